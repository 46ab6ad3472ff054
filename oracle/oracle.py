"""TEST INFRASTRUCTURE ONLY: numpy front end of the CPU oracle (hp_oracle.cpp).

Used by tests/, the smoke check and bench.py's CPU-baseline leg as the checker
of the CUDA path; nothing in the product imports it.  `build()` compiles the
C++ restatement with the Makefile next to this file.
"""
import ctypes
import fcntl
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhp_oracle.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32


class OraCamera(ctypes.Structure):
    _fields_ = [("c2w", ctypes.c_float * 12), ("w2c", ctypes.c_float * 12), ("K", ctypes.c_float * 9),
                ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("width", _i32), ("height", _i32)]


class OraOptions(ctypes.Structure):
    _fields_ = [("kernel_size", _i32), ("t_intvl", ctypes.c_float), ("radius_threshold", ctypes.c_float),
                ("num_sample_points_per_ray", _i32), ("num_point_cloud_per_sp", _i32),
                ("num_point_per_ray", _i32), ("sdf2weight_gaussian_alpha", ctypes.c_float),
                ("sdf2weight_gaussian_gamma", ctypes.c_float)]


def build(force=False):
    """make the oracle library; processes that build at once take turns on a lock file."""
    srcs = [os.path.join(HERE, f) for f in ("hp_oracle.cpp", "hp_oracle.h")]

    def stale():
        return force or not os.path.exists(LIB_PATH) or any(os.path.getmtime(LIB_PATH) < os.path.getmtime(f)
                                                              for f in srcs)

    if stale():
        os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
        with open(os.path.join(os.path.dirname(LIB_PATH), ".build.lock"), "w") as lock:
            try:
                fcntl.flock(lock, fcntl.LOCK_EX)
                locked = True
            except OSError:  # a filesystem without locks: build unserialised
                locked = False
            try:
                if stale():
                    subprocess.run(["make", "-C", HERE, "-B" if force else "all"], check=True,
                                   stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
            finally:
                if locked:
                    fcntl.flock(lock, fcntl.LOCK_UN)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        cp = ctypes.POINTER(OraCamera)
        op = ctypes.POINTER(OraOptions)
        L.ora_project_mode.argtypes = [_f32p, _i64, cp, _i32, _i32, _i32p, _f32p]
        L.ora_project.argtypes = [_f32p, _i64, cp, _i32p, _f32p]
        L.ora_project_f64.argtypes = [_f32p, _i64, cp, _f64p]
        L.ora_projection_rounding.argtypes = [_i64, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]
        L.ora_sort_by_pixel.argtypes = [_i32p, _f32p, _i64, _i32, _i32p, _f32p, _i32p]
        L.ora_scatter_hashtable.argtypes = [_i32p, _i32p, _f32p, _i64, _i32, _i32, _i32, _i32p, _f32p, _i32p]
        L.ora_pts2plane.argtypes = [_f32p, _i64, cp, _i32, _i32p, _f32p, _i32p]
        L.ora_quick_sampling_dirs.argtypes = [_f32p, _i64, cp, op, _i32p, _i32p, _vp, _f32p, _i32p, _f32p, _u8p,
                                              _f32p, _vp, _i64, _i32]
        L.ora_quick_sampling_dirs.restype = ctypes.c_int
        L.ora_quick_sampling_f64.argtypes = [_f32p, _i64, cp, op, _i32p, _i32p, _f64p, _f64p, _u8p, _i32]
        L.ora_quick_sampling_f64.restype = ctypes.c_int
        L.ora_ray_dirs.argtypes = [cp, _f32p]
        L.ora_quick_query_dirs.argtypes = [_f32p, _i64, cp, op, _i32p, _i32p, _i32p, _i64, _vp, _i32p, _i32p, _f32p]
        L.ora_quick_query_dirs.restype = ctypes.c_int
        L.ora_scatter_multibin.argtypes = [_i32p, _i32p, _f32p, _i64, _i32, _i32, _i32, _f32p, _i32p]
        _lib = L
    return _lib


def camera(c2w, w2c, K, width, height, fx=None, fy=None, cx=None, cy=None):
    c2w = np.asarray(c2w, np.float32)
    w2c = np.asarray(w2c, np.float32)
    K = np.asarray(K, np.float32)
    c = OraCamera()
    c.c2w[:] = c2w[:3, :4].reshape(-1).tolist()
    c.w2c[:] = w2c[:3, :4].reshape(-1).tolist()
    c.K[:] = K.reshape(-1).tolist()
    c.fx = float(K[0, 0]) if fx is None else float(fx)
    c.fy = float(K[1, 1]) if fy is None else float(fy)
    c.cx = float(K[0, 2]) if cx is None else float(cx)
    c.cy = float(K[1, 2]) if cy is None else float(cy)
    c.width, c.height = int(width), int(height)
    return c


def camera_from(cam):
    """From an object with c2w, w2c, K, width, height (e.g. hashpoint.synth.PinholeCamera)."""
    return camera(cam.c2w, cam.w2c, cam.K, cam.width, cam.height)


def options(opt):
    o = OraOptions()
    for name, _ in OraOptions._fields_:
        setattr(o, name, getattr(opt, name))
    return o


def _c32(a):
    return np.ascontiguousarray(a, np.float32)


def _ci32(a):
    return np.ascontiguousarray(a, np.int32)


def projection_rounding(n):
    a, b = _i32(), _i32()
    lib().ora_projection_rounding(int(n), ctypes.byref(a), ctypes.byref(b))
    return int(a.value), int(b.value)


def project(xyz, cam, mode=None):
    xyz = _c32(xyz)
    n = len(xyz)
    pid = np.empty(n, np.int32)
    dep = np.empty(n, np.float32)
    if mode is None:
        lib().ora_project(xyz, n, ctypes.byref(cam), pid, dep)
    else:
        lib().ora_project_mode(xyz, n, ctypes.byref(cam), int(mode[0]), int(mode[1]), pid, dep)
    return pid, dep


def project_f64(xyz, cam):
    xyz = _c32(xyz)
    out = np.empty(len(xyz), np.float64)
    lib().ora_project_f64(xyz, len(xyz), ctypes.byref(cam), out)
    return out


def sort_by_pixel(pid, depth, hw):
    n = len(pid)
    ps = np.empty(n, np.int32)
    ds = np.empty(n, np.float32)
    ix = np.empty(n, np.int32)
    lib().ora_sort_by_pixel(_ci32(pid), _c32(depth), n, int(hw), ps, ds, ix)
    return ps, ds, ix


def scatter_hashtable(point_idx, point2img, depth, height, width, sort):
    n = len(point_idx)
    oi = np.empty(n, np.int32)
    od = np.empty(n, np.float32)
    hs = np.empty((height * width, 2), np.int32)
    lib().ora_scatter_hashtable(_ci32(point_idx), _ci32(point2img), _c32(depth), n, int(height), int(width),
                                int(bool(sort)), oi, od, hs)
    return oi, od, hs


def pts2plane(xyz, cam, sort=False):
    xyz = _c32(xyz)
    n = len(xyz)
    oi = np.empty(n, np.int32)
    od = np.empty(n, np.float32)
    hs = np.empty((cam.height * cam.width, 2), np.int32)
    lib().ora_pts2plane(xyz, n, ctypes.byref(cam), int(bool(sort)), oi, od, hs)
    return oi, od, hs


def ray_dirs(cam):
    out = np.empty((cam.height * cam.width, 3), np.float32)
    lib().ora_ray_dirs(ctypes.byref(cam), out)
    return out


def quick_sampling(xyz, cam, opt, sorted_idx, hash_table, dirs=None, rays=None, nthreads=1):
    """Returns sp_xyz [H,W,S,3], pc_idx [H,W,S,P], sp_t [H,W,S], mask [H,W,S] (bool), margin [H*W].

    With `rays` (linear pixel ids) the outputs are compact: [R,S,3], [R,S,P], [R,S], [R,S], [R].
    `dirs` [H*W,3] overrides the ray directions (e.g. the CUDA library's own)."""
    H, W = cam.height, cam.width
    o = options(opt)
    S, P = o.num_sample_points_per_ray, o.num_point_cloud_per_sp
    xyz = _c32(xyz)
    lead = (H, W) if rays is None else (len(rays),)
    sp_xyz = np.zeros(lead + (S, 3), np.float32)
    pc_idx = np.full(lead + (S, P), -1, np.int32)
    sp_t = np.zeros(lead + (S,), np.float32)
    mask = np.zeros(lead + (S,), np.uint8)
    margin = np.full(int(np.prod(lead)), np.inf, np.float32)
    dirs_c = None if dirs is None else _c32(dirs).reshape(-1, 3)
    rays_c = None if rays is None else _ci32(rays)
    rc = lib().ora_quick_sampling_dirs(
        xyz, len(xyz), ctypes.byref(cam), ctypes.byref(o), _ci32(sorted_idx), _ci32(hash_table).reshape(-1),
        None if dirs_c is None else dirs_c.ctypes.data, sp_xyz, pc_idx, sp_t, mask, margin,
        None if rays_c is None else rays_c.ctypes.data, 0 if rays_c is None else len(rays_c), int(nthreads))
    if rc != 0:
        raise ValueError("oracle quick_sampling rejected the options (code %d)" % rc)
    return sp_xyz, pc_idx, sp_t, mask.astype(bool), margin


def quick_sampling_f64(xyz, cam, opt, sorted_idx, hash_table, nthreads=1):
    H, W = cam.height, cam.width
    o = options(opt)
    S = o.num_sample_points_per_ray
    sp_xyz = np.zeros((H, W, S, 3), np.float64)
    sp_t = np.zeros((H, W, S), np.float64)
    mask = np.zeros((H, W, S), np.uint8)
    rc = lib().ora_quick_sampling_f64(_c32(xyz), len(xyz), ctypes.byref(cam), ctypes.byref(o), _ci32(sorted_idx),
                                      _ci32(hash_table).reshape(-1), sp_xyz, sp_t, mask, int(nthreads))
    if rc != 0:
        raise ValueError("oracle quick_sampling_f64 rejected the options (code %d)" % rc)
    return sp_xyz, sp_t, mask.astype(bool)


def quick_query(xyz, cam, opt, sorted_idx, hash_table, ray_ids, dirs=None):
    o = options(opt)
    ray_ids = _ci32(ray_ids)
    n = len(ray_ids)
    cap = o.num_point_per_ray
    out = np.empty((n, cap), np.int32)
    cnt = np.empty(n, np.int32)
    mg = np.empty(n, np.float32)
    dirs_c = None if dirs is None else _c32(dirs).reshape(-1, 3)
    rc = lib().ora_quick_query_dirs(_c32(xyz), len(xyz), ctypes.byref(cam), ctypes.byref(o), _ci32(sorted_idx),
                                    _ci32(hash_table).reshape(-1), ray_ids, n,
                                    None if dirs_c is None else dirs_c.ctypes.data, out, cnt, mg)
    if rc != 0:
        raise ValueError("oracle quick_query rejected the options (code %d)" % rc)
    return out, cnt, mg


def scatter_multibin(point_idx, point2img, depth, height, width, bins):
    hw = height * width
    od = np.empty((hw, bins), np.float32)
    oi = np.empty((hw, bins), np.int32)
    lib().ora_scatter_multibin(_ci32(point_idx), _ci32(point2img), _c32(depth), len(point_idx), int(height),
                               int(width), int(bins), od, oi)
    return od, oi
