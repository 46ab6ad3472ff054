"""ctypes binding of the hashpoint_b200 C ABI (include/hashpoint_b200.h).

`build()` compiles csrc/*.cu for sm_100a into hashpoint/lib/libhashpoint_b200.so
(in-tree).  `lib()` loads it; there is no fallback: if the shared library is
missing or a call fails, an exception is raised.

The tensor-level helpers here are the plumbing between torch (device memory,
the current stream) and the C ABI: they validate dtypes/devices/contiguity,
allocate outputs and workspaces with torch's caching allocator on the current
device, and pass raw pointers plus torch's current CUDA stream.
"""
import ctypes
import fcntl
import os
import subprocess
import threading
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                       # hashpoint-code_b200/
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_NAME = "libhashpoint_b200.so"
LIB_PATH = os.path.join(LIB_DIR, LIB_NAME)
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
SOURCES = ["hp_api.cu", "hp_build.cu", "hp_sample.cu", "hp_query.cu", "hp_feature.cu", "hp_aggregator.cu",
           "hp_tc_check.cu"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]

# C-ABI symbols declared in include/hashpoint_b200.h
EXPORTS = ["hp_version", "hp_last_error", "hp_projection_rounding", "hp_pts2plane_workspace_size", "hp_pts2plane",
           "hp_pts2plane_noalloc", "hp_scatter_hashtable", "hp_quick_sampling_workspace_size", "hp_quick_sampling",
           "hp_quick_sampling_batch_workspace_size", "hp_quick_sampling_batch", "hp_quick_query_for_nearby_point",
           "hp_scatter", "hp_ray_directions", "hp_mask_scan", "hp_mask_scan_workspace_size", "hp_feature_query",
           "hp_clamp_t", "hp_render", "hp_aggregator_packed_size", "hp_aggregator_pack",
           "hp_aggregator_workspace_size", "hp_aggregator_forward", "hp_aggregator_status",
           "hp_tc_check_image_bytes", "hp_tc_check_mma"]

HP_OK = 0


class HashPointError(RuntimeError):
    pass


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _deps():
    deps = _sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(INCLUDE, "hashpoint_b200.h"))
    return deps


def needs_build():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force=False, verbose=False, extra_flags=()):
    """Compile the CUDA sources for sm_100a into the in-tree shared library.

    Processes that build at once (the ranks of a torchrun job, test workers)
    take turns on a lock file next to the library; each re-checks after taking
    it, so the first one builds and the others find the library current."""
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    with open(os.path.join(LIB_DIR, ".build.lock"), "w") as lock:
        try:
            fcntl.flock(lock, fcntl.LOCK_EX)
        except OSError:  # a filesystem without locks: build unserialised, as before
            return _build_locked(verbose, extra_flags)
        try:
            if not force and not needs_build():
                return LIB_PATH
            return _build_locked(verbose, extra_flags)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)


def _build_locked(verbose, extra_flags):
    objs = [os.path.join(LIB_DIR, os.path.basename(s) + ".o") for s in _sources()]

    def compile_one(pair):
        src, obj = pair
        cmd = [NVCC, "-c", src, "-o", obj, "-I" + INCLUDE] + NVCC_FLAGS + list(extra_flags)
        p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if p.returncode != 0:
            raise HashPointError("nvcc failed for %s:\n%s" % (src, p.stdout))
        return p.stdout

    with ThreadPoolExecutor(max_workers=len(objs)) as ex:
        outs = list(ex.map(compile_one, zip(_sources(), objs)))
    tmp = LIB_PATH + ".tmp"
    p = subprocess.run([NVCC, "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a"],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise HashPointError("link failed:\n%s" % p.stdout)
    os.replace(tmp, LIB_PATH)
    for o in objs:
        os.remove(o)
    if verbose:
        print("".join(outs))
    return LIB_PATH


# ----------------------------------------------------------------------------
# C structs
# ----------------------------------------------------------------------------
class HpCamera(ctypes.Structure):
    _fields_ = [("c2w", ctypes.c_void_p), ("w2c", ctypes.c_void_p), ("K", ctypes.c_void_p),
                ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32)]


class HpOptions(ctypes.Structure):
    _fields_ = [("kernel_size", ctypes.c_int32), ("t_intvl", ctypes.c_float),
                ("radius_threshold", ctypes.c_float), ("num_sample_points_per_ray", ctypes.c_int32),
                ("num_point_cloud_per_sp", ctypes.c_int32), ("num_point_per_ray", ctypes.c_int32),
                ("sdf2weight_gaussian_alpha", ctypes.c_float), ("sdf2weight_gaussian_gamma", ctypes.c_float)]


class HpPointAttrs(ctypes.Structure):
    _fields_ = [("xyz", ctypes.c_void_p), ("rgb", ctypes.c_void_p), ("dir", ctypes.c_void_p), ("feat", ctypes.c_void_p),
                ("feat_dim", ctypes.c_int32), ("feat_half", ctypes.c_int32), ("n_points", ctypes.c_int64)]


class HpAggregatorWeights(ctypes.Structure):
    """The Aggregator's nine nn.Linear layers (weight [out, in], bias), module order."""
    _fields_ = [("weight", ctypes.c_void_p * 9), ("bias", ctypes.c_void_p * 9)]


class HpTuning(ctypes.Structure):
    """Launch tuning of hp_quick_sampling_batch (0 = default)."""
    _fields_ = [("heavy_window", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32)]


class HpView(ctypes.Structure):
    """One view of hp_quick_sampling_batch (include/hashpoint_b200.h)."""
    _fields_ = [("xyz", ctypes.c_void_p), ("n_points", ctypes.c_int64), ("sorted_point_idx", ctypes.c_void_p),
                ("n_sorted", ctypes.c_int64), ("hash_table", ctypes.c_void_p), ("sp_xyz", ctypes.c_void_p),
                ("pc_idx", ctypes.c_void_p), ("sp_t", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("cam", HpCamera), ("opt", HpOptions)]


_lib = None
_lock = threading.Lock()


def lib():
    """Load the shared library (raises HashPointError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise HashPointError("CUDA library %s is missing: build it with hashpoint.native.build() "
                                 "(there is no CPU fallback)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
        cam_p, opt_p = ctypes.POINTER(HpCamera), ctypes.POINTER(HpOptions)
        L.hp_version.restype = i32
        L.hp_last_error.restype = ctypes.c_char_p
        L.hp_projection_rounding.argtypes = [i64, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        L.hp_projection_rounding.restype = None
        L.hp_pts2plane_workspace_size.argtypes = [i64, i32, i32]
        L.hp_pts2plane_workspace_size.restype = sz
        L.hp_pts2plane.argtypes = [vp, i64, cam_p, i32, vp, vp, vp, vp, sz, vp]
        L.hp_pts2plane.restype = i32
        L.hp_pts2plane_noalloc.argtypes = [vp, i64, cam_p, i32, vp, vp, vp, vp]
        L.hp_pts2plane_noalloc.restype = i32
        L.hp_scatter_hashtable.argtypes = [vp, vp, vp, i64, i32, i32, i32, vp, vp, vp, vp]
        L.hp_scatter_hashtable.restype = i32
        L.hp_quick_sampling_workspace_size.argtypes = [i64, i32, i32]
        L.hp_quick_sampling_workspace_size.restype = sz
        L.hp_quick_sampling.argtypes = [vp, i64, cam_p, opt_p, vp, i64, vp, vp, vp, vp, vp, vp, sz, vp]
        L.hp_quick_sampling.restype = i32
        view_p = ctypes.POINTER(HpView)
        L.hp_quick_sampling_batch_workspace_size.argtypes = [view_p, i32]
        L.hp_quick_sampling_batch_workspace_size.restype = sz
        L.hp_quick_sampling_batch.argtypes = [view_p, vp, i32, ctypes.POINTER(HpTuning), vp, sz, vp]
        L.hp_quick_sampling_batch.restype = i32
        L.hp_mask_scan.argtypes = [vp, i64, vp, vp, vp, sz, vp]
        L.hp_mask_scan.restype = i32
        L.hp_mask_scan_workspace_size.argtypes = [i64]
        L.hp_mask_scan_workspace_size.restype = sz
        L.hp_feature_query.argtypes = [ctypes.POINTER(HpPointAttrs), vp, vp, vp, i64, i32, i32, vp, cam_p, vp,
                                       vp, vp, vp, vp, vp, vp, vp, vp]
        L.hp_feature_query.restype = i32
        L.hp_clamp_t.argtypes = [vp, i64, i32, ctypes.c_float, vp, vp]
        L.hp_clamp_t.restype = i32
        L.hp_render.argtypes = [vp, vp, ctypes.c_float, vp, vp, i64, i32, i32, vp, vp]
        L.hp_render.restype = i32
        L.hp_aggregator_packed_size.argtypes = []
        L.hp_aggregator_packed_size.restype = sz
        L.hp_aggregator_pack.argtypes = [ctypes.POINTER(HpAggregatorWeights), vp, sz, vp]
        L.hp_aggregator_pack.restype = i32
        L.hp_aggregator_workspace_size.argtypes = [i64]
        L.hp_aggregator_workspace_size.restype = sz
        L.hp_aggregator_forward.argtypes = [vp, vp, vp, vp, vp, i32, vp, vp, vp, i64, i32, vp, vp, i64, vp, vp, vp,
                                            sz, vp]
        L.hp_aggregator_forward.restype = i32
        L.hp_aggregator_status.argtypes = [vp, i64, vp]
        L.hp_aggregator_status.restype = i32
        L.hp_tc_check_image_bytes.argtypes = [i32]
        L.hp_tc_check_image_bytes.restype = sz
        L.hp_tc_check_mma.argtypes = [vp, vp, i32, ctypes.c_uint32, i32, ctypes.c_uint32, vp, vp]
        L.hp_tc_check_mma.restype = i32
        L.hp_quick_query_for_nearby_point.argtypes = [vp, i64, cam_p, opt_p, vp, i64, vp, vp, i64, vp, vp]
        L.hp_quick_query_for_nearby_point.restype = i32
        L.hp_scatter.argtypes = [vp, vp, vp, i64, i32, i32, i32, vp, vp, vp]
        L.hp_scatter.restype = i32
        L.hp_ray_directions.argtypes = [cam_p, vp, vp]
        L.hp_ray_directions.restype = i32
        _lib = L
        return _lib


def check(rc, what):
    if rc != HP_OK:
        msg = lib().hp_last_error().decode(errors="replace")
        raise HashPointError("%s failed (%d): %s" % (what, rc, msg))


def projection_rounding(n_points):
    a, b = ctypes.c_int32(), ctypes.c_int32()
    lib().hp_projection_rounding(int(n_points), ctypes.byref(a), ctypes.byref(b))
    return int(a.value), int(b.value)
