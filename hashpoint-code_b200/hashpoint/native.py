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
import shutil
import subprocess
import tempfile
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
SOURCES = ["hp_api.cu", "hp_build.cu", "hp_sample.cu", "hp_query.cu", "hp_feature.cu", "hp_aggregator.cu"]
# The test-only library (include/hashpoint_b200_testing.h): the tensor-core operand-form self-check and a
# wait-expiry test of the Aggregator, compiled with the sources they exercise; never loaded by the product.
TESTING_LIB_NAME = "libhashpoint_b200_testing.so"
TESTING_LIB_PATH = os.path.join(LIB_DIR, TESTING_LIB_NAME)
TESTING_SOURCES = ["hp_api.cu", "hp_build.cu", "hp_aggregator.cu", "hp_tc_check.cu"]
TESTING_FLAGS = ["-DHP_TESTING"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]

# C-ABI symbols declared in include/hashpoint_b200.h
EXPORTS = ["hp_version", "hp_last_error", "hp_projection_rounding", "hp_pts2plane_workspace_size", "hp_pts2plane",
           "hp_pts2plane_noalloc", "hp_pts2plane_status", "hp_pts2plane_noalloc_status", "hp_scatter_hashtable", "hp_quick_sampling_workspace_size", "hp_quick_sampling",
           "hp_quick_sampling_tuned", "hp_stage_config_info",
           "hp_quick_sampling_batch_workspace_size", "hp_quick_sampling_batch", "hp_quick_query_for_nearby_point",
           "hp_scatter", "hp_ray_directions", "hp_mask_scan", "hp_mask_scan_workspace_size", "hp_feature_query",
           "hp_clamp_t", "hp_render", "hp_aggregator_packed_size", "hp_aggregator_pack",
           "hp_aggregator_workspace_size", "hp_aggregator_forward", "hp_aggregator_status"]
# declared in include/hashpoint_b200_testing.h, exported by the test-only library
TESTING_EXPORTS = ["hp_tc_check_image_bytes", "hp_tc_check_mma", "hp_aggregator_forward_withheld",
                   "hp_pts2plane_withheld"]

HP_OK = 0


class HashPointError(RuntimeError):
    pass


def _sources(names=None):
    return [os.path.join(CSRC, s) for s in (names or SOURCES)]


def _deps(names=None):
    deps = _sources(names) + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return deps


def needs_build(path=None, names=None):
    path = path or LIB_PATH
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    return any(os.path.getmtime(d) > t for d in _deps(names))


def build(force=False, verbose=False, extra_flags=()):
    """Compile the CUDA sources for sm_100a into the in-tree shared library.

    Every build compiles into a directory of its own and links to a file name
    of its own, then renames the result over the library (atomic), so builders
    that run at once -- the ranks of a torchrun job, test workers -- never
    read or delete each other's files.  A lock file next to the library only
    saves duplicate work: each builder re-checks after taking it, so the first
    one builds and the others find the library current.  On a filesystem
    without locks they simply all build."""
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    with open(os.path.join(LIB_DIR, ".build.lock"), "w") as lock:
        try:
            fcntl.flock(lock, fcntl.LOCK_EX)
        except OSError:  # a filesystem without locks: private build directories keep builders apart
            return _build_private(verbose, extra_flags)
        try:
            if not force and not needs_build():
                return LIB_PATH
            return _build_private(verbose, extra_flags)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)


def build_testing(force=False, verbose=False):
    """Compile the test-only library (TESTING_SOURCES with -DHP_TESTING) beside the product library,
    under the same lock and private-directory protocol as build()."""
    if not force and not needs_build(TESTING_LIB_PATH, TESTING_SOURCES):
        return TESTING_LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    with open(os.path.join(LIB_DIR, ".build.lock"), "w") as lock:
        try:
            fcntl.flock(lock, fcntl.LOCK_EX)
        except OSError:
            return _build_private(verbose, TESTING_FLAGS, TESTING_SOURCES, TESTING_LIB_PATH)
        try:
            if not force and not needs_build(TESTING_LIB_PATH, TESTING_SOURCES):
                return TESTING_LIB_PATH
            return _build_private(verbose, TESTING_FLAGS, TESTING_SOURCES, TESTING_LIB_PATH)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)


def _build_private(verbose, extra_flags, names=None, path=None):
    work = tempfile.mkdtemp(prefix=".build-", dir=LIB_DIR)
    try:
        return _compile_and_link(work, verbose, extra_flags, names, path or LIB_PATH)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _compile_and_link(work, verbose, extra_flags, names=None, path=None):
    path = path or LIB_PATH
    srcs = _sources(names)
    objs = [os.path.join(work, os.path.basename(s) + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        cmd = [NVCC, "-c", src, "-o", obj, "-I" + INCLUDE] + NVCC_FLAGS + list(extra_flags)
        p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if p.returncode != 0:
            raise HashPointError("nvcc failed for %s:\n%s" % (src, p.stdout))
        return p.stdout

    with ThreadPoolExecutor(max_workers=len(objs)) as ex:
        outs = list(ex.map(compile_one, zip(srcs, objs)))
    tmp = os.path.join(work, os.path.basename(path))
    p = subprocess.run([NVCC, "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a"],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        raise HashPointError("link failed:\n%s" % p.stdout)
    os.replace(tmp, path)
    if verbose:
        print("".join(outs))
    return path


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
    """Launch tuning of hp_quick_sampling_tuned / _batch (0 = default; see include/hashpoint_b200.h)."""
    _fields_ = [("heavy_window", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("stage_config", ctypes.c_int32)]


STAGE_CONFIGS = (1, 2, 3, 4, 5)  # hp_tuning.stage_config values (see include/hashpoint_b200.h)


def stage_config_info(config):
    """{tile_h, tile_w, stage_points, blocks_per_sm} of a stage configuration (hp_stage_config_info)."""
    L = lib()
    v = [ctypes.c_int32() for _ in range(4)]
    check(L.hp_stage_config_info(int(config), *[ctypes.byref(x) for x in v]), "hp_stage_config_info", L)
    return dict(zip(("tile_h", "tile_w", "stage_points", "blocks_per_sm"), (x.value for x in v)))


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
        L.hp_pts2plane_status.argtypes = [vp, i64, i32, i32, vp]
        L.hp_pts2plane_status.restype = i32
        L.hp_pts2plane_noalloc_status.argtypes = [i64, i32, i32, vp]
        L.hp_pts2plane_noalloc_status.restype = i32
        L.hp_scatter_hashtable.argtypes = [vp, vp, vp, i64, i32, i32, i32, vp, vp, vp, vp]
        L.hp_scatter_hashtable.restype = i32
        L.hp_quick_sampling_workspace_size.argtypes = [i64, i32, i32]
        L.hp_quick_sampling_workspace_size.restype = sz
        L.hp_quick_sampling.argtypes = [vp, i64, cam_p, opt_p, vp, i64, vp, vp, vp, vp, vp, vp, sz, vp]
        L.hp_quick_sampling.restype = i32
        L.hp_quick_sampling_tuned.argtypes = [vp, i64, cam_p, opt_p, vp, i64, vp, vp, vp, vp, vp,
                                              ctypes.POINTER(HpTuning), vp, sz, vp]
        L.hp_quick_sampling_tuned.restype = i32
        ip = ctypes.POINTER(ctypes.c_int32)
        L.hp_stage_config_info.argtypes = [i32, ip, ip, ip, ip]
        L.hp_stage_config_info.restype = i32
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
        L.hp_quick_query_for_nearby_point.argtypes = [vp, i64, cam_p, opt_p, vp, i64, vp, vp, i64, vp, vp]
        L.hp_quick_query_for_nearby_point.restype = i32
        L.hp_scatter.argtypes = [vp, vp, vp, i64, i32, i32, i32, vp, vp, vp]
        L.hp_scatter.restype = i32
        L.hp_ray_directions.argtypes = [cam_p, vp, vp]
        L.hp_ray_directions.restype = i32
        _lib = L
        return _lib


_testing = None


def testing_lib():
    """Load the test-only library (raises HashPointError if it is missing)."""
    global _testing
    with _lock:
        if _testing is not None:
            return _testing
        if not os.path.exists(TESTING_LIB_PATH):
            raise HashPointError("test library %s is missing: build it with hashpoint.native.build_testing()"
                                 % TESTING_LIB_PATH)
        T = ctypes.CDLL(TESTING_LIB_PATH)
        vp, i32, i64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
        T.hp_last_error.restype = ctypes.c_char_p
        T.hp_tc_check_image_bytes.argtypes = [i32]
        T.hp_tc_check_image_bytes.restype = sz
        T.hp_tc_check_mma.argtypes = [vp, vp, i32, ctypes.c_uint32, i32, ctypes.c_uint32, vp, vp]
        T.hp_tc_check_mma.restype = i32
        T.hp_aggregator_workspace_size.argtypes = [i64]
        T.hp_aggregator_workspace_size.restype = sz
        T.hp_aggregator_status.argtypes = [vp, i64, vp]
        T.hp_aggregator_status.restype = i32
        T.hp_aggregator_forward_withheld.argtypes = [vp, vp, vp, vp, vp, i32, vp, vp, vp, i64, i32, vp, vp, i64, vp,
                                                     vp, vp, sz, i32, vp]
        T.hp_aggregator_forward_withheld.restype = i32
        cam_p = ctypes.POINTER(HpCamera)
        T.hp_pts2plane_workspace_size.argtypes = [i64, i32, i32]
        T.hp_pts2plane_workspace_size.restype = sz
        T.hp_pts2plane_withheld.argtypes = [vp, i64, cam_p, i32, vp, vp, vp, vp, sz, i32, vp]
        T.hp_pts2plane_withheld.restype = i32
        T.hp_pts2plane_status.argtypes = [vp, i64, i32, i32, vp]
        T.hp_pts2plane_status.restype = i32
        _testing = T
        return _testing


def check(rc, what, L=None):
    """Raise HashPointError with the library's message when rc is not HP_OK (L: the library that
    made the call, default the product library)."""
    if rc != HP_OK:
        msg = (L or lib()).hp_last_error().decode(errors="replace")
        raise HashPointError("%s failed (%d): %s" % (what, rc, msg))


def projection_rounding(n_points):
    a, b = ctypes.c_int32(), ctypes.c_int32()
    lib().hp_projection_rounding(int(n_points), ctypes.byref(a), ctypes.byref(b))
    return int(a.value), int(b.value)
