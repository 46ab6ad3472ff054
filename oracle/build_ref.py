"""Build recipe for the reference's own CUDA extension, used only as a test checker.

This script compiles the reference's `epcq/csrc` sources *where they lie* under
the read-only reference checkout (the HP_REFERENCE_ROOT environment variable,
else `/root/reference`) with plain
`nvcc`/`g++` invocations (it does not run the reference's setup.py), for
sm_100a, and links them into `oracle/_ref/epcq_ref_csrc.so`, a CPython
extension module named `epcq_ref_csrc` that exposes the same pybind surface as
the reference's `epcq.csrc` (`scatter`, `scatter_hashtable`, `quick_sampling`,
`quick_query_for_nearby_point` and the four spec classes, registered at
epcq/csrc/epcq.cpp:10-56).

Only the three translation units that carry code are compiled: epcq.cpp,
rasterization.cu and epcq_render_topk.cu.  optimize.cu and
epcq_render_topk_bk.cu are entirely commented out in the reference.

Compiler flags mirror what torch's CUDAExtension passes for the reference's
setup.py (setup.py:38-49 adds only the include dir), plus the sm_100a gencode.
The output directory is git-ignored; the built .so travels with the repository
snapshot to GPU machines, where the reference checkout itself is absent.

Usage:  python oracle/build_ref.py [--ref REFERENCE_ROOT] [--force]
"""
import argparse
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
MODULE = "epcq_ref_csrc"
SO_PATH = os.path.join(OUT_DIR, MODULE + ".so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")


def default_root():
    """Location of the reference checkout: $HP_REFERENCE_ROOT, else where this build reads it."""
    return os.environ.get("HP_REFERENCE_ROOT", "/root/reference")


def _torch_paths():
    import torch
    tdir = os.path.dirname(torch.__file__)
    inc = [os.path.join(tdir, "include"),
           os.path.join(tdir, "include", "torch", "csrc", "api", "include")]
    lib = os.path.join(tdir, "lib")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return inc, lib, abi


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed (%d): %s\n%s" % (proc.returncode, " ".join(cmd), proc.stdout))
    return proc.stdout


def build(ref_root=None, force=False, verbose=True):
    """Compile the reference extension into oracle/_ref; return the .so path.

    Skips the build when the .so is newer than every source (unless force).
    Raises FileNotFoundError when the reference checkout is absent.
    """
    ref_root = ref_root or default_root()
    csrc = os.path.join(ref_root, "epcq", "csrc")
    if not os.path.isdir(csrc):
        raise FileNotFoundError("reference sources not found at %s" % csrc)
    sources = [os.path.join(csrc, f) for f in ("epcq.cpp", "rasterization.cu", "epcq_render_topk.cu")]
    if (not force and os.path.exists(SO_PATH)
            and all(os.path.getmtime(SO_PATH) > os.path.getmtime(s) for s in sources)):
        return SO_PATH
    os.makedirs(OUT_DIR, exist_ok=True)
    tinc, tlib, abi = _torch_paths()
    pyinc = sysconfig.get_paths()["include"]
    incs = ["-I" + os.path.join(csrc, "include")] + ["-I" + p for p in tinc] + \
           ["-I" + pyinc, "-I" + os.path.join(CUDA_HOME, "include")]
    defs = ["-DTORCH_API_INCLUDE_EXTENSION_H", "-DTORCH_EXTENSION_NAME=" + MODULE,
            "-D_GLIBCXX_USE_CXX11_ABI=%d" % abi]
    nvcc_flags = ["-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
                  "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
                  "--expt-relaxed-constexpr", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-gencode", "arch=compute_100a,code=sm_100a"]
    jobs = []
    objs = []
    for s in sources:
        obj = os.path.join(OUT_DIR, os.path.basename(s) + ".o")
        objs.append(obj)
        if s.endswith(".cu"):
            jobs.append([NVCC, "-c", s, "-o", obj] + nvcc_flags + defs + incs)
        else:
            jobs.append(["g++", "-c", s, "-o", obj, "-O2", "-fPIC", "-std=c++17"] + defs + incs)
    if verbose:
        print("[build_ref] compiling %d reference sources -> %s" % (len(jobs), OUT_DIR), flush=True)
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        list(ex.map(_run, jobs))
    link = ["g++", "-shared", "-o", SO_PATH] + objs + [
        "-L" + tlib, "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python", "-lc10_cuda", "-ltorch_cuda",
        "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-Wl,-rpath," + tlib]
    _run(link)
    for o in objs:
        os.remove(o)
    if verbose:
        print("[build_ref] built", SO_PATH, flush=True)
    return SO_PATH


def load():
    """Import the built reference extension module (requires torch imported)."""
    import importlib.util
    import torch  # noqa: F401  (the module links against libtorch)
    if not os.path.exists(SO_PATH):
        raise FileNotFoundError(SO_PATH)
    spec = importlib.util.spec_from_file_location(MODULE, SO_PATH)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: $HP_REFERENCE_ROOT or the build's)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(a.ref, a.force)
    except FileNotFoundError as e:
        print("[build_ref] skipped:", e)
        sys.exit(0)
