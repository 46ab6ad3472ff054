"""The reference's own CPU point-ray searchers, timed on this machine's host cores.

The reference benchmarks its GPU path against pure-Python CPU searchers in
point_ray_search_benchmark/: KDTreeRaySearch (kdtree.py:128-184) and
UniformGrid (uniform_grid.py:9-97), driven by benchmark.py:77,111 with
voxel_size 0.2 and max_points_per_node 100.  This module is baseline
infrastructure, not product: bench.py's CPU-baseline leg runs it.

  stage(ref_root)  copies those three source files (tools.py, kdtree.py,
                   uniform_grid.py), unmodified, from the reference checkout
                   into baseline/_ref/point_ray_search_benchmark/ (git-ignored;
                   it travels with the working tree to GPU machines, where the
                   checkout is absent)
  run(...)         in a child process (the stubs below must not reach the
                   caller's modules): imports them with empty stand-ins for the
                   modules they import but never use on this path (open3d,
                   matplotlib, graphviz, the reference's dataset, epcq and
                   utils.config), builds both structures once on the 100k-point
                   sphere workload, then forks one worker per host core, each
                   searching a slice of 4096 seed-0 pixel-centre rays
                   (o = c2w[:3, 3], d = R ((u + .5 - cx) / fx, (v + .5 - cy) / fy, 1),
                   the GPU path's rays), radius 0.01.

Reported per searcher: rays/s (rays / wall time of the parallel search),
build seconds, and whether its result sets equal a brute-force search
(distance <= radius, the reference's tools.correct_answer) on 32 of the rays.
The reference's UniformGrid initialises its DDA t_max wrongly
(uniform_grid.py:46) and misses points; the flag records that.

Usage:  python oracle/ref_cpu.py --stage <reference checkout>
        python oracle/ref_cpu.py --json
"""
import argparse
import json
import os
import platform
import shutil
import subprocess
import sys
import time
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
STAGE_DIR = os.path.join(ROOT, "baseline", "_ref", "point_ray_search_benchmark")
FILES = ("tools.py", "kdtree.py", "uniform_grid.py")


def staged():
    return all(os.path.exists(os.path.join(STAGE_DIR, f)) for f in FILES)


def stage(ref_root):
    """Copy the searchers' sources from the reference checkout (no-op when already current)."""
    src = os.path.join(ref_root, "point_ray_search_benchmark")
    if not all(os.path.exists(os.path.join(src, f)) for f in FILES):
        raise FileNotFoundError("point_ray_search_benchmark not found under %s" % ref_root)
    os.makedirs(STAGE_DIR, exist_ok=True)
    for f in FILES:
        a, b = os.path.join(src, f), os.path.join(STAGE_DIR, f)
        if not os.path.exists(b) or os.path.getmtime(b) < os.path.getmtime(a):
            shutil.copy2(a, b)
    return STAGE_DIR


def _install_stubs():
    """Empty stand-ins for modules the searchers import but never use on the ray-search path."""
    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    class _Unused:
        def __init__(self, *a, **k):
            raise RuntimeError("not available in the CPU baseline")

    mod("open3d")
    mpl = mod("matplotlib")
    mpl.pyplot = mod("matplotlib.pyplot")
    mod("graphviz")
    ds = mod("dataset")
    ds.nerfsynthesis = mod("dataset.nerfsynthesis", NeRFSynthesis=_Unused)
    ep = mod("epcq")
    ep.epcq = mod("epcq.epcq", CameraSpec=_Unused)
    ut = mod("utils")
    ut.config = mod("utils.config", parser=None)


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


_STATE = {}


def _search_slice(args):
    which, lo, hi = args
    st = _STATE
    n = 0
    for i in range(lo, hi):
        o, d = st["o"], st["d"][i]
        if which == "kdtree":
            res = st["kdtree"].ray_search_radius_vector3d(st["kdtree"].root, o, d, st["r"])
        else:
            res = st["grid"].ray_search_radius_vector3d(o, d, st["r"])
        n += len(res)
    return n


def _child(n_rays, seed, workers, n_check):
    import multiprocessing as mp

    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "hashpoint-code_b200"))
    from hashpoint import synth
    _install_stubs()
    sys.path.insert(0, STAGE_DIR)
    import kdtree as K  # noqa: E402  (the reference's kdtree.py)
    import uniform_grid as U  # noqa: E402  (the reference's uniform_grid.py)

    sc = synth.make_sphere()
    cam = sc.cameras[0]
    r = float(sc.options.radius_threshold)
    xyz = sc.xyz.astype(np.float32)
    rng = np.random.default_rng(seed)
    pix = rng.choice(cam.width * cam.height, size=n_rays, replace=False)
    u, v = pix % cam.width, pix // cam.width
    R = cam.c2w[:3, :3].astype(np.float64)
    d = np.stack([(u + 0.5 - cam.cx) / cam.fx, (v + 0.5 - cam.cy) / cam.fy, np.ones(n_rays)], 1) @ R.T
    o = cam.c2w[:3, 3].astype(np.float64)
    out = {"rays": n_rays, "cores": workers, "cpu_model": _cpu_model(), "radius": r, "points": len(xyz),
           "workload": "sphere-100k-400x400 (pixel-centre rays, seed 0)"}
    t0 = time.perf_counter()
    grid = U.UniformGrid(xyz, 0.2)
    t1 = time.perf_counter()
    tree = K.KDTreeRaySearch(xyz, max_points_per_node=100)
    t2 = time.perf_counter()
    _STATE.update(kdtree=tree, grid=grid, o=o, d=d, r=r)
    ctx = mp.get_context("fork")  # a fresh CPU-only process: nothing here touches a GPU
    chunks = max(workers * 4, 1)
    bounds = [(n_rays * i // chunks, n_rays * (i + 1) // chunks) for i in range(chunks)]
    for which, build_s in (("kdtree", t2 - t1), ("uniform_grid", t1 - t0)):
        with ctx.Pool(workers) as pool:
            s0 = time.perf_counter()
            found = sum(pool.map(_search_slice, [(which, a, b) for a, b in bounds]))
            wall = time.perf_counter() - s0
        # result sets against brute force on the first n_check rays
        ok = 0
        for i in range(n_check):
            q = xyz.astype(np.float64) - o
            dn = d[i] / np.linalg.norm(d[i])
            dist = np.linalg.norm(q - (q @ dn)[:, None] * dn, axis=1)
            truth = set(np.nonzero(dist <= r)[0].tolist())
            if which == "kdtree":
                got = tree.ray_search_radius_vector3d(tree.root, o, d[i], r)
            else:
                got = grid.ray_search_radius_vector3d(o, d[i], r)
            ok += int(set(p.name for p in got) == truth)
        out[which] = {"rays_per_s": n_rays / wall, "search_s": wall, "build_s": build_s, "points_found": int(found),
                      "correct_rays": ok, "checked_rays": n_check, "correct": ok == n_check}
    return out


def run(n_rays=4096, seed=0, workers=None, n_check=32, timeout=600):
    """Time both searchers in a child process; returns the result dict (raises if not staged)."""
    if not staged():
        raise FileNotFoundError("reference CPU searchers not staged under %s" % STAGE_DIR)
    workers = workers or os.cpu_count() or 1
    cmd = [sys.executable, os.path.abspath(__file__), "--json", "--rays", str(n_rays), "--seed", str(seed),
           "--workers", str(workers), "--check", str(n_check)]
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError("reference CPU searchers failed:\n" + p.stderr[-2000:])
    return json.loads(p.stdout.strip().splitlines()[-1])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", metavar="REFERENCE_ROOT")
    ap.add_argument("--json", action="store_true")
    ap.add_argument("--rays", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--check", type=int, default=32)
    a = ap.parse_args()
    if a.stage:
        print(stage(a.stage))
    if a.json:
        print(json.dumps(_child(a.rays, a.seed, a.workers or os.cpu_count() or 1, a.check)), flush=True)
