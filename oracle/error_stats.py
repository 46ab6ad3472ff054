"""Error of the FP32 search+sample path against the FP64 oracle (test and
baseline infrastructure: the GPU tests and bench.py's CPU-baseline leg use it
as a checker; nothing in the product path does).

What is measured, on one view:
  depth     camera depth of every in-image point (sorted_depth) against the
            projection in double (epcq/epcq.py:251-257; ora_project_f64)
  t         sample depths sp_t against the FP64 twin of the sampling steps
            (ora_quick_sampling_f64: rays, tmin/tmax, t-bins and the walk of
            epcq_render_topk.cu:82-220 in double), over sampled rays whose
            emitted slots agree in both
  xyz       sample positions sp_xyz against the same twin (relative to |x|)
  ray_dist  distance of each selected point to its pixel ray
            (PointRayInterset, cuda_util.cuh:215-236) as the kernels compute
            it -- float32, in their operation order, on the library's own ray
            directions -- against the distance to the FP64 ray; absolute, and
            relative to the query radius

Rays where FP32 and FP64 make a different discrete choice (a point on the
radius changes the kept set and so tmin, a t on a bin edge changes the bin,
alpha * T on 1e-3 changes what is emitted) emit different slots or shift
their samples by a visible fraction of t_intvl; they are counted as
`decision_flips` (a sample depth more than 1e-5 relative off is one: rounding
alone stays two orders of magnitude below that), not folded into the error
figures.
"""
import numpy as np

import oracle


def _fma32(a, b, c):
    # a * b is exact in double for float32 operands; one rounding to double, one to float
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _dot3_32(a, b):
    # the kernels' dot3: fma(a2, b2, fma(a0, b0, a1 * b1))
    return _fma32(a[..., 2], b[..., 2], _fma32(a[..., 0], b[..., 0], (a[..., 1] * b[..., 1]).astype(np.float32)))


def _quantiles(x):
    if x.size == 0:
        return {"max": None, "median": None, "p99": None, "n": 0}
    return {"max": float(x.max()), "median": float(np.median(x)), "p99": float(np.quantile(x, 0.99)),
            "n": int(x.size)}


def fp64_error(xyz, cam, opt, sidx, sdep, hsh, sp_xyz, sp_t, mask, pc_idx, dirs, n_rays=4000, seed=0, nthreads=8):
    """Error statement of one view's FP32 outputs (numpy arrays from the CUDA path) against FP64.

    cam: a synth.PinholeCamera; dirs: [H*W, 3] ray directions of the library (hp_ray_directions)."""
    H, W = cam.height, cam.width
    ocam = oracle.camera_from(cam)
    xyz = np.ascontiguousarray(xyz, np.float32)
    # projection depth
    n_in = int((sidx >= 0).sum())
    ids = sidx[:n_in]
    d64 = oracle.project_f64(xyz, ocam)[ids]
    depth_rel = np.abs(sdep[:n_in].astype(np.float64) - d64) / np.maximum(np.abs(d64), 1e-30)
    # samples against the FP64 twin
    x64, t64, m64 = oracle.quick_sampling_f64(xyz, ocam, opt, sidx, hsh, nthreads=nthreads)
    rng = np.random.default_rng(seed)
    rays = rng.choice(H * W, size=min(n_rays, H * W), replace=False)
    vv, uu = rays // W, rays % W
    m32, mm = mask[vv, uu], m64[vv, uu]
    same = np.all(m32 == mm, axis=1)
    t32s, t64s = sp_t[vv, uu].astype(np.float64), t64[vv, uu]
    sel = same[:, None] & m32
    t_rel = np.abs(t32s[sel] - t64s[sel]) / np.maximum(np.abs(t64s[sel]), 1e-30)
    # a different kept set (tmin) or t-bin moves t far beyond rounding: a decision
    bin_flip = t_rel > 1e-5
    x32s, x64s = sp_xyz[vv, uu].astype(np.float64)[sel], x64[vv, uu][sel]
    x_rel = np.linalg.norm(x32s - x64s, axis=-1) / np.maximum(np.linalg.norm(x64s, axis=-1), 1e-30)
    # ray distances of the selected points, kernel arithmetic vs FP64
    c2w = cam.c2w.astype(np.float32)
    o32 = c2w[:3, 3]
    R64 = cam.c2w.astype(np.float64)[:3, :3]
    ray_of = np.repeat(np.arange(len(rays)), pc_idx.shape[2] * pc_idx.shape[3])
    sel_ids = pc_idx[vv, uu].reshape(-1)
    keep = (sel_ids >= 0) & np.repeat(same, pc_idx.shape[2] * pc_idx.shape[3])
    ray_of, sel_ids = ray_of[keep], sel_ids[keep]
    p = xyz[sel_ids]
    d32 = np.asarray(dirs, np.float32).reshape(-1, 3)[rays[ray_of]]
    s32 = (p - o32).astype(np.float32)
    num = _dot3_32(s32, d32)
    dd = _dot3_32(d32, d32)
    t = np.where(dd == 1.0, num, (num / dd).astype(np.float32)).astype(np.float32)
    e32 = np.stack([(p[:, i] - _fma32(t, d32[:, i], np.full_like(t, o32[i]))).astype(np.float32) for i in range(3)], 1)
    dist32 = np.linalg.norm(e32.astype(np.float64), axis=1).astype(np.float32).astype(np.float64)
    u64 = (uu[ray_of] + 0.5 - cam.cx) / cam.fx
    v64 = (vv[ray_of] + 0.5 - cam.cy) / cam.fy
    dir64 = np.stack([u64, v64, np.ones_like(u64)], 1) @ R64.T
    dir64 /= np.linalg.norm(dir64, axis=1, keepdims=True)
    q = p.astype(np.float64) - cam.c2w.astype(np.float64)[:3, 3]
    dist64 = np.linalg.norm(q - np.sum(q * dir64, 1, keepdims=True) * dir64, axis=1)
    r = float(opt.radius_threshold)
    big = dist64 > 1e-3 * r  # relative error is meaningless for points on the ray
    return {
        "rays": int(len(rays)), "rays_same_slots": int(same.sum()),
        "depth_rel": _quantiles(depth_rel),
        "t_rel": _quantiles(t_rel[~bin_flip]),
        "xyz_rel": _quantiles(x_rel[~bin_flip]),
        "ray_dist_abs_over_radius": _quantiles(np.abs(dist32 - dist64) / r),
        "ray_dist_rel": _quantiles(np.abs(dist32 - dist64)[big] / dist64[big]),
        "decision_flips": {"rays_with_other_slots": int((~same).sum()), "samples_moved": int(bin_flip.sum())},
    }
