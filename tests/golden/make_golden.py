"""Generate golden fixtures by running the reference's own CUDA extension.

Runs on a CUDA machine.  It loads the reference extension compiled from the
reference's sources by oracle/build_ref.py (oracle/_ref/epcq_ref_csrc.so) and
drives it exactly as the reference's Python layer does:

  projection   epcq/epcq.py:251-274  (torch matmuls, divide, int32 cast, where)
  sort+gather  epcq/epcq.py:283-286  (torch.sort by pixel id, gathers)
  hash table   _C.scatter_hashtable  (epcq/csrc/rasterization.cu:130-171)
  sampling     _C.quick_sampling     (epcq/csrc/epcq_render_topk.cu:341-417)
  ray query    _C.quick_query_for_nearby_point (epcq_render_topk.cu:287-339)
  multi-bin    _C.scatter            (rasterization.cu:88-128)

Inputs are kept inside the envelope where the reference kernels are free of
their known out-of-bounds accesses and divergent-barrier hazards:
  * point2img is passed as a view of a buffer with one extra sentinel element,
    so the bucket walk at rasterization.cu:23 stops at index N;
  * quick_sampling runs with num_point_cloud_per_sp = 8 (the id buffer of
    epcq_render_topk.cu:35,77 holds 8 entries);
  * kernel_size <= 5 (window lists hold 32 cells);
  * quick_query runs on scenes whose every pixel is occupied and with a ray
    count that fills whole blocks, so no thread leaves before the
    __syncthreads at epcq_render_topk.cu:270;
  * scatter only sees positive depths (rasterization.cu:56 never advances on a
    negative depth) and bins >= 5 (its block size is 48 KiB / (bins * 9.6 B),
    which exceeds 1024 threads below 5 bins, rasterization.cu:114-118).

Each case is written as a compressed .npz into --out.  The fixtures committed
under tests/golden/ were produced by:  python tests/golden/make_golden.py --out <dir>
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "hashpoint-code_b200"))

from hashpoint import synth  # noqa: E402
from ref_pipeline import OPT_FIELDS, RefPipeline  # noqa: E402,F401  (RefPipeline: used by the parity tests too)


def plane_cloud(rng, n, cam, depth=2.0, jitter=0.0):
    """Points on the plane z_cam = depth covering the whole image (every pixel occupied)."""
    u = rng.uniform(0.0, cam.width, size=n)
    v = rng.uniform(0.0, cam.height, size=n)
    z = depth + rng.normal(0.0, jitter, size=n) if jitter else np.full(n, depth)
    xc = (u - cam.cx) / cam.fx * z
    yc = (v - cam.cy) / cam.fy * z
    pc = np.stack([xc, yc, z, np.ones(n)], 1)
    pw = pc @ cam.c2w.astype(np.float64).T
    return pw[:, :3].astype(np.float32)


def build_cases():
    cases = []
    # 1. sphere, 3x3 window, id-ordered buckets
    rng = np.random.default_rng(101)
    cam = synth.look_at_camera((0, 0, 4), (0, 0, 0), 64, 64, 80.0)
    cases.append(dict(name="sphere_64_k3", xyz=synth.sphere_cloud(rng, 6000), cam=cam, sort=False,
                      opt=synth.Options(kernel_size=3, radius_threshold=0.04, num_sample_points_per_ray=8,
                                        num_point_cloud_per_sp=8), scatter_bins=[6, 8, 16]))
    # 2. shapes, 5x5 window, depth-ordered buckets, non-square image
    rng = np.random.default_rng(102)
    xyz = synth.shapes_cloud(rng, 20000)
    cam = synth.orbit_cameras(rng, 1, 4.0, 96, 80, 110.0, 48.0, 40.0)[0]
    cases.append(dict(name="shapes_96x80_k5_sorted", xyz=xyz, cam=cam, sort=True,
                      opt=synth.Options(kernel_size=5, radius_threshold=0.03, num_sample_points_per_ray=8,
                                        num_point_cloud_per_sp=8), scatter_bins=[8]))
    # 3. clusters: deep buckets (exercises the 48-per-cell cap), S=16, wider bins
    rng = np.random.default_rng(103)
    xyz = synth.clusters_cloud(rng, 30000)
    cam = synth.orbit_cameras(rng, 1, None, 80, 64, 150.0, 40.0, 32.0, elev_deg=(40, 70),
                              radius_range=(2.5, 3.5))[0]
    cases.append(dict(name="clusters_80x64_k5", xyz=xyz, cam=cam, sort=False,
                      opt=synth.Options(kernel_size=5, radius_threshold=0.02, t_intvl=0.02,
                                        num_sample_points_per_ray=16, num_point_cloud_per_sp=8)))
    # 4. even window, off-centre camera (off-image tail), camera inside the cloud's hull so
    #    some points are behind the camera and alias into the image (no z filter in the reference)
    rng = np.random.default_rng(104)
    xyz = synth.sphere_cloud(rng, 8000)
    cam = synth.look_at_camera((0.3, 0.2, 1.4), (0.9, -0.4, 0.0), 72, 56, 60.0, 60.0, 30.0, 31.0)
    cases.append(dict(name="sphere_72x56_k4_behind", xyz=xyz, cam=cam, sort=True,
                      opt=synth.Options(kernel_size=4, radius_threshold=0.05, num_sample_points_per_ray=8,
                                        num_point_cloud_per_sp=8)))
    # 5. tiny windows and a soft T-walk (more samples per ray)
    rng = np.random.default_rng(105)
    xyz = synth.shapes_cloud(rng, 15000)
    cam = synth.orbit_cameras(rng, 1, 4.0, 64, 64, 90.0)[0]
    for k in (1, 2):
        cases.append(dict(name="shapes_64_k%d_soft" % k, xyz=xyz, cam=cam, sort=False,
                          opt=synth.Options(kernel_size=k, radius_threshold=0.05, num_sample_points_per_ray=8,
                                            num_point_cloud_per_sp=8, sdf2weight_gaussian_gamma=0.3,
                                            sdf2weight_gaussian_alpha=0.05)))
    # 6. full-frame plane: every pixel occupied, border windows clamp onto duplicates
    rng = np.random.default_rng(106)
    cam = synth.look_at_camera((0.1, -0.2, 3.0), (0, 0, 0), 48, 40, 50.0)
    xyz = plane_cloud(rng, 48 * 40 * 24, cam, depth=2.0, jitter=0.01)
    cases.append(dict(name="plane_48x40_k5_dense", xyz=xyz, cam=cam, sort=False,
                      opt=synth.Options(kernel_size=5, radius_threshold=0.03, num_sample_points_per_ray=8,
                                        num_point_cloud_per_sp=8),
                      query=dict(n_rays=64, num_point_per_ray=[256, 16]), scatter_bins=[6]))
    cases.append(dict(name="plane_48x40_k3_query", xyz=xyz, cam=cam, sort=True,
                      opt=synth.Options(kernel_size=3, radius_threshold=0.02, num_sample_points_per_ray=16,
                                        num_point_cloud_per_sp=8),
                      query=dict(n_rays=96, num_point_per_ray=[256, 8])))
    return cases


def run_case(rp, case, dev):
    cam = case["cam"]
    H, W = cam.height, cam.width
    opt = case["opt"]
    assert opt.num_point_cloud_per_sp == 8 and 1 <= opt.kernel_size <= 5
    xyz = torch.from_numpy(case["xyz"]).to(dev).contiguous()
    c2w = torch.from_numpy(cam.c2w).to(dev).contiguous()
    w2c = torch.from_numpy(cam.w2c).to(dev).contiguous()
    K = torch.from_numpy(cam.K).to(dev).contiguous()
    pid, depth, sx, sy, pts_c = rp.project(xyz, w2c, K, H, W)
    pid_s, perm, depth_s, idx_s = rp.sort(pid, depth)
    pid_st, perm_st = torch.sort(pid, stable=True)
    stable_equal = bool(torch.equal(perm, perm_st))
    sidx, sdep, hsh = rp.scatter_hashtable(idx_s, pid_s, depth_s, H, W, case["sort"])
    npspec = rp.C.NeuralPointsSpec()
    npspec.xyz_data = xyz
    cspec = rp.camera_spec(c2w, w2c, cam)
    ospec = rp.options_spec(opt)
    outs = rp.C.quick_sampling(npspec, cspec, ospec, sidx, hsh)
    torch.cuda.synchronize()
    reruns = []
    for _ in range(3):
        o2 = rp.C.quick_sampling(npspec, cspec, ospec, sidx, hsh)
        reruns.append([int((a != b).sum()) for a, b in zip(outs, o2)])
    sp_xyz, pc_idx, sp_t, mask = [t.cpu().numpy() for t in outs]
    rec = dict(
        xyz=case["xyz"], c2w=cam.c2w, w2c=cam.w2c, K=cam.K,
        cam_f=np.array([cam.fx, cam.fy, cam.cx, cam.cy], np.float32), hw=np.array([H, W], np.int32),
        options=json.dumps({f: getattr(opt, f) for f in OPT_FIELDS}), sort=np.array(case["sort"]),
        point2img=pid.cpu().numpy(), depth=depth.cpu().numpy(),
        screen_x=sx.cpu().numpy(), screen_y=sy.cpu().numpy(), pts_c=pts_c.cpu().numpy(),
        perm=perm.cpu().numpy(), sort_is_stable=np.array(stable_equal),
        sorted_point_idx=sidx.cpu().numpy(), sorted_depth=sdep.cpu().numpy(), hash_table=hsh.cpu().numpy(),
        sp_xyz=sp_xyz, pc_idx=pc_idx, sp_t=sp_t, mask=mask, rerun_mismatch=np.array(reruns, np.int64),
    )
    q = case.get("query")
    if q is not None:
        occupied = int((hsh[:, 1] > 0).sum())
        assert occupied == H * W, "quick_query golden needs every pixel occupied"
        assert q["n_rays"] % 4 == 0
        rng = np.random.default_rng(7)
        rays = rng.choice(H * W, size=q["n_rays"], replace=False).astype(np.int32)
        rays_t = torch.from_numpy(rays).to(dev)
        rec["query_rays"] = rays
        for npr in q["num_point_per_ray"]:
            o = synth.Options(**{f: getattr(opt, f) for f in OPT_FIELDS})
            o.num_point_per_ray = npr
            out = rp.C.quick_query_for_nearby_point(npspec, cspec, rp.options_spec(o), sidx, hsh, rays_t)
            torch.cuda.synchronize()
            rec["query_out_%d" % npr] = np.sort(out.cpu().numpy(), axis=1)
            rec["query_count_%d" % npr] = (out >= 0).sum(1).cpu().numpy().astype(np.int32)
    for bins in case.get("scatter_bins", []):
        bd, bi = rp.scatter(idx_s, pid_s, depth_s, H, W, bins)
        torch.cuda.synchronize()
        rec["scatter_depth_%d" % bins] = bd.cpu().numpy()
        rec["scatter_idx_%d" % bins] = bi.cpu().numpy()
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    import build_ref
    mod = build_ref.load()
    dev = torch.device("cuda:0")
    rp = RefPipeline(mod, dev)
    os.makedirs(a.out, exist_ok=True)
    for case in build_cases():
        t0 = time.time()
        rec = run_case(rp, case, dev)
        np.savez_compressed(os.path.join(a.out, case["name"] + ".npz"), **rec)
        print("%-28s N=%d HW=%dx%d emitted=%d maxbucket=%d stable=%s rerun=%s (%.2fs)" % (
            case["name"], len(case["xyz"]), rec["hw"][0], rec["hw"][1], int(rec["mask"].sum()),
            int(rec["hash_table"][:, 1].max()), bool(rec["sort_is_stable"]),
            rec["rerun_mismatch"].max(0).tolist(), time.time() - t0), flush=True)


if __name__ == "__main__":
    main()
