"""Golden fixtures for the rows downstream of sampling: FeatureQuery.forward,
clamp_t, render and Aggregator.forward, produced by running the reference's
own Python code.

Those four are plain torch in the reference (epcq/epcq.py:328-529),
so this script imports the reference module from a checkout of the reference
(argument --ref, read only; the module's optional `open3d` import is replaced
by an empty stand-in, and its CUDA extension is not needed by these
functions) and runs them on the CPU.  The sampling outputs they consume are
taken from the committed quick_sampling fixtures (themselves outputs of the
reference's CUDA extension); point colours, directions and features are seeded
random values.  Writes fd_*.npz beside this script:

  python tests/golden/make_golden_downstream.py --ref <reference checkout>
"""
import argparse
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref):
    sys.modules.setdefault("open3d", types.ModuleType("open3d"))
    sys.path.insert(0, ref)
    import epcq.epcq as E  # the reference's module
    return E


def feature_case(E, src, name, seed, feat_dim, half, n_uv=None):
    g = np.load(os.path.join(HERE, src + ".npz"))
    rng = np.random.default_rng(seed)
    H, W = int(g["hw"][0]), int(g["hw"][1])
    fx, fy, cx, cy = [float(x) for x in g["cam_f"]]
    xyz = torch.from_numpy(g["xyz"]).float()
    n = xyz.shape[0]
    pts = types.SimpleNamespace(
        xyz_data=xyz,
        rgb_data=torch.from_numpy(rng.random((n, 3), dtype=np.float32)),
        dir_data=torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)),
        feat_data=torch.from_numpy(rng.standard_normal((n, feat_dim)).astype(np.float16 if half else np.float32)))
    sp_xyz = torch.from_numpy(g["sp_xyz"])
    pc_idx = torch.from_numpy(g["pc_idx"].astype(np.int64))
    mask = torch.from_numpy(g["mask"].astype(bool))
    c2w = torch.from_numpy(g["c2w"])
    cam = E.CameraSpec(c2w=c2w, w2c=torch.from_numpy(g["w2c"]), K=torch.from_numpy(g["K"]),
                       fx=torch.tensor(fx), fy=torch.tensor(fy), cx=torch.tensor(cx), cy=torch.tensor(cy),
                       width=torch.tensor(W), height=torch.tensor(H))
    uv = torch.zeros((0, 2), dtype=torch.int64)
    if n_uv:
        u = rng.integers(0, W, size=n_uv)
        v = rng.integers(0, H, size=n_uv)
        uv = torch.from_numpy(np.stack([u, v], 1).astype(np.int64))
        sp_xyz, pc_idx, mask = sp_xyz[uv[:, 1], uv[:, 0]], pc_idx[uv[:, 1], uv[:, 0]], mask[uv[:, 1], uv[:, 0]]
    out = E.FeatureQuery()(pts, sp_xyz, pc_idx, mask, cam, uv)
    keys = ("pc_xyz", "pc_rgb", "pc_dir", "pc_feat", "out_sp_xyz", "valid", "rays_d")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), kind="feature", xyz=g["xyz"], rgb=pts.rgb_data.numpy(),
                        dir=pts.dir_data.numpy(), feat=pts.feat_data.numpy(), sp_xyz=sp_xyz.numpy(),
                        pc_idx=pc_idx.numpy().astype(np.int32), mask=mask.numpy(), c2w=g["c2w"],
                        cam_f=np.array([fx, fy, cx, cy], np.float32), width=W, uv=uv.numpy().astype(np.int32),
                        **{k: v.numpy() for k, v in zip(keys, out)})
    print(name, "valid samples", out[0].shape[0])


def render_case(E, name, seed, R, S):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(2.0, 6.0, size=(R, S)).astype(np.float32), axis=1)
    # some exact repeats (gap 0) and some wide gaps, as clamp_t guards against
    t[:, 3] = t[:, 2]
    t[::7, 5:] += 0.5
    t = torch.from_numpy(t)
    sig = torch.from_numpy(rng.exponential(20.0, size=(R, S)).astype(np.float32))
    rgb = torch.from_numpy(rng.random((R, S, 3), dtype=np.float32))
    vsize = 0.004
    d = E.clamp_t(t, vsize)
    black = E.render(d, sig, rgb, white_bg=False)
    white = E.render(d, sig, rgb, white_bg=True)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), kind="render", t_val=t.numpy(), sigmas=sig.numpy(),
                        rgbs=rgb.numpy(), vsize=np.float32(vsize), t_dist=d.numpy(), color=black.numpy(),
                        color_white=white.numpy())
    print(name, R, S)


def aggregator_case(E, src, name, seed, n_rays):
    """Aggregator.forward on FeatureQuery outputs of n_rays rays (with samples) of a sampling
    fixture.  Features are fp32 of fp16-representable values (stored as fp16); the module is
    built with torch.manual_seed(seed) (xavier weights) and given random biases, and all its
    parameters are rounded to fp16-representable values (stored as fp16) before it runs.  The
    same inputs run with mask_out as [rays, S] (training layout) and as [h, w, S] (inference)."""
    g = np.load(os.path.join(HERE, src + ".npz"))
    rng = np.random.default_rng(seed)
    H, W = int(g["hw"][0]), int(g["hw"][1])
    fx, fy, cx, cy = [float(x) for x in g["cam_f"]]
    xyz = torch.from_numpy(g["xyz"]).float()
    n = xyz.shape[0]
    pts = types.SimpleNamespace(
        xyz_data=xyz,
        rgb_data=torch.from_numpy(rng.random((n, 3), dtype=np.float32)),
        dir_data=torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)),
        feat_data=torch.from_numpy(rng.standard_normal((n, 32)).astype(np.float16).astype(np.float32)))
    hit = np.flatnonzero(g["mask"].reshape(H * W, -1).any(-1))
    pick = np.sort(rng.choice(hit, n_rays, replace=False))
    uv = torch.from_numpy(np.stack([pick % W, pick // W], 1).astype(np.int64))
    sp_xyz = torch.from_numpy(g["sp_xyz"])[uv[:, 1], uv[:, 0]]
    pc_idx = torch.from_numpy(g["pc_idx"].astype(np.int64))[uv[:, 1], uv[:, 0]]
    mask = torch.from_numpy(g["mask"].astype(bool))[uv[:, 1], uv[:, 0]]
    cam = E.CameraSpec(c2w=torch.from_numpy(g["c2w"]), w2c=torch.from_numpy(g["w2c"]), K=torch.from_numpy(g["K"]),
                       fx=torch.tensor(fx), fy=torch.tensor(fy), cx=torch.tensor(cx), cy=torch.tensor(cy),
                       width=torch.tensor(W), height=torch.tensor(H))
    fq = E.FeatureQuery()(pts, sp_xyz, pc_idx, mask, cam, uv)
    pc_xyz, pc_rgb, pc_dir, pc_feat, out_sp, valid, rays_d = fq
    torch.manual_seed(seed)
    agg = E.Aggregator()
    params = {}
    with torch.no_grad():
        for mod_name, mod in agg.named_modules():
            if isinstance(mod, torch.nn.Linear):
                mod.bias.uniform_(-0.1, 0.1)
                mod.weight.copy_(mod.weight.half().float())
                mod.bias.copy_(mod.bias.half().float())
                params[mod_name] = (mod.weight.numpy().astype(np.float16), mod.bias.numpy().astype(np.float16))
        train = agg(pc_xyz, pc_rgb, pc_dir, pc_feat, out_sp, valid, mask, rays_d)
        side = int(round(n_rays ** 0.5))
        mask3 = mask.reshape(side, n_rays // side, -1)
        infer = agg(pc_xyz, pc_rgb, pc_dir, pc_feat, out_sp, valid, mask3, rays_d)
    arrays = {"w_" + k: w for k, (w, b) in params.items()}
    arrays.update({"b_" + k: b for k, (w, b) in params.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), kind="aggregator", pc_xyz=pc_xyz.numpy(),
                        pc_rgb=pc_rgb.numpy(), pc_dir=pc_dir.numpy(), pc_feat=pc_feat.numpy().astype(np.float16),
                        sp_xyz=out_sp.numpy(), valid=valid.numpy(), rays_d=rays_d.numpy(), mask=mask.numpy(),
                        mask3=mask3.numpy(), alpha_train=train[0].numpy(), color_train=train[1].numpy(),
                        alpha_infer=infer[0].numpy(), color_infer=infer[1].numpy(), **arrays)
    print(name, "samples", pc_xyz.shape[0], "valid points", int(valid.sum()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    args = ap.parse_args()
    E = load_reference(args.ref)
    torch.manual_seed(0)
    # (the reference's FeatureQuery needs float32 features: with float16 its index_put fails)
    feature_case(E, "shapes_96x80_k5_sorted", "fd_feature_shapes_uv", 1, 16, False, n_uv=1500)
    feature_case(E, "sphere_64_k3", "fd_feature_sphere", 2, 8, False)
    feature_case(E, "clusters_80x64_k5", "fd_feature_clusters_f3", 3, 3, False)
    render_case(E, "fd_render", 4, 2000, 16)
    aggregator_case(E, "shapes_96x80_k5_sorted", "fd_aggregator", 5, 256)


if __name__ == "__main__":
    main()
