"""CPU oracle (test infrastructure only) for the rows downstream of sampling:
FeatureQuery.forward's gather, clamp_t, render and the Aggregator MLP.

Each function restates the reference's torch code in float32 numpy:
  feature_query        epcq/epcq.py:333-387  (generate_rays :333-341, forward :344-387)
  clamp_t              epcq/epcq.py:508-515
  render               epcq/epcq.py:517-529
  positional_encoding  epcq/epcq.py:389-404  (ori=False)
  aggregator           epcq/epcq.py:406-507  (Aggregator.forward)
Gathers and copies are exact.  Ray directions, opacities and colours are
float32 expressions whose summation order (torch.sum, torch.cumprod) is not
specified by the reference, so they agree with it to within a few ulp; the
tests state their tolerance.  Parity is pinned by the fd_*.npz fixtures under
tests/golden/, made by running the reference's own code.
"""
import numpy as np


def generate_rays_d(c2w, fx, fy, cx, cy, width, height):
    """[H, W, 3] directions through pixel corners: ((u - cx) / fx, (v - cy) / fy, 1) @ R^T (epcq.py:333-341)."""
    f32 = np.float32
    y, x = np.meshgrid(np.arange(height, dtype=f32), np.arange(width, dtype=f32), indexing="ij")
    d = np.stack([(x - f32(cx)) / f32(fx), (y - f32(cy)) / f32(fy), np.ones_like(x)], -1).astype(f32)
    R = np.asarray(c2w, f32)[:3, :3]
    p = d[:, :, None, :] * R[None, None, :, :]       # products rounded to float32
    return ((p[..., 0] + p[..., 1]) + p[..., 2]).astype(f32)


def feature_query(xyz, rgb, dir_, feat, sp_xyz, pc_idx, mask, c2w, fx, fy, cx, cy, width, uv=None):
    """(pc_xyz, pc_rgb, pc_dir, pc_feat, out_sp_xyz, valid, rays_d) for the masked samples (epcq.py:344-387)."""
    S, P = pc_idx.shape[-2], pc_idx.shape[-1]
    m = np.asarray(mask, bool).reshape(-1)
    sp = np.asarray(sp_xyz, np.float32).reshape(-1, 3)[m]
    ids = np.asarray(pc_idx).reshape(-1, P)[m]
    valid = ids != -1
    def take(a):
        a = np.asarray(a)
        out = np.zeros(ids.shape + (a.shape[-1],), np.float32)
        out[valid] = a[ids[valid]].astype(np.float32)
        return out
    if uv is not None and len(uv):
        height = int(np.max(uv[:, 1])) + 1
        rd = generate_rays_d(c2w, fx, fy, cx, cy, width, height)[uv[:, 1], uv[:, 0]]
    else:
        height = (np.asarray(mask).size // S) // width
        rd = generate_rays_d(c2w, fx, fy, cx, cy, width, height).reshape(-1, 3)
    rd = np.repeat(rd.reshape(-1, 3), S, axis=0)[m]
    return take(xyz), take(rgb), take(dir_), take(feat), sp, valid, rd


def clamp_t(t_val, vsize=0.004):
    """Spacings t[s+1] - t[s] (last: vsize) with gaps < 1e-8 or > 2 vsize set to vsize (epcq.py:508-515)."""
    f32 = np.float32
    t = np.asarray(t_val, f32)
    d = np.concatenate([t[:, 1:] - t[:, :-1], np.full_like(t[:, :1], f32(vsize))], -1)
    mk = ((d < f32(1e-8)) | (d > f32(2) * f32(vsize))).astype(f32)
    return (d * (f32(1) - mk) + mk * f32(vsize)).astype(f32)


def render(deltas, sigmas, rgbs, white_bg=False):
    """Front-to-back composite, sequential in float32 (epcq.py:517-529)."""
    f32 = np.float32
    d, s, c = np.asarray(deltas, f32), np.asarray(sigmas, f32), np.asarray(rgbs, f32)
    R, S = s.shape
    op = (f32(1) - np.exp((-s * d).astype(f32))).astype(f32)
    trans = np.ones(R, f32)
    col = np.zeros((R, 3), f32)
    last = trans
    for k in range(S):
        last = trans
        col = (col + (op[:, k] * trans)[:, None] * c[:, k]).astype(f32)
        trans = (trans * ((f32(1) - op[:, k]) + f32(1e-10))).astype(f32)
    bg = f32(1) if white_bg else f32(0)
    return (col + last[:, None] * bg).astype(f32)


# the Aggregator's nn.Linear layers in module order: (name, out, in)
AGG_LAYERS = (("block1.0", 256, 284), ("block1.2", 256, 256), ("block3.0", 256, 263), ("block3.2", 256, 256),
              ("alpha_branch.0", 1, 256), ("color_branch.0", 128, 280), ("color_branch.2", 128, 128),
              ("color_branch.4", 128, 128), ("color_branch.6", 3, 128))


def positional_encoding(x, freqs):
    """[..., C] -> [..., 2 C freqs]: for channel c and band f (index c * freqs + f), sin and cos of
    x_c * 2^f, interleaved (epcq.py:389-404 with ori=False)."""
    f32 = np.float32
    x = np.asarray(x, f32)
    bands = (f32(2) ** np.arange(freqs)).astype(f32)
    p = (x[..., None] * bands).reshape(x.shape[:-1] + (freqs * x.shape[-1],)).astype(f32)
    return np.stack([np.sin(p), np.cos(p)], -1).reshape(p.shape[:-1] + (2 * p.shape[-1],)).astype(f32)


def aggregator(params, pc_xyz, pc_rgb, pc_dir, pc_feat, sp_xyz, valid, mask_out, rays_d):
    """(alphas, colors) of Aggregator.forward (epcq.py:441-507) in float32.

    params: {layer name: (weight [out, in], bias [out])}.  Inputs as FeatureQuery returns them:
    pc_* [M, P, *], sp_xyz and rays_d [M, 3], valid [M, P]; mask_out is the sampling mask,
    [H, W, S] (inference: alphas [H*W, S], colors [H*W, S, 3]) or [R, S] (training: [R, S],
    [R, S, 3]).  The reference's 20000-sample chunks do not change the per-row arithmetic."""
    f32 = np.float32
    Wt = {k: (np.asarray(w, f32), np.asarray(b, f32)) for k, (w, b) in params.items()}

    def lin(x, k):
        return (x @ Wt[k][0].T + Wt[k][1]).astype(f32)

    def leaky(x):
        return np.where(x > 0, x, x * f32(0.01)).astype(f32)

    pc_xyz, pc_rgb, pc_dir, pc_feat, sp_xyz, rays_d = (np.asarray(a, f32) for a in
                                                        (pc_xyz, pc_rgb, pc_dir, pc_feat, sp_xyz, rays_d))
    valid = np.asarray(valid, bool)
    M, P = valid.shape
    v = valid.reshape(-1)
    dist = (pc_xyz - sp_xyz[:, None, :]).astype(f32)
    distpow = (pc_xyz ** 2 - sp_xyz[:, None, :] ** 2).astype(f32)
    norm = np.sqrt((dist * dist).sum(-1)).astype(f32)
    inv = ((f32(1) / (norm + f32(1e-6))) * valid.astype(f32)).astype(f32)
    weights = (inv / (inv.sum(-1, keepdims=True) + f32(1e-6))).astype(f32)

    dist_feat = np.concatenate([dist, distpow], -1).reshape(-1, 6)[v]
    feat_in = pc_feat.reshape(-1, pc_feat.shape[-1])[v]
    rgb = pc_rgb.reshape(-1, 3)[v]
    dr = pc_dir.reshape(-1, 3)[v]
    rd = np.repeat(rays_d, P, axis=0)[v]
    x = np.concatenate([feat_in, positional_encoding(feat_in, 3), positional_encoding(dist_feat, 5)], -1)
    x = leaky(lin(leaky(lin(x, "block1.0")), "block1.2"))
    x = np.concatenate([x, rgb, dr - rd, (dr * rd).sum(-1, keepdims=True)], -1).astype(f32)
    x = leaky(lin(leaky(lin(x, "block3.0")), "block3.2"))
    z = lin(x, "alpha_branch.0") - f32(1)
    alphas = np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, f32(20))))).astype(f32)
    a = np.zeros((M * P, 1), f32)
    a[v] = alphas
    alpha_pred = (a.reshape(M, P) * weights).sum(-1, keepdims=True).astype(f32)
    canvas = np.zeros((M * P, x.shape[1]), f32)
    canvas[v] = x
    canvas = (canvas.reshape(M, P, -1) * weights[..., None]).sum(-2).astype(f32)
    c = np.concatenate([canvas, positional_encoding(rays_d, 4)], -1)
    c = leaky(lin(c, "color_branch.0"))
    c = leaky(lin(c, "color_branch.2"))
    c = leaky(lin(c, "color_branch.4"))
    c = lin(c, "color_branch.6")
    color = ((f32(1) / (f32(1) + np.exp(-c))) * f32(1 + 2 * 0.001) - f32(0.001)).astype(f32)

    m = np.asarray(mask_out, bool)
    fa = np.zeros(m.size, f32)
    fa[m.reshape(-1)] = alpha_pred.reshape(-1)
    fc = np.zeros((m.size, 3), f32)
    fc[m.reshape(-1)] = color
    rows = m.shape[0] * m.shape[1] if m.ndim == 3 else m.shape[0]
    S = m.shape[-1]
    return fa.reshape(rows, S), fc.reshape(rows, S, 3)
