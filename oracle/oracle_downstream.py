"""CPU oracle (test infrastructure only) for the rows downstream of sampling:
FeatureQuery.forward's gather, clamp_t and render.

Each function restates the reference's torch code in float32 numpy:
  feature_query  epcq/epcq.py:333-387  (generate_rays :333-341, forward :344-387)
  clamp_t        epcq/epcq.py:508-515
  render         epcq/epcq.py:517-529
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
