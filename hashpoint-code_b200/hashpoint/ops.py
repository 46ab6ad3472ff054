"""Tensor-level entry points over the C ABI.

Each function validates its tensors the way the reference's TORCH_CHECKs do
(CUDA, contiguous; epcq/csrc/include/util.hpp:4-9), allocates its outputs with
torch on the inputs' device, and launches on torch's current CUDA stream.
Nothing here computes on the CPU: the work is the CUDA library's.
"""
import ctypes

import torch

from . import native

_vp = ctypes.c_void_p


def _ptr(t):
    return _vp(t.data_ptr()) if t is not None and t.numel() > 0 else _vp(0)


def _stream(device):
    return _vp(torch.cuda.current_stream(device).cuda_stream)


def check_input(t, name, dtype=None):
    if not isinstance(t, torch.Tensor):
        raise RuntimeError("%s must be a tensor" % name)
    if not t.is_cuda:
        raise RuntimeError("%s must be a CUDA tensor" % name)
    if not t.is_contiguous():
        raise RuntimeError("%s must be contiguous" % name)
    if dtype is not None and t.dtype != dtype:
        raise RuntimeError("%s must be %s, got %s" % (name, dtype, t.dtype))
    return t


def check_matrix(t, name, rows=3, cols=4):
    check_input(t, name, torch.float32)
    if t.dim() != 2 or t.shape[1] != cols or t.shape[0] < rows:
        raise RuntimeError("%s must be a [>=%d, %d] float32 matrix, got %s" % (name, rows, cols, tuple(t.shape)))
    return t


def make_camera(c2w=None, w2c=None, K=None, fx=0.0, fy=0.0, cx=0.0, cy=0.0, width=0, height=0):
    """HpCamera over device tensors (the caller keeps the tensors alive)."""
    cam = native.HpCamera()
    cam.c2w = _ptr(c2w).value
    cam.w2c = _ptr(w2c).value
    cam.K = _ptr(K).value
    cam.fx, cam.fy, cam.cx, cam.cy = float(fx), float(fy), float(cx), float(cy)
    cam.width, cam.height = int(width), int(height)
    return cam


def make_options(opt):
    o = native.HpOptions()
    o.kernel_size = int(opt.kernel_size)
    o.t_intvl = float(opt.t_intvl)
    o.radius_threshold = float(opt.radius_threshold)
    o.num_sample_points_per_ray = int(opt.num_sample_points_per_ray)
    o.num_point_cloud_per_sp = int(opt.num_point_cloud_per_sp)
    o.num_point_per_ray = int(opt.num_point_per_ray)
    o.sdf2weight_gaussian_alpha = float(opt.sdf2weight_gaussian_alpha)
    o.sdf2weight_gaussian_gamma = float(opt.sdf2weight_gaussian_gamma)
    return o


def pts2plane(xyz, w2c, K, height, width, sort=False):
    """Projection + hash table: (sorted_point_idx int32[N], sorted_depth f32[N], hash int32[H*W, 2])."""
    check_input(xyz, "xyz", torch.float32)
    if xyz.dim() != 2 or xyz.shape[1] != 3:
        raise RuntimeError("xyz must be [N, 3], got %s" % (tuple(xyz.shape),))
    check_matrix(w2c, "w2c")
    check_input(K, "K", torch.float32)
    if tuple(K.shape) != (3, 3):
        raise RuntimeError("K must be [3, 3], got %s" % (tuple(K.shape),))
    dev = xyz.device
    H, W = int(height), int(width)
    n = xyz.shape[0]
    L = native.lib()
    ws_bytes = L.hp_pts2plane_workspace_size(n, H, W)
    if ws_bytes == 0:
        raise RuntimeError("pts2plane: invalid sizes N=%d H=%d W=%d" % (n, H, W))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    sidx = torch.empty(n, dtype=torch.int32, device=dev)
    sdep = torch.empty(n, dtype=torch.float32, device=dev)
    hsh = torch.empty((H * W, 2), dtype=torch.int32, device=dev)
    cam = make_camera(w2c=w2c, K=K, width=W, height=H)
    rc = L.hp_pts2plane(_ptr(xyz), n, ctypes.byref(cam), int(bool(sort)), _ptr(sidx), _ptr(sdep), _ptr(hsh),
                        _ptr(ws), ws_bytes, _stream(dev))
    native.check(rc, "hp_pts2plane")
    return sidx, sdep, hsh


def scatter_hashtable(point_idx, point2img, depth, height, width, sort=False):
    check_input(point_idx, "point_idx_list", torch.int32)
    check_input(point2img, "point2img_idx_list", torch.int32)
    check_input(depth, "depth_list", torch.float32)
    n = point_idx.shape[0]
    if point2img.shape[0] != n or depth.shape[0] != n:
        raise RuntimeError("scatter_hashtable: input lengths differ")
    dev = point_idx.device
    H, W = int(height), int(width)
    sidx = torch.empty(n, dtype=torch.int32, device=dev)
    sdep = torch.empty(n, dtype=torch.float32, device=dev)
    hsh = torch.empty((H * W, 2), dtype=torch.int32, device=dev)
    rc = native.lib().hp_scatter_hashtable(_ptr(point_idx), _ptr(point2img), _ptr(depth), n, H, W, int(bool(sort)),
                                           _ptr(sidx), _ptr(sdep), _ptr(hsh), _stream(dev))
    native.check(rc, "hp_scatter_hashtable")
    return sidx, sdep, hsh


def _hash_view(hash_table, height, width):
    check_input(hash_table, "hashtable", torch.int32)
    if hash_table.dim() == 2:
        hash_table = hash_table.view(height, width, 2)
    if hash_table.dim() != 3 or tuple(hash_table.shape) != (height, width, 2):
        raise RuntimeError("hashtable size error: %s" % (tuple(hash_table.shape),))
    return hash_table


def make_tuning(heavy_window=0, blocks_per_sm=0, stage_config=0):
    """HpTuning for the sampling launches (0 = default for every field)."""
    return native.HpTuning(int(heavy_window), int(blocks_per_sm), int(stage_config))


def quick_sampling(xyz, c2w, fx, fy, cx, cy, width, height, opt, sorted_point_idx, hash_table, tuning=None):
    """(sp_xyz f32[H,W,S,3], pc_idx i32[H,W,S,P], sp_t f32[H,W,S], mask bool[H,W,S]).

    tuning: optional HpTuning (make_tuning); outputs do not depend on it."""
    check_input(xyz, "xyz_data", torch.float32)
    check_matrix(c2w, "c2w")
    check_input(sorted_point_idx, "sorted_point_idx_list", torch.int32)
    H, W = int(height), int(width)
    hash_table = _hash_view(hash_table, H, W)
    dev = xyz.device
    S, P = int(opt.num_sample_points_per_ray), int(opt.num_point_cloud_per_sp)
    sp_xyz = torch.empty((H, W, S, 3), dtype=torch.float32, device=dev)
    pc_idx = torch.empty((H, W, S, P), dtype=torch.int32, device=dev)
    sp_t = torch.empty((H, W, S), dtype=torch.float32, device=dev)
    mask = torch.empty((H, W, S), dtype=torch.bool, device=dev)
    cam = make_camera(c2w=c2w, fx=fx, fy=fy, cx=cx, cy=cy, width=W, height=H)
    o = make_options(opt)
    L = native.lib()
    ws_bytes = L.hp_quick_sampling_workspace_size(sorted_point_idx.numel(), H, W)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    rc = L.hp_quick_sampling_tuned(_ptr(xyz), xyz.shape[0], ctypes.byref(cam), ctypes.byref(o),
                                   _ptr(sorted_point_idx), sorted_point_idx.numel(), _ptr(hash_table), _ptr(sp_xyz),
                                   _ptr(pc_idx), _ptr(sp_t), _ptr(mask),
                                   ctypes.byref(tuning) if tuning is not None else None, _ptr(ws), ws_bytes,
                                   _stream(dev))
    native.check(rc, "hp_quick_sampling")
    return sp_xyz, pc_idx, sp_t, mask


def sampling_outputs(height, width, opt, device):
    """Uninitialised quick_sampling outputs (every element is written by the kernel)."""
    H, W = int(height), int(width)
    S, P = int(opt.num_sample_points_per_ray), int(opt.num_point_cloud_per_sp)
    return (torch.empty((H, W, S, 3), dtype=torch.float32, device=device),
            torch.empty((H, W, S, P), dtype=torch.int32, device=device),
            torch.empty((H, W, S), dtype=torch.float32, device=device),
            torch.empty((H, W, S), dtype=torch.bool, device=device))


def make_view(xyz, c2w, fx, fy, cx, cy, width, height, opt, sorted_point_idx, hash_table, outputs):
    """HpView for hp_quick_sampling_batch (the caller keeps the tensors alive)."""
    check_input(xyz, "xyz_data", torch.float32)
    check_matrix(c2w, "c2w")
    check_input(sorted_point_idx, "sorted_point_idx_list", torch.int32)
    H, W = int(height), int(width)
    hash_table = _hash_view(hash_table, H, W)
    sp_xyz, pc_idx, sp_t, mask = outputs
    v = native.HpView()
    v.xyz, v.n_points = _ptr(xyz).value, xyz.shape[0]
    v.sorted_point_idx, v.n_sorted = _ptr(sorted_point_idx).value, sorted_point_idx.numel()
    v.hash_table = _ptr(hash_table).value
    v.sp_xyz, v.pc_idx, v.sp_t, v.mask = (_ptr(sp_xyz).value, _ptr(pc_idx).value, _ptr(sp_t).value,
                                          _ptr(mask).value)
    v.cam = make_camera(c2w=c2w, fx=fx, fy=fy, cx=cx, cy=cy, width=W, height=H)
    v.opt = make_options(opt)
    return v


def batch_workspace_size(views):
    n = len(views)
    return native.lib().hp_quick_sampling_batch_workspace_size((native.HpView * n)(*views), n)


def quick_sampling_batch(views, device, views_device=None, workspace=None, heavy_window=0, blocks_per_sm=0,
                         stage_config=0):
    """hp_quick_sampling_batch over a list of HpView (see make_view); outputs are the views' own tensors.

    views_device: optional uint8 CUDA tensor holding the same table (for CUDA-graph capture).
    workspace: optional uint8 CUDA tensor of at least batch_workspace_size(views) bytes.
    heavy_window, blocks_per_sm, stage_config: launch tuning (0 = default); outputs do not depend on it."""
    L = native.lib()
    n = len(views)
    table = (native.HpView * n)(*views)
    ws_bytes = L.hp_quick_sampling_batch_workspace_size(table, n)
    if ws_bytes == 0:
        raise RuntimeError("hp_quick_sampling_batch: invalid views")
    if workspace is None:
        workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    tuning = make_tuning(heavy_window, blocks_per_sm, stage_config)
    rc = L.hp_quick_sampling_batch(table, _ptr(views_device), n, ctypes.byref(tuning), _ptr(workspace),
                                   workspace.numel(), _stream(torch.device(device)))
    native.check(rc, "hp_quick_sampling_batch")


def quick_query(xyz, c2w, fx, fy, cx, cy, width, height, opt, sorted_point_idx, hash_table, ray_ids):
    check_input(xyz, "xyz_data", torch.float32)
    check_matrix(c2w, "c2w")
    check_input(sorted_point_idx, "sorted_point_idx_list", torch.int32)
    check_input(ray_ids, "indices_of_ray", torch.int32)
    H, W = int(height), int(width)
    hash_table = _hash_view(hash_table, H, W)
    dev = xyz.device
    R = ray_ids.shape[0]
    cap = int(opt.num_point_per_ray)
    out = torch.full((R, cap), -1, dtype=torch.int32, device=dev) if R == 0 or cap == 0 else \
        torch.empty((R, cap), dtype=torch.int32, device=dev)
    cam = make_camera(c2w=c2w, fx=fx, fy=fy, cx=cx, cy=cy, width=W, height=H)
    o = make_options(opt)
    rc = native.lib().hp_quick_query_for_nearby_point(_ptr(xyz), xyz.shape[0], ctypes.byref(cam), ctypes.byref(o),
                                                      _ptr(sorted_point_idx), sorted_point_idx.numel(),
                                                      _ptr(hash_table), _ptr(ray_ids), R, _ptr(out), _stream(dev))
    native.check(rc, "hp_quick_query_for_nearby_point")
    return out


def scatter_multibin(point_idx, point2img, depth, height, width, bins):
    check_input(point_idx, "point_idx_list", torch.int32)
    check_input(point2img, "point2img_idx_list", torch.int32)
    check_input(depth, "depth_list", torch.float32)
    dev = point_idx.device
    H, W = int(height), int(width)
    bd = torch.empty((H * W, int(bins)), dtype=torch.float32, device=dev)
    bi = torch.empty((H * W, int(bins)), dtype=torch.int32, device=dev)
    rc = native.lib().hp_scatter(_ptr(point_idx), _ptr(point2img), _ptr(depth), point_idx.shape[0], H, W, int(bins),
                                 _ptr(bd), _ptr(bi), _stream(dev))
    native.check(rc, "hp_scatter")
    return bd, bi


def ray_directions(c2w, fx, fy, cx, cy, width, height):
    check_matrix(c2w, "c2w")
    H, W = int(height), int(width)
    out = torch.empty((H * W, 3), dtype=torch.float32, device=c2w.device)
    cam = make_camera(c2w=c2w, fx=fx, fy=fy, cx=cx, cy=cy, width=W, height=H)
    rc = native.lib().hp_ray_directions(ctypes.byref(cam), _ptr(out), _stream(c2w.device))
    native.check(rc, "hp_ray_directions")
    return out


# ---------------------------------------------------------------------------
# downstream of sampling: FeatureQuery gather, clamp_t, render
# ---------------------------------------------------------------------------
def mask_scan(mask):
    """(offsets int32 [n], count int32 [1]) of a bool/uint8 mask: the exclusive scan of its set entries."""
    check_input(mask, "mask")
    if mask.dtype not in (torch.bool, torch.uint8):
        raise RuntimeError("mask must be bool or uint8")
    n = mask.numel()
    dev = mask.device
    offsets = torch.empty(n, dtype=torch.int32, device=dev)
    count = torch.empty(1, dtype=torch.int32, device=dev)
    L = native.lib()
    ws_bytes = L.hp_mask_scan_workspace_size(n)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    rc = L.hp_mask_scan(_ptr(mask), n, _ptr(offsets), _ptr(count), _ptr(ws), ws_bytes, _stream(dev))
    native.check(rc, "hp_mask_scan")
    return offsets, count


def feature_query(xyz, rgb, dir_, feat, sp_xyz, pc_idx, mask, c2w, fx, fy, cx, cy, width, ray_uv=None):
    """FeatureQuery.forward's gather (epcq/epcq.py:345-387) on the GPU.

    Returns (pc_xyz [M,P,3], pc_rgb [M,P,3], pc_dir [M,P,3], pc_feat [M,P,F] f32, sp_xyz [M,3],
    valid bool [M,P], rays_d [M,3]) for the M samples whose mask is set.  The sample count is read
    back to size the outputs (one host synchronisation, as the reference's boolean indexing does)."""
    for t, nme in ((xyz, "xyz_data"), (rgb, "rgb_data"), (dir_, "dir_data"), (sp_xyz, "output_sp_xyz")):
        check_input(t, nme, torch.float32)
    check_input(feat, "feat_data")
    if feat.dtype not in (torch.float32, torch.float16):
        raise RuntimeError("feat_data must be float32 or float16")
    check_input(pc_idx, "output_pc_idx", torch.int32)
    check_matrix(c2w, "c2w")
    S, P = int(pc_idx.shape[-2]), int(pc_idx.shape[-1])
    n_rays = pc_idx.numel() // max(S * P, 1)
    if mask.numel() != n_rays * S or sp_xyz.numel() != n_rays * S * 3:
        raise RuntimeError("mask_out / output_sp_xyz do not match output_pc_idx")
    if ray_uv is not None:
        ray_uv = ray_uv.to(device=xyz.device, dtype=torch.int32).contiguous()
        if ray_uv.shape != (n_rays, 2):
            raise RuntimeError("ray_index_uv must be [rays, 2] (u, v)")
    mask = mask.contiguous()
    offsets, count = mask_scan(mask)
    M = int(count.item())
    dev = xyz.device
    F = int(feat.shape[-1]) if feat.dim() == 2 else 0
    out = (torch.empty((M, P, 3), dtype=torch.float32, device=dev), torch.empty((M, P, 3), dtype=torch.float32, device=dev),
           torch.empty((M, P, 3), dtype=torch.float32, device=dev), torch.empty((M, P, F), dtype=torch.float32, device=dev),
           torch.empty((M, 3), dtype=torch.float32, device=dev), torch.empty((M, P), dtype=torch.bool, device=dev),
           torch.empty((M, 3), dtype=torch.float32, device=dev))
    if M == 0:
        return out
    pts = native.HpPointAttrs(_ptr(xyz).value, _ptr(rgb).value, _ptr(dir_).value, _ptr(feat).value, F,
                              int(feat.dtype == torch.float16), xyz.shape[0])
    cam = make_camera(c2w=c2w, fx=fx, fy=fy, cx=cx, cy=cy, width=width, height=1)
    rc = native.lib().hp_feature_query(ctypes.byref(pts), _ptr(sp_xyz), _ptr(pc_idx), _ptr(mask), n_rays, S, P,
                                       _ptr(offsets), ctypes.byref(cam), _ptr(ray_uv), *[_ptr(t) for t in out[:4]],
                                       _ptr(out[4]), _ptr(out[5]), _ptr(out[6]), _stream(dev))
    native.check(rc, "hp_feature_query")
    return out


def clamp_t(t_val, vsize=0.004):
    """clamp_t (epcq/epcq.py:508-515) on the GPU: t_val [R, S] -> t_dist [R, S]."""
    check_input(t_val, "t_val", torch.float32)
    R, S = t_val.shape
    out = torch.empty_like(t_val)
    rc = native.lib().hp_clamp_t(_ptr(t_val), R, S, float(vsize), _ptr(out), _stream(t_val.device))
    native.check(rc, "hp_clamp_t")
    return out


def render(deltas, sigmas, rgbs, white_bg=False, t_val=None, vsize=0.004):
    """render (epcq/epcq.py:517-529) on the GPU: colour [R, 3].  With deltas None, the spacings are
    clamp_t(t_val, vsize), computed inside the same kernel."""
    check_input(sigmas, "sigmas", torch.float32)
    check_input(rgbs, "rgbs", torch.float32)
    R, S = sigmas.shape
    if rgbs.shape != (R, S, 3):
        raise RuntimeError("rgbs must be [rays, samples, 3]")
    if deltas is not None:
        check_input(deltas, "deltas", torch.float32)
        if deltas.shape != (R, S):
            raise RuntimeError("deltas must match sigmas")
    elif t_val is None or tuple(t_val.shape) != (R, S):
        raise RuntimeError("render needs deltas or t_val of the sigmas' shape")
    else:
        check_input(t_val, "t_val", torch.float32)
    color = torch.empty((R, 3), dtype=torch.float32, device=sigmas.device)
    rc = native.lib().hp_render(_ptr(deltas), _ptr(t_val), float(vsize), _ptr(sigmas), _ptr(rgbs), R, S,
                                int(bool(white_bg)), _ptr(color), _stream(sigmas.device))
    native.check(rc, "hp_render")
    return color


# ---------------------------------------------------------------------------
# Aggregator (epcq/epcq.py:406-507) on the tensor cores
# ---------------------------------------------------------------------------
# the nine nn.Linear layers in module order: (name, out, in)
AGG_LAYERS = (("block1.0", 256, 284), ("block1.2", 256, 256), ("block3.0", 256, 263), ("block3.2", 256, 256),
              ("alpha_branch.0", 1, 256), ("color_branch.0", 128, 280), ("color_branch.2", 128, 128),
              ("color_branch.4", 128, 128), ("color_branch.6", 3, 128))


def aggregator_pack(weights, biases):
    """Pack the Aggregator's nine layers (fp32 weight [out, in] and bias [out] device tensors, module
    order) into the bf16 operand tiles + fp32 parameters the forward kernels read (uint8 tensor)."""
    if len(weights) != 9 or len(biases) != 9:
        raise RuntimeError("aggregator_pack: nine layers expected")
    w = native.HpAggregatorWeights()
    keep = []
    for i, ((name, n_out, n_in), W, b) in enumerate(zip(AGG_LAYERS, weights, biases)):
        W = W.detach().to(torch.float32).contiguous()
        b = b.detach().to(torch.float32).contiguous()
        if tuple(W.shape) != (n_out, n_in) or tuple(b.shape) != (n_out,) or not W.is_cuda or not b.is_cuda:
            raise RuntimeError("aggregator_pack: %s must be CUDA fp32 [%d, %d] with bias [%d]" %
                               (name, n_out, n_in, n_out))
        keep += [W, b]
        w.weight[i] = W.data_ptr()
        w.bias[i] = b.data_ptr()
    dev = keep[0].device
    L = native.lib()
    size = L.hp_aggregator_packed_size()
    packed = torch.empty(size, dtype=torch.uint8, device=dev)
    rc = L.hp_aggregator_pack(ctypes.byref(w), _ptr(packed), size, _stream(dev))
    native.check(rc, "hp_aggregator_pack")
    packed._hp_keep = keep  # the sources stay alive until the packing kernel has run
    return packed


def aggregator_forward(packed, pc_xyz, pc_rgb, pc_dir, pc_feat, output_sp_xyz, valid_sp_mask_out, mask_out, rays_d,
                       check_status=False):
    """Aggregator.forward (epcq/epcq.py:441-507) on the GPU: (alphas, colors) -- [H*W, S] and
    [H*W, S, 3] for a sampling mask [H, W, S], [R, S] and [R, S, 3] for [R, S] -- zeros where
    mask_out is not set.  bf16 operands, fp32 accumulation.  check_status synchronises and raises
    if a wait inside the kernels gave up."""
    for t, nme in ((pc_xyz, "pc_xyz"), (pc_rgb, "pc_rgb"), (pc_dir, "pc_dir"), (pc_feat, "pc_feat"),
                   (output_sp_xyz, "output_sp_xyz"), (rays_d, "rays_d")):
        check_input(t, nme, torch.float32)
    check_input(valid_sp_mask_out, "valid_sp_mask_out")
    check_input(mask_out, "mask_out")
    if mask_out.dim() not in (2, 3):
        raise ValueError("mask_out shape error")
    if valid_sp_mask_out.dim() != 2:
        raise RuntimeError("valid_sp_mask_out must be [samples, points]")
    M, P = valid_sp_mask_out.shape
    if (pc_xyz.shape != (M, P, 3) or pc_rgb.shape != (M, P, 3) or pc_dir.shape != (M, P, 3) or
            pc_feat.dim() != 3 or pc_feat.shape[:2] != (M, P) or output_sp_xyz.shape != (M, 3) or
            rays_d.shape != (M, 3)):
        raise RuntimeError("aggregator: inputs do not match valid_sp_mask_out [%d, %d]" % (M, P))
    dev = pc_xyz.device
    S = mask_out.shape[-1]
    rows = mask_out.numel() // max(S, 1)
    alphas = torch.empty((rows, S), dtype=torch.float32, device=dev)
    colors = torch.empty((rows, S, 3), dtype=torch.float32, device=dev)
    offsets, _ = mask_scan(mask_out)
    L = native.lib()
    ws_bytes = L.hp_aggregator_workspace_size(M)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    rc = L.hp_aggregator_forward(_ptr(packed), _ptr(pc_xyz), _ptr(pc_rgb), _ptr(pc_dir), _ptr(pc_feat),
                                 int(pc_feat.shape[2]), _ptr(output_sp_xyz), _ptr(valid_sp_mask_out), _ptr(rays_d),
                                 M, P, _ptr(mask_out), _ptr(offsets), mask_out.numel(), _ptr(alphas), _ptr(colors),
                                 _ptr(ws), ws_bytes, _stream(dev))
    native.check(rc, "hp_aggregator_forward")
    if check_status:
        native.check(L.hp_aggregator_status(_ptr(ws), M, _stream(dev)), "hp_aggregator_forward")
    return alphas, colors
