"""Drop-in `epcq.epcq` module: the reference's point searching and sampling API.

Mirrors the reference's epcq/epcq.py entry points, tensor layouts and return
signatures for the search+sample path:

  CameraSpec, RenderOptions (same defaults), NeuralPointsGrads   (:15-145)
  NeuralPoints(pc_type in {'pointnerf', 'gt_pc', 'pc'})          (:147-221)
    .pts2plane(cam, opt, pc_xyz=None, sort=False)                (:279-295)
        -> sorted_point_idx_list int32[N], sorted_depth_list f32[N], hash_table int32[H*W, 2]
    .render_image_hashtable_topk(cam, opt, idx, depth, hash)      (:297-327)
        -> sp_xyz f32[H,W,S,3], pc_idx int32[H,W,S,P], sp_t f32[H,W,S], mask bool[H,W,S]

  FeatureQuery().forward(neuralpoints, sp_xyz, pc_idx, mask, cam, ray_index_uv) (:328-387)
  positional_encoding(positions, freqs, ori=False)                (:389-404)
  Aggregator().forward(pc_xyz, pc_rgb, pc_dir, pc_feat, sp_xyz, valid, mask_out, rays_d) (:406-507)
  clamp_t(t_val, vsize), render(deltas, sigmas, rgbs, white_bg)   (:508-529)

pts2plane runs the projection, the per-pixel counting sort and the bucket
order in the CUDA library (one call, no torch.sort); render_image_hashtable_topk
runs the fused search/sample kernel.  Both launch on torch's current stream.
"""
import os
from dataclasses import dataclass
from typing import Union

import torch
import torch.nn as nn

from . import utils
from hashpoint import ops

_C = utils._get_c_extension()


def _scalar(v):
    return v.item() if isinstance(v, torch.Tensor) else v


def _host_values(*vals):
    """The values of Python numbers and one-element tensors as Python numbers, the tensors read
    back with one device-to-host copy per device (the reference's callers pass 0-d CUDA tensors for
    fx..height, opt/render_image.py:61-68; reading each with .item() waits on the stream once per
    value).  Tensors holding integers come back as int, the rest as float (float32 values and
    integers below 2^53 survive the float64 round trip exactly)."""
    out = list(vals)
    groups = {}
    for i, v in enumerate(vals):
        if isinstance(v, torch.Tensor):
            if v.numel() != 1:
                raise RuntimeError("a camera scalar must hold one element, got shape %s" % (tuple(v.shape),))
            groups.setdefault(v.device, []).append(i)
    for dev, idx in groups.items():
        if len(idx) == 1 or dev.type != "cuda":
            for i in idx:
                out[i] = vals[i].item()
            continue
        host = torch.stack([vals[i].reshape(()).to(torch.float64) for i in idx]).cpu().tolist()
        for i, h in zip(idx, host):
            is_int = not (vals[i].dtype.is_floating_point or vals[i].dtype.is_complex)
            out[i] = int(h) if is_int else h
    return out


@dataclass
class CameraSpec:
    c2w: torch.Tensor
    w2c: torch.Tensor
    K: torch.Tensor
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int

    def _host(self):
        """(fx, fy, cx, cy, width, height) as Python numbers.  Tensor fields are read back
        together and the values kept on the camera while its fields are the same objects at the
        same version (an in-place change bumps a tensor's version), so the calls of one view --
        pts2plane, then render_image_hashtable_topk -- read them once."""
        fields = (self.fx, self.fy, self.cx, self.cy, self.width, self.height)
        versions = tuple(f._version if isinstance(f, torch.Tensor) else None for f in fields)
        hit = self.__dict__.get("_host_cache")
        if hit is not None and all(a is b for a, b in zip(hit[0], fields)) and hit[1] == versions:
            return hit[2]
        vals = tuple(_host_values(*fields))
        if any(isinstance(f, torch.Tensor) for f in fields):
            self.__dict__["_host_cache"] = (fields, versions, vals)
        return vals

    def _to_cpp(self):
        spec = _C.CameraSpec()
        spec.c2w = self.c2w
        spec.w2c = self.w2c
        spec.fx, spec.fy, spec.cx, spec.cy, spec.width, spec.height = self._host()
        return spec

    @staticmethod
    def decomposeK(K: torch.Tensor):
        """(fx, fy, cx, cy) as 0-d tensors, like the reference."""
        return K[0, 0], K[1, 1], K[0, 2], K[1, 2]

    def _save2torch(self, filename):
        torch.save({"c2w": self.c2w, "w2c": self.w2c,
                    **{k: torch.as_tensor(_scalar(getattr(self, k))) for k in
                       ("fx", "fy", "cx", "cy", "width", "height")}}, filename)

    def pixelidx2hwidx(self, pixelidx):
        return pixelidx // self.width, pixelidx % self.width

    def hwidx2pixelidx(self, h_idx, w_idx):
        return h_idx * self.width + w_idx


@dataclass
class RenderOptions:
    kernel_size: int = 5
    t_intvl: float = 0.01
    radius_threshold: float = 0.016
    sigma_threshold: float = 1e-4
    background_brightness: float = 1.0
    stop_threshold: float = 0.001
    num_sample_points_per_ray: int = 16
    num_point_cloud_per_sp: int = 4
    num_point_per_ray: int = 256
    sdf2weight_gaussian_alpha: float = 0.2
    sdf2weight_gaussian_gamma: float = 0.9
    sparsity_loss_w: float = 5e-4
    topK: int = 8

    _CPP_FIELDS = ("kernel_size", "t_intvl", "radius_threshold", "sigma_threshold", "background_brightness",
                   "stop_threshold", "num_sample_points_per_ray", "num_point_cloud_per_sp", "num_point_per_ray",
                   "sdf2weight_gaussian_alpha", "sdf2weight_gaussian_gamma", "topK")

    def _to_cpp(self):
        opt = _C.RenderOptions()
        for f in self._CPP_FIELDS:
            setattr(opt, f, getattr(self, f))
        return opt

    def _save2torch(self, filename):
        torch.save({f: torch.as_tensor(getattr(self, f)) for f in self._CPP_FIELDS}, filename)


@dataclass
class NeuralPointsGrads:
    grad_sigma: torch.Tensor
    grad_sh: torch.Tensor
    mask_out: torch.Tensor

    def _to_cpp(self):
        grads = _C.NeuralPointsGrads()
        grads.grad_sigma_out = self.grad_sigma
        grads.grad_sh_out = self.grad_sh
        grads.mask_out = self.mask_out
        return grads


def _read_ply_xyz_rgb(path):
    """Vertices (and colours, if present) of a PLY file: float64 [N,3], float64 [N,3] in [0,1] or None.

    Stands in for open3d.io.read_point_cloud, which the reference uses for
    pc_type='gt_pc' (epcq.py:182) and which is not required here.
    """
    import numpy as np
    with open(path, "rb") as f:
        header = []
        while True:
            line = f.readline().decode("ascii", errors="replace").strip()
            header.append(line)
            if line == "end_header":
                break
        body = f.read()
    fmt = [h.split()[1] for h in header if h.startswith("format")][0]
    n = 0
    props = []
    in_vertex = False
    for h in header:
        t = h.split()
        if t[:2] == ["element", "vertex"]:
            n, in_vertex = int(t[2]), True
        elif t and t[0] == "element":
            in_vertex = False
        elif in_vertex and t and t[0] == "property":
            props.append((t[2], t[1]))
    tmap = {"float": "f4", "float32": "f4", "double": "f8", "float64": "f8", "uchar": "u1", "uint8": "u1",
            "char": "i1", "int8": "i1", "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
            "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4"}
    if fmt == "ascii":
        rows = np.array(body.decode("ascii").split(), dtype=np.float64)[: n * len(props)].reshape(n, len(props))
        cols = {name: rows[:, i] for i, (name, _) in enumerate(props)}
    else:
        endian = "<" if fmt == "binary_little_endian" else ">"
        dt = np.dtype([(name, endian + tmap[typ]) for name, typ in props])
        arr = np.frombuffer(body, dtype=dt, count=n)
        cols = {name: arr[name].astype(np.float64) for name, _ in props}
    xyz = np.stack([cols["x"], cols["y"], cols["z"]], 1)
    rgb = None
    if all(c in cols for c in ("red", "green", "blue")):
        rgb = np.stack([cols["red"], cols["green"], cols["blue"]], 1)
        if dict(props)["red"] in ("uchar", "uint8"):
            rgb = rgb / 255.0
    return xyz, rgb


class NeuralPoints(nn.Module):
    def __init__(self,
                 basis_dim: int = 9,
                 device: Union[torch.device, str] = "cuda:0",
                 pc_type: str = "pointnerf",
                 gt_pc_path: str = None,
                 pointnerf_path: str = "pointnerf_ckpt/nerf_synthesis/lego.pth",
                 alpha: float = 5.0,
                 points=None):
        super().__init__()
        assert pc_type in ["pointnerf", "gt_pc", "pc"]
        self.pc_type = pc_type
        if pc_type == "pointnerf":
            if not str(pointnerf_path).endswith(".pth"):
                raise ValueError("Unsupported pointnerf_path: {}".format(pointnerf_path))
            ckpt = torch.load(pointnerf_path)
            self.xyz_data = nn.Parameter(ckpt["neural_points.xyz"], requires_grad=False)
            self.rgb_data = nn.Parameter(ckpt["neural_points.points_color"].squeeze(0), requires_grad=True)
            self.dir_data = nn.Parameter(ckpt["neural_points.points_dir"].squeeze(0), requires_grad=True)
            self.density_data = nn.Parameter(ckpt["neural_points.points_conf"].squeeze(0), requires_grad=True)
            self.feat_data = nn.Parameter(ckpt["neural_points.points_embeding"].squeeze(0), requires_grad=True)
            self.capacity = self.xyz_data.shape[0]
        elif pc_type == "gt_pc":
            if gt_pc_path is None:
                raise ValueError("gt_pc_path is required")
            xyz, rgb = _read_ply_xyz_rgb(gt_pc_path)
            self.xyz_data = nn.Parameter(torch.tensor(xyz, dtype=torch.float32, device=device), requires_grad=False)
            rgb_t = torch.zeros_like(self.xyz_data) if rgb is None else \
                torch.tensor(rgb, dtype=torch.float32, device=device)
            self.rgb_data = nn.Parameter(rgb_t, requires_grad=True)
            self.dir_data = nn.Parameter(torch.zeros_like(self.xyz_data), requires_grad=True)
            self.capacity = self.xyz_data.shape[0]
            self.basis_dim = basis_dim
            self.density_data = nn.Parameter(torch.zeros(self.capacity, 1, dtype=torch.float32, device=device),
                                             requires_grad=True)
            self.feat_data = nn.Parameter(torch.zeros(self.capacity, 32, dtype=torch.float32, device=device),
                                          requires_grad=True)
        else:
            assert points is not None
            self.xyz_data = nn.Parameter(points, requires_grad=False)
            self.rgb_data = nn.Parameter(torch.zeros_like(points), requires_grad=False)
            self.dir_data = nn.Parameter(torch.zeros_like(points), requires_grad=False)
            self.density_data = nn.Parameter(torch.zeros((points.shape[0], 1)), requires_grad=False)
            self.feat_data = nn.Parameter(torch.zeros_like(points), requires_grad=False)
            self.capacity = self.xyz_data.shape[0]
        self.multi_bins_rasterize = _C.scatter
        self.rasterize_hashtable = _C.scatter_hashtable
        self.quick_sampling = _C.quick_sampling

    def _load_ckpt(self, ckpt):
        """Restore a 'gt_pc' cloud from a checkpoint (a dict or a path to one) (epcq.py:223-233).

        The reference assigns 'sh_data' (and 'alpha_data') to attributes NeuralPoints never
        defines, so the call fails there.  Here 'sh_data' goes to feat_data, the tensor
        _save2torch stores under that key, so a saved cloud loads back; 'alpha_data' is kept
        as a plain attribute.  Other pc_types raise NotImplementedError, as in the reference."""
        if self.pc_type != "gt_pc":
            raise NotImplementedError
        if isinstance(ckpt, str):
            ckpt = torch.load(ckpt)
        self.density_data.data = ckpt["density_data"]
        self.feat_data.data = ckpt["sh_data"]
        self.xyz_data.data = ckpt["xyz_data"]
        self.capacity = self.xyz_data.shape[0]
        if "alpha_data" in ckpt:
            self.alpha_data = ckpt["alpha_data"]

    def _to_cpp(self):
        spec = _C.NeuralPointsSpec()
        spec.xyz_data = self.xyz_data.data
        return spec

    def _save2torch(self, filename):
        torch.save({"density_data": self.density_data.data, "sh_data": self.feat_data.data,
                    "xyz_data": self.xyz_data.data, "basis_dim": torch.tensor(9)}, filename)

    # -- torch helpers of the reference's projection, kept for callers that use
    #    them directly (pts2plane below does not: it runs in the CUDA library) --
    def _world2cam(self, cam: CameraSpec, pc_xyz: torch.Tensor = None):
        xyz = self.xyz_data if pc_xyz is None else pc_xyz
        pts_c = (cam.w2c[:3, :3] @ xyz.t() + cam.w2c[:3, 3:4]).t()
        return pts_c, pts_c[:, 2:3]

    def _cam2image(self, pts_c: torch.Tensor, cam: CameraSpec):
        scrn = cam.K @ pts_c.t()
        scrn = scrn / scrn[2:3, :]
        return scrn[0, :], scrn[1, :], scrn[0, :].to(torch.int32), scrn[1, :].to(torch.int32)

    def _convetpixel(self, screen_x, screen_y, hw):
        inside = (0 <= screen_x) & (screen_x < hw[1]) & (0 <= screen_y) & (screen_y < hw[0])
        return torch.where(inside, screen_x + screen_y * hw[1], torch.full_like(screen_x, hw[0] * hw[1]))

    def _uv2ray_index(self, uv, width):
        return (uv[:, 1] * width + uv[:, 0]).to(torch.int32)

    def pts2plane(self, cam: CameraSpec, opt: RenderOptions, pc_xyz: torch.Tensor = None, sort: bool = False):
        """Projection + per-pixel hash table (epcq.py:279-295), in one CUDA library call."""
        xyz = (self.xyz_data if pc_xyz is None else pc_xyz).detach()
        width, height = cam._host()[4:]
        return ops.pts2plane(xyz, cam.w2c, cam.K, height, width, sort)

    def render_image_hashtable_topk(self, cam: CameraSpec, opt: RenderOptions,
                                    sorted_point_idx_list: torch.Tensor,
                                    sorted_depth_list: torch.Tensor,
                                    hashtable: torch.Tensor,
                                    save_variables_for_debug: bool = False):
        """Window search + sampling + per-sample points (epcq.py:297-327)."""
        if save_variables_for_debug:
            out_dir = os.environ.get("EPCQ_DEBUG_DIR", ".")
            os.makedirs(out_dir, exist_ok=True)
            torch.save({"sorted_point_idx_list": sorted_point_idx_list}, os.path.join(out_dir, "sorted_point_idx_list.pt"))
            torch.save({"sorted_depth_list": sorted_depth_list}, os.path.join(out_dir, "sorted_depth_list.pt"))
            torch.save({"hashtable": hashtable}, os.path.join(out_dir, "hashtable.pt"))
            self._save2torch(os.path.join(out_dir, "epcq.pt"))
            cam._save2torch(os.path.join(out_dir, "cam.pt"))
            opt._save2torch(os.path.join(out_dir, "opt.pt"))
        return self.quick_sampling(self._to_cpp(), cam._to_cpp(), opt._to_cpp(), sorted_point_idx_list, hashtable)


class FeatureQuery(nn.Module):
    """Per-sample point attributes for the aggregator (epcq.py:328-387).

    forward gathers, for every sample whose mask is set, the xyz / rgb / dir /
    feat rows of its P point ids (zeros where the id is -1), its sample point
    and the direction of its pixel ray -- the same seven tensors as the
    reference, produced by one CUDA gather after a scan of the mask."""

    def generate_rays(self, cam: CameraSpec):
        """(rays_o, rays_d) [H, W, 3] through pixel corners, as the reference builds them (epcq.py:333-341)."""
        dev = cam.c2w.device
        fx, fy, cx, cy, W, H = cam._host()
        fx, fy, cx, cy, W, H = float(fx), float(fy), float(cx), float(cy), int(W), int(H)
        y, x = torch.meshgrid(torch.arange(H, dtype=torch.float32, device=dev),
                              torch.arange(W, dtype=torch.float32, device=dev), indexing="ij")
        d = torch.stack([(x - cx) / fx, (y - cy) / fy, torch.ones_like(x)], dim=-1)
        rays_d = torch.sum(d[:, :, None, :] * cam.c2w[:3, :3][None, None, :, :], dim=-1)
        rays_o = cam.c2w[:3, 3].expand_as(rays_d)
        return rays_o, rays_d

    def forward(self, neuralpoints, output_sp_xyz: torch.Tensor, output_pc_idx: torch.Tensor,
                mask_out: torch.Tensor, cam: CameraSpec, ray_index_uv: torch.Tensor = None):
        """-> (pc_xyz, pc_rgb, pc_dir, pc_feat, output_sp_xyz, valid_sp_mask_out, rays_d) for the M valid samples."""
        uv = ray_index_uv if ray_index_uv is not None and len(ray_index_uv) != 0 else None
        pc_idx = output_pc_idx if output_pc_idx.dtype == torch.int32 else output_pc_idx.to(torch.int32)
        feat = neuralpoints.feat_data.detach()
        fx, fy, cx, cy, width = cam._host()[:5]
        return ops.feature_query(neuralpoints.xyz_data.detach().contiguous(), neuralpoints.rgb_data.detach().contiguous(),
                                 neuralpoints.dir_data.detach().contiguous(), feat.contiguous(),
                                 output_sp_xyz.contiguous(), pc_idx.contiguous(), mask_out, cam.c2w,
                                 fx, fy, cx, cy, width, uv)


def positional_encoding(positions, freqs, ori=False):
    """sin / cos of every channel times 2^f, f < freqs (epcq.py:389-404): interleaved per argument
    ([sin a0, cos a0, sin a1, ...], argument c * freqs + f) or, with ori, [positions, all sines,
    all cosines]."""
    bands = 2.0 ** torch.arange(freqs, dtype=torch.float32, device=positions.device)
    args = (positions[..., None] * bands).flatten(-2)
    if ori:
        return torch.cat([positions, torch.sin(args), torch.cos(args)], dim=-1)
    return torch.stack([torch.sin(args), torch.cos(args)], dim=-1).flatten(-2)


class Aggregator(nn.Module):
    """The per-point MLP, alpha branch, inverse-distance aggregation and colour branch (epcq.py:406-507).

    Same layers, names, initialisation and forward signature as the reference's module, so its
    state_dict loads unchanged.  forward runs on the tensor cores: the weights are packed to bf16
    operand tiles once per parameter change, and two fused kernels compute the whole forward
    (bf16 operands, fp32 accumulation; outputs within about 1e-3 of the fp32 reference).  It is
    an inference path: with autograd recording and parameters that require grad it raises."""

    def __init__(self) -> None:
        super().__init__()

        def act():
            return nn.LeakyReLU(inplace=True)

        self.block1 = nn.Sequential(nn.Linear(284, 256), act(), nn.Linear(256, 256), act())
        self.block3 = nn.Sequential(nn.Linear(263, 256), act(), nn.Linear(256, 256), act())
        self.alpha_branch = nn.Sequential(nn.Linear(256, 1))
        self.alpha_act = nn.Softplus()
        self.color_branch = nn.Sequential(nn.Linear(280, 128), act(), nn.Linear(128, 128), act(),
                                          nn.Linear(128, 128), act(), nn.Linear(128, 3))
        self.color_act = nn.Sigmoid()
        for m in self.modules():
            if isinstance(m, nn.Linear):
                nn.init.xavier_uniform_(m.weight)
                nn.init.zeros_(m.bias)
        self.chunksize = 20000  # the reference's sample chunk; the fused kernels need none
        self._packed = None
        self._packed_key = None

    def calculate_weight(self, dist, mask=None):
        """Inverse-distance weights over the last axis, masked entries 0 (epcq.py:432-435)."""
        inv = 1 / (dist + 1e-6)
        if mask is not None:
            inv = inv * mask.float()
        return inv / (torch.sum(inv, dim=-1, keepdim=True) + 1e-6)

    def _linears(self):
        return [self.block1[0], self.block1[2], self.block3[0], self.block3[2], self.alpha_branch[0],
                self.color_branch[0], self.color_branch[2], self.color_branch[4], self.color_branch[6]]

    def packed_weights(self):
        """The bf16 operand tiles of the current parameters (re-packed when any of them changed)."""
        params = [t for m in self._linears() for t in (m.weight, m.bias)]
        key = tuple((t.data_ptr(), t._version, t.device) for t in params)
        if self._packed is None or self._packed_key != key:
            lin = self._linears()
            self._packed = ops.aggregator_pack([m.weight for m in lin], [m.bias for m in lin])
            self._packed_key = key
        return self._packed

    def forward(self, pc_xyz, pc_rgb, pc_dir, pc_feat, output_sp_xyz, valid_sp_mask_out, mask_out, rays_d):
        """-> (alphas, colors): [H*W, S] and [H*W, S, 3] for mask_out [H, W, S] (inference), [R, S]
        and [R, S, 3] for [R, S] (training layout); zeros where mask_out is not set."""
        if mask_out.dim() not in (2, 3):
            raise ValueError('mask_out shape error')
        if torch.is_grad_enabled() and any(p.requires_grad for p in self.parameters()):
            raise RuntimeError("Aggregator: the tensor-core forward has no backward; run it under torch.no_grad()")
        valid = valid_sp_mask_out if valid_sp_mask_out.dtype in (torch.bool, torch.uint8) else valid_sp_mask_out.bool()
        mask = mask_out if mask_out.dtype in (torch.bool, torch.uint8) else mask_out.bool()
        f32 = [t.detach().to(torch.float32).contiguous() for t in (pc_xyz, pc_rgb, pc_dir, pc_feat, output_sp_xyz,
                                                                    rays_d)]
        return ops.aggregator_forward(self.packed_weights(), f32[0], f32[1], f32[2], f32[3], f32[4],
                                      valid.contiguous(), mask.contiguous(), f32[5])


def clamp_t(t_val, vsize=0.004):
    """Sample spacings with out-of-range gaps set to vsize (epcq.py:508-515), on the GPU."""
    return ops.clamp_t(t_val.contiguous(), vsize)


def render(deltas, sigmas, rgbs, white_bg=False):
    """Front-to-back compositing of [R, S] samples into [R, 3] colours (epcq.py:517-529), on the GPU."""
    return ops.render(deltas.contiguous(), sigmas.contiguous(), rgbs.contiguous(), white_bg)
