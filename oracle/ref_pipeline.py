"""The reference's Python-side steps of the search+sample path, restated over
torch, driving the reference's own CUDA extension (oracle/_ref, built by
oracle/build_ref.py).  Test and baseline infrastructure only: the golden
fixtures, the live-reference parity tests and bench.py's reference-GPU leg
use it; nothing in the product path does.

  project            epcq/epcq.py:251-274  (torch matmuls, divide, int32 cast, where)
  sort               epcq/epcq.py:283-286  (torch.sort by pixel id, gathers)
  scatter_hashtable  _C.scatter_hashtable  (epcq/csrc/rasterization.cu:130-171)
  quick_sampling     _C.quick_sampling     (epcq/csrc/epcq_render_topk.cu:341-417)
  scatter            _C.scatter            (rasterization.cu:88-128)

The reference's bucket walk reads point2img[N] (rasterization.cu:23), one past
the sorted ids; scatter_hashtable and scatter hand it a view of a buffer with
one extra sentinel element, so that read stays in bounds and stops the walk.
"""
import torch

OPT_FIELDS = ["kernel_size", "t_intvl", "radius_threshold", "sigma_threshold", "background_brightness",
              "stop_threshold", "num_sample_points_per_ray", "num_point_cloud_per_sp", "num_point_per_ray",
              "sdf2weight_gaussian_alpha", "sdf2weight_gaussian_gamma", "topK"]


class RefPipeline:
    """The reference's per-view steps over torch tensors, feeding the reference _C module `mod`."""

    def __init__(self, mod, dev):
        self.C = mod
        self.dev = dev

    def camera_spec(self, c2w, w2c, cam):
        s = self.C.CameraSpec()
        s.c2w, s.w2c = c2w, w2c
        s.fx, s.fy, s.cx, s.cy = cam.fx, cam.fy, cam.cx, cam.cy
        s.width, s.height = cam.width, cam.height
        return s

    def options_spec(self, opt):
        o = self.C.RenderOptions()
        for f in OPT_FIELDS:
            setattr(o, f, getattr(opt, f))
        return o

    def project(self, xyz, w2c, K, H, W):
        pts_c = (w2c[:3, :3] @ xyz.t() + w2c[:3, 3:4]).t()
        depth = pts_c[:, 2:3]
        scrn = K @ pts_c.t()
        scrn = scrn / scrn[2:3, :]
        sx, sy = scrn[0, :], scrn[1, :]
        sxi, syi = sx.to(torch.int32), sy.to(torch.int32)
        pid = sxi + syi * W
        inb = (0 <= sxi) & (sxi < W) & (0 <= syi) & (syi < H)
        pid = torch.where(inb, pid, torch.full_like(pid, H * W))
        return pid, depth.squeeze(1), sx, sy, pts_c

    def sort(self, pid, depth):
        n = pid.shape[0]
        point_idx = torch.arange(n, dtype=torch.int32, device=pid.device)
        pid_s, perm = torch.sort(pid.squeeze(), dim=-1, descending=False)
        return pid_s, perm, depth[perm], point_idx[perm]

    @staticmethod
    def _sentinel(pid_s):
        n = pid_s.shape[0]
        pad = torch.empty(n + 1, dtype=torch.int32, device=pid_s.device)
        pad[:n] = pid_s
        pad[n] = -7  # stops the bucket walk at index n
        return pad[:n]

    def scatter_hashtable(self, idx_s, pid_s, depth_s, H, W, sort):
        return self.C.scatter_hashtable(idx_s, self._sentinel(pid_s), depth_s, [H, W], sort)

    def scatter(self, idx_s, pid_s, depth_s, H, W, bins):
        assert bool((depth_s[pid_s < H * W] >= 0).all())
        return self.C.scatter(idx_s, self._sentinel(pid_s), depth_s, [H, W], bins)

    def pts2plane(self, xyz, w2c, K, H, W, sort=False):
        """NeuralPoints.pts2plane (epcq.py:279-295): (sorted_point_idx, sorted_depth, hash_table)."""
        pid, depth, _, _, _ = self.project(xyz, w2c, K, H, W)
        pid_s, _, depth_s, idx_s = self.sort(pid, depth)
        return self.scatter_hashtable(idx_s, pid_s, depth_s, H, W, sort)

    def render(self, xyz, c2w, w2c, K, cam, opt, sort=False):
        """pts2plane then render_image_hashtable_topk's _C.quick_sampling (epcq.py:279-325):
        (sp_xyz, pc_idx, sp_t, mask)."""
        sidx, _, hsh = self.pts2plane(xyz, w2c, K, cam.height, cam.width, sort)
        spec = self.C.NeuralPointsSpec()
        spec.xyz_data = xyz
        return self.C.quick_sampling(spec, self.camera_spec(c2w, w2c, cam), self.options_spec(opt), sidx, hsh)
