"""Per-view pipeline over preallocated device buffers (the plain per-view launch).

A ViewPipeline owns the workspace and the output buffers for one problem shape
(point count, image size, options) and renders a view with two C-ABI calls:
hp_pts2plane (projection + hash table) and hp_quick_sampling (search + sample +
per-sample points).  Camera matrices are read from device memory, so many
views can be described by a device-resident camera table and launched
back-to-back without host synchronisation.
"""
import ctypes

import torch

from . import native
from .ops import make_options, make_tuning

_vp = ctypes.c_void_p


class CameraTable:
    """Device-resident cameras: c2w/w2c [V,4,4], K [V,3,3] float32, plus host intrinsics."""

    def __init__(self, cams, device):
        import numpy as np
        self.n = len(cams)
        self.c2w = torch.from_numpy(np.stack([c.c2w for c in cams]).astype(np.float32)).to(device).contiguous()
        self.w2c = torch.from_numpy(np.stack([c.w2c for c in cams]).astype(np.float32)).to(device).contiguous()
        self.K = torch.from_numpy(np.stack([c.K for c in cams]).astype(np.float32)).to(device).contiguous()
        self.intr = [(c.fx, c.fy, c.cx, c.cy, c.width, c.height) for c in cams]

    def struct(self, i):
        fx, fy, cx, cy, W, H = self.intr[i]
        cam = native.HpCamera()
        cam.c2w = self.c2w.data_ptr() + i * 64
        cam.w2c = self.w2c.data_ptr() + i * 64
        cam.K = self.K.data_ptr() + i * 36
        cam.fx, cam.fy, cam.cx, cam.cy = fx, fy, cx, cy
        cam.width, cam.height = W, H
        return cam


class ViewPipeline:
    """pts2plane + quick_sampling for a fixed (N, H, W, S, P), buffers allocated once."""

    def __init__(self, n_points, height, width, options, device, sort=False, tuning=None):
        self.n, self.H, self.W = int(n_points), int(height), int(width)
        self.tuning = tuning  # HpTuning of the sampling launch (None = defaults)
        self.opt = make_options(options)
        self.sort = int(bool(sort))
        self.device = torch.device(device)
        S, P = self.opt.num_sample_points_per_ray, self.opt.num_point_cloud_per_sp
        L = native.lib()
        self.ws_bytes = L.hp_pts2plane_workspace_size(self.n, self.H, self.W)
        dev = self.device
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=dev)
        self.sidx = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.sdep = torch.empty(self.n, dtype=torch.float32, device=dev)
        self.hash = torch.empty((self.H * self.W, 2), dtype=torch.int32, device=dev)
        self.sp_xyz = torch.empty((self.H, self.W, S, 3), dtype=torch.float32, device=dev)
        self.pc_idx = torch.empty((self.H, self.W, S, P), dtype=torch.int32, device=dev)
        self.sp_t = torch.empty((self.H, self.W, S), dtype=torch.float32, device=dev)
        self.mask = torch.empty((self.H, self.W, S), dtype=torch.bool, device=dev)
        self.ws_sample_bytes = L.hp_quick_sampling_workspace_size(self.n, self.H, self.W)
        self.ws_sample = torch.empty(self.ws_sample_bytes, dtype=torch.uint8, device=dev)

    def build(self, xyz, cam, stream):
        rc = native.lib().hp_pts2plane(_vp(xyz.data_ptr()), self.n, ctypes.byref(cam), self.sort,
                                       _vp(self.sidx.data_ptr()), _vp(self.sdep.data_ptr()),
                                       _vp(self.hash.data_ptr()), _vp(self.ws.data_ptr()), self.ws_bytes,
                                       _vp(stream.cuda_stream))
        native.check(rc, "hp_pts2plane")

    def sample(self, xyz, cam, stream):
        rc = native.lib().hp_quick_sampling_tuned(
            _vp(xyz.data_ptr()), self.n, ctypes.byref(cam), ctypes.byref(self.opt), _vp(self.sidx.data_ptr()), self.n,
            _vp(self.hash.data_ptr()), _vp(self.sp_xyz.data_ptr()), _vp(self.pc_idx.data_ptr()),
            _vp(self.sp_t.data_ptr()), _vp(self.mask.data_ptr()),
            ctypes.byref(self.tuning) if self.tuning is not None else None, _vp(self.ws_sample.data_ptr()),
            self.ws_sample_bytes, _vp(stream.cuda_stream))
        native.check(rc, "hp_quick_sampling")

    def tune(self, xyz, cams, stream=None, reps=2):
        """Pick the fastest stage configuration of the sampling kernel (hp_tuning.stage_config) for
        this shape on the given views, timed with CUDA events; outputs never depend on it.  Returns
        the configuration, which later sample() calls use."""
        import torch
        stream = stream or torch.cuda.current_stream(self.device)
        best = None
        for cfg in native.STAGE_CONFIGS:
            self.tuning = make_tuning(stage_config=cfg)
            ms = []
            for rep in range(reps + 1):
                tot = 0.0
                for cam in cams:
                    self.build(xyz, cam, stream)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    self.sample(xyz, cam, stream)
                    e1.record(stream)
                    e1.synchronize()
                    tot += e0.elapsed_time(e1)
                if rep:  # the first pass loads and warms the configuration's kernels
                    ms.append(tot)
            if best is None or min(ms) < best[0]:
                best = (min(ms), cfg)
        self.tuning = make_tuning(stage_config=best[1])
        return best[1]

    def render(self, xyz, cam, stream=None):
        stream = stream or torch.cuda.current_stream(self.device)
        self.build(xyz, cam, stream)
        self.sample(xyz, cam, stream)
        return self.sp_xyz, self.pc_idx, self.sp_t, self.mask

    # kernels each render() launches (hp_pts2plane: project/count, scan,
    # scatter, order, huge-bucket sort; hp_quick_sampling: tile work with the
    # packing, tile order, sampling)
    KERNELS_PER_VIEW = 8


class ViewRing:
    """Many views of one shape through per-view launches, pipelined over `depth` streams.

    View i runs on pipeline i % depth (its own buffers) and that pipeline's stream, so view i+1's
    hash-table build and tile scheduling run while view i's persistent sampling kernel drains its
    last work items, and its sampling kernel's blocks start as view i's retire.  Every view is
    still hp_pts2plane + hp_quick_sampling, each with the outputs the plain launch gives.  A
    view's outputs stay in its pipeline's buffers until view i + depth reuses them on the same
    stream: `on_view(i, pipe, stream)` is called right after view i is enqueued, so work it
    enqueues on `stream` reads them before they are overwritten."""

    def __init__(self, n_points, height, width, options, device, depth=3, sort=False, tuning=None):
        self.device = torch.device(device)
        self.pipes = [ViewPipeline(n_points, height, width, options, device, sort, tuning) for _ in range(depth)]
        self.streams = [torch.cuda.Stream(self.device) for _ in range(depth)]

    @property
    def depth(self):
        return len(self.pipes)

    def set_tuning(self, tuning):
        for p in self.pipes:
            p.tuning = tuning

    def tune(self, xyz, cams, stream=None, reps=2):
        """Pick the stage configuration of the sampling kernel for this shape by timing
        render_many over `cams` in each (CUDA events on `stream`): with launches overlapping
        across streams, the fastest configuration can differ from the one-stream choice
        (ViewPipeline.tune).  Outputs never depend on it."""
        main = stream or torch.cuda.current_stream(self.device)
        best = None
        for cfg in native.STAGE_CONFIGS:
            self.set_tuning(make_tuning(stage_config=cfg))
            ms = []
            for rep in range(reps + 1):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(main)
                self.render_many(xyz, cams, main)
                e1.record(main)
                e1.synchronize()
                if rep:  # the first pass loads and warms the configuration's kernels
                    ms.append(e0.elapsed_time(e1))
            if best is None or min(ms) < best[0]:
                best = (min(ms), cfg)
        self.set_tuning(make_tuning(stage_config=best[1]))
        return best[1]

    def render_many(self, xyz, cams, stream=None, on_view=None):
        """Render `cams` (HpCamera structs); the views' work starts after, and `stream` waits for,
        everything enqueued on `stream` before the call."""
        main = stream or torch.cuda.current_stream(self.device)
        start = torch.cuda.Event()
        start.record(main)
        for s in self.streams:
            s.wait_event(start)
        for i, cam in enumerate(cams):
            k = i % self.depth
            p, s = self.pipes[k], self.streams[k]
            p.build(xyz, cam, s)
            p.sample(xyz, cam, s)
            if on_view is not None:
                on_view(i, p, s)
        for s in self.streams:
            done = torch.cuda.Event()
            done.record(s)
            main.wait_event(done)
