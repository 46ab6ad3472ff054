"""Batched multi-view search+sample: one persistent sampling launch over many views.

The reference renders a view at a time: `pts2plane` then `quick_sampling`
(epcq/epcq.py:279-325), one kernel launch each.  `BatchRenderer` takes many
views at once -- different clouds, cameras, image sizes -- builds every view's
hash table (hp_pts2plane, spread over a few streams so small builds overlap)
and then runs hp_quick_sampling_batch: the tiles of all views in one queue,
heaviest first, served by one persistent kernel, so the tail of one view
overlaps the work of the others.  Each view's outputs are bit-identical to the
per-view launch.

The whole batch can be captured once as a CUDA graph and replayed (`capture`,
`replay`): buffers and the device view table are allocated up front and never
move, and no call in the batch synchronises with the host.

`Autotuner` picks the launch tuning of hp_quick_sampling_batch -- the stage
configuration of the sampling pipeline (items in flight per block, staged
points per item, blocks per SM; which items get split into row bands follows
from the staged capacity) and which rays a whole warp serves -- by timing the
candidates on the first batch of a shape class and caching the winner;
outputs never depend on the choice.
"""
import ctypes
import math
import threading

import numpy as np
import torch

from . import native, ops

_vp = ctypes.c_void_p


def _dev_tensor(a, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)


class _View:
    """Device camera tensors, build buffers and outputs of one view."""

    def __init__(self, cloud, n_points, cam, opt, device, sort):
        self.cloud = cloud
        self.H, self.W = int(cam.height), int(cam.width)
        self.fx, self.fy, self.cx, self.cy = float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy)
        self.c2w = _dev_tensor(cam.c2w, device)
        self.w2c = _dev_tensor(cam.w2c, device)
        self.K = _dev_tensor(cam.K, device)
        self.n = int(n_points)
        self.sort = int(bool(sort))
        L = native.lib()
        self.ws_bytes = L.hp_pts2plane_workspace_size(self.n, self.H, self.W)
        self.ws = torch.empty(max(self.ws_bytes, 1), dtype=torch.uint8, device=device)
        self.sidx = torch.empty(self.n, dtype=torch.int32, device=device)
        self.sdep = torch.empty(self.n, dtype=torch.float32, device=device)
        self.hash = torch.empty((self.H * self.W, 2), dtype=torch.int32, device=device)
        self.out = ops.sampling_outputs(self.H, self.W, opt, device)
        self.cam = ops.make_camera(c2w=self.c2w, w2c=self.w2c, K=self.K, fx=self.fx, fy=self.fy, cx=self.cx,
                                   cy=self.cy, width=self.W, height=self.H)

    @property
    def rays(self):
        return self.H * self.W


class BatchRenderer:
    """Search+sample for a fixed set of views over resident clouds.

    clouds: list of float32 [N_i, 3] tensors on `device` (kept resident).
    views:  list of (cloud index, camera) with camera.c2w/w2c/K and intrinsics
            (for example hashpoint.synth.PinholeCamera).
    options: RenderOptions-like (kernel_size, t_intvl, radius_threshold, ...).
    """

    def __init__(self, clouds, views, options, device="cuda", sort=False, build_streams=4):
        self.device = torch.device(device)
        self.clouds = [ops.check_input(c, "cloud", torch.float32) for c in clouds]
        self.options = options
        self.views = [_View(ci, self.clouds[ci].shape[0], cam, options, self.device, sort) for ci, cam in views]
        self.hp_views = [ops.make_view(self.clouds[v.cloud], v.c2w, v.fx, v.fy, v.cx, v.cy, v.W, v.H, options,
                                       v.sidx, v.hash, v.out) for v in self.views]
        n = len(self.hp_views)
        self.table = (native.HpView * n)(*self.hp_views)
        raw = bytes(memoryview(self.table).cast("B"))
        self.table_device = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device)
        self.ws_bytes = native.lib().hp_quick_sampling_batch_workspace_size(self.table, n)
        if self.ws_bytes == 0:
            raise RuntimeError("BatchRenderer: invalid views")
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, int(build_streams)))]
        self.tuning = ops.make_tuning()
        self.graph = None

    # -- work ---------------------------------------------------------------
    @property
    def rays(self):
        return sum(v.rays for v in self.views)

    def build(self):
        """hp_pts2plane for every view, round-robin over the build streams (joined back)."""
        main = torch.cuda.current_stream(self.device)
        L = native.lib()
        for s in self.streams:
            s.wait_stream(main)
        for i, v in enumerate(self.views):
            s = self.streams[i % len(self.streams)]
            xyz = self.clouds[v.cloud]
            rc = L.hp_pts2plane(_vp(xyz.data_ptr()), v.n, ctypes.byref(v.cam), v.sort, _vp(v.sidx.data_ptr()),
                                _vp(v.sdep.data_ptr()), _vp(v.hash.data_ptr()), _vp(v.ws.data_ptr()), v.ws_bytes,
                                _vp(s.cuda_stream))
            native.check(rc, "hp_pts2plane")
        for s in self.streams:
            main.wait_stream(s)

    def sample(self):
        """One hp_quick_sampling_batch over all views on the current stream."""
        L = native.lib()
        rc = L.hp_quick_sampling_batch(self.table, _vp(self.table_device.data_ptr()), len(self.hp_views),
                                       ctypes.byref(self.tuning), _vp(self.ws.data_ptr()), self.ws_bytes,
                                       _vp(torch.cuda.current_stream(self.device).cuda_stream))
        native.check(rc, "hp_quick_sampling_batch")

    def run(self):
        self.build()
        self.sample()

    def run_per_view(self):
        """The plain per-view launch over the same buffers, for comparison: hp_pts2plane then
        hp_quick_sampling, one view at a time on the current stream."""
        L = native.lib()
        st = _vp(torch.cuda.current_stream(self.device).cuda_stream)
        if getattr(self, "_pv_ws", None) is None:
            need = max(L.hp_quick_sampling_workspace_size(v.n, v.H, v.W) for v in self.views)
            self._pv_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
            self._pv_opt = ops.make_options(self.options)
        ws = self._pv_ws
        for v in self.views:
            xyz = self.clouds[v.cloud]
            rc = L.hp_pts2plane(_vp(xyz.data_ptr()), v.n, ctypes.byref(v.cam), v.sort, _vp(v.sidx.data_ptr()),
                                _vp(v.sdep.data_ptr()), _vp(v.hash.data_ptr()), _vp(v.ws.data_ptr()), v.ws_bytes, st)
            native.check(rc, "hp_pts2plane")
            sp_xyz, pc_idx, sp_t, mask = v.out
            rc = L.hp_quick_sampling(_vp(xyz.data_ptr()), v.n, ctypes.byref(v.cam), ctypes.byref(self._pv_opt),
                                     _vp(v.sidx.data_ptr()), v.n, _vp(v.hash.data_ptr()), _vp(sp_xyz.data_ptr()),
                                     _vp(pc_idx.data_ptr()), _vp(sp_t.data_ptr()), _vp(mask.data_ptr()),
                                     _vp(ws.data_ptr()), ws.numel(), st)
            native.check(rc, "hp_quick_sampling")

    # -- CUDA graph -----------------------------------------------------------
    def capture(self):
        """Capture build + sample as one CUDA graph (run once eagerly first to load the kernels)."""
        self.run()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def release(self):
        self.graph = None

    # -- results --------------------------------------------------------------
    def outputs(self, i):
        """(sp_xyz, pc_idx, sp_t, mask) of view i."""
        return self.views[i].out

    def hash_table(self, i):
        """(sorted_point_idx, sorted_depth, hash_table) of view i."""
        v = self.views[i]
        return v.sidx, v.sdep, v.hash


class Autotuner:
    """Per shape class, the fastest hp_quick_sampling_batch tuning (cached, thread-safe).

    A shape class is (views, log2 of the rays, log2 of the points, k, S, P).
    Candidates are timed with CUDA events on the renderer's own batch; the
    cache is filled once per class and then only read."""

    HEAVY = (224, 320)
    STAGES = native.STAGE_CONFIGS

    def __init__(self, reps=3):
        self.reps = int(reps)
        self.cache = {}
        self.lock = threading.Lock()

    def key(self, r):
        pts = sum(c.shape[0] for c in r.clouds)
        o = r.options
        return (len(r.views), int(math.log2(max(r.rays, 1))), int(math.log2(max(pts, 1))), int(o.kernel_size),
                int(o.num_sample_points_per_ray), int(o.num_point_cloud_per_sp))

    def _time(self, r):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        r.sample()  # warm
        best = float("inf")
        for _ in range(self.reps):
            ev[0].record()
            r.sample()
            ev[1].record()
            ev[1].synchronize()
            best = min(best, ev[0].elapsed_time(ev[1]))
        return best

    def tune(self, r):
        """Set r.tuning to the cached or newly measured best; returns (stage_config, heavy_window)."""
        k = self.key(r)
        with self.lock:
            hit = self.cache.get(k)
        if hit is None:
            r.build()
            results = []
            for c in self.STAGES:
                for h in self.HEAVY:
                    r.tuning = ops.make_tuning(heavy_window=h, stage_config=c)
                    results.append((self._time(r), c, h))
            _, c, h = min(results)
            with self.lock:
                hit = self.cache.setdefault(k, (c, h))
        r.tuning = ops.make_tuning(heavy_window=hit[1], stage_config=hit[0])
        return hit
