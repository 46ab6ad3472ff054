"""Serving: a request loop over resident scenes with continuous batching.

Scenes (point clouds) stay on the device, and so do their hash tables, cached
per (scene, camera pose, resolution).  Render requests -- (scene, pose,
resolution) -- arrive over time.  The loop

  * admits waiting requests in arrival order while the HBM budget allows
    (resident scenes + cached hash tables + outputs of every admitted request);
    a request that can never fit is rejected;
  * packs the admitted requests into a batch and launches it on a free stream:
    hash-table builds for cache misses (hp_pts2plane) and one
    hp_quick_sampling_batch over all of the batch's views;
  * keeps up to `streams` batches in flight, so requests that arrive while
    others are on the GPU are admitted as soon as a slot and memory free up,
    and their work overlaps the running batches on the device;
  * retires finished batches (their outputs are handed to a callback, then
    freed) and records each request's latency from its arrival to its
    batch's completion on the GPU.

The host work per batch is kept small and free of allocation: output buffers
come from a pool per resolution, each in-flight slot owns a sampling and a
build workspace that only grow, and every cached hash table carries its
hp_view template (only the output pointers are filled in per request).  A
Server is meant to live across runs: its pool and workspaces are filled by the
first requests and reused afterwards (a device allocation inside the loop --
hundreds of MB of outputs for a 1600 x 1200 view -- stalls it for tens of ms).  The loop spins on its events and
the next arrival for the last stretch before either is due instead of
sleeping through it, so a request is noticed within microseconds.

Each request's outputs are exactly those of a plain per-view launch: the batch
runs the same per-ray code, and a hash table is the same whether built for the
request or found in the cache.
"""
import collections
import gc
import ctypes
import time

import numpy as np
import torch

from . import native, ops, synth

_vp = ctypes.c_void_p


class Request:
    __slots__ = ("rid", "scene", "pose", "width", "height", "arrival", "done_ms", "outputs", "status", "reserved")

    def __init__(self, rid, scene, pose, width, height, arrival):
        self.rid, self.scene, self.pose = int(rid), int(scene), int(pose)
        self.width, self.height = int(width), int(height)
        self.arrival = float(arrival)  # seconds after the start of the run
        self.done_ms = None            # completion, ms after the start of the run (GPU clock)
        self.outputs = None
        self.status = "waiting"
        self.reserved = False  # holds a cached table since admission

    @property
    def rays(self):
        return self.width * self.height


def camera_for(pose_c2w, width, height, f_at_800=1111.0):
    """Pinhole camera with the pose of `pose_c2w` at a resolution (f scaled with the width)."""
    f = f_at_800 * width / 800.0
    K = np.array([[f, 0, width / 2], [0, f, height / 2], [0, 0, 1]], np.float32)
    c2w = np.asarray(pose_c2w, np.float32)
    w2c = np.linalg.inv(c2w.astype(np.float64)).astype(np.float32)
    return synth.PinholeCamera(c2w, w2c, K, int(width), int(height))


class _Entry:
    """A cached hash table: (scene, pose, width, height) -> sorted ids, depths, table, and the
    hp_view of a request for it (output pointers left to fill)."""

    def __init__(self, n, H, W, device):
        # one allocation, three 256-byte aligned views (a miss costs one device allocation, not three)
        nb = (4 * n + 255) // 256 * 256
        buf = torch.empty(2 * nb + 8 * H * W, dtype=torch.uint8, device=device)
        self.sidx = buf[:4 * n].view(torch.int32)
        self.sdep = buf[nb:nb + 4 * n].view(torch.float32)
        self.hash = buf[2 * nb:].view(torch.int32).view(H * W, 2)
        self.ready = None  # event recorded after the build
        self.bytes = 8 * n + 8 * H * W
        self.users = 0     # in-flight batches that read it
        self.view = None   # native.HpView template


class SceneStore:
    """Resident scenes, their camera poses and the hash-table cache."""

    def __init__(self, clouds, poses, options, device="cuda"):
        self.device = torch.device(device)
        self.clouds = [ops.check_input(c, "cloud", torch.float32) for c in clouds]
        self.poses = poses  # poses[scene] = list of 4x4 c2w
        self.options = options
        self.cache = collections.OrderedDict()
        self.cams = {}
        self.scene_bytes = sum(12 * c.shape[0] for c in self.clouds)
        self.bytes = self.scene_bytes  # scenes + cached tables
        self.hits = 0    # lookups served from the cache
        self.misses = 0  # lookups that built a table

    def camera(self, scene, pose, width, height):
        key = (scene, pose, width, height)
        c = self.cams.get(key)
        if c is None:
            cam = camera_for(self.poses[scene][pose], width, height)
            c = (cam, torch.from_numpy(cam.c2w).to(self.device), torch.from_numpy(cam.w2c).to(self.device),
                 torch.from_numpy(cam.K).to(self.device))
            self.cams[key] = c
        return c

    def entry_bytes(self, req):
        key = (req.scene, req.pose, req.width, req.height)
        if key in self.cache:
            return 0
        return 8 * self.clouds[req.scene].shape[0] + 8 * req.rays

    def evict(self, need, budget, other_bytes):
        """Drop least recently used tables no batch is reading until `need` more bytes fit; True if they do."""
        for key in list(self.cache.keys()):
            if self.bytes + other_bytes + need <= budget:
                break
            e = self.cache[key]
            if e.users == 0:
                del self.cache[key]
                self.bytes -= e.bytes
        return self.bytes + other_bytes + need <= budget

    def reserve(self, req):
        """At admission: pin the request's cached table (if any) so eviction leaves it."""
        e = self.cache.get((req.scene, req.pose, req.width, req.height))
        if e is None:
            return False
        e.users += 1
        return True

    def lookup(self, req, stream, build_ws):
        """The request's hash table, pinned for its batch; built on `stream` on a miss (other streams
        wait on its event)."""
        key = (req.scene, req.pose, req.width, req.height)
        e = self.cache.get(key)
        if e is not None:
            self.hits += 1
            self.cache.move_to_end(key)
            if not req.reserved:
                e.users += 1
            if e.ready is not None:
                stream.wait_event(e.ready)
            return e
        self.misses += 1
        xyz = self.clouds[req.scene]
        n = xyz.shape[0]
        cam, c2w, w2c, K = self.camera(req.scene, req.pose, req.width, req.height)
        e = _Entry(n, req.height, req.width, self.device)
        hc = ops.make_camera(c2w=c2w, w2c=w2c, K=K, fx=cam.fx, fy=cam.fy, cx=cam.cx, cy=cam.cy, width=req.width,
                             height=req.height)
        L = native.lib()
        need = L.hp_pts2plane_workspace_size(n, req.height, req.width)
        ws = build_ws(need)
        rc = L.hp_pts2plane(_vp(xyz.data_ptr()), n, ctypes.byref(hc), 0, _vp(e.sidx.data_ptr()),
                            _vp(e.sdep.data_ptr()), _vp(e.hash.data_ptr()), _vp(ws.data_ptr()), need,
                            _vp(stream.cuda_stream))
        native.check(rc, "hp_pts2plane")
        e.ready = torch.cuda.Event()
        e.ready.record(stream)
        e.users = 1
        e.view = ops.make_view(xyz, c2w, cam.fx, cam.fy, cam.cx, cam.cy, req.width, req.height, self.options, e.sidx,
                               e.hash, (None, None, None, None))
        self.cache[key] = e
        self.bytes += e.bytes
        return e


def output_bytes(req, opt):
    S, P = int(opt.num_sample_points_per_ray), int(opt.num_point_cloud_per_sp)
    return req.rays * S * (12 + 4 + 1 + 4 * P)


class _Batch:
    def __init__(self, reqs, slot, stream, done, hold):
        self.reqs, self.slot, self.stream, self.done, self.hold = reqs, slot, stream, done, hold


class OutputPool:
    """Reusable quick_sampling output buffers per resolution (sp_xyz, pc_idx, sp_t, mask)."""

    def __init__(self, options, device):
        self.options, self.device = options, device
        self.free = collections.defaultdict(list)

    def take(self, width, height):
        lst = self.free[(width, height)]
        return lst.pop() if lst else ops.sampling_outputs(height, width, self.options, self.device)

    def give(self, width, height, out):
        self.free[(width, height)].append(out)


class Server:
    """Continuous-batching request loop (see the module docstring).

    budget_bytes: HBM the loop may use for scenes, cached tables and outputs.
    streams: batches in flight at once; max_views: requests per batch.
    on_result(request): called with each finished request (outputs attached)
    before its outputs are released."""

    def __init__(self, store, budget_bytes, streams=3, max_views=16, on_result=None, tuning=None):
        self.store = store
        self.budget = int(budget_bytes)
        self.max_views = int(max_views)
        self.on_result = on_result
        self.device = store.device
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, int(streams)))]
        self.free_slots = list(range(len(self.streams)))
        self.tuning = tuning if tuning is not None else ops.make_tuning()
        self.out_bytes = 0
        self.batches = 0
        self.pool = OutputPool(store.options, self.device)
        self.ws = [None] * len(self.streams)        # sampling workspace per slot (grows, never shrinks)
        self.build_ws = [None] * len(self.streams)  # hash-table build workspace per slot (likewise)
        self.tables = [(native.HpView * self.max_views)() for _ in self.streams]

    def _build_ws(self, slot, nbytes):
        ws = self.build_ws[slot]
        if ws is None or ws.numel() < nbytes:
            ws = self.build_ws[slot] = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return ws

    def tune(self, requests, tuner=None):
        """Pick the batch launch tuning (stage configuration, heavy-ray threshold) on a sample of
        requests, as a service would once at start-up: hashpoint.batch.Autotuner over one batch of
        their views.  Returns (stage_config, heavy_window); outputs never depend on it."""
        from . import batch
        views = []
        for r in requests[: self.max_views]:
            cam, _, _, _ = self.store.camera(r.scene, r.pose, r.width, r.height)
            views.append((r.scene, cam))
        renderer = batch.BatchRenderer(self.store.clouds, views, self.store.options, self.device)
        choice = (tuner or batch.Autotuner(reps=1)).tune(renderer)
        self.tuning = renderer.tuning
        del renderer
        torch.cuda.empty_cache()
        return choice

    def _bytes_needed(self, req):
        return output_bytes(req, self.store.options) + self.store.entry_bytes(req)

    def _launch(self, reqs, slot, t0_event):
        # heavy views first: the batch takes its views' tiles in table order
        reqs = sorted(reqs, key=lambda r: -self.store.clouds[r.scene].shape[0])
        s = self.streams[slot]
        hold = []  # cached tables the batch reads
        table = self.tables[slot]
        n = len(reqs)
        with torch.cuda.stream(s):
            for i, r in enumerate(reqs):
                e = self.store.lookup(r, s, lambda b: self._build_ws(slot, b))
                out = self.pool.take(r.width, r.height)
                r.outputs = out
                table[i] = e.view
                v = table[i]  # shares the table's memory
                v.sp_xyz, v.pc_idx, v.sp_t, v.mask = (out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                                                      out[3].data_ptr())
                hold.append(e)
                r.status = "running"
            L = native.lib()
            ws_bytes = L.hp_quick_sampling_batch_workspace_size(table, n)
            ws = self.ws[slot]
            if ws is None or ws.numel() < ws_bytes:
                ws = self.ws[slot] = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
            rc = L.hp_quick_sampling_batch(table, None, n, ctypes.byref(self.tuning), _vp(ws.data_ptr()), ws.numel(),
                                           _vp(s.cuda_stream))
            native.check(rc, "hp_quick_sampling_batch")
            done = torch.cuda.Event(enable_timing=True)
            done.record(s)
        self.batches += 1
        return _Batch(reqs, slot, s, done, hold)

    def _retire(self, b, t0_event):
        done_ms = t0_event.elapsed_time(b.done)
        for h in b.hold:
            if isinstance(h, _Entry):
                h.users -= 1
        for r in b.reqs:
            r.done_ms = done_ms
            r.status = "done"
            if self.on_result is not None:
                self.on_result(r)
            self.out_bytes -= output_bytes(r, self.store.options)
            self.pool.give(r.width, r.height, r.outputs)
            r.outputs = None
        self.free_slots.append(b.slot)

    def run(self, requests, poll_s=200e-6, time_limit_s=600.0):
        """Serve `requests` (arrival times relative to the start) in real time; returns stats.
        Python's cyclic garbage collector is paused while the loop runs (a collection pass
        stalls the launch loop for milliseconds) and restored afterwards.  The loop sleeps
        only while the next arrival is more than poll_s away and nothing can be launched;
        otherwise it spins."""
        gc_was = gc.isenabled()
        gc.disable()
        try:
            return self._run(requests, poll_s, time_limit_s)
        finally:
            if gc_was:
                gc.enable()

    def _run(self, requests, poll_s, time_limit_s):
        hits0, misses0, batches0 = self.store.hits, self.store.misses, self.batches
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        inflight = []
        rejected = []
        torch.cuda.synchronize(self.device)
        t0_event = torch.cuda.Event(enable_timing=True)
        t0_event.record(torch.cuda.current_stream(self.device))
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        while pending or waiting or inflight:
            now = time.perf_counter() - t0
            if now > time_limit_s:
                raise RuntimeError("serve: time limit exceeded")
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            still = []
            for b in inflight:
                if b.done.query():
                    self._retire(b, t0_event)
                else:
                    still.append(b)
            inflight = still
            if waiting and self.free_slots:
                batch, pending_bytes = [], 0  # new tables and outputs of this batch
                while waiting and len(batch) < self.max_views:
                    r = waiting[0]
                    need = self._bytes_needed(r)
                    if self.store.scene_bytes + need > self.budget:  # can never fit
                        waiting.popleft()
                        r.status = "rejected"
                        rejected.append(r)
                        continue
                    if not self.store.evict(need, self.budget, self.out_bytes + pending_bytes):
                        break
                    r.reserved = self.store.reserve(r)
                    waiting.popleft()
                    batch.append(r)
                    pending_bytes += need
                    self.out_bytes += output_bytes(r, self.store.options)
                    pending_bytes -= output_bytes(r, self.store.options)
                if batch:
                    inflight.append(self._launch(batch, self.free_slots.pop(0), t0_event))
                    continue
            if not inflight and not waiting and pending:
                # idle until the next arrival: sleep through all but its last poll_s, then spin
                gap = pending[0].arrival - (time.perf_counter() - t0)
                if gap > 2 * poll_s:
                    time.sleep(gap - poll_s)
        torch.cuda.synchronize(self.device)
        done = [r for r in requests if r.status == "done"]
        lat = np.array([r.done_ms - 1e3 * r.arrival for r in done]) if done else np.zeros(0)
        span_ms = (max(r.done_ms for r in done) - 1e3 * min(r.arrival for r in done)) if done else 0.0
        rays = sum(r.rays for r in done)
        return {
            "requests": len(requests), "done": len(done), "rejected": len(rejected), "batches": self.batches - batches0,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_ms": float(lat.mean()) if len(lat) else None,
            "rays": rays, "span_ms": span_ms, "rays_per_s": rays / (span_ms * 1e-3) if span_ms > 0 else None,
            "cache_entries": len(self.store.cache), "cache_hits": self.store.hits - hits0,
            "cache_misses": self.store.misses - misses0,
        }


def poisson_requests(rng, n, rate_per_s, n_scenes, n_poses, resolutions, first_id=0):
    """n requests with exponential inter-arrival times (rate_per_s), uniform scene, pose and resolution."""
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))
    reqs = []
    for i in range(n):
        W, H = resolutions[int(rng.integers(len(resolutions)))]
        reqs.append(Request(first_id + i, int(rng.integers(n_scenes)), int(rng.integers(n_poses)), W, H, float(t[i])))
    return reqs


def make_scenes(rng, n_scenes=16, total_points=40_000_000, size_range=(5e5, 6e6), n_poses=16):
    """Scene clouds as in the `shapes` workload with sizes log-uniform in size_range, rescaled to
    total_points, and n_poses camera poses per scene on the radius-4 sphere."""
    lo, hi = np.log(size_range[0]), np.log(size_range[1])
    sizes = np.exp(rng.uniform(lo, hi, size=n_scenes))
    sizes = np.maximum(1, np.round(sizes * total_points / sizes.sum())).astype(np.int64)
    clouds = [synth.shapes_cloud(rng, int(n)) for n in sizes]
    poses = [[c.c2w for c in synth.orbit_cameras(rng, n_poses, 4.0, 800, 800, 1111.0, 400.0, 400.0)]
             for _ in range(n_scenes)]
    return clouds, poses
