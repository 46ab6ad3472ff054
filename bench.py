"""Search+sample throughput benchmark (rays/s) on the 1M-point / 800x800 / 100-view workload.

Workload ("shapes"): 1,000,000 FP32 points area-uniform on 32 random boxes and
ellipsoids in [-1.5,1.5]^3 (each point also carries an fp16[32] feature the path
never reads), 100 cameras on a radius-4 sphere looking at the origin,
800x800 pixels, f=1111, radius 0.008, 5x5 window, K=8 samples, 8 points per
sample, one launch per view.  Seeded synthetic data (seed 0).

One step = all 100 views through per-view launches: for each view
hp_pts2plane (projection + per-pixel hash table) then hp_quick_sampling
(window search, primary-surface selection, sample emission, per-sample
points), every output written to HBM.  The views are spread over three
streams, each with its own buffers (hashpoint.engine.ViewRing), so one view's
build and tile scheduling run in the previous view's sampling tail; the line
also gives the same launches one after another on one stream
("single_stream").  With N GPUs (torchrun) every rank renders its own 100
views (weak scaling; no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Beside the plain per-view figure the line carries the two system forms, run on
one GPU only: "batched" (the same 100 views as one CUDA-graph-captured
persistent launch, and an uneven 64-view batch over 8 clouds of 50k-4M points
at 256^2..1600x1200) and "served" (16 resident scenes, 40M points, Poisson
requests, continuous batching, p50/p99 latency), each against the plain
per-view launches of the same kernels.

Also on the line, outside every timed region: "reference_gpu" (the
reference's own CUDA path, built from its sources into oracle/_ref, on the
same GPU and views), the other workloads' rooflines, and in "cpu_baseline" the
oracle port, the reference's own CPU point-ray searchers (KDTreeRaySearch,
UniformGrid) on the host cores, and the FP32 path's error against the FP64
oracle on three full-size views.

--impl reference times the reference algorithm's CPU implementation (the
oracle port, oracle/hp_oracle.cpp) on this machine's host cores on a bounded
sample of the same workload, rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hashpoint-code_b200"))

METRIC = "rays/s search+sample on 1 B200; served p50/p99 ms vs plain per-view launch"
RING_DEPTH = 3  # streams (and buffer sets) the per-view launches of a step are spread over
UNIT = "rays/s"
WORKLOAD = "shapes-1M-800x800-100views"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hashpoint", choices=["hashpoint", "reference"])
    ap.add_argument("--views", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-systems", action="store_true", help="skip the batched and served measurements")
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--served-only", action="store_true",
                    help="run only the served measurement and print its JSON (the main run starts this in a fresh "
                         "process)")
    ap.add_argument("--kernels-once", action="store_true",
                    help="run one view of the workload once through every kernel of the path and exit (for profilers)")
    ap.add_argument("--agg-case", type=int, default=0, metavar="N",
                    help="run the Aggregator twice on N seeded random samples (8 points each) and exit (for profilers)")
    return ap.parse_args()


def config_dict(args, extra=None):
    d = {"workload": WORKLOAD, "points": 1_000_000, "width": 800, "height": 800, "views_per_step": args.views,
         "kernel_size": 5, "radius": 0.008, "samples_per_ray": 8, "points_per_sample": 8,
         "rays_per_step": 800 * 800 * args.views, "parallelism": "views sharded across ranks (replicas)"}
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port on the host cores, the reference's own CPU
# searchers, and the FP32 path's error against the FP64 oracle
# ---------------------------------------------------------------------------
def cpu_baseline(n_views=3, scene=None, searchers=True, error_views=None):
    """Oracle (C++ restatement) on `n_views` full views of the workload, all host threads.

    rays/s = rays / (hash-table build time + sampling time), both on the CPU; the build (one
    thread) and the search+sample (all threads) are also reported apart.  With `searchers`, the
    reference's own KDTreeRaySearch / UniformGrid (point_ray_search_benchmark, staged by
    oracle/ref_cpu.py) on the 100k-point sphere workload beside it.  `error_views`: GPU outputs of
    full-size views ({name: (xyz, cam, opt, outputs...)}) whose error against the FP64 oracle is
    stated (oracle/error_stats.py).
    """
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hashpoint import synth
    oracle.build()
    sc = scene or synth.make_shapes(n_views=max(n_views, 1), with_feat=False)
    cores = os.cpu_count() or 1
    total_rays, t_build, t_search = 0, 0.0, 0.0
    for cam in sc.cameras[:n_views]:
        oc = oracle.camera_from(cam)
        t0 = time.perf_counter()
        oi, od, oh = oracle.pts2plane(sc.xyz, oc, False)
        t1 = time.perf_counter()
        oracle.quick_sampling(sc.xyz, oc, sc.options, oi, oh, nthreads=cores)
        t2 = time.perf_counter()
        t_build += t1 - t0
        t_search += t2 - t1
        total_rays += cam.width * cam.height
    t_total = t_build + t_search
    out = {"value": total_rays / t_total, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": "%d full view(s) (800x800, 1M points) of the workload: hash-table build single-threaded "
                     "(%.3f s), search+sample on %d threads (%.3f s); %.2f s wall" % (n_views, t_build, cores,
                                                                                   t_search, t_total),
           "build_s_per_view": t_build / n_views, "search_sample_rays_per_s": total_rays / t_search}
    if searchers:
        import ref_cpu
        if ref_cpu.staged():
            try:
                out["reference_searchers"] = ref_cpu.run()
            except Exception as e:  # noqa: BLE001 -- reported, the baseline leg goes on
                out["reference_searchers"] = {"unavailable": str(e).splitlines()[0][:200]}
        else:
            out["reference_searchers"] = {"unavailable": "point_ray_search_benchmark not staged (oracle/ref_cpu.py)"}
    if error_views:
        import error_stats
        out["fp64_error"] = {name: error_stats.fp64_error(*v, nthreads=cores) for name, v in error_views.items()}
    return out


def stage_desc(stage_config, heavy_window=None):
    """A tuning choice as the tile, stage capacity and occupancy it stands for."""
    from hashpoint import native
    d = {"stage_config": int(stage_config), **native.stage_config_info(stage_config)}
    if heavy_window is not None:
        d["heavy_window"] = int(heavy_window)
    return d


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for nm, v in zip(names, r[4:]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# main GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from hashpoint import native, synth
    from hashpoint.engine import CameraTable, ViewPipeline, ViewRing

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    native.build()

    from hashpoint import shard
    sc = synth.make_shapes(n_views=args.views, seed=0, with_feat=True)
    if rank > 0:  # the same cloud, this rank's own cameras
        cams = synth.orbit_cameras(np.random.default_rng(shard.view_seed(0, rank)), args.views, 4.0, 800, 800, 1111.0,
                                   400.0, 400.0)
        sc.cameras[:] = cams
    xyz = torch.from_numpy(sc.xyz).to(dev)
    feat = torch.from_numpy(sc.feat).to(dev)  # resident, never read by the path
    cams = CameraTable(sc.cameras, dev)
    ring = ViewRing(len(sc.xyz), 800, 800, sc.options, dev, depth=RING_DEPTH)
    pipe = ring.pipes[0]  # the single-stream form, the tuning and the roofline use one pipeline
    stream = torch.cuda.Stream(dev)
    structs = [cams.struct(i) for i in range(cams.n)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # the sampling kernel's stage configuration for this workload (outputs never depend on it)
    with torch.cuda.stream(stream):
        stage = ring.tune(xyz, structs[:12], stream)

    # in-image point count per view (for the algorithmic byte count), outside timing
    n_in = []
    with torch.cuda.stream(stream):
        for s in structs:
            pipe.build(xyz, s, stream)
            n_in.append(int((pipe.hash[:, 1].clamp(min=0)).sum().item()))

    S, P = sc.options.num_sample_points_per_ray, sc.options.num_point_cloud_per_sp
    HW = 800 * 800
    out_bytes = HW * S * (12 + 4 + 1 + 4 * P)
    samp_bytes = [16 * ni + 8 * HW + out_bytes for ni in n_in]

    def step():  # the timed step: per-view launches over the ring's streams
        ring.render_many(xyz, structs, stream)

    def step_single(ev_samp=None):  # the same launches on one stream, each sampling call timed
        for i, s in enumerate(structs):
            pipe.build(xyz, s, stream)
            if ev_samp is not None:
                ev_samp[i][0].record(stream)
            pipe.sample(xyz, s, stream)
            if ev_samp is not None:
                ev_samp[i][1].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1)
            step()
            flush.fill_(1)
            step_single()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t_wall0 = time.perf_counter()
    step_ms = []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flushed between steps, outside the step events
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            stream.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t_wall = time.perf_counter() - t_wall0
    value, ms_per_step = shard.job_rays_per_s(HW * len(structs), sum(step_ms) / len(step_ms), dev)

    # the same on one stream: the sequential per-view figure, and each sampling launch's duration
    single_ms, samp_ms = [], []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in structs]
            e0.record(stream)
            step_single(ev)
            e1.record(stream)
            stream.synchronize()
            single_ms.append(e0.elapsed_time(e1))
            samp_ms.extend(a.elapsed_time(b) for a, b in ev)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    single_value, single_ms_per_step = shard.job_rays_per_s(HW * len(structs), sum(single_ms) / len(single_ms), dev)

    # roofline of the dominant kernel (k_quick_sampling)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    samp_avg_ms = sum(samp_ms) / len(samp_ms)
    achieved = (sum(samp_bytes) / len(samp_bytes)) / (samp_avg_ms * 1e-3) / 1e9
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = tr.get("k_quick_sampling", {}).get(WORKLOAD)
    except (OSError, ValueError):
        pass

    # end to end through the epcq API with host buffers
    e2e = run_e2e(args, sc, dev, pipe_hw=HW)

    # the two system forms beside the plain per-view launch (one GPU runs them alone), the other
    # workloads, and the reference's own CUDA path on the same GPU
    batched = served = downstream = others = refgpu = error_views = None
    if world == 1 and not args.no_systems:
        served = run_served_isolated(args)  # a process of its own: the real-time loop is sensitive to process state
        torch.cuda.empty_cache()
        downstream = run_downstream(args, dev, xyz, feat, sc, pipe, structs, stream, peak, flush)
        others = run_other_workloads(dev, flush, peak)
        del pipe, ring
        torch.cuda.empty_cache()
        refgpu = run_reference_gpu(dev, flush, {
            WORKLOAD.rsplit("-", 1)[0]: single_ms_per_step / len(structs),
            "sphere-100k-400x400": others["sphere_100k_400x400"]["ms_per_view"],
            "clusters-3M-1600x1200": others["clusters_3M_1600x1200"]["ms_per_view"]})
        torch.cuda.empty_cache()
        batched = run_batched(args, dev, xyz, sc, flush)
        torch.cuda.empty_cache()
        error_views = collect_error_views(dev)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no public dataset)",
        "config": config_dict(args, {"l2": "flushed between steps (256 MiB write)",
                                     "path": "per-view launches (hp_pts2plane + hp_quick_sampling for each view) "
                                             "over %d streams with a buffer set each (hashpoint.engine.ViewRing)"
                                             % RING_DEPTH,
                                     "sampling_stage_config": stage_desc(stage)}),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_quick_sampling", "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": sum(samp_bytes) / len(samp_bytes),
                     "avg_launch_ms": samp_avg_ms},
        "clocks": clk, "e2e": e2e,
        "gpu_launches": ViewPipeline.KERNELS_PER_VIEW * len(structs) * args.steps,
        "wall_s_timed_region": t_wall,
        "stages_ms_per_view": {"build_plus_sample": single_ms_per_step / len(structs), "sample": samp_avg_ms},
        "single_stream": {"value": single_value, "ms_per_step": single_ms_per_step,
                          "path": "the same per-view launches one after another on one stream"},
    }
    if downstream is not None:
        result["downstream"] = downstream
    if others is not None:
        result["other_workloads"] = others
    if batched is not None:
        result["batched"] = batched
    if served is not None:
        result["served"] = served
    if refgpu is not None:
        result["reference_gpu"] = refgpu
    if rank == 0 and world == 1:
        result["cpu_baseline"] = cpu_baseline(searchers=not args.no_systems, error_views=error_views)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    del feat


def run_e2e(args, sc, dev, pipe_hw):
    """The same metric through the public epcq API, inputs copied from pinned host memory every step."""
    import numpy as np
    import torch

    from epcq import epcq as E
    from hashpoint import shard

    xyz_h = torch.from_numpy(sc.xyz).pin_memory()
    c2w_h = torch.from_numpy(np.stack([c.c2w for c in sc.cameras])).pin_memory()
    w2c_h = torch.from_numpy(np.stack([c.w2c for c in sc.cameras])).pin_memory()
    K_h = torch.from_numpy(np.stack([c.K for c in sc.cameras])).pin_memory()
    opt = E.RenderOptions(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8,
                          num_point_cloud_per_sp=8)
    counts_h = torch.empty(len(sc.cameras), dtype=torch.int64).pin_memory()
    h2d = xyz_h.numel() * 4 + (c2w_h.numel() + w2c_h.numel() + K_h.numel()) * 4
    d2h = counts_h.numel() * 8
    model = E.NeuralPoints(pc_type="pc", points=torch.empty_like(xyz_h, device=dev))
    c2w, w2c, K = (torch.empty_like(t, device=dev) for t in (c2w_h, w2c_h, K_h))

    # the reference's own caller (opt/render_image.py:61-68) passes fx..cy as 0-d CUDA tensors taken
    # from K and the image size as a CUDA tensor; the library reads them back once per view
    hw_h = torch.tensor([[c.height, c.width] for c in sc.cameras], dtype=torch.int64).pin_memory()
    hw = torch.empty_like(hw_h, device=dev)
    side = [torch.cuda.Stream(dev) for _ in range(RING_DEPTH)]

    def view(i, counts, device_scalars):
        if device_scalars:
            fx, fy, cx, cy = E.CameraSpec.decomposeK(K[i])
            cam = E.CameraSpec(c2w=c2w[i], w2c=w2c[i], K=K[i], fx=fx, fy=fy, cx=cx, cy=cy, height=hw[i, 0],
                               width=hw[i, 1])
        else:
            c = sc.cameras[i]
            cam = E.CameraSpec(c2w=c2w[i], w2c=w2c[i], K=K[i], fx=c.fx, fy=c.fy, cx=c.cx, cy=c.cy,
                               width=c.width, height=c.height)
        idx, dep, hsh = model.pts2plane(cam, opt)
        sp_xyz, pc_idx, sp_t, mask = model.render_image_hashtable_topk(cam, opt, idx, dep, hsh)
        counts[i] = mask.sum()

    def step(device_scalars=False, streams=None):
        main = torch.cuda.current_stream(dev)
        model.xyz_data.data.copy_(xyz_h, non_blocking=True)
        c2w.copy_(c2w_h, non_blocking=True)
        w2c.copy_(w2c_h, non_blocking=True)
        K.copy_(K_h, non_blocking=True)
        hw.copy_(hw_h, non_blocking=True)
        counts = torch.empty(len(sc.cameras), dtype=torch.int64, device=dev)
        if streams is None:
            for i in range(len(sc.cameras)):
                view(i, counts, device_scalars)
        else:
            # views dealt round-robin over torch streams, as a caller overlapping views would: each
            # call launches on the current stream and allocates its outputs and workspaces there
            for s in streams:
                s.wait_stream(main)
            for i in range(len(sc.cameras)):
                with torch.cuda.stream(streams[i % len(streams)]):
                    view(i, counts, device_scalars)
            for s in streams:
                main.wait_stream(s)
        counts_h.copy_(counts, non_blocking=True)

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(max(args.e2e_steps, 1)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
        return sum(ts) / len(ts)

    # whole job: every rank's rays over the slowest rank's step (every rank takes the same three steps)
    rate_ms = [shard.job_rays_per_s(pipe_hw * len(sc.cameras), timed(fn), dev)
               for fn in (lambda: step(streams=side), step, lambda: step(device_scalars=True, streams=side))]
    (value, ms), (value_one, ms_one), (value_dev, ms_dev) = rate_ms
    h2d_all = h2d + hw_h.numel() * 8
    return {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d_all, "d2h_bytes_per_step": d2h,
            "ms_per_step": ms, "api": f"epcq.NeuralPoints.pts2plane + render_image_hashtable_topk per view, the "
            f"views dealt round-robin over {len(side)} torch streams; xyz, cameras and image sizes copied from "
            "pinned host memory each step, per-view emitted-sample counts read back",
            "one_stream": {"value": value_one, "unit": UNIT, "ms_per_step": ms_one,
                           "api": "the same calls, every view on the current stream"},
            "device_scalars": {"value": value_dev, "unit": UNIT, "ms_per_step": ms_dev,
                               "api": "the same calls over the same streams with fx..cy as 0-d CUDA tensors "
                                      "from K and the image size as a CUDA tensor, as the reference's renderer "
                                      "passes them (the six scalars read back to the host once per view)"}}


def _event_ms(fn, reps, flush=None):
    import torch
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def run_downstream(args, dev, xyz, feat, sc, pipe, structs, stream, peak, flush):
    """The rows after sampling on the same views: the FeatureQuery gather (mask scan + gather of
    xyz/rgb/dir and the fp16[32] features of every selected point) and render (clamp_t fused),
    timed per view with CUDA events; HBM fraction from the bytes each must move."""
    import numpy as np
    import torch

    from hashpoint import ops

    n = xyz.shape[0]
    rng = np.random.default_rng(3)
    rgb = torch.from_numpy(rng.random((n, 3), dtype=np.float32)).to(dev)
    dr = torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)).to(dev)
    S, P, F = sc.options.num_sample_points_per_ray, sc.options.num_point_cloud_per_sp, feat.shape[1]
    fq_ms, fq_bytes, r_ms, r_bytes = [], [], [], []
    # Aggregator: seeded random weights of the reference's layer shapes
    lay = ops.AGG_LAYERS
    agg_w = [torch.from_numpy((rng.standard_normal((o, i)) / np.sqrt(i)).astype(np.float32)).to(dev) for _, o, i in lay]
    agg_b = [torch.from_numpy((rng.standard_normal(o) * 0.05).astype(np.float32)).to(dev) for _, o, _ in lay]
    packed = ops.aggregator_pack(agg_w, agg_b)
    ag_ms, ag_alg, ag_exec = [], [], []
    pair_flops = 2 * sum(o * i for name, o, i in lay if not name.startswith("color"))
    color_flops = 2 * sum(o * i for name, o, i in lay if name.startswith("color"))
    with torch.cuda.stream(stream):
        for i in range(min(10, len(structs))):
            pipe.render(xyz, structs[i], stream)
            c = sc.cameras[i]
            sp_xyz, pc_idx, sp_t, mask = (t.clone() for t in (pipe.sp_xyz, pipe.pc_idx, pipe.sp_t, pipe.mask))
            c2w = torch.from_numpy(c.c2w).to(dev)
            R = c.width * c.height
            sig = torch.rand((R, S), device=dev) * 50
            rgbs = torch.rand((R, S, 3), device=dev)
            t_val = sp_t.view(R, S)
            for rep in range(2):  # the second is timed
                flush.fill_(1)
                e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                e[0].record(stream)
                out = ops.feature_query(xyz, rgb, dr, feat, sp_xyz, pc_idx, mask, c2w, c.fx, c.fy, c.cx, c.cy, c.width)
                e[1].record(stream)
                flush.fill_(1)
                e[2].record(stream)
                ops.render(None, sig, rgbs, t_val=t_val)
                e[3].record(stream)
                stream.synchronize()
            M = out[0].shape[0]
            # mask read, offsets written and read, sample rows and ids read, P ids' rows gathered, outputs written
            fq_bytes.append(R * S * (1 + 8) + M * (12 + 4 * P) + M * P * (36 + 2 * F) +
                            M * (P * (36 + 4 * F + 1) + 24))
            fq_ms.append(e[0].elapsed_time(e[1]))
            r_bytes.append(R * S * (4 + 4 + 12) + R * 12)
            r_ms.append(e[2].elapsed_time(e[3]))
            for rep in range(2):  # the second is timed
                flush.fill_(1)
                ea = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ea[0].record(stream)
                ops.aggregator_forward(packed, *out[:6], mask, out[6])
                ea[1].record(stream)
                stream.synchronize()
            n_valid = int(out[5].sum())
            ag_ms.append(ea[0].elapsed_time(ea[1]))
            ag_alg.append(n_valid * pair_flops + M * color_flops)
            ag_exec.append(M * P * 2 * 256 * (320 + 256 + 256 + 16 + 256) + M * 2 * 128 * (320 + 128 + 128))
    fq = statistics.median(fq_ms)
    rr = statistics.median(r_ms)
    fqb = sum(fq_bytes) / len(fq_bytes)
    rb = sum(r_bytes) / len(r_bytes)
    return {"feature_query": {"ms_per_view": fq, "bytes_per_view": fqb, "gbs": fqb / (fq * 1e-3) / 1e9,
                              "frac_of_hbm": fqb / (fq * 1e-3) / 1e9 / peak,
                              "note": "includes the mask scan and the read-back of the sample count"},
            "render": {"ms_per_view": rr, "bytes_per_view": rb, "gbs": rb / (rr * 1e-3) / 1e9,
                       "frac_of_hbm": rb / (rr * 1e-3) / 1e9 / peak, "note": "clamp_t fused"},
            "aggregator": _aggregator_figures(ag_ms, ag_alg, ag_exec),
            "views": len(fq_ms)}


def _aggregator_figures(ms, alg, executed):
    """Aggregator per view: algorithmic TFLOP/s (the reference's layers over its valid (sample, point)
    pairs and samples) and the tensor-core rate actually executed (all pair rows, K padded to 64),
    each against the measured dense bf16 peak."""
    peak = _measured("bf16_tflops")
    t = statistics.median(ms)
    a = sum(alg) / len(alg)
    x = sum(executed) / len(executed)
    return {"ms_per_view": t, "tflops": a / (t * 1e-3) / 1e12, "executed_tflops": x / (t * 1e-3) / 1e12,
            "peak_tflops": peak, "frac_of_peak": (a / (t * 1e-3) / 1e12) / peak if peak else None,
            "executed_frac_of_peak": (x / (t * 1e-3) / 1e12) / peak if peak else None,
            "note": "bf16 operands, fp32 accumulation; peak = measured burst bf16 GEMM"}


def _measured(key):
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key])
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}.get(key)


def sampling_bytes(n_in, H, W, S, P):
    """Algorithmic bytes of one k_quick_sampling launch: the in-image points' (x, y, z, id) records and
    the hash table read once, every output element written once."""
    HW = H * W
    return 16 * n_in + 8 * HW + HW * S * (12 + 4 + 1 + 4 * P)


def run_other_workloads(dev, flush, peak):
    """The 100k-point sphere at 400x400 (k=3) and the 3M-point clusters at 1600x1200 (K=16) through
    the same plain per-view launch (CUDA events, L2 flushed before each view), with the stage
    configuration the pipeline's tune() picks for the workload: build + sample per view, the
    sampling launch alone, and its fraction of the HBM roofline."""
    import torch

    from hashpoint import synth
    from hashpoint.engine import CameraTable, ViewPipeline

    out = {}
    for name, sc in (("sphere_100k_400x400", synth.make_sphere()), ("clusters_3M_1600x1200", synth.make_clusters(n_views=4))):
        X = torch.from_numpy(sc.xyz).to(dev)
        c0 = sc.cameras[0]
        pipe = ViewPipeline(len(sc.xyz), c0.height, c0.width, sc.options, dev)
        cams = CameraTable(sc.cameras, dev)
        structs = [cams.struct(i) for i in range(cams.n)]
        st = torch.cuda.current_stream(dev)
        stage = pipe.tune(X, structs[:2], st)
        n_in = []
        for s_ in structs:
            pipe.render(X, s_)
            n_in.append(int(pipe.hash[:, 1].clamp(min=0).sum().item()))
        ts, ss = [], []
        for _ in range(3):
            for s_ in structs:
                flush.fill_(1)
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e[0].record()
                pipe.build(X, s_, st)
                e[1].record()
                pipe.sample(X, s_, st)
                e[2].record()
                e[2].synchronize()
                ts.append(e[0].elapsed_time(e[2]))
                ss.append(e[1].elapsed_time(e[2]))
        ms, sms = statistics.median(ts), statistics.median(ss)
        S, P = sc.options.num_sample_points_per_ray, sc.options.num_point_cloud_per_sp
        nbytes = sum(sampling_bytes(ni, c0.height, c0.width, S, P) for ni in n_in) / len(n_in)
        achieved = nbytes / (sms * 1e-3) / 1e9
        out[name] = {"rays_per_s": c0.width * c0.height / (ms * 1e-3), "ms_per_view": ms, "sample_ms": sms,
                     "views": len(structs), "points": len(sc.xyz), "sampling_stage_config": stage_desc(stage),
                     "roofline": {"bound": "hbm", "kernel": "k_quick_sampling", "achieved": achieved, "peak": peak,
                                  "unit": "GB/s", "frac": achieved / peak, "algorithmic_bytes_per_launch": nbytes}}
        del pipe, X
        torch.cuda.empty_cache()
    return out


def collect_error_views(dev):
    """View 0 of the sphere, shapes and clusters workloads through the CUDA path, as host arrays
    (the inputs of oracle/error_stats.fp64_error)."""
    import torch

    from hashpoint import ops, synth

    out = {}
    for name, sc in (("sphere", synth.make_sphere()), ("shapes", synth.make_shapes(n_views=1, with_feat=False)),
                     ("clusters", synth.make_clusters(n_views=1))):
        cam = sc.cameras[0]
        X = torch.from_numpy(sc.xyz).to(dev)
        c2w, w2c, K = (torch.from_numpy(a).to(dev) for a in (cam.c2w, cam.w2c, cam.K))
        sidx, sdep, hsh = ops.pts2plane(X, w2c, K, cam.height, cam.width, False)
        sp_xyz, pc_idx, sp_t, mask = ops.quick_sampling(X, c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height,
                                                        sc.options, sidx, hsh)
        dirs = ops.ray_directions(c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height)
        H = lambda t: t.cpu().numpy()
        out[name] = (sc.xyz, cam, sc.options, H(sidx), H(sdep), H(hsh), H(sp_xyz), H(sp_t), H(mask), H(pc_idx), H(dirs))
        del X
    torch.cuda.empty_cache()
    return out


def run_reference_gpu(dev, flush, ours):
    """The reference's own CUDA path on the same GPU and inputs: its extension (oracle/_ref, built
    from the reference's sources) driven as epcq.py:279-325 drives it -- torch projection and
    sort, _C.scatter_hashtable, _C.quick_sampling -- timed per view with CUDA events (L2 flushed
    before each step of views), beside this library's plain per-view launch of the same views.
    `ours`: {workload: ms per view} of this library."""
    import numpy as np
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_ref
    from ref_pipeline import RefPipeline
    from hashpoint import synth

    if not os.path.exists(build_ref.SO_PATH):
        return {"unavailable": "the reference's CUDA build (oracle/_ref) is not present"}
    rp = RefPipeline(build_ref.load(), dev)
    out = {}
    for name, sc, nv in (("shapes-1M-800x800", synth.make_shapes(n_views=10, with_feat=False), 10),
                         ("sphere-100k-400x400", synth.make_sphere(), 1),
                         ("clusters-3M-1600x1200", synth.make_clusters(n_views=4), 4)):
        X = torch.from_numpy(sc.xyz).to(dev)
        cams = [(torch.from_numpy(c.c2w).to(dev), torch.from_numpy(c.w2c).to(dev), torch.from_numpy(c.K).to(dev), c)
                for c in sc.cameras[:nv]]
        for c2w, w2c, K, c in cams:  # warm-up
            rp.render(X, c2w, w2c, K, c, sc.options)
        steps = []
        for _ in range(3 if nv > 1 else 10):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for c2w, w2c, K, c in cams:
                rp.render(X, c2w, w2c, K, c, sc.options)
            e1.record()
            e1.synchronize()
            steps.append(e0.elapsed_time(e1) / nv)
        ms = statistics.median(steps)
        rays = sc.cameras[0].width * sc.cameras[0].height
        out[name] = {"ms_per_view": ms, "rays_per_s": rays / (ms * 1e-3), "views": nv,
                     "ms_per_view_here": ours.get(name), "speedup_over_reference_gpu":
                     ms / ours[name] if ours.get(name) else None}
        del X, cams
        torch.cuda.empty_cache()
    out["path"] = ("reference extension built from the reference's epcq/csrc for sm_100a, driven as epcq.py "
                   "pts2plane + render_image_hashtable_topk (P=8); the sorted pixel ids get a sentinel element "
                   "after the end (the reference's bucket walk reads one past them)")
    return out


def run_batched(args, dev, xyz, sc, flush):
    """Batching: the same 100 views as one graph-captured persistent launch; and the uneven
    multi-cloud batch (64 views over 8 clouds of 50k-4M points at 256^2..1600x1200), each
    against the plain per-view launches of the same kernels over the same buffers."""
    import torch

    from hashpoint import batch, synth

    out = {}
    tuner = batch.Autotuner()
    # same workload as the headline: 100 views of the 1M-point cloud, one batch
    r = batch.BatchRenderer([xyz], [(0, c) for c in sc.cameras], sc.options, dev)
    tuning = tuner.tune(r)
    r.capture()
    r.run_per_view()
    torch.cuda.synchronize(dev)
    pv = _event_ms(r.run_per_view, 3, flush)
    g = _event_ms(r.replay, max(args.steps, 3), flush)
    out["shapes_100views"] = {"rays_per_s": r.rays / (g * 1e-3), "ms": g, "per_view_rays_s": r.rays / (pv * 1e-3),
                              "per_view_ms": pv, "speedup": pv / g, "tuning": stage_desc(*tuning),
                              "path": "hp_pts2plane x100 on 4 streams + one hp_quick_sampling_batch, CUDA graph"}
    r.release()
    del r
    torch.cuda.empty_cache()
    # uneven batch: 8 clouds log-uniform in 50k-4M points, 64 views, mixed resolutions
    mb = synth.make_mixed(n_clouds=8, n_views=64, seed=0)
    clouds = [torch.from_numpy(c).to(dev) for c in mb.clouds]
    order = sorted(range(len(mb.views)), key=lambda i: -len(mb.clouds[mb.views[i][0]]))  # heavy views first
    r = batch.BatchRenderer(clouds, [mb.views[i] for i in order], mb.options, dev)
    tuning = tuner.tune(r)
    r.capture()
    r.run_per_view()
    torch.cuda.synchronize(dev)
    pv = _event_ms(r.run_per_view, 3, flush)
    g = _event_ms(r.replay, max(args.steps, 3), flush)
    out["mixed_64views_8clouds"] = {
        "rays_per_s": r.rays / (g * 1e-3), "ms": g, "per_view_rays_s": r.rays / (pv * 1e-3), "per_view_ms": pv,
        "speedup": pv / g, "tuning": stage_desc(*tuning), "rays": r.rays, "points": [int(c.shape[0]) for c in clouds],
        "path": "one CUDA graph: 64 hash-table builds on 4 streams + one persistent sampling launch"}
    r.release()
    del r, clouds
    return out


def run_served_isolated(args):
    """run_served in a fresh process on the same GPU, as a server would run: the request loop is
    a real-time host loop, and in the benchmark process -- after the timed sections' allocations,
    streams and host threads -- its latency was an order of magnitude worse than in a process of
    its own on the same machine."""
    cmd = [sys.executable, os.path.abspath(__file__), "--served-only", "--serve-requests", str(args.serve_requests)]
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env, timeout=1200)
    if p.returncode != 0:
        return {"unavailable": "served run failed: " + p.stderr.strip().splitlines()[-1][:200] if p.stderr else "?"}
    out = json.loads(p.stdout.strip().splitlines()[-1])
    out["process"] = "fresh (bench.py --served-only)"
    return out


def run_served(args, dev):
    """Serving: 16 resident scenes (40M points), Poisson requests at 2000/s (mixed resolutions,
    K=8), 120 GB budget, continuous batching; p50/p99 latency and rays/s against serial plain
    launches of the same requests (hash tables cached per scene, camera pose and resolution)."""
    import numpy as np
    import torch

    from hashpoint import ops, serve, synth

    clouds, poses = serve.make_scenes(np.random.default_rng(0))
    opt = synth.Options(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8, num_point_cloud_per_sp=8)
    store = serve.SceneStore([torch.from_numpy(c).to(dev) for c in clouds], poses, opt, dev)
    n = max(int(args.serve_requests), 10)

    def requests(rate, count):
        return serve.poisson_requests(np.random.default_rng(1), count, rate, len(clouds), len(poses[0]),
                                      synth.MIXED_RESOLUTIONS)

    budget = 120 << 30
    torch.cuda.empty_cache()
    server = serve.Server(store, budget)  # one server for every run, as a service would keep it
    tuned = server.tune(requests(2000.0, n))  # once at start-up, on one batch of requests
    server.run(requests(2000.0, n))  # warm: hash-table cache, output pool, workspaces

    def median_run(rate, count, runs=3):
        # The first run meets cold hash-table caches (every new scene/pose builds its table);
        # it is reported on its own as the cold start.  Batch formation under a Poisson arrival
        # stream depends on timing, so warm runs vary too: report the warm run with the median
        # p50 and every run's figures in order.
        cold = server.run(requests(rate, count))
        runs_ = [server.run(requests(rate, count)) for _ in range(runs)]
        res = sorted(runs_, key=lambda r: r["p50_ms"])
        med = dict(res[len(res) // 2])
        med["runs_rays_per_s"] = [r["rays_per_s"] for r in runs_]
        keys = ("p50_ms", "p99_ms", "batches", "cache_misses")
        med["cold_run"] = {k: cold[k] for k in keys}
        med["runs_in_order"] = [{k: r[k] for k in keys} for r in runs_]
        return med

    hot = median_run(2000.0, n)
    light = median_run(200.0, max(n // 3, 10))
    # the same requests through serial plain launches (cached tables, one request at a time)
    reqs = requests(2000.0, n)
    mk = lambda b: torch.empty(max(b, 1), dtype=torch.uint8, device=dev)

    def serial():
        s = torch.cuda.current_stream(dev)
        for q in reqs:
            e = store.lookup(q, s, mk)
            e.users -= 1
            cam, c2w, _, _ = store.camera(q.scene, q.pose, q.width, q.height)
            ops.quick_sampling(store.clouds[q.scene], c2w, cam.fx, cam.fy, cam.cx, cam.cy, q.width, q.height, opt,
                               e.sidx, e.hash, tuning=server.tuning)  # the served launches' stage configuration

    ser = _event_ms(serial, 1)
    rays = sum(q.rays for q in reqs)
    keep = ("requests", "done", "rejected", "batches", "p50_ms", "p99_ms", "mean_ms", "rays_per_s", "span_ms",
            "runs_rays_per_s", "cache_hits", "cache_misses", "cold_run", "runs_in_order")
    return {"scenes": len(clouds), "points": int(sum(len(c) for c in clouds)), "budget_gb": 120,
            "tuning": stage_desc(*tuned),
            "lambda_2000": {k: hot[k] for k in keep}, "lambda_200": {k: light[k] for k in keep},
            "serial_plain_rays_per_s": rays / (ser * 1e-3), "serial_plain_ms": ser,
            "speedup_vs_serial_plain": (hot["rays_per_s"] or 0) / (rays / (ser * 1e-3)),
            "note": "one cold run (cold_run: every scene/pose table built on first use), then the warm run "
                    "with the median p50 of 3; at 2000 requests/s the offered load exceeds the GPU's capacity, "
                    "so latency is mostly queueing; 200 requests/s is below it; cameras: 16 fixed poses per scene "
                    "(hash tables cached per scene, pose and resolution); cache_misses counts the tables built "
                    "during the reported run"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from hashpoint import synth
    sc = synth.make_shapes(n_views=1, with_feat=False)
    for _ in range(args.warmup):
        cpu_baseline(n_views=1, scene=sc, searchers=False)
    vals = [cpu_baseline(n_views=1, scene=sc, searchers=False) for _ in range(args.steps)]
    value = sum(v["value"] for v in vals) / len(vals)
    base = dict(vals[-1])
    base["value"] = value
    base["sample"] = "per step " + base["sample"]
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 640000 / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no public dataset)",
        "config": config_dict(args, {"views_per_step": 1, "rays_per_step": 640000}), "impl": "reference",
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_kernels_once(args):
    """One view of the workload through every kernel once, after one untimed pass: the projection and
    hash-table build, the per-view sampling launch, a 4-view batched launch, the listed-ray query,
    ray directions, the FeatureQuery gather (fp16[32] features), the Aggregator (random weights),
    clamp_t and render.  Prints no bench line: this is the command the per-kernel profiles are
    captured on."""
    import numpy as np
    import torch

    from hashpoint import batch, native, ops, synth

    native.build()
    dev = torch.device("cuda", 0)
    sc = synth.make_shapes(n_views=4, seed=0, with_feat=True)
    xyz = torch.from_numpy(sc.xyz).to(dev)
    feat = torch.from_numpy(sc.feat).to(dev)
    rng = np.random.default_rng(3)
    n = xyz.shape[0]
    rgb = torch.from_numpy(rng.random((n, 3), dtype=np.float32)).to(dev)
    dr = torch.from_numpy(rng.standard_normal((n, 3)).astype(np.float32)).to(dev)
    cam = sc.cameras[0]
    c2w, w2c, K = (torch.from_numpy(np.asarray(a, np.float32)).to(dev) for a in (cam.c2w, cam.w2c, cam.K))
    S = sc.options.num_sample_points_per_ray
    R = cam.width * cam.height
    ray_ids = torch.from_numpy(rng.choice(R, 65536, replace=False).astype(np.int32)).to(dev)
    sig = torch.rand((R, S), device=dev) * 50
    rgbs = torch.rand((R, S, 3), device=dev)
    r = batch.BatchRenderer([xyz], [(0, c) for c in sc.cameras], sc.options, dev)
    lay = ops.AGG_LAYERS
    packed = ops.aggregator_pack(
        [torch.from_numpy((rng.standard_normal((o, i)) / np.sqrt(i)).astype(np.float32)).to(dev) for _, o, i in lay],
        [torch.from_numpy((rng.standard_normal(o) * 0.05).astype(np.float32)).to(dev) for _, o, _ in lay])
    for _ in range(2):  # the first pass loads the library and warms up
        sidx, _, hsh = ops.pts2plane(xyz, w2c, K, cam.height, cam.width)
        sp_xyz, pc_idx, sp_t, mask = ops.quick_sampling(xyz, c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width,
                                                        cam.height, sc.options, sidx, hsh)
        r.run()
        ops.quick_query(xyz, c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height, sc.options, sidx, hsh,
                        ray_ids)
        ops.ray_directions(c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height)
        fq = ops.feature_query(xyz, rgb, dr, feat, sp_xyz, pc_idx, mask, c2w, cam.fx, cam.fy, cam.cx, cam.cy,
                               cam.width)
        ops.aggregator_forward(packed, *fq[:6], mask, fq[6])
        d = ops.clamp_t(sp_t.view(R, S))
        ops.render(d, sig, rgbs)
        torch.cuda.synchronize(dev)
    print("kernels-once: ok", flush=True)


def run_agg_case(n):
    """The Aggregator alone on n seeded random samples of 8 points (features N(0, 1), weights of the
    reference's shapes), twice, with the status check at the end.  No bench line."""
    import numpy as np
    import torch

    from hashpoint import native, ops

    native.build()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(1)
    P = 8
    sp = rng.standard_normal((n, 3)).astype(np.float32)
    pc_xyz = (sp[:, None, :] + 0.01 * rng.standard_normal((n, P, 3))).astype(np.float32)

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    ins = [T(pc_xyz), T(rng.random((n, P, 3), dtype=np.float32)), T(rng.standard_normal((n, P, 3)).astype(np.float32)),
           T(rng.standard_normal((n, P, 32)).astype(np.float32)), T(sp), T(rng.random((n, P)) < 0.75)]
    rays_d = T(rng.standard_normal((n, 3)).astype(np.float32))
    mask = torch.ones((n, 1), dtype=torch.bool, device=dev)
    lay = ops.AGG_LAYERS
    packed = ops.aggregator_pack([T((rng.standard_normal((o, i)) / np.sqrt(i)).astype(np.float32)) for _, o, i in lay],
                                 [T((rng.standard_normal(o) * 0.05).astype(np.float32)) for _, o, _ in lay])
    for rep in range(2):
        ops.aggregator_forward(packed, *ins, mask, rays_d, check_status=rep == 1)
    print("agg-case: ok, %d samples" % n, flush=True)


def main():
    args = parse()
    if args.served_only:
        import torch
        from hashpoint import native
        native.build()
        print(json.dumps(run_served(args, torch.device("cuda", 0))), flush=True)
    elif args.kernels_once:
        run_kernels_once(args)
    elif args.agg_case > 0:
        run_agg_case(args.agg_case)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
