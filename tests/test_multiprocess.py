"""The multi-GPU form on CPU: two gloo ranks (world size 2, 127.0.0.1).

Each rank builds its own view set (weak scaling), renders a small view of it
with the CPU oracle, and the job time is the slowest rank's: the ranks' camera
sets differ, each rank's result is the same as rendering that view alone, and
the reduction returns the maximum on every rank.  No GPU is used.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "hashpoint-code_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hashpoint import shard, synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(shard.view_seed(0, rank))
        cams = synth.orbit_cameras(rng, 3, 4.0, 48, 40, 60.0, 24.0, 20.0)
        xyz = synth.shapes_cloud(np.random.default_rng(7), 20000)
        opt = synth.Options(kernel_size=3, radius_threshold=0.02, num_sample_points_per_ray=4,
                            num_point_cloud_per_sp=8)
        cam = O.camera_from(cams[0])
        sidx, sdep, hsh = O.pts2plane(xyz, cam)
        res = O.quick_sampling(xyz, cam, opt, sidx, hsh)
        emitted = int(np.asarray(res[3]).sum())
        centre = torch.tensor(cams[0].c2w[:3, 3].astype(np.float64))
        gathered = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, centre)
        t_max = shard.max_over_ranks(10.0 + rank)
        value, ms = shard.job_rays_per_s(48 * 40, 1.0 + rank)
        out[rank] = (emitted, [g.tolist() for g in gathered], t_max, value, ms)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_views_and_reduce_time():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    r0, r1 = out[0], out[1]
    assert r0[1] == r1[1] and r0[1][0] != r0[1][1]   # both ranks see both camera centres; they differ
    assert r0[2] == r1[2] == 11.0                       # max over ranks
    assert r0[4] == r1[4] == 2.0                        # slowest rank's step time
    assert abs(r0[3] - 2 * 48 * 40 / 2e-3) < 1e-6      # all ranks' rays over the slowest time
    assert r0[0] > 0 and r1[0] > 0
