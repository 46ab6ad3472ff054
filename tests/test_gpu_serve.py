"""Serving loop (hashpoint.serve): continuous batching over resident scenes.

Each request's result must be the same served in a mix of overlapping
requests as rendered alone with the plain per-view launch (bit-exact), under
a roomy budget (many requests per batch, several batches in flight) and under
a tight one (admission waits for memory to free up); a request that can never
fit the budget is rejected, and the others still complete.
"""
import numpy as np
import pytest
import torch

from hashpoint import native, ops, serve, synth
from hp_testutil import bits

pytestmark = pytest.mark.gpu

RES = ((64, 64), (128, 96), (200, 150))


@pytest.fixture(scope="module")
def store():
    native.build()
    rng = np.random.default_rng(11)
    clouds, poses = serve.make_scenes(rng, n_scenes=3, total_points=400_000, size_range=(5e4, 2e5), n_poses=4)
    opt = synth.Options(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8, num_point_cloud_per_sp=8)
    return serve.SceneStore([torch.from_numpy(c).cuda() for c in clouds], poses, opt, "cuda")


def _alone(store, r):
    cam, c2w, w2c, K = store.camera(r.scene, r.pose, r.width, r.height)
    xyz = store.clouds[r.scene]
    sidx, _, hsh = ops.pts2plane(xyz, w2c, K, r.height, r.width)
    return ops.quick_sampling(xyz, c2w, cam.fx, cam.fy, cam.cx, cam.cy, r.width, r.height, store.options, sidx, hsh)


def _collect():
    got = {}

    def on_result(r):
        got[r.rid] = tuple(t.clone() for t in r.outputs)

    return got, on_result


def _check(store, reqs, got):
    for r in reqs:
        if r.status != "done":
            continue
        ref = _alone(store, r)
        for a, b in zip(got[r.rid], ref):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            if a.dtype == np.float32:
                assert np.array_equal(bits(a), bits(b)), r.rid
            else:
                assert np.array_equal(a, b), r.rid


def test_served_results_equal_alone(store):
    rng = np.random.default_rng(1)
    reqs = serve.poisson_requests(rng, 48, 20000.0, 3, 4, RES)
    got, on_result = _collect()
    srv = serve.Server(store, 8 << 30, streams=3, max_views=8, on_result=on_result)
    stage, heavy = srv.tune(reqs[:8])  # start-up tuning; results must not depend on it
    assert srv.tuning.stage_config == stage and srv.tuning.heavy_window == heavy
    stats = srv.run(reqs)
    assert stats["done"] == 48 and stats["rejected"] == 0
    assert stats["batches"] < 48  # requests were batched
    assert stats["cache_entries"] <= 3 * 4 * len(RES)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    _check(store, reqs, got)


def test_tight_budget_admission_and_rejection(store):
    rng = np.random.default_rng(2)
    reqs = serve.poisson_requests(rng, 12, 5000.0, 3, 4, RES, first_id=100)
    # one request larger than the whole budget
    reqs.append(serve.Request(999, 0, 0, 1600, 1200, 0.0))
    got, on_result = _collect()
    one = serve.output_bytes(serve.Request(0, 0, 0, 200, 150, 0.0), store.options)
    budget = store.scene_bytes + 3 * one + 2 * (8 * 200_000 + 8 * 200 * 150)
    srv = serve.Server(store, budget, streams=2, max_views=4, on_result=on_result)
    stats = srv.run(reqs)
    assert stats["rejected"] == 1 and reqs[-1].status == "rejected"
    assert stats["done"] == 12
    _check(store, reqs, got)
