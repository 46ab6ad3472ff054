"""Host-side logic on the CPU: the serving loop's camera construction, byte
accounting, hash-table cache (LRU eviction, pinning) and request stream; the
autotuner's shape classes; and every entry point's rejection of host tensors.
No device work: the cache entries and renderers here are stand-ins."""
import collections
import types

import numpy as np
import pytest
import torch

from hashpoint import batch, serve, synth
from epcq.epcq import RenderOptions


def test_camera_for_scales_focal_length_with_width():
    c2w = synth.orbit_cameras(np.random.default_rng(0), 1, 4.0, 800, 800, 1111.0, 400.0, 400.0)[0].c2w
    for W, H in ((256, 256), (800, 800), (1600, 1200)):
        cam = serve.camera_for(c2w, W, H)
        assert cam.width == W and cam.height == H
        assert np.isclose(cam.fx, 1111.0 * W / 800) and np.isclose(cam.fy, cam.fx)
        assert cam.cx == W / 2 and cam.cy == H / 2
        np.testing.assert_allclose(cam.w2c @ cam.c2w, np.eye(4), atol=1e-5)


def test_output_bytes_counts_the_four_sampling_outputs():
    opt = RenderOptions()
    opt.num_sample_points_per_ray, opt.num_point_cloud_per_sp = 8, 8
    r = serve.Request(0, 0, 0, 800, 600, 0.0)
    # sp_xyz f32[3] + sp_t f32 + mask u8 + pc_idx i32[P] per sample
    assert serve.output_bytes(r, opt) == 800 * 600 * 8 * (12 + 4 + 1 + 4 * 8)
    assert r.rays == 480000


def _store(n_points_per_scene):
    """A SceneStore without device tensors: only what the accounting reads."""
    s = serve.SceneStore.__new__(serve.SceneStore)
    s.clouds = [torch.empty((n, 3)) for n in n_points_per_scene]
    s.cache = collections.OrderedDict()
    s.scene_bytes = sum(12 * n for n in n_points_per_scene)
    s.bytes = s.scene_bytes
    return s


def _add(store, key, nbytes, users=0):
    store.cache[key] = types.SimpleNamespace(bytes=nbytes, users=users)
    store.bytes += nbytes


def test_entry_bytes_is_zero_for_a_cached_table():
    s = _store([1000, 2000])
    r = serve.Request(0, 1, 3, 64, 32, 0.0)
    assert s.entry_bytes(r) == 8 * 2000 + 8 * 64 * 32  # sorted ids + depths, (start, count) per pixel
    _add(s, (1, 3, 64, 32), 123)
    assert s.entry_bytes(r) == 0


def test_evict_drops_least_recently_used_tables_not_in_use():
    s = _store([100])  # 1200 bytes of scenes
    _add(s, "a", 100)
    _add(s, "b", 200, users=1)  # a batch in flight reads it
    _add(s, "c", 300)
    budget = 1200 + 600
    # 600 cached + 100 other + 150 needed = 850 > 600 spare: "a" goes (LRU first), then "b" is pinned, "c" goes
    assert s.evict(150, budget, other_bytes=100)
    assert list(s.cache) == ["b"] and s.bytes == 1200 + 200
    # nothing left to drop: 200 + 100 + 350 > 600
    assert not s.evict(350, budget, other_bytes=100)
    assert list(s.cache) == ["b"]
    # it fits once the batch is done with "b"
    s.cache["b"].users = 0
    assert s.evict(350, budget, other_bytes=100) and not s.cache and s.bytes == 1200


def test_evict_keeps_everything_when_it_fits():
    s = _store([100])
    _add(s, "a", 100)
    _add(s, "b", 100)
    assert s.evict(10, 1200 + 300, other_bytes=0)
    assert list(s.cache) == ["a", "b"]


def test_reserve_pins_a_cached_table():
    s = _store([100])
    r = serve.Request(0, 0, 1, 8, 8, 0.0)
    assert not s.reserve(r)  # nothing cached: built at launch
    _add(s, (0, 1, 8, 8), 50)
    assert s.reserve(r) and s.cache[(0, 1, 8, 8)].users == 1
    assert not s.evict(10_000, 1200 + 50, other_bytes=0)  # pinned: not evicted
    assert (0, 1, 8, 8) in s.cache


def test_poisson_requests():
    rng = np.random.default_rng(3)
    res = ((256, 256), (512, 512), (1600, 1200))
    reqs = serve.poisson_requests(rng, 4000, 2000.0, 16, 5, res, first_id=10)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) >= 0)
    assert abs(len(reqs) / t[-1] - 2000.0) < 2000.0 * 0.05  # the mean rate
    assert [r.rid for r in reqs] == list(range(10, 4010))
    assert {r.scene for r in reqs} <= set(range(16)) and {r.pose for r in reqs} <= set(range(5))
    assert {(r.width, r.height) for r in reqs} == set(res)
    assert all(r.status == "waiting" and r.outputs is None for r in reqs)


def test_autotuner_shape_classes():
    opt = RenderOptions()
    opt.kernel_size, opt.num_sample_points_per_ray, opt.num_point_cloud_per_sp = 5, 8, 8

    def renderer(n_views, rays, points):
        return types.SimpleNamespace(clouds=[torch.empty((p, 3)) for p in points], options=opt,
                                     views=[None] * n_views, rays=rays)

    a = batch.Autotuner()
    k = a.key(renderer(4, 800 * 800 * 4, [1_000_000, 500_000]))
    assert k == (4, 21, 20, 5, 8, 8)  # log2 of 2.56e6 rays and 1.5e6 points
    # within a class (same power-of-two bins) the key and so the tuning is shared
    assert a.key(renderer(4, 800 * 800 * 4 + 1000, [1_200_000, 400_000])) == k
    assert a.key(renderer(8, 800 * 800 * 4, [1_000_000, 500_000])) != k
    assert a.key(renderer(1, 0, [0])) == (1, 0, 0, 5, 8, 8)


def _cpu_calls():
    from epcq import epcq as E
    from hashpoint import ops
    opt = synth.Options()
    f, i, m4, K = torch.zeros(4, 3), torch.zeros(4, dtype=torch.int32), torch.eye(4), torch.eye(3)
    h = torch.zeros(16, 2, dtype=torch.int32)
    sp, pc, mk = torch.zeros(2, 2, 3), torch.zeros(2, 2, 8, dtype=torch.int32), torch.zeros(2, 2, dtype=torch.bool)
    return {
        "pts2plane": (lambda: ops.pts2plane(f, m4, K, 4, 4), "xyz"),
        "scatter_hashtable": (lambda: ops.scatter_hashtable(i, i, torch.zeros(4), 4, 4), "point_idx"),
        "quick_sampling": (lambda: ops.quick_sampling(f, m4, 1., 1., 2., 2., 4, 4, opt, i, h), "xyz"),
        "quick_query": (lambda: ops.quick_query(f, m4, 1., 1., 2., 2., 4, 4, opt, i, h, i), "xyz"),
        "scatter_multibin": (lambda: ops.scatter_multibin(i, i, torch.zeros(4), 4, 4, 5), "point_idx"),
        "ray_directions": (lambda: ops.ray_directions(m4, 1., 1., 2., 2., 4, 4), "c2w"),
        "mask_scan": (lambda: ops.mask_scan(torch.zeros(4, dtype=torch.bool)), "mask"),
        "feature_query": (lambda: ops.feature_query(f, f, f, torch.zeros(4, 32), sp, pc, mk, m4, 1., 1., 2., 2., 2), "xyz"),
        "clamp_t": (lambda: ops.clamp_t(torch.zeros(2, 8)), "t_val"),
        "render": (lambda: ops.render(torch.zeros(2, 8), torch.zeros(2, 8), torch.zeros(2, 8, 3)), "sigmas"),
        "aggregator_pack": (lambda: ops.aggregator_pack([torch.zeros(o, k) for _, o, k in ops.AGG_LAYERS],
                                                        [torch.zeros(o) for _, o, _ in ops.AGG_LAYERS]), "block1.0"),
        "_C.scatter": (lambda: E._C.scatter(i, i, torch.zeros(4), [4, 4], 5), "point_idx"),
        "_C.scatter_hashtable": (lambda: E._C.scatter_hashtable(i, i, torch.zeros(4), (4, 4), False), "point_idx"),
    }


@pytest.mark.parametrize("name", sorted(_cpu_calls()))
def test_entry_points_reject_host_tensors(name):
    """Like the reference's TORCH_CHECKs: a tensor argument in host memory is a RuntimeError that names
    it, raised before any device work (there is no CPU fallback)."""
    call, arg = _cpu_calls()[name]
    with pytest.raises(RuntimeError, match=arg) as e:
        call()
    assert "CUDA" in str(e.value)
