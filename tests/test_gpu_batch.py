"""Batched search+sample (hp_quick_sampling_batch, hashpoint.batch) against the
per-view launch and the reference's golden outputs.

Every view of a batch must come out bit-identical to the same view launched
alone: the golden fixtures (reference CUDA outputs, mixed options and sizes)
as one batch, a mixed multi-cloud batch against per-view launches, the device
view table and a CUDA graph replay, and every launch tuning.
"""
import numpy as np
import pytest
import torch

from hashpoint import batch, native, ops, synth
from hp_testutil import Golden, bits, golden_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _setup():
    native.build()


def D(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def H(t):
    return t.cpu().numpy()


def _same(a, b):
    """Bit-identical quick_sampling outputs."""
    for x, y in zip(a, b):
        x, y = H(x), H(y)
        if x.dtype == np.float32:
            assert np.array_equal(bits(x), bits(y))
        else:
            assert np.array_equal(x, y)


def test_golden_views_as_one_batch():
    keep, views, outs = [], [], []
    for name in golden_names():
        g = Golden(name)
        t = dict(xyz=D(g["xyz"]), c2w=D(g["c2w"]), sidx=D(g["sorted_point_idx"]), hash=D(g["hash_table"]))
        out = ops.sampling_outputs(g.H, g.W, g.opt, "cuda")
        views.append(ops.make_view(t["xyz"], t["c2w"], g.fx, g.fy, g.cx, g.cy, g.W, g.H, g.opt, t["sidx"], t["hash"],
                                   out))
        keep.append((t, g))
        outs.append(out)
    ops.quick_sampling_batch(views, "cuda")
    torch.cuda.synchronize()
    for (t, g), (sp_xyz, pc_idx, sp_t, mask) in zip(keep, outs):
        assert np.array_equal(H(mask), g["mask"]), g.name
        assert np.array_equal(H(pc_idx), g["pc_idx"]), g.name
        assert np.array_equal(bits(H(sp_t)), bits(g["sp_t"])), g.name
        assert np.array_equal(bits(H(sp_xyz)), bits(g["sp_xyz"])), g.name


def _mixed_renderer(seed=3, sort=False):
    mb = synth.make_mixed(n_clouds=4, n_views=10, seed=seed, size_range=(2e3, 3e5),
                          resolutions=((64, 64), (96, 80), (200, 150), (256, 256)))
    clouds = [D(c) for c in mb.clouds]
    return batch.BatchRenderer(clouds, mb.views, mb.options, "cuda", sort=sort), mb


@pytest.mark.parametrize("sort", [False, True])
def test_mixed_batch_matches_per_view(sort):
    r, mb = _mixed_renderer(sort=sort)
    r.run()
    torch.cuda.synchronize()
    emitted = 0
    for i, v in enumerate(r.views):
        xyz = r.clouds[v.cloud]
        sidx, sdep, hsh = ops.pts2plane(xyz, v.w2c, v.K, v.H, v.W, sort)
        b_sidx, b_sdep, b_hash = r.hash_table(i)
        assert torch.equal(sidx, b_sidx) and torch.equal(hsh, b_hash)
        ref = ops.quick_sampling(xyz, v.c2w, v.fx, v.fy, v.cx, v.cy, v.W, v.H, mb.options, sidx, hsh)
        _same(r.outputs(i), ref)
        emitted += int(ref[3].sum())
    assert emitted > 0


def test_graph_replay_and_device_table():
    r, _ = _mixed_renderer(seed=5)
    r.run()
    torch.cuda.synchronize()
    first = [tuple(t.clone() for t in r.outputs(i)) for i in range(len(r.views))]
    r.capture()
    for _ in range(2):
        for i in range(len(r.views)):
            for t in r.outputs(i):
                t.zero_()
        r.replay()
        torch.cuda.synchronize()
        for i in range(len(r.views)):
            _same(r.outputs(i), first[i])
    r.release()


def test_tuning_does_not_change_outputs():
    r, _ = _mixed_renderer(seed=7)
    r.run()
    torch.cuda.synchronize()
    first = [tuple(t.clone() for t in r.outputs(i)) for i in range(len(r.views))]
    cases = [(1, 0, 1), (64, 1, 2), (160, 2, 3), (320, 3, 4), (224, 0, 5), (4096, 0, 4), (1, 0, 5)]
    cases += [(320, 0, c) for c in native.STAGE_CONFIGS]
    for heavy, blocks, stage in cases:
        r.tuning = ops.make_tuning(heavy_window=heavy, blocks_per_sm=blocks, stage_config=stage)
        r.sample()
        torch.cuda.synchronize()
        for i in range(len(r.views)):
            _same(r.outputs(i), first[i])


def test_autotuner_caches_per_shape_class():
    r, _ = _mixed_renderer(seed=9)
    tuner = batch.Autotuner(reps=1)
    choice = tuner.tune(r)
    assert choice[0] in batch.Autotuner.STAGES and choice[1] in batch.Autotuner.HEAVY
    assert tuner.cache[tuner.key(r)] == choice
    assert tuner.tune(r) == choice
    assert (r.tuning.stage_config, r.tuning.heavy_window) == choice


def test_view_pipeline_tune_keeps_outputs():
    """ViewPipeline.tune picks one of the stage configurations and the per-view outputs stay the same."""
    from hashpoint.engine import CameraTable, ViewPipeline
    sc = synth.make_sphere(n=30000, width=160, height=120, f=220.0)
    X = torch.from_numpy(sc.xyz).cuda()
    cams = CameraTable(sc.cameras, "cuda")
    s = cams.struct(0)
    pipe = ViewPipeline(len(sc.xyz), 120, 160, sc.options, "cuda")
    before = [t.clone() for t in pipe.render(X, s)]
    cfg = pipe.tune(X, [s], reps=1)
    assert cfg in native.STAGE_CONFIGS and pipe.tuning.stage_config == cfg
    after = pipe.render(X, s)
    torch.cuda.synchronize()
    for a, b in zip(before, after):
        assert torch.equal(a.view(torch.uint8), b.view(torch.uint8))


def test_view_ring_matches_one_stream():
    """ViewRing (per-view launches over 3 streams, a buffer set each) gives every view the outputs
    of the same launches one after another on one stream; on_view sees each view's outputs before
    its buffers are reused."""
    from hashpoint.engine import CameraTable, ViewPipeline, ViewRing
    sc = synth.make_shapes(n=60000, n_views=7, width=160, height=128, f=220.0, with_feat=False)
    X = torch.from_numpy(sc.xyz).cuda()
    cams = CameraTable(sc.cameras, "cuda")
    structs = [cams.struct(i) for i in range(cams.n)]
    pipe = ViewPipeline(len(sc.xyz), 128, 160, sc.options, "cuda")
    ref = [[t.clone() for t in pipe.render(X, s)] for s in structs]
    ring = ViewRing(len(sc.xyz), 128, 160, sc.options, "cuda", depth=3)
    cfg = ring.tune(X, structs, reps=1)
    assert cfg in native.STAGE_CONFIGS and all(p.tuning.stage_config == cfg for p in ring.pipes)
    got = [None] * len(structs)

    def keep(i, p, stream):
        with torch.cuda.stream(stream):
            got[i] = [t.clone() for t in (p.sp_xyz, p.pc_idx, p.sp_t, p.mask)]

    main = torch.cuda.current_stream()
    ring.render_many(X, structs, main, on_view=keep)
    torch.cuda.synchronize()
    for a_view, b_view in zip(ref, got):
        for a, b in zip(a_view, b_view):
            assert torch.equal(a.view(torch.uint8), b.view(torch.uint8))
    assert any(bool(v[3].any()) for v in got)


def test_epcq_calls_over_streams_match_one_stream():
    """The drop-in epcq calls launch on torch's current stream and take their workspaces and
    outputs from torch's allocator, so a caller may deal views over several streams: every view's
    hash table and samples equal those of the same calls on one stream."""
    from epcq import epcq as E
    sc = synth.make_shapes(n=60000, n_views=7, width=160, height=128, f=220.0, with_feat=False)
    model = E.NeuralPoints(pc_type="pc", points=torch.from_numpy(sc.xyz).cuda())
    opt = E.RenderOptions(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8,
                          num_point_cloud_per_sp=8)
    cams = [E.CameraSpec(c2w=D(c.c2w), w2c=D(c.w2c), K=D(c.K), fx=c.fx, fy=c.fy, cx=c.cx, cy=c.cy,
                         width=c.width, height=c.height) for c in sc.cameras]

    def run(cam):
        idx, dep, hsh = model.pts2plane(cam, opt)
        return [idx, dep, hsh, *model.render_image_hashtable_topk(cam, opt, idx, dep, hsh)]

    ref = [run(c) for c in cams]
    torch.cuda.synchronize()
    main = torch.cuda.current_stream()
    side = [torch.cuda.Stream() for _ in range(3)]
    got = [None] * len(cams)
    for s in side:
        s.wait_stream(main)
    for i, c in enumerate(cams):
        with torch.cuda.stream(side[i % 3]):
            got[i] = run(c)
    for s in side:
        main.wait_stream(s)
    torch.cuda.synchronize()
    for a_view, b_view in zip(ref, got):
        for a, b in zip(a_view, b_view):
            assert torch.equal(a.view(torch.uint8), b.view(torch.uint8))
    assert any(bool(v[6].any()) for v in got)
