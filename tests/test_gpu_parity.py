"""GPU parity: the CUDA path through the C ABI against the reference's golden
outputs (bit-exact), against the CPU oracle on seeded cases, and against
size-independent properties at the full workload sizes.

Tolerances: integer outputs (pixel ids, hash tables, masks, point ids) are
compared exactly.  Float outputs are compared bit for bit against the
reference's own CUDA outputs; against the oracle fed the library's ray
directions they are bit-exact too, and rays whose decisions the oracle flags
as within rounding of a threshold (CUDA's norm3df / __expf vs the oracle's
correctly rounded stand-ins) may differ, bounded in number.
"""
import numpy as np
import pytest
import torch

import oracle as O
from hashpoint import native, ops, synth
from hp_testutil import Golden, bits, golden_names, ray_mismatch

pytestmark = pytest.mark.gpu
NAMES = golden_names()


@pytest.fixture(scope="module", autouse=True)
def _setup():
    native.build()
    O.build()


def D(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def H(t):
    return t.cpu().numpy()


# ---------------------------------------------------------------------------
# golden fixtures (outputs of the reference's CUDA extension on a B200)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", NAMES)
def test_pts2plane_bit_exact_vs_reference(name):
    g = Golden(name)
    sidx, sdep, hsh = ops.pts2plane(D(g["xyz"]), D(g["w2c"]), D(g["K"]), g.H, g.W, g.sort)
    assert np.array_equal(H(hsh), g["hash_table"])
    assert np.array_equal(H(sidx), g["sorted_point_idx"])
    assert np.array_equal(bits(H(sdep)), bits(g["sorted_depth"]))


@pytest.mark.parametrize("name", NAMES)
def test_quick_sampling_bit_exact_vs_reference(name):
    g = Golden(name)
    sp_xyz, pc_idx, sp_t, mask = ops.quick_sampling(D(g["xyz"]), D(g["c2w"]), g.fx, g.fy, g.cx, g.cy, g.W, g.H,
                                                    g.opt, D(g["sorted_point_idx"]), D(g["hash_table"]))
    assert mask.dtype == torch.bool
    assert np.array_equal(H(mask), g["mask"])
    assert np.array_equal(H(pc_idx), g["pc_idx"])
    assert np.array_equal(bits(H(sp_t)), bits(g["sp_t"]))
    assert np.array_equal(bits(H(sp_xyz)), bits(g["sp_xyz"]))


@pytest.mark.parametrize("stage", native.STAGE_CONFIGS)
def test_every_stage_config_bit_exact_vs_reference(stage):
    """Each stage configuration of the sampling kernel (staged points per tile, blocks per SM)
    reproduces every golden fixture; the tuning changes speed only."""
    for name in NAMES:
        g = Golden(name)
        for heavy in (0, 1, 4096):  # default, every ray warp-served, none
            t = ops.make_tuning(heavy_window=heavy, stage_config=stage)
            sp_xyz, pc_idx, sp_t, mask = ops.quick_sampling(D(g["xyz"]), D(g["c2w"]), g.fx, g.fy, g.cx, g.cy, g.W,
                                                            g.H, g.opt, D(g["sorted_point_idx"]),
                                                            D(g["hash_table"]), tuning=t)
            assert np.array_equal(H(mask), g["mask"]), (name, heavy)
            assert np.array_equal(H(pc_idx), g["pc_idx"]), (name, heavy)
            assert np.array_equal(bits(H(sp_t)), bits(g["sp_t"])), (name, heavy)
            assert np.array_equal(bits(H(sp_xyz)), bits(g["sp_xyz"])), (name, heavy)


@pytest.mark.parametrize("name", NAMES)
def test_scatter_hashtable_bit_exact_vs_reference(name):
    g = Golden(name)
    perm = g["perm"].astype(np.int64)
    pid_s = g["point2img"][perm]
    sidx, sdep, hsh = ops.scatter_hashtable(D(perm.astype(np.int32)), D(pid_s), D(g["depth"][perm]), g.H, g.W,
                                            g.sort)
    assert np.array_equal(H(hsh), g["hash_table"])
    assert np.array_equal(H(sidx), g["sorted_point_idx"])
    assert np.array_equal(bits(H(sdep)), bits(g["sorted_depth"]))


@pytest.mark.parametrize("name", [n for n in NAMES if "query" in n or "dense" in n])
def test_quick_query_vs_reference(name):
    g = Golden(name)
    for k in g.g.files:
        if not k.startswith("query_out_"):
            continue
        cap = int(k.split("_")[-1])
        g.opt.num_point_per_ray = cap
        out = H(ops.quick_query(D(g["xyz"]), D(g["c2w"]), g.fx, g.fy, g.cx, g.cy, g.W, g.H, g.opt,
                                D(g["sorted_point_idx"]), D(g["hash_table"]), D(g["query_rays"])))
        assert np.array_equal((out >= 0).sum(1), g["query_count_%d" % cap])
        if cap >= 256:
            assert np.array_equal(np.sort(out, 1), g[k])
        # deterministic order: identical to the oracle's window-cell / bucket order
        ref, cnt, _ = O.quick_query(g["xyz"], g.ora_camera(), g.opt, g["sorted_point_idx"], g["hash_table"],
                                    g["query_rays"], dirs=H(ops.ray_directions(D(g["c2w"]), g.fx, g.fy, g.cx, g.cy,
                                                                                g.W, g.H)))
        assert np.array_equal(out, ref)


@pytest.mark.parametrize("name", [n for n in NAMES if "sphere_64" in n or "shapes_96" in n or "dense" in n])
def test_scatter_multibin_vs_reference(name):
    g = Golden(name)
    perm = g["perm"].astype(np.int64)
    for k in g.g.files:
        if k.startswith("scatter_idx_"):
            bins = int(k.split("_")[-1])
            bd, bi = ops.scatter_multibin(D(perm.astype(np.int32)), D(g["point2img"][perm]), D(g["depth"][perm]),
                                          g.H, g.W, bins)
            assert np.array_equal(H(bi), g[k])
            assert np.array_equal(bits(H(bd)), bits(g["scatter_depth_%d" % bins]))


# ---------------------------------------------------------------------------
# projection rounding at the switch points of the reference's cuBLAS GEMMs
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", list(range(1, 17)) + [1535, 1536, 1537, 1538, 233022, 233023, 233024, 233025])
def test_projection_vs_reference_torch(n):
    """Pixel ids and depths of hp_pts2plane against the reference's own torch projection
    (epcq.py:251-274, run here with this machine's torch and cuBLAS) at point counts that bracket
    the GEMM-rounding switch points of hp_projection_rounding.  Depths are compared bit for bit:
    a wrong rounding form changes most of them by an ulp.  N = 1 (a 3x3 by 3x1 product) matched
    neither rounding form when the switch points were measured, so there only pixel ids must
    agree and depths within 1 ulp."""
    from ref_pipeline import RefPipeline
    rng = np.random.default_rng(1000 + n)
    cam = synth.look_at_camera((0.3, -0.2, 4.0), (0, 0, 0), 64, 48, 70.0)
    xyz = (rng.standard_normal((n, 3)) * 0.5).astype(np.float32)
    X, w2c, K = D(xyz), D(cam.w2c), D(cam.K)
    pid, depth, _, _, _ = RefPipeline(None, X.device).project(X, w2c, K, cam.height, cam.width)
    pid_h, dep_h = H(pid).astype(np.int32), H(depth).astype(np.float32)
    perm = np.argsort(pid_h, kind="stable").astype(np.int32)
    r_sidx, r_sdep, r_hsh = O.scatter_hashtable(perm, pid_h[perm], dep_h[perm], cam.height, cam.width, False)
    sidx, sdep, hsh = (H(t) for t in ops.pts2plane(X, w2c, K, cam.height, cam.width, False))
    assert np.array_equal(hsh, r_hsh) and np.array_equal(sidx, r_sidx)
    if n == 1:
        assert np.all(np.abs(bits(sdep).astype(np.int64) - bits(r_sdep).astype(np.int64)) <= 1)
    else:
        assert np.array_equal(bits(sdep), bits(r_sdep))


# ---------------------------------------------------------------------------
# seeded cases against the oracle
# ---------------------------------------------------------------------------
def _case(kind, seed, n, W, Hh, f, k, r, S=8, P=8, t_intvl=0.01, sort=False, **kw):
    rng = np.random.default_rng(seed)
    if kind == "sphere":
        xyz = synth.sphere_cloud(rng, n)
        cam = synth.look_at_camera((0, 0, 4), (0, 0, 0), W, Hh, f)
    elif kind == "shapes":
        xyz = synth.shapes_cloud(rng, n)
        cam = synth.orbit_cameras(rng, 1, 4.0, W, Hh, f)[0]
    else:
        xyz = synth.clusters_cloud(rng, n)
        cam = synth.orbit_cameras(rng, 1, None, W, Hh, f, elev_deg=(30, 70), radius_range=(2.5, 3.5))[0]
    opt = synth.Options(kernel_size=k, radius_threshold=r, num_sample_points_per_ray=S, num_point_cloud_per_sp=P,
                        t_intvl=t_intvl, **kw)
    return xyz, cam, opt, sort


CASES = {
    "sphere_200x160_k3": ("sphere", 1, 60000, 200, 160, 280.0, 3, 0.012),
    "shapes_256_k5_sorted": ("shapes", 2, 200000, 256, 256, 360.0, 5, 0.01, 8, 8, 0.01, True),
    "clusters_192x160_k5_S16": ("clusters", 3, 200000, 192, 160, 350.0, 5, 0.006, 16, 8, 0.01),
    "shapes_128_k4_P4": ("shapes", 4, 80000, 128, 128, 180.0, 4, 0.02, 8, 4),
    "shapes_128_k2_P12_S3": ("shapes", 5, 80000, 128, 128, 180.0, 2, 0.02, 3, 12),
    "sphere_97x61_k1_soft": ("sphere", 6, 30000, 97, 61, 120.0, 1, 0.03, 8, 8, 0.01, False),
}


def _run_case(xyz, cam, opt, sort):
    c2w, w2c, K = D(cam.c2w), D(cam.w2c), D(cam.K)
    sidx, sdep, hsh = ops.pts2plane(D(xyz), w2c, K, cam.height, cam.width, sort)
    outs = ops.quick_sampling(D(xyz), c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height, opt, sidx, hsh)
    dirs = ops.ray_directions(c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height)
    return (H(sidx), H(sdep), H(hsh)), [H(o) for o in outs], H(dirs)


@pytest.mark.parametrize("case", sorted(CASES))
def test_vs_oracle(case):
    args = CASES[case]
    xyz, cam, opt, sort = _case(*args)
    (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), dirs = _run_case(xyz, cam, opt, sort)
    ocam = O.camera_from(cam)
    oi, od, oh = O.pts2plane(xyz, ocam, sort)
    assert np.array_equal(hsh, oh)
    assert np.array_equal(sidx, oi)
    assert np.array_equal(bits(sdep), bits(od))
    r_xyz, r_idx, r_t, r_mask, margin = O.quick_sampling(xyz, ocam, opt, sidx, hsh, dirs=dirs, nthreads=8)
    Hh, W = cam.height, cam.width
    bad = ray_mismatch(mask, pc_idx, r_mask, r_idx, Hh, W)
    assert np.all(margin[bad] < 1e-6), margin[bad][:8]
    assert np.count_nonzero(bad) <= max(2, Hh * W // 20000)
    ok = ~bad.reshape(Hh, W)
    assert np.array_equal(bits(sp_t[ok]), bits(r_t[ok]))
    assert np.array_equal(bits(sp_xyz[ok]), bits(r_xyz[ok]))
    assert mask.sum() > 0


def test_edge_cases():
    rng = np.random.default_rng(9)
    opt = synth.Options(kernel_size=3, radius_threshold=0.05, num_sample_points_per_ray=4, num_point_cloud_per_sp=8)
    # every point projects to the same pixel (8, 6): one bucket of 6000 (deep, sorted in global memory)
    cam = synth.look_at_camera((0, 0, 4), (0, 0, 0), 16, 12, 0.5, 0.5, 8.5, 6.5)
    xyz = (rng.normal(size=(6000, 3)) * 0.2).astype(np.float32)
    for sort in (False, True):
        (sidx, sdep, hsh), outs, dirs = _run_case(xyz, cam, opt, sort)
        oi, od, oh = O.pts2plane(xyz, O.camera_from(cam), sort)
        assert np.array_equal(hsh, oh) and np.array_equal(sidx, oi) and np.array_equal(bits(sdep), bits(od))
        assert hsh[:, 1].max() == 6000
    # three buckets above 2048 entries (k_sort_huge_list: the CTAs share the scan's list)
    cam3 = synth.look_at_camera((0, 0, 4), (0, 0, 0), 16, 12, 50.0, 50.0, 8.5, 6.5)
    xyz3 = np.concatenate([rng.normal(size=(3000, 3)) * 0.001 + np.array([dx, 0.0, 0.0])
                           for dx in (-0.16, 0.0, 0.16)]).astype(np.float32)
    for sort in (False, True):
        (sidx, sdep, hsh), _, _ = _run_case(xyz3, cam3, opt, sort)
        oi, od, oh = O.pts2plane(xyz3, O.camera_from(cam3), sort)
        assert np.array_equal(hsh, oh) and np.array_equal(sidx, oi) and np.array_equal(bits(sdep), bits(od))
        assert (hsh[:, 1] > 2048).sum() == 3
    # empty cloud
    (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), _ = _run_case(np.zeros((0, 3), np.float32), cam, opt, False)
    assert sidx.size == 0 and np.all(hsh == -1) and not mask.any() and np.all(pc_idx == -1) and np.all(sp_t == 0)
    # all points off-image (beside the camera's field of view): -1 everywhere
    far = np.tile(np.array([[100.0, 0.0, 0.0]], np.float32), (500, 1))
    (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), _ = _run_case(far, cam, opt, False)
    assert np.all(sidx == -1) and np.all(sdep == -1) and np.all(hsh == -1) and not mask.any()
    # 1x1, 1xW and Hx1 images
    for W, Hh in ((1, 1), (37, 1), (1, 29)):
        cam2 = synth.look_at_camera((0, 0, 4), (0, 0, 0), W, Hh, 40.0)
        xyz2 = synth.sphere_cloud(rng, 3000)
        (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), dirs = _run_case(xyz2, cam2, opt, False)
        oc = O.camera_from(cam2)
        oi, od, oh = O.pts2plane(xyz2, oc, False)
        assert np.array_equal(hsh, oh) and np.array_equal(sidx, oi)
        r = O.quick_sampling(xyz2, oc, opt, sidx, hsh, dirs=dirs)
        assert np.array_equal(mask, r[3]) and np.array_equal(pc_idx, r[1])


def test_more_huge_buckets_than_ctas():
    """170 buckets of 2100+ entries: more than the 148 CTAs that order the buckets above 2048
    entries, so each CTA takes several from the list the scan writes; both bucket orders, and
    hp_scatter_hashtable's depth order over the same runs (it finds them by scanning)."""
    rng = np.random.default_rng(21)
    W, Hh, f = 20, 10, 40.0
    cam = synth.look_at_camera((0, 0, 4), (0, 0, 0), W, Hh, f)
    c2w, K = cam.c2w.astype(np.float64), cam.K.astype(np.float64)
    pix = rng.choice(W * Hh, size=170, replace=False)
    pts = []
    for p in pix:
        u, v = p % W + 0.25, p // W + 0.25          # inside pixel (p % W, p // W) under floor and round alike
        d = rng.uniform(2.0, 6.0, size=2100 + int(rng.integers(0, 60)))
        ray = np.linalg.solve(K, np.array([u, v, 1.0]))
        cam_pts = d[:, None] * ray[None, :]
        pts.append(cam_pts @ c2w[:3, :3].T + c2w[:3, 3])
    xyz = np.concatenate(pts)[rng.permutation(sum(len(q) for q in pts))].astype(np.float32)
    oc = O.camera_from(cam)
    for sort in (False, True):
        sidx, sdep, hsh = (H(t) for t in ops.pts2plane(D(xyz), D(cam.w2c), D(cam.K), Hh, W, sort))
        oi, od, oh = O.pts2plane(xyz, oc, sort)
        assert (oh[:, 1] > 2048).sum() == 170
        assert np.array_equal(hsh, oh) and np.array_equal(sidx, oi) and np.array_equal(bits(sdep), bits(od))
    # runs already grouped by pixel (the stable order), then depth-sorted inside each run
    oi, od, oh = O.pts2plane(xyz, oc, False)
    pid = np.repeat(np.arange(W * Hh, dtype=np.int32), np.maximum(oh[:, 1], 0))
    s_idx, s_dep, s_h = (H(t) for t in ops.scatter_hashtable(D(oi), D(pid), D(od), Hh, W, True))
    r_idx, r_dep, r_h = O.scatter_hashtable(oi, pid, od, Hh, W, True)
    assert np.array_equal(s_h, r_h) and np.array_equal(s_idx, r_idx) and np.array_equal(bits(s_dep), bits(r_dep))


def test_epcq_camera_scalars_on_the_device():
    """Through the drop-in epcq API, a camera whose fx..cy are 0-d CUDA tensors taken from K and
    whose size is a CUDA tensor (as the reference's renderer builds it) gives the same outputs, bit
    for bit, as the same camera with Python numbers."""
    from epcq import epcq as E
    rng = np.random.default_rng(31)
    xyz = synth.shapes_cloud(rng, 20000)
    cam = synth.orbit_cameras(rng, 1, 4.0, 96, 80, 120.0)[0]
    K = D(cam.K)
    model = E.NeuralPoints(pc_type="pc", points=D(xyz))
    opt = E.RenderOptions(kernel_size=5, radius_threshold=0.05, num_sample_points_per_ray=8, num_point_cloud_per_sp=8)
    fx, fy, cx, cy = E.CameraSpec.decomposeK(K)
    hw = torch.tensor([cam.height, cam.width], device="cuda")
    cams = [E.CameraSpec(c2w=D(cam.c2w), w2c=D(cam.w2c), K=K, fx=cam.fx, fy=cam.fy, cx=cam.cx, cy=cam.cy,
                         width=cam.width, height=cam.height),
            E.CameraSpec(c2w=D(cam.c2w), w2c=D(cam.w2c), K=K, fx=fx, fy=fy, cx=cx, cy=cy, height=hw[0], width=hw[1])]
    outs = []
    for c in cams:
        idx, dep, hsh = model.pts2plane(c, opt)
        outs.append([H(t) for t in (idx, dep, hsh) + tuple(model.render_image_hashtable_topk(c, opt, idx, dep, hsh))])
    for a, b in zip(*outs):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert outs[0][-1].any()


def test_scan_wait_gives_up_and_reports():
    """The hash-table scan's waits are bounded: with one scan block withheld (test library), the
    blocks after it give up, hp_pts2plane_status reports it, and the next plain call on the same
    workspace and context is correct again and reports nothing."""
    import ctypes
    native.build_testing()
    T, L = native.testing_lib(), native.lib()
    rng = np.random.default_rng(41)
    xyz = synth.shapes_cloud(rng, 20000)
    cam = synth.orbit_cameras(rng, 1, 4.0, 160, 128, 180.0)[0]  # 20480 pixels: five 4096-pixel scan blocks
    n, Hh, W = len(xyz), cam.height, cam.width
    X, w2c, K = D(xyz), D(cam.w2c), D(cam.K)  # kept alive: the camera struct holds their device pointers
    hc = ops.make_camera(w2c=w2c, K=K, width=W, height=Hh)
    ws_bytes = L.hp_pts2plane_workspace_size(n, Hh, W)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    sidx = torch.empty(n, dtype=torch.int32, device="cuda")
    sdep = torch.empty(n, dtype=torch.float32, device="cuda")
    hsh = torch.empty((Hh * W, 2), dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptrs = [ctypes.c_void_p(t.data_ptr()) for t in (sidx, sdep, hsh, ws)]
    rc = T.hp_pts2plane_withheld(ctypes.c_void_p(X.data_ptr()), n, ctypes.byref(hc), 0, *ptrs, ws_bytes, 0, stream)
    native.check(rc, "hp_pts2plane_withheld", T)
    assert T.hp_pts2plane_status(ptrs[3], n, Hh, W, stream) != 0
    assert "gave up" in T.hp_last_error().decode()
    rc = L.hp_pts2plane(ctypes.c_void_p(X.data_ptr()), n, ctypes.byref(hc), 0, *ptrs, ws_bytes, stream)
    native.check(rc, "hp_pts2plane")
    native.check(L.hp_pts2plane_status(ptrs[3], n, Hh, W, stream), "hp_pts2plane_status")
    oi, od, oh = O.pts2plane(xyz, O.camera_from(cam), False)
    assert np.array_equal(H(hsh), oh) and np.array_equal(H(sidx), oi) and np.array_equal(bits(H(sdep)), bits(od))


def test_repeatable():
    xyz, cam, opt, sort = _case(*CASES["clusters_192x160_k5_S16"])
    a = _run_case(xyz, cam, opt, sort)
    b = _run_case(xyz, cam, opt, sort)
    for x, y in zip(a[0] + tuple(a[1]), b[0] + tuple(b[1])):
        assert np.array_equal(x, y)


# ---------------------------------------------------------------------------
# full-size workloads: properties plus an oracle check on sampled rays
# ---------------------------------------------------------------------------
def _full(name):
    if name == "sphere":
        sc = synth.make_sphere()
    elif name == "shapes":
        sc = synth.make_shapes(n_views=1, with_feat=False)
    else:
        sc = synth.make_clusters(n_views=1)
    return sc.xyz, sc.cameras[0], sc.options


@pytest.mark.parametrize("name", ["shapes", "clusters"])
def test_full_size_every_stage_config_identical(name):
    """At full size every stage configuration gives the default's outputs bit for bit (the
    configurations split and stage different work items, so they take different code paths)."""
    xyz, cam, opt = _full(name)
    X, c2w, w2c, K = D(xyz), D(cam.c2w), D(cam.w2c), D(cam.K)
    sidx, _, hsh = ops.pts2plane(X, w2c, K, cam.height, cam.width, False)
    run = lambda t: [H(o) for o in ops.quick_sampling(X, c2w, cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height,
                                                      opt, sidx, hsh, tuning=t)]
    base = run(None)
    for stage in native.STAGE_CONFIGS:
        for a, b in zip(run(ops.make_tuning(stage_config=stage)), base):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), stage


@pytest.mark.parametrize("name", ["sphere", "shapes", "clusters"])
def test_full_size(name):
    xyz, cam, opt = _full(name)
    Hh, W = cam.height, cam.width
    (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), dirs = _run_case(xyz, cam, opt, False)
    ocam = O.camera_from(cam)
    # projection + hash table: exact against the oracle
    oi, od, oh = O.pts2plane(xyz, ocam, False)
    assert np.array_equal(hsh, oh) and np.array_equal(sidx, oi) and np.array_equal(bits(sdep), bits(od))
    # hash invariants
    occ = hsh[:, 1] > 0
    n_in = int(hsh[occ, 1].sum())
    assert np.all(sidx[n_in:] == -1) and np.all(sidx[:n_in] >= 0)
    assert np.array_equal(np.sort(sidx[:n_in]), np.unique(sidx[:n_in]))
    starts = hsh[occ, 0]
    assert np.all(np.diff(starts) > 0) and starts[0] == 0
    # mask is a prefix per ray; unused slots hold defaults
    m = mask.reshape(Hh * W, -1)
    assert np.all(m[:, 1:] <= m[:, :-1])
    assert np.all(sp_t[~mask] == 0) and np.all(pc_idx[~mask] == -1)
    # sampled rays against the oracle
    rng = np.random.default_rng(0)
    rays = rng.choice(Hh * W, size=4000, replace=False).astype(np.int32)
    r_xyz, r_idx, r_t, r_mask, margin = O.quick_sampling(xyz, ocam, opt, sidx, hsh, dirs=dirs, rays=rays, nthreads=8)
    vv, uu = rays // W, rays % W
    bad = ~(np.all(mask[vv, uu] == r_mask, 1) & np.all(pc_idx[vv, uu].reshape(len(rays), -1) ==
                                                          r_idx.reshape(len(rays), -1), 1))
    assert np.all(margin[bad] < 1e-6)
    assert np.count_nonzero(bad) <= 4
    ok = ~bad
    assert np.array_equal(bits(sp_t[vv, uu][ok]), bits(r_t[ok]))
    # selected ids are within the radius of their sample (float64 check, small slack)
    sel = pc_idx[vv, uu]
    samp = sp_xyz[vv, uu]
    ii = np.nonzero(sel >= 0)
    d = np.linalg.norm(xyz[sel[ii]].astype(np.float64) - samp[ii[0], ii[1]].astype(np.float64), axis=-1)
    assert np.all(d < opt.radius_threshold * (1 + 1e-5))


@pytest.mark.parametrize("name", ["sphere", "shapes", "clusters"])
def test_fp64_error_statement(name):
    """The FP32 path's error against the FP64 oracle on 4000 sampled rays of a full-size view
    (oracle/error_stats.py): camera depths and sample depths within 1e-6 relative, sample
    positions within 1e-5 relative at the 99th percentile, ray distances within 1e-3 of the
    radius, and rays whose discrete choices differ from FP64 under 1%."""
    import error_stats
    xyz, cam, opt = _full(name)
    (sidx, sdep, hsh), (sp_xyz, pc_idx, sp_t, mask), dirs = _run_case(xyz, cam, opt, False)
    st = error_stats.fp64_error(xyz, cam, opt, sidx, sdep, hsh, sp_xyz, sp_t, mask, pc_idx, dirs)
    assert st["depth_rel"]["max"] <= 1e-6, st["depth_rel"]
    assert st["t_rel"]["n"] > 500 and st["t_rel"]["max"] <= 1e-6, st["t_rel"]
    assert st["xyz_rel"]["p99"] <= 1e-5, st["xyz_rel"]
    assert st["ray_dist_abs_over_radius"]["max"] <= 1e-3, st["ray_dist_abs_over_radius"]
    flips = st["decision_flips"]
    assert flips["rays_with_other_slots"] + flips["samples_moved"] <= 0.01 * st["rays"], flips


# ---------------------------------------------------------------------------
# the reference's own CUDA build (present when oracle/_ref travels with the repo)
# ---------------------------------------------------------------------------
def _ref_module():
    import os
    import build_ref
    if not os.path.exists(build_ref.SO_PATH):
        pytest.skip("reference build oracle/_ref not present")
    return build_ref.load()


def _mixed_view_1600():
    """A 1600x1200 view of the uneven multi-cloud workload (its largest resolution), on its cloud."""
    mb = synth.make_mixed(n_clouds=8, n_views=64, seed=0)
    ci, cam = next((c, v) for c, v in mb.views if v.width == 1600)
    return mb.clouds[ci], cam, mb.options


@pytest.mark.parametrize("name", ["sphere", "shapes", "clusters", "mixed_1600x1200"])
def test_full_size_vs_reference_cuda(name):
    """Whole pipeline vs the reference's CUDA extension driven as epcq.py drives it (P = 8): the
    100k-point sphere, the 1M-point shapes view, the 3M-point clusters view at 1600x1200 with
    K = 16 (deep buckets, the 48-per-cell cap, warp-served and unstaged work), and a 1600x1200
    view of the uneven multi-cloud workload."""
    from ref_pipeline import RefPipeline
    mod = _ref_module()
    xyz, cam, opt = _mixed_view_1600() if name == "mixed_1600x1200" else _full(name)
    rp = RefPipeline(mod, torch.device("cuda:0"))
    X = D(xyz)
    c2w, w2c, K = D(cam.c2w), D(cam.w2c), D(cam.K)
    pid, depth, _, _, _ = rp.project(X, w2c, K, cam.height, cam.width)
    pid_s, perm, depth_s, idx_s = rp.sort(pid, depth)
    r_sidx, r_sdep, r_hsh = rp.scatter_hashtable(idx_s, pid_s, depth_s, cam.height, cam.width, False)
    npspec = mod.NeuralPointsSpec()
    npspec.xyz_data = X
    r_out = mod.quick_sampling(npspec, rp.camera_spec(c2w, w2c, cam), rp.options_spec(opt), r_sidx, r_hsh)
    (sidx, sdep, hsh), outs, _ = _run_case(xyz, cam, opt, False)
    assert np.array_equal(hsh, H(r_hsh)) and np.array_equal(sidx, H(r_sidx))
    assert np.array_equal(bits(sdep), bits(H(r_sdep)))
    names = ["sp_xyz", "pc_idx", "sp_t", "mask"]
    for nm, a, b in zip(names, outs, r_out):
        b = H(b)
        if a.dtype == np.float32:
            assert np.array_equal(bits(a), bits(b)), nm
        else:
            assert np.array_equal(a, b), nm


def _pixel_rays64(cam, u, v):
    """FP64 pixel-centre rays (origin, unit direction) of the sampling path's definition."""
    c2w = np.asarray(cam.c2w, np.float64)
    d = np.stack([(u + 0.5 - cam.cx) / cam.fx, (v + 0.5 - cam.cy) / cam.fy, np.ones_like(u, np.float64)], -1)
    d = d @ c2w[:3, :3].T
    return c2w[:3, 3], d / np.linalg.norm(d, axis=-1, keepdims=True)


def _ray_dist64(xyz, o, d):
    e = xyz.astype(np.float64) - o
    return np.linalg.norm(e - (e @ d)[:, None] * d, axis=-1)


@pytest.mark.parametrize("name", ["sphere", "shapes", "clusters"])
def test_quick_query_sets_vs_brute_force(name):
    """The listed-ray query at full size against a brute-force FP64 search of each ray's window
    cells: every returned id lies within the radius of its pixel-centre ray (up to 2e-4 of the
    radius, the FP32 rounding of the ray and the distance), and every window point more than 2e-4
    of the radius inside it is returned -- unless the ray's row or one of its cells reached its cap
    (num_point_per_ray, 32 per cell).  Rays whose windows touch the image border (clamped, so
    repeated, cells) are left out."""
    xyz, cam, opt = _full(name)
    W, Hh, k = cam.width, cam.height, opt.kernel_size
    lo = (k + 1) // 2 - 1
    X = D(xyz)
    sidx, _, hsh = ops.pts2plane(X, D(cam.w2c), D(cam.K), Hh, W, False)
    rng = np.random.default_rng(11)
    u = rng.integers(lo, W - (k - 1 - lo), 2048)
    v = rng.integers(lo, Hh - (k - 1 - lo), 2048)
    rays = (v * W + u).astype(np.int32)
    out = H(ops.quick_query(X, D(cam.c2w), cam.fx, cam.fy, cam.cx, cam.cy, W, Hh, opt, sidx, hsh, D(rays)))
    si, hs = H(sidx), H(hsh).reshape(-1, 2)
    o, d = _pixel_rays64(cam, u.astype(np.float64), v.astype(np.float64))
    r, cap, tol = float(opt.radius_threshold), int(opt.num_point_per_ray), 2e-4
    checked = found = 0
    for i in range(len(rays)):
        ids, full_cell = [], False
        for dv in range(-lo, k - lo):
            for du in range(-lo, k - lo):
                s, c = hs[(v[i] + dv) * W + u[i] + du]
                if s < 0 or c <= 0:
                    continue
                cell = si[s:s + c]
                near = _ray_dist64(xyz[cell], o, d[i]) < r * (1 + tol)
                full_cell |= int(near.sum()) >= 32
                ids.append(cell)
        ids = np.concatenate(ids) if ids else np.zeros(0, np.int32)
        dist = _ray_dist64(xyz[ids], o, d[i]) if len(ids) else np.zeros(0)
        got = out[i][out[i] >= 0]
        assert len(np.unique(got)) == len(got), i  # no repeated cell, so no repeated id
        assert set(got.tolist()) <= set(ids[dist < r * (1 + tol)].tolist()), i
        if len(got) < cap and not full_cell:
            sure = set(ids[dist < r * (1 - tol)].tolist())
            assert sure <= set(got.tolist()), i
            checked += 1
            found += len(sure)
    assert checked > len(rays) // 2 and found > 0


@pytest.mark.parametrize("name", ["sphere", "shapes", "clusters"])
def test_sample_points_within_radius(name):
    """Per-sample point selection at full size: every id chosen for an emitted sample lies within
    the radius of that sample point (FP64 distance, up to 2e-4 of the radius), an emitted sample's
    ids fill its first slots, and samples that were not emitted carry -1 everywhere."""
    xyz, cam, opt = _full(name)
    X = D(xyz)
    sidx, _, hsh = ops.pts2plane(X, D(cam.w2c), D(cam.K), cam.height, cam.width, False)
    sp_xyz, pc_idx, sp_t, mask = (H(t) for t in ops.quick_sampling(
        X, D(cam.c2w), cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height, opt, sidx, hsh))
    P = pc_idx.shape[-1]
    m = mask.reshape(-1).astype(bool)
    idx = pc_idx.reshape(-1, P)
    assert (idx[~m] == -1).all()
    ids, sp = idx[m], sp_xyz.reshape(-1, 3)[m].astype(np.float64)
    valid = ids >= 0
    # -1 only after the last chosen id of a sample
    assert not (~valid[:, :-1] & valid[:, 1:]).any()
    rows, cols = np.nonzero(valid)
    dist = np.linalg.norm(xyz[ids[rows, cols]].astype(np.float64) - sp[rows], axis=-1)
    assert len(dist) > 0 and (dist < float(opt.radius_threshold) * (1 + 2e-4)).all()
