"""The C-ABI libraries load and export every symbol their headers declare:
include/hashpoint_b200.h (the product library) and include/hashpoint_b200_testing.h
(the test-only library).

No compute is launched here: argument validation runs on the host and returns
before any CUDA call, so these checks need no GPU.
"""
import ctypes
import os
import re

import pytest

from hashpoint import native

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADER = os.path.join(INCLUDE, "hashpoint_b200.h")
TESTING_HEADER = os.path.join(INCLUDE, "hashpoint_b200_testing.h")


def declared_symbols(header=HEADER):
    text = open(header).read()
    return sorted(set(re.findall(r"HP_API\s+[\w\s\*]+?\b(hp_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    native.build()
    return native.lib()


@pytest.fixture(scope="module")
def T():
    native.build_testing()
    return native.testing_lib()


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "hp_quick_sampling" in syms and "hp_pts2plane" in syms
    assert set(syms) == set(native.EXPORTS)
    assert set(declared_symbols(TESTING_HEADER)) == set(native.TESTING_EXPORTS)


def test_library_exports_every_declared_symbol(L):
    for s in declared_symbols():
        assert hasattr(L, s), s


def test_testing_library_exports_its_symbols_and_the_product_keeps_them_out(L, T):
    for s in declared_symbols(TESTING_HEADER):
        assert hasattr(T, s), s
        with pytest.raises(AttributeError):
            getattr(L, s)


def test_version(L):
    assert L.hp_version() >= 100


def test_projection_rounding_matches_oracle(L):
    import oracle
    oracle.build()
    for n in [0, 1, 2, 1536, 1537, 4099, 65536, 100000, 233023, 233024, 1_000_000, 3_000_000]:
        assert native.projection_rounding(n) == oracle.projection_rounding(n), n


def test_projection_rounding_switch_points(L):
    # measured on B200: cuBLAS fuses the w2c product from N=1537 and the K product from N=233024
    assert native.projection_rounding(1536) == (0, 0)
    assert native.projection_rounding(1537) == (1, 0)
    assert native.projection_rounding(233023) == (1, 0)
    assert native.projection_rounding(233024) == (1, 1)


def test_workspace_size(L):
    a = L.hp_pts2plane_workspace_size(1000, 10, 10)
    b = L.hp_pts2plane_workspace_size(2000, 10, 10)
    c = L.hp_pts2plane_workspace_size(1000, 100, 100)
    assert 0 < a < b and a < c
    assert L.hp_pts2plane_workspace_size(10, 0, 10) == 0
    assert L.hp_pts2plane_workspace_size(-1, 10, 10) == 0


def _cam(w=8, h=8, c2w=0x1000):
    cam = native.HpCamera()
    cam.c2w = c2w
    cam.w2c = c2w
    cam.K = c2w
    cam.fx = cam.fy = 10.0
    cam.cx = cam.cy = 4.0
    cam.width, cam.height = w, h
    return cam


def _opt(k=3, S=8, P=8, t=0.01):
    o = native.HpOptions()
    o.kernel_size, o.t_intvl, o.radius_threshold = k, t, 0.01
    o.num_sample_points_per_ray, o.num_point_cloud_per_sp, o.num_point_per_ray = S, P, 256
    o.sdf2weight_gaussian_alpha, o.sdf2weight_gaussian_gamma = 0.2, 0.9
    return o


def _err(L):
    return L.hp_last_error().decode()


@pytest.mark.parametrize("k,S,P,t,msg", [(0, 8, 8, 0.01, "kernel_size"), (6, 8, 8, 0.01, "kernel_size"),
                                         (3, 0, 8, 0.01, "num_sample_points_per_ray"),
                                         (3, 8, 0, 0.01, "num_point_cloud_per_sp"), (3, 8, 8, 0.0, "t_intvl")])
def test_quick_sampling_rejects_bad_options(L, k, S, P, t, msg):
    p = ctypes.c_void_p(0x1000)
    rc = L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt(k, S, P, t)), p, 10, p, p, p, p, p, p, 1 << 20,
                             None)
    assert rc == -1 and msg in _err(L)


def test_quick_sampling_rejects_null_and_misaligned(L):
    p = ctypes.c_void_p(0x1000)
    ws, big = ctypes.c_void_p(0x10000), 1 << 20
    assert L.hp_quick_sampling(p, 10, None, ctypes.byref(_opt()), p, 10, p, p, p, p, p, ws, big, None) == -1
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt()), p, 10, None, p, p, p, p, ws, big,
                               None) == -1
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt()), p, 10, ctypes.c_void_p(0x1004),
                               p, p, p, p, ws, big, None) == -1
    assert "aligned" in _err(L)
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam(w=0)), ctypes.byref(_opt()), p, 10, p, p, p, p, p, ws, big,
                               None) == -1
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt()), p, -1, p, p, p, p, p, ws, big,
                               None) == -1
    need = L.hp_quick_sampling_workspace_size(10, 8, 8)
    assert need > 0
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt()), p, 10, p, p, p, p, p, ws, need - 1,
                               None) == -2
    assert L.hp_quick_sampling(p, 10, ctypes.byref(_cam()), ctypes.byref(_opt()), p, 10, p, p, p, p, p, None, need,
                               None) == -2


def _view(w=8, h=8, k=3):
    v = native.HpView()
    p = 0x1000
    v.xyz, v.n_points, v.sorted_point_idx, v.n_sorted, v.hash_table = p, 10, p, 10, p
    v.sp_xyz = v.pc_idx = v.sp_t = v.mask = p
    v.cam = _cam(w, h)
    v.opt = _opt(k)
    return v


def test_batch_workspace_and_validation(L):
    one = (native.HpView * 1)(_view())
    two = (native.HpView * 2)(_view(), _view(64, 48))
    a = L.hp_quick_sampling_batch_workspace_size(one, 1)
    b = L.hp_quick_sampling_batch_workspace_size(two, 2)
    assert 0 < a < b
    assert L.hp_quick_sampling_batch_workspace_size(two, 0) == 0
    assert L.hp_quick_sampling_batch_workspace_size((native.HpView * 1)(_view(w=0)), 1) == 0
    ws = ctypes.c_void_p(0x100000)
    t = native.HpTuning()
    bad = (native.HpView * 2)(_view(), _view(k=9))
    assert L.hp_quick_sampling_batch(bad, None, 2, ctypes.byref(t), ws, 1 << 30, None) == -1
    assert "view 1" in _err(L) and "kernel_size" in _err(L)
    assert L.hp_quick_sampling_batch(two, None, 0, ctypes.byref(t), ws, 1 << 30, None) == -1
    assert L.hp_quick_sampling_batch(two, None, 2, ctypes.byref(t), ws, b - 1, None) == -2
    for bad_t in (native.HpTuning(4097), native.HpTuning(0, -1), native.HpTuning(0, 0, 6), native.HpTuning(0, 0, -1)):
        assert L.hp_quick_sampling_batch(two, None, 2, ctypes.byref(bad_t), ws, b, None) == -1
        assert "tuning" in _err(L)


def test_stage_config_info(L):
    shapes = {c: native.stage_config_info(c) for c in native.STAGE_CONFIGS}
    assert native.stage_config_info(0) == shapes[4]  # the default
    for c, d in shapes.items():
        assert d["tile_h"] * d["tile_w"] == 256 and d["stage_points"] > 0 and d["blocks_per_sm"] >= 1
    assert {(d["tile_h"], d["tile_w"]) for d in shapes.values()} == {(8, 32), (16, 16)}
    # a larger stage means fewer resident blocks
    assert shapes[1]["stage_points"] < shapes[2]["stage_points"] < shapes[3]["stage_points"]
    assert shapes[1]["blocks_per_sm"] > shapes[2]["blocks_per_sm"] > shapes[3]["blocks_per_sm"]
    for bad in (6, -1):
        assert L.hp_stage_config_info(bad, None, None, None, None) == -1
        assert "stage_config" in _err(L)


def test_pts2plane_status_validation(L):
    assert L.hp_pts2plane_status(None, 10, 8, 8, None) == -1
    assert L.hp_pts2plane_status(ctypes.c_void_p(0x1000), -1, 8, 8, None) == -1
    assert L.hp_pts2plane_status(ctypes.c_void_p(0x1000), 10, 0, 8, None) == -1
    assert "bad arguments" in _err(L)
    assert L.hp_pts2plane_noalloc_status(262145, 8, 8, None) == -1
    assert L.hp_pts2plane_noalloc_status(10, 1025, 1024, None) == -1


def test_pts2plane_checks_workspace(L):
    p = ctypes.c_void_p(0x1000)
    need = L.hp_pts2plane_workspace_size(10, 8, 8)
    rc = L.hp_pts2plane(p, 10, ctypes.byref(_cam()), 0, p, p, p, ctypes.c_void_p(0x10000), need - 1, None)
    assert rc == -2 and "workspace" in _err(L)
    rc = L.hp_pts2plane(p, 10, ctypes.byref(_cam()), 0, p, p, p, None, need, None)
    assert rc == -2
    rc = L.hp_pts2plane(p, 10, ctypes.byref(_cam()), 0, p, p, p, ctypes.c_void_p(0x10010), need, None)
    assert rc == -2  # not 256-byte aligned


def test_query_and_scatter_validation(L):
    p = ctypes.c_void_p(0x1000)
    o = _opt(k=32)
    assert L.hp_quick_query_for_nearby_point(p, 10, ctypes.byref(_cam()), ctypes.byref(o), p, 10, p, p, 4, p,
                                             None) == -1
    assert L.hp_scatter(p, p, p, 10, 8, 8, 0, p, p, None) == -1
    assert L.hp_scatter(p, p, p, 10, 8, 8, 65, p, p, None) == -1
    assert L.hp_scatter_hashtable(p, p, p, 10, 0, 8, 0, p, p, p, None) == -1
    # nothing to do: no launch, success
    o = _opt(k=3)
    assert L.hp_quick_query_for_nearby_point(p, 10, ctypes.byref(_cam()), ctypes.byref(o), p, 10, p, p, 0, p,
                                             None) == 0


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(native.HashPointError):
        native.lib()


def test_aggregator_sizes_and_validation(L):
    """The Aggregator's host-side contract: packed-weight and workspace sizes, and the argument
    checks that run before any device work (feature width, points per sample, alignment, workspace)."""
    packed = L.hp_aggregator_packed_size()
    assert packed == 34 * 16384 + 8192 + 9 * 16384 + 2056 * 4  # pair chunks, W3b, colour chunks, fp32 parameters
    assert L.hp_aggregator_workspace_size(-1) == 0
    w0, w1 = L.hp_aggregator_workspace_size(0), L.hp_aggregator_workspace_size(1000)
    assert 0 < w0 < w1 and w1 % 256 == 0
    p = ctypes.c_void_p(0x100000)

    def call(feat_dim=32, P=8, ws_bytes=w1, feat=p):
        return L.hp_aggregator_forward(p, p, p, p, feat, feat_dim, p, p, p, 1000, P, p, p, 8000, p, p, p, ws_bytes, None)

    assert call(feat_dim=16) == -1 and "feature width" in _err(L)
    for P in (0, 3, 64):
        assert call(P=P) == -1 and "points per sample" in _err(L)
    assert call(feat=ctypes.c_void_p(0x100004)) == -1 and "aligned" in _err(L)
    assert call(ws_bytes=w1 - 1) == -2 and "workspace" in _err(L)
    w = native.HpAggregatorWeights()
    assert L.hp_aggregator_pack(ctypes.byref(w), p, packed - 1, None) == -2
    assert L.hp_aggregator_pack(ctypes.byref(w), p, packed, None) == -1 and "layer 0" in _err(L)


def test_tc_check_validation(T):
    """The operand-form self-check's argument checks, which run before any device work."""
    L = T
    assert L.hp_tc_check_image_bytes(0) == 81920 and L.hp_tc_check_image_bytes(1) == 32768
    p = ctypes.c_void_p(0x100000)
    PLAIN, SW128, SW64 = 0, 1, 2
    bad = [
        (None, SW128, 0, SW64, 0, "null"),
        (ctypes.c_void_p(0x100008), SW128, 0, SW64, 0, "aligned"),
        (p, 3, 0, SW64, 0, "form"),
        (p, SW128, 8, SW64, 0, "offset"),                     # not on a 16-byte boundary
        (p, SW128, 65536 + 112, SW64, 0, "offset"),           # the K window leaves its 128-byte row
        (p, SW128, 65536 + 1024, SW64, 0, "offset"),          # 128 rows past the image's end
        (p, PLAIN, 81920 - 4080, SW64, 0, "offset"),
        (p, SW128, 0, SW128, 128, "offset"),                  # not in an atom's first row
        (p, SW128, 0, SW64, 48, "offset"),
    ]
    for a, af, ao, bf, bo, msg in bad:
        assert L.hp_tc_check_mma(a, p, af, ao, bf, bo, p, None) == -1, (af, ao, bf, bo)
        assert msg in _err(L)
