"""The downstream oracle (oracle/oracle_downstream.py) against the reference's
own FeatureQuery / clamp_t / render / Aggregator outputs (tests/golden/fd_*.npz).

Gathered rows, sample points, validity flags and clamp_t are exact; ray
directions and colours are float32 sums whose order the reference leaves to
torch, compared with rtol 1e-6 and atol 1e-7.  The Aggregator's float32 MLP
(matmul and sum orders left to torch) agrees with it to atol 1e-6.
"""
import numpy as np
import pytest

import oracle_downstream as OD
from hp_testutil import aggregator_inputs, aggregator_params, bits, downstream_files

RTOL, ATOL = 1e-6, 1e-7


@pytest.mark.parametrize("path", downstream_files("feature"))
def test_feature_query_oracle_vs_reference(path):
    g = np.load(path)
    fx, fy, cx, cy = [float(x) for x in g["cam_f"]]
    uv = g["uv"] if len(g["uv"]) else None
    out = OD.feature_query(g["xyz"], g["rgb"], g["dir"], g["feat"], g["sp_xyz"], g["pc_idx"], g["mask"], g["c2w"],
                           fx, fy, cx, cy, int(g["width"]), uv)
    for key, got in zip(("pc_xyz", "pc_rgb", "pc_dir", "pc_feat", "out_sp_xyz", "valid"), out[:6]):
        assert got.shape == g[key].shape, key
        if got.dtype == np.float32:
            assert np.array_equal(bits(got), bits(g[key])), key
        else:
            assert np.array_equal(got, g[key]), key
    np.testing.assert_allclose(out[6], g["rays_d"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("path", downstream_files("render"))
def test_render_oracle_vs_reference(path):
    g = np.load(path)
    d = OD.clamp_t(g["t_val"], float(g["vsize"]))
    assert np.array_equal(bits(d), bits(g["t_dist"]))
    np.testing.assert_allclose(OD.render(d, g["sigmas"], g["rgbs"]), g["color"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(OD.render(d, g["sigmas"], g["rgbs"], True), g["color_white"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("path", downstream_files("aggregator"))
def test_aggregator_oracle_vs_reference(path):
    g = np.load(path)
    params = aggregator_params(g)
    for mask, a_key, c_key in (("mask", "alpha_train", "color_train"), ("mask3", "alpha_infer", "color_infer")):
        alphas, colors = OD.aggregator(params, *aggregator_inputs(g), g[mask], g["rays_d"])
        assert alphas.shape == g[a_key].shape and colors.shape == g[c_key].shape
        np.testing.assert_allclose(alphas, g[a_key], rtol=0, atol=1e-6)
        np.testing.assert_allclose(colors, g[c_key], rtol=0, atol=1e-6)
        unset = ~g[mask].reshape(-1)
        assert not alphas.reshape(-1)[unset].any() and not colors.reshape(-1, 3)[unset].any()


def test_positional_encoding_layout():
    """Interleaved sin / cos, argument index channel * freqs + band (epcq.py:389-404)."""
    x = np.array([[0.5, -2.0]], np.float32)
    pe = OD.positional_encoding(x, 3)
    args = np.array([0.5, 1.0, 2.0, -2.0, -4.0, -8.0], np.float32)
    want = np.stack([np.sin(args), np.cos(args)], -1).reshape(1, 12)
    assert np.array_equal(pe, want)
