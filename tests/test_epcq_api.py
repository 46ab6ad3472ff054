"""Host-side behaviour of the drop-in `epcq` API (no GPU needed)."""
import pytest
import torch

import epcq
from epcq import epcq as E


def test_module_surface():
    C = E._C
    for f in ("scatter", "scatter_hashtable", "quick_sampling", "quick_query_for_nearby_point"):
        assert callable(getattr(C, f))
    for c in ("CameraSpec", "NeuralPointsSpec", "RenderOptions", "NeuralPointsGrads"):
        assert isinstance(getattr(C, c), type)
    assert epcq.NeuralPoints is E.NeuralPoints


def test_render_options_defaults_match_reference():
    o = E.RenderOptions()
    # epcq/epcq.py:83-96
    assert (o.kernel_size, o.t_intvl, o.radius_threshold, o.sigma_threshold, o.background_brightness,
            o.stop_threshold, o.num_sample_points_per_ray, o.num_point_cloud_per_sp, o.num_point_per_ray,
            o.sdf2weight_gaussian_alpha, o.sdf2weight_gaussian_gamma, o.sparsity_loss_w, o.topK) == \
        (5, 0.01, 0.016, 1e-4, 1.0, 0.001, 16, 4, 256, 0.2, 0.9, 5e-4, 8)


def test_spec_fields_accept_zero_dim_tensors():
    c = E._C.CameraSpec()
    c.fx = torch.tensor(555.0)
    c.cx = 200
    c.width = torch.tensor(400)
    c.height = 300.0
    assert (c.fx, c.cx, c.width, c.height) == (555.0, 200.0, 400, 300)
    with pytest.raises(AttributeError):
        c.not_a_field = 1
    with pytest.raises(TypeError):
        c.c2w = [1, 2]


def test_camera_scalars_read_back_together():
    """CameraSpec._to_cpp takes Python numbers or one-element tensors (the reference's renderer
    passes 0-d tensors from K and the image size); the values, and int for integer tensors,
    survive the shared read-back."""
    K = torch.tensor([[1111.5, 0, 400.25], [0, 1110.75, 399.5], [0, 0, 1]], dtype=torch.float32)
    fx, fy, cx, cy = E.CameraSpec.decomposeK(K)
    hw = torch.tensor([800, 640])
    cam = E.CameraSpec(c2w=torch.eye(4), w2c=torch.eye(4), K=K, fx=fx, fy=fy, cx=cx, cy=cy, height=hw[0],
                       width=hw[1])
    spec = cam._to_cpp()
    assert (spec.fx, spec.fy, spec.cx, spec.cy, spec.width, spec.height) == (1111.5, 1110.75, 400.25, 399.5, 640, 800)
    vals = E._host_values(fx, 3, 2.5, hw[1], torch.tensor(0.1, dtype=torch.float32))
    assert vals[:4] == [1111.5, 3, 2.5, 640] and isinstance(vals[3], int)
    assert vals[4] == float(torch.tensor(0.1, dtype=torch.float32))  # the float32 value, exactly
    with pytest.raises(RuntimeError):
        E._host_values(torch.zeros(2))


def test_camera_scalars_read_once_per_camera(monkeypatch):
    """A view's calls share one read-back of its camera's tensor scalars; an in-place change of
    one of them, or a new field object, reads them again."""
    calls = []
    real = E._host_values
    monkeypatch.setattr(E, "_host_values", lambda *v: calls.append(1) or real(*v))
    K = torch.tensor([[100.0, 0, 32.0], [0, 90.0, 24.0], [0, 0, 1]])
    fx, fy, cx, cy = E.CameraSpec.decomposeK(K)
    hw = torch.tensor([48, 64])
    cam = E.CameraSpec(c2w=torch.eye(4), w2c=torch.eye(4), K=K, fx=fx, fy=fy, cx=cx, cy=cy, height=hw[0],
                       width=hw[1])
    assert cam._host() == (100.0, 90.0, 32.0, 24.0, 64, 48)
    cam._to_cpp()
    assert len(calls) == 1
    K[0, 0] = 120.0  # in place: fx's version moves
    assert cam._host()[0] == 120.0 and len(calls) == 2
    cam.width = 80  # a new object
    assert cam._host()[4] == 80 and len(calls) == 3
    plain = E.CameraSpec(c2w=torch.eye(4), w2c=torch.eye(4), K=K, fx=1.0, fy=2.0, cx=3.0, cy=4.0, width=5, height=6)
    assert plain._host() == (1.0, 2.0, 3.0, 4.0, 5, 6)


def test_options_to_cpp_roundtrip():
    o = E.RenderOptions(kernel_size=3, num_point_cloud_per_sp=8)
    cpp = o._to_cpp()
    assert cpp.kernel_size == 3 and cpp.num_point_cloud_per_sp == 8
    assert abs(cpp.t_intvl - 0.01) < 1e-12


def test_cpu_tensors_rejected_like_torch_check():
    pts = torch.zeros(10, 3)
    npnt = E.NeuralPoints(pc_type="pc", points=pts)
    cam = E.CameraSpec(c2w=torch.eye(4), w2c=torch.eye(4), K=torch.eye(3), fx=1.0, fy=1.0, cx=0.0, cy=0.0,
                       width=4, height=4)
    with pytest.raises(RuntimeError, match="CUDA"):
        npnt.pts2plane(cam, E.RenderOptions())
    with pytest.raises(RuntimeError, match="CUDA"):
        npnt.render_image_hashtable_topk(cam, E.RenderOptions(), torch.zeros(10, dtype=torch.int32),
                                         torch.zeros(10), torch.zeros(16, 2, dtype=torch.int32))


def test_ply_reader(tmp_path):
    import numpy as np
    p = tmp_path / "c.ply"
    xyz = np.array([[0.0, 1.0, 2.0], [3.0, 4.0, 5.0]], np.float32)
    rgb = np.array([[255, 0, 0], [0, 255, 0]], np.uint8)
    hdr = ("ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float x\nproperty float y\n"
           "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n")
    rec = np.zeros(2, dtype=[("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("r", "u1"), ("g", "u1"), ("b", "u1")])
    rec["x"], rec["y"], rec["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    rec["r"], rec["g"], rec["b"] = rgb[:, 0], rgb[:, 1], rgb[:, 2]
    p.write_bytes(hdr.encode() + rec.tobytes())
    a, c = E._read_ply_xyz_rgb(str(p))
    assert np.allclose(a, xyz) and np.allclose(c, rgb / 255.0)


def test_aggregator_module_matches_reference_layout():
    """Same parameter names and shapes as the reference's Aggregator (its state_dict loads), and the
    same initialisation: built after the same seed, its weights are the reference's (the fixture holds
    them rounded to fp16)."""
    import numpy as np

    import oracle_downstream as OD
    from hp_testutil import downstream_files
    torch.manual_seed(5)
    a = E.Aggregator()
    sd = a.state_dict()
    assert list(sd) == [k + s for k, _, _ in OD.AGG_LAYERS for s in (".weight", ".bias")]
    for k, n_out, n_in in OD.AGG_LAYERS:
        assert tuple(sd[k + ".weight"].shape) == (n_out, n_in) and tuple(sd[k + ".bias"].shape) == (n_out,)
    g = np.load(downstream_files("aggregator")[0])
    for k, _, _ in OD.AGG_LAYERS:
        assert np.array_equal(sd[k + ".weight"].numpy().astype(np.float16), g["w_" + k]), k
    assert a.chunksize == 20000


def test_aggregator_cpu_inputs_rejected():
    a = E.Aggregator()
    M, P = 4, 8
    z = torch.zeros(M, P, 3)
    with torch.no_grad(), pytest.raises(RuntimeError, match="CUDA"):
        a(z, z, z, torch.zeros(M, P, 32), torch.zeros(M, 3), torch.ones(M, P, dtype=torch.bool),
          torch.ones(2, 2, dtype=torch.bool), torch.zeros(M, 3))
    with pytest.raises(RuntimeError, match="no_grad"):
        a(z, z, z, torch.zeros(M, P, 32), torch.zeros(M, 3), torch.ones(M, P, dtype=torch.bool),
          torch.ones(2, 2, dtype=torch.bool), torch.zeros(M, 3))


def test_positional_encoding_matches_oracle():
    import numpy as np

    import oracle_downstream as OD
    x = torch.randn(5, 6)
    for ori in (False, True):
        pe = E.positional_encoding(x, 4, ori).numpy()
        want = OD.positional_encoding(x.numpy(), 4)
        if ori:
            args = (x.numpy()[..., None] * (2.0 ** np.arange(4, dtype=np.float32))).reshape(5, -1)
            want = np.concatenate([x.numpy(), np.sin(args), np.cos(args)], -1)
        np.testing.assert_allclose(pe, want, rtol=1e-6, atol=1e-6)


def test_checkpoint_round_trip(tmp_path):
    """_save2torch then _load_ckpt restores a 'gt_pc' cloud (density, features, positions); other
    point-cloud types raise NotImplementedError as in the reference."""
    import numpy as np
    p = tmp_path / "c.ply"
    hdr = "ply\nformat binary_little_endian 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\nend_header\n"
    p.write_bytes(hdr.encode() + np.arange(9, dtype="<f4").tobytes())
    a = E.NeuralPoints(pc_type="gt_pc", gt_pc_path=str(p), device="cpu")
    with torch.no_grad():
        a.density_data.add_(torch.arange(3.0)[:, None])
        a.feat_data.add_(1.5)
    ck = tmp_path / "np.pth"
    a._save2torch(str(ck))
    b = E.NeuralPoints(pc_type="gt_pc", gt_pc_path=str(p), device="cpu")
    b._load_ckpt(str(ck))
    assert torch.equal(b.density_data, a.density_data) and torch.equal(b.feat_data, a.feat_data)
    assert torch.equal(b.xyz_data, a.xyz_data) and b.capacity == 3
    b._load_ckpt(dict(torch.load(str(ck)), alpha_data=torch.ones(3)))
    assert torch.equal(b.alpha_data, torch.ones(3))
    c = E.NeuralPoints(pc_type="pc", points=torch.zeros(4, 3))
    with pytest.raises(NotImplementedError):
        c._load_ckpt(str(ck))
