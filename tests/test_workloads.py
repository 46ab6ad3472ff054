"""The seeded synthetic workloads, on the CPU: point counts, bounds,
resolutions, focal lengths, principal points, search options and camera
geometry as the benchmark names them, every point in front of every camera
(the projection has no z > 0 filter, so a point behind a camera could alias
into its image), and the same data for the same seed."""
import numpy as np
import pytest

from hashpoint import synth


def _look_at_origin(cam, radius=None):
    c2w = np.asarray(cam.c2w, np.float64)
    eye = c2w[:3, 3]
    if radius is not None:
        assert np.isclose(np.linalg.norm(eye), radius, rtol=1e-5)
    fwd = c2w[:3, 2]  # OpenCV convention: the camera looks along +z
    np.testing.assert_allclose(fwd, -eye / np.linalg.norm(eye), atol=1e-5)
    np.testing.assert_allclose(np.asarray(cam.w2c, np.float64) @ c2w, np.eye(4), atol=1e-5)


def _options(opt, k, r, S, P):
    assert (opt.kernel_size, opt.num_sample_points_per_ray, opt.num_point_cloud_per_sp) == (k, S, P)
    assert np.isclose(opt.radius_threshold, r)


def test_sphere_workload():
    sc = synth.make_sphere()
    assert sc.xyz.shape == (100_000, 3) and sc.xyz.dtype == np.float32
    rad = np.linalg.norm(sc.xyz, axis=1)
    assert abs(rad.mean() - 1.0) < 1e-3 and rad.std() < 0.01
    (cam,) = sc.cameras
    assert (cam.width, cam.height, cam.fx, cam.fy, cam.cx, cam.cy) == (400, 400, 555.0, 555.0, 200.0, 200.0)
    _look_at_origin(cam, 4.0)
    _options(sc.options, 3, 0.01, 8, 8)
    assert synth.check_in_front(sc.xyz, cam)


def test_shapes_workload():
    sc = synth.make_shapes(n_views=100)
    assert sc.xyz.shape == (1_000_000, 3) and np.abs(sc.xyz).max() <= 1.5 + 1e-6
    assert sc.feat.shape == (1_000_000, 32) and sc.feat.dtype == np.float16
    assert len(sc.cameras) == 100
    elev = []
    for cam in sc.cameras:
        assert (cam.width, cam.height, cam.fx, cam.cx, cam.cy) == (800, 800, 1111.0, 400.0, 400.0)
        _look_at_origin(cam, 4.0)
        assert synth.check_in_front(sc.xyz, cam)
        eye = np.asarray(cam.c2w)[:3, 3]
        elev.append(np.degrees(np.arcsin(eye[2] / np.linalg.norm(eye))))
    assert -80.0 <= min(elev) and max(elev) <= 80.0
    _options(sc.options, 5, 0.008, 8, 8)


def test_clusters_workload():
    sc = synth.make_clusters()
    assert sc.xyz.shape == (3_000_000, 3)
    for cam in sc.cameras:
        assert (cam.width, cam.height, cam.fx, cam.cx, cam.cy) == (1600, 1200, 2890.0, 800.0, 600.0)
        _look_at_origin(cam)
        assert 2.5 <= np.linalg.norm(np.asarray(cam.c2w)[:3, 3]) <= 3.5
        assert synth.check_in_front(sc.xyz, cam)
    _options(sc.options, 5, 0.005, 16, 8)


def test_mixed_batch_workload():
    mb = synth.make_mixed()
    sizes = [len(c) for c in mb.clouds]
    assert len(sizes) == 8 and min(sizes) >= 5e4 and max(sizes) <= 4e6
    assert len(mb.views) == 64
    for c, cam in mb.views:
        assert 0 <= c < 8 and (cam.width, cam.height) in synth.MIXED_RESOLUTIONS
        assert np.isclose(cam.fx, 1111.0 * cam.width / 800.0)
        assert (cam.cx, cam.cy) == (cam.width / 2, cam.height / 2)
        _look_at_origin(cam, 4.0)
        assert synth.check_in_front(mb.clouds[c], cam)
    _options(mb.options, 5, 0.008, 8, 8)


@pytest.mark.parametrize("make", [lambda s: synth.make_sphere(n=5000, seed=s),
                                  lambda s: synth.make_shapes(n=5000, n_views=3, seed=s)])
def test_same_seed_same_data(make):
    a, b, c = make(7), make(7), make(8)
    assert np.array_equal(a.xyz, b.xyz) and not np.array_equal(a.xyz, c.xyz)
    for ca, cb in zip(a.cameras, b.cameras):
        assert np.array_equal(ca.c2w, cb.c2w)


def test_serving_scenes():
    """The served scenes (here scaled down 20x): sizes log-uniform, rescaled to the total, and each
    scene's camera poses on the radius-4 sphere looking at the origin."""
    from hashpoint import serve
    clouds, poses = serve.make_scenes(np.random.default_rng(0), n_scenes=16, total_points=2_000_000,
                                      size_range=(25_000, 300_000), n_poses=16)
    sizes = np.array([len(c) for c in clouds])
    assert len(clouds) == 16 and abs(int(sizes.sum()) - 2_000_000) <= 16
    assert sizes.max() / sizes.min() > 2  # uneven
    assert len(poses) == 16 and all(len(p) == 16 for p in poses)
    for c2w in poses[0]:
        eye = np.asarray(c2w, np.float64)[:3, 3]
        assert np.isclose(np.linalg.norm(eye), 4.0, rtol=1e-5)
        np.testing.assert_allclose(np.asarray(c2w, np.float64)[:3, 2], -eye / 4.0, atol=1e-5)
