"""hp_pts2plane_noalloc: projection + hash table without any device allocation.

Some callers cannot allocate device memory -- for example a host plugin that
the embedding application hands nothing but device pointers for its inputs and
outputs, or a service that must keep its device footprint fixed once it has
started -- so they cannot give hp_pts2plane the workspace it needs.
hp_pts2plane_noalloc takes the same inputs and outputs and uses scratch built
into the library instead.  These tests call it through the C ABI and check,
on two calls in a row with different inputs, that it returns exactly what
hp_pts2plane returns (integer outputs equal, depths equal bit for bit), and
that a problem larger than its built-in scratch is refused with a clear error.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from hashpoint import native, ops, synth

pytestmark = pytest.mark.gpu

MAX_POINTS = 262144
MAX_PIXELS = 1048576


def _noalloc(xyz, w2c, K, height, width, sort):
    L = native.lib()
    n = xyz.shape[0]
    sidx = torch.empty(n, dtype=torch.int32, device=xyz.device)
    sdep = torch.empty(n, dtype=torch.float32, device=xyz.device)
    hsh = torch.empty((height * width, 2), dtype=torch.int32, device=xyz.device)
    cam = ops.make_camera(w2c=w2c, K=K, width=width, height=height)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.hp_pts2plane_noalloc(ctypes.c_void_p(xyz.data_ptr()), n, ctypes.byref(cam), int(sort),
                                ctypes.c_void_p(sidx.data_ptr()), ctypes.c_void_p(sdep.data_ptr()),
                                ctypes.c_void_p(hsh.data_ptr()), stream)
    native.check(rc, "hp_pts2plane_noalloc")
    native.check(L.hp_pts2plane_noalloc_status(n, height, width, stream), "hp_pts2plane_noalloc_status")
    return sidx, sdep, hsh


def _scene(seed, n, width, height, f):
    rng = np.random.default_rng(seed)
    xyz = synth.shapes_cloud(rng, n)
    cam = synth.orbit_cameras(rng, 1, 4.0, width, height, f)[0]
    dev = torch.device("cuda:0")
    return (torch.from_numpy(xyz).to(dev), torch.from_numpy(cam.w2c).to(dev), torch.from_numpy(cam.K).to(dev),
            cam.height, cam.width)


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    native.build()
    cases = [(_scene(11, 200000, 640, 480, 900.0), False), (_scene(12, 50000, 321, 207, 400.0), True)]
    for (xyz, w2c, K, H, W), sort in cases:
        a = _noalloc(xyz, w2c, K, H, W, sort)
        b = ops.pts2plane(xyz, w2c, K, H, W, sort)
        torch.cuda.synchronize()
        assert torch.equal(a[0], b[0])
        assert torch.equal(a[2], b[2])
        assert torch.equal(a[1].view(torch.int32), b[1].view(torch.int32))
        assert int((a[2][:, 1] > 0).sum()) > 0


def test_noalloc_at_its_limits():
    """Exactly the largest problem the built-in scratch takes (262144 points on a 1024 x 1024
    image, whose scratch offsets are the tightest), checked against hp_pts2plane and the CPU
    oracle; then no points at all on the same image."""
    native.build()
    O.build()
    rng = np.random.default_rng(13)
    xyz = synth.shapes_cloud(rng, MAX_POINTS)
    cam = synth.orbit_cameras(rng, 1, 4.0, 1024, 1024, 1400.0)[0]
    assert cam.width * cam.height == MAX_PIXELS
    dev = torch.device("cuda:0")
    X, w2c, K = (torch.from_numpy(a).to(dev) for a in (xyz, cam.w2c, cam.K))
    for sort in (False, True):
        a = _noalloc(X, w2c, K, cam.height, cam.width, sort)
        b = ops.pts2plane(X, w2c, K, cam.height, cam.width, sort)
        torch.cuda.synchronize()
        for x, y in zip(a, b):
            assert torch.equal(x.view(torch.int32), y.view(torch.int32))
        oi, od, oh = O.pts2plane(xyz, O.camera_from(cam), sort)
        assert np.array_equal(a[0].cpu().numpy(), oi) and np.array_equal(a[2].cpu().numpy(), oh)
        assert np.array_equal(a[1].cpu().numpy().view(np.int32), od.view(np.int32))
    empty = torch.empty((0, 3), dtype=torch.float32, device=dev)
    sidx, sdep, hsh = _noalloc(empty, w2c, K, cam.height, cam.width, False)
    torch.cuda.synchronize()
    assert sidx.numel() == 0 and sdep.numel() == 0 and bool((hsh == -1).all())


def test_noalloc_refuses_problems_beyond_its_scratch():
    native.build()
    L = native.lib()
    cam = ops.make_camera(width=64, height=64)
    p = ctypes.c_void_p(0x1000)
    rc = L.hp_pts2plane_noalloc(p, MAX_POINTS + 1, ctypes.byref(cam), 0, p, p, p, None)
    assert rc == -1 and "scratch" in L.hp_last_error().decode()
    big = ops.make_camera(width=1025, height=1024)
    rc = L.hp_pts2plane_noalloc(p, 10, ctypes.byref(big), 0, p, p, p, None)
    assert rc == -1 and str(MAX_PIXELS) in L.hp_last_error().decode()
