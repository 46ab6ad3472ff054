"""Size-independent properties of the oracle's outputs on seeded scenes, on the
CPU, beside its bit-exact pinning to the reference's goldens:

  pts2plane     the (start, count) table partitions the in-image points into
                contiguous buckets in pixel order; every id in a bucket
                projects to that pixel; ids ascend inside a bucket (depths,
                then ids, when sorted); depths are the ids' own; the
                off-image tail is -1.
  sampling      a ray's samples are a prefix of its S slots with strictly
                increasing t, at o + t d; unused slots are zero / -1; a
                sample's point ids are listed first and lie within the radius
                of the sample.
  ray query     at most num_point_per_ray ids, within the radius of the ray.
  z-buffer      each pixel keeps the `bins` smallest depths of its points, in
                ascending order, each with its own point's id; -1 padded.
Ids repeat only where the k x k window meets the image border: the reference
clamps the window's cells to the image, so a border cell is visited more
than once; away from the border every id is listed once.
"""
import numpy as np
import pytest

import oracle as O
from hashpoint import synth

SCENES = {
    # a sphere in full view, 3x3 windows
    "sphere": lambda: synth.make_sphere(n=20000, seed=1, width=96, height=80, f=555.0 * 96 / 400),
    # boxes and ellipsoids that overflow the image, 5x5 windows
    "shapes": lambda: synth.make_shapes(n=60000, n_views=2, seed=2, width=128, height=96, f=1111.0 * 128 / 800,
                                        with_feat=False),
}


def interior(rays, cam, k):
    """Rays whose k x k pixel window lies inside the image."""
    v, u = rays // cam.width, rays % cam.width
    h = k // 2
    return (u >= h) & (u < cam.width - h) & (v >= h) & (v < cam.height - h)


@pytest.fixture(scope="module", autouse=True)
def _build_oracle():
    O.build()


@pytest.fixture(scope="module", params=sorted(SCENES))
def scene(request):
    sc = SCENES[request.param]()
    return sc, O.camera_from(sc.cameras[-1])


@pytest.mark.parametrize("sort", [False, True])
def test_hash_table_partitions_the_in_image_points(scene, sort):
    sc, cam = scene
    H, W = cam.height, cam.width
    pid, depth = O.project(sc.xyz, cam)
    inside = pid < H * W
    oi, od, oh = O.pts2plane(sc.xyz, cam, sort)
    n_in = int(inside.sum())
    assert 0 < n_in <= len(oi)
    start, count = oh[:, 0], oh[:, 1]
    empty = count <= 0
    assert np.all(start[empty] == -1) and np.all(count[empty] == -1)
    full = np.nonzero(~empty)[0]
    assert count[full].sum() == n_in
    assert start[full[0]] == 0 and np.all(start[full[1:]] == start[full[:-1]] + count[full[:-1]])
    assert np.all(oi[n_in:] == -1) and np.all(od[n_in:] == -1)
    ids = oi[:n_in]
    assert len(np.unique(ids)) == n_in and np.all(inside[ids])
    assert np.array_equal(od[:n_in], depth[ids])  # each id's own depth
    bucket_pixel = np.repeat(full, count[full])
    assert np.array_equal(pid[ids], bucket_pixel)  # every id in its pixel's bucket
    same = bucket_pixel[1:] == bucket_pixel[:-1]
    if sort:  # (depth, id) ascending inside a bucket
        d0, d1 = od[:n_in - 1][same], od[1:n_in][same]
        assert np.all((d0 < d1) | ((d0 == d1) & (ids[:-1][same] < ids[1:][same])))
    else:
        assert np.all(ids[:-1][same] < ids[1:][same])


def test_samples_and_their_points(scene):
    sc, cam = scene
    opt = sc.options
    oi, od, oh = O.pts2plane(sc.xyz, cam, False)
    sp, pc, t, m, _ = O.quick_sampling(sc.xyz, cam, opt, oi, oh)
    S, P = m.shape[-1], pc.shape[-1]
    m2, t2, sp2, pc2 = m.reshape(-1, S), t.reshape(-1, S), sp.reshape(-1, S, 3), pc.reshape(-1, S, P)
    assert m2.any()
    assert np.all(np.diff(m2.astype(np.int8), axis=1) <= 0)  # a prefix of the slots
    assert np.all(t2[~m2] == 0) and np.all(sp2[~m2] == 0) and np.all(pc2[~m2] == -1)
    both = m2[:, 1:] & m2[:, :-1]
    assert np.all(np.diff(t2, axis=1)[both] > 0)
    # the sample points lie on their rays
    dirs = O.ray_dirs(cam).astype(np.float64)
    o = np.asarray(sc.cameras[-1].c2w, np.float64)[:3, 3]
    ray, slot = np.nonzero(m2)
    on_ray = o + t2[ray, slot, None].astype(np.float64) * dirs[ray]
    np.testing.assert_allclose(sp2[ray, slot], on_ray, rtol=0, atol=1e-6)
    # ball query: ids listed first, within the radius of the sample, unique away from the border
    ids = pc2[ray, slot]
    valid = ids >= 0
    n_valid = valid.sum(1)
    assert np.array_equal(valid, np.arange(P)[None, :] < n_valid[:, None])
    inner = interior(ray, cam, int(opt.kernel_size))
    assert inner.any()
    for row in ids[inner]:
        v = row[row >= 0]
        assert len(np.unique(v)) == len(v)
    pts = sc.xyz[np.where(valid, ids, 0)].astype(np.float64)
    dist = np.linalg.norm(pts - sp2[ray, slot, None, :], axis=2)
    r = float(opt.radius_threshold)
    assert np.all(dist[valid] < r * (1 + 1e-5))


def test_ray_query_points_are_near_the_ray(scene):
    sc, cam = scene
    opt = sc.options
    oi, od, oh = O.pts2plane(sc.xyz, cam, False)
    rays = np.arange(0, cam.height * cam.width, 5, dtype=np.int32)
    out, cnt, _ = O.quick_query(sc.xyz, cam, opt, oi, oh, rays)
    assert np.all((cnt >= 0) & (cnt <= opt.num_point_per_ray)) and cnt.sum() > 0
    dirs = O.ray_dirs(cam).astype(np.float64)
    o = np.asarray(sc.cameras[-1].c2w, np.float64)[:3, 3]
    r = float(opt.radius_threshold)
    inner = interior(rays, cam, int(opt.kernel_size))
    for i, ray in enumerate(rays):
        ids = out[i, :cnt[i]]
        if inner[i]:
            assert len(np.unique(ids)) == len(ids)
        if len(ids):
            d = dirs[ray] / np.linalg.norm(dirs[ray])
            v = sc.xyz[ids].astype(np.float64) - o
            dist = np.linalg.norm(v - (v @ d)[:, None] * d, axis=1)
            assert np.all(dist < r * (1 + 1e-5))


@pytest.mark.parametrize("bins", [1, 4, 8])
def test_multibin_keeps_the_nearest_points(scene, bins):
    sc, cam = scene
    H, W = cam.height, cam.width
    pid, depth = O.project(sc.xyz, cam)
    ps, ds, ix = O.sort_by_pixel(pid, depth, H * W)
    od, oi = O.scatter_multibin(ix, ps, ds, H, W, bins)
    valid = oi >= 0
    n = valid.sum(1)
    assert np.array_equal(valid, np.arange(bins)[None, :] < n[:, None])
    assert np.all(od[~valid] == -1)
    inside = pid < H * W
    per_pixel = np.bincount(pid[inside], minlength=H * W)
    assert np.array_equal(n, np.minimum(per_pixel, bins))
    assert np.all(np.diff(od, axis=1)[valid[:, 1:]] >= 0)
    px, slot = np.nonzero(valid)
    ids = oi[px, slot]
    assert np.array_equal(pid[ids], px) and np.array_equal(depth[ids], od[px, slot])
    # the kept depths are the pixel's smallest ones
    order = np.lexsort((depth[inside], pid[inside]))
    pix_sorted, dep_sorted = pid[inside][order], depth[inside][order]
    first = np.searchsorted(pix_sorted, np.arange(H * W))
    for p in np.nonzero(n)[0][::7]:
        np.testing.assert_array_equal(od[p, :n[p]], dep_sorted[first[p]:first[p] + n[p]])
