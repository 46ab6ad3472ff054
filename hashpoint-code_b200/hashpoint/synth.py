"""Seeded synthetic scenes and cameras for the search+sample workloads.

The reference benchmarks on the NeRF-Synthetic lego scene and Point-NeRF
checkpoints (point_ray_search_benchmark/benchmark.py:33, opt/render_image.py:139),
which are not available here; these generators stand in for them with the
shapes, sizes and value distributions of the five named workloads:

  sphere   : N points uniform on the unit sphere, radial noise N(0, 0.005);
             camera at (0,0,4) looking at the origin; 400x400, f=555, c=200;
             radius 0.01, 3x3 window, 8 samples per ray.
  shapes   : N points area-uniform on 16 random boxes + 16 random ellipsoids
             inside [-1.5,1.5]^3 (extents U(0.1,0.6)), each point with an
             fp16[32] feature; cameras on a radius-4 sphere looking at the
             origin; 800x800, f=1111, c=400; radius 0.008, 5x5 window, K=8.
  clusters : 70% of N from 64 anisotropic Gaussians (sigma U(0.01,0.1) per
             axis) with z snapped to a height field (8 random sinusoids of
             amplitude 0.2), 30% uniform in [-1,1]^3; 1600x1200, f=2890,
             c=(800,600); camera distance U(2.5,3.5); radius 0.005, 5x5, K=16.

Cameras follow the OpenCV convention used by the reference's datasets
(dataset/nerfsynthesis.py:106): x right, y down, z forward; c2w is 4x4 and
w2c its inverse, both float32.  Everything is numpy only.
"""
from dataclasses import dataclass, field

import numpy as np


# ----------------------------------------------------------------------------
# cameras
# ----------------------------------------------------------------------------
@dataclass
class PinholeCamera:
    c2w: np.ndarray          # float32 [4,4]
    w2c: np.ndarray          # float32 [4,4]
    K: np.ndarray            # float32 [3,3]
    width: int
    height: int

    @property
    def fx(self):
        return float(self.K[0, 0])

    @property
    def fy(self):
        return float(self.K[1, 1])

    @property
    def cx(self):
        return float(self.K[0, 2])

    @property
    def cy(self):
        return float(self.K[1, 2])


def look_at_camera(eye, target, width, height, fx, fy=None, cx=None, cy=None, up=(0.0, 0.0, 1.0)):
    """OpenCV-convention camera at `eye` looking at `target` (float64 maths, float32 out).

    World up is +z; when the view direction is (anti)parallel to it, +y is used.
    """
    eye = np.asarray(eye, np.float64)
    target = np.asarray(target, np.float64)
    fwd = target - eye
    fwd /= np.linalg.norm(fwd)
    up = np.asarray(up, np.float64)
    if abs(np.dot(fwd, up)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = right, down, fwd, eye
    w2c = np.linalg.inv(c2w)
    fy = fx if fy is None else fy
    cx = width / 2.0 if cx is None else cx
    cy = height / 2.0 if cy is None else cy
    K = np.array([[fx, 0.0, cx], [0.0, fy, cy], [0.0, 0.0, 1.0]])
    return PinholeCamera(c2w.astype(np.float32), w2c.astype(np.float32), K.astype(np.float32),
                         int(width), int(height))


def orbit_cameras(rng, n, radius, width, height, f, cx=None, cy=None,
                  elev_deg=(-80.0, 80.0), radius_range=None):
    """`n` cameras at random azimuth/elevation on a sphere, looking at the origin."""
    cams = []
    for _ in range(n):
        az = rng.uniform(0.0, 2.0 * np.pi)
        el = np.deg2rad(rng.uniform(*elev_deg))
        r = radius if radius_range is None else rng.uniform(*radius_range)
        eye = r * np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])
        cams.append(look_at_camera(eye, (0, 0, 0), width, height, f, f, cx, cy))
    return cams


# ----------------------------------------------------------------------------
# point clouds
# ----------------------------------------------------------------------------
def sphere_cloud(rng, n, noise=0.005):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = 1.0 + rng.normal(0.0, noise, size=(n, 1))
    return (d * r).astype(np.float32)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _box_surface(rng, n, ext):
    a, b, c = ext  # half extents
    areas = np.array([b * c, b * c, a * c, a * c, a * b, a * b])
    face = rng.choice(6, size=n, p=areas / areas.sum())
    u = rng.uniform(-1.0, 1.0, size=n)
    v = rng.uniform(-1.0, 1.0, size=n)
    p = np.empty((n, 3))
    s = np.where(face % 2 == 0, 1.0, -1.0)
    ax = face // 2
    p[ax == 0] = np.stack([s * a, u * b, v * c], 1)[ax == 0]
    p[ax == 1] = np.stack([u * a, s * b, v * c], 1)[ax == 1]
    p[ax == 2] = np.stack([u * a, v * b, s * c], 1)[ax == 2]
    return p


def _ellipsoid_surface(rng, n, ext):
    a, b, c = ext
    gmax = max(b * c, a * c, a * b)
    out = []
    need = n
    while need > 0:
        m = int(need * 1.6) + 16
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        g = np.sqrt((b * c * d[:, 0]) ** 2 + (a * c * d[:, 1]) ** 2 + (a * b * d[:, 2]) ** 2)
        keep = rng.uniform(0.0, gmax, size=m) < g
        d = d[keep][:need]
        out.append(d * np.array([a, b, c]))
        need -= len(d)
    return np.concatenate(out, 0)


def _box_area(ext):
    a, b, c = ext
    return 8.0 * (a * b + b * c + a * c)


def _ellipsoid_area(ext):
    a, b, c = ext
    p = 1.6075  # Knud Thomsen's approximation
    return 4.0 * np.pi * (((a * b) ** p + (a * c) ** p + (b * c) ** p) / 3.0) ** (1.0 / p)


def shapes_cloud(rng, n, n_boxes=16, n_ellipsoids=16, bound=1.5, ext_range=(0.1, 0.6)):
    """Area-uniform points on random boxes and ellipsoids inside [-bound, bound]^3.

    `ext_range` bounds each shape's full extent per axis.
    """
    kinds = [0] * n_boxes + [1] * n_ellipsoids
    shapes = []
    for k in kinds:
        ext = rng.uniform(*ext_range, size=3) / 2.0
        rot = _random_rotation(rng)
        rmax = np.linalg.norm(ext)
        ctr = rng.uniform(-bound + rmax, bound - rmax, size=3)
        area = _box_area(ext) if k == 0 else _ellipsoid_area(ext)
        shapes.append((k, ext, rot, ctr, area))
    areas = np.array([s[4] for s in shapes])
    counts = rng.multinomial(n, areas / areas.sum())
    pts = []
    for (k, ext, rot, ctr, _), m in zip(shapes, counts):
        if m == 0:
            continue
        p = _box_surface(rng, m, ext) if k == 0 else _ellipsoid_surface(rng, m, ext)
        pts.append(p @ rot.T + ctr)
    pts = np.concatenate(pts, 0)
    pts = pts[rng.permutation(len(pts))]
    return pts.astype(np.float32)


def height_field(rng, n_waves=8, amp=0.2):
    k = rng.uniform(0.5, 4.0, size=(n_waves, 2)) * rng.choice([-1, 1], size=(n_waves, 2))
    ph = rng.uniform(0.0, 2 * np.pi, size=n_waves)

    def h(x, y):
        z = np.zeros_like(x)
        for i in range(n_waves):
            z += amp * np.sin(k[i, 0] * x + k[i, 1] * y + ph[i])
        return z
    return h


def clusters_cloud(rng, n, n_clusters=64, frac_clustered=0.7, sigma_range=(0.01, 0.1)):
    nc = int(round(n * frac_clustered))
    h = height_field(rng)
    centers = rng.uniform(-1.0, 1.0, size=(n_clusters, 3))
    sig = rng.uniform(*sigma_range, size=(n_clusters, 3))
    lab = rng.integers(0, n_clusters, size=nc)
    p = centers[lab] + rng.normal(size=(nc, 3)) * sig[lab]
    p[:, 2] = h(p[:, 0], p[:, 1])
    bg = rng.uniform(-1.0, 1.0, size=(n - nc, 3))
    pts = np.concatenate([p, bg], 0)
    pts = pts[rng.permutation(n)]
    return pts.astype(np.float32)


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
@dataclass
class Options:
    """Mirror of the reference RenderOptions fields used by the path (epcq.py:82-96)."""
    kernel_size: int = 5
    t_intvl: float = 0.01
    radius_threshold: float = 0.016
    sigma_threshold: float = 1e-4
    background_brightness: float = 1.0
    stop_threshold: float = 0.001
    num_sample_points_per_ray: int = 16
    num_point_cloud_per_sp: int = 4
    num_point_per_ray: int = 256
    sdf2weight_gaussian_alpha: float = 0.2
    sdf2weight_gaussian_gamma: float = 0.9
    topK: int = 8


@dataclass
class Scene:
    name: str
    xyz: np.ndarray
    cameras: list
    options: Options
    feat: np.ndarray = None
    meta: dict = field(default_factory=dict)


def make_sphere(n=100_000, seed=0, width=400, height=400, f=555.0):
    rng = np.random.default_rng(seed)
    xyz = sphere_cloud(rng, n)
    cam = look_at_camera((0, 0, 4), (0, 0, 0), width, height, f, f, width / 2, height / 2)
    opt = Options(kernel_size=3, radius_threshold=0.01, num_sample_points_per_ray=8,
                  num_point_cloud_per_sp=8)
    return Scene("sphere", xyz, [cam], opt)


def make_shapes(n=1_000_000, n_views=100, seed=0, width=800, height=800, f=1111.0, with_feat=True):
    rng = np.random.default_rng(seed)
    xyz = shapes_cloud(rng, n)
    cams = orbit_cameras(rng, n_views, 4.0, width, height, f, width / 2, height / 2)
    feat = None
    if with_feat:
        feat = rng.standard_normal(size=(n, 32), dtype=np.float32).astype(np.float16)
    opt = Options(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8,
                  num_point_cloud_per_sp=8)
    return Scene("shapes", xyz, cams, opt, feat)


def make_clusters(n=3_000_000, n_views=4, seed=0, width=1600, height=1200, f=2890.0):
    rng = np.random.default_rng(seed)
    xyz = clusters_cloud(rng, n)
    cams = orbit_cameras(rng, n_views, None, width, height, f, 800.0 * width / 1600, 600.0 * height / 1200,
                         elev_deg=(20.0, 80.0), radius_range=(2.5, 3.5))
    opt = Options(kernel_size=5, radius_threshold=0.005, num_sample_points_per_ray=16,
                  num_point_cloud_per_sp=8)
    return Scene("clusters", xyz, cams, opt)


def check_in_front(xyz, cam):
    """True when every point has positive camera depth (no behind-camera aliasing)."""
    z = xyz.astype(np.float64) @ cam.w2c[2, :3].astype(np.float64) + float(cam.w2c[2, 3])
    return bool(np.all(z > 0))


@dataclass
class MixedBatch:
    """Several clouds and views over them (view = (cloud index, camera))."""
    clouds: list
    views: list
    options: Options


MIXED_RESOLUTIONS = ((256, 256), (512, 512), (800, 800), (1600, 1200))


def make_mixed(n_clouds=8, n_views=64, seed=0, size_range=(5e4, 4e6), resolutions=MIXED_RESOLUTIONS):
    """Uneven multi-cloud batch: clouds as in `shapes` with sizes log-uniform in
    size_range; each view picks a cloud and a resolution uniformly, f = 1111 * W / 800,
    camera on the radius-4 sphere looking at the origin."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(size_range[0]), np.log(size_range[1])
    sizes = np.exp(rng.uniform(lo, hi, size=n_clouds)).astype(np.int64)
    clouds = [shapes_cloud(rng, int(n)) for n in sizes]
    views = []
    for _ in range(n_views):
        c = int(rng.integers(n_clouds))
        W, H = resolutions[int(rng.integers(len(resolutions)))]
        f = 1111.0 * W / 800.0
        cam = orbit_cameras(rng, 1, 4.0, W, H, f, W / 2, H / 2)[0]
        views.append((c, cam))
    opt = Options(kernel_size=5, radius_threshold=0.008, num_sample_points_per_ray=8, num_point_cloud_per_sp=8)
    return MixedBatch(clouds, views, opt)
