// Window search, primary-surface selection, K-sample emission and per-sample
// point selection, fused into one kernel.
//
// Replaces _C.quick_sampling (epcq/csrc/epcq_render_topk.cu:341-417), which
// zero-fills all four outputs, runs quick_sampling_kernel (:82-220, one warp
// per ray, one lane per window cell, a 128-bin shared-memory histogram built
// with float atomics and a serial walk on lane 0) and then
// quick_search_nearby_pc (:10-81, one thread per (ray, sample slot) re-walking
// the window).  Here one thread owns one ray end to end and writes every
// output element of that ray exactly once:
//
//   pass A  kept candidates (ray distance < radius, at most 48 per window cell,
//           cells row-major and clamped, bucket order) -> tmin, tmax
//   pass B  the same candidates binned by int((t - tmin) / t_intvl); instead of
//           a 128-bin histogram the thread keeps the 8 smallest distinct bins
//           (count, distance sum) in registers -- exactly the bins the walk
//           reaches first -- and re-collects further bins only if the walk
//           goes past them
//   walk    bins with >= 2 points in ascending order: alpha = gamma *
//           exp(-mean_dist / alpha_g), emit when alpha * T > 1e-3, T -= alpha,
//           stop when T < 1e-3 or S samples are out
//   ball    per emitted sample, the reference's 8-entry id buffer over the
//           whole window (including its quirk that, while the buffer fills, the
//           tracked "farthest" entry is the nearest one)
//
// Bin sums are accumulated in window-cell then bucket order; the reference
// adds them with shared-memory atomics in an unspecified order, so a bin's
// mean distance can differ from the reference's in the last bit -- which moves
// an output only if alpha * T or T sits within that bit of 1e-3.
#include "hp_common.cuh"

namespace hp {

constexpr int kTileW = 32;   // pixels of one image row per warp
constexpr int kTileH = 4;    // rows per block
constexpr int kBinList = 8;  // distinct t-bins collected per candidate pass

struct SampleArgs {
  const float* __restrict__ xyz;
  const int* __restrict__ sidx;
  const int2* __restrict__ hash;
  int n_points;  // ids outside [0, n_points) are skipped
  int n_sorted;  // bucket ranges are clipped to [0, n_sorted)
  DevCamera cam;
  DevOptions opt;
  float* __restrict__ sp_xyz;
  int* __restrict__ pc_idx;
  float* __restrict__ sp_t;
  uint8_t* __restrict__ mask;
};

// Kept candidates in the reference's order: window cells 0..ncell-1, bucket
// order, at most kKeptPerCell kept per cell; f(t, dist) for each.
template <typename F>
__device__ __forceinline__ void for_each_kept(const SampleArgs& a, const Ray& r, int v, int u, int ncell, F&& f) {
  const int H = a.cam.height, W = a.cam.width, k = a.opt.k;
  for (int l = 0; l < ncell; l++) {
    int vv, uu;
    window_cell(v, u, k, H, W, l, vv, uu);
    const int2 h = __ldg(a.hash + (size_t)vv * W + uu);
    if (h.y <= 0 || h.x < 0) continue;
    int nk = 0;
    const int end = min(h.x + min(h.y, a.n_sorted), a.n_sorted);
    for (int j = h.x; j < end && nk < kKeptPerCell; j++) {
      const int id = __ldg(a.sidx + j);
      if ((unsigned)id >= (unsigned)a.n_points) continue;
      const float4 p = load_point(a.xyz, id);
      float t, dist;
      intersect(r, p.x, p.y, p.z, t, dist);
      if (dist < a.opt.radius) {
        nk++;
        f(t, dist);
      }
    }
  }
}

// Every window point (all k*k cells, no cap), f(id, point).
template <typename F>
__device__ __forceinline__ void for_each_window_point(const SampleArgs& a, int v, int u, int k2, F&& f) {
  const int H = a.cam.height, W = a.cam.width, k = a.opt.k;
  for (int l = 0; l < k2; l++) {
    int vv, uu;
    window_cell(v, u, k, H, W, l, vv, uu);
    const int2 h = __ldg(a.hash + (size_t)vv * W + uu);
    if (h.y < 0 || h.x < 0) continue;
    const int end = min(h.x + min(h.y, a.n_sorted), a.n_sorted);
    for (int j = h.x; j < end; j++) {
      const int id = __ldg(a.sidx + j);
      if ((unsigned)id >= (unsigned)a.n_points) continue;
      f(id, load_point(a.xyz, id));
    }
  }
}

__global__ void __launch_bounds__(kTileW* kTileH) k_quick_sampling(SampleArgs a) {
  const int u = blockIdx.x * kTileW + (threadIdx.x & 31);
  const int v = blockIdx.y * kTileH + (threadIdx.x >> 5);
  const int W = a.cam.width, H = a.cam.height;
  if (u >= W || v >= H) return;
  const int ray = v * W + u;
  const int S = a.opt.S, P = a.opt.P, k = a.opt.k, k2 = k * k;
  const int ncell = k2 < kLaneCells ? k2 : kLaneCells;

  Ray r;
  make_ray(a.cam.c2w, a.cam.fx, a.cam.fy, a.cam.cx, a.cam.cy, u, v, r);

  // pass A: tmin / tmax over the kept candidates (epcq_render_topk.cu:132-161)
  float tmin = 1e3f, tmax = -1e3f;
  for_each_kept(a, r, v, u, ncell, [&](float t, float) {
    if (tmin > t) tmin = t;
    if (tmax < t) tmax = t;
  });

  float* o_xyz = a.sp_xyz + (size_t)ray * S * 3;
  float* o_t = a.sp_t + (size_t)ray * S;
  uint8_t* o_m = a.mask + (size_t)ray * S;
  int* o_idx = a.pc_idx + (size_t)ray * S * P;
  int emitted = 0;

  if (!(tmin > tmax)) {
    float transmit = 1.0f;
    int lo = 0;
    for (;;) {
      // pass B: the kBinList smallest distinct bins in [lo, cut) with full stats
      int lb[kBinList], lc[kBinList];
      float ls[kBinList];
#pragma unroll
      for (int q = 0; q < kBinList; q++) lb[q] = 0x7fffffff, lc[q] = 0, ls[q] = 0.0f;
      int m = 0, cut = kBins;
      for_each_kept(a, r, v, u, ncell, [&](float t, float dist) {
        const int b = __float2int_rz(__fdiv_rn(__fsub_rn(t, tmin), a.opt.t_intvl));
        if (b < lo || b >= cut) return;
        bool found = false;
#pragma unroll
        for (int q = 0; q < kBinList; q++)
          if (q < m && lb[q] == b) {
            lc[q] += 1;
            ls[q] = __fadd_rn(ls[q], dist);
            found = true;
          }
        if (found) return;
        if (m == kBinList && b > lb[kBinList - 1]) {
          cut = b;
          return;
        }
        int pos = 0;
#pragma unroll
        for (int q = 0; q < kBinList; q++) pos += (q < m && lb[q] < b) ? 1 : 0;
        if (m == kBinList) cut = lb[kBinList - 1];
#pragma unroll
        for (int q = kBinList - 1; q >= 0; q--) {
          if (q > pos) {
            lb[q] = lb[q - 1];
            lc[q] = lc[q - 1];
            ls[q] = ls[q - 1];
          } else if (q == pos) {
            lb[q] = b;
            lc[q] = 1;
            ls[q] = dist;
          }
        }
        m = m < kBinList ? m + 1 : kBinList;
      });
      // primary-surface walk (epcq_render_topk.cu:181-204)
      bool done = false;
#pragma unroll
      for (int q = 0; q < kBinList; q++) {
        if (q >= m || done) break;
        if (lc[q] < 2) continue;
        if (transmit < 1e-3f || emitted >= S) {
          done = true;
          break;
        }
        const float sdf = __fdiv_rn(ls[q], __fadd_rn((float)lc[q], 1e-6f));
        const float alpha = __fmul_rn(a.opt.gamma, __expf(__fdiv_rn(-sdf, a.opt.alpha_g)));
        const float weight = __fmul_rn(alpha, transmit);
        if (weight > 1e-3f) {
          const float t = __fmaf_rn((float)lb[q], a.opt.t_intvl, tmin);
          o_xyz[emitted * 3 + 0] = __fmaf_rn(t, r.d[0], r.o[0]);
          o_xyz[emitted * 3 + 1] = __fmaf_rn(t, r.d[1], r.o[1]);
          o_xyz[emitted * 3 + 2] = __fmaf_rn(t, r.d[2], r.o[2]);
          o_t[emitted] = t;
          o_m[emitted] = 1;
          emitted++;
        }
        transmit = __fsub_rn(transmit, alpha);
      }
      if (done || cut >= kBins) break;
      lo = cut;
    }
  }

  // per-sample point selection (epcq_render_topk.cu:10-81)
  for (int s = 0; s < emitted; s++) {
    const float sx = o_xyz[s * 3 + 0], sy = o_xyz[s * 3 + 1], sz = o_xyz[s * 3 + 2];
    float bd[kBallBuf];
    int bi[kBallBuf];
#pragma unroll
    for (int q = 0; q < kBallBuf; q++) bd[q] = 0.0f, bi[q] = -1;
    int bsize = 0, maxi = 0;
    float maxd = 1e3f;
    for_each_window_point(a, v, u, k2, [&](int id, float4 p) {
      const float dist = norm3df(__fsub_rn(sx, p.x), __fsub_rn(sy, p.y), __fsub_rn(sz, p.z));
      if (!(dist < a.opt.radius)) return;
      if (bsize < kBallBuf) {
#pragma unroll
        for (int q = 0; q < kBallBuf; q++)
          if (q == bsize) bd[q] = dist, bi[q] = id;
        if (maxd > dist) {
          maxd = dist;
          maxi = bsize;
        }
        bsize++;
      } else if (dist < maxd) {
#pragma unroll
        for (int q = 0; q < kBallBuf; q++)
          if (q == maxi) bd[q] = dist, bi[q] = id;
        maxd = dist;
#pragma unroll
        for (int q = 0; q < kBallBuf; q++)
          if (bd[q] > maxd) {
            maxd = bd[q];
            maxi = q;
          }
      }
    });
    int* row = o_idx + (size_t)s * P;
#pragma unroll
    for (int q = 0; q < kBallBuf; q++)
      if (q < P) row[q] = q < bsize ? bi[q] : -1;
    for (int q = kBallBuf; q < P; q++) row[q] = -1;
  }

  // defaults for the slots nothing was emitted into
  for (int s = emitted; s < S; s++) {
    o_xyz[s * 3 + 0] = 0.0f;
    o_xyz[s * 3 + 1] = 0.0f;
    o_xyz[s * 3 + 2] = 0.0f;
    o_t[s] = 0.0f;
    o_m[s] = 0;
    int* row = o_idx + (size_t)s * P;
    for (int q = 0; q < P; q++) row[q] = -1;
  }
}

__global__ void k_ray_directions(DevCamera cam, float* __restrict__ dirs) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= cam.width * cam.height) return;
  Ray r;
  make_ray(cam.c2w, cam.fx, cam.fy, cam.cx, cam.cy, p % cam.width, p / cam.width, r);
  dirs[3 * (size_t)p + 0] = r.d[0];
  dirs[3 * (size_t)p + 1] = r.d[1];
  dirs[3 * (size_t)p + 2] = r.d[2];
}

int32_t check_camera(const hp_camera* cam, const char* who) {
  if (!cam) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: cam is NULL", who);
  if (cam->height <= 0 || cam->width <= 0 || (int64_t)cam->height * cam->width >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: bad image size %dx%d", who, cam->height, cam->width);
  if (!cam->c2w) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: c2w is NULL", who);
  return HP_OK;
}

DevCamera dev_camera(const hp_camera* cam) {
  DevCamera d;
  d.c2w = cam->c2w;
  d.fx = cam->fx;
  d.fy = cam->fy;
  d.cx = cam->cx;
  d.cy = cam->cy;
  d.width = cam->width;
  d.height = cam->height;
  return d;
}

DevOptions dev_options(const hp_options* o) {
  DevOptions d;
  d.k = o->kernel_size;
  d.t_intvl = o->t_intvl;
  d.radius = o->radius_threshold;
  d.S = o->num_sample_points_per_ray;
  d.P = o->num_point_cloud_per_sp;
  d.num_point_per_ray = o->num_point_per_ray;
  d.alpha_g = o->sdf2weight_gaussian_alpha;
  d.gamma = o->sdf2weight_gaussian_gamma;
  return d;
}

}  // namespace hp

using namespace hp;

extern "C" int32_t hp_quick_sampling(const float* xyz, int64_t n_points, const hp_camera* cam, const hp_options* opt,
                                     const int32_t* sorted_point_idx, int64_t n_sorted, const int32_t* hash_table,
                                     float* sp_xyz, int32_t* pc_idx, float* sp_t, uint8_t* mask, hp_stream_t stream) {
  if (int32_t rc = check_camera(cam, "hp_quick_sampling")) return rc;
  if (!opt) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: opt is NULL");
  if (opt->kernel_size < 1 || opt->kernel_size > kMaxKernel)
    return set_error(HP_ERR_INVALID_ARGUMENT,
                     "hp_quick_sampling: kernel_size %d outside 1..%d (the reference's windows hold 32 cells)",
                     opt->kernel_size, kMaxKernel);
  if (!(opt->t_intvl > 0.0f))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: t_intvl must be > 0");
  if (opt->num_sample_points_per_ray < 1 || opt->num_point_cloud_per_sp < 1)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: num_sample_points_per_ray and "
                     "num_point_cloud_per_sp must be >= 1");
  const int64_t hw = (int64_t)cam->height * cam->width;
  if (hw * opt->num_sample_points_per_ray * (int64_t)(opt->num_point_cloud_per_sp > 3 ? opt->num_point_cloud_per_sp : 3) >=
      (1ll << 40))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: output too large");
  if (n_points < 0 || n_points >= (1ll << 31) || n_sorted < 0 || n_sorted >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: n_points / n_sorted out of range");
  if (!hash_table || !sp_xyz || !pc_idx || !sp_t || !mask || (n_points > 0 && !xyz) ||
      (n_sorted > 0 && !sorted_point_idx))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: null pointer");
  if (((uintptr_t)hash_table & 7) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_quick_sampling: hash_table must be 8-byte aligned");
  SampleArgs a;
  a.xyz = xyz;
  a.sidx = sorted_point_idx;
  a.hash = (const int2*)hash_table;
  a.n_points = (int)n_points;
  a.n_sorted = (int)n_sorted;
  a.cam = dev_camera(cam);
  a.opt = dev_options(opt);
  a.sp_xyz = sp_xyz;
  a.pc_idx = pc_idx;
  a.sp_t = sp_t;
  a.mask = mask;
  const dim3 grid((cam->width + kTileW - 1) / kTileW, (cam->height + kTileH - 1) / kTileH);
  k_quick_sampling<<<grid, kTileW * kTileH, 0, (cudaStream_t)stream>>>(a);
  return check_launch("k_quick_sampling");
}

extern "C" int32_t hp_ray_directions(const hp_camera* cam, float* dirs, hp_stream_t stream) {
  if (int32_t rc = check_camera(cam, "hp_ray_directions")) return rc;
  if (!dirs) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_ray_directions: dirs is NULL");
  const int hw = cam->width * cam->height;
  k_ray_directions<<<(hw + 255) / 256, 256, 0, (cudaStream_t)stream>>>(dev_camera(cam), dirs);
  return check_launch("k_ray_directions");
}
