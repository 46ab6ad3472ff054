// TEST INFRASTRUCTURE ONLY -- CPU oracle for the HashPoint search+sample path.
//
// CPU restatement of the reference algorithm, used by tests/, the smoke check
// and bench.py's CPU-baseline leg as the checker; never part of the product.
// See hp_oracle.h for the parity statement.
//
// FP32 arithmetic mirrors the GPU operation by operation.  Where nvcc or
// cuBLAS fuse a multiply-add the restatement calls fmaf explicitly; the
// fusion pattern of every expression was established by diffing GPU outputs
// (no compiled code was read).  Build with -ffp-contract=off so the host
// compiler adds no fusion of its own.
#include "hp_oracle.h"

#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

// Point counts above which cuBLAS used an FMA chain for the world->camera and
// the camera->image 3x3 @ 3xN GEMMs of epcq.py:253,261 (see ora_projection_rounding).
#ifndef ORA_WORLD_FUSED_ABOVE
#define ORA_WORLD_FUSED_ABOVE 1536
#endif
#ifndef ORA_IMAGE_FUSED_ABOVE
#define ORA_IMAGE_FUSED_ABOVE 233023
#endif

namespace {

constexpr int kLaneCells = 32;      // cells a sampling warp covers (cuda_util.cuh:11, epcq_render_topk.cu:125)
constexpr int kKeptPerCell = 48;    // per-lane projection buffer (cuda_util.cuh:17, epcq_render_topk.cu:135-139)
constexpr int kBins = 128;          // t-histogram bins (cuda_util.cuh:19)
constexpr int kBallBuf = 8;         // per-sample id buffer (cuda_util.cuh:13, epcq_render_topk.cu:35)
constexpr int kQueryPerCell = 32;   // per-lane id buffer in the ray query (epcq_render_topk.cu:256-259)

// ---------------------------------------------------------------------------
// arithmetic mirrors
// ---------------------------------------------------------------------------
// float -> int32 conversion with round-toward-zero and saturation (cvt.rzi.s32.f32,
// what static_cast<int> and torch's .to(torch.int32) do on the GPU).
inline int f2i_rz(double q) {
  if (q != q) return 0;
  if (q >= 2147483648.0) return INT_MAX;
  if (q <= -2147483649.0) return INT_MIN;
  return (int)q;
}

// _dot3d (cuda_util.cuh:57) as nvcc contracts it: fma(a2,b2, fma(a0,b0, a1*b1)).
inline float dot3(const float* a, const float* b) { return fmaf(a[2], b[2], fmaf(a[0], b[0], a[1] * b[1])); }
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Stand-ins for CUDA's norm3df / rnorm3df / __expf: correctly rounded via double.
inline float norm3(float x, float y, float z) {
  return (float)std::sqrt((double)x * x + (double)y * y + (double)z * z);
}
inline double norm3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }
inline float rnorm3(float x, float y, float z) {
  return (float)(1.0 / std::sqrt((double)x * x + (double)y * y + (double)z * z));
}
inline double rnorm3(double x, double y, double z) { return 1.0 / std::sqrt(x * x + y * y + z * z); }
inline float fexp(float x) { return (float)std::exp((double)x); }
inline double fexp(double x) { return std::exp(x); }
inline float fmadd(float a, float b, float c) { return fmaf(a, b, c); }
inline double fmadd(double a, double b, double c) { return a * b + c; }

template <typename T>
struct Ray {
  T o[3];
  T d[3];
};

// cam2world_ray (cuda_util.cuh:338-354): pixel centre in double, cast to float;
// d_i = fma(c_i0, x, c_i1*y) + c_i2 (z = 1 folded); normalised by rnorm3df.
template <typename T>
inline void make_ray(const ora_camera* cam, int u, int v, const float* dir_override, Ray<T>* r);

template <>
inline void make_ray<float>(const ora_camera* cam, int u, int v, const float* dir_override, Ray<float>* r) {
  const float* c = cam->c2w;
  for (int i = 0; i < 3; i++) r->o[i] = c[4 * i + 3];
  if (dir_override) {
    for (int i = 0; i < 3; i++) r->d[i] = dir_override[i];
    return;
  }
  float x = (float)(((double)u + 0.5 - (double)cam->cx) / (double)cam->fx);
  float y = (float)(((double)v + 0.5 - (double)cam->cy) / (double)cam->fy);
  float d[3];
  for (int i = 0; i < 3; i++) d[i] = fmaf(c[4 * i + 0], x, c[4 * i + 1] * y) + c[4 * i + 2];
  float rn = rnorm3(d[0], d[1], d[2]);
  for (int i = 0; i < 3; i++) r->d[i] = d[i] * rn;
}

template <>
inline void make_ray<double>(const ora_camera* cam, int u, int v, const float*, Ray<double>* r) {
  const float* c = cam->c2w;
  for (int i = 0; i < 3; i++) r->o[i] = c[4 * i + 3];
  double x = ((double)u + 0.5 - (double)cam->cx) / (double)cam->fx;
  double y = ((double)v + 0.5 - (double)cam->cy) / (double)cam->fy;
  double d[3];
  for (int i = 0; i < 3; i++) d[i] = (double)c[4 * i + 0] * x + (double)c[4 * i + 1] * y + (double)c[4 * i + 2];
  double rn = rnorm3(d[0], d[1], d[2]);
  for (int i = 0; i < 3; i++) r->d[i] = d[i] * rn;
}

// PointRayInterset (cuda_util.cuh:215-236): t = (p-o).d / d.d; proj = fma(t,d,o);
// dist = norm3df(p - proj).
template <typename T>
inline void intersect(const Ray<T>& r, const float* pf, T* t_out, T* dist_out) {
  T p[3] = {(T)pf[0], (T)pf[1], (T)pf[2]};
  T s[3] = {p[0] - r.o[0], p[1] - r.o[1], p[2] - r.o[2]};
  T t = dot3(s, r.d) / dot3(r.d, r.d);
  T e[3];
  for (int i = 0; i < 3; i++) e[i] = p[i] - fmadd(t, r.d[i], r.o[i]);
  *t_out = t;
  *dist_out = norm3(e[0], e[1], e[2]);
}

// calculate_neighbor_uv (cuda_util.cuh:382-388): row-major k x k window,
// offsets from ceil() of float divisions (restated in exact integer form),
// coordinates clamped into the image.
inline void window_cell(int v, int u, int k, int H, int W, int l, int* vv, int* uu) {
  const int koff = (k + 1) / 2;                 // ceil(k / 2.0f)
  const int voff = (l + k) / k - koff;          // ceil((l+1)/k) - koff
  const int uoff = (l % k) - (koff - 1);
  int a = v + voff, b = u + uoff;
  *vv = a < 0 ? 0 : (a > H - 1 ? H - 1 : a);
  *uu = b < 0 ? 0 : (b > W - 1 ? W - 1 : b);
}

// Dynamic parallel-for over [0, n) in chunks on `nthreads` std::threads
// (nthreads <= 1 runs inline).
template <typename F>
void parallel_for(int64_t n, int nthreads, F&& body) {
  if (nthreads <= 1 || n < 256) {
    body(0, n);
    return;
  }
  std::atomic<int64_t> next(0);
  const int64_t chunk = 64;
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; t++)
    pool.emplace_back([&]() {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        body(b, b + chunk < n ? b + chunk : n);
      }
    });
  for (auto& th : pool) th.join();
}

inline void note(float* margin, double slack) {
  if (slack < 0) slack = -slack;
  if (slack < *margin) *margin = (float)slack;
}

struct Kept {
  float t, dist;
};

// ---------------------------------------------------------------------------
// quick_sampling, one ray (FP32 mirror)
// ---------------------------------------------------------------------------
void sample_ray_f32(const float* xyz, const ora_camera* cam, const ora_options* opt, const int32_t* sorted_idx,
                    const int32_t* hash, const float* dirs, int ray, int64_t out_i, float* sp_xyz, int32_t* pc_idx,
                    float* sp_t, uint8_t* mask, float* margin_out, std::vector<Kept>& kept,
                    std::vector<int>& kept_cell_n) {
  const int W = cam->width, H = cam->height;
  const int u = ray % W, v = ray / W;
  const int k = opt->kernel_size;
  const int k2 = k * k;
  const int S = opt->num_sample_points_per_ray, P = opt->num_point_cloud_per_sp;
  const float r_thr = opt->radius_threshold;
  float margin = 1e30f;

  float* o_xyz = sp_xyz + (size_t)out_i * S * 3;
  int32_t* o_idx = pc_idx + (size_t)out_i * S * P;
  float* o_t = sp_t + (size_t)out_i * S;
  uint8_t* o_m = mask + (size_t)out_i * S;
  for (int i = 0; i < S * 3; i++) o_xyz[i] = 0.0f;
  for (int i = 0; i < S * P; i++) o_idx[i] = -1;
  for (int i = 0; i < S; i++) o_t[i] = 0.0f, o_m[i] = 0;

  Ray<float> rr;
  make_ray<float>(cam, u, v, dirs ? dirs + (size_t)ray * 3 : nullptr, &rr);
  const double scale = 1.0 + std::fabs(rr.o[0]) + std::fabs(rr.o[1]) + std::fabs(rr.o[2]);

  // Step 1 (epcq_render_topk.cu:118-161): per window cell keep up to 48 points
  // with ray distance < radius; tmin/tmax over the kept points.
  kept.clear();
  kept_cell_n.assign(kLaneCells, 0);
  const int ncell = k2 < kLaneCells ? k2 : kLaneCells;
  std::vector<int> cell_begin(ncell + 1, 0);
  float tmin = 1e3f, tmax = -1e3f;
  for (int l = 0; l < ncell; l++) {
    cell_begin[l] = (int)kept.size();
    int vv, uu;
    window_cell(v, u, k, H, W, l, &vv, &uu);
    const int32_t start = hash[2 * ((size_t)vv * W + uu)], cnt = hash[2 * ((size_t)vv * W + uu) + 1];
    if (cnt <= 0) continue;
    int nk = 0;
    for (int j = start; j < start + cnt && nk < kKeptPerCell; j++) {
      const float* p = xyz + 3 * (size_t)sorted_idx[j];
      float t, dist;
      intersect<float>(rr, p, &t, &dist);
      note(&margin, (dist - r_thr) / scale);
      if (dist < r_thr) {
        if (tmin > t) tmin = t;
        if (tmax < t) tmax = t;
        kept.push_back({t, dist});
        nk++;
      }
    }
    kept_cell_n[l] = nk;
  }
  cell_begin[ncell] = (int)kept.size();
  if (tmin > tmax) {
    if (margin_out) margin_out[out_i] = margin;
    return;
  }

  // Step 2 (:167-179): histogram of mean ray distance per t-bin.  The
  // reference adds with shared-memory atomics; here the adds run in
  // window-cell order, then bucket order.
  float sums[kBins], cnts[kBins];
  for (int b = 0; b < kBins; b++) sums[b] = 0.0f, cnts[b] = 0.0f;
  for (const Kept& q : kept) {
    float quo = (q.t - tmin) / opt->t_intvl;
    if (q.t != tmin) {  // the minimum itself lands on bin 0 exactly
      double fr = (double)quo - std::floor((double)quo);
      if (fr > 0.5) fr = 1.0 - fr;
      note(&margin, fr * opt->t_intvl / scale);
    }
    int b = f2i_rz(quo);
    if (b >= kBins) continue;
    sums[b] += q.dist;
    cnts[b] += 1.0f;
  }
  for (int b = 0; b < kBins; b++) sums[b] /= (cnts[b] + 1e-6f);

  // Step 3 (:181-219): primary-surface walk with subtractive transmittance.
  float transmit = 1.0f;
  int slot = 0;
  for (int b = 0; b < kBins; b++) {
    if (cnts[b] < 2.0f) continue;
    note(&margin, (double)transmit - 1e-3);
    if (transmit < 1e-3f) break;
    if (slot >= S) break;
    float sdf = sums[b];
    float alpha = opt->sdf2weight_gaussian_gamma * fexp(-sdf / opt->sdf2weight_gaussian_alpha);
    float weight = alpha * transmit;
    note(&margin, (double)weight - 1e-3);
    if (weight > 1e-3f) {
      float t = fmaf((float)b, opt->t_intvl, tmin);
      for (int j = 0; j < 3; j++) o_xyz[slot * 3 + j] = fmaf(t, rr.d[j], rr.o[j]);
      o_m[slot] = 1;
      o_t[slot] = t;
      slot++;
    }
    transmit -= alpha;
  }

  // quick_search_nearby_pc (:10-81): per emitted sample, ball query over the
  // whole window with the 8-entry buffer.  While the buffer fills, the tracked
  // "max" is the running minimum (:54-57); once full, the first eviction
  // therefore replaces the closest point, after which the true maximum is tracked.
  for (int s = 0; s < slot; s++) {
    const float sp[3] = {o_xyz[s * 3 + 0], o_xyz[s * 3 + 1], o_xyz[s * 3 + 2]};
    const double bscale = scale + std::fabs(o_t[s]);
    float bd[kBallBuf];
    int bi[kBallBuf];
    int bsize = 0, maxi = 0;
    float maxd = 1e3f;
    for (int l = 0; l < k2; l++) {
      int vv, uu;
      window_cell(v, u, k, H, W, l, &vv, &uu);
      const int32_t start = hash[2 * ((size_t)vv * W + uu)], cnt = hash[2 * ((size_t)vv * W + uu) + 1];
      if (cnt < 0) continue;
      for (int j = start; j <= start + cnt - 1; j++) {
        const int id = sorted_idx[j];
        const float* p = xyz + 3 * (size_t)id;
        float dist = norm3(sp[0] - p[0], sp[1] - p[1], sp[2] - p[2]);
        note(&margin, (dist - r_thr) / bscale);
        if (!(dist < r_thr)) continue;
        // comparisons of a point with itself (clamped windows repeat cells) are exact ties
        if (bsize == 0 || bi[maxi] != id) note(&margin, (dist - maxd) / bscale);
        if (bsize < kBallBuf) {
          bd[bsize] = dist;
          bi[bsize] = id;
          if (maxd > dist) {
            maxd = dist;
            maxi = bsize;
          }
          bsize++;
        } else if (dist < maxd) {
          bd[maxi] = dist;
          bi[maxi] = id;
          maxd = dist;
          for (int q = 0; q < kBallBuf; q++) {
            if (bi[q] != bi[maxi]) note(&margin, (bd[q] - maxd) / bscale);
            if (bd[q] > maxd) {
              maxd = bd[q];
              maxi = q;
            }
          }
        }
      }
    }
    const int nw = bsize < P ? bsize : P;
    for (int q = 0; q < nw; q++) o_idx[s * P + q] = bi[q];
  }
  if (margin_out) margin_out[out_i] = margin;
}

// FP64 twin of steps 1-3 (no ball query): emitted t / xyz in double.
void sample_ray_f64(const float* xyz, const ora_camera* cam, const ora_options* opt, const int32_t* sorted_idx,
                    const int32_t* hash, int ray, double* sp_xyz, double* sp_t, uint8_t* mask) {
  const int W = cam->width, H = cam->height;
  const int u = ray % W, v = ray / W;
  const int k = opt->kernel_size, k2 = k * k;
  const int S = opt->num_sample_points_per_ray;
  const double r_thr = opt->radius_threshold;
  double* o_xyz = sp_xyz + (size_t)ray * S * 3;
  double* o_t = sp_t + (size_t)ray * S;
  uint8_t* o_m = mask + (size_t)ray * S;
  for (int i = 0; i < S * 3; i++) o_xyz[i] = 0.0;
  for (int i = 0; i < S; i++) o_t[i] = 0.0, o_m[i] = 0;
  Ray<double> rr;
  make_ray<double>(cam, u, v, nullptr, &rr);
  std::vector<double> kt, kd;
  const int ncell = k2 < kLaneCells ? k2 : kLaneCells;
  double tmin = 1e3, tmax = -1e3;
  for (int l = 0; l < ncell; l++) {
    int vv, uu;
    window_cell(v, u, k, H, W, l, &vv, &uu);
    const int32_t start = hash[2 * ((size_t)vv * W + uu)], cnt = hash[2 * ((size_t)vv * W + uu) + 1];
    if (cnt <= 0) continue;
    int nk = 0;
    for (int j = start; j < start + cnt && nk < kKeptPerCell; j++) {
      double t, dist;
      intersect<double>(rr, xyz + 3 * (size_t)sorted_idx[j], &t, &dist);
      if (dist < r_thr) {
        tmin = t < tmin ? t : tmin;
        tmax = t > tmax ? t : tmax;
        kt.push_back(t);
        kd.push_back(dist);
        nk++;
      }
    }
  }
  if (tmin > tmax) return;
  double sums[kBins], cnts[kBins];
  for (int b = 0; b < kBins; b++) sums[b] = 0.0, cnts[b] = 0.0;
  for (size_t i = 0; i < kt.size(); i++) {
    int b = f2i_rz((kt[i] - tmin) / (double)opt->t_intvl);
    if (b >= kBins) continue;
    sums[b] += kd[i];
    cnts[b] += 1.0;
  }
  double transmit = 1.0;
  int slot = 0;
  for (int b = 0; b < kBins; b++) {
    if (cnts[b] < 2.0) continue;
    if (transmit < 1e-3) break;
    if (slot >= S) break;
    double sdf = sums[b] / (cnts[b] + 1e-6);
    double alpha = (double)opt->sdf2weight_gaussian_gamma * std::exp(-sdf / (double)opt->sdf2weight_gaussian_alpha);
    if (alpha * transmit > 1e-3) {
      double t = tmin + b * (double)opt->t_intvl;
      for (int j = 0; j < 3; j++) o_xyz[slot * 3 + j] = rr.o[j] + t * rr.d[j];
      o_m[slot] = 1;
      o_t[slot] = t;
      slot++;
    }
    transmit -= alpha;
  }
}

int check_options(const ora_camera* cam, const ora_options* opt) {
  if (cam->width <= 0 || cam->height <= 0) return -1;
  if (opt->kernel_size < 1 || opt->kernel_size > 5) return -2;
  if (!(opt->t_intvl > 0.0f)) return -3;
  if (opt->num_sample_points_per_ray < 1 || opt->num_point_cloud_per_sp < 1) return -4;
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// projection (epcq.py:251-274)
// ---------------------------------------------------------------------------
extern "C" void ora_project_mode(const float* xyz, int64_t n, const ora_camera* cam, int32_t fused_world,
                                 int32_t fused_image, int32_t* point2img, float* depth) {
  const float* w = cam->w2c;
  const float* K = cam->K;
  const int H = cam->height, W = cam->width;
  for (int64_t i = 0; i < n; i++) {
    const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    float pc[3];
    for (int r = 0; r < 3; r++) {
      const float* a = w + 4 * r;
      float g = fused_world ? fmaf(a[2], z, fmaf(a[1], y, a[0] * x)) : (a[0] * x + a[1] * y) + a[2] * z;
      pc[r] = g + a[3];
    }
    float s[3];
    for (int r = 0; r < 3; r++) {
      const float* a = K + 3 * r;
      s[r] = fused_image ? fmaf(a[2], pc[2], fmaf(a[1], pc[1], a[0] * pc[0]))
                         : (a[0] * pc[0] + a[1] * pc[1]) + a[2] * pc[2];
    }
    const int ix = f2i_rz(s[0] / s[2]), iy = f2i_rz(s[1] / s[2]);
    const bool inb = 0 <= ix && ix < W && 0 <= iy && iy < H;
    point2img[i] = inb ? ix + iy * W : H * W;
    depth[i] = pc[2];
  }
}

// Which GEMM arithmetic torch/cuBLAS used for the projection's two 3x3 @ 3xN
// products on a B200 (torch 2.11, cuBLAS 12.8), established by diffing its
// outputs: an FMA chain above a size threshold, separately rounded products
// below it.  Must match hp_projection_rounding in the product library.
extern "C" void ora_projection_rounding(int64_t n, int32_t* fused_world, int32_t* fused_image) {
  *fused_world = n > ORA_WORLD_FUSED_ABOVE;
  *fused_image = n > ORA_IMAGE_FUSED_ABOVE;
}

extern "C" void ora_project(const float* xyz, int64_t n, const ora_camera* cam, int32_t* point2img, float* depth) {
  int32_t fw, fi;
  ora_projection_rounding(n, &fw, &fi);
  ora_project_mode(xyz, n, cam, fw, fi, point2img, depth);
}

extern "C" void ora_project_f64(const float* xyz, int64_t n, const ora_camera* cam, double* depth) {
  const float* w = cam->w2c;
  for (int64_t i = 0; i < n; i++) {
    depth[i] = (double)w[8] * xyz[3 * i] + (double)w[9] * xyz[3 * i + 1] + (double)w[10] * xyz[3 * i + 2] +
               (double)w[11];
  }
}

// ---------------------------------------------------------------------------
// sort + hash table
// ---------------------------------------------------------------------------
extern "C" void ora_sort_by_pixel(const int32_t* point2img, const float* depth, int64_t n, int32_t hw,
                                  int32_t* pid_sorted, float* depth_sorted, int32_t* idx_sorted) {
  // stable counting sort over keys [0, hw]
  std::vector<int64_t> off((size_t)hw + 2, 0);
  for (int64_t i = 0; i < n; i++) off[(size_t)point2img[i] + 1]++;
  for (int64_t p = 0; p <= hw; p++) off[p + 1] += off[p];
  for (int64_t i = 0; i < n; i++) {
    int64_t dst = off[point2img[i]]++;
    pid_sorted[dst] = point2img[i];
    depth_sorted[dst] = depth[i];
    idx_sorted[dst] = (int32_t)i;
  }
}

extern "C" void ora_scatter_hashtable(const int32_t* point_idx, const int32_t* point2img, const float* depth,
                                      int64_t n, int32_t height, int32_t width, int32_t sort, int32_t* out_idx,
                                      float* out_depth, int32_t* hash) {
  const int64_t hw = (int64_t)height * width;
  for (int64_t i = 0; i < n; i++) out_idx[i] = -1, out_depth[i] = -1.0f;
  for (int64_t p = 0; p < 2 * hw; p++) hash[p] = -1;
  // binary_search (cuda_util.cuh:558-579) finds the first index of each pixel
  // id; the walk (rasterization.cu:23-28) copies the run.
  int64_t i = 0;
  while (i < n) {
    const int32_t p = point2img[i];
    int64_t j = i;
    while (j < n && point2img[j] == p) j++;
    if (p >= 0 && p < hw) {
      for (int64_t q = i; q < j; q++) out_idx[q] = point_idx[q], out_depth[q] = depth[q];
      if (sort) {
        // bubble_sort ascending (cuda_util.cuh:291-313): stable by depth
        const int64_t m = j - i;
        for (int64_t a = 0; a < m; a++) {
          bool swapped = false;
          for (int64_t b = i; b < j - a - 1; b++) {
            if (out_depth[b] > out_depth[b + 1]) {
              float td = out_depth[b];
              out_depth[b] = out_depth[b + 1];
              out_depth[b + 1] = td;
              int32_t ti = out_idx[b];
              out_idx[b] = out_idx[b + 1];
              out_idx[b + 1] = ti;
              swapped = true;
            }
          }
          if (!swapped) break;
        }
      }
      hash[2 * p] = (int32_t)i;
      hash[2 * p + 1] = (int32_t)(j - i);
    }
    i = j;
  }
}

extern "C" void ora_pts2plane(const float* xyz, int64_t n, const ora_camera* cam, int32_t sort, int32_t* out_idx,
                              float* out_depth, int32_t* hash) {
  const int32_t hw = cam->width * cam->height;
  std::vector<int32_t> pid(n), pid_s(n), idx_s(n);
  std::vector<float> dep(n), dep_s(n);
  ora_project(xyz, n, cam, pid.data(), dep.data());
  ora_sort_by_pixel(pid.data(), dep.data(), n, hw, pid_s.data(), dep_s.data(), idx_s.data());
  ora_scatter_hashtable(idx_s.data(), pid_s.data(), dep_s.data(), n, cam->height, cam->width, sort, out_idx,
                        out_depth, hash);
}

// ---------------------------------------------------------------------------
// sampling
// ---------------------------------------------------------------------------
extern "C" int ora_quick_sampling_dirs(const float* xyz, int64_t n_points, const ora_camera* cam,
                                       const ora_options* opt, const int32_t* sorted_idx, const int32_t* hash,
                                       const float* dirs, float* sp_xyz, int32_t* pc_idx, float* sp_t,
                                       uint8_t* mask, float* margin, const int32_t* rays, int64_t n_rays,
                                       int32_t nthreads) {
  (void)n_points;
  int rc = check_options(cam, opt);
  if (rc) return rc;
  const int64_t hw = (int64_t)cam->width * cam->height;
  const int64_t total = rays ? n_rays : hw;
  parallel_for(total, nthreads, [&](int64_t b, int64_t e) {
    std::vector<Kept> kept;
    std::vector<int> kn;
    kept.reserve(1024);
    for (int64_t i = b; i < e; i++) {
      const int ray = rays ? rays[i] : (int)i;
      sample_ray_f32(xyz, cam, opt, sorted_idx, hash, dirs, ray, i, sp_xyz, pc_idx, sp_t, mask, margin, kept, kn);
    }
  });
  return 0;
}

extern "C" int ora_quick_sampling(const float* xyz, int64_t n_points, const ora_camera* cam, const ora_options* opt,
                                  const int32_t* sorted_idx, const int32_t* hash, float* sp_xyz, int32_t* pc_idx,
                                  float* sp_t, uint8_t* mask, float* margin, const int32_t* rays, int64_t n_rays,
                                  int32_t nthreads) {
  return ora_quick_sampling_dirs(xyz, n_points, cam, opt, sorted_idx, hash, nullptr, sp_xyz, pc_idx, sp_t, mask,
                                 margin, rays, n_rays, nthreads);
}

extern "C" int ora_quick_sampling_f64(const float* xyz, int64_t n_points, const ora_camera* cam,
                                      const ora_options* opt, const int32_t* sorted_idx, const int32_t* hash,
                                      double* sp_xyz, double* sp_t, uint8_t* mask, int32_t nthreads) {
  (void)n_points;
  int rc = check_options(cam, opt);
  if (rc) return rc;
  const int64_t hw = (int64_t)cam->width * cam->height;
  parallel_for(hw, nthreads, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) sample_ray_f64(xyz, cam, opt, sorted_idx, hash, (int)i, sp_xyz, sp_t, mask);
  });
  return 0;
}

// Per-pixel normalised ray directions (cam2world_ray with the rnorm stand-in).
extern "C" void ora_ray_dirs(const ora_camera* cam, float* dirs) {
  for (int v = 0; v < cam->height; v++)
    for (int u = 0; u < cam->width; u++) {
      Ray<float> r;
      make_ray<float>(cam, u, v, nullptr, &r);
      float* d = dirs + 3 * ((size_t)v * cam->width + u);
      d[0] = r.d[0], d[1] = r.d[1], d[2] = r.d[2];
    }
}

// ---------------------------------------------------------------------------
// ray query (epcq_render_topk.cu:222-283)
// ---------------------------------------------------------------------------
extern "C" int ora_quick_query_dirs(const float* xyz, int64_t n_points, const ora_camera* cam,
                                    const ora_options* opt, const int32_t* sorted_idx, const int32_t* hash,
                                    const int32_t* ray_ids, int64_t n_rays, const float* dirs, int32_t* out,
                                    int32_t* count, float* margin) {
  (void)n_points;
  const int W = cam->width, H = cam->height, k = opt->kernel_size, k2 = k * k;
  const int cap = opt->num_point_per_ray;
  if (W <= 0 || H <= 0 || k < 1 || cap < 0) return -1;
  const float r_thr = opt->radius_threshold;
  for (int64_t i = 0; i < n_rays; i++) {
    int32_t* row = out + (size_t)i * cap;
    for (int q = 0; q < cap; q++) row[q] = -1;
    int n_out = 0;
    float mg = 1e30f;
    const int ray = ray_ids[i];
    if (ray < 0 || (int64_t)ray >= (int64_t)W * H) {
      count[i] = 0;
      if (margin) margin[i] = mg;
      continue;
    }
    const int u = ray % W, v = ray / W;
    Ray<float> rr;
    make_ray<float>(cam, u, v, dirs ? dirs + 3 * (size_t)ray : nullptr, &rr);
    const double scale = 1.0 + std::fabs(rr.o[0]) + std::fabs(rr.o[1]) + std::fabs(rr.o[2]);
    for (int l = 0; l < k2; l++) {
      int vv, uu;
      window_cell(v, u, k, H, W, l, &vv, &uu);
      const int32_t start = hash[2 * ((size_t)vv * W + uu)], cnt = hash[2 * ((size_t)vv * W + uu) + 1];
      if (cnt < 0) continue;
      int nl = 0;
      for (int j = start; j <= start + cnt - 1 && nl < kQueryPerCell; j++) {
        float t, dist;
        intersect<float>(rr, xyz + 3 * (size_t)sorted_idx[j], &t, &dist);
        note(&mg, (dist - r_thr) / scale);
        if (dist < r_thr) {
          if (n_out < cap) row[n_out] = sorted_idx[j];
          n_out++;
          nl++;
        }
      }
    }
    count[i] = n_out < cap ? n_out : cap;
    if (margin) margin[i] = mg;
  }
  return 0;
}

extern "C" int ora_quick_query(const float* xyz, int64_t n_points, const ora_camera* cam, const ora_options* opt,
                               const int32_t* sorted_idx, const int32_t* hash, const int32_t* ray_ids,
                               int64_t n_rays, int32_t* out, int32_t* count, float* margin) {
  return ora_quick_query_dirs(xyz, n_points, cam, opt, sorted_idx, hash, ray_ids, n_rays, nullptr, out, count,
                              margin);
}

// ---------------------------------------------------------------------------
// multi-bin z-buffer (rasterization.cu:36-86)
// ---------------------------------------------------------------------------
extern "C" void ora_scatter_multibin(const int32_t* point_idx, const int32_t* point2img, const float* depth,
                                     int64_t n, int32_t height, int32_t width, int32_t bins, float* out_depth,
                                     int32_t* out_idx) {
  const int64_t hw = (int64_t)height * width;
  for (int64_t i = 0; i < hw * bins; i++) out_depth[i] = -1.0f, out_idx[i] = -1;
  std::vector<float> bd(bins);
  std::vector<int32_t> bi(bins);
  int64_t i = 0;
  while (i < n) {
    const int32_t p = point2img[i];
    int64_t j = i;
    while (j < n && point2img[j] == p) j++;
    if (p >= 0 && p < hw) {
      int size = 0, maxi = -1;
      float maxz = -1000.0f;
      for (int64_t q = i; q < j; q++) {
        const float d = depth[q];
        if (d < 0) continue;  // the reference spins here (no advance); skipped instead
        if (size < bins) {
          bd[size] = d;
          bi[size] = point_idx[q];
          if (d > maxz) maxz = d, maxi = size;
          size++;
        } else if (d < maxz) {
          bd[maxi] = d;
          bi[maxi] = point_idx[q];
          maxz = d;
          for (int a = 0; a < bins; a++)
            if (bd[a] > maxz) maxz = bd[a], maxi = a;
        }
      }
      // bubble_sort<PixSpec> ascending by depth (stable)
      for (int a = 0; a < size; a++) {
        bool swapped = false;
        for (int b = 0; b < size - a - 1; b++) {
          if (bd[b] > bd[b + 1]) {
            std::swap(bd[b], bd[b + 1]);
            std::swap(bi[b], bi[b + 1]);
            swapped = true;
          }
        }
        if (!swapped) break;
      }
      for (int a = 0; a < size; a++) out_depth[(size_t)p * bins + a] = bd[a], out_idx[(size_t)p * bins + a] = bi[a];
    }
    i = j;
  }
}
