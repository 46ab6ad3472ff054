// Window search, primary-surface selection, K-sample emission and per-sample
// point selection, fused into one kernel.
//
// Replaces _C.quick_sampling (epcq/csrc/epcq_render_topk.cu:341-417), which
// zero-fills all four outputs, runs quick_sampling_kernel (:82-220, one warp
// per ray, one lane per window cell, a 128-bin shared-memory histogram built
// with float atomics and a serial walk on lane 0) and then
// quick_search_nearby_pc (:10-81, one thread per (ray, sample slot) re-walking
// the window).  Here a CTA owns an 8x32 pixel tile: it stages the points of
// the tile's window halo (clamped to the image) into shared memory once as
// float4 (x, y, z, id) with coalesced gathers (bands of rows when the whole
// halo does not fit), then one thread owns one ray end to end and writes
// every output element of that ray exactly once:
//
//   pass A  kept candidates (ray distance < radius, at most 48 per window cell,
//           cells row-major and clamped, bucket order) -> tmin, tmax
//   pass B  the same candidates binned by int((t - tmin) / t_intvl); instead of
//           a 128-bin histogram the thread keeps the 4 smallest distinct bins
//           (count, distance sum) in registers -- exactly the bins the walk
//           reaches first -- and re-collects further bins only if the walk
//           goes past them
//   walk    bins with >= 2 points in ascending order: alpha = gamma *
//           exp(-mean_dist / alpha_g), emit when alpha * T > 1e-3, T -= alpha,
//           stop when T < 1e-3 or S samples are out
//   ball    per emitted sample, the reference's 8-entry id buffer over the
//           whole window (including its quirk that, while the buffer fills, the
//           tracked "farthest" entry is the nearest one).  Candidates whose
//           position along the ray is further than radius (+ a rounding
//           margin orders of magnitude above float error) from the sample are
//           skipped before the distance is computed: they cannot be within
//           the radius, so the buffer sees exactly the same sequence.
//
// Each pass walks the ray's window as one flat candidate sequence, and the
// tile's rays are ranked by window size before they are handed to threads, so
// the lanes of a warp run loops of similar length instead of diverging on
// every cell's bucket size.  The radius test decides on the squared distance
// when it is clear of the threshold and calls norm3df only near it (see
// RadiusTest); the mean distance of a bin is computed only for bins the walk
// can reach.  A one-row band whose halo still holds more than kStageCap
// points reads its candidates straight from global memory through the same
// code.
//
// Bin sums are accumulated in window-cell then bucket order; the reference
// adds them with shared-memory atomics in an unspecified order, so a bin's
// mean distance can differ from the reference's in the last bit -- which moves
// an output only if alpha * T or T sits within that bit of 1e-3.
#include <mutex>

#include "hp_common.cuh"

namespace hp {

constexpr int kTileW = 32;   // pixels of one image row per warp
constexpr int kTileH = 8;    // rows per block
constexpr int kThreads = kTileW * kTileH;
constexpr int kHaloMax = (kTileH + kMaxKernel - 1) * (kTileW + kMaxKernel - 1);
constexpr int kCellsPerThread = (kHaloMax + kThreads - 1) / kThreads;
constexpr int kStageCap = 4096;  // staged points per band (64 KB)
constexpr int kBinList = 4;      // distinct t-bins collected per candidate pass
constexpr int kTeReg = 4;        // emitted sample depths kept in registers

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

struct Stage {
  float4 cand[kStageCap];  // x, y, z, id (as int bits; -1 = invalid id)
  int4 work[kThreads / 4]; // per pixel of the tile: (window candidates << 8) | pixel
  int order[kThreads];     // pixel each thread processes, most work first
  int off[kHaloMax + 1];   // staged offset of each halo cell, exclusive prefix
  int start[kHaloMax];     // the cell's first index in sorted_point_idx
  int warp_tot[kThreads / 32];
};

// Clipped bucket range of a hash entry: [x, x + count) within [0, n_sorted).
__device__ __forceinline__ int2 bucket_range(int2 h, int n_sorted) {
  if (h.x < 0 || h.y <= 0 || h.x >= n_sorted) return make_int2(0, 0);
  return make_int2(h.x, h.x + min(h.y, n_sorted - h.x));
}

// Candidates from the tile's shared-memory stage.
struct SrcStaged {
  static constexpr bool kStaged = true;
  const Stage* st;
  int rv0, ru0, nu;
  __device__ __forceinline__ int cell(int vv, int uu) const { return (vv - rv0) * nu + (uu - ru0); }
  __device__ __forceinline__ int2 range(const SampleArgs&, int vv, int uu) const {
    const int c = cell(vv, uu);
    return make_int2(st->off[c], st->off[c + 1]);
  }
  __device__ __forceinline__ float4 fetch(const SampleArgs&, int i) const { return st->cand[i]; }
};

// Candidates straight from global memory (one-row bands whose halo overflows the stage).
struct SrcGlobal {
  static constexpr bool kStaged = false;
  __device__ __forceinline__ int cell(int, int) const { return 0; }
  __device__ __forceinline__ int2 range(const SampleArgs& a, int vv, int uu) const {
    return bucket_range(__ldg(a.hash + (size_t)vv * a.cam.width + uu), a.n_sorted);
  }
  __device__ __forceinline__ float4 fetch(const SampleArgs& a, int j) const {
    const int id = __ldg(a.sidx + j);
    if ((unsigned)id >= (unsigned)a.n_points) return make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    const float4 p = load_point(a.xyz, id);
    return make_float4(p.x, p.y, p.z, __int_as_float(id));
  }
};

// Visit a ray's window candidates in the reference's order -- window rows
// top to bottom, cells left to right (coordinates clamped into the image, so
// border windows repeat cells), entries in bucket order -- calling
// body(point) for each; body returns true when it accepts the candidate, and
// a cell is left once `cap` of its candidates were accepted.
//
// Staged tiles: a window row whose columns need no clamping is a run of
// consecutive halo cells, i.e. one contiguous range of the stage, so the loop
// only watches for cell boundaries (for the cap).  Other rows, and tiles read
// from global memory, go cell by cell.  No integer division per cell.
template <class Src, class Body>
__device__ __forceinline__ void walk_window(const SampleArgs& a, const Src& src, int v, int u, int cap, Body&& body) {
  const int H = a.cam.height, W = a.cam.width, k = a.opt.k;
  const int koff = (k + 1) >> 1, lo = koff - 1, hi = k - koff;
  const bool cols_clamped = (u - lo < 0) || (u + hi > W - 1);
  for (int dv = -lo; dv <= hi; dv++) {
    const int vv = min(max(v + dv, 0), H - 1);
    bool done_row = false;
    if constexpr (Src::kStaged) {
      if (!cols_clamped) {
        const int c0 = src.cell(vv, u - lo);
        const int* off = src.st->off;
        int j = off[c0];
        const int jend = off[c0 + k];
        int c = c0, cell_end = off[c0 + 1], nk = 0;
        while (j < jend) {
          while (j >= cell_end) {  // entered the next non-empty cell
            c++;
            cell_end = off[c + 1];
            nk = 0;
          }
          if (nk >= cap) {
            j = cell_end;
            continue;
          }
          if (body(src.fetch(a, j))) nk++;
          j++;
        }
        done_row = true;
      }
    }
    if (!done_row) {
      for (int du = -lo; du <= hi; du++) {
        const int uu = min(max(u + du, 0), W - 1);
        const int2 rg = src.range(a, vv, uu);
        int nk = 0;
        for (int j = rg.x; j < rg.y && nk < cap; j++)
          if (body(src.fetch(a, j))) nk++;
      }
    }
  }
}

// Fill n elements from p with v using 16-byte stores where aligned.
template <typename T>
__device__ __forceinline__ void fill_run(T* p, int n, T v) {
  constexpr int kVec = 16 / sizeof(T);
  int i = 0;
  while (i < n && (((uintptr_t)(p + i)) & 15) != 0) p[i++] = v;
  if (i + kVec <= n) {
    T vv[kVec];
#pragma unroll
    for (int q = 0; q < kVec; q++) vv[q] = v;
    const int4 pack = *reinterpret_cast<const int4*>(vv);
    for (; i + kVec <= n; i += kVec) *reinterpret_cast<int4*>(p + i) = pack;
  }
  for (; i < n; i++) p[i] = v;
}

// The reference keeps a candidate when norm3df(e) < radius (e = point minus its
// projection on the ray).  The squared length e2 (three roundings) decides it
// without the square root whenever e2 is outside a band of relative width
// 2^-16 around radius^2 -- far wider than the few-ulp errors of e2 and
// norm3df -- and norm3df decides inside the band, so the result is identical.
struct RadiusTest {
  float r, lo2, hi2;
  bool fast;
};

__device__ __forceinline__ RadiusTest make_radius_test(float r) {
  RadiusTest rt;
  rt.r = r;
  const double r2 = (double)r * (double)r;
  rt.fast = r2 > 1e-30 && r2 < 1e30;
  rt.lo2 = (float)(r2 * (1.0 - 1.0 / 65536.0));
  rt.hi2 = (float)(r2 * (1.0 + 1.0 / 65536.0));
  return rt;
}

__device__ __forceinline__ bool within_radius(const RadiusTest& rt, float e0, float e1, float e2) {
  if (rt.fast) {
    const float q = __fmaf_rn(e2, e2, __fmaf_rn(e1, e1, __fmul_rn(e0, e0)));
    if (q < rt.lo2) return true;
    if (q > rt.hi2) return false;
  }
  return norm3df(e0, e1, e2) < rt.r;
}

// PointRayInterset's t (cuda_util.cuh:227); dividing by d.d == 1 is exact, so it is skipped then.
__device__ __forceinline__ float ray_t(const Ray& r, bool unit, float px, float py, float pz, float& s0, float& s1,
                                      float& s2) {
  s0 = __fsub_rn(px, r.o[0]);
  s1 = __fsub_rn(py, r.o[1]);
  s2 = __fsub_rn(pz, r.o[2]);
  const float num = dot3(s0, s1, s2, r.d[0], r.d[1], r.d[2]);
  return unit ? num : __fdiv_rn(num, r.dd);
}

template <class Src>
__device__ __forceinline__ void sample_ray(const SampleArgs& a, const Src& src, int v, int u) {
  const int W = a.cam.width;
  const int ray = v * W + u;
  const int S = a.opt.S, P = a.opt.P;
  const float radius = a.opt.radius;

  Ray r;
  make_ray(a.cam.c2w, a.cam.fx, a.cam.fy, a.cam.cx, a.cam.cy, u, v, r);
  const bool unit = r.dd == 1.0f;
  const RadiusTest rt = make_radius_test(radius);

  // pass A: tmin / tmax over the kept candidates (epcq_render_topk.cu:132-161)
  float tmin = 1e3f, tmax = -1e3f;
  walk_window(a, src, v, u, kKeptPerCell, [&](const float4& p) -> bool {
    if (__float_as_int(p.w) < 0) return false;
    float s0, s1, s2;
    const float t = ray_t(r, unit, p.x, p.y, p.z, s0, s1, s2);
    const float e0 = __fsub_rn(p.x, __fmaf_rn(t, r.d[0], r.o[0]));
    const float e1 = __fsub_rn(p.y, __fmaf_rn(t, r.d[1], r.o[1]));
    const float e2 = __fsub_rn(p.z, __fmaf_rn(t, r.d[2], r.o[2]));
    if (!within_radius(rt, e0, e1, e2)) return false;
    if (tmin > t) tmin = t;
    if (tmax < t) tmax = t;
    return true;
  });

  float* o_xyz = a.sp_xyz + (size_t)ray * S * 3;
  float* o_t = a.sp_t + (size_t)ray * S;
  uint8_t* o_m = a.mask + (size_t)ray * S;
  int* o_idx = a.pc_idx + (size_t)ray * S * P;
  int emitted = 0;
  float te[kTeReg];
#pragma unroll
  for (int q = 0; q < kTeReg; q++) te[q] = 0.0f;

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
      walk_window(a, src, v, u, kKeptPerCell, [&](const float4& p) -> bool {
        if (__float_as_int(p.w) < 0) return false;
        float s0, s1, s2;
        const float t = ray_t(r, unit, p.x, p.y, p.z, s0, s1, s2);
        const float e0 = __fsub_rn(p.x, __fmaf_rn(t, r.d[0], r.o[0]));
        const float e1 = __fsub_rn(p.y, __fmaf_rn(t, r.d[1], r.o[1]));
        const float e2 = __fsub_rn(p.z, __fmaf_rn(t, r.d[2], r.o[2]));
        if (!within_radius(rt, e0, e1, e2)) return false;
        const int b = __float2int_rz(__fdiv_rn(__fsub_rn(t, tmin), a.opt.t_intvl));
        if (b < lo || b >= cut) return true;
        if (m == kBinList && b > lb[kBinList - 1]) {
          cut = b;
          return true;
        }
        const float dist = norm3df(e0, e1, e2);
        bool found = false;
#pragma unroll
        for (int q = 0; q < kBinList; q++)
          if (q < m && lb[q] == b) {
            lc[q] += 1;
            ls[q] = __fadd_rn(ls[q], dist);
            found = true;
          }
        if (found) return true;
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
        return true;
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
#pragma unroll
          for (int e = 0; e < kTeReg; e++)
            if (e == emitted) te[e] = t;
          emitted++;
        }
        transmit = __fsub_rn(transmit, alpha);
      }
      if (done || cut >= kBins) break;
      lo = cut;
    }
  }

  // per-sample point selection (epcq_render_topk.cu:10-81)
  const float omax = fmaxf(fabsf(r.o[0]), fmaxf(fabsf(r.o[1]), fabsf(r.o[2])));
  for (int s = 0; s < emitted; s++) {
    float ts = o_t[s];
#pragma unroll
    for (int e = 0; e < kTeReg; e++)
      if (e == s) ts = te[e];
    const float sx = __fmaf_rn(ts, r.d[0], r.o[0]), sy = __fmaf_rn(ts, r.d[1], r.o[1]),
                sz = __fmaf_rn(ts, r.d[2], r.o[2]);
    // |position along the ray - ts| beyond this cannot be within the radius
    const float reach = radius * 1.001f + 1e-5f * (1.0f + fabsf(ts) + omax);
    float bd[kBallBuf];
    int bi[kBallBuf];
#pragma unroll
    for (int q = 0; q < kBallBuf; q++) bd[q] = 0.0f, bi[q] = -1;
    int bsize = 0, maxi = 0;
    float maxd = 1e3f;
    walk_window(a, src, v, u, 0x7fffffff, [&](const float4& p) -> bool {
      const int id = __float_as_int(p.w);
      if (id < 0) return false;
      const float along = dot3(p.x - r.o[0], p.y - r.o[1], p.z - r.o[2], r.d[0], r.d[1], r.d[2]);
      if (fabsf(along - ts) > reach) return false;
      const float dist = norm3df(__fsub_rn(sx, p.x), __fsub_rn(sy, p.y), __fsub_rn(sz, p.z));
      if (!(dist < radius)) return false;
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
      return false;
    });
    int* row = o_idx + (size_t)s * P;
#pragma unroll
    for (int q = 0; q < kBallBuf; q++)
      if (q < P) row[q] = q < bsize ? bi[q] : -1;
    if (P > kBallBuf) fill_run(row + kBallBuf, P - kBallBuf, -1);
  }

  // defaults for the slots nothing was emitted into
  if (emitted < S) {
    fill_run(o_xyz + emitted * 3, (S - emitted) * 3, 0.0f);
    fill_run(o_t + emitted, S - emitted, 0.0f);
    fill_run(o_m + emitted, S - emitted, (uint8_t)0);
    fill_run(o_idx + (size_t)emitted * P, (S - emitted) * P, -1);
  }
}

// Cell table of the halo of rows [vb, vb + rows) of the tile's columns: global
// start and clipped count per halo cell, block-wide exclusive prefix in
// st.off.  Returns the number of points in the halo (every thread gets it).
struct Band {
  int vb, rows, rv0, ru0, nu, ncells;
};

__device__ __forceinline__ int stage_table(const SampleArgs& a, Stage& st, Band& bd, int u0) {
  const int W = a.cam.width, H = a.cam.height, k = a.opt.k;
  const int koff = (k + 1) >> 1, lo = koff - 1, hi = k - koff;
  bd.rv0 = max(0, bd.vb - lo);
  const int rv1 = min(H - 1, bd.vb + bd.rows - 1 + hi);
  bd.ru0 = max(0, u0 - lo);
  const int ru1 = min(W - 1, u0 + kTileW - 1 + hi);
  bd.nu = ru1 - bd.ru0 + 1;
  bd.ncells = (rv1 - bd.rv0 + 1) * bd.nu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int cnt[kCellsPerThread];
  int local = 0;
#pragma unroll
  for (int q = 0; q < kCellsPerThread; q++) {
    const int c = tid * kCellsPerThread + q;
    cnt[q] = 0;
    if (c < bd.ncells) {
      const int vv = bd.rv0 + c / bd.nu, uu = bd.ru0 + c % bd.nu;
      const int2 rg = bucket_range(__ldg(a.hash + (size_t)vv * W + uu), a.n_sorted);
      st.start[c] = rg.x;
      // capped so the prefix cannot overflow; a capped cell alone exceeds the stage
      cnt[q] = min(rg.y - rg.x, kStageCap + 1);
    }
    local += cnt[q];
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();  // previous readers of st are done
  if (lane == 31) st.warp_tot[warp] = incl;
  __syncthreads();
  int base = incl - local;
  for (int q = 0; q < warp; q++) base += st.warp_tot[q];
  int total = 0;
#pragma unroll
  for (int q = 0; q < kThreads / 32; q++) total += st.warp_tot[q];
#pragma unroll
  for (int q = 0; q < kCellsPerThread; q++) {
    const int c = tid * kCellsPerThread + q;
    if (c < bd.ncells) st.off[c] = base;
    base += cnt[q];
  }
  if (tid == 0) st.off[bd.ncells] = total;
  __syncthreads();
  return total;
}

__device__ __forceinline__ void stage_points(const SampleArgs& a, Stage& st, const Band& bd, int total) {
  for (int i = threadIdx.x; i < total; i += kThreads) {
    int lo_c = 0, hi_c = bd.ncells;  // off[lo_c] <= i < off[hi_c]
    while (hi_c - lo_c > 1) {
      const int mid = (lo_c + hi_c) >> 1;
      if (st.off[mid] <= i)
        lo_c = mid;
      else
        hi_c = mid;
    }
    const int id = __ldg(a.sidx + st.start[lo_c] + (i - st.off[lo_c]));
    float4 p = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    if ((unsigned)id < (unsigned)a.n_points) {
      const float4 q = load_point(a.xyz, id);
      p = make_float4(q.x, q.y, q.z, __int_as_float(id));
    }
    st.cand[i] = p;
  }
  __syncthreads();
}

// A CTA owns an 8x32 tile.  It stages the halo of the whole tile when it fits
// in the stage, otherwise of bands of 4, 2 or 1 rows in turn (a one-row band
// that still overflows reads global memory).  The band's rays are ranked by
// window size and handed out most-work-first.
__global__ void __launch_bounds__(kThreads, 3) k_quick_sampling(SampleArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Stage& st = *reinterpret_cast<Stage*>(smem_raw);
  const int W = a.cam.width, H = a.cam.height, k = a.opt.k;
  const int v0 = blockIdx.y * kTileH, u0 = blockIdx.x * kTileW;
  const int v_end = min(H, v0 + kTileH);
  const int tid = threadIdx.x;
  for (int vb = v0; vb < v_end;) {
    Band bd;
    bd.vb = vb;
    bd.rows = v_end - vb;
    int total = stage_table(a, st, bd, u0);
    while (total > kStageCap && bd.rows > 1) {
      bd.rows = (bd.rows + 1) >> 1;
      total = stage_table(a, st, bd, u0);
    }
    const bool staged = total <= kStageCap;
    if (staged) stage_points(a, st, bd, total);
    const int nrays = bd.rows * kTileW;
    // rank the band's rays by window size (most work first)
    {
      const int pu = u0 + (tid & 31), pv = vb + (tid >> 5);
      int work = 0;
      if (tid < nrays && pu < W) {
        work = 1;
        if (staged) {
          const SrcStaged ss{&st, bd.rv0, bd.ru0, bd.nu};
          for (int l = 0; l < k * k; l++) {
            int vv, uu;
            window_cell(pv, pu, k, H, W, l, vv, uu);
            const int2 rg = ss.range(a, vv, uu);
            work += rg.y - rg.x;
          }
        }
      }
      int* work_flat = reinterpret_cast<int*>(st.work);
      work_flat[tid] = (min(work, 0x7fffff) << 8) | tid;
      __syncthreads();
      const int mine = work_flat[tid];
      int rank = 0;
#pragma unroll 8
      for (int q = 0; q < kThreads / 4; q++) {
        const int4 w4 = st.work[q];
        rank += (w4.x > mine) + (w4.y > mine) + (w4.z > mine) + (w4.w > mine);
      }
      st.order[rank] = tid;
      __syncthreads();
    }
    const int px = st.order[tid];
    const int u = u0 + (px & 31), v = vb + (px >> 5);
    if (px < nrays && u < W) {
      if (staged)
        sample_ray(a, SrcStaged{&st, bd.rv0, bd.ru0, bd.nu}, v, u);
      else
        sample_ray(a, SrcGlobal{}, v, u);
    }
    vb += bd.rows;
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

// The stage exceeds the 48 KB default of dynamic shared memory: opt the kernel
// in once per device.
int32_t allow_stage_smem() {
  static std::mutex mu;
  static bool done[128] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return set_error(HP_ERR_CUDA, "hp_quick_sampling: cudaGetDevice failed");
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_quick_sampling, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Stage));
    if (e != cudaSuccess) return set_error(HP_ERR_CUDA, "hp_quick_sampling: cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    done[dev] = true;
  }
  return HP_OK;
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
  if (int32_t rc = allow_stage_smem()) return rc;
  k_quick_sampling<<<grid, kThreads, sizeof(Stage), (cudaStream_t)stream>>>(a);
  return check_launch("k_quick_sampling");
}

extern "C" int32_t hp_ray_directions(const hp_camera* cam, float* dirs, hp_stream_t stream) {
  if (int32_t rc = check_camera(cam, "hp_ray_directions")) return rc;
  if (!dirs) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_ray_directions: dirs is NULL");
  const int hw = cam->width * cam->height;
  k_ray_directions<<<(hw + 255) / 256, 256, 0, (cudaStream_t)stream>>>(dev_camera(cam), dirs);
  return check_launch("k_ray_directions");
}
