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
// float4 (x, y, z, id) with coalesced gathers, then one thread owns one ray
// end to end and writes every output element of that ray exactly once:
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
//           tracked "farthest" entry is the nearest one), all samples of a ray
//           in one walk.  Candidates whose position along the ray is further
//           than radius (+ a rounding margin orders of magnitude above float
//           error) from a sample are skipped for it before the distance is
//           computed: they cannot be within the radius, so each buffer sees
//           exactly the same sequence.
//
// Each pass walks the ray's window as one flat candidate sequence, and the
// tile's rays are ranked by window size before they are handed to threads, so
// the lanes of a warp run loops of similar length instead of diverging on
// every cell's bucket size.  The radius test decides on the squared distance
// when it is clear of the threshold and calls norm3df only near it (see
// RadiusTest); the mean distance of a bin is computed only for bins the walk
// can reach.  Tiles
// whose halo holds more points than the stage read candidates straight from
// global memory through the same code.
//
// Bin sums are accumulated in window-cell then bucket order; the reference
// adds them with shared-memory atomics in an unspecified order, so a bin's
// mean distance can differ from the reference's in the last bit -- which moves
// an output only if alpha * T or T sits within that bit of 1e-3.
#include <cstdio>
#include <mutex>

#include "hp_common.cuh"

namespace hp {

#ifndef HP_BIN_LIST
#define HP_BIN_LIST 6
#endif
constexpr int kBinList = HP_BIN_LIST;  // distinct t-bins collected per candidate pass
constexpr int kTeReg = 4;        // emitted sample depths kept in registers
constexpr int kBallPass = 2;     // samples served by one ball-query walk
constexpr int kHeavyWindow = 320;  // default: rays with more window candidates get a whole warp
constexpr int kMaxHeavyWindow = 4096;  // largest tunable threshold
constexpr int kMaskWords = (kHeavyWindow + 31) / 32;  // kept-candidate mask of a thread-served ray (larger windows run unmasked)
constexpr int kClasses = 64;     // window-size classes used to group a tile's rays
constexpr int kWalkBatch = 4;    // bins whose sums one walk pass of a warp-served ray gathers

struct SampleArgs {
  const float* __restrict__ xyz;
  const int* __restrict__ sidx;
  const float4* __restrict__ pts;  // sorted_point_idx packed: (x, y, z, id as int bits; -1 = invalid)
  const int2* __restrict__ hash;
  int n_points;  // ids outside [0, n_points) are skipped
  int n_sorted;  // bucket ranges are clipped to [0, n_sorted)
  DevCamera cam;
  DevOptions opt;
  float* __restrict__ sp_xyz;
  int* __restrict__ pc_idx;
  float* __restrict__ sp_t;
  uint8_t* __restrict__ mask;
  int heavy;  // rays with more window candidates than this are served by a whole warp
};

// Stage configurations: kCap staged points per tile, kBlocks resident blocks
// per SM, and the tile: kTileH rows x kTileW pixels, one thread per pixel
// (kThreads = 256 or 128 threads per block).  Shared memory per SM bounds
// stage and blocks together, and registers per thread follow from the
// resident threads: 64 at 4 x 256 or 8 x 128, 80 at 3 x 256 or 6 x 128, 128 at
// 2 x 256.  A larger stage splits fewer dense tiles into row bands (less
// re-staging of shared halo rows) but keeps fewer warps resident; a square
// tile stages a smaller window halo per ray (20 x 20 cells for 256 rays
// against 12 x 36 at k = 5).  Which wins depends on how the cloud's points
// spread over the image, so the launch picks one (hp_tuning.stage_config) and
// hashpoint.batch.Autotuner searches them.  (128-thread blocks on 8 x 16 tiles
// -- 4 warps waiting at a tile's end instead of 8, for a 12 x 20 halo per 128
// rays -- measured 3-5% slower on the shapes views and 12-17% on the clustered
// ones, with 1216 points x 8 blocks and 1856 x 6, so none is offered.)
template <int kCap_, int kBlocks_, int kTileH_, int kTileW_>
struct StageCfg {
  static constexpr int kCap = kCap_;
  static constexpr int kBlocks = kBlocks_;
  static constexpr int kTileH = kTileH_;
  static constexpr int kTileW = kTileW_;
  static constexpr int kThreads = kTileH * kTileW;
  static constexpr int kHaloMax = (kTileH + kMaxKernel - 1) * (kTileW + kMaxKernel - 1);
  static constexpr int kItemsPerTile = kTileH * 4;  // rows, each in up to four column quarters
  static_assert((kThreads == 256 || kThreads == 128) && kTileW >= 4 && kTileW <= 32 && kTileH <= 16, "tile shape");
};
using Cfg2560x4 = StageCfg<2560, 4, 8, 32>;     // 40 KB stage, 4 blocks per SM, 8 x 32 tiles
using Cfg3712x3 = StageCfg<3712, 3, 8, 32>;     // 58 KB stage, 3 blocks per SM
using Cfg5888x2 = StageCfg<5888, 2, 8, 32>;     // 92 KB stage, 2 blocks per SM
using Cfg2560x4Sq = StageCfg<2560, 4, 16, 16>;  // 16 x 16 tiles
using Cfg3712x3Sq = StageCfg<3712, 3, 16, 16>;
constexpr int kStageConfigs = 5;      // hp_tuning.stage_config 1..5 (0 = the default)
// The default: 16 x 16 tiles with 2560 staged points x 4 blocks, measured
// fastest or level on the shapes, clustered and multi-view workloads (the
// small sphere view prefers 5888 x 2, which a tuner finds).
constexpr int kDefaultStageConfig = 4;
constexpr int kMaxItemsPerTile = 64;  // over the configurations (16 rows, four column ranges each)
constexpr int kCellsPerThread = 2;    // halo cells per thread (<= 432 = the largest halo)

template <class Cfg>
struct Stage {
  float4 cand[Cfg::kCap];   // x, y, z, id (as int bits; -1 = invalid id)
  int cls[kClasses];        // rays per window-size class
  int cls_base[kClasses];   // first rank of each class
  int order[Cfg::kThreads];  // pixel of each rank, heaviest class first
  int off[Cfg::kHaloMax + 1];  // staged offset of each halo cell, exclusive prefix
  int start[Cfg::kHaloMax];    // the cell's first index in sorted_point_idx
  int warp_tot[Cfg::kThreads / 32];
  int next_unit;            // next work unit of the tile (see process_tile)
  unsigned kept[kMaskWords][Cfg::kThreads];  // per thread: window positions pass A accepted
};
// kBlocks CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA)
template <class Cfg>
constexpr bool fits_sm() {
  return Cfg::kBlocks * (sizeof(Stage<Cfg>) + 16 + 1024) <= 228 * 1024 && Cfg::kItemsPerTile <= kMaxItemsPerTile &&
         Cfg::kHaloMax <= kCellsPerThread * Cfg::kThreads;
}
static_assert(fits_sm<Cfg2560x4>() && fits_sm<Cfg3712x3>() && fits_sm<Cfg5888x2>() && fits_sm<Cfg2560x4Sq>() &&
                  fits_sm<Cfg3712x3Sq>(),
              "a stage configuration exceeds the shared memory of its blocks per SM");

// Clipped bucket range of a hash entry: [x, x + count) within [0, n_sorted).
__device__ __forceinline__ int2 bucket_range(int2 h, int n_sorted) {
  if (h.x < 0 || h.y <= 0 || h.x >= n_sorted) return make_int2(0, 0);
  return make_int2(h.x, h.x + min(h.y, n_sorted - h.x));
}

// Candidates from the tile's shared-memory stage.
template <class Cfg>
struct SrcStaged {
  static constexpr bool kStaged = true;
  static constexpr int kKeptStride = Cfg::kThreads;  // the kept masks' word stride (one column per thread)
  const Stage<Cfg>* st;
  int rv0, ru0, nu;
  __device__ __forceinline__ int cell(int vv, int uu) const { return (vv - rv0) * nu + (uu - ru0); }
  __device__ __forceinline__ int2 range(const SampleArgs&, int vv, int uu) const {
    const int c = cell(vv, uu);
    return make_int2(st->off[c], st->off[c + 1]);
  }
  __device__ __forceinline__ float4 fetch(const SampleArgs&, int i) const { return st->cand[i]; }
};

// Candidates straight from global memory (tiles whose halo overflows the stage).
struct SrcGlobal {
  static constexpr bool kStaged = false;
  static constexpr int kKeptStride = 1;  // no kept masks
  __device__ __forceinline__ int cell(int, int) const { return 0; }
  __device__ __forceinline__ int2 range(const SampleArgs& a, int vv, int uu) const {
    return bucket_range(__ldg(a.hash + (size_t)vv * a.cam.width + uu), a.n_sorted);
  }
  __device__ __forceinline__ float4 fetch(const SampleArgs& a, int j) const { return __ldg(a.pts + j); }
};

// Pack the candidates once per launch: pts[j] = (xyz of sorted_point_idx[j],
// its id), or id -1 when the id is outside [0, n_points).  Every later fetch
// of candidate j -- staging or global -- is then one 16-byte load instead of
// an id load and a dependent point gather.
__device__ __forceinline__ float4 packed_point(const int* __restrict__ sidx, int j, const float* __restrict__ xyz,
                                               int n_points) {
  const int id = __ldg(sidx + j);
  float4 p = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
  if ((unsigned)id < (unsigned)n_points) {
    const float4 q = load_point(xyz, id);
    p = make_float4(q.x, q.y, q.z, __int_as_float(id));
  }
  return p;
}

// Candidates [j0, j1) packed by one warp, four per lane in flight.
__device__ __forceinline__ void pack_range(const int* __restrict__ sidx, int j0, int j1, const float* __restrict__ xyz,
                                           int n_points, float4* __restrict__ pts) {
  const int lane = threadIdx.x & 31;
  for (int j = j0 + lane; j < j1; j += 128) {
    float4 p[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (j + 32 * q < j1) p[q] = packed_point(sidx, j + 32 * q, xyz, n_points);
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (j + 32 * q < j1) pts[j + 32 * q] = p[q];
  }
}

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

// Staged tiles, unclamped window columns: the same visit as walk_window's
// fast path, also passing each candidate's position f in the window's
// candidate sequence (window rows concatenated, entries in stage order).
template <class Src, class Body>
__device__ __forceinline__ void walk_rows(const SampleArgs& a, const Src& src, int v, int u, int cap, Body&& body) {
  const int H = a.cam.height, k = a.opt.k;
  const int lo = ((k + 1) >> 1) - 1;
  const int* off = src.st->off;
  int f0 = 0;
  for (int r = 0; r < k; r++) {
    const int c0 = src.cell(min(max(v - lo + r, 0), H - 1), u - lo);
    const int jb = off[c0], jend = off[c0 + k];
    int j = jb, c = c0, cell_end = off[c0 + 1], nk = 0;
    while (j < jend) {
      while (j >= cell_end) {
        c++;
        cell_end = off[c + 1];
        nk = 0;
      }
      if (nk >= cap) {
        j = cell_end;
        continue;
      }
      if (body(src.fetch(a, j), f0 + (j - jb))) nk++;
      j++;
    }
    f0 += jend - jb;
  }
}

// Visit the candidates whose window positions are set in a kept mask (nw
// words, stride Src::kKeptStride), in order; the position is mapped back to the stage
// row by row.
template <class Src, class Body>
__device__ __forceinline__ void walk_kept(const SampleArgs& a, const Src& src, int v, int u, const unsigned* mask,
                                          int nw, Body&& body) {
  const int H = a.cam.height, k = a.opt.k;
  const int lo = ((k + 1) >> 1) - 1;
  const int* off = src.st->off;
  int r = -1, rf0 = 0, rf1 = 0, jb = 0;
  for (int w = 0; w < nw; w++) {
    unsigned m = mask[w * Src::kKeptStride];
    while (m) {
      const int f = (w << 5) + __ffs(m) - 1;
      m &= m - 1;
      while (f >= rf1) {
        r++;
        const int c0 = src.cell(min(max(v - lo + r, 0), H - 1), u - lo);
        jb = off[c0];
        rf0 = rf1;
        rf1 += off[c0 + k] - jb;
      }
      body(src.fetch(a, jb + (f - rf0)));
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

// t-bin index int((t - tmin) / t_intvl) of a kept candidate (x = t - tmin >= 0).
// y = x * RN(1 / t_intvl) is within 3.1 * 2^-24 * q of the quotient q and of
// its rounding RN(q), so when y widened by 2^-21 relative on both sides
// truncates to one integer, that integer is int(RN(q)); otherwise (a bin
// edge within a few ulps) the division is done exactly.
struct BinDiv {
  float intvl, inv;
  bool fast;
};

__device__ __forceinline__ BinDiv make_bin_div(float intvl) {
  BinDiv bd;
  bd.intvl = intvl;
  bd.inv = __frcp_rn(intvl);
  bd.fast = intvl > 0.0f && bd.inv < 0x1p100f && intvl < 0x1p100f;
  return bd;
}

__device__ __forceinline__ int bin_index(const BinDiv& bd, float x) {
  if (bd.fast) {
    const float y = __fmul_rn(x, bd.inv);
    const int lo = __float2int_rz(__fmul_rn(y, 1.0f - 0x1p-21f));
    if (lo == __float2int_rz(__fmul_rn(y, 1.0f + 0x1p-21f))) return lo;
  }
  return __float2int_rz(__fdiv_rn(x, bd.intvl));
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

// `kept` (staged tiles only; else null) is this thread's kept-candidate mask
// (kMaskWords words, stride Src::kKeptStride).  For windows with unclamped columns and
// at most kMaskWords * 32 candidates, pass A records the positions it keeps
// there and pass B visits only those, without the radius test or the cap.
template <class Src>
__device__ __forceinline__ void sample_ray(const SampleArgs& a, const Src& src, int v, int u, unsigned* kept) {
  const int W = a.cam.width;
  const int ray = v * W + u;
  const int S = a.opt.S, P = a.opt.P;
  const float radius = a.opt.radius;

  Ray r;
  make_ray(a.cam.c2w, a.cam.fx, a.cam.fy, a.cam.cx, a.cam.cy, u, v, r);
  const bool unit = r.dd == 1.0f;
  const RadiusTest rt = make_radius_test(radius);

  // the window's candidate count when the kept mask is used, else -1
  int masked_T = -1;
  if constexpr (Src::kStaged) {
    const int k = a.opt.k, lo = ((k + 1) >> 1) - 1, hi = k - 1 - lo;
    if (kept && u - lo >= 0 && u + hi <= W - 1) {
      int T = 0;
      for (int q = 0; q < k; q++) {
        const int c0 = src.cell(min(max(v - lo + q, 0), a.cam.height - 1), u - lo);
        T += src.st->off[c0 + k] - src.st->off[c0];
      }
      if (T <= kMaskWords * 32) {
        masked_T = T;
        for (int w = 0; w < (T + 31) >> 5; w++) kept[w * Src::kKeptStride] = 0u;
      }
    }
  }

  // pass A: tmin / tmax over the kept candidates (epcq_render_topk.cu:132-161)
  float tmin = 1e3f, tmax = -1e3f;
  auto keep = [&](const float4& p) -> bool {
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
  };
  bool masked = false;
  if constexpr (Src::kStaged) {
    if (masked_T >= 0) {
      masked = true;
      unsigned word = 0u;
      int wi = 0;
      walk_rows(a, src, v, u, kKeptPerCell, [&](const float4& p, int f) -> bool {
        if (!keep(p)) return false;
        if ((f >> 5) != wi) {
          if (word) kept[wi * Src::kKeptStride] = word;
          wi = f >> 5;
          word = 0u;
        }
        word |= 1u << (f & 31);
        return true;
      });
      if (word) kept[wi * Src::kKeptStride] = word;
    }
  }
  if (!masked) walk_window(a, src, v, u, kKeptPerCell, keep);

  float* o_xyz = a.sp_xyz + (size_t)ray * S * 3;
  float* o_t = a.sp_t + (size_t)ray * S;
  uint8_t* o_m = a.mask + (size_t)ray * S;
  int* o_idx = a.pc_idx + (size_t)ray * S * P;
  int emitted = 0;
  float te[kTeReg];
#pragma unroll
  for (int q = 0; q < kTeReg; q++) te[q] = 0.0f;

  if (!(tmin > tmax)) {
    const BinDiv bdiv = make_bin_div(a.opt.t_intvl);
    float transmit = 1.0f;
    int lo = 0;
    for (;;) {
      // pass B: the kBinList smallest distinct bins in [lo, cut) with full stats
      int lb[kBinList], lc[kBinList];
      float ls[kBinList];
#pragma unroll
      for (int q = 0; q < kBinList; q++) lb[q] = 0x7fffffff, lc[q] = 0, ls[q] = 0.0f;
      int m = 0, cut = kBins;
      // a kept candidate at depth t: into the list if its bin is among the
      // kBinList smallest in [lo, cut); dist() gives its distance to the ray
      auto collect = [&](float t, auto&& dist) {
        const int b = bin_index(bdiv, __fsub_rn(t, tmin));
        if (b < lo || b >= cut) return;
        if (m == kBinList && b > lb[kBinList - 1]) {
          cut = b;
          return;
        }
        const float d = dist();
        bool found = false;
#pragma unroll
        for (int q = 0; q < kBinList; q++)
          if (q < m && lb[q] == b) {
            lc[q] += 1;
            ls[q] = __fadd_rn(ls[q], d);
            found = true;
          }
        if (found) return;
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
            ls[q] = d;
          }
        }
        m = m < kBinList ? m + 1 : kBinList;
      };
      bool visited = false;
      if constexpr (Src::kStaged) {
        if (masked) {
          visited = true;
          walk_kept(a, src, v, u, kept, (masked_T + 31) >> 5, [&](const float4& p) {
            float s0, s1, s2;
            const float t = ray_t(r, unit, p.x, p.y, p.z, s0, s1, s2);
            collect(t, [&] {
              return norm3df(__fsub_rn(p.x, __fmaf_rn(t, r.d[0], r.o[0])), __fsub_rn(p.y, __fmaf_rn(t, r.d[1], r.o[1])),
                             __fsub_rn(p.z, __fmaf_rn(t, r.d[2], r.o[2])));
            });
          });
        }
      }
      if (!visited) {
        walk_window(a, src, v, u, kKeptPerCell, [&](const float4& p) -> bool {
          if (__float_as_int(p.w) < 0) return false;
          float s0, s1, s2;
          const float t = ray_t(r, unit, p.x, p.y, p.z, s0, s1, s2);
          const float e0 = __fsub_rn(p.x, __fmaf_rn(t, r.d[0], r.o[0]));
          const float e1 = __fsub_rn(p.y, __fmaf_rn(t, r.d[1], r.o[1]));
          const float e2 = __fsub_rn(p.z, __fmaf_rn(t, r.d[2], r.o[2]));
          if (!within_radius(rt, e0, e1, e2)) return false;
          collect(t, [&] { return norm3df(e0, e1, e2); });
          return true;
        });
      }
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

  // per-sample point selection (epcq_render_topk.cu:10-81).  One walk over the
  // window serves up to kBallPass samples: each candidate's position along the
  // ray is compared with every sample's reach (samples are in ascending t), and
  // only candidates within a sample's reach get the exact distance.  The
  // per-sample buffers live in a small local array touched only on hits.
  const float omax = fmaxf(fabsf(r.o[0]), fmaxf(fabsf(r.o[1]), fabsf(r.o[2])));
  for (int s0 = 0; s0 < emitted; s0 += kBallPass) {
    const int ns = min(kBallPass, emitted - s0);
    float ts[kBallPass], reach[kBallPass], spx[kBallPass], spy[kBallPass], spz[kBallPass], maxd[kBallPass];
    float bd[kBallPass][kBallBuf];
    int bi[kBallPass][kBallBuf], bsize[kBallPass], maxi[kBallPass];
#pragma unroll
    for (int q = 0; q < kBallPass; q++) {
      float t = 0.0f;
      if (q < ns) {
        t = o_t[s0 + q];
#pragma unroll
        for (int e = 0; e < kTeReg; e++)
          if (e == s0 + q) t = te[e];
      }
      ts[q] = t;
      // |position along the ray - t| beyond this cannot be within the radius
      reach[q] = q < ns ? radius * 1.001f + 1e-5f * (1.0f + fabsf(t) + omax) : -1.0f;
      spx[q] = __fmaf_rn(t, r.d[0], r.o[0]);
      spy[q] = __fmaf_rn(t, r.d[1], r.o[1]);
      spz[q] = __fmaf_rn(t, r.d[2], r.o[2]);
      bsize[q] = 0;
      maxi[q] = 0;
      maxd[q] = 1e3f;
#pragma unroll
      for (int e = 0; e < kBallBuf; e++) bd[q][e] = 0.0f, bi[q][e] = -1;
    }
    const float t_first = ts[0] - reach[0], t_last = ts[ns - 1 > 0 ? 1 : 0] + reach[ns - 1 > 0 ? 1 : 0];
    walk_window(a, src, v, u, 0x7fffffff, [&](const float4& p) -> bool {
      const int id = __float_as_int(p.w);
      if (id < 0) return false;
      const float along = dot3(p.x - r.o[0], p.y - r.o[1], p.z - r.o[2], r.d[0], r.d[1], r.d[2]);
      if (along < t_first || along > t_last) return false;
#pragma unroll
      for (int q = 0; q < kBallPass; q++) {
        if (!(fabsf(along - ts[q]) <= reach[q])) continue;
        const float dist = norm3df(__fsub_rn(spx[q], p.x), __fsub_rn(spy[q], p.y), __fsub_rn(spz[q], p.z));
        if (!(dist < radius)) continue;
        if (bsize[q] < kBallBuf) {
          bd[q][bsize[q]] = dist;  // one indexed store into the local-memory buffer
          bi[q][bsize[q]] = id;
          if (maxd[q] > dist) {
            maxd[q] = dist;
            maxi[q] = bsize[q];
          }
          bsize[q]++;
        } else if (dist < maxd[q]) {
          bd[q][maxi[q]] = dist;
          bi[q][maxi[q]] = id;
          float md = dist;
          int mi = maxi[q];
#pragma unroll
          for (int e = 0; e < kBallBuf; e++)
            if (bd[q][e] > md) {
              md = bd[q][e];
              mi = e;
            }
          maxd[q] = md;
          maxi[q] = mi;
        }
      }
      return false;
    });
#pragma unroll
    for (int q = 0; q < kBallPass; q++) {
      if (q >= ns) break;
      int* row = o_idx + (size_t)(s0 + q) * P;
#pragma unroll
      for (int e = 0; e < kBallBuf; e++)
        if (e < P) row[e] = e < bsize[q] ? bi[q][e] : -1;
      if (P > kBallBuf) fill_run(row + kBallBuf, P - kBallBuf, -1);
    }
  }

  // defaults for the slots nothing was emitted into
  if (emitted < S) {
    fill_run(o_xyz + emitted * 3, (S - emitted) * 3, 0.0f);
    fill_run(o_t + emitted, S - emitted, 0.0f);
    fill_run(o_m + emitted, S - emitted, (uint8_t)0);
    fill_run(o_idx + (size_t)emitted * P, (S - emitted) * P, -1);
  }
}

// Lanes [lo, hi) of a warp as a bit mask (0 <= lo <= hi <= 32).
__device__ __forceinline__ unsigned lane_span(int lo, int hi) {
  const unsigned below_hi = hi >= 32 ? 0xffffffffu : (1u << hi) - 1u;
  const unsigned below_lo = lo >= 32 ? 0xffffffffu : (1u << lo) - 1u;
  return below_hi & ~below_lo;
}

// Warp-cooperative sample_ray.  The ray's k*k window cells (reference order:
// rows, then columns, clamped) are concatenated into one candidate sequence:
// lane c < k*k holds cell c's range and its exclusive prefix, and each chunk
// of 32 consecutive candidates is spread over the lanes, every lane finding its
// cell by a binary search over the prefixes (shuffles).  Everything
// order-dependent reproduces sample_ray exactly: the 48-per-cell cap from
// ballot ranks plus a per-cell carry, bin sums added one candidate at a time
// in sequence order, and the 8-entry ball buffers fed hits in sequence order.
// A ray costs about ceil(candidates / 32) chunks per pass, so heavy rays finish
// in a fraction of the time one thread would need for them.
template <class Src>
__device__ __forceinline__ void sample_ray_warp(const SampleArgs& a, const Src& src, int v, int u, unsigned* wbuf) {
  const unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int W = a.cam.width, H = a.cam.height, k = a.opt.k;
  const int lo = ((k + 1) >> 1) - 1;
  const int ray = v * W + u;
  const int S = a.opt.S, P = a.opt.P;
  const float radius = a.opt.radius;
  Ray r;
  make_ray(a.cam.c2w, a.cam.fx, a.cam.fy, a.cam.cx, a.cam.cy, u, v, r);
  const bool unit = r.dd == 1.0f;
  const RadiusTest rt = make_radius_test(radius);

  // lane c < k*k: cell c's first index and count; exclusive prefix over cells
  int cbase = 0, ccnt = 0;
  if (lane < k * k) {
    const int q = lane / k;
    const int vv = min(max(v + q - lo, 0), H - 1), uu = min(max(u + (lane - q * k) - lo, 0), W - 1);
    const int2 rg = src.range(a, vv, uu);
    cbase = rg.x;
    ccnt = rg.y - rg.x;
  }
  int cpre = ccnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kAll, cpre, o);
    if (lane >= o) cpre += t;
  }
  const int total = __shfl_sync(kAll, cpre, 31);
  cpre -= ccnt;
  const bool capped = __any_sync(kAll, ccnt > kKeptPerCell);

  // body(j0, valid, idx, cell, pc) per lane and chunk: candidate j0 + lane of
  // the sequence, its index for src.fetch, its cell and the cell's first j
  auto chunks = [&](auto&& body) {
    for (int j0 = 0; j0 < total; j0 += 32) {
      const int j = j0 + lane;
      int c = 0;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1)
        if (__shfl_sync(kAll, cpre, c + s) <= j) c += s;
      const int pc = __shfl_sync(kAll, cpre, c);
      const int idx = __shfl_sync(kAll, cbase, c) + (j - pc);
      body(j0, j < total, idx, c, pc);
    }
  };
  // The same for the capped passes (A, B and the walk sums; carry = the
  // pass's per-cell kept counts): when the cell the chunk ended in already
  // has its 48 kept candidates, the rest of it is skipped -- none of them can
  // be kept.
  auto capped_chunks = [&](const int& carry, auto&& body) {
    for (int j0 = 0; j0 < total;) {
      const int j = j0 + lane;
      int c = 0;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1)
        if (__shfl_sync(kAll, cpre, c + s) <= j) c += s;
      const int pc = __shfl_sync(kAll, cpre, c);
      const int idx = __shfl_sync(kAll, cbase, c) + (j - pc);
      body(j0, j < total, idx, c, pc);
      j0 += 32;
      if (capped) {
        const int last = __shfl_sync(kAll, c, 31);
        if (__shfl_sync(kAll, carry, last) >= kKeptPerCell) j0 = max(j0, __shfl_sync(kAll, cpre + ccnt, last));
      }
    }
  };
  // the candidate's t and offset from the ray; true when within the radius
  auto eval = [&](bool valid, int idx, float& t, float& e0, float& e1, float& e2) -> bool {
    if (!valid) return false;
    const float4 p = src.fetch(a, idx);
    if (__float_as_int(p.w) < 0) return false;
    float s0, s1, s2;
    t = ray_t(r, unit, p.x, p.y, p.z, s0, s1, s2);
    e0 = __fsub_rn(p.x, __fmaf_rn(t, r.d[0], r.o[0]));
    e1 = __fsub_rn(p.y, __fmaf_rn(t, r.d[1], r.o[1]));
    e2 = __fsub_rn(p.z, __fmaf_rn(t, r.d[2], r.o[2]));
    return within_radius(rt, e0, e1, e2);
  };
  // kept candidates that are among the first 48 kept of their cell; `carry`
  // (lane c's copy is cell c's) counts a cell's kept candidates of earlier chunks
  auto accept = [&](bool kept, int j0, int cell, int pc, int& carry) -> bool {
    if (!capped) return kept;
    const unsigned m = __ballot_sync(kAll, kept);
    const int before = __shfl_sync(kAll, carry, cell) + __popc(m & below & ~lane_span(0, max(pc - j0, 0)));
    carry += __popc(m & lane_span(min(max(cpre - j0, 0), 32), min(max(cpre + ccnt - j0, 0), 32)));
    return kept && before < kKeptPerCell;
  };
  const BinDiv bdiv = make_bin_div(a.opt.t_intvl);
  auto bin_of = [&](float t, float tmin) {
    return bin_index(bdiv, __fsub_rn(t, tmin));
  };

  // pass A: tmin / tmax
  float tmin = 1e3f, tmax = -1e3f;
  {
    int carry = 0;
    capped_chunks(carry, [&](int j0, bool valid, int idx, int cell, int pc) {
      float t = 0.f, e0, e1, e2;
      if (accept(eval(valid, idx, t, e0, e1, e2), j0, cell, pc, carry)) {
        if (tmin > t) tmin = t;
        if (tmax < t) tmax = t;
      }
    });
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float a0 = __shfl_xor_sync(kAll, tmin, o), a1 = __shfl_xor_sync(kAll, tmax, o);
    if (tmin > a0) tmin = a0;
    if (tmax < a1) tmax = a1;
  }

  float* o_xyz = a.sp_xyz + (size_t)ray * S * 3;
  float* o_t = a.sp_t + (size_t)ray * S;
  uint8_t* o_m = a.mask + (size_t)ray * S;
  int* o_idx = a.pc_idx + (size_t)ray * S * P;
  int emitted = 0;
  float te[kTeReg];
#pragma unroll
  for (int q = 0; q < kTeReg; q++) te[q] = 0.0f;

  if (!(tmin > tmax)) {
    // pass B: which bins hold >= 2 kept points (the only ones the walk uses)
    unsigned s1[kBins / 32], s2[kBins / 32];
#pragma unroll
    for (int q = 0; q < kBins / 32; q++) s1[q] = 0u, s2[q] = 0u;
    {
      int carry = 0;
      capped_chunks(carry, [&](int j0, bool valid, int idx, int cell, int pc) {
        float t = 0.f, e0, e1, e2;
        if (accept(eval(valid, idx, t, e0, e1, e2), j0, cell, pc, carry)) {
          const int b = bin_of(t, tmin);
          if (b < kBins) {
            const unsigned bit = 1u << (b & 31);
#pragma unroll
            for (int q = 0; q < kBins / 32; q++)
              if (q == (b >> 5)) {
                s2[q] |= s1[q] & bit;
                s1[q] |= bit;
              }
          }
        }
      });
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int q = 0; q < kBins / 32; q++) {
        const unsigned o1 = __shfl_xor_sync(kAll, s1[q], o), o2 = __shfl_xor_sync(kAll, s2[q], o);
        s2[q] = s2[q] | o2 | (s1[q] & o1);
        s1[q] |= o1;
      }
    }
    // first bin >= from holding >= 2 points (kBins if none)
    auto next_bin = [&](int from) {
      int b = kBins;
#pragma unroll
      for (int q = kBins / 32 - 1; q >= 0; q--) {
        unsigned m = s2[q];
        if (q * 32 + 32 <= from)
          m = 0u;
        else if (q * 32 < from)
          m &= ~0u << (from - q * 32);
        if (m) b = q * 32 + __ffs(m) - 1;
      }
      return b;
    };
    // walk: the bins' sums are gathered kWalkBatch bins per pass, in ascending order
    float transmit = 1.0f;
    int from = 0;
    bool done = false;
    while (!done) {
      int bb[kWalkBatch];
      int nb = 0;
#pragma unroll
      for (int q = 0; q < kWalkBatch; q++) {
        bb[q] = next_bin(q == 0 ? from : bb[q - 1] + 1);
        nb += bb[q] < kBins ? 1 : 0;
      }
      if (nb == 0) break;
      float bsum[kWalkBatch];
      int bcnt[kWalkBatch];
#pragma unroll
      for (int q = 0; q < kWalkBatch; q++) bsum[q] = 0.0f, bcnt[q] = 0;
      int carry = 0;
      capped_chunks(carry, [&](int j0, bool valid, int idx, int cell, int pc) {
        float t = 0.f, e0 = 0.f, e1 = 0.f, e2 = 0.f;
        int mine = -1;
        float dist = 0.0f;
        if (accept(eval(valid, idx, t, e0, e1, e2), j0, cell, pc, carry)) {
          const int b = bin_of(t, tmin);
#pragma unroll
          for (int q = 0; q < kWalkBatch; q++)
            if (bb[q] == b) mine = q;
          if (mine >= 0) dist = norm3df(e0, e1, e2);
        }
#pragma unroll
        for (int q = 0; q < kWalkBatch; q++) {
          unsigned mm = __ballot_sync(kAll, mine == q);
          while (mm) {
            const int l = __ffs(mm) - 1;
            mm &= mm - 1;
            bsum[q] = __fadd_rn(bsum[q], __shfl_sync(kAll, dist, l));
            bcnt[q]++;
          }
        }
      });
#pragma unroll
      for (int q = 0; q < kWalkBatch; q++) {
        if (q >= nb) break;
        if (transmit < 1e-3f || emitted >= S) {
          done = true;
          break;
        }
        const float sdf = __fdiv_rn(bsum[q], __fadd_rn((float)bcnt[q], 1e-6f));
        const float alpha = __fmul_rn(a.opt.gamma, __expf(__fdiv_rn(-sdf, a.opt.alpha_g)));
        const float weight = __fmul_rn(alpha, transmit);
        if (weight > 1e-3f) {
          const float t = __fmaf_rn((float)bb[q], a.opt.t_intvl, tmin);
          if (lane == 0) {
            o_xyz[emitted * 3 + 0] = __fmaf_rn(t, r.d[0], r.o[0]);
            o_xyz[emitted * 3 + 1] = __fmaf_rn(t, r.d[1], r.o[1]);
            o_xyz[emitted * 3 + 2] = __fmaf_rn(t, r.d[2], r.o[2]);
            o_t[emitted] = t;
            o_m[emitted] = 1;
          }
#pragma unroll
          for (int e = 0; e < kTeReg; e++)
            if (e == emitted) te[e] = t;
          emitted++;
        }
        transmit = __fsub_rn(transmit, alpha);
      }
      if (nb < kWalkBatch) break;
      from = bb[kWalkBatch - 1] + 1;
    }
  }
  __syncwarp();

  // per-sample point selection, two samples per pass, buffers fed hits in
  // order.  The buffers (distance and id of kBallBuf hits per sample) live in
  // the serving warp's 32 words of shared memory (wbuf), written by lane 0;
  // their size, minimum-then-maximum tracking and state are warp-uniform
  // registers.
  static_assert(2 * kBallPass * kBallBuf <= 32, "ball buffers exceed the warp's words");
  float* sbd = reinterpret_cast<float*>(wbuf);              // [kBallPass][kBallBuf] distances
  int* sbi = reinterpret_cast<int*>(wbuf) + kBallPass * kBallBuf;  // [kBallPass][kBallBuf] ids
  const float omax = fmaxf(fabsf(r.o[0]), fmaxf(fabsf(r.o[1]), fabsf(r.o[2])));
  for (int s0 = 0; s0 < emitted; s0 += kBallPass) {
    const int ns = min(kBallPass, emitted - s0);
    float ts[kBallPass], reach[kBallPass], spx[kBallPass], spy[kBallPass], spz[kBallPass], maxd[kBallPass];
    int bsize[kBallPass], maxi[kBallPass];
    bool settled[kBallPass];
#pragma unroll
    for (int q = 0; q < kBallPass; q++) {
      float t = 0.0f;
      if (q < ns) {
        t = o_t[s0 + q];
#pragma unroll
        for (int e = 0; e < kTeReg; e++)
          if (e == s0 + q) t = te[e];
      }
      ts[q] = t;
      reach[q] = q < ns ? radius * 1.001f + 1e-5f * (1.0f + fabsf(t) + omax) : -1.0f;
      spx[q] = __fmaf_rn(t, r.d[0], r.o[0]);
      spy[q] = __fmaf_rn(t, r.d[1], r.o[1]);
      spz[q] = __fmaf_rn(t, r.d[2], r.o[2]);
      bsize[q] = 0;
      maxi[q] = 0;
      maxd[q] = 1e3f;
      settled[q] = false;
    }
    chunks([&](int, bool valid, int idx, int, int) {
      float dq[kBallPass];
      bool hq[kBallPass];
      int id = -1;
#pragma unroll
      for (int q = 0; q < kBallPass; q++) dq[q] = 0.0f, hq[q] = false;
      if (valid) {
        const float4 p = src.fetch(a, idx);
        id = __float_as_int(p.w);
        if (id >= 0) {
          const float along = dot3(p.x - r.o[0], p.y - r.o[1], p.z - r.o[2], r.d[0], r.d[1], r.d[2]);
#pragma unroll
          for (int q = 0; q < kBallPass; q++)
            if (fabsf(along - ts[q]) <= reach[q]) {
              dq[q] = norm3df(__fsub_rn(spx[q], p.x), __fsub_rn(spy[q], p.y), __fsub_rn(spz[q], p.z));
              hq[q] = dq[q] < radius;
            }
        }
      }
#pragma unroll
      for (int q = 0; q < kBallPass; q++) {
        // Which of the chunk's hits can change the buffer (bsize, settled and
        // maxd are the same in every lane).  While filling: all of them.  Once
        // full and replaced at least once, maxd is the buffer's true maximum and
        // only decreases, so only hits below it.  Full but never replaced, maxd
        // is the minimum of the first eight (the reference's quirk) and the
        // buffer stays as it is until a hit falls below it; from that hit on,
        // maxd becomes the true maximum, so every later hit is looked at.
        unsigned mm;
        if (bsize[q] < kBallBuf || settled[q]) {
          mm = __ballot_sync(kAll, hq[q] && (bsize[q] < kBallBuf || dq[q] < maxd[q]));
        } else {
          const unsigned first = __ballot_sync(kAll, hq[q] && dq[q] < maxd[q]);
          const unsigned all = __ballot_sync(kAll, hq[q]);
          mm = first ? all & ~((1u << (__ffs(first) - 1)) - 1u) : 0u;
        }
        while (mm) {
          const int l = __ffs(mm) - 1;
          mm &= mm - 1;
          const float dist = __shfl_sync(kAll, dq[q], l);
          const int cid = __shfl_sync(kAll, id, l);
          if (bsize[q] < kBallBuf) {
            if (lane == 0) {
              sbd[q * kBallBuf + bsize[q]] = dist;
              sbi[q * kBallBuf + bsize[q]] = cid;
            }
            if (maxd[q] > dist) {
              maxd[q] = dist;
              maxi[q] = bsize[q];
            }
            bsize[q]++;
          } else if (dist < maxd[q]) {
            if (lane == 0) {
              sbd[q * kBallBuf + maxi[q]] = dist;
              sbi[q * kBallBuf + maxi[q]] = cid;
            }
            __syncwarp();
            // the new maximum; a scan from the replaced slot's value keeps the
            // replaced slot when it holds the maximum, else the first slot that does
            const float ve = lane < kBallBuf ? sbd[q * kBallBuf + lane] : -1.0f;
            float md = ve;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) md = fmaxf(md, __shfl_xor_sync(kAll, md, o));
            const unsigned at = __ballot_sync(kAll, lane < kBallBuf && ve == md);
            maxi[q] = md == dist ? maxi[q] : __ffs(at) - 1;
            maxd[q] = md;
            settled[q] = true;
          }
        }
      }
    });
#pragma unroll
    for (int q = 0; q < kBallPass; q++) {
      if (q >= ns) break;
      int* row = o_idx + (size_t)(s0 + q) * P;
      __syncwarp();
      const int val = lane < bsize[q] ? sbi[q * kBallBuf + lane] : -1;
      if (lane < min(P, kBallBuf)) row[lane] = val;
      if (P > kBallBuf)
        for (int e = kBallBuf + lane; e < P; e += 32) row[e] = -1;
    }
  }
  if (emitted < S) {
    const int n3 = (S - emitted) * 3, n1 = S - emitted, np = (S - emitted) * P;
    for (int e = lane; e < n3; e += 32) o_xyz[emitted * 3 + e] = 0.0f;
    for (int e = lane; e < n1; e += 32) o_t[emitted + e] = 0.0f, o_m[emitted + e] = 0;
    for (int e = lane; e < np; e += 32) o_idx[(size_t)emitted * P + e] = -1;
  }
  __syncwarp();
}

// Tile scheduling.  A tile's cost grows with the points in its window halo
// and is very uneven (dense objects vs background).  Work items are tiles of
// 8 rows x 32 pixels; a tile whose halo does not fit the stage is split into
// items of 4, 2 or 1 rows (each staged on its own, so they run concurrently
// on different SMs), and a single row whose halo still does not fit into
// column halves and then quarters, each staging its own, narrower halo; only
// what does not fit even then reads candidates from global memory.  Items are
// handed out heaviest first (a counting sort on
// log2 of the halo's point count; halos still too large to stage weighted up)
// to a persistent grid of SMs x resident blocks that takes the next item from
// an atomic counter, so heavy items start first and light ones fill in
// around them.
struct Sched {
  int* work;    // [max items] estimated cost
  int* item;    // [max items] item_code(tile, first row, rows)
  int* cols;    // [max items] (first column << 8) | end column, within the tile
  int* view;    // [max items] view of the item (batched launches; else null)
  int* order;   // [max items] item indices, heaviest first
  int* counts;  // [32] items per cost class
  int* fill;    // [32] placement cursors
  int* next;    // [1] next position in `order` to hand out
  int* n_items; // [1]
};

__device__ __forceinline__ int cost_class(int w) { return 31 - __clz(w | 1); }

// A work item: tile t (< 2^21, local to its view), first row and row count
// (<= 16) within the tile.
__host__ __device__ constexpr int item_code(int t, int row, int rows) { return (t << 10) | (row << 5) | rows; }
__device__ __forceinline__ int item_tile(int it) { return it >> 10; }
__device__ __forceinline__ int item_row(int it) { return (it >> 5) & 31; }
__device__ __forceinline__ int item_rows(int it) { return it & 31; }
constexpr int64_t kMaxTilesPerView = 1 << 21;

// Items of tile t (local to its view) of an H x W image, appended to the queue.
// The clipped point counts of the tile's whole window halo (up to
// (kTileH + 4) rows x (kTileW + 4) columns) are loaded once, up to two columns
// per lane; the halo of any row band or column range of the tile is a
// sub-rectangle of it, summed from those registers with one warp reduction.
template <int kTileH, int kTileW>
__device__ __forceinline__ void tile_work(const int2* __restrict__ hash, int n_sorted, int H, int W, int k, int tiles_x,
                                          int t, int view, int cap, Sched& sc) {
  constexpr int kHaloRows = kTileH + kMaxKernel - 1;
  const int lane = threadIdx.x & 31;
  const int v0 = (t / tiles_x) * kTileH, u0 = (t % tiles_x) * kTileW;
  const int v_end = min(H, v0 + kTileH);
  const int koff = (k + 1) >> 1, lo = koff - 1, hi = k - koff;
  const int hv0 = max(0, v0 - lo), hv1 = min(H - 1, v_end - 1 + hi);
  const int hu0 = max(0, u0 - lo), hu1 = min(W - 1, u0 + kTileW - 1 + hi);
  // a second halo column per lane only where the halo is wider than a warp
  constexpr bool kTwoCols = kTileW + kMaxKernel - 1 > 32;
  const int ua = hu0 + lane, ub = hu0 + 32 + lane;  // this lane's halo columns
  int ca[kHaloRows], cb[kTwoCols ? kHaloRows : 1];
#pragma unroll
  for (int h = 0; h < kHaloRows; h++) {
    ca[h] = 0;
    if constexpr (kTwoCols) cb[h] = 0;
    const int vv = hv0 + h;
    if (vv <= hv1) {
      if (ua <= hu1) {
        const int2 rg = bucket_range(__ldg(hash + (size_t)vv * W + ua), n_sorted);
        ca[h] = min(rg.y - rg.x, cap + 1);
      }
      if constexpr (kTwoCols) {
        if (ub <= hu1) {
          const int2 rg = bucket_range(__ldg(hash + (size_t)vv * W + ub), n_sorted);
          cb[h] = min(rg.y - rg.x, cap + 1);
        }
      }
    }
  }
  // points in the halo of rows [vb, vb + rows) and tile columns [c0, c1)
  auto halo = [&](int vb, int rows, int c0, int c1) {
    const int r0 = max(0, vb - lo), r1 = min(H - 1, vb + rows - 1 + hi);
    const int x0 = max(0, u0 + c0 - lo), x1 = min(W - 1, u0 + c1 - 1 + hi);
    const bool ia = ua >= x0 && ua <= x1, ib = kTwoCols && ub >= x0 && ub <= x1;
    int sum = 0;
#pragma unroll
    for (int h = 0; h < kHaloRows; h++) {
      const int vv = hv0 + h;
      if (vv >= r0 && vv <= r1) {
        sum += ia ? ca[h] : 0;
        if constexpr (kTwoCols) sum += ib ? cb[h] : 0;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    return sum;
  };
  // The tile's items are collected in shared memory first and then given
  // queue positions with one atomic per tile: a chain of returning atomics on
  // the shared item counter, one per item, made tiles that split into many
  // items wait on it item by item.  One tile per warp, eight warps per block.
  __shared__ int3 s_item[8][kTileH * 4];  // (cost, item code, columns)
  const int wp = threadIdx.x >> 5;
  int n_it = 0;  // warp-uniform
  // split the tile's rows until each item's halo holds at most `cap` points
  // (the stage's capacity, so no item runs much longer than the average) or
  // is one row
  for (int vb = v0; vb < v_end;) {
    int rows = v_end - vb;
    int sum = halo(vb, rows, 0, kTileW);
    while (sum > cap && rows > 1) {
      rows = (rows + 1) >> 1;
      sum = halo(vb, rows, 0, kTileW);
    }
    // cost estimate: the halo's points scaled by the share of its rows (and
    // columns) that hold the item's rays; unstaged items count 4x
    auto emit = [&](int hs, int c0, int c1) {
      if (lane == 0) {
        const int c = (int)(((long long)min(hs, 1 << 24) * rows * kTileH * (c1 - c0)) /
                            ((long long)(rows + k - 1) * (c1 - c0 + k - 1)));
        const int w = hs > cap ? c * 4 : c;
        s_item[wp][n_it] = make_int3(w, item_code(t, vb - v0, rows), (c0 << 8) | c1);
      }
      n_it++;
    };
    if (sum <= cap) {
      emit(sum, 0, kTileW);
    } else {  // one row: halves, then quarters, until the halo fits
      for (int c0 = 0; c0 < kTileW && u0 + c0 < W; c0 += kTileW / 2) {
        const int hs = halo(vb, rows, c0, c0 + kTileW / 2);
        if (hs <= cap) {
          emit(hs, c0, c0 + kTileW / 2);
          continue;
        }
        for (int q0 = c0; q0 < c0 + kTileW / 2 && u0 + q0 < W; q0 += kTileW / 4)
          emit(halo(vb, rows, q0, q0 + kTileW / 4), q0, q0 + kTileW / 4);
      }
    }
    vb += rows;
  }
  __syncwarp();
  int first = 0;
  if (lane == 0) first = atomicAdd(sc.n_items, n_it);
  first = __shfl_sync(0xffffffffu, first, 0);
  for (int j = lane; j < n_it; j += 32) {
    const int3 e = s_item[wp][j];
    const int i = first + j;
    sc.work[i] = e.x;
    sc.item[i] = e.y;
    sc.cols[i] = e.z;
    if (sc.view) sc.view[i] = view;
    atomicAdd(sc.counts + (sc.view ? view * 32 : 0) + cost_class(e.x), 1);  // result unused: a reduction
  }
}

// One warp per tile: its work items, then its share of the candidate packing
// (packing needs no result of the tile pass, so its loads overlap the tile
// pass's latency instead of taking a launch of their own).  Three blocks per
// SM, so one view's tiles (2500 warps at 800 x 800) run in one wave.
template <int kTileH, int kTileW>
__global__ void __launch_bounds__(256, 3) k_tile_work(const int2* __restrict__ hash, int n_sorted, int H, int W, int k,
                                                   int tiles_x, int ntiles, int cap, Sched sc,
                                                   const int* __restrict__ sidx, const float* __restrict__ xyz,
                                                   int n_points, float4* __restrict__ pts) {
  const int t = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (t >= ntiles) return;
  tile_work<kTileH, kTileW>(hash, n_sorted, H, W, k, tiles_x, t, 0, cap, sc);
  const int per = (n_sorted + ntiles - 1) / ntiles;
  const int j0 = min(n_sorted, t * per);
  pack_range(sidx, j0, min(n_sorted, j0 + per), xyz, n_points, pts);
}

__global__ void __launch_bounds__(256) k_tile_order(Sched sc) {
  __shared__ int base[32];
  if (threadIdx.x < 32) {
    int b = 0;  // items in heavier classes
    for (int c = 31; c > (int)threadIdx.x; c--) b += sc.counts[c];
    base[threadIdx.x] = b;
  }
  __syncthreads();
  const int n = *sc.n_items;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = cost_class(sc.work[i]);
    sc.order[base[c] + atomicAdd(sc.fill + c, 1)] = i;
  }
}

// Batched queue order: view by view (in table order), heaviest class first
// within a view, so only a view or two are in flight at a time -- their
// points stay in L2 -- while one view's tail still overlaps the next view's
// head.  base[v * 32 + c] = first queue position of view v's class-c items
// (one block: exclusive scan over the n_views * 32 buckets).
__global__ void __launch_bounds__(1024) k_batch_order_scan(Sched sc, int n_views, int* __restrict__ base) {
  __shared__ int warp_sum[32];
  const int n = n_views * 32;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(n, b0 + per);
  // bucket order: view ascending, class descending
  auto at = [&](int r) { return (r / 32) * 32 + (31 - r % 32); };
  int local = 0;
  for (int r = b0; r < b1; r++) local += sc.counts[at(r)];
  int incl = local;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  int off = 0;
  for (int w = 0; w < warp; w++) off += warp_sum[w];
  int run = off + incl - local;
  for (int r = b0; r < b1; r++) {
    base[at(r)] = run;
    run += sc.counts[at(r)];
  }
}

__global__ void __launch_bounds__(256) k_batch_order_place(Sched sc, const int* __restrict__ base) {
  const int n = *sc.n_items;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int b = sc.view[i] * 32 + cost_class(sc.work[i]);
    sc.order[base[b] + atomicAdd(sc.fill + b, 1)] = i;
  }
}

// Rays of rows [v0, v0 + rows) and tile columns [c0, c1) of the tile at u0
// (u0 + c0 < width).  Thread tid is tile pixel (tid / kTileW, tid % kTileW);
// a ray is named by that pixel index in the rank order.
template <class Cfg>
__device__ __forceinline__ void process_tile(const SampleArgs& a, Stage<Cfg>& st, int v0, int rows, int u0, int c0,
                                             int c1) {
  constexpr int kTileW = Cfg::kTileW;
  constexpr int kCap = Cfg::kCap;
  const int W = a.cam.width, H = a.cam.height, k = a.opt.k;
  const int koff = (k + 1) >> 1, lo = koff - 1, hi = k - koff;
  const int rv0 = max(0, v0 - lo), rv1 = min(H - 1, v0 + rows - 1 + hi);
  const int ru0 = max(0, u0 + c0 - lo), ru1 = min(W - 1, u0 + c1 - 1 + hi);
  const int nu = ru1 - ru0 + 1, ncells = (rv1 - rv0 + 1) * nu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // halo cell table: global start, clipped count, block-wide exclusive prefix
  int cnt[kCellsPerThread];
  int local = 0;
#pragma unroll
  for (int q = 0; q < kCellsPerThread; q++) {
    const int c = tid * kCellsPerThread + q;
    cnt[q] = 0;
    if (c < ncells) {
      const int vv = rv0 + c / nu, uu = ru0 + c % nu;
      const int2 rg = bucket_range(__ldg(a.hash + (size_t)vv * W + uu), a.n_sorted);
      st.start[c] = rg.x;
      // capped so the prefix cannot overflow; a capped cell alone exceeds the stage
      cnt[q] = min(rg.y - rg.x, kCap + 1);
    }
    local += cnt[q];
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) st.warp_tot[warp] = incl;
  __syncthreads();
  int base = incl - local;
  for (int q = 0; q < warp; q++) base += st.warp_tot[q];
  int total = 0;
#pragma unroll
  for (int q = 0; q < Cfg::kThreads / 32; q++) total += st.warp_tot[q];
#pragma unroll
  for (int q = 0; q < kCellsPerThread; q++) {
    const int c = tid * kCellsPerThread + q;
    if (c < ncells) st.off[c] = base;
    base += cnt[q];
  }
  if (tid == 0) st.off[ncells] = total;
  __syncthreads();

  const bool staged = total <= kCap;
  if (staged) {
    for (int i = tid; i < total; i += Cfg::kThreads) {
      int lo_c = 0, hi_c = ncells;  // off[lo_c] <= i < off[hi_c]
      while (hi_c - lo_c > 1) {
        const int mid = (lo_c + hi_c) >> 1;
        if (st.off[mid] <= i)
          lo_c = mid;
        else
          hi_c = mid;
      }
      st.cand[i] = __ldg(a.pts + st.start[lo_c] + (i - st.off[lo_c]));
    }
    __syncthreads();
  }

  // Group the tile's rays by their window's candidate count (a counting sort
  // over size classes; the order within a class does not affect any output).
  // The warps then pull work units, longest first: groups of 32 consecutive ranks below
  // a.heavy candidates (one ray per thread, similar loop lengths; a group
  // runs as long as its heaviest ray), then one unit per heavier ray (served by
  // the whole warp, sample_ray_warp, in about a 32nd of that time).  Warps that
  // finish early take the next unit, so a tile ends within about one short
  // unit of its total work divided by its warps.
  int nheavy, nvalid;
  {
    const int col = tid % kTileW, row = tid / kTileW;
    const int pu = u0 + col, pv = v0 + row;
    int T = -1;  // window candidates; -1: no ray at this pixel
    if (pu < W && pv < H && row < rows && col >= c0 && col < c1) {
      T = 0;
      if (staged && pu - lo >= 0 && pu + hi <= W - 1) {
        // unclamped columns: each window row is a run of k consecutive halo cells
        for (int dv = -lo; dv <= hi; dv++) {
          const int c0 = (min(max(pv + dv, 0), H - 1) - rv0) * nu + (pu - lo - ru0);
          T += st.off[c0 + k] - st.off[c0];
        }
      } else {
        for (int l = 0; l < k * k; l++) {
          int vv, uu;
          window_cell(pv, pu, k, H, W, l, vv, uu);
          const int2 rg = staged ? SrcStaged<Cfg>{&st, rv0, ru0, nu}.range(a, vv, uu) : SrcGlobal{}.range(a, vv, uu);
          T += rg.y - rg.x;
        }
      }
    }
    if (tid < kClasses) st.cls[tid] = 0;
    if (tid == 0) st.next_unit = 0;
    __syncthreads();
    // class 0: warp-served rays; then light rays by descending window size; last: no ray
    const int cw = max(1, a.heavy / 40);  // candidates per class
    const int c = T < 0 ? kClasses - 1 : (T > a.heavy ? 0 : 1 + min(kClasses - 3, (a.heavy - T) / cw));
    const int local = atomicAdd(&st.cls[c], 1);
    __syncthreads();
    if (tid < 32) {
      const int n0 = st.cls[2 * tid], n1 = st.cls[2 * tid + 1];
      int incl = n0 + n1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (tid >= o) incl += t;
      }
      st.cls_base[2 * tid] = incl - n0 - n1;
      st.cls_base[2 * tid + 1] = incl - n1;
    }
    __syncthreads();
    st.order[st.cls_base[c] + local] = tid;
    nheavy = st.cls[0];
    nvalid = Cfg::kThreads - st.cls[kClasses - 1];
    __syncthreads();
  }
  const int ngroups = (nvalid - nheavy + 31) >> 5;
  for (;;) {
    int unit = 0;
    if (lane == 0) unit = atomicAdd(&st.next_unit, 1);
    unit = __shfl_sync(0xffffffffu, unit, 0);
    if (unit < ngroups) {
      const int rk = nheavy + unit * 32 + lane;
      if (rk < nvalid) {
        const int px = st.order[rk];
        if (staged)
          sample_ray(a, SrcStaged<Cfg>{&st, rv0, ru0, nu}, v0 + px / kTileW, u0 + px % kTileW, &st.kept[0][tid]);
        else
          sample_ray(a, SrcGlobal{}, v0 + px / kTileW, u0 + px % kTileW, nullptr);
      }
      continue;
    }
    const int h = unit - ngroups;
    if (h >= nheavy) break;
    const int px = st.order[h];
    if (staged)
      sample_ray_warp(a, SrcStaged<Cfg>{&st, rv0, ru0, nu}, v0 + px / kTileW, u0 + px % kTileW,
                      &st.kept[0][warp * 32]);
    else
      sample_ray_warp(a, SrcGlobal{}, v0 + px / kTileW, u0 + px % kTileW, &st.kept[0][warp * 32]);
  }
  __syncthreads();  // the stage is reused by the next tile
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::kThreads, Cfg::kBlocks) k_quick_sampling(SampleArgs a, Sched sc, int tiles_x) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Stage<Cfg>& st = *reinterpret_cast<Stage<Cfg>*>(smem_raw);
  __shared__ int s_next;
  const int n = *sc.n_items;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(sc.next, 1);
    __syncthreads();
    const int i = s_next;
    if (i >= n) break;
    const int j = sc.order[i];
    const int it = sc.item[j], cc = sc.cols[j];
    const int t = item_tile(it);
    process_tile(a, st, (t / tiles_x) * Cfg::kTileH + item_row(it), item_rows(it), (t % tiles_x) * Cfg::kTileW,
                 cc >> 8, cc & 255);
  }
}

// ---------------------------------------------------------------------------
// Batched launch: the tiles of many views (different clouds, cameras, image
// sizes and options) in one queue and one persistent sampling kernel, so a
// view's tail overlaps the other views' work.  Every ray runs the same code as
// in a per-view launch, so the outputs are identical.

// Device view table -> per-view kernel arguments and the first global tile of
// each view (exclusive scan; tile_base[n_views] = all tiles).  One warp.
// Also the first packed-point slot of each view (pack_base; regions padded to
// 16 slots) and the views' packed-point arrays inside `pts`.
__global__ void k_batch_setup(const hp_view* __restrict__ views, int n_views, int heavy, int tile_h, int tile_w,
                              SampleArgs* __restrict__ args, int* __restrict__ tile_base, int* __restrict__ pack_base,
                              float4* __restrict__ pts) {
  const int lane = threadIdx.x;
  int run = 0, prun = 0;
  for (int b = 0; b < n_views; b += 32) {
    const int v = b + lane;
    int tiles = 0, slots = 0;
    if (v < n_views) slots = ((int)views[v].n_sorted + 15) & ~15;
    int pincl = slots;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, pincl, o);
      if (lane >= o) pincl += t;
    }
    const int pfirst = prun + pincl - slots;
    if (v < n_views) pack_base[v] = pfirst;
    prun += __shfl_sync(0xffffffffu, pincl, 31);
    if (v < n_views) {
      const hp_view& hv = views[v];
      SampleArgs a;
      a.xyz = hv.xyz;
      a.sidx = hv.sorted_point_idx;
      a.pts = pts + pfirst;
      a.hash = (const int2*)hv.hash_table;
      a.n_points = (int)hv.n_points;
      a.n_sorted = (int)hv.n_sorted;
      a.cam.c2w = hv.cam.c2w;
      a.cam.fx = hv.cam.fx;
      a.cam.fy = hv.cam.fy;
      a.cam.cx = hv.cam.cx;
      a.cam.cy = hv.cam.cy;
      a.cam.width = hv.cam.width;
      a.cam.height = hv.cam.height;
      a.opt.k = hv.opt.kernel_size;
      a.opt.t_intvl = hv.opt.t_intvl;
      a.opt.radius = hv.opt.radius_threshold;
      a.opt.S = hv.opt.num_sample_points_per_ray;
      a.opt.P = hv.opt.num_point_cloud_per_sp;
      a.opt.num_point_per_ray = hv.opt.num_point_per_ray;
      a.opt.alpha_g = hv.opt.sdf2weight_gaussian_alpha;
      a.opt.gamma = hv.opt.sdf2weight_gaussian_gamma;
      a.sp_xyz = hv.sp_xyz;
      a.pc_idx = hv.pc_idx;
      a.sp_t = hv.sp_t;
      a.mask = hv.mask;
      a.heavy = heavy;
      args[v] = a;
      tiles = ((hv.cam.width + tile_w - 1) / tile_w) * ((hv.cam.height + tile_h - 1) / tile_h);
    }
    int incl = tiles;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (v < n_views) tile_base[v] = run + incl - tiles;
    run += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) {
    tile_base[n_views] = run;
    pack_base[n_views] = prun;
  }
}

// Pack every view's candidates (see packed_point); slot g of the batch.
__global__ void k_batch_pack(const SampleArgs* __restrict__ args, const int* __restrict__ pack_base, int n_views,
                             int total) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  int lo = 0, hi = n_views;  // pack_base[lo] <= g < pack_base[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pack_base[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  const SampleArgs& a = args[lo];
  const int j = g - pack_base[lo];
  if (j >= a.n_sorted) return;
  const_cast<float4*>(a.pts)[j] = packed_point(a.sidx, j, a.xyz, a.n_points);
}

// One warp per global tile: find its view, then queue the tile's items.
template <int kTileH, int kTileW>
__global__ void __launch_bounds__(256, 3) k_batch_tile_work(const SampleArgs* __restrict__ args,
                                                         const int* __restrict__ tile_base, int n_views,
                                                         int total_tiles, int cap, Sched sc) {
  const int g = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (g >= total_tiles) return;
  int lo = 0, hi = n_views;  // tile_base[lo] <= g < tile_base[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tile_base[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  const SampleArgs& a = args[lo];
  const int tiles_x = (a.cam.width + kTileW - 1) / kTileW;
  tile_work<kTileH, kTileW>(a.hash, a.n_sorted, a.cam.height, a.cam.width, a.opt.k, tiles_x, g - tile_base[lo], lo,
                            cap, sc);
}

// The persistent sampling kernel over the batch's queue; each item's view
// arguments are loaded into shared memory before the tile is processed.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::kThreads, Cfg::kBlocks)
    k_quick_sampling_batch(const SampleArgs* __restrict__ args, Sched sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Stage<Cfg>& st = *reinterpret_cast<Stage<Cfg>*>(smem_raw);
  __shared__ int s_next;
  __shared__ SampleArgs s_args;
  const int n = *sc.n_items;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(sc.next, 1);
    __syncthreads();
    const int i = s_next;
    if (i >= n) break;
    const int j = sc.order[i];
    if (threadIdx.x == 0) s_args = args[sc.view[j]];
    __syncthreads();
    const int it = sc.item[j], cc = sc.cols[j];
    const int t = item_tile(it);
    const int tiles_x = (s_args.cam.width + Cfg::kTileW - 1) / Cfg::kTileW;
    process_tile(s_args, st, (t / tiles_x) * Cfg::kTileH + item_row(it), item_rows(it), (t % tiles_x) * Cfg::kTileW,
                 cc >> 8, cc & 255);
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

// The kernels and shapes of each stage configuration.
struct SamplingKernels {
  void (*view)(SampleArgs, Sched, int);
  void (*batch)(const SampleArgs*, Sched);
  void (*tile_work)(const int2*, int, int, int, int, int, int, int, Sched, const int*, const float*, int, float4*);
  void (*batch_tile_work)(const SampleArgs*, const int*, int, int, int, Sched);
  size_t smem;
  int cap, blocks, threads, tile_h, tile_w, items_per_tile;
};
template <class Cfg>
static SamplingKernels sampling_kernels() {
  return {k_quick_sampling<Cfg>,
          k_quick_sampling_batch<Cfg>,
          k_tile_work<Cfg::kTileH, Cfg::kTileW>,
          k_batch_tile_work<Cfg::kTileH, Cfg::kTileW>,
          sizeof(Stage<Cfg>),
          Cfg::kCap,
          Cfg::kBlocks,
          Cfg::kThreads,
          Cfg::kTileH,
          Cfg::kTileW,
          Cfg::kItemsPerTile};
}
static const SamplingKernels& stage_kernels(int config) {  // config 1..kStageConfigs
  static const SamplingKernels table[kStageConfigs] = {
      sampling_kernels<Cfg2560x4>(),   sampling_kernels<Cfg3712x3>(), sampling_kernels<Cfg5888x2>(),
      sampling_kernels<Cfg2560x4Sq>(), sampling_kernels<Cfg3712x3Sq>()};
  return table[config - 1];
}

static int64_t tiles_of(int64_t H, int64_t W, int tile_h, int tile_w) {
  return ((W + tile_w - 1) / tile_w) * ((H + tile_h - 1) / tile_h);
}

// Schedule entries an H x W view can need under any configuration (workspaces
// are sized for the largest, so one workspace serves every tuning).
static int64_t max_view_items(int64_t H, int64_t W) {
  int64_t m = 0;
  for (int c = 1; c <= kStageConfigs; c++) {
    const SamplingKernels& K = stage_kernels(c);
    const int64_t items = tiles_of(H, W, K.tile_h, K.tile_w) * K.items_per_tile;
    if (items > m) m = items;
  }
  return m;
}

// The stage exceeds the 48 KB default of dynamic shared memory: opt the
// configuration's kernels in once per device and size the persistent grid
// from their occupancy.
int32_t sampling_grid(int config, int* blocks, int* sm_count = nullptr) {
  static std::mutex mu;
  static int grid[128][kStageConfigs] = {{0}}, sm_counts[128] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(HP_ERR_CUDA, "hp_quick_sampling: cudaGetDevice failed");
  if (dev < 0 || dev >= 128)
    return set_error(HP_ERR_UNSUPPORTED, "hp_quick_sampling: device ordinal %d is beyond the 128 devices it tracks",
                     dev);
  std::lock_guard<std::mutex> lock(mu);
  int& g = grid[dev][config - 1];
  if (!g) {
    const SamplingKernels& K = stage_kernels(config);
    cudaError_t e = cudaFuncSetAttribute(K.view, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(K.batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K.smem);
    int sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, K.view, K.threads, K.smem);
    if (e != cudaSuccess) return set_error(HP_ERR_CUDA, "hp_quick_sampling: kernel set-up: %s", cudaGetErrorString(e));
    g = sms * (per_sm > 0 ? per_sm : 1);
    sm_counts[dev] = sms;
  }
  *blocks = g;
  if (sm_count) *sm_count = sm_counts[dev];
  return HP_OK;
}

// Launch tuning shared by both entry points; outputs never depend on it.
struct Tune {
  int heavy = kHeavyWindow, per_sm = 0, config = kDefaultStageConfig;
};

static int32_t read_tuning(const char* who, const hp_tuning* tuning, Tune& t) {
  if (!tuning) return HP_OK;
  if (tuning->heavy_window < 0 || tuning->heavy_window > kMaxHeavyWindow || tuning->blocks_per_sm < 0 ||
      tuning->stage_config < 0 || tuning->stage_config > kStageConfigs)
    return set_error(HP_ERR_INVALID_ARGUMENT,
                     "%s: tuning out of range (heavy_window 0..%d, blocks_per_sm >= 0, stage_config 0..%d)", who,
                     kMaxHeavyWindow, kStageConfigs);
  if (tuning->heavy_window > 0) t.heavy = tuning->heavy_window;
  t.per_sm = tuning->blocks_per_sm;
  if (tuning->stage_config > 0) t.config = tuning->stage_config;
  return HP_OK;
}

static constexpr size_t align256s(size_t x) { return (x + 255) & ~(size_t)255; }

struct SchedLayout {
  size_t work, item, cols, order, view, small, pts, total;
};

// up to items_per_tile items per tile (every row its own item, in quarters)
static SchedLayout sched_layout(int64_t H, int64_t W, int64_t n_sorted) {
  const size_t per = align256s(sizeof(int) * (size_t)max_view_items(H, W));
  SchedLayout L;
  L.work = 0;
  L.item = per;
  L.cols = 2 * per;
  L.order = 3 * per;
  L.view = 0;  // single view: none
  L.small = 4 * per;
  L.pts = L.small + 512;  // counts[32], fill[32], next, n_items
  L.total = L.pts + align256s(sizeof(float4) * (size_t)n_sorted);
  return L;
}

// Batched launch: the queue over all views' tiles, then the per-view
// arguments, the views' first tiles and room for a copy of the view table.
struct BatchLayout {
  SchedLayout q;
  size_t args, tile_base, pack_base, views, buckets, pts, total;
};

static BatchLayout batch_layout(int64_t total_items, int n_views, int64_t total_slots) {
  BatchLayout B;
  const size_t per = align256s(sizeof(int) * (size_t)total_items);
  B.q.work = 0;
  B.q.item = per;
  B.q.cols = 2 * per;
  B.q.order = 3 * per;
  B.q.view = 4 * per;
  B.q.small = 5 * per;
  B.q.total = B.q.small + 512;  // next, n_items (counts and fill live in `buckets`)
  B.args = B.q.total;
  B.tile_base = B.args + align256s(sizeof(SampleArgs) * (size_t)n_views);
  B.pack_base = B.tile_base + align256s(sizeof(int) * (size_t)(n_views + 1));
  B.views = B.pack_base + align256s(sizeof(int) * (size_t)(n_views + 1));
  B.buckets = B.views + align256s(sizeof(hp_view) * (size_t)n_views);  // counts, fill, base: n_views * 32 each
  B.pts = B.buckets + 3 * align256s(sizeof(int) * 32 * (size_t)n_views);
  B.total = B.pts + sizeof(float4) * (size_t)total_slots;
  return B;
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

extern "C" size_t hp_quick_sampling_workspace_size(int64_t n_sorted, int32_t height, int32_t width) {
  if (height <= 0 || width <= 0 || n_sorted < 0) return 0;
  return sched_layout(height, width, n_sorted).total;
}

// Argument checks shared by the per-view and batched entry points.
static int32_t check_sampling(const char* who, const float* xyz, int64_t n_points, const hp_camera* cam,
                              const hp_options* opt, const int32_t* sorted_point_idx, int64_t n_sorted,
                              const int32_t* hash_table, const float* sp_xyz, const int32_t* pc_idx, const float* sp_t,
                              const uint8_t* mask) {
  if (int32_t rc = check_camera(cam, who)) return rc;
  if (!opt) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: opt is NULL", who);
  if (opt->kernel_size < 1 || opt->kernel_size > kMaxKernel)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: kernel_size %d outside 1..%d (the reference's windows hold 32 cells)",
                     who, opt->kernel_size, kMaxKernel);
  if (!(opt->t_intvl > 0.0f)) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: t_intvl must be > 0", who);
  if (opt->num_sample_points_per_ray < 1 || opt->num_point_cloud_per_sp < 1)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: num_sample_points_per_ray and num_point_cloud_per_sp must be >= 1",
                     who);
  const int64_t hw = (int64_t)cam->height * cam->width;
  if (tiles_of(cam->height, cam->width, 16, 16) >= kMaxTilesPerView ||
      tiles_of(cam->height, cam->width, 8, 32) >= kMaxTilesPerView)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: image too large (%lld pixels)", who, (long long)hw);
  if (hw * opt->num_sample_points_per_ray * (int64_t)(opt->num_point_cloud_per_sp > 3 ? opt->num_point_cloud_per_sp : 3) >=
      (1ll << 40))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: output too large", who);
  if (n_points < 0 || n_points >= (1ll << 31) || n_sorted < 0 || n_sorted >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: n_points / n_sorted out of range", who);
  if (!hash_table || !sp_xyz || !pc_idx || !sp_t || !mask || (n_points > 0 && !xyz) ||
      (n_sorted > 0 && !sorted_point_idx))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: null pointer", who);
  if (((uintptr_t)hash_table & 7) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: hash_table must be 8-byte aligned", who);
  return HP_OK;
}

extern "C" int32_t hp_stage_config_info(int32_t config, int32_t* tile_h, int32_t* tile_w, int32_t* stage_points,
                                        int32_t* blocks_per_sm) {
  if (config == 0) config = kDefaultStageConfig;
  if (config < 1 || config > kStageConfigs)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_stage_config_info: stage_config %d outside 0..%d", config,
                     kStageConfigs);
  const SamplingKernels& K = stage_kernels(config);
  if (tile_h) *tile_h = K.tile_h;
  if (tile_w) *tile_w = K.tile_w;
  if (stage_points) *stage_points = K.cap;
  if (blocks_per_sm) *blocks_per_sm = K.blocks;
  return HP_OK;
}

extern "C" int32_t hp_quick_sampling_tuned(const float* xyz, int64_t n_points, const hp_camera* cam,
                                           const hp_options* opt, const int32_t* sorted_point_idx, int64_t n_sorted,
                                           const int32_t* hash_table, float* sp_xyz, int32_t* pc_idx, float* sp_t,
                                           uint8_t* mask, const hp_tuning* tuning, void* workspace,
                                           size_t workspace_bytes, hp_stream_t stream) {
  if (int32_t rc = check_sampling("hp_quick_sampling", xyz, n_points, cam, opt, sorted_point_idx, n_sorted, hash_table,
                                  sp_xyz, pc_idx, sp_t, mask))
    return rc;
  Tune tn;
  if (int32_t rc = read_tuning("hp_quick_sampling", tuning, tn)) return rc;
  const SchedLayout L = sched_layout(cam->height, cam->width, n_sorted);
  if (!workspace || workspace_bytes < L.total || ((uintptr_t)workspace & 255) != 0)
    return set_error(HP_ERR_WORKSPACE, "hp_quick_sampling: workspace needs %zu bytes, 256-byte aligned (got %zu)",
                     L.total, workspace_bytes);
  SampleArgs a;
  a.xyz = xyz;
  a.sidx = sorted_point_idx;
  a.pts = (const float4*)((char*)workspace + L.pts);
  a.hash = (const int2*)hash_table;
  a.n_points = (int)n_points;
  a.n_sorted = (int)n_sorted;
  a.cam = dev_camera(cam);
  a.opt = dev_options(opt);
  a.sp_xyz = sp_xyz;
  a.pc_idx = pc_idx;
  a.sp_t = sp_t;
  a.mask = mask;
  a.heavy = tn.heavy;
  int blocks = 0, sms = 0;
  if (int32_t rc = sampling_grid(tn.config, &blocks, &sms)) return rc;
  if (tn.per_sm > 0 && tn.per_sm * sms < blocks) blocks = tn.per_sm * sms;
  const SamplingKernels& K = stage_kernels(tn.config);
  const int tiles_x = (cam->width + K.tile_w - 1) / K.tile_w;
  const int ntiles = (int)tiles_of(cam->height, cam->width, K.tile_h, K.tile_w);
  char* ws = (char*)workspace;
  Sched sc;
  sc.work = (int*)(ws + L.work);
  sc.item = (int*)(ws + L.item);
  sc.cols = (int*)(ws + L.cols);
  sc.order = (int*)(ws + L.order);
  sc.view = nullptr;
  sc.counts = (int*)(ws + L.small);
  sc.fill = sc.counts + 32;
  sc.next = sc.counts + 64;
  sc.n_items = sc.counts + 65;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(sc.counts, 0, 512, st) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "hp_quick_sampling: cudaMemsetAsync failed");
  K.tile_work<<<(ntiles + 7) / 8, 256, 0, st>>>(a.hash, a.n_sorted, cam->height, cam->width, opt->kernel_size, tiles_x,
                                                 ntiles, K.cap, sc, sorted_point_idx, xyz, (int)n_points,
                                                 (float4*)(ws + L.pts));
  if (int32_t rc = check_launch("k_tile_work")) return rc;
  k_tile_order<<<(ntiles + 255) / 256 < 148 ? (ntiles + 255) / 256 : 148, 256, 0, st>>>(sc);
  if (int32_t rc = check_launch("k_tile_order")) return rc;
  // a split tile yields up to items_per_tile items: size the persistent grid by those, not by tiles
  const int64_t max_items = (int64_t)ntiles * K.items_per_tile;
  K.view<<<blocks < max_items ? blocks : (int)max_items, K.threads, K.smem, st>>>(a, sc, tiles_x);
  return check_launch("k_quick_sampling");
}

extern "C" int32_t hp_quick_sampling(const float* xyz, int64_t n_points, const hp_camera* cam, const hp_options* opt,
                                     const int32_t* sorted_point_idx, int64_t n_sorted, const int32_t* hash_table,
                                     float* sp_xyz, int32_t* pc_idx, float* sp_t, uint8_t* mask, void* workspace,
                                     size_t workspace_bytes, hp_stream_t stream) {
  return hp_quick_sampling_tuned(xyz, n_points, cam, opt, sorted_point_idx, n_sorted, hash_table, sp_xyz, pc_idx, sp_t,
                                 mask, nullptr, workspace, workspace_bytes, stream);
}

// packed-point slots of a batch: each view's n_sorted rounded up to 16
static int64_t batch_slots(const hp_view* views, int32_t n_views) {
  int64_t total = 0;
  for (int32_t v = 0; v < n_views; v++) total += (views[v].n_sorted + 15) & ~(int64_t)15;
  return total;
}

static int64_t batch_tiles(const hp_view* views, int32_t n_views, int tile_h, int tile_w) {
  int64_t total = 0;
  for (int32_t v = 0; v < n_views; v++) total += tiles_of(views[v].cam.height, views[v].cam.width, tile_h, tile_w);
  return total;
}

// Schedule entries a batch can need under any configuration.
static int64_t batch_max_items(const hp_view* views, int32_t n_views) {
  int64_t m = 0;
  for (int c = 1; c <= kStageConfigs; c++) {
    const SamplingKernels& K = stage_kernels(c);
    const int64_t items = batch_tiles(views, n_views, K.tile_h, K.tile_w) * K.items_per_tile;
    if (items > m) m = items;
  }
  return m;
}

extern "C" size_t hp_quick_sampling_batch_workspace_size(const hp_view* views, int32_t n_views) {
  if (!views || n_views <= 0) return 0;
  for (int32_t v = 0; v < n_views; v++)
    if (views[v].cam.width <= 0 || views[v].cam.height <= 0 || views[v].n_sorted < 0) return 0;
  return batch_layout(batch_max_items(views, n_views), n_views, batch_slots(views, n_views)).total;
}

extern "C" int32_t hp_quick_sampling_batch(const hp_view* views, const hp_view* views_device, int32_t n_views,
                                           const hp_tuning* tuning, void* workspace, size_t workspace_bytes,
                                           hp_stream_t stream) {
  static const char* who = "hp_quick_sampling_batch";
  if (!views || n_views <= 0) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: no views", who);
  Tune tn;
  if (int32_t rc = read_tuning(who, tuning, tn)) return rc;
  for (int32_t v = 0; v < n_views; v++) {
    const hp_view& hv = views[v];
    if (int32_t rc = check_sampling(who, hv.xyz, hv.n_points, &hv.cam, &hv.opt, hv.sorted_point_idx, hv.n_sorted,
                                    hv.hash_table, hv.sp_xyz, hv.pc_idx, hv.sp_t, hv.mask)) {
      char msg[256];
      snprintf(msg, sizeof(msg), "%s", hp_last_error());
      return set_error(rc, "%s (view %d)", msg, v);
    }
  }
  const int64_t max_items = batch_max_items(views, n_views);
  const int64_t total_slots = batch_slots(views, n_views);
  if (max_items >= (1ll << 31) || total_slots >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: too many tiles or points in one batch", who);
  const BatchLayout B = batch_layout(max_items, n_views, total_slots);
  if (!workspace || workspace_bytes < B.total || ((uintptr_t)workspace & 255) != 0)
    return set_error(HP_ERR_WORKSPACE, "%s: workspace needs %zu bytes, 256-byte aligned (got %zu)", who, B.total,
                     workspace_bytes);
  int blocks = 0, sms = 0;
  if (int32_t rc = sampling_grid(tn.config, &blocks, &sms)) return rc;
  if (tn.per_sm > 0 && tn.per_sm * sms < blocks) blocks = tn.per_sm * sms;
  const SamplingKernels& K = stage_kernels(tn.config);
  const int64_t total_tiles = batch_tiles(views, n_views, K.tile_h, K.tile_w);
  char* ws = (char*)workspace;
  cudaStream_t st = (cudaStream_t)stream;
  if (!views_device) {  // copy the table into the workspace
    if (cudaMemcpyAsync(ws + B.views, views, sizeof(hp_view) * (size_t)n_views, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return set_error(HP_ERR_CUDA, "%s: copying the view table failed", who);
    views_device = (const hp_view*)(ws + B.views);
  }
  Sched sc;
  sc.work = (int*)(ws + B.q.work);
  sc.item = (int*)(ws + B.q.item);
  sc.cols = (int*)(ws + B.q.cols);
  sc.order = (int*)(ws + B.q.order);
  sc.view = (int*)(ws + B.q.view);
  const size_t bucket_bytes = align256s(sizeof(int) * 32 * (size_t)n_views);
  sc.counts = (int*)(ws + B.buckets);
  sc.fill = (int*)(ws + B.buckets + bucket_bytes);
  int* base = (int*)(ws + B.buckets + 2 * bucket_bytes);
  sc.next = (int*)(ws + B.q.small);
  sc.n_items = sc.next + 1;
  SampleArgs* args = (SampleArgs*)(ws + B.args);
  int* tile_base = (int*)(ws + B.tile_base);
  if (cudaMemsetAsync(ws + B.q.small, 0, 512, st) != cudaSuccess ||
      cudaMemsetAsync(ws + B.buckets, 0, 2 * bucket_bytes, st) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "%s: memset failed", who);
  int* pack_base = (int*)(ws + B.pack_base);
  k_batch_setup<<<1, 32, 0, st>>>(views_device, n_views, tn.heavy, K.tile_h, K.tile_w, args, tile_base, pack_base,
                                  (float4*)(ws + B.pts));
  if (int32_t rc = check_launch("k_batch_setup")) return rc;
  if (total_slots > 0) {
    k_batch_pack<<<(unsigned)((total_slots + 255) / 256), 256, 0, st>>>(args, pack_base, n_views, (int)total_slots);
    if (int32_t rc = check_launch("k_batch_pack")) return rc;
  }
  const int nt = (int)total_tiles;
  K.batch_tile_work<<<(nt + 7) / 8, 256, 0, st>>>(args, tile_base, n_views, nt, K.cap, sc);
  if (int32_t rc = check_launch("k_batch_tile_work")) return rc;
  k_batch_order_scan<<<1, 1024, 0, st>>>(sc, n_views, base);
  if (int32_t rc = check_launch("k_batch_order_scan")) return rc;
  k_batch_order_place<<<(nt + 255) / 256 < 148 ? (nt + 255) / 256 : 148, 256, 0, st>>>(sc, base);
  if (int32_t rc = check_launch("k_batch_order_place")) return rc;
  const int64_t grid_items = (int64_t)nt * K.items_per_tile;
  K.batch<<<blocks < grid_items ? blocks : (int)grid_items, K.threads, K.smem, st>>>(args, sc);
  return check_launch("k_quick_sampling_batch");
}

extern "C" int32_t hp_ray_directions(const hp_camera* cam, float* dirs, hp_stream_t stream) {
  if (int32_t rc = check_camera(cam, "hp_ray_directions")) return rc;
  if (!dirs) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_ray_directions: dirs is NULL");
  const int hw = cam->width * cam->height;
  k_ray_directions<<<(hw + 255) / 256, 256, 0, (cudaStream_t)stream>>>(dev_camera(cam), dirs);
  return check_launch("k_ray_directions");
}
