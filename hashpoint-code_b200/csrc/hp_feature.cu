// Downstream of sampling: the per-sample point-attribute gather and the
// volume-rendering composite.
//
// hp_feature_query replaces FeatureQuery.forward (epcq/epcq.py:345-387).  The
// reference selects the valid samples with boolean indexing, gathers xyz /
// rgb / dir / feat of every selected point id with four torch.gather calls,
// scatters them into zero-filled canvases, and builds the per-pixel ray
// directions (generate_rays, epcq.py:333-341) for the whole image before
// selecting them.  Here the valid samples are numbered by an exclusive scan of
// the mask (hp_mask_scan) and one kernel writes, for each valid sample, its
// sample point, its ray direction, its P validity flags and the P gathered
// attribute rows -- each output element once, point rows read with coalesced
// warp loads.
//
// hp_clamp_t and hp_render replace clamp_t and render (epcq.py:508-529): per
// ray, the sample spacing with out-of-range gaps replaced by vsize, opacity
// 1 - exp(-sigma * delta), transmittance as the running product of
// (1 - opacity + 1e-10), and the weighted colour sum plus the background
// times the transmittance in front of the last sample.  One thread walks one
// ray's samples in order; hp_render can take t values instead of spacings and
// apply clamp_t on the fly.
#include <cuda_fp16.h>

#include "hp_common.cuh"

namespace hp {

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;  // mask bytes per thread (one 16-byte load)
constexpr int kScanTile = kScanThreads * kScanPerThread;

__device__ __forceinline__ int count_bytes(uint4 w) {
  // mask bytes are 0 or 1 (bool); count the nonzero ones
  auto c = [](unsigned x) { return __popc(__vcmpne4(x, 0u) & 0x01010101u); };
  return c(w.x) + c(w.y) + c(w.z) + c(w.w);
}

// Per tile of kScanTile mask bytes: its count.
__global__ void __launch_bounds__(kScanThreads) k_mask_tile_counts(const uint8_t* __restrict__ mask, int64_t n,
                                                                   int* __restrict__ tile_counts) {
  __shared__ int warp_sum[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPerThread;
  int c = 0;
  if (base + kScanPerThread <= n && ((uintptr_t)(mask + base) & 15) == 0) {
    c = count_bytes(*reinterpret_cast<const uint4*>(mask + base));
  } else {
    for (int q = 0; q < kScanPerThread; q++)
      if (base + q < n) c += mask[base + q] != 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kScanThreads / 32; w++) t += warp_sum[w];
    tile_counts[blockIdx.x] = t;
  }
}

// Exclusive scan of the tile counts in place (one block), total to *count.
__global__ void __launch_bounds__(1024) k_mask_scan_tiles(int* __restrict__ tile_counts, int n_tiles,
                                                          int* __restrict__ count) {
  __shared__ int warp_sum[32];
  const int per = (n_tiles + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(n_tiles, b0 + per);
  int local = 0;
  for (int i = b0; i < b1; i++) local += tile_counts[i];
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
  for (int i = b0; i < b1; i++) {
    const int c = tile_counts[i];
    tile_counts[i] = run;
    run += c;
  }
  if (threadIdx.x == blockDim.x - 1) *count = run;
}

// offsets[i] = valid samples before i (tile base + block-local exclusive scan).
__global__ void __launch_bounds__(kScanThreads) k_mask_offsets(const uint8_t* __restrict__ mask, int64_t n,
                                                               const int* __restrict__ tile_base,
                                                               int* __restrict__ offsets) {
  __shared__ int warp_sum[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPerThread;
  uint8_t v[kScanPerThread];
  if (base + kScanPerThread <= n && ((uintptr_t)(mask + base) & 15) == 0) {
    const uint4 w = *reinterpret_cast<const uint4*>(mask + base);
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < kScanPerThread; q++) v[q] = ((ws[q >> 2] >> (8 * (q & 3))) & 0xffu) != 0;
  } else {
#pragma unroll
    for (int q = 0; q < kScanPerThread; q++) v[q] = base + q < n ? mask[base + q] != 0 : 0;
  }
  int local = 0;
#pragma unroll
  for (int q = 0; q < kScanPerThread; q++) local += v[q];
  int incl = local;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  int run = tile_base[blockIdx.x] + incl - local;
  for (int w = 0; w < warp; w++) run += warp_sum[w];
  int o[kScanPerThread];
#pragma unroll
  for (int q = 0; q < kScanPerThread; q++) {
    o[q] = run;
    run += v[q];
  }
  if (base + kScanPerThread <= n && ((uintptr_t)(offsets + base) & 15) == 0) {
    int4* dst = reinterpret_cast<int4*>(offsets + base);  // this thread's 64 contiguous bytes
#pragma unroll
    for (int q = 0; q < kScanPerThread / 4; q++) dst[q] = make_int4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
  } else {
#pragma unroll
    for (int q = 0; q < kScanPerThread; q++)
      if (base + q < n) offsets[base + q] = o[q];
  }
}

struct FeatArgs {
  const float* xyz;
  const float* rgb;
  const float* dir;
  const void* feat;
  int feat_dim, feat_half;
  int n_points;
  const float* sp_xyz;
  const int* pc_idx;
  const uint8_t* mask;
  const int* offsets;
  int64_t n_samples;  // rays * S
  int S, P;
  const float* c2w;
  float fx, fy, cx, cy;
  int width;
  const int* ray_uv;  // [rays, 2] (u, v) or null: ray r is pixel (r % width, r / width)
  float* o_xyz;
  float* o_rgb;
  float* o_dir;
  float* o_feat;
  float* o_sp;
  uint8_t* o_valid;
  float* o_rays;
};

// One warp per 32 consecutive samples; the warp serves their valid ones in
// turn, spreading each sample's outputs over its lanes.
__global__ void __launch_bounds__(256) k_feature_query(FeatArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t i0 = ((int64_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * 32;
  if (i0 >= a.n_samples) return;
  const int64_t my = i0 + lane;
  const bool valid = my < a.n_samples && a.mask[my] != 0;
  unsigned todo = __ballot_sync(0xffffffffu, valid);
  const int my_off = valid ? a.offsets[my] : 0;
  const int P = a.P, F = a.feat_dim;
  while (todo) {
    const int l = __ffs(todo) - 1;
    todo &= todo - 1;
    const int64_t i = i0 + l;
    const int64_t m = __shfl_sync(0xffffffffu, my_off, l);
    const unsigned ray = (unsigned)i / (unsigned)a.S;  // sample counts are below 2^31: 32-bit division
    // sample point and ray direction (generate_rays: ((u - cx) / fx, (v - cy) / fy, 1) rotated by c2w)
    if (lane < 3) a.o_sp[m * 3 + lane] = a.sp_xyz[i * 3 + lane];
    if (lane >= 3 && lane < 6) {
      const int c = lane - 3;
      int u, v;
      if (a.ray_uv) {
        u = a.ray_uv[2 * (int64_t)ray];
        v = a.ray_uv[2 * (int64_t)ray + 1];
      } else {
        v = (int)(ray / (unsigned)a.width);
        u = (int)(ray - (unsigned)v * (unsigned)a.width);
      }
      const float dx = __fdiv_rn(__fsub_rn((float)u, a.cx), a.fx);
      const float dy = __fdiv_rn(__fsub_rn((float)v, a.cy), a.fy);
      const float* R = a.c2w + 4 * c;
      a.o_rays[m * 3 + c] = __fadd_rn(__fadd_rn(__fmul_rn(dx, R[0]), __fmul_rn(dy, R[1])), R[2]);
    }
    // validity flags and xyz / rgb / dir rows: lane = (point, component) over 3 * P lanes per pass
    const int* ids = a.pc_idx + i * P;
    for (int e = lane; e < 3 * P; e += 32) {
      const int p = e / 3, c = e - 3 * p;
      const int id = ids[p];
      const bool ok = (unsigned)id < (unsigned)a.n_points;
      if (c == 0) a.o_valid[m * P + p] = ok;
      const int64_t o = (m * P + p) * 3 + c;
      a.o_xyz[o] = ok ? a.xyz[(int64_t)id * 3 + c] : 0.0f;
      a.o_rgb[o] = ok ? a.rgb[(int64_t)id * 3 + c] : 0.0f;
      a.o_dir[o] = ok ? a.dir[(int64_t)id * 3 + c] : 0.0f;
    }
    // feature rows: P * F consecutive floats
    float* of = a.o_feat + m * P * F;
    for (int e = lane; e < P * F; e += 32) {
      const int p = e / F, f = e - p * F;
      const int id = ids[p];
      float val = 0.0f;
      if ((unsigned)id < (unsigned)a.n_points) {
        if (a.feat_half)
          val = __half2float(reinterpret_cast<const __half*>(a.feat)[(int64_t)id * F + f]);
        else
          val = reinterpret_cast<const float*>(a.feat)[(int64_t)id * F + f];
      }
      of[e] = val;
    }
  }
}

// The same gather with 16-byte moves, for feature rows whose bytes are a
// multiple of 16 (F = 32 fp16 or fp32 features, the Aggregator's width): the
// two half-warps serve two valid samples at a time, each lane moving 16-byte
// chunks of the feature rows (fp16 chunks widened to two float4 stores) and
// loading its two chunks or elements before storing either, so a pair of
// samples waits on one round of gathers.
template <int kHalf>
__global__ void __launch_bounds__(256) k_feature_query_vec(FeatArgs a) {
  constexpr int kEsz = kHalf ? 2 : 4;
  const unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31, hl = lane & 15, half = lane >> 4;
  const int64_t i0 = ((int64_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * 32;
  if (i0 >= a.n_samples) return;
  const int64_t my = i0 + lane;
  const bool valid = my < a.n_samples && a.mask[my] != 0;
  unsigned todo = __ballot_sync(kAll, valid);
  const int my_off = valid ? a.offsets[my] : 0;
  const int P = a.P, F = a.feat_dim;
  const int cpp = F * kEsz / 16;  // 16-byte chunks per feature row
  const int cshift = (cpp & (cpp - 1)) == 0 ? __ffs(cpp) - 1 : -1;  // log2(cpp) when a power of two
  const int nch = P * cpp;
  const char* feat = reinterpret_cast<const char*>(a.feat);
  while (todo) {
    const int l0 = __ffs(todo) - 1;
    todo &= todo - 1;
    int l1 = -1;
    if (todo) {
      l1 = __ffs(todo) - 1;
      todo &= todo - 1;
    }
    const int l = half ? l1 : l0;
    const int64_t m = __shfl_sync(kAll, my_off, l < 0 ? 0 : l);
    if (l < 0) continue;
    const int64_t i = i0 + l;
    const int* ids = a.pc_idx + i * P;  // the same few words for the half-warp (L1)
    if (hl < 3) a.o_sp[m * 3 + hl] = a.sp_xyz[i * 3 + hl];
    if (hl >= 3 && hl < 6) {
      const int c = hl - 3;
      const unsigned ray = (unsigned)i / (unsigned)a.S;  // sample counts are below 2^31: 32-bit division
      int u, v;
      if (a.ray_uv) {
        u = a.ray_uv[2 * (int64_t)ray];
        v = a.ray_uv[2 * (int64_t)ray + 1];
      } else {
        v = (int)(ray / (unsigned)a.width);
        u = (int)(ray - (unsigned)v * (unsigned)a.width);
      }
      const float dx = __fdiv_rn(__fsub_rn((float)u, a.cx), a.fx);
      const float dy = __fdiv_rn(__fsub_rn((float)v, a.cy), a.fy);
      const float* R = a.c2w + 4 * c;
      a.o_rays[m * 3 + c] = __fadd_rn(__fadd_rn(__fmul_rn(dx, R[0]), __fmul_rn(dy, R[1])), R[2]);
    }
    // xyz / rgb / dir rows: element e = (point, component), two per lane per pass
    for (int e = hl; e < 3 * P; e += 32) {
      float x[2], g[2], d[2];
      bool ok[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ee = e + 16 * h;
        x[h] = g[h] = d[h] = 0.0f;
        ok[h] = false;
        if (ee < 3 * P) {
          const int p = ee / 3, c = ee - 3 * p;
          const int id = ids[p];
          ok[h] = (unsigned)id < (unsigned)a.n_points;
          if (ok[h]) {
            x[h] = a.xyz[(int64_t)id * 3 + c];
            g[h] = a.rgb[(int64_t)id * 3 + c];
            d[h] = a.dir[(int64_t)id * 3 + c];
          }
        }
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ee = e + 16 * h;
        if (ee < 3 * P) {
          const int p = ee / 3, c = ee - 3 * p;
          if (c == 0) a.o_valid[m * P + p] = ok[h];
          const int64_t o = (m * P + p) * 3 + c;
          a.o_xyz[o] = x[h];
          a.o_rgb[o] = g[h];
          a.o_dir[o] = d[h];
        }
      }
    }
    // feature rows: chunk q of point p, two per lane per pass
    float* of = a.o_feat + m * P * F;
    for (int c = hl; c < nch; c += 32) {
      uint4 v[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int cc = c + 16 * h;
        v[h] = make_uint4(0u, 0u, 0u, 0u);
        if (cc < nch) {
          const int p = cshift >= 0 ? cc >> cshift : cc / cpp, q = cc - p * cpp;
          const int id = ids[p];
          if ((unsigned)id < (unsigned)a.n_points)
            v[h] = __ldg(reinterpret_cast<const uint4*>(feat + ((int64_t)id * cpp + q) * 16));
        }
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int cc = c + 16 * h;
        if (cc < nch) {
          const int p = cshift >= 0 ? cc >> cshift : cc / cpp, q = cc - p * cpp;
          if constexpr (kHalf) {
            const __half2* hh = reinterpret_cast<const __half2*>(&v[h]);
            const float2 f0 = __half22float2(hh[0]), f1 = __half22float2(hh[1]), f2 = __half22float2(hh[2]),
                         f3 = __half22float2(hh[3]);
            float4* dst = reinterpret_cast<float4*>(of + p * F + q * 8);
            dst[0] = make_float4(f0.x, f0.y, f1.x, f1.y);
            dst[1] = make_float4(f2.x, f2.y, f3.x, f3.y);
          } else {
            *reinterpret_cast<uint4*>(of + p * F + q * 4) = v[h];
          }
        }
      }
    }
  }
}

// clamp_t: gaps outside (1e-8, 2 vsize], and the last sample's, become vsize.
__device__ __forceinline__ float clamped_gap(const float* t, int s, int S, float vsize) {
  const float d = s + 1 < S ? __fsub_rn(t[s + 1], t[s]) : vsize;
  const float m = (d < 1e-8f || d > __fmul_rn(2.0f, vsize)) ? 1.0f : 0.0f;
  return __fadd_rn(__fmul_rn(d, __fsub_rn(1.0f, m)), __fmul_rn(m, vsize));
}

// one thread per (ray, sample): consecutive threads read and write consecutive elements
__global__ void k_clamp_t(const float* __restrict__ t_val, int64_t rays, int S, float vsize, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rays * S) return;
  const int s = i < 0x7fffffff ? (int)((unsigned)i % (unsigned)S) : (int)(i % S);
  out[i] = clamped_gap(t_val + (i - s), s, S, vsize);
}

// render (with the deltas given, or derived from t_val by clamp_t when deltas is null)
__global__ void k_render(const float* __restrict__ deltas, const float* __restrict__ t_val, float vsize,
                         const float* __restrict__ sigmas, const float* __restrict__ rgbs, int64_t rays, int S,
                         int white_bg, float* __restrict__ color) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rays) return;
  float trans = 1.0f;  // transmittance before this sample
  float bg_trans = 1.0f;  // the background sees the transmittance before the last sample
  float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  for (int s = 0; s < S; s++) {
    bg_trans = trans;
    const float d = deltas ? deltas[r * S + s] : clamped_gap(t_val + r * S, s, S, vsize);
    const float opacity = __fsub_rn(1.0f, expf(__fmul_rn(-sigmas[r * S + s], d)));
    const float w = __fmul_rn(opacity, trans);
    const float* c = rgbs + (r * S + s) * 3;
    c0 = __fadd_rn(c0, __fmul_rn(w, c[0]));
    c1 = __fadd_rn(c1, __fmul_rn(w, c[1]));
    c2 = __fadd_rn(c2, __fmul_rn(w, c[2]));
    trans = __fmul_rn(trans, __fadd_rn(__fsub_rn(1.0f, opacity), 1e-10f));
  }
  const float bg = white_bg ? 1.0f : 0.0f;
  color[r * 3 + 0] = __fadd_rn(c0, __fmul_rn(bg_trans, bg));
  color[r * 3 + 1] = __fadd_rn(c1, __fmul_rn(bg_trans, bg));
  color[r * 3 + 2] = __fadd_rn(c2, __fmul_rn(bg_trans, bg));
}

// The same for S = kS (a multiple of 4) with 16-byte aligned bases: a ray's
// sigma, t (or delta) and rgb rows are loaded as 16-byte vectors before any
// arithmetic, so a thread waits on one round of loads instead of one per
// sample; the arithmetic and its order are k_render's.
template <int kS>
__global__ void __launch_bounds__(256) k_render_vec(const float* __restrict__ deltas, const float* __restrict__ t_val,
                                                    float vsize, const float* __restrict__ sigmas,
                                                    const float* __restrict__ rgbs, int64_t rays, int white_bg,
                                                    float* __restrict__ color) {
  static_assert(kS % 4 == 0, "kS must be a multiple of 4");
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rays) return;
  float sg[kS], tv[kS], cl[3 * kS];
  const float4* s4 = reinterpret_cast<const float4*>(sigmas + r * kS);
  const float4* t4 = reinterpret_cast<const float4*>((deltas ? deltas : t_val) + r * kS);
  const float4* c4 = reinterpret_cast<const float4*>(rgbs + r * kS * 3);
#pragma unroll
  for (int q = 0; q < kS / 4; q++) {
    const float4 x = __ldg(s4 + q), y = __ldg(t4 + q);
    sg[4 * q] = x.x, sg[4 * q + 1] = x.y, sg[4 * q + 2] = x.z, sg[4 * q + 3] = x.w;
    tv[4 * q] = y.x, tv[4 * q + 1] = y.y, tv[4 * q + 2] = y.z, tv[4 * q + 3] = y.w;
  }
#pragma unroll
  for (int q = 0; q < 3 * kS / 4; q++) {
    const float4 x = __ldg(c4 + q);
    cl[4 * q] = x.x, cl[4 * q + 1] = x.y, cl[4 * q + 2] = x.z, cl[4 * q + 3] = x.w;
  }
  float trans = 1.0f, bg_trans = 1.0f;
  float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
#pragma unroll
  for (int s = 0; s < kS; s++) {
    bg_trans = trans;
    const float d = deltas ? tv[s] : clamped_gap(tv, s, kS, vsize);
    const float opacity = __fsub_rn(1.0f, expf(__fmul_rn(-sg[s], d)));
    const float w = __fmul_rn(opacity, trans);
    c0 = __fadd_rn(c0, __fmul_rn(w, cl[3 * s]));
    c1 = __fadd_rn(c1, __fmul_rn(w, cl[3 * s + 1]));
    c2 = __fadd_rn(c2, __fmul_rn(w, cl[3 * s + 2]));
    trans = __fmul_rn(trans, __fadd_rn(__fsub_rn(1.0f, opacity), 1e-10f));
  }
  const float bg = white_bg ? 1.0f : 0.0f;
  color[r * 3 + 0] = __fadd_rn(c0, __fmul_rn(bg_trans, bg));
  color[r * 3 + 1] = __fadd_rn(c1, __fmul_rn(bg_trans, bg));
  color[r * 3 + 2] = __fadd_rn(c2, __fmul_rn(bg_trans, bg));
}

}  // namespace hp

using namespace hp;

static size_t mask_tiles(int64_t n) { return (size_t)((n + kScanTile - 1) / kScanTile); }

extern "C" size_t hp_mask_scan_workspace_size(int64_t n) {
  if (n < 0) return 0;
  return ((mask_tiles(n) + 1) * sizeof(int) + 255) & ~(size_t)255;
}

extern "C" int32_t hp_mask_scan(const uint8_t* mask, int64_t n, int32_t* offsets, int32_t* count, void* workspace,
                                size_t workspace_bytes, hp_stream_t stream) {
  if (n < 0 || n >= (1ll << 31)) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_mask_scan: n out of range");
  if ((n > 0 && (!mask || !offsets)) || !count)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_mask_scan: null pointer");
  if (!workspace || workspace_bytes < hp_mask_scan_workspace_size(n))
    return set_error(HP_ERR_WORKSPACE, "hp_mask_scan: workspace needs %zu bytes", hp_mask_scan_workspace_size(n));
  cudaStream_t st = (cudaStream_t)stream;
  const int tiles = (int)mask_tiles(n);
  int* tile = (int*)workspace;
  if (tiles == 0) {
    if (cudaMemsetAsync(count, 0, sizeof(int32_t), st) != cudaSuccess)
      return set_error(HP_ERR_CUDA, "hp_mask_scan: memset failed");
    return HP_OK;
  }
  k_mask_tile_counts<<<tiles, kScanThreads, 0, st>>>(mask, n, tile);
  if (int32_t rc = check_launch("k_mask_tile_counts")) return rc;
  k_mask_scan_tiles<<<1, 1024, 0, st>>>(tile, tiles, count);
  if (int32_t rc = check_launch("k_mask_scan_tiles")) return rc;
  k_mask_offsets<<<tiles, kScanThreads, 0, st>>>(mask, n, tile, offsets);
  return check_launch("k_mask_offsets");
}

extern "C" int32_t hp_feature_query(const hp_point_attrs* pts, const float* sp_xyz, const int32_t* pc_idx,
                                    const uint8_t* mask, int64_t n_rays, int32_t S, int32_t P,
                                    const int32_t* offsets, const hp_camera* cam, const int32_t* ray_uv,
                                    float* pc_xyz, float* pc_rgb, float* pc_dir, float* pc_feat, float* out_sp_xyz,
                                    uint8_t* valid, float* rays_d, hp_stream_t stream) {
  static const char* who = "hp_feature_query";
  if (!pts || !cam) return set_error(HP_ERR_INVALID_ARGUMENT, "%s: null pointer", who);
  if (n_rays < 0 || S < 1 || P < 1 || n_rays * S >= (1ll << 31) || pts->n_points < 0 || pts->n_points >= (1ll << 31) ||
      pts->feat_dim < 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: sizes out of range", who);
  if (!cam->c2w || (!ray_uv && cam->width <= 0) || !(cam->fx != 0.0f) || !(cam->fy != 0.0f))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: bad camera", who);
  if (n_rays == 0) return HP_OK;
  if (!sp_xyz || !pc_idx || !mask || !offsets || !pc_xyz || !pc_rgb || !pc_dir || !out_sp_xyz || !valid || !rays_d ||
      (pts->feat_dim > 0 && (!pc_feat || !pts->feat)) || (pts->n_points > 0 && (!pts->xyz || !pts->rgb || !pts->dir)))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: null pointer", who);
  FeatArgs a;
  a.xyz = pts->xyz;
  a.rgb = pts->rgb;
  a.dir = pts->dir;
  a.feat = pts->feat;
  a.feat_dim = pts->feat_dim;
  a.feat_half = pts->feat_half;
  a.n_points = (int)pts->n_points;
  a.sp_xyz = sp_xyz;
  a.pc_idx = pc_idx;
  a.mask = mask;
  a.offsets = offsets;
  a.n_samples = n_rays * S;
  a.S = S;
  a.P = P;
  a.c2w = cam->c2w;
  a.fx = cam->fx;
  a.fy = cam->fy;
  a.cx = cam->cx;
  a.cy = cam->cy;
  a.width = cam->width;
  a.ray_uv = ray_uv;
  a.o_xyz = pc_xyz;
  a.o_rgb = pc_rgb;
  a.o_dir = pc_dir;
  a.o_feat = pc_feat;
  a.o_sp = out_sp_xyz;
  a.o_valid = valid;
  a.o_rays = rays_d;
  const int64_t warps = (a.n_samples + 31) / 32;
  const int esz = a.feat_half ? 2 : 4;
  // 16-byte moves when the rows and both base addresses allow them
  const bool vec = a.feat_dim > 0 && (a.feat_dim * esz) % 16 == 0 && ((uintptr_t)a.feat & 15) == 0 &&
                   ((uintptr_t)a.o_feat & 15) == 0;
  if (vec && a.feat_half)
    k_feature_query_vec<1><<<(unsigned)((warps + 7) / 8), 256, 0, (cudaStream_t)stream>>>(a);
  else if (vec)
    k_feature_query_vec<0><<<(unsigned)((warps + 7) / 8), 256, 0, (cudaStream_t)stream>>>(a);
  else
    k_feature_query<<<(unsigned)((warps + 7) / 8), 256, 0, (cudaStream_t)stream>>>(a);
  return check_launch("k_feature_query");
}

extern "C" int32_t hp_clamp_t(const float* t_val, int64_t n_rays, int32_t S, float vsize, float* t_dist,
                              hp_stream_t stream) {
  if (n_rays < 0 || S < 1 || n_rays * S >= (1ll << 39))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_clamp_t: sizes out of range");
  if (n_rays == 0) return HP_OK;
  if (!t_val || !t_dist) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_clamp_t: null pointer");
  k_clamp_t<<<(unsigned)((n_rays * S + 255) / 256), 256, 0, (cudaStream_t)stream>>>(t_val, n_rays, S, vsize, t_dist);
  return check_launch("k_clamp_t");
}

extern "C" int32_t hp_render(const float* deltas, const float* t_val, float vsize, const float* sigmas,
                             const float* rgbs, int64_t n_rays, int32_t S, int32_t white_bg, float* color,
                             hp_stream_t stream) {
  if (n_rays < 0 || S < 1) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_render: sizes out of range");
  if (n_rays == 0) return HP_OK;
  if ((!deltas && !t_val) || !sigmas || !rgbs || !color)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_render: null pointer");
  const unsigned blocks = (unsigned)((n_rays + 255) / 256);
  cudaStream_t st = (cudaStream_t)stream;
  const bool aligned = (((uintptr_t)(deltas ? deltas : t_val) | (uintptr_t)sigmas | (uintptr_t)rgbs) & 15) == 0;
  if (aligned && S == 8)
    k_render_vec<8><<<blocks, 256, 0, st>>>(deltas, t_val, vsize, sigmas, rgbs, n_rays, white_bg, color);
  else if (aligned && S == 16)
    k_render_vec<16><<<blocks, 256, 0, st>>>(deltas, t_val, vsize, sigmas, rgbs, n_rays, white_bg, color);
  else if (aligned && S == 4)
    k_render_vec<4><<<blocks, 256, 0, st>>>(deltas, t_val, vsize, sigmas, rgbs, n_rays, white_bg, color);
  else
    k_render<<<blocks, 256, 0, st>>>(deltas, t_val, vsize, sigmas, rgbs, n_rays, S, white_bg, color);
  return check_launch("k_render");
}
