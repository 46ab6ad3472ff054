// Per-pixel hash-table build: projection, counting sort by pixel, bucket order.
//
// Replaces NeuralPoints.pts2plane (epcq/epcq.py:279-295) + _C.scatter_hashtable
// (epcq/csrc/rasterization.cu:130-171).  The reference projects with two cuBLAS
// GEMMs, radix-sorts all N pixel ids with torch.sort, and then has one thread
// per pixel binary-search the sorted array and copy its run.  Here the pixel
// ids are a small dense key range, so the sort is a counting sort:
//
//   k_project_count   one pass over xyz, four points per thread: pixel id +
//                     depth with the reference's exact rounding, atomic slot
//                     within the pixel's bucket (four atomics in flight)
//   k_scan_hash       single-pass exclusive scan of the H*W counts (tiles
//                     add up the totals of the tiles before them) ->
//                     hash_table (start, count) / (-1, -1)
//   k_scatter         every point to start + slot of a scratch copy, one
//                     16-byte (id, depth, bucket start, bucket count) record
//                     per entry; -1 into the off-image tail of the outputs
//   k_order           one thread per bucket entry: its rank among its bucket's
//                     entries gives its final position (buckets <= 2048)
//   k_sort_huge_list  buckets above 2048 entries, which k_scan_hash lists as
//                     it writes the table: one CTA each, bitonic sort in place
//                     in global memory (k_sort_huge_scan finds them by
//                     scanning the table where there is no workspace)
//
// The atomic slots make the order inside a bucket arbitrary; ranking restores
// the reference's order: ascending point id (the stable sort's order) when
// sort == 0, (depth, id) when sort != 0 (its stable bubble sort).  Rank
// sorting costs sum(c^2) comparisons over buckets of c entries, which for
// point clouds (a few to a few hundred points per pixel) is far cheaper than
// a serial sort per bucket, and every thread does useful work.
#include <cstdio>
#include <mutex>

#include "hp_common.cuh"
#ifdef HP_TESTING
#include "../../include/hashpoint_b200_testing.h"
#endif

namespace hp {

constexpr int kRankMax = 2048;                   // largest bucket ordered by ranking
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;                    // counts per thread in the scan
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kHugeThreads = 512;
// Look-back words of the scan: a status bit above the tile's total in the
// low 32 bits (0 = not yet published).
constexpr unsigned long long kAggregate = 1ull << 62;
constexpr int kLookBackSpins = 1 << 16;  // polls of one predecessor (about 64 ns apart) before giving up
constexpr int kScanMaxTiles = 256;       // blocks of the scan (each a run of chunks of kScanTile pixels)

// Bucket sort key: the point id (sort == 0) or (depth, id) with depth mapped to
// an order-preserving integer (-0.0 folded onto +0.0 as float comparison does).
__device__ __forceinline__ unsigned long long sort_key(int id, float depth, int by_depth) {
  if (!by_depth) return (unsigned long long)(unsigned)id;
  unsigned b = __float_as_uint(depth == 0.0f ? 0.0f : depth);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  return ((unsigned long long)b << 32) | (unsigned)id;
}

// ---------------------------------------------------------------------------
// projection + count (epcq.py:251-274 restated with the GEMMs' rounding)
// ---------------------------------------------------------------------------
// One point: (pixel id, slot in its bucket, depth bits), pixel id H*W when off
// the image.
__device__ __forceinline__ int3 project_point(const float* w, const float* k, float x, float y, float z, int H, int W,
                                              int fused_world, int fused_image, int* __restrict__ counts) {
  float pc[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float* a = w + 4 * r;
    const float g = fused_world ? __fmaf_rn(a[2], z, __fmaf_rn(a[1], y, __fmul_rn(a[0], x)))
                                : __fadd_rn(__fadd_rn(__fmul_rn(a[0], x), __fmul_rn(a[1], y)), __fmul_rn(a[2], z));
    pc[r] = __fadd_rn(g, a[3]);
  }
  float s[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float* a = k + 3 * r;
    s[r] = fused_image ? __fmaf_rn(a[2], pc[2], __fmaf_rn(a[1], pc[1], __fmul_rn(a[0], pc[0])))
                       : __fadd_rn(__fadd_rn(__fmul_rn(a[0], pc[0]), __fmul_rn(a[1], pc[1])), __fmul_rn(a[2], pc[2]));
  }
  const int ix = __float2int_rz(__fdiv_rn(s[0], s[2]));
  const int iy = __float2int_rz(__fdiv_rn(s[1], s[2]));
  const bool inb = 0 <= ix && ix < W && 0 <= iy && iy < H;
  const int p = inb ? ix + iy * W : H * W;
  const int slot = inb ? atomicAdd(counts + p, 1) : 0;
  return make_int3(p, slot, __float_as_int(pc[2]));
}

// Four consecutive points per thread: xyz as three 16-byte loads when it is
// 16-byte aligned (the last partial group, and unaligned inputs, point by
// point), the (pixel, slot) pairs as two 16-byte stores and the depths as one.
__global__ void __launch_bounds__(256) k_project_count(const float* __restrict__ xyz, int n,
                                                       const float* __restrict__ w2c, const float* __restrict__ K,
                                                       int H, int W, int fused_world, int fused_image,
                                                       int* __restrict__ counts, int2* __restrict__ pid_slot,
                                                       float* __restrict__ depth) {
  float w[12], k[9];
#pragma unroll
  for (int i = 0; i < 12; i++) w[i] = __ldg(w2c + i);
#pragma unroll
  for (int i = 0; i < 9; i++) k[i] = __ldg(K + i);
  const bool vec = ((uintptr_t)xyz & 15) == 0;
  const int groups = (n + 3) >> 2;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x) {
    const int i0 = g << 2;
    if (vec && i0 + 3 < n) {
      const float4* x4 = reinterpret_cast<const float4*>(xyz) + 3 * (size_t)g;
      const float4 a = __ldg(x4), b = __ldg(x4 + 1), c = __ldg(x4 + 2);
      const int3 o0 = project_point(w, k, a.x, a.y, a.z, H, W, fused_world, fused_image, counts);
      const int3 o1 = project_point(w, k, a.w, b.x, b.y, H, W, fused_world, fused_image, counts);
      const int3 o2 = project_point(w, k, b.z, b.w, c.x, H, W, fused_world, fused_image, counts);
      const int3 o3 = project_point(w, k, c.y, c.z, c.w, H, W, fused_world, fused_image, counts);
      int4* ps = reinterpret_cast<int4*>(pid_slot + i0);
      ps[0] = make_int4(o0.x, o0.y, o1.x, o1.y);
      ps[1] = make_int4(o2.x, o2.y, o3.x, o3.y);
      *reinterpret_cast<int4*>(depth + i0) = make_int4(o0.z, o1.z, o2.z, o3.z);
    } else {
      for (int i = i0; i < n && i < i0 + 4; i++) {
        const int3 o = project_point(w, k, __ldg(xyz + 3 * (size_t)i), __ldg(xyz + 3 * (size_t)i + 1),
                                     __ldg(xyz + 3 * (size_t)i + 2), H, W, fused_world, fused_image, counts);
        pid_slot[i] = make_int2(o.x, o.y);
        depth[i] = __int_as_float(o.z);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// scan over the per-pixel counts
// ---------------------------------------------------------------------------
__device__ __forceinline__ int block_reduce_sum(int v, int* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = lane < nw ? sh[lane] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Single-pass exclusive scan of counts -> hash_table.  The image's pixels are
// cut into chunks of kScanTile; at most kScanMaxTiles blocks ("tiles") each
// take a contiguous run of chunks, in the order the tiles start (their index
// comes from a counter), so a tile only ever waits on tiles already running.
// A tile sums its run and publishes the total; its first warp then adds up
// the totals of all earlier tiles (a look-back over totals alone: no tile
// waits on another's running total, so there is no chain), and the tile scans
// its run chunk by chunk from that carry.  Every poll of an earlier tile is
// bounded (`spins` polls, kLookBackSpins in the product); a tile that gives up
// counts that tile as empty and sets scalars[3], which hp_pts2plane_status
// reports (the table is then wrong; this does not happen while the tiles it
// waits on are running).  `withhold` >= 0 names a tile that never publishes
// its total, so that a test can make the others give up.  Also lists the pixels whose
// buckets exceed kRankMax (count in scalars[1]), for k_sort_huge_list.
// scalars[2]: the tile counter; scalars[0]: the points inside the image.
__global__ void __launch_bounds__(kScanThreads) k_scan_hash(const int* __restrict__ counts, int hw, int chunks_per_tile,
                                                            unsigned long long* __restrict__ look,
                                                            int2* __restrict__ hash, int* __restrict__ scalars,
                                                            int* __restrict__ huge, int withhold, int spins) {
  __shared__ int sh[32];
  __shared__ int warp_tot[32];
  __shared__ int s_tile, s_carry;
  if (threadIdx.x == 0) s_tile = atomicAdd(scalars + 2, 1);
  __syncthreads();
  const int tile = s_tile;
  const int nchunks = (hw + kScanTile - 1) / kScanTile;
  const int ch0 = min(nchunks, tile * chunks_per_tile), ch1 = min(nchunks, ch0 + chunks_per_tile);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  static_assert(kScanItems == 4, "one int4 of counts per thread");
  // a thread's four counts (an int4: base is a multiple of 4 and counts is 256-byte aligned)
  auto load4 = [&](int base, int* c) {
    if (base + 3 < hw) {
      const int4 v = *reinterpret_cast<const int4*>(counts + base);
      c[0] = v.x, c[1] = v.y, c[2] = v.z, c[3] = v.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) c[j] = base + j < hw ? counts[base + j] : 0;
    }
  };
  // the run's total
  int part = 0;
  for (int ch = ch0; ch < ch1; ch++) {
    int c[4];
    load4(ch * kScanTile + threadIdx.x * kScanItems, c);
    part += c[0] + c[1] + c[2] + c[3];
  }
  const int total = block_reduce_sum(part, sh);
  if (warp == 0) {
    if (lane == 0 && tile != withhold) atomicExch(look + tile, kAggregate | (unsigned)total);
    int carry = 0;
    for (int q = lane; q < tile; q += 32) {
      unsigned long long f = *(volatile unsigned long long*)(look + q);
      for (int spin = 0; (f >> 62) == 0; spin++) {
        if (spin == spins) {
          atomicExch(scalars + 3, 1);
          f = kAggregate;  // counted as empty
          break;
        }
        __nanosleep(64);
        f = *(volatile unsigned long long*)(look + q);
      }
      carry += (int)(unsigned)(f & 0xffffffffu);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) carry += __shfl_xor_sync(0xffffffffu, carry, o);
    if (lane == 0) s_carry = carry;
  }
  __syncthreads();
  int run = s_carry;  // points before the current chunk

  for (int ch = ch0; ch < ch1; ch++) {
    const int base = ch * kScanTile + threadIdx.x * kScanItems;
    int c[kScanItems];
    load4(base, c);
    const int local = c[0] + c[1] + c[2] + c[3];
    // block exclusive scan of `local`
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int wt = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
      int wi = wt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      warp_tot[lane] = wi - wt;
      sh[lane] = wi;  // sh[31]: the chunk's total
    }
    __syncthreads();
    int off = run + warp_tot[warp] + incl - local;
    int o[kScanItems];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
      o[j] = off;
      if (c[j] > kRankMax && base + j < hw) huge[atomicAdd(scalars + 1, 1)] = base + j;
      off += c[j];
    }
    auto entry = [&](int j) { return c[j] > 0 ? make_int2(o[j], c[j]) : make_int2(-1, -1); };
    if (base + 3 < hw) {  // 16-byte stores (hash_table is 8-byte aligned: two int4 need 16)
      const int2 e0 = entry(0), e1 = entry(1), e2 = entry(2), e3 = entry(3);
      if (((uintptr_t)(hash + base) & 15) == 0) {
        reinterpret_cast<int4*>(hash + base)[0] = make_int4(e0.x, e0.y, e1.x, e1.y);
        reinterpret_cast<int4*>(hash + base)[1] = make_int4(e2.x, e2.y, e3.x, e3.y);
      } else {
        hash[base] = e0, hash[base + 1] = e1, hash[base + 2] = e2, hash[base + 3] = e3;
      }
    } else {
#pragma unroll
      for (int j = 0; j < kScanItems; j++)
        if (base + j < hw) hash[base + j] = entry(j);
    }
    run += sh[31];
    __syncthreads();  // warp_tot and sh are rewritten by the next chunk
  }
  if (ch1 == nchunks && ch0 < ch1 && threadIdx.x == 0) scalars[0] = run;  // points inside the image
}

// ---------------------------------------------------------------------------
// scatter into buckets
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_scatter(int n, int hw, const int2* __restrict__ pid_slot,
                                                 const float* __restrict__ depth, const int2* __restrict__ hash,
                                                 const int* __restrict__ scalars, int4* __restrict__ tmp,
                                                 int* __restrict__ out_idx, float* __restrict__ out_depth) {
  const int n_in = scalars[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 ps = pid_slot[i];
    if (ps.x < hw) {
      const int2 h = hash[ps.x];
      tmp[h.x + ps.y] = make_int4(i, __float_as_int(depth[i]), h.x, h.y);
    }
    if (i >= n_in) {
      out_idx[i] = -1;
      out_depth[i] = -1.0f;
    }
  }
}

// ---------------------------------------------------------------------------
// per-bucket order
// ---------------------------------------------------------------------------
// Entry keys are (hi, lo): hi = order-preserving depth bits (0 when ordering by
// id alone), lo = the point id, or -- for hp_scatter_hashtable, whose input
// order inside a run must survive depth ties -- the entry's input position.
struct BucketOrder {
  int by_depth;
  int by_position;  // tie-break on the input position instead of the id
};

__device__ __forceinline__ unsigned long long entry_key(const BucketOrder& bo, int id, float depth, int pos) {
  return sort_key(bo.by_position ? pos : id, depth, bo.by_depth);
}

// Bucket entries in position order: hp_pts2plane's packed scratch records,
// which carry their bucket ...
struct PackedEntries {
  const int4* rec;  // (id, depth bits, bucket start, bucket count)
  // entry j: its bucket (start, count) and (id, depth bits); false if none
  __device__ __forceinline__ bool entry(int j, const int2*, int, int2& bucket, int2& e) const {
    const int4 r = __ldg(rec + j);
    bucket = make_int2(r.z, r.w);
    e = make_int2(r.x, r.y);
    return true;
  }
  __device__ __forceinline__ int2 id_depth(int j) const { return __ldg(reinterpret_cast<const int2*>(rec + j)); }
  __device__ __forceinline__ int id_at(int j) const { return __ldg(reinterpret_cast<const int*>(rec + j)); }
};

// ... or the caller's sorted arrays (hp_scatter_hashtable), whose buckets come
// from the hash table.
struct SplitEntries {
  const int* id;
  const float* depth;
  const int* pid;
  __device__ __forceinline__ bool entry(int j, const int2* hash, int hw, int2& bucket, int2& e) const {
    const int p = __ldg(pid + j);
    if (p < 0 || p >= hw) return false;
    bucket = __ldg(hash + p);
    e = id_depth(j);
    return true;
  }
  __device__ __forceinline__ int2 id_depth(int j) const {
    return make_int2(__ldg(id + j), __float_as_int(__ldg(depth + j)));
  }
  __device__ __forceinline__ int id_at(int j) const { return __ldg(id + j); }
};

// One thread per entry j < n_in of the scratch copy: rank among the entries of
// its bucket -> final position.  Buckets of one entry are copied; buckets above
// kRankMax are left to k_sort_huge_list / k_sort_huge_scan.  The order mode
// is a template argument so that the rank loop -- the kernel's instructions
// are mostly its iterations -- compares ids alone when ordering by id.
template <class Entries, int kByDepth, int kByPosition>
__global__ void __launch_bounds__(256) k_order(Entries in, const int2* __restrict__ hash, int hw,
                                               const int* __restrict__ scalars, int n_fixed,
                                               int* __restrict__ out_idx, float* __restrict__ out_depth) {
  const BucketOrder bo{kByDepth, kByPosition};
  const int n_in = n_fixed >= 0 ? n_fixed : scalars[0];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_in; j += gridDim.x * blockDim.x) {
    int2 h, e;
    if (!in.entry(j, hash, hw, h, e)) continue;
    // a bucket inside [0, n_in) -- always, unless the scan gave up waiting (hp_pts2plane_status),
    // when the scratch may hold records no point wrote: then outputs are wrong but stay in bounds
    if (h.x < 0 || h.y < 1 || h.y > n_in - h.x) continue;
    if (h.y > kRankMax) continue;
    const float d = __int_as_float(e.y);
    int pos = h.x;
    if (h.y > 1) {
      int rank = 0;
      if constexpr (!kByDepth && !kByPosition) {
        for (int q = h.x; q < h.x + h.y; q++) rank += in.id_at(q) < e.x;
      } else {
        const unsigned long long kj = entry_key(bo, e.x, d, j);
        for (int q = h.x; q < h.x + h.y; q++) {
          const int2 eq = in.id_depth(q);
          rank += entry_key(bo, eq.x, __int_as_float(eq.y), q) < kj;
        }
      }
      pos += rank;
    }
    out_idx[pos] = e.x;
    out_depth[pos] = d;
  }
}

// Compare-exchange of positions i < l (ascending) in a bucket of c entries;
// positions >= c act as +inf and are never touched (the "flip" bitonic
// variant compares only towards the larger index, ascending).  While sorting,
// idx holds input positions in the by_position mode.
__device__ __forceinline__ void cx_global(const BucketOrder& bo, int* idx, float* dep, int i, int l, int c) {
  if (l >= c) return;
  const unsigned long long ki = sort_key(idx[i], dep[i], bo.by_depth), kl = sort_key(idx[l], dep[l], bo.by_depth);
  if (ki > kl) {
    const int t = idx[i];
    idx[i] = idx[l];
    idx[l] = t;
    const float d = dep[i];
    dep[i] = dep[l];
    dep[l] = d;
  }
}

// One bucket above kRankMax entries (pathological inputs), sorted by one CTA in
// place in global memory after copying it from the scratch entries (indexed by
// position).
template <class Entries>
__device__ __forceinline__ void sort_bucket(int2 h, Entries in, int* __restrict__ out_idx, float* __restrict__ out_depth,
                                            const BucketOrder& bo) {
  const int c = h.y;
  int* idx = out_idx + h.x;
  float* dep = out_depth + h.x;
  for (int i = threadIdx.x; i < c; i += blockDim.x) {
    const int2 e = in.id_depth(h.x + i);
    idx[i] = bo.by_position ? h.x + i : e.x;
    dep[i] = __int_as_float(e.y);
  }
  __syncthreads();
  int npow = 1;
  while (npow < c) npow <<= 1;
  for (int k = 2; k <= npow; k <<= 1) {
    for (int i = threadIdx.x; i < npow / 2; i += blockDim.x) {
      const int blk = i / (k >> 1), off = i % (k >> 1);
      const int a = blk * k + off, b = blk * k + k - 1 - off;
      if (a < c) cx_global(bo, idx, dep, a, b, c);
    }
    __syncthreads();
    for (int j = k >> 2; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < npow / 2; i += blockDim.x) {
        const int blk = i / j, off = i % j;
        const int a = blk * 2 * j + off;
        if (a < c) cx_global(bo, idx, dep, a, a + j, c);
      }
      __syncthreads();
    }
  }
  if (bo.by_position)
    for (int i = threadIdx.x; i < c; i += blockDim.x) idx[i] = in.id_depth(idx[i]).x;
  __syncthreads();
}

// hp_pts2plane: the buckets k_scan_hash listed, one CTA each in turn.
template <class Entries>
__global__ void __launch_bounds__(kHugeThreads) k_sort_huge_list(const int* __restrict__ huge,
                                                                 const int* __restrict__ scalars, Entries in,
                                                                 const int2* __restrict__ hash,
                                                                 int* __restrict__ out_idx,
                                                                 float* __restrict__ out_depth, BucketOrder bo) {
  const int n = scalars[1];
  for (int q = blockIdx.x; q < n; q += gridDim.x) sort_bucket(hash[huge[q]], in, out_idx, out_depth, bo);
}

// hp_scatter_hashtable (no workspace for a list): each CTA scans a contiguous
// range of pixels blockDim at a time and queues the huge ones in shared memory.
template <class Entries>
__global__ void __launch_bounds__(kHugeThreads) k_sort_huge_scan(int hw, Entries in, const int2* __restrict__ hash,
                                                                 int* __restrict__ out_idx,
                                                                 float* __restrict__ out_depth, BucketOrder bo) {
  __shared__ int queue[kHugeThreads];
  __shared__ int qn;
  const int per = (hw + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per, hi = min(hw, lo + per);
  for (int base = lo; base < hi; base += blockDim.x) {
    if (threadIdx.x == 0) qn = 0;
    __syncthreads();
    const int p = base + threadIdx.x;
    if (p < hi && hash[p].y > kRankMax) queue[atomicAdd(&qn, 1)] = p;
    __syncthreads();
    const int nq = qn;
    for (int q = 0; q < nq; q++) sort_bucket(hash[queue[q]], in, out_idx, out_depth, bo);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// standalone scatter_hashtable over inputs already sorted by pixel id
// ---------------------------------------------------------------------------
__global__ void k_fill_hash(int hw, int2* __restrict__ hash) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < hw; p += gridDim.x * blockDim.x) hash[p] = make_int2(-1, -1);
}

__global__ void __launch_bounds__(256) k_runs(const int* __restrict__ point_idx, const int* __restrict__ point2img,
                                              const float* __restrict__ depth, int n, int hw,
                                              int* __restrict__ out_idx, float* __restrict__ out_depth,
                                              int2* __restrict__ hash) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p = point2img[i];
    const bool valid = 0 <= p && p < hw;
    out_idx[i] = valid ? point_idx[i] : -1;
    out_depth[i] = valid ? depth[i] : -1.0f;
    if (valid && (i == 0 || point2img[i - 1] != p)) {
      int e = i + 1;
      while (e < n && point2img[e] == p) e++;
      hash[p] = make_int2(i, e - i);
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Scratch of hp_pts2plane.  The look-back words and the scalars are adjacent,
// so one memset clears both.
struct BuildLayout {
  size_t counts, pid_slot, depth, tmp, huge, look, scalars, total;
};

static constexpr BuildLayout build_layout(int64_t n, int64_t hw) {
  const int64_t nchunks = (hw + kScanTile - 1) / kScanTile;
  const int64_t tiles = nchunks < kScanMaxTiles ? nchunks : kScanMaxTiles;
  BuildLayout L{};
  size_t o = 0;
  L.counts = o;
  o += align256(sizeof(int) * (size_t)(hw > 0 ? hw : 1));
  L.pid_slot = o;
  o += align256(sizeof(int2) * (size_t)(n > 0 ? n : 1));
  L.depth = o;
  o += align256(sizeof(float) * (size_t)(n > 0 ? n : 1));
  L.tmp = o;
  o += align256(sizeof(int4) * (size_t)(n > 0 ? n : 1));
  L.huge = o;  // pixels of buckets above kRankMax entries: at most n / (kRankMax + 1)
  o += align256(sizeof(int) * (size_t)(n / (kRankMax + 1) + 1));
  L.look = o;
  o += sizeof(unsigned long long) * (size_t)(tiles > 0 ? tiles : 1);
  o = align256(o);
  L.scalars = o;
  o += 256;
  L.total = o;
  return L;
}

static int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = 148 * 16;
  if (g > cap) g = cap;
  return (int)(g > 0 ? g : 1);
}

// Bucket order shared by hp_pts2plane (packed scratch records, count on the
// device) and hp_scatter_hashtable (entries in the caller's sorted input).
// huge: the list of buckets above kRankMax (count in scalars[1]), or null to
// find them by scanning the hash table.
template <class Entries>
static int32_t launch_order(int hw, int n_fixed, int n_grid, Entries in, const int2* hash, const int* scalars,
                            const int* huge, int* out_idx, float* out_depth, BucketOrder bo, cudaStream_t st) {
  if (n_grid > 0) {
    const int g = grid_for(n_grid, 256);
    if (!bo.by_depth && !bo.by_position)
      k_order<Entries, 0, 0><<<g, 256, 0, st>>>(in, hash, hw, scalars, n_fixed, out_idx, out_depth);
    else if (!bo.by_position)
      k_order<Entries, 1, 0><<<g, 256, 0, st>>>(in, hash, hw, scalars, n_fixed, out_idx, out_depth);
    else
      k_order<Entries, 1, 1><<<g, 256, 0, st>>>(in, hash, hw, scalars, n_fixed, out_idx, out_depth);
    if (int32_t rc = check_launch("k_order")) return rc;
  }
  if (huge) {
    k_sort_huge_list<<<148, kHugeThreads, 0, st>>>(huge, scalars, in, hash, out_idx, out_depth, bo);
    return check_launch("k_sort_huge_list");
  }
  const int blocks = (hw + kHugeThreads - 1) / kHugeThreads < 148 * 2 ? (hw + kHugeThreads - 1) / kHugeThreads : 148 * 2;
  k_sort_huge_scan<<<blocks, kHugeThreads, 0, st>>>(hw, in, hash, out_idx, out_depth, bo);
  return check_launch("k_sort_huge_scan");
}

}  // namespace hp

using namespace hp;

extern "C" void hp_projection_rounding(int64_t n_points, int32_t* fused_world, int32_t* fused_image) {
  // Point counts above which torch's cuBLAS GEMM for the 3x3 @ 3xN products of
  // epcq.py:253 (w2c, transposed xyz operand) and epcq.py:261 (K) used a fused
  // multiply-add chain on B200; below them it rounded each product separately.
  if (fused_world) *fused_world = n_points > HP_WORLD_FUSED_ABOVE;
  if (fused_image) *fused_image = n_points > HP_IMAGE_FUSED_ABOVE;
}

extern "C" size_t hp_pts2plane_workspace_size(int64_t n_points, int32_t height, int32_t width) {
  if (n_points < 0 || height <= 0 || width <= 0) return 0;
  return build_layout(n_points, (int64_t)height * width).total;
}

// hp_pts2plane with the scan's test hooks (withhold: see k_scan_hash).
static int32_t pts2plane(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                         int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table, void* workspace,
                         size_t workspace_bytes, hp_stream_t stream, int withhold, int spins) {
  if (!cam) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: cam is NULL");
  const int H = cam->height, W = cam->width;
  if (H <= 0 || W <= 0 || (int64_t)H * W >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: bad image size %dx%d", H, W);
  if (n_points < 0 || n_points > (1ll << 30))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: n_points %lld out of range", (long long)n_points);
  if (!cam->w2c || !cam->K) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: w2c and K are required");
  if ((n_points > 0 && (!xyz || !sorted_point_idx || !sorted_depth)) || !hash_table)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: null input/output pointer");
  if (((uintptr_t)hash_table & 7) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane: hash_table must be 8-byte aligned");
  const int64_t hw = (int64_t)H * W;
  const BuildLayout L = build_layout(n_points, hw);
  if (!workspace || workspace_bytes < L.total || ((uintptr_t)workspace & 255) != 0)
    return set_error(HP_ERR_WORKSPACE, "hp_pts2plane: workspace needs %zu bytes, 256-byte aligned (got %zu)",
                     L.total, workspace_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  int* counts = (int*)(ws + L.counts);
  int2* pid_slot = (int2*)(ws + L.pid_slot);
  float* depth = (float*)(ws + L.depth);
  int4* tmp = (int4*)(ws + L.tmp);
  int* huge = (int*)(ws + L.huge);
  unsigned long long* look = (unsigned long long*)(ws + L.look);
  int* scalars = (int*)(ws + L.scalars);
  int2* hash = (int2*)hash_table;
  const int n = (int)n_points;
  int32_t fw, fi;
  hp_projection_rounding(n_points, &fw, &fi);

  if (cudaMemsetAsync(counts, 0, sizeof(int) * hw, st) != cudaSuccess ||
      cudaMemsetAsync(look, 0, L.total - L.look, st) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "hp_pts2plane: cudaMemsetAsync failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (n > 0) {
    k_project_count<<<grid_for((n + 3) / 4, 256), 256, 0, st>>>(xyz, n, cam->w2c, cam->K, H, W, fw, fi, counts,
                                                                pid_slot, depth);
    if (int32_t rc = check_launch("k_project_count")) return rc;
  }
  const int nchunks = (int)((hw + kScanTile - 1) / kScanTile);
  const int per_tile = (nchunks + kScanMaxTiles - 1) / kScanMaxTiles;
  const int tiles = (nchunks + per_tile - 1) / per_tile;
  k_scan_hash<<<tiles, kScanThreads, 0, st>>>(counts, (int)hw, per_tile, look, hash, scalars, huge, withhold, spins);
  if (int32_t rc = check_launch("k_scan_hash")) return rc;
  if (n > 0) {
    k_scatter<<<grid_for(n, 256), 256, 0, st>>>(n, (int)hw, pid_slot, depth, hash, scalars, tmp,
                                                sorted_point_idx, sorted_depth);
    if (int32_t rc = check_launch("k_scatter")) return rc;
  }
  return launch_order((int)hw, -1, n, PackedEntries{tmp}, hash, scalars, huge, sorted_point_idx, sorted_depth,
                      BucketOrder{sort != 0, 0}, st);
}

extern "C" int32_t hp_pts2plane(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                                int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table, void* workspace,
                                size_t workspace_bytes, hp_stream_t stream) {
  return pts2plane(xyz, n_points, cam, sort, sorted_point_idx, sorted_depth, hash_table, workspace, workspace_bytes,
                   stream, -1, kLookBackSpins);
}

extern "C" int32_t hp_pts2plane_status(const void* workspace, int64_t n_points, int32_t height, int32_t width,
                                       hp_stream_t stream) {
  if (!workspace || n_points < 0 || height <= 0 || width <= 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane_status: bad arguments");
  const BuildLayout L = build_layout(n_points, (int64_t)height * width);
  int flag = 0;
  if (cudaMemcpyAsync(&flag, (const char*)workspace + L.scalars + 3 * sizeof(int), sizeof(int),
                      cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "hp_pts2plane_status: %s", cudaGetErrorString(cudaGetLastError()));
  if (flag) return set_error(HP_ERR_CUDA, "hp_pts2plane: the hash-table scan gave up waiting for a block");
  return HP_OK;
}

#ifdef HP_TESTING
extern "C" int32_t hp_pts2plane_withheld(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                                         int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                                         void* workspace, size_t workspace_bytes, int32_t withhold_tile,
                                         hp_stream_t stream) {
  if (withhold_tile < 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane_withheld: withhold_tile must be >= 0");
  return pts2plane(xyz, n_points, cam, sort, sorted_point_idx, sorted_depth, hash_table, workspace, workspace_bytes,
                   stream, withhold_tile, 1024);
}
#endif

extern "C" int32_t hp_scatter_hashtable(const int32_t* point_idx, const int32_t* point2img, const float* depth,
                                        int64_t n, int32_t height, int32_t width, int32_t sort,
                                        int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                                        hp_stream_t stream) {
  if (height <= 0 || width <= 0 || (int64_t)height * width >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter_hashtable: bad image size %dx%d", height, width);
  if (n < 0 || n > (1ll << 30))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter_hashtable: n %lld out of range", (long long)n);
  if ((n > 0 && (!point_idx || !point2img || !depth || !sorted_point_idx || !sorted_depth)) || !hash_table)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter_hashtable: null pointer");
  if (((uintptr_t)hash_table & 7) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_scatter_hashtable: hash_table must be 8-byte aligned");
  const int hw = height * width;
  cudaStream_t st = (cudaStream_t)stream;
  int2* hash = (int2*)hash_table;
  k_fill_hash<<<grid_for(hw, 256), 256, 0, st>>>(hw, hash);
  if (int32_t rc = check_launch("k_fill_hash")) return rc;
  if (n > 0) {
    k_runs<<<grid_for(n, 256), 256, 0, st>>>(point_idx, point2img, depth, (int)n, hw, sorted_point_idx, sorted_depth,
                                             hash);
    if (int32_t rc = check_launch("k_runs")) return rc;
  }
  if (!sort) return HP_OK;
  // depth order inside each run, ties kept in input order
  return launch_order(hw, (int)n, (int)n, SplitEntries{point_idx, depth, point2img}, hash, nullptr, nullptr,
                      sorted_point_idx, sorted_depth, BucketOrder{1, 1}, st);
}

// ---------------------------------------------------------------------------
// hp_pts2plane_noalloc: hp_pts2plane over a scratch array built into the library
// ---------------------------------------------------------------------------
// For callers that cannot allocate device memory (see the header): the
// scratch hp_pts2plane needs lives in this file-scope __device__ array, which
// every GPU that loads the library holds until the process exits.  Sized for
// the largest problem the entry point accepts.
namespace hp {
constexpr int64_t kNoAllocMaxPoints = HP_NOALLOC_MAX_POINTS;
constexpr int64_t kNoAllocMaxPixels = HP_NOALLOC_MAX_PIXELS;
// build_layout grows with both sizes, so the largest accepted problem bounds every call's scratch
constexpr size_t kNoAllocScratchBytes = build_layout(kNoAllocMaxPoints, kNoAllocMaxPixels).total;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device.  It is looked up again on
// every call made outside stream capture (the lookup is cheap, and a
// cudaDeviceReset since the last call would have reloaded the module at a new
// address); a call made while its stream is being captured uses the address
// its device's last uncaptured call found.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[128] = {nullptr};
}  // namespace hp

extern "C" int32_t hp_pts2plane_noalloc(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                                        int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                                        hp_stream_t stream) {
  if (!cam) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane_noalloc: cam is NULL");
  const int64_t hw = (int64_t)cam->height * cam->width;
  if (n_points > kNoAllocMaxPoints || hw > kNoAllocMaxPixels)
    return set_error(HP_ERR_INVALID_ARGUMENT,
                     "hp_pts2plane_noalloc: %lld points / %lld pixels exceed its built-in scratch "
                     "(at most %lld points and %lld pixels); use hp_pts2plane with a workspace",
                     (long long)n_points, (long long)hw, (long long)kNoAllocMaxPoints, (long long)kNoAllocMaxPixels);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "hp_pts2plane_noalloc: cudaGetDevice failed");
  if (dev < 0 || dev >= 128)
    return set_error(HP_ERR_UNSUPPORTED, "hp_pts2plane_noalloc: device ordinal %d is beyond the 128 devices it tracks",
                     dev);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  const bool capturing =
      cudaStreamIsCapturing((cudaStream_t)stream, &capture) != cudaSuccess || capture != cudaStreamCaptureStatusNone;
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!capturing) {
      const cudaError_t e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_noalloc_addr[dev] = nullptr;
        return set_error(HP_ERR_CUDA, "hp_pts2plane_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      }
    }
    scratch = g_noalloc_addr[dev];
  }
  if (!scratch)
    return set_error(HP_ERR_CUDA,
                     "hp_pts2plane_noalloc: called under stream capture before any uncaptured call on device %d "
                     "(make one call outside capture first)",
                     dev);
  return hp_pts2plane(xyz, n_points, cam, sort, sorted_point_idx, sorted_depth, hash_table, scratch,
                      kNoAllocScratchBytes, stream);
}

extern "C" int32_t hp_pts2plane_noalloc_status(int64_t n_points, int32_t height, int32_t width, hp_stream_t stream) {
  if (n_points < 0 || n_points > kNoAllocMaxPoints || height <= 0 || width <= 0 ||
      (int64_t)height * width > kNoAllocMaxPixels)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane_noalloc_status: bad arguments");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return set_error(HP_ERR_CUDA, "hp_pts2plane_noalloc_status: no usable device");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    scratch = g_noalloc_addr[dev];
  }
  if (!scratch)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_pts2plane_noalloc_status: no hp_pts2plane_noalloc call on device %d",
                     dev);
  return hp_pts2plane_status(scratch, n_points, height, width, stream);
}
