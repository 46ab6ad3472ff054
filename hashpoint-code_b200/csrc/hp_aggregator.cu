// Aggregator forward (epcq/epcq.py:406-507) on the tcgen05 tensor cores.
//
// The reference runs, per valid (sample, point) pair, the 284-wide input
// [feat, PE(feat, 3), PE(dist_feat, 5)] through block1 (284->256->256,
// LeakyReLU) and, with [rgb, dir - ray_d, dir . ray_d] appended, block3
// (263->256->256); the alpha branch (256->1, softplus(x - 1)) and the
// inverse-distance weights then reduce each sample's P points to one alpha and
// one 256-wide feature, which with PE(ray_d, 4) goes through the colour branch
// (280->128->128->128->3, sigmoid).  Everything is fp32 torch, chunked by
// 20000 samples, with boolean-mask gathers and scatters between the layers.
//
// Here two persistent kernels do the whole forward, GEMMs in bf16 with fp32
// accumulation in TMEM:
//
//   k_agg_pairs   one CTA = 128 pair rows (128 / P samples).  Its 256 threads
//                 build the 284-wide inputs (positional encodings with
//                 __sincosf) straight into shared memory as the A operand,
//                 then four layers run back to back: one thread issues
//                 tcgen05.mma over 32-wide K chunks of the pre-packed weights,
//                 which stream through a 4-stage ring of bulk copies
//                 (cp.async.bulk, mbarrier completion); every thread reads its
//                 row's accumulator columns with tcgen05.ld, adds the bias,
//                 applies LeakyReLU and writes the next layer's bf16 A operand
//                 in place.  The last epilogue computes the alpha branch and
//                 the weighted reduction over each sample's P rows (warp
//                 shuffles: a sample's rows are adjacent lanes) and writes the
//                 sample's alpha and its colour-branch input row.
//   k_agg_color   one CTA = 128 samples: the colour-branch input tile arrives
//                 with one bulk copy, three layers on the tensor cores, the
//                 final 128->3 layer and the sigmoid on the CUDA cores.
//   k_agg_scatter alpha and colour of sample m to the m-th set position of
//                 mask_out, zeros elsewhere.
//
// Rows of invalid points are computed like the others (their inputs are the
// zero rows FeatureQuery wrote) and enter the reductions with weight 0, as in
// the reference, where their canvas rows are zeros times weight 0.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "hp_common.cuh"
#include "hp_tc.cuh"

namespace hp {

constexpr int kAggRows = 128;     // pair rows (or samples) per tile = MMA M
constexpr int kAggThreads = 256;  // two threads per row in the epilogues
constexpr int kChunkK = 32;       // K columns of one streamed weight chunk
constexpr int kStages = 4;        // weight chunks in flight
constexpr int kFeatDim = 32;      // pc_feat width the layer sizes imply (284 = 32 + 192 + 60)

// pair layers L = 0..3: K (padded to 32), the layer's real input width, N
__host__ __device__ constexpr int pair_k(int L) { return (L & 1) ? 256 : 288; }
__host__ __device__ constexpr int pair_real_k(int L) { return L == 0 ? 284 : L == 2 ? 263 : 256; }
constexpr int kPairN = 256;
constexpr int kPairChunks = (288 + 256 + 288 + 256) / kChunkK;  // 34
constexpr unsigned kPairChunkBytes = kPairN * kChunkK * 2;       // 16 KB
// colour layers L = 0..2
__host__ __device__ constexpr int color_k(int L) { return L == 0 ? 288 : 128; }
__host__ __device__ constexpr int color_real_k(int L) { return L == 0 ? 280 : 128; }
constexpr int kColorN = 128;
constexpr int kColorChunks = (288 + 128 + 128) / kChunkK;       // 17
constexpr unsigned kColorChunkBytes = kColorN * kChunkK * 2;      // 8 KB
constexpr unsigned kColorTileBytes = kAggRows * 288 * 2;          // one colour-input tile (K = 288)

// packed weight buffer: pair chunks, colour chunks, then fp32 parameters
constexpr size_t kPairBytes = (size_t)kPairChunks * kPairChunkBytes;
constexpr size_t kColorBytes = (size_t)kColorChunks * kColorChunkBytes;
constexpr size_t kParamOff = kPairBytes + kColorBytes;
enum : int {
  kPB1 = 0, kPB2 = 256, kPB3 = 512, kPB4 = 768, kPWA = 1024, kPBA = 1280,
  kPCB1 = 1284, kPCB2 = 1412, kPCB3 = 1540, kPWC4 = 1668, kPCB4 = 2052, kParams = 2056
};
constexpr size_t kPackedBytes = kParamOff + (size_t)kParams * 4;

// shared memory of the two tensor-core kernels
constexpr unsigned kAOff = 0;
constexpr unsigned kPairStageOff = kAggRows * 288 * 2;                         // 73728
constexpr unsigned kPairBarOff = kPairStageOff + kStages * kPairChunkBytes;    // 139264
constexpr unsigned kColorStageOff = kAggRows * 288 * 2;
constexpr unsigned kColorBarOff = kColorStageOff + kStages * kColorChunkBytes;  // 106496

struct Ring {  // barriers and bookkeeping of one CTA's weight stream (thread 0)
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t done;   // all MMAs of a layer completed
  uint64_t aload;  // colour-input tile landed
  uint32_t tmem;
};

struct PairScratch {
  float wgt[kAggRows];         // aggregation weight of each row
  float extra[kAggRows][8];    // rgb, dir - ray_d, dir . ray_d
  float apart[2][kAggRows];    // alpha-branch partial dot products
};

struct ColorScratch {
  float opart[2][kAggRows][4];
};

// Weight chunk stream: chunk g of this CTA is packed chunk g % n_chunks.
struct ChunkStream {
  const uint8_t* base;
  int n_chunks;
  unsigned bytes;
  long long issued, consumed, total;
};

__device__ __forceinline__ bool refill(ChunkStream& s, uint8_t* stages, Ring& ring) {
  while (s.issued < s.total && s.issued < s.consumed + kStages - 1) {
    const int st = (int)(s.issued % kStages);
    if (s.issued >= kStages && !tc::mbar_wait(&ring.empty[st], (unsigned)(((s.issued / kStages) - 1) & 1)))
      return false;
    tc::mbar_arrive_expect_tx(&ring.full[st], s.bytes);
    tc::bulk_load(stages + (size_t)st * s.bytes, s.base + (size_t)(s.issued % s.n_chunks) * s.bytes, s.bytes,
                  &ring.full[st]);
    s.issued++;
  }
  return true;
}

// One layer: D[tmem] = A (K wide, shared memory) * W^T over K / 32 streamed
// chunks, then a commit on ring.done.  Thread 0 only.
__device__ __forceinline__ bool issue_layer(ChunkStream& s, uint8_t* stages, Ring& ring, uint32_t a_addr, int K,
                                            uint32_t d_tmem, uint32_t idesc) {
  bool ok = true;
  for (int c = 0; c < K / kChunkK && ok; c++) {
    const int st = (int)(s.consumed % kStages);
    if (!tc::mbar_wait(&ring.full[st], (unsigned)((s.consumed / kStages) & 1))) {
      ok = false;
      break;
    }
    tc::tc_fence_after();
    const uint32_t b_addr = tc::smem_addr(stages + (size_t)st * s.bytes);
#pragma unroll
    for (int j = 0; j < kChunkK / 16; j++) {
      const int k0 = c * kChunkK + j * 16;
      const uint64_t ad = tc::smem_desc(a_addr + (uint32_t)k0 * 16u, 128u, (uint32_t)K * 16u);
      const uint64_t bd = tc::smem_desc(b_addr + (uint32_t)j * 256u, 128u, (uint32_t)kChunkK * 16u);
      tc::mma_bf16(d_tmem, ad, bd, idesc, (c > 0 || j > 0) ? 1u : 0u);
    }
    tc::mma_commit(&ring.empty[st]);
    s.consumed++;
    ok = refill(s, stages, ring);
  }
  tc::mma_commit(&ring.done);  // also on failure, so the other threads' wait ends
  return ok;
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ void store_unit(uint8_t* A, int r, int u, int K, const float* v) {
  uint4 w;
  w.x = pack2(v[0], v[1]);
  w.y = pack2(v[2], v[3]);
  w.z = pack2(v[4], v[5]);
  w.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4*>(A + tc::operand_offset(r, u * 8, K)) = w;
}

__device__ __forceinline__ float leaky(float x) { return x > 0.0f ? x : __fmul_rn(x, 0.01f); }

__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

// sin / cos column pair j (even: sin, odd: cos) of PE(x, freqs) over C channels:
// argument a = j / 2 is channel a / freqs times 2^(a % freqs).
template <int kFreqs>
__device__ __forceinline__ void pe_pair(const float* x, int a, float& s, float& c) {
  const float arg = __fmul_rn(x[a / kFreqs], (float)(1 << (a % kFreqs)));
  __sincosf(arg, &s, &c);
}

struct AggArgs {
  const uint8_t* packed;
  const float* pc_xyz;   // [M, P, 3]
  const float* pc_rgb;   // [M, P, 3]
  const float* pc_dir;   // [M, P, 3]
  const float* pc_feat;  // [M, P, 32]
  const float* sp_xyz;   // [M, 3]
  const uint8_t* valid;  // [M, P]
  const float* rays_d;   // [M, 3]
  long long M;
  int P;
  uint8_t* color_in;  // colour-branch input tiles (operand layout, K = 288)
  float* alpha;       // [M]
  float* color;       // [M, 3]
  int* status;
};

// ---------------------------------------------------------------------------
// pair MLP: block1, block3, alpha branch, weighted reduction
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAggThreads, 1) k_agg_pairs(AggArgs g, long long n_tiles) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* A = smem + kAOff;
  uint8_t* stages = smem + kPairStageOff;
  Ring& ring = *reinterpret_cast<Ring*>(smem + kPairBarOff);
  PairScratch& sc = *reinterpret_cast<PairScratch*>(smem + kPairBarOff + 256);
  const float* prm = reinterpret_cast<const float*>(g.packed + kParamOff);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int P = g.P, spt = kAggRows / P;

  if (tid == 0) {
    for (int i = 0; i < kStages; i++) {
      tc::mbar_init(&ring.full[i], 1);
      tc::mbar_init(&ring.empty[i], 1);
    }
    tc::mbar_init(&ring.done, 1);
    tc::mbar_init(&ring.aload, 1);
    tc::mbar_init_fence();
  }
  if (warp == 0) tc::tmem_alloc(&ring.tmem, 256);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = ring.tmem;
  const long long my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  ChunkStream cs{g.packed, kPairChunks, kPairChunkBytes, 0, 0, my_tiles * kPairChunks};
  bool fail = false;  // this thread saw a wait give up
  if (tid == 0) fail = !refill(cs, stages, ring);
  int stop = __syncthreads_or(fail);  // every thread takes the same branches
  unsigned done_phase = 0;
  const uint32_t idesc = tc::idesc_bf16(kAggRows, kPairN);

  // this thread's row and column half in the epilogues (TMEM lane quarter = warp % 4)
  const int er = 32 * (warp & 3) + lane, eh = warp >> 2;
  const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);

  for (long long t = blockIdx.x; t < n_tiles && !stop; t += gridDim.x) {
    // ---- inputs: row r = tid % 128, threads 0..127 build units 0..17, 128..255 units 18..35
    {
      const int r = tid & (kAggRows - 1), h = tid >> 7;
      const long long m = t * spt + r / P;
      const int p = r % P;
      const bool in = r < spt * P && m < g.M;
      const long long e = m * P + p;
      float feat[kFeatDim], df[6];
      float inv = 0.0f;
#pragma unroll
      for (int i = 0; i < kFeatDim; i++) feat[i] = 0.0f;
#pragma unroll
      for (int i = 0; i < 6; i++) df[i] = 0.0f;
      if (in) {
        const float4* fp = reinterpret_cast<const float4*>(g.pc_feat + e * kFeatDim);
#pragma unroll
        for (int i = 0; i < kFeatDim / 4; i++) {
          const float4 q = __ldg(fp + i);
          feat[4 * i] = q.x, feat[4 * i + 1] = q.y, feat[4 * i + 2] = q.z, feat[4 * i + 3] = q.w;
        }
        float d2 = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const float x = __ldg(g.pc_xyz + e * 3 + i), s = __ldg(g.sp_xyz + m * 3 + i);
          df[i] = __fsub_rn(x, s);
          df[3 + i] = __fsub_rn(__fmul_rn(x, x), __fmul_rn(s, s));
          d2 = __fmaf_rn(df[i], df[i], d2);
        }
        if (__ldg(g.valid + e)) inv = __fdiv_rn(1.0f, __fadd_rn(sqrtf(d2), 1e-6f));
      }
      if (h == 0) {
        // aggregation weight: inv / (sum over the sample's P rows + 1e-6); the rows are adjacent lanes
        float sum = inv;
        for (int o = 1; o < P; o <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        sc.wgt[r] = __fdiv_rn(inv, __fadd_rn(sum, 1e-6f));
      } else {
        float ex[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (in) {
          float dot = 0.0f;
#pragma unroll
          for (int i = 0; i < 3; i++) {
            const float dv = __ldg(g.pc_dir + e * 3 + i), rd = __ldg(g.rays_d + m * 3 + i);
            ex[i] = __ldg(g.pc_rgb + e * 3 + i);
            ex[3 + i] = __fsub_rn(dv, rd);
            dot = i == 0 ? __fmul_rn(dv, rd) : __fmaf_rn(dv, rd, dot);
          }
          ex[6] = dot;
        }
#pragma unroll
        for (int i = 0; i < 8; i++) sc.extra[r][i] = ex[i];
      }
      // the 284 input columns (+4 zeros) as 36 units of 8: feat 0..3, PE(feat) 4..27, PE(dist_feat) 28..35
#pragma unroll
      for (int u = 0; u < 36; u++) {
        if ((u >= 18) != (h == 1)) continue;
        float v[8];
        if (u < 4) {
#pragma unroll
          for (int i = 0; i < 8; i++) v[i] = feat[8 * u + i];
        } else if (u < 28) {
#pragma unroll
          for (int i = 0; i < 4; i++) pe_pair<3>(feat, (8 * (u - 4)) / 2 + i, v[2 * i], v[2 * i + 1]);
        } else {
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int a = (8 * (u - 28)) / 2 + i;
            if (a < 30) {
              pe_pair<5>(df, a, v[2 * i], v[2 * i + 1]);
            } else {
              v[2 * i] = 0.0f;
              v[2 * i + 1] = 0.0f;
            }
          }
        }
        if (!in) {
#pragma unroll
          for (int i = 0; i < 8; i++) v[i] = 0.0f;
        }
        store_unit(A, r, u, 288, v);
      }
    }
    tc::fence_async_smem();
    tc::tc_fence_before();
    __syncthreads();

    for (int L = 0; L < 4 && !stop; L++) {
      if (tid == 0) {
        tc::tc_fence_after();
        if (!issue_layer(cs, stages, ring, tc::smem_addr(A), pair_k(L), tmem, idesc)) fail = true;
      }
      if (!tc::mbar_wait(&ring.done, done_phase & 1)) fail = true;
      done_phase++;
      tc::tc_fence_after();
      const float* bias = prm + (L == 0 ? kPB1 : L == 1 ? kPB2 : L == 2 ? kPB3 : kPB4);
      const int Knext = L == 1 ? 288 : 256;
      if (L < 3) {
#pragma unroll 1
        for (int cc = 0; cc < 4; cc++) {
          const int col0 = 128 * eh + 32 * cc;
          float v[32];
          tc::tmem_ld32(lane_addr + (uint32_t)col0, v);
#pragma unroll
          for (int i = 0; i < 32; i++) v[i] = leaky(__fadd_rn(v[i], __ldg(bias + col0 + i)));
#pragma unroll
          for (int q = 0; q < 4; q++) store_unit(A, er, col0 / 8 + q, Knext, v + 8 * q);
        }
        if (L == 1 && eh == 1) {  // block3's extra inputs, columns 256..262, zeros to 287
          float v[8];
#pragma unroll
          for (int i = 0; i < 8; i++) v[i] = i < 7 ? sc.extra[er][i] : 0.0f;
          store_unit(A, er, 32, 288, v);
#pragma unroll
          for (int i = 0; i < 8; i++) v[i] = 0.0f;
          store_unit(A, er, 33, 288, v);
          store_unit(A, er, 34, 288, v);
          store_unit(A, er, 35, 288, v);
        }
      } else {
        // block3 output: alpha-branch dot product and the weighted sum over the sample's rows
        const long long m = t * spt + er / P;
        const int p = er % P;
        const bool in = er < spt * P && m < g.M;
        const float w = sc.wgt[er];
        const float* wa = prm + kPWA;
        uint8_t* crow = g.color_in + (size_t)(m / kAggRows) * kColorTileBytes;
        const int cr = (int)(m % kAggRows);
        float adot = 0.0f;
#pragma unroll 1
        for (int cc = 0; cc < 4; cc++) {
          const int col0 = 128 * eh + 32 * cc;
          float v[32];
          tc::tmem_ld32(lane_addr + (uint32_t)col0, v);
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const float f = leaky(__fadd_rn(v[i], __ldg(bias + col0 + i)));
            adot = __fmaf_rn(f, __ldg(wa + col0 + i), adot);
            float x = __fmul_rn(f, w);
            for (int o = 1; o < P; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            v[i] = x;
          }
          if (in) {
#pragma unroll
            for (int q = 0; q < 4; q++)
              if (q % P == p) store_unit(crow, cr, col0 / 8 + q, 288, v + 8 * q);
          }
        }
        sc.apart[eh][er] = adot;
        if (eh == 1 && in && p == 0) {  // PE(ray_d, 4) -> columns 256..279, zeros to 287
          float rd[3];
#pragma unroll
          for (int i = 0; i < 3; i++) rd[i] = __ldg(g.rays_d + m * 3 + i);
#pragma unroll
          for (int u = 0; u < 4; u++) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int a = 4 * u + i;
              if (a < 12) {
                pe_pair<4>(rd, a, v[2 * i], v[2 * i + 1]);
              } else {
                v[2 * i] = 0.0f;
                v[2 * i + 1] = 0.0f;
              }
            }
            store_unit(crow, cr, 32 + u, 288, v);
          }
        }
      }
      tc::tc_fence_before();
      tc::fence_async_smem();
      stop = __syncthreads_or(fail);
    }
    if (stop) break;
    // alpha: softplus(branch - 1) of each valid row, weighted sum over the sample
    if (tid < kAggRows) {
      const int r = tid;
      const long long m = t * spt + r / P;
      const int p = r % P;
      const bool in = r < spt * P && m < g.M;
      float a = 0.0f;
      if (in && __ldg(g.valid + m * P + p)) {
        const float z = __fadd_rn(__fadd_rn(sc.apart[0][r], sc.apart[1][r]), prm[kPBA]);
        a = softplus(__fsub_rn(z, 1.0f));
      }
      float x = __fmul_rn(a, sc.wgt[r]);
      for (int o = 1; o < P; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (in && p == 0) g.alpha[m] = x;
    }
    __syncthreads();
  }

  // drain: every issued copy has landed and every MMA completed before TMEM is freed
  if (tid == 0) {
    for (long long q = cs.consumed; q < cs.issued; q++)
      if (!tc::mbar_wait(&ring.full[q % kStages], (unsigned)((q / kStages) & 1))) fail = true;
    tc::mma_commit(&ring.done);
    if (!tc::mbar_wait(&ring.done, done_phase & 1)) fail = true;
  }
  if (fail) atomicExch(g.status, 1);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 256);
  }
}

// ---------------------------------------------------------------------------
// colour branch
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAggThreads, 2) k_agg_color(AggArgs g, long long n_tiles) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* A = smem + kAOff;
  uint8_t* stages = smem + kColorStageOff;
  Ring& ring = *reinterpret_cast<Ring*>(smem + kColorBarOff);
  ColorScratch& sc = *reinterpret_cast<ColorScratch*>(smem + kColorBarOff + 256);
  const float* prm = reinterpret_cast<const float*>(g.packed + kParamOff);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int i = 0; i < kStages; i++) {
      tc::mbar_init(&ring.full[i], 1);
      tc::mbar_init(&ring.empty[i], 1);
    }
    tc::mbar_init(&ring.done, 1);
    tc::mbar_init(&ring.aload, 1);
    tc::mbar_init_fence();
  }
  if (warp == 0) tc::tmem_alloc(&ring.tmem, 128);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = ring.tmem;
  const long long my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  ChunkStream cs{g.packed + kPairBytes, kColorChunks, kColorChunkBytes, 0, 0, my_tiles * kColorChunks};
  bool fail = false;
  if (tid == 0) fail = !refill(cs, stages, ring);
  int stop = __syncthreads_or(fail);
  unsigned done_phase = 0, a_phase = 0;
  bool a_pending = false;
  const uint32_t idesc = tc::idesc_bf16(kAggRows, kColorN);
  const int er = 32 * (warp & 3) + lane, eh = warp >> 2;
  const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);

  for (long long t = blockIdx.x; t < n_tiles && !stop; t += gridDim.x) {
    for (int L = 0; L < 3 && !stop; L++) {
      if (tid == 0) {
        bool ok = true;
        if (L == 0) {  // this tile's inputs (the previous tile's MMAs have completed)
          tc::mbar_arrive_expect_tx(&ring.aload, kColorTileBytes);
          tc::bulk_load(A, g.color_in + (size_t)t * kColorTileBytes, kColorTileBytes, &ring.aload);
          a_pending = true;
          ok = tc::mbar_wait(&ring.aload, a_phase & 1);
          if (ok) a_pending = false;
          a_phase++;
        }
        tc::tc_fence_after();
        if (!ok) {
          fail = true;
          tc::mma_commit(&ring.done);
        } else if (!issue_layer(cs, stages, ring, tc::smem_addr(A), color_k(L), tmem, idesc)) {
          fail = true;
        }
      }
      if (!tc::mbar_wait(&ring.done, done_phase & 1)) fail = true;
      done_phase++;
      tc::tc_fence_after();
      const float* bias = prm + (L == 0 ? kPCB1 : L == 1 ? kPCB2 : kPCB3);
      if (L < 2) {
#pragma unroll 1
        for (int cc = 0; cc < 2; cc++) {
          const int col0 = 64 * eh + 32 * cc;
          float v[32];
          tc::tmem_ld32(lane_addr + (uint32_t)col0, v);
#pragma unroll
          for (int i = 0; i < 32; i++) v[i] = leaky(__fadd_rn(v[i], __ldg(bias + col0 + i)));
#pragma unroll
          for (int q = 0; q < 4; q++) store_unit(A, er, col0 / 8 + q, 128, v + 8 * q);
        }
      } else {
        float o[3] = {0.0f, 0.0f, 0.0f};
        const float* wc = prm + kPWC4;
#pragma unroll 1
        for (int cc = 0; cc < 2; cc++) {
          const int col0 = 64 * eh + 32 * cc;
          float v[32];
          tc::tmem_ld32(lane_addr + (uint32_t)col0, v);
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const float f = leaky(__fadd_rn(v[i], __ldg(bias + col0 + i)));
#pragma unroll
            for (int j = 0; j < 3; j++) o[j] = __fmaf_rn(f, __ldg(wc + j * 128 + col0 + i), o[j]);
          }
        }
#pragma unroll
        for (int j = 0; j < 3; j++) sc.opart[eh][er][j] = o[j];
      }
      tc::tc_fence_before();
      tc::fence_async_smem();
      stop = __syncthreads_or(fail);
    }
    if (stop) break;
    if (tid < kAggRows) {
      const long long m = t * kAggRows + tid;
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const float z = __fadd_rn(__fadd_rn(sc.opart[0][tid][j], sc.opart[1][tid][j]), prm[kPCB4 + j]);
          const float s = 1.0f / (1.0f + expf(-z));
          g.color[m * 3 + j] = __fsub_rn(__fmul_rn(s, 1.002f), 0.001f);
        }
      }
    }
    __syncthreads();
  }

  if (tid == 0) {
    if (a_pending && !tc::mbar_wait(&ring.aload, (a_phase - 1) & 1)) fail = true;
    for (long long q = cs.consumed; q < cs.issued; q++)
      if (!tc::mbar_wait(&ring.full[q % kStages], (unsigned)((q / kStages) & 1))) fail = true;
    tc::mma_commit(&ring.done);
    if (!tc::mbar_wait(&ring.done, done_phase & 1)) fail = true;
  }
  if (fail) atomicExch(g.status, 1);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 128);
  }
}

// alpha / colour of sample offsets[i] at every set position i of mask_out, zeros elsewhere
__global__ void k_agg_scatter(const uint8_t* __restrict__ mask, const int* __restrict__ offsets, long long n,
                              long long M, const float* __restrict__ alpha, const float* __restrict__ color,
                              float* __restrict__ alpha_out, float* __restrict__ color_out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long m = offsets[i];
  const bool set = mask[i] != 0 && m < M;
  alpha_out[i] = set ? alpha[m] : 0.0f;
#pragma unroll
  for (int j = 0; j < 3; j++) color_out[i * 3 + j] = set ? color[m * 3 + j] : 0.0f;
}

// ---------------------------------------------------------------------------
// weight packing: fp32 nn.Linear weights -> bf16 chunks in operand layout
// ---------------------------------------------------------------------------
struct PackArgs {
  const float* w[9];
  const float* b[9];
};

// element e of a chunk stream of N-row chunks -> (chunk, n, k within the chunk)
__device__ __forceinline__ void chunk_coords(long long e, int N, int& chunk, int& n, int& k) {
  const int per = N * kChunkK;
  chunk = (int)(e / per);
  const int o = (int)(e % per) * 2;  // byte offset in the chunk
  const int ng = o / (kChunkK * 16), rem = o % (kChunkK * 16);
  const int kk = rem / 128, rem2 = rem % 128;
  n = ng * 8 + rem2 / 16;
  k = kk * 8 + (rem2 % 16) / 2;
}

__global__ void k_agg_pack(PackArgs a, uint8_t* __restrict__ packed) {
  const long long n_pair = (long long)kPairBytes / 2, n_color = (long long)kColorBytes / 2;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  __nv_bfloat16* out = reinterpret_cast<__nv_bfloat16*>(packed);
  if (e < n_pair) {
    int chunk, n, k;
    chunk_coords(e, kPairN, chunk, n, k);
    int L = 0, c0 = 0;
    while (chunk >= c0 + pair_k(L) / kChunkK) c0 += pair_k(L++) / kChunkK;
    const int kk = (chunk - c0) * kChunkK + k;
    const int wi = L;  // block1.0, block1.2, block3.0, block3.2
    out[e] = __float2bfloat16_rn(kk < pair_real_k(L) ? a.w[wi][(size_t)n * pair_real_k(L) + kk] : 0.0f);
  } else if (e < n_pair + n_color) {
    const long long f = e - n_pair;
    int chunk, n, k;
    chunk_coords(f, kColorN, chunk, n, k);
    int L = 0, c0 = 0;
    while (chunk >= c0 + color_k(L) / kChunkK) c0 += color_k(L++) / kChunkK;
    const int kk = (chunk - c0) * kChunkK + k;
    const int wi = 5 + L;  // color_branch.0, .2, .4
    out[e] = __float2bfloat16_rn(kk < color_real_k(L) ? a.w[wi][(size_t)n * color_real_k(L) + kk] : 0.0f);
  } else if (e < n_pair + n_color + kParams) {
    const int q = (int)(e - n_pair - n_color);
    float* prm = reinterpret_cast<float*>(packed + kParamOff);
    float v = 0.0f;
    if (q < kPWA) v = a.b[q / 256][q % 256];
    else if (q < kPBA) v = a.w[4][q - kPWA];
    else if (q < kPCB1) v = q == kPBA ? a.b[4][0] : 0.0f;
    else if (q < kPWC4) v = a.b[5 + (q - kPCB1) / 128][(q - kPCB1) % 128];
    else if (q < kPCB4) v = a.w[8][q - kPWC4];
    else v = q < kPCB4 + 3 ? a.b[8][q - kPCB4] : 0.0f;
    prm[q] = v;
  }
}

static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess || n <= 0)
      n = 148;
  }
  return n;
}

}  // namespace hp

using namespace hp;

namespace {
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct AggLayout {
  size_t color_in, alpha, color, status, total;
};

AggLayout agg_layout(long long M) {
  AggLayout L;
  const long long tiles = (M + kAggRows - 1) / kAggRows;
  size_t o = 0;
  L.color_in = o;
  o += align256((size_t)(tiles > 0 ? tiles : 1) * kColorTileBytes);
  L.alpha = o;
  o += align256(sizeof(float) * (size_t)(M > 0 ? M : 1));
  L.color = o;
  o += align256(sizeof(float) * 3 * (size_t)(M > 0 ? M : 1));
  L.status = o;
  o += 256;
  L.total = o;
  return L;
}

constexpr unsigned kPairSmem = kPairBarOff + 256 + sizeof(PairScratch) + 1024;
constexpr unsigned kColorSmem = kColorBarOff + 256 + sizeof(ColorScratch) + 1024;
static_assert(sizeof(Ring) <= 256, "barrier block");
static_assert(kPairSmem <= 227 * 1024 && kColorSmem <= 227 * 1024, "shared memory");
}  // namespace

extern "C" size_t hp_aggregator_packed_size(void) { return kPackedBytes; }

extern "C" int32_t hp_aggregator_pack(const hp_aggregator_weights* w, void* packed, size_t packed_bytes,
                                      hp_stream_t stream) {
  if (!w || !packed) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_aggregator_pack: null pointer");
  if (packed_bytes < kPackedBytes || ((uintptr_t)packed & 255) != 0)
    return set_error(HP_ERR_WORKSPACE, "hp_aggregator_pack: needs %zu bytes, 256-byte aligned", kPackedBytes);
  PackArgs a;
  for (int i = 0; i < 9; i++) {
    if (!w->weight[i] || !w->bias[i]) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_aggregator_pack: layer %d", i);
    a.w[i] = w->weight[i];
    a.b[i] = w->bias[i];
  }
  const long long n = (long long)(kPairBytes + kColorBytes) / 2 + kParams;
  k_agg_pack<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, (uint8_t*)packed);
  return check_launch("k_agg_pack");
}

extern "C" size_t hp_aggregator_workspace_size(int64_t n_samples) {
  if (n_samples < 0) return 0;
  return agg_layout(n_samples).total;
}

extern "C" int32_t hp_aggregator_forward(const void* packed, const float* pc_xyz, const float* pc_rgb,
                                         const float* pc_dir, const float* pc_feat, int32_t feat_dim,
                                         const float* sp_xyz, const uint8_t* valid, const float* rays_d,
                                         int64_t n_samples, int32_t P, const uint8_t* mask_out,
                                         const int32_t* mask_offsets, int64_t n_positions, float* alpha_out,
                                         float* color_out, void* workspace, size_t workspace_bytes,
                                         hp_stream_t stream) {
  static const char* who = "hp_aggregator_forward";
  if (feat_dim != kFeatDim)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: feature width %d (the layers take %d)", who, feat_dim, kFeatDim);
  if (P < 1 || P > 32 || (P & (P - 1)) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: points per sample %d (1, 2, 4, ..., 32 supported)", who, P);
  if (n_samples < 0 || n_samples * P >= (1ll << 40) || n_positions < 0 || n_positions >= (1ll << 31))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: sizes out of range", who);
  if (!packed || !workspace || (n_positions > 0 && (!mask_out || !mask_offsets || !alpha_out || !color_out)) ||
      (n_samples > 0 && (!pc_xyz || !pc_rgb || !pc_dir || !pc_feat || !sp_xyz || !valid || !rays_d)))
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: null pointer", who);
  if (((uintptr_t)pc_feat & 15) != 0 || ((uintptr_t)packed & 255) != 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "%s: pc_feat must be 16-byte and packed 256-byte aligned", who);
  const AggLayout L = agg_layout(n_samples);
  if (workspace_bytes < L.total || ((uintptr_t)workspace & 255) != 0)
    return set_error(HP_ERR_WORKSPACE, "%s: workspace needs %zu bytes, 256-byte aligned", who, L.total);
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  AggArgs g;
  g.packed = (const uint8_t*)packed;
  g.pc_xyz = pc_xyz;
  g.pc_rgb = pc_rgb;
  g.pc_dir = pc_dir;
  g.pc_feat = pc_feat;
  g.sp_xyz = sp_xyz;
  g.valid = valid;
  g.rays_d = rays_d;
  g.M = n_samples;
  g.P = P;
  g.color_in = (uint8_t*)(ws + L.color_in);
  g.alpha = (float*)(ws + L.alpha);
  g.color = (float*)(ws + L.color);
  g.status = (int*)(ws + L.status);
  if (cudaMemsetAsync(g.status, 0, sizeof(int), st) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "%s: memset failed", who);
  if (n_samples > 0) {
    static bool attr = false;
    if (!attr) {
      if (cudaFuncSetAttribute(k_agg_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmem) != cudaSuccess ||
          cudaFuncSetAttribute(k_agg_color, cudaFuncAttributeMaxDynamicSharedMemorySize, kColorSmem) != cudaSuccess)
        return set_error(HP_ERR_CUDA, "%s: cudaFuncSetAttribute failed", who);
      attr = true;
    }
    const int spt = kAggRows / P;
    const long long pair_tiles = (n_samples + spt - 1) / spt;
    const long long color_tiles = (n_samples + kAggRows - 1) / kAggRows;
    const int sms = sm_count();
    const unsigned pg = (unsigned)(pair_tiles < sms ? pair_tiles : sms);
    const unsigned cg = (unsigned)(color_tiles < 2 * sms ? color_tiles : 2 * sms);
    k_agg_pairs<<<pg, kAggThreads, kPairSmem, st>>>(g, pair_tiles);
    if (int32_t rc = check_launch("k_agg_pairs")) return rc;
    k_agg_color<<<cg, kAggThreads, kColorSmem, st>>>(g, color_tiles);
    if (int32_t rc = check_launch("k_agg_color")) return rc;
  }
  if (n_positions > 0) {
    k_agg_scatter<<<(unsigned)((n_positions + 255) / 256), 256, 0, st>>>(mask_out, mask_offsets, n_positions,
                                                                         n_samples, g.alpha, g.color, alpha_out,
                                                                         color_out);
    if (int32_t rc = check_launch("k_agg_scatter")) return rc;
  }
  return HP_OK;
}

extern "C" int32_t hp_aggregator_status(const void* workspace, int64_t n_samples, hp_stream_t stream) {
  if (!workspace || n_samples < 0) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_aggregator_status: bad arguments");
  const AggLayout L = agg_layout(n_samples);
  int flag = 0;
  if (cudaMemcpyAsync(&flag, (const char*)workspace + L.status, sizeof(int), cudaMemcpyDeviceToHost,
                      (cudaStream_t)stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "hp_aggregator_status: %s", cudaGetErrorString(cudaGetLastError()));
  if (flag) return set_error(HP_ERR_CUDA, "hp_aggregator_forward: a tensor-core wait timed out");
  return HP_OK;
}
