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
//   k_agg_pairs   one tile = 128 pair rows (128 / P samples), one CTA per SM,
//                 warp-specialised:
//                   warps 0-15 build the tile's 284-wide inputs (positional
//                              encodings: one __sincosf per channel, higher
//                              bands by the double-angle formulas) into the
//                              layer-1 operand A0, and run the epilogues: read
//                              the accumulator with tcgen05.ld, add the bias,
//                              LeakyReLU, write the next layer's bf16 operand
//                              A1 in 64-column blocks, each released to the
//                              MMA warp by its own barrier, so the next layer
//                              starts while later blocks are being written
//                              (block3's seven extra inputs go to a separate
//                              16-wide operand E);
//                              (warp w: TMEM lane quarter w % 4, columns
//                              64 (w / 4) .. + 63 of its row);
//                   warp 16    issues tcgen05.mma (M 128, N 256, K 16) from
//                              A0 / A1 / E and the streamed weights;
//                   warp 17    streams the pre-packed weights (256 outputs x 32
//                              K, 16 KB, 64-byte swizzled) from L2 into a
//                              4-stage ring with cp.async.bulk.
//                 Two TMEM accumulators (layers alternate), so the next
//                 tile's layer 1 runs while this tile's last epilogue
//                 computes the alpha branch and the weighted reduction over
//                 each sample's rows, and the next tile's inputs are built
//                 while this tile's layer 4 runs.
//   k_agg_color   one CTA = 128 samples: the colour-branch input tile arrives
//                 with one bulk copy, three layers on the tensor cores, the
//                 final 128->3 layer and the sigmoid on the CUDA cores.
//   k_agg_scatter alpha and colour of sample m to the m-th set position of
//                 mask_out, zeros elsewhere.
//
// Rows of invalid points are computed like the others (their inputs are the
// zero rows FeatureQuery wrote) and enter the reductions with weight 0, as in
// the reference, where their canvas rows are zeros times weight 0.  Every
// wait is bounded; a wait that gives up sets the CTA's abort flag (the other
// roles' waits then give up at once) and the status word.
#include <cuda_bf16.h>

#include <mutex>

#include "hp_common.cuh"
#include "hp_tc.cuh"
#ifdef HP_TESTING
#include "../../include/hashpoint_b200_testing.h"
#endif

namespace hp {

constexpr int kAggRows = 128;                      // pair rows (or samples) per tile = MMA M
constexpr int kMathThreads = 512;                  // warps 0..15
constexpr int kPairThreads = kMathThreads + 64;    // + MMA warp + load warp
constexpr int kColorThreads = 256;
constexpr int kMmaWarp = 16, kLoadWarp = 17;
constexpr int kPairChunkK = 32;                    // pair weight chunk: 256 outputs x 32 K, 64-byte swizzled
constexpr int kChunkK = 64;                        // colour weight chunk: 128 outputs x 64 K, 128-byte swizzled
constexpr int kChunkN = 128;
constexpr unsigned kChunkBytes = 16384;            // either chunk
constexpr int kStages = 4;                         // weight chunks in flight
constexpr int kFeatDim = 32;                       // pc_feat width the layer sizes imply (284 = 32 + 192 + 60)

// pair layers L = 0..3: padded K of the streamed operand (block3.0's seven
// extra inputs, columns 256..262, go through their own K = 16 MMA), real input width
__host__ __device__ constexpr int pair_k(int L) { return L == 0 ? 320 : 256; }
__host__ __device__ constexpr int pair_real_k(int L) { return L == 0 ? 284 : L == 2 ? 263 : 256; }
constexpr int kPairN = 256;
constexpr int kPairChunks = (320 + 256 + 256 + 256) / kPairChunkK;  // 34
// colour layers L = 0..2
__host__ __device__ constexpr int color_k(int L) { return L == 0 ? 320 : 128; }
__host__ __device__ constexpr int color_real_k(int L) { return L == 0 ? 280 : 128; }
constexpr int kColorN = 128;
constexpr int kColorChunks = (320 + 128 + 128) / kChunkK;  // 9
constexpr int kWideK = 320;
constexpr unsigned kATileBytes = kAggRows * kWideK * 2;     // 80 KB: A0, or one colour-input tile
constexpr unsigned kA1Bytes = kAggRows * 256 * 2;           // 64 KB
constexpr unsigned kEBytes = kAggRows * 16 * 2;             // extras operand, no swizzle
constexpr unsigned kW3bBytes = kPairN * 16 * 2;             // block3.0 columns 256..262 (+ zeros), no swizzle

// packed weight buffer: pair chunks, W3b, colour chunks, fp32 parameters
constexpr size_t kPairBytes = (size_t)kPairChunks * kChunkBytes;
constexpr size_t kW3bOff = kPairBytes;
constexpr size_t kColorOff = kW3bOff + kW3bBytes;
constexpr size_t kColorBytes = (size_t)kColorChunks * kChunkBytes;
constexpr size_t kParamOff = kColorOff + kColorBytes;
enum : int {
  kPB1 = 0, kPB2 = 256, kPB3 = 512, kPB4 = 768, kPWA = 1024, kPBA = 1280,
  kPCB1 = 1284, kPCB2 = 1412, kPCB3 = 1540, kPWC4 = 1668, kPCB4 = 2052, kParams = 2056
};
constexpr size_t kPackedBytes = kParamOff + (size_t)kParams * 4;

// pair kernel shared memory (from a 1024-byte aligned base)
constexpr unsigned kPA0 = 0;
constexpr unsigned kPA1 = kPA0 + kATileBytes;
constexpr unsigned kPStages = kPA1 + kA1Bytes;
constexpr unsigned kPE = kPStages + kStages * kChunkBytes;
constexpr unsigned kPW3b = kPE + kEBytes;
constexpr unsigned kPBar = kPW3b + kW3bBytes;
constexpr unsigned kPScratch = kPBar + 256;
// colour kernel shared memory
constexpr unsigned kCStages = kATileBytes;
constexpr unsigned kCBar = kCStages + kStages * kChunkBytes;
constexpr unsigned kCScratch = kCBar + 256;
constexpr int kRed = 32;  // the last epilogue's transpose buffer: 32 x 32 floats per warp, column c of row r at c ^ r

struct PairBars {
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t acc_full[2];  // MMA warp -> math warps: a layer completed into accumulator i
  uint64_t a0_ready;     // math warps -> MMA warp: a tile's layer-1 operand is written (256 arrivals)
  uint64_t a1_blk[4];    // math warps -> MMA warp: 64-column block i of the next layer's operand is written
  uint64_t w3b;          // W3b landed
  uint64_t idle;         // MMA warp: everything it issued has completed
  uint32_t tmem;
  int abort;
};

struct PairScratch {
  float wgt[2][kAggRows];    // aggregation weight of each row, by tile parity
  float apart[4][kAggRows];  // alpha-branch partial dot products (column quarters)
};

struct Ring {  // colour kernel: barriers and bookkeeping of one CTA's weight stream (thread 0)
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t done;   // all MMAs of a layer completed
  uint64_t aload;  // colour-input tile landed
  uint32_t tmem;
};

struct ColorScratch {
  float opart[2][kAggRows][4];
};

// Wait for a phase; gives up (and raises the CTA's abort flag) after limit_ns,
// or at once when another role raised it.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, unsigned parity, volatile int* abort,
                                              unsigned long long limit_ns) {
  if (tc::mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = tc::global_ns();
  for (;;) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
    if (tc::global_ns() - t0 > limit_ns) {
      *abort = 1;
      return false;
    }
  }
}

// Weight chunk stream of the colour kernel: chunk g of this CTA is packed chunk g % n_chunks.
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

// One colour layer: D[tmem] = A (K wide) * W^T over K / 64 streamed chunks, then a
// commit on ring.done.  Thread 0 only.
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
    for (int j = 0; j < kChunkK / 16; j++)
      tc::mma_bf16(d_tmem, tc::smem_desc_sw128(a_addr + (uint32_t)c * (kAggRows * 128) + (uint32_t)j * 32u),
                   tc::smem_desc_sw128(b_addr + (uint32_t)j * 32u), idesc, (c > 0 || j > 0) ? 1u : 0u);
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

__device__ __forceinline__ uint4 pack8(const float* v) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

// columns 8u .. 8u + 7 of row r of a 128-row swizzled operand
__device__ __forceinline__ void store_unit(uint8_t* A, int r, int u, const float* v) {
  *reinterpret_cast<uint4*>(A + tc::operand_offset(r, u * 8, kAggRows)) = pack8(v);
}

__device__ __forceinline__ void zero_unit(uint8_t* A, int r, int u) {
  *reinterpret_cast<uint4*>(A + tc::operand_offset(r, u * 8, kAggRows)) = make_uint4(0, 0, 0, 0);
}

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  const uint32_t a = tc::smem_addr(p);
  return p + (((a + 1023u) & ~1023u) - a);
}

// LeakyReLU(0.01): max(x, 0.01 x) is x for x >= 0 and 0.01 x below.
__device__ __forceinline__ float leaky(float x) { return fmaxf(x, __fmul_rn(x, 0.01f)); }

__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

// sin / cos of x * 2^f, f < F: one __sincosf, then sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a.
template <int F>
__device__ __forceinline__ void bands(float x, float* s, float* c) {
  __sincosf(x, &s[0], &c[0]);
#pragma unroll
  for (int f = 1; f < F; f++) {
    s[f] = __fmul_rn(2.0f, __fmul_rn(s[f - 1], c[f - 1]));
    c[f] = __fmaf_rn(-2.0f * s[f - 1], s[f - 1], 1.0f);
  }
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
  uint8_t* color_in;  // colour-branch input tiles (operand layout, K = 320)
  float* alpha;       // [M]
  float* color;       // [M, 3]
  int* status;
  unsigned long long wait_ns;  // limit of each wait of the pair kernel's roles (tc::kWaitNs)
  int withhold_w3b;            // a test of those waits: W3b is never loaded, so its wait gives up
};

// Layer-1 operand units U0 .. U1-1 of row r: columns 0..31 feat, 32..223 PE(feat, 3)
// (argument a = channel * 3 + band at columns 32 + 2a (sin), 33 + 2a (cos)), 224..283
// PE(dist_feat, 5), 284 the constant 1 (its weight column holds block1.0's bias),
// 285..319 zeros.
template <int U0, int U1>
__device__ __forceinline__ void input_units(uint8_t* A0, int r, bool in, const float* feat, const float* df) {
  float sf[3], cf[3], sd[5], cd[5];
  int chf = -1, chd = -1;
#pragma unroll
  for (int u = U0; u < U1; u++) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int col = 8 * u + i;
      float x = 0.0f;
      if (col < 32) {
        x = feat[col];
      } else if (col < 224) {
        const int a = (col - 32) >> 1, c = a / 3, f = a % 3;
        if (c != chf) {
          bands<3>(feat[c], sf, cf);
          chf = c;
        }
        x = ((col - 32) & 1) ? cf[f] : sf[f];
      } else if (col < 284) {
        const int a = (col - 224) >> 1, c = a / 5, f = a % 5;
        if (c != chd) {
          bands<5>(df[c], sd, cd);
          chd = c;
        }
        x = ((col - 224) & 1) ? cd[f] : sd[f];
      } else if (col == 284) {
        x = 1.0f;
      }
      v[i] = in ? x : 0.0f;
    }
    store_unit(A0, r, u, v);
  }
}

// The math warps' view of one tile's inputs: builds A0 and the rows' aggregation weights.
__device__ __forceinline__ void build_inputs(const AggArgs& g, long long t, int spt, uint8_t* A0, float* wgt,
                                             int tid) {
  const int P = g.P;
  const int r = tid & (kAggRows - 1), h = tid >> 7;  // h: which 10 of the row's 40 units
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
    wgt[r] = __fdiv_rn(inv, __fadd_rn(sum, 1e-6f));
    input_units<0, 10>(A0, r, in, feat, df);
  } else if (h == 1) {
    input_units<10, 20>(A0, r, in, feat, df);
  } else if (h == 2) {
    input_units<20, 30>(A0, r, in, feat, df);
  } else {
    input_units<30, 40>(A0, r, in, feat, df);
  }
}

// Epilogue of a hidden layer, written in K order so the next layer's MMAs can
// start on a block while later blocks are still being written: in round kb
// every math thread converts columns 64 kb + 16 g .. + 15 (g = warp / 4) of its
// row er -> LeakyReLU(x + bias) -> bf16 into the next operand (A1), then
// arrives on block kb's barrier.  `last` runs before the final arrival.  bias is
// null for the layers whose bias came in through the MMA.
template <class Last>
__device__ __forceinline__ void epilogue_hidden(uint32_t acc_addr, const float* bias, uint8_t* A1, int er, int g,
                                                uint64_t* blk, Last&& last) {
#pragma unroll 1
  for (int kb = 0; kb < 4; kb++) {
    const int col0 = 64 * kb + 16 * g;
    float v[16];
    tc::tmem_ld16(acc_addr + (uint32_t)col0, v);
    if (bias) {
      const float4* b4 = reinterpret_cast<const float4*>(bias + col0);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 b = __ldg(b4 + q);
        v[4 * q] = __fadd_rn(v[4 * q], b.x);
        v[4 * q + 1] = __fadd_rn(v[4 * q + 1], b.y);
        v[4 * q + 2] = __fadd_rn(v[4 * q + 2], b.z);
        v[4 * q + 3] = __fadd_rn(v[4 * q + 3], b.w);
      }
    }
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = leaky(v[i]);
    store_unit(A1, er, col0 / 8, v);
    store_unit(A1, er, col0 / 8 + 1, v + 8);
    if (kb == 3) last();
    tc::tc_fence_before();
    tc::fence_async_smem();
    tc::mbar_arrive(&blk[kb]);
  }
}

// Column sums over each sample's P rows of one warp's 32 x 32 transpose buffer (row =
// pair row, column = this lane's feature column; written in place into rows 0..G-1),
// then the sums to the colour-input rows, 8 columns per store.
template <int P>
__device__ __forceinline__ void sample_sums(float* red, int lane, long long m0, long long M, uint8_t* color_in,
                                            int col0) {
  constexpr int G = 32 / P;
#pragma unroll
  for (int gs = 0; gs < G; gs++) {
    float v[P];
#pragma unroll
    for (int p = 0; p < P; p++) v[p] = red[(gs * P + p) * kRed + (lane ^ (gs * P + p))];
    float acc = v[0];
#pragma unroll
    for (int p = 1; p < P; p++) acc = __fadd_rn(acc, v[p]);
    if (P > 1) red[gs * kRed + (lane ^ gs)] = acc;  // rows below gs * P are read already
  }
  __syncwarp();
  for (int un = lane; un < G * 4; un += 32) {
    const int gs = un >> 2, q = un & 3;
    const long long m = m0 + gs;
    if (m < M) {
      float o[8];
#pragma unroll
      for (int i = 0; i < 8; i++) o[i] = red[gs * kRed + ((8 * q + i) ^ gs)];
      store_unit(color_in + (size_t)(m / kAggRows) * kATileBytes, (int)(m % kAggRows), col0 / 8 + q, o);
    }
  }
}

// ---------------------------------------------------------------------------
// pair MLP: block1, block3, alpha branch, weighted reduction
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPairThreads, 1) k_agg_pairs(AggArgs g, long long n_tiles) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* A0 = smem + kPA0;
  uint8_t* A1 = smem + kPA1;
  uint8_t* stages = smem + kPStages;
  uint8_t* E = smem + kPE;
  uint8_t* W3b = smem + kPW3b;
  PairBars& bar = *reinterpret_cast<PairBars*>(smem + kPBar);
  PairScratch& sc = *reinterpret_cast<PairScratch*>(smem + kPScratch);
  volatile int* abort = &bar.abort;
  const float* prm = reinterpret_cast<const float*>(g.packed + kParamOff);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int P = g.P, spt = kAggRows / P;

  if (tid == 0) {
    for (int i = 0; i < kStages; i++) {
      tc::mbar_init(&bar.full[i], 1);
      tc::mbar_init(&bar.empty[i], 1);
    }
    tc::mbar_init(&bar.acc_full[0], 1);
    tc::mbar_init(&bar.acc_full[1], 1);
    tc::mbar_init(&bar.a0_ready, kMathThreads);
    for (int i = 0; i < 4; i++) tc::mbar_init(&bar.a1_blk[i], kMathThreads);
    tc::mbar_init(&bar.w3b, 1);
    tc::mbar_init(&bar.idle, 1);
    bar.abort = 0;
    tc::mbar_init_fence();
  }
  if (warp == 0) tc::tmem_alloc(&bar.tmem, 512);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = bar.tmem;
  const long long my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  bool fail = false;

  if (warp == kLoadWarp) {
    // ---- weight loads: W3b once, then the pair chunk stream, 34 chunks per tile
    if (lane == 0) {
      if (!g.withhold_w3b) {
        tc::mbar_arrive_expect_tx(&bar.w3b, kW3bBytes);
        tc::bulk_load(W3b, g.packed + kW3bOff, kW3bBytes, &bar.w3b);
      }
      const long long total = my_tiles * kPairChunks;
      long long q = 0;
      for (; q < total; q++) {
        const int st = (int)(q % kStages);
        if (q >= kStages && !wait_or_abort(&bar.empty[st], (unsigned)(((q / kStages) - 1) & 1), abort, g.wait_ns))
          break;
        tc::mbar_arrive_expect_tx(&bar.full[st], kChunkBytes);
        tc::bulk_load(stages + (size_t)st * kChunkBytes, g.packed + (size_t)(q % kPairChunks) * kChunkBytes,
                      kChunkBytes, &bar.full[st]);
      }
      // the last copy into each stage has landed before the CTA ends
      for (long long d = q - 1; d >= 0 && d >= q - kStages; d--)
        if (!tc::mbar_wait(&bar.full[d % kStages], (unsigned)((d / kStages) & 1))) fail = true;
      if (!g.withhold_w3b && !tc::mbar_wait(&bar.w3b, 0)) fail = true;
    }
    __syncwarp();  // the warp's other lanes wait for lane 0 here, not at the block barrier
  } else if (warp == kMmaWarp) {
    // ---- MMA issue: per tile, layers 0..3 into accumulators 0, 1, 0, 1
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16(kAggRows, kPairN);
      unsigned a0_ph = 0, a1_ph = 0;
      long long q = 0;
      bool ok = wait_or_abort(&bar.w3b, 0, abort, g.wait_ns);
      for (long long t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        for (int L = 0; L < 4 && ok; L++) {
          if (L == 0) {
            if (!(ok = wait_or_abort(&bar.a0_ready, (a0_ph++) & 1, abort, g.wait_ns))) break;
            tc::tc_fence_after();
          }
          const uint32_t acc = tmem + (uint32_t)(L & 1) * 256u;
          const uint32_t a_addr = tc::smem_addr(L == 0 ? A0 : A1);
          const int nk = pair_k(L) / kPairChunkK;
          for (int kc = 0; kc < nk; kc++, q++) {
            if (L > 0 && (kc & 1) == 0) {  // A1's 64-column block kc / 2 is written
              if (!(ok = wait_or_abort(&bar.a1_blk[kc >> 1], a1_ph & 1, abort, g.wait_ns))) break;
              tc::tc_fence_after();
            }
            const int st = (int)(q % kStages);
            if (!(ok = wait_or_abort(&bar.full[st], (unsigned)((q / kStages) & 1), abort, g.wait_ns))) break;
            tc::tc_fence_after();
            const uint32_t b_addr = tc::smem_addr(stages + (size_t)st * kChunkBytes);
#pragma unroll
            for (int j = 0; j < kPairChunkK / 16; j++) {
              const int k0 = kc * kPairChunkK + 16 * j;  // A: 64-wide 128-byte-swizzled blocks
              tc::mma_bf16(acc, tc::smem_desc_sw128(a_addr + (uint32_t)(k0 >> 6) * (kAggRows * 128) + (k0 & 63) * 2),
                           tc::smem_desc_sw64(b_addr + 32u * j), idesc, (kc > 0 || j > 0) ? 1u : 0u);
            }
            tc::mma_commit(&bar.empty[st]);
          }
          if (ok && L == 2)  // block3.0's extra inputs: E (K 16, written before block 3's arrival) times W3b
            tc::mma_bf16(acc, tc::smem_desc_plain(tc::smem_addr(E), 128u, 256u),
                         tc::smem_desc_plain(tc::smem_addr(W3b), 128u, 256u), idesc, 1u);
          if (L > 0) a1_ph++;
          tc::mma_commit(&bar.acc_full[L & 1]);
        }
      }
      if (!ok) fail = true;
      tc::mma_commit(&bar.idle);
      if (!tc::mbar_wait(&bar.idle, 0)) fail = true;
    }
    __syncwarp();
  } else {
    // ---- math warps: inputs, epilogues, reductions
    const int er = 32 * (warp & 3) + lane, cq = warp >> 2;  // cq: also the column group of the epilogues
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    auto nothing = [] {};
    unsigned acc_ph[2] = {0, 0};
    int stop = 0, slot = 0;
    if (my_tiles > 0) {
      build_inputs(g, blockIdx.x, spt, A0, sc.wgt[0], tid);
      tc::fence_async_smem();
      tc::mbar_arrive(&bar.a0_ready);
    }
    for (long long t = blockIdx.x; t < n_tiles && !stop; t += gridDim.x, slot ^= 1) {
      // layer 1 -> A1
      if (!wait_or_abort(&bar.acc_full[0], (acc_ph[0]++) & 1, abort, g.wait_ns)) fail = true;
      tc::tc_fence_after();
      epilogue_hidden(lane_addr, nullptr, A1, er, cq, bar.a1_blk, nothing);  // bias: A0 column 284
      // layer 2 -> A1, and block3's extra inputs -> E
      if (!wait_or_abort(&bar.acc_full[1], (acc_ph[1]++) & 1, abort, g.wait_ns)) fail = true;
      tc::tc_fence_after();
      epilogue_hidden(lane_addr + 256u, prm + kPB2, A1, er, cq, bar.a1_blk, [&] {
      if (cq == 3) {
        const long long m = t * spt + er / P;
        const long long e = m * P + er % P;
        float ex[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (er < spt * P && m < g.M) {
          float dot = 0.0f;
#pragma unroll
          for (int i = 0; i < 3; i++) {
            const float dv = __ldg(g.pc_dir + e * 3 + i), rd = __ldg(g.rays_d + m * 3 + i);
            ex[i] = __ldg(g.pc_rgb + e * 3 + i);
            ex[3 + i] = __fsub_rn(dv, rd);
            dot = i == 0 ? __fmul_rn(dv, rd) : __fmaf_rn(dv, rd, dot);
          }
          ex[6] = dot;
          ex[7] = 1.0f;  // its W3b column holds block3.0's bias
        }
        *reinterpret_cast<uint4*>(E + tc::plain16_offset(er, 0)) = pack8(ex);
        *reinterpret_cast<uint4*>(E + tc::plain16_offset(er, 8)) = make_uint4(0, 0, 0, 0);
      }
      });
      // layer 3 -> A1
      if (!wait_or_abort(&bar.acc_full[0], (acc_ph[0]++) & 1, abort, g.wait_ns)) fail = true;
      tc::tc_fence_after();
      epilogue_hidden(lane_addr, nullptr, A1, er, cq, bar.a1_blk, nothing);  // bias: E column 7
      // the next tile's inputs (A0's reader, this tile's layer 1, has completed) while layer 4 runs
      if (t + gridDim.x < n_tiles) {
        build_inputs(g, t + gridDim.x, spt, A0, sc.wgt[slot ^ 1], tid);
        tc::fence_async_smem();
        tc::mbar_arrive(&bar.a0_ready);
      }
      // layer 4: alpha-branch dot product per row, and the weighted sum over each sample's
      // rows: the warp's 32 rows x 32 columns go through a transpose buffer (in A1, whose
      // last reader, layer 4, has completed), lane l sums column l of each sample in place,
      // and the sums are written to the colour-input rows 8 columns at a time.
      if (!wait_or_abort(&bar.acc_full[1], (acc_ph[1]++) & 1, abort, g.wait_ns)) fail = true;
      tc::tc_fence_after();
      {
        const float w = sc.wgt[slot][er];
        const float* wa = prm + kPWA;
        const float* bias = prm + kPB4;
        float* red = reinterpret_cast<float*>(A1) + warp * (32 * kRed);
        const long long m0 = (t * kAggRows + 32 * (warp & 3)) / P;  // the warp's first sample
        float adot = 0.0f;
#pragma unroll 1
        for (int cc = 0; cc < 2; cc++) {
          const int col0 = 64 * cq + 32 * cc;
          float v[32];
          tc::tmem_ld32(lane_addr + 256u + (uint32_t)col0, v);
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const float4 b = __ldg(reinterpret_cast<const float4*>(bias + col0) + q);
            const float4 a = __ldg(reinterpret_cast<const float4*>(wa + col0) + q);
            const float bb[4] = {b.x, b.y, b.z, b.w}, aa[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const float f = leaky(__fadd_rn(v[4 * q + i], bb[i]));
              adot = __fmaf_rn(f, aa[i], adot);
              red[lane * kRed + ((4 * q + i) ^ lane)] = __fmul_rn(f, w);
            }
          }
          __syncwarp();
          switch (P) {
            case 1: sample_sums<1>(red, lane, m0, g.M, g.color_in, col0); break;
            case 2: sample_sums<2>(red, lane, m0, g.M, g.color_in, col0); break;
            case 4: sample_sums<4>(red, lane, m0, g.M, g.color_in, col0); break;
            case 8: sample_sums<8>(red, lane, m0, g.M, g.color_in, col0); break;
            case 16: sample_sums<16>(red, lane, m0, g.M, g.color_in, col0); break;
            default: sample_sums<32>(red, lane, m0, g.M, g.color_in, col0); break;
          }
          __syncwarp();
        }
        sc.apart[cq][er] = adot;
        const long long m = t * spt + er / P;
        if (cq == 3 && er % P == 0 && er < spt * P && m < g.M) {  // PE(ray_d, 4) -> columns 256..279, zeros to 319
          uint8_t* crow = g.color_in + (size_t)(m / kAggRows) * kATileBytes;
          const int cr = (int)(m % kAggRows);
          float s4[3][4], c4[3][4];
#pragma unroll
          for (int i = 0; i < 3; i++) bands<4>(__ldg(g.rays_d + m * 3 + i), s4[i], c4[i]);
#pragma unroll
          for (int u = 0; u < 3; u++) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int a = 4 * u + i;
              v[2 * i] = s4[a / 4][a % 4];
              v[2 * i + 1] = c4[a / 4][a % 4];
            }
            store_unit(crow, cr, 32 + u, v);
          }
#pragma unroll
          for (int u = 35; u < 40; u++) zero_unit(crow, cr, u);
        }
      }
      tc::tc_fence_before();
      stop = tc::named_sync_or(fail || *abort, kMathThreads);
      if (stop) break;
      // alpha: softplus(branch - 1) of each valid row, weighted sum over the sample
      if (tid < kAggRows) {
        const int r = tid;
        const long long m = t * spt + r / P;
        const int p = r % P;
        const bool in = r < spt * P && m < g.M;
        float a = 0.0f;
        if (in && __ldg(g.valid + m * P + p)) {
          const float z = __fadd_rn(__fadd_rn(__fadd_rn(sc.apart[0][r], sc.apart[1][r]),
                                              __fadd_rn(sc.apart[2][r], sc.apart[3][r])), prm[kPBA]);
          a = softplus(__fsub_rn(z, 1.0f));
        }
        float x = __fmul_rn(a, sc.wgt[slot][r]);
        for (int o = 1; o < P; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (in && p == 0) g.alpha[m] = x;
      }
      stop = tc::named_sync_or(fail || *abort, kMathThreads);  // apart and A1 are rewritten next tile
    }
  }

  if (fail) atomicExch(g.status, 1);
  if (tid == 0 && bar.abort) atomicExch(g.status, 1);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------
// colour branch
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kColorThreads, 1) k_agg_color(AggArgs g, long long n_tiles) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  uint8_t* A = smem;
  uint8_t* stages = smem + kCStages;
  Ring& ring = *reinterpret_cast<Ring*>(smem + kCBar);
  ColorScratch& sc = *reinterpret_cast<ColorScratch*>(smem + kCScratch);
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
  ChunkStream cs{g.packed + kColorOff, kColorChunks, kChunkBytes, 0, 0, my_tiles * kColorChunks};
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
          tc::mbar_arrive_expect_tx(&ring.aload, kATileBytes);
          tc::bulk_load(A, g.color_in + (size_t)t * kATileBytes, kATileBytes, &ring.aload);
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
          for (int q = 0; q < 4; q++) store_unit(A, er, col0 / 8 + q, v + 8 * q);
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

// element e of the colour chunk stream -> (chunk, n, k within the chunk); a chunk is
// 128 rows x 64 K, 128-byte swizzled (tc::operand_offset with one K block)
__device__ __forceinline__ void chunk_coords(long long e, int& chunk, int& n, int& k) {
  const int per = kChunkN * kChunkK;
  chunk = (int)(e / per);
  const int o = (int)(e % per) * 2;  // byte offset in the chunk
  n = o >> 7;
  const int c = ((o >> 4) & 7) ^ (n & 7);
  k = c * 8 + ((o & 15) >> 1);
}

__global__ void k_agg_pack(PackArgs a, uint8_t* __restrict__ packed) {
  const long long n_pair = (long long)kPairBytes / 2, n_w3b = kW3bBytes / 2, n_color = (long long)kColorBytes / 2;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  __nv_bfloat16* out = reinterpret_cast<__nv_bfloat16*>(packed);
  if (e < n_pair) {  // pair chunk: 256 rows x 32 K, 64-byte swizzled (tc::sw64_offset)
    const int chunk = (int)(e / (kPairN * kPairChunkK));
    const int o = (int)(e % (kPairN * kPairChunkK)) * 2;
    const int row = o >> 6, k = ((((o >> 4) & 3) ^ ((row >> 1) & 3)) << 3) + ((o & 15) >> 1);
    int L = 0, c0 = 0;
    while (chunk >= c0 + pair_k(L) / kPairChunkK) c0 += pair_k(L++) / kPairChunkK;
    const int col = (chunk - c0) * kPairChunkK + k;
    const int streamed = L == 2 ? 256 : pair_real_k(L);  // block3.0's columns 256.. go to W3b
    float w = col < streamed ? a.w[L][(size_t)row * pair_real_k(L) + col] : 0.0f;
    if (L == 0 && col == 284) w = a.b[0][row];  // block1.0's bias, against the constant input column
    out[e] = __float2bfloat16_rn(w);
  } else if (e < n_pair + n_w3b) {
    const int o = (int)(e - n_pair) * 2;  // W3b: 256 rows x 16 K, no swizzle (tc::plain16_offset)
    const int row = (o / 256) * 8 + (o % 128) / 16, col = ((o % 256) / 128) * 8 + (o % 16) / 2;
    out[e] = __float2bfloat16_rn(col < 7 ? a.w[2][(size_t)row * 263 + 256 + col] : col == 7 ? a.b[2][row] : 0.0f);
  } else if (e < n_pair + n_w3b + n_color) {
    int chunk, n, k;
    chunk_coords(e - n_pair - n_w3b, chunk, n, k);
    int L = 0, c0 = 0;
    while (chunk >= c0 + color_k(L) / kChunkK) c0 += color_k(L++) / kChunkK;
    const int col = (chunk - c0) * kChunkK + k;
    out[e] = __float2bfloat16_rn(col < color_real_k(L) ? a.w[5 + L][(size_t)n * color_real_k(L) + col] : 0.0f);
  } else if (e < n_pair + n_w3b + n_color + kParams) {
    const int q = (int)(e - n_pair - n_w3b - n_color);
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

// The two tensor-core kernels exceed the 48 KB default of dynamic shared
// memory: opt them in once per device, and note the device's SM count.
static int32_t agg_setup(unsigned pair_smem, unsigned color_smem, int* sms) {
  static std::mutex mu;
  static int sm_counts[128] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return set_error(HP_ERR_CUDA, "hp_aggregator_forward: cudaGetDevice failed");
  std::lock_guard<std::mutex> lock(mu);
  if (!sm_counts[dev]) {
    int n = 0;
    cudaError_t e = cudaFuncSetAttribute(k_agg_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_agg_color, cudaFuncAttributeMaxDynamicSharedMemorySize, color_smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || n <= 0)
      return set_error(HP_ERR_CUDA, "hp_aggregator_forward: kernel set-up: %s", cudaGetErrorString(e));
    sm_counts[dev] = n;
  }
  *sms = sm_counts[dev];
  return HP_OK;
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
  o += align256((size_t)(tiles > 0 ? tiles : 1) * kATileBytes);
  L.alpha = o;
  o += align256(sizeof(float) * (size_t)(M > 0 ? M : 1));
  L.color = o;
  o += align256(sizeof(float) * 3 * (size_t)(M > 0 ? M : 1));
  L.status = o;
  o += 256;
  L.total = o;
  return L;
}

constexpr unsigned kPairSmem = kPScratch + sizeof(PairScratch) + 1024;
constexpr unsigned kColorSmem = kCScratch + sizeof(ColorScratch) + 1024;
static_assert(sizeof(PairBars) <= 256 && sizeof(Ring) <= 256, "barrier block");
static_assert(kPairSmem <= 227 * 1024 && kColorSmem <= 227 * 1024, "shared memory");
static_assert(kMathThreads / 32 * 32 * kRed * 4 <= kA1Bytes, "transpose buffers fit in A1");
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
  const long long n = (long long)(kPairBytes + kW3bBytes + kColorBytes) / 2 + kParams;
  k_agg_pack<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, (uint8_t*)packed);
  return check_launch("k_agg_pack");
}

extern "C" size_t hp_aggregator_workspace_size(int64_t n_samples) {
  if (n_samples < 0) return 0;
  return agg_layout(n_samples).total;
}

static int32_t agg_forward(const void* packed, const float* pc_xyz, const float* pc_rgb, const float* pc_dir,
                           const float* pc_feat, int32_t feat_dim, const float* sp_xyz, const uint8_t* valid,
                           const float* rays_d, int64_t n_samples, int32_t P, const uint8_t* mask_out,
                           const int32_t* mask_offsets, int64_t n_positions, float* alpha_out, float* color_out,
                           void* workspace, size_t workspace_bytes, hp_stream_t stream, unsigned long long wait_ns,
                           int withhold_w3b) {
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
  g.wait_ns = wait_ns;
  g.withhold_w3b = withhold_w3b;
  if (cudaMemsetAsync(g.status, 0, sizeof(int), st) != cudaSuccess)
    return set_error(HP_ERR_CUDA, "%s: memset failed", who);
  if (n_samples > 0) {
    int sms = 0;
    if (int32_t rc = agg_setup(kPairSmem, kColorSmem, &sms)) return rc;
    const int spt = kAggRows / P;
    const long long pair_tiles = (n_samples + spt - 1) / spt;
    const long long color_tiles = (n_samples + kAggRows - 1) / kAggRows;
    const unsigned pg = (unsigned)(pair_tiles < sms ? pair_tiles : sms);
    const unsigned cg = (unsigned)(color_tiles < sms ? color_tiles : sms);
    k_agg_pairs<<<pg, kPairThreads, kPairSmem, st>>>(g, pair_tiles);
    if (int32_t rc = check_launch("k_agg_pairs")) return rc;
    k_agg_color<<<cg, kColorThreads, kColorSmem, st>>>(g, color_tiles);
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

extern "C" int32_t hp_aggregator_forward(const void* packed, const float* pc_xyz, const float* pc_rgb,
                                         const float* pc_dir, const float* pc_feat, int32_t feat_dim,
                                         const float* sp_xyz, const uint8_t* valid, const float* rays_d,
                                         int64_t n_samples, int32_t P, const uint8_t* mask_out,
                                         const int32_t* mask_offsets, int64_t n_positions, float* alpha_out,
                                         float* color_out, void* workspace, size_t workspace_bytes,
                                         hp_stream_t stream) {
  return agg_forward(packed, pc_xyz, pc_rgb, pc_dir, pc_feat, feat_dim, sp_xyz, valid, rays_d, n_samples, P, mask_out,
                     mask_offsets, n_positions, alpha_out, color_out, workspace, workspace_bytes, stream, tc::kWaitNs,
                     0);
}

#ifdef HP_TESTING
// Test library only (include/hashpoint_b200_testing.h): the forward with the
// pair kernel's W3b block never loaded, so the tensor-core warp's bounded wait
// for it gives up after wait_limit_us, every other role's wait ends at once,
// the kernels return and hp_aggregator_status reports the failure.
extern "C" int32_t hp_aggregator_forward_withheld(const void* packed, const float* pc_xyz, const float* pc_rgb,
                                                  const float* pc_dir, const float* pc_feat, int32_t feat_dim,
                                                  const float* sp_xyz, const uint8_t* valid, const float* rays_d,
                                                  int64_t n_samples, int32_t P, const uint8_t* mask_out,
                                                  const int32_t* mask_offsets, int64_t n_positions, float* alpha_out,
                                                  float* color_out, void* workspace, size_t workspace_bytes,
                                                  int32_t wait_limit_us, hp_stream_t stream) {
  if (wait_limit_us <= 0)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_aggregator_forward_withheld: wait_limit_us must be > 0");
  return agg_forward(packed, pc_xyz, pc_rgb, pc_dir, pc_feat, feat_dim, sp_xyz, valid, rays_d, n_samples, P, mask_out,
                     mask_offsets, n_positions, alpha_out, color_out, workspace, workspace_bytes, stream,
                     1000ull * (unsigned long long)wait_limit_us, 1);
}
#endif

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
