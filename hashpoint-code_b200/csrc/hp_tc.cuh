// Blackwell (sm_100a) tensor-core plumbing written as inline PTX: mbarriers,
// bulk global->shared copies, TMEM allocation, tcgen05.mma (bf16 x bf16 ->
// fp32 in TMEM) and tcgen05.ld.
//
// Operand layout.  Every shared-memory operand is stored K-major with the
// 128-byte swizzle of tcgen05: K is cut into blocks of 64 bf16 (one 128-byte
// row per matrix row), a block of R rows is R * 128 contiguous bytes (8-row
// atoms of 1024 bytes, SBO = 1024), and inside a row the eight 16-byte chunks
// are permuted by chunk ^ (row % 8).  So element (r, k) of an operand with R
// rows sits at
//   (k / 64) * (R * 128) + r * 128 + (((k / 8) % 8) ^ (r % 8)) * 16 + (k % 8) * 2.
// Blocks start 1024-byte aligned.  One MMA consumes 16 K; within a block the
// next K step starts 32 bytes further on (the swizzle is applied to the
// address bits, so the descriptor's start address simply advances).
//
// Waits are bounded: every mbarrier wait gives up after kWaitNs of
// %globaltimer and reports failure, so a kernel whose copies or MMAs never
// complete returns an error status instead of hanging.
#pragma once

#include <stdint.h>

namespace hp {
namespace tc {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// --- mbarrier ---------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Wait until the phase of the given parity has completed; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}

// --- bulk copy (no tensor map; the issuing CTA is the only destination) -------
// bytes: a multiple of 16; both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst_smem)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Generic-proxy shared-memory writes -> visible to the async proxy (tcgen05.mma).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// --- TMEM --------------------------------------------------------------------
// One full warp; the column base is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// --- descriptors -------------------------------------------------------------
// Shared-memory matrix descriptor of a K-major 128-byte-swizzled operand:
// start address >> 4 (bits 0-13), LBO 16 bytes (unused inside one swizzle
// row; bits 16-29), SBO 1024 bytes between 8-row atoms (bits 32-45), version
// 1 (bits 46-47), base offset 0, layout SWIZZLE_128B = 2 (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  const uint64_t lo = (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)1 << 16);
  const uint64_t hi = (uint64_t)(1024u >> 4) | (1ull << 14) | (2ull << 29);
  return lo | (hi << 32);
}

// Descriptor of a K-major operand in the canonical no-swizzle layout (8x8
// core matrices of 128 contiguous bytes): lbo = bytes between K-adjacent core
// matrices, sbo = bytes between 8-row groups; layout type 0.
__device__ __forceinline__ uint64_t smem_desc_plain(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  const uint64_t lo = (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16);
  const uint64_t hi = (uint64_t)((sbo >> 4) & 0x3fffu) | (1ull << 14);
  return lo | (hi << 32);
}

// Descriptor of a K-major 64-byte-swizzled operand: rows of 32 bf16 (64
// bytes), 8-row atoms of 512 bytes (SBO), the 16-byte chunks of a row permuted
// by chunk ^ ((row / 2) % 4); layout SWIZZLE_64B = 4 (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t addr) {
  const uint64_t lo = (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)1 << 16);
  const uint64_t hi = (uint64_t)(512u >> 4) | (1ull << 14) | (4ull << 29);
  return lo | (hi << 32);
}

// Instruction descriptor of kind::f16: D fp32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, M x N x 16; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

// Arrive on bar when every tcgen05 operation this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// 32 consecutive fp32 columns of this thread's TMEM lane (the warp reads lanes
// 32 * (warp % 4) .. + 31); taddr = base + (lane0 << 16) + column.  The wait
// for the load is in the same asm statement: as a statement of its own it
// would name none of the destination registers, and the compiler could move
// arithmetic on them above it, onto registers the load has not yet written.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (n, k), k < 32, in a K-major 64-byte-swizzled block.
__host__ __device__ __forceinline__ uint32_t sw64_offset(int n, int k) {
  return (uint32_t)(n * 64 + ((((k >> 3) & 3) ^ ((n >> 1) & 3)) << 4) + (k & 7) * 2);
}

// Byte offset of element (r, k) of a 16-wide K-major operand in the no-swizzle
// layout (lbo 128, sbo 256).
__host__ __device__ __forceinline__ uint32_t plain16_offset(int r, int k) {
  return (uint32_t)((r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Barrier 1 over the first n threads of the block (warps 0 .. n/32 - 1), with
// an OR of pred over them returned to all.
__device__ __forceinline__ int named_sync_or(int pred, int n) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(pred), "r"(n)
      : "memory");
  return r;
}

// Byte offset of element (r, k) in a K-major 128-byte-swizzled operand of R rows.
__host__ __device__ __forceinline__ uint32_t operand_offset(int r, int k, int R) {
  return (uint32_t)((k >> 6) * (R * 128) + r * 128 + ((((k >> 3) & 7) ^ (r & 7)) << 4) + (k & 7) * 2);
}

}  // namespace tc
}  // namespace hp
