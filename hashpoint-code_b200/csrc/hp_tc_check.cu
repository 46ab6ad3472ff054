// Self-check of the tensor-core operand forms of hp_tc.cuh (test library
// only, include/hashpoint_b200_testing.h): one tcgen05.mma,
// D [128, 256] fp32 = A [128 x 16] * B [256 x 16]^T (bf16), from operand
// images the caller laid out as shared memory, with the descriptor of each
// operand starting at a chosen byte offset into its image.  The tests compare
// D with a host product for each form the Aggregator's kernels use.
#include "../../include/hashpoint_b200_testing.h"
#include "hp_common.cuh"
#include "hp_tc.cuh"

namespace hp {

constexpr int kCheckM = 128, kCheckN = 256;
constexpr unsigned kCheckABytes = 81920;  // the Aggregator's largest A operand (128 rows x 320 K)
constexpr unsigned kCheckBBytes = 32768;  // 256 rows x 64 K

__device__ __forceinline__ uint64_t check_desc(int form, uint32_t addr) {
  if (form == HP_TC_PLAIN) return tc::smem_desc_plain(addr, 128u, 256u);
  if (form == HP_TC_SW128) return tc::smem_desc_sw128(addr);
  return tc::smem_desc_sw64(addr);
}

__global__ void __launch_bounds__(128, 1) k_tc_check(const uint4* __restrict__ a, const uint4* __restrict__ b,
                                                     int a_form, uint32_t a_off, int b_form, uint32_t b_off,
                                                     float* __restrict__ d, int* __restrict__ status) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t done;
  __shared__ uint32_t tmem_base;
  const uint32_t raw = tc::smem_addr(smem_raw);
  uint8_t* A = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* B = A + kCheckABytes;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (unsigned i = tid; i < kCheckABytes / 16; i += blockDim.x) reinterpret_cast<uint4*>(A)[i] = a[i];
  for (unsigned i = tid; i < kCheckBBytes / 16; i += blockDim.x) reinterpret_cast<uint4*>(B)[i] = b[i];
  tc::fence_async_smem();
  if (tid == 0) {
    tc::mbar_init(&done, 1);
    tc::mbar_init_fence();
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base, kCheckN);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    tc::mma_bf16(tmem, check_desc(a_form, tc::smem_addr(A) + a_off), check_desc(b_form, tc::smem_addr(B) + b_off),
                 tc::idesc_bf16(kCheckM, kCheckN), 0u);
    tc::mma_commit(&done);
  }
  __syncwarp();
  const bool ok = tc::mbar_wait(&done, 0);
  tc::tc_fence_after();
  if (__syncthreads_and(ok)) {
    const int row = 32 * warp + lane;
    for (int c = 0; c < kCheckN; c += 32) {
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, v);
#pragma unroll
      for (int j = 0; j < 32; j++) d[(size_t)row * kCheckN + c + j] = v[j];
    }
  } else if (tid == 0) {
    *status = 1;
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, kCheckN);
  }
}

// Whether a K = 16 window of `rows` rows starting `off` bytes into an image
// stays inside it: 8-row groups of 256 bytes for the no-swizzle form; for the
// swizzled forms the start lies in the first row of an 8-row atom (the K step
// inside a row, as the kernels use it) and the rows are 128 / 64 bytes.
static bool check_window(int form, uint32_t off, unsigned rows, unsigned image) {
  if (off % 16) return false;
  if (form == HP_TC_PLAIN) return off + rows * 32 <= image;
  const unsigned row_bytes = form == HP_TC_SW128 ? 128 : 64, atom = 8 * row_bytes;
  if ((off % atom) + 32 > row_bytes) return false;
  return (off / atom) * atom + rows * row_bytes <= image;
}

}  // namespace hp

using namespace hp;

HP_API size_t hp_tc_check_image_bytes(int32_t operand) { return operand == 0 ? kCheckABytes : kCheckBBytes; }

HP_API int32_t hp_tc_check_mma(const void* a_image, const void* b_image, int32_t a_form, uint32_t a_offset,
                               int32_t b_form, uint32_t b_offset, float* d, hp_stream_t stream) {
  const auto form_ok = [](int32_t f) { return f == HP_TC_PLAIN || f == HP_TC_SW128 || f == HP_TC_SW64; };
  if (!a_image || !b_image || !d) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_tc_check_mma: null pointer");
  if ((reinterpret_cast<uintptr_t>(a_image) | reinterpret_cast<uintptr_t>(b_image)) & 15)
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_tc_check_mma: images must be 16-byte aligned");
  if (!form_ok(a_form) || !form_ok(b_form)) return set_error(HP_ERR_INVALID_ARGUMENT, "hp_tc_check_mma: form");
  if (!check_window(a_form, a_offset, kCheckM, kCheckABytes) || !check_window(b_form, b_offset, kCheckN, kCheckBBytes))
    return set_error(HP_ERR_INVALID_ARGUMENT, "hp_tc_check_mma: offset outside the image or its row");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned smem = kCheckABytes + kCheckBBytes + 1024;
  int* status = nullptr;
  cudaError_t e = cudaFuncSetAttribute(k_tc_check, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) e = cudaMallocAsync(&status, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    k_tc_check<<<1, 128, smem, s>>>(static_cast<const uint4*>(a_image), static_cast<const uint4*>(b_image), a_form,
                                    a_offset, b_form, b_offset, d, status);
    e = cudaGetLastError();
  }
  int flag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (status) cudaFreeAsync(status, s);
  if (e != cudaSuccess) return set_error(HP_ERR_CUDA, "hp_tc_check_mma: %s", cudaGetErrorString(e));
  if (flag) return set_error(HP_ERR_CUDA, "hp_tc_check_mma: the MMA did not complete");
  return HP_OK;
}
