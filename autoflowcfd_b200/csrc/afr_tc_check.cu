// Tensor-core self-check: one CTA computes D[128 x n] = A[128 x k] * B[n x k]^T
// with tcgen05.mma (BF16 in, FP32 accumulate in tensor memory) through the
// same shared-memory layout, descriptors and waits that the mixed-precision
// kernels use.  Diagnostic entry point; no counterpart in the reference.
#include <cuda_runtime.h>
#include <cstdint>

#include "afr_tc.cuh"
#include "../../include/afr_b200.h"

namespace afr {
namespace {

__device__ unsigned g_tc_check_status;

__global__ void __launch_bounds__(128, 1) k_tc_check(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                     float* __restrict__ D, int n, int kd, uint32_t ncols) {
  extern __shared__ __align__(1024) uint16_t sm_tc[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int done;
  uint16_t* sA = sm_tc;            // 128 x kd, K-major canonical
  uint16_t* sB = sm_tc + 128 * kd; // n x kd
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int t = tid; t < 128 * kd; t += blockDim.x) sA[tc::kmajor_index(t / kd, t % kd, 128)] = A[t];
  for (int t = tid; t < n * kd; t += blockDim.x) sB[tc::kmajor_index(t / kd, t % kd, n)] = B[t];
  if (warp == 0) tc::tmem_alloc(&tbase, ncols);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    const uint32_t idesc = tc::idesc_bf16(128, n);
    const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
    for (int ks = 0; ks < kd / 16; ++ks) {
      const uint64_t ad = tc::make_desc(a0 + ks * 2 * 128 * 16, 128 * 16, 128);
      const uint64_t bd = tc::make_desc(b0 + ks * 2 * n * 16, n * 16, 128);
      tc::mma_bf16(tmem, ad, bd, idesc, ks > 0 ? 1u : 0u);
    }
    tc::commit(&bar);
    const bool ok = tc::mbar_wait(&bar, 0);
    done = ok ? 1 : 0;
    if (!ok) atomicOr(&g_tc_check_status, 1u);
  }
  __syncthreads();
  tc::fence_after();
  if (done) {
    const int row = warp * 32 + lane;
    for (int c = 0; c < n; c += 8) {
      float v[8];
      tc::tmem_ld8(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c, v);
#pragma unroll
      for (int j = 0; j < 8; ++j) D[(size_t)row * n + c + j] = v[j];
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tmem, ncols);
  }
}

}  // namespace
}  // namespace afr

extern "C" int afr_tc_check(int n, int k, const void* A, const void* B, float* D, void* stream) {
  if (n < 16 || n > 256 || n % 16 || k < 16 || k > 256 || k % 16 || !A || !B || !D) return AFR_EINVAL;
  uint32_t ncols = 32;
  while (ncols < static_cast<uint32_t>(n)) ncols <<= 1;
  const size_t smem = static_cast<size_t>(128 + n) * k * sizeof(uint16_t);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaFuncSetAttribute(afr::k_tc_check, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
      cudaSuccess)
    return AFR_ECUDA;
  const unsigned zero = 0;
  if (cudaMemcpyToSymbolAsync(afr::g_tc_check_status, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return AFR_ECUDA;
  afr::k_tc_check<<<1, 128, smem, s>>>(static_cast<const uint16_t*>(A), static_cast<const uint16_t*>(B), D, n, k,
                                       ncols);
  unsigned st = 0;
  if (cudaGetLastError() != cudaSuccess) return AFR_ECUDA;
  if (cudaMemcpyFromSymbolAsync(&st, afr::g_tc_check_status, sizeof(st), 0, cudaMemcpyDeviceToHost, s) !=
      cudaSuccess)
    return AFR_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return AFR_ECUDA;
  return st ? AFR_ECUDA : AFR_OK;
}
