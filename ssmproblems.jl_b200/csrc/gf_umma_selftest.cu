// gf_umma_selftest.cu -- diagnostic entry point: D = A * B^T on the tensor
// cores (tcgen05 kind::tf32, 1x or 3x split precision) for one 128-row tile,
// so tests can check the operand layout, descriptors and TMEM read-back
// against a host matmul.  Not part of the filtering API (gf_b200_diag.h).
#include <cuda_runtime.h>

#include <vector>

#include "gf_umma.cuh"

namespace gf {

__global__ void __launch_bounds__(128) umma_selftest_kernel(const float* __restrict__ A,
                                                          const float* __restrict__ B, float* D,
                                                          int N, int K, int split3, int* status) {
  extern __shared__ __align__(128) unsigned char smem[];
  float* sAh = reinterpret_cast<float*>(smem);
  float* sAl = sAh + 128 * K;
  float* sBh = sAl + 128 * K;
  float* sBl = sBh + N * K;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int r = threadIdx.x;
  for (int k = 0; k < K; ++k) {
    const float v = A[r * K + k];
    const float h = umma::to_tf32(v);
    const uint32_t off = umma::kmajor_offset(r, k, K) / 4;
    sAh[off] = h;
    sAl[off] = umma::to_tf32(v - h);
  }
  for (int n = r; n < N; n += 128)
    for (int k = 0; k < K; ++k) {
      const float v = B[n * K + k];
      const float h = umma::to_tf32(v);
      const uint32_t off = umma::kmajor_offset(n, k, K) / 4;
      sBh[off] = h;
      sBl[off] = umma::to_tf32(v - h);
    }
  if (r == 0) {
    umma::mbar_init(&mbar, 1);
    umma::fence_mbar_init();
  }
  umma::fence_async_smem();
  __syncthreads();
  const uint32_t ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  if (r < 32) umma::tmem_alloc(&tmem_base, ncols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (r == 0) {
    const uint32_t kstride = 128, mstride = (uint32_t)(K / 4) * 128;
    const uint32_t idesc = umma::idesc_tf32(128, N);
    for (int s = 0; s < K / 8; ++s) {
      const uint32_t koff = (uint32_t)s * 2 * kstride;
      const uint64_t ah = umma::desc(umma::smem_u32(sAh) + koff, kstride, mstride);
      const uint64_t al = umma::desc(umma::smem_u32(sAl) + koff, kstride, mstride);
      const uint64_t bh = umma::desc(umma::smem_u32(sBh) + koff, kstride, mstride);
      const uint64_t bl = umma::desc(umma::smem_u32(sBl) + koff, kstride, mstride);
      umma::mma_tf32(tbase, ah, bh, idesc, s > 0 ? 1u : 0u);
      if (split3) {
        umma::mma_tf32(tbase, ah, bl, idesc, 1u);
        umma::mma_tf32(tbase, al, bh, idesc, 1u);
      }
    }
    umma::mma_commit(&mbar);
  }
  const bool ok = umma::mbar_wait(&mbar, 0, 1u << 20);
  if (!ok && r == 0) atomicExch(status, 4);
  umma::fence_after_sync();
  if (ok) {
    const int w = r >> 5;
    for (int c = 0; c < N; c += 16) {
      float v[16];
      umma::tmem_ld16(tbase + ((uint32_t)(32 * w) << 16) + (uint32_t)c, v);
      umma::tmem_wait_ld();
      for (int j = 0; j < 16 && c + j < N; ++j) D[r * N + c + j] = v[j];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (r < 32) umma::tmem_dealloc(tbase, ncols);
}

}  // namespace gf

// Host wrapper: A [128 x K], B [N x K] row-major FP32 host arrays, D [128 x N].
// K a multiple of 8, N a multiple of 16 in [16, 256].  Returns 0 on success.
extern "C" int gfx_umma_selftest(const float* A, const float* B, float* D, int N, int K,
                                 int split3) {
  if (K % 8 || N % 16 || N < 16 || N > 256 || K > 256) return 6;
  float *dA, *dB, *dD;
  int* dst;
  size_t smem = sizeof(float) * (2 * 128 * K + 2 * N * K);
  if (smem > 200 * 1024) return 6;
  if (cudaMalloc(&dA, sizeof(float) * 128 * K) || cudaMalloc(&dB, sizeof(float) * N * K) ||
      cudaMalloc(&dD, sizeof(float) * 128 * N) || cudaMalloc(&dst, sizeof(int)))
    return 5;
  cudaMemcpy(dA, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice);
  cudaMemset(dD, 0, sizeof(float) * 128 * N);
  cudaMemset(dst, 0, sizeof(int));
  cudaFuncSetAttribute(gf::umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  gf::umma_selftest_kernel<<<1, 128, smem>>>(dA, dB, dD, N, K, split3, dst);
  cudaError_t e = cudaDeviceSynchronize();
  int st = 0;
  cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost);
  cudaMemcpy(D, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(dst);
  if (e != cudaSuccess) return 5;
  return st;
}
