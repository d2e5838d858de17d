// gf_wait_selftest.cu -- diagnostic entry point for the bounded device waits.
//
// The library's kernels never wait without a limit: the decoupled lookback of
// the cumulative-weight scan polls a predecessor's flag at most kSpinLimit
// times, and the tensor-core propagate polls its MMA-completion mbarrier at
// most TC_WAIT times; each sets GF_ERR_TIMEOUT in the job status when the
// limit runs out.  This entry point runs the same wait routines against a flag
// that is either published beforehand or never set, with a caller-chosen
// (short) limit, so a test can watch the timeout path return an error status
// while the context stays usable.  Not part of the filtering API
// (gf_b200_diag.h).
#include <cuda_runtime.h>

#include "gf_pf_kernels.cuh"
#include "gf_umma.cuh"

namespace gf {

// Tile 1 of a two-tile lookback: tile 0's inclusive prefix is `pred` when
// `publish` is set, otherwise nothing ever writes it.
__global__ void wait_lookback_kernel(unsigned long long* flags, int publish,
                                     unsigned long long pred, long long limit,
                                     unsigned long long* excl_out, int* status) {
  unsigned long long* fagg = flags;
  unsigned long long* finc = flags + 2;
  if (publish && threadIdx.x == 0) atomicExch(finc, kReady | pred);
  __syncwarp();
  bool fail = false;
  const unsigned long long excl = lookback_exclusive(fagg, finc, 1, 7ull, limit, &fail);
  if (threadIdx.x == 0) {
    *status = fail ? GF_ERR_TIMEOUT : GF_OK;
    *excl_out = excl;
  }
}

// An mbarrier expecting one arrival, which thread 0 gives when `publish` is
// set; every thread then waits on phase 0 with at most `limit` polls.
__global__ void wait_mbarrier_kernel(int publish, uint32_t limit, int* status) {
  __shared__ uint64_t mbar;
  if (threadIdx.x == 0) {
    umma::mbar_init(&mbar, 1);
    umma::fence_mbar_init();
  }
  __syncthreads();
  if (publish && threadIdx.x == 0) {
    uint64_t token;
    asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];"
                 : "=l"(token)
                 : "r"(umma::smem_u32(&mbar))
                 : "memory");
    (void)token;
  }
  const bool ok = umma::mbar_wait(&mbar, 0u, limit);
  const unsigned all_ok = __syncthreads_and(ok ? 1 : 0);
  if (threadIdx.x == 0) *status = all_ok ? GF_OK : GF_ERR_TIMEOUT;
}

}  // namespace gf

extern "C" int gfx_wait_selftest(int which, int publish, long long limit, int* status_out,
                                 unsigned long long* excl_out) {
  if (!status_out || limit < 1 || (which != 0 && which != 1)) return GF_ERR_ARG;
  unsigned long long* dflags = nullptr;
  int* dst = nullptr;
  if (cudaMalloc(&dflags, 5 * sizeof(unsigned long long)) != cudaSuccess) return GF_ERR_CUDA;
  if (cudaMalloc(&dst, sizeof(int)) != cudaSuccess) {
    cudaFree(dflags);
    return GF_ERR_CUDA;
  }
  cudaMemset(dflags, 0, 5 * sizeof(unsigned long long));
  cudaMemset(dst, 0xff, sizeof(int));
  if (which == 0) {
    gf::wait_lookback_kernel<<<1, 32>>>(dflags, publish, 5ull, limit, dflags + 4, dst);
  } else {
    const uint32_t lim = limit > 0xFFFFFFFFll ? 0xFFFFFFFFu : (uint32_t)limit;
    gf::wait_mbarrier_kernel<<<1, 128>>>(publish, lim, dst);
  }
  cudaError_t e = cudaDeviceSynchronize();
  int st = -1;
  unsigned long long ex = 0ull;
  if (e == cudaSuccess) e = cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&ex, dflags + 4, sizeof ex, cudaMemcpyDeviceToHost);
  cudaFree(dflags);
  cudaFree(dst);
  if (e != cudaSuccess) return GF_ERR_CUDA;
  *status_out = st;
  if (excl_out) *excl_out = ex;
  return GF_OK;
}
