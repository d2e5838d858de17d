// gf_noalloc.cu -- gf_sample_ancestors_noalloc: ancestor sampling for callers
// that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at the point where they
// resample: a caller running inside a memory-pool-managed framework that
// forbids foreign allocations, a real-time loop that must not take the
// allocator's locks or trigger a device synchronisation, or code sized
// up front that must never fail with out-of-memory mid-run.  For them this
// entry point does the work of gf_sample_ancestors with all of its scratch
// (cumulative weights, lookback flags, partial sums, scalars and the job
// descriptor) in one file-scope device array of fixed size instead of
// per-call allocations.  The caller still provides the weights, uniforms and
// the ancestor output buffer.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "gf_internal.hpp"
#include "gf_pf_kernels.cuh"

namespace gf {

// Largest particle count the fixed scratch supports.
constexpr int64_t kNoAllocMaxN = int64_t(1) << 18;
constexpr int kNoAllocTiles = (int)((kNoAllocMaxN + SCAN_TILE - 1) / SCAN_TILE);
constexpr int kNoAllocParts = 256;

struct NoAllocScratch {
  double key[kNoAllocMaxN];                          // cumulative weights
  unsigned long long flags[2 * kNoAllocTiles];       // lookback flags (cleared per call)
  double part[kNoAllocParts];                        // partial weight sums
  PfScalars sc;                                      // per-call scalars (re-initialised per call)
  PfJob job;                                         // job descriptor (rewritten per call)
};

// One copy per device that loads the library, held until the process exits
// (about 2.1 MB).  Shared by every call on that device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Kernels of gf_resample.cu reused unchanged.
__global__ void sa_partial_sum(const double* __restrict__ w, int64_t n, double* __restrict__ part);
__global__ void sa_setup(const double* __restrict__ part, int nparts, PfScalars* sc,
                         const double* __restrict__ unif, int kind);
__global__ void sa_search(const PfJob* __restrict__ jobs, int64_t* __restrict__ anc);

// Writes the call's job descriptor into the scratch array: the descriptor
// travels as a kernel argument, so no host-to-device copy from pageable
// memory is needed.
__global__ void na_write_job(PfJob job, PfJob* dst) { *dst = job; }

// Device address of the scratch array, resolved once per device and cached
// for the life of the process (a cudaDeviceReset would leave it stale).
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {nullptr};

static cudaError_t noalloc_scratch(int device, NoAllocScratch** out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = p;
  }
  *out = reinterpret_cast<NoAllocScratch*>(g_noalloc_ptr[device]);
  return cudaSuccess;
}

}  // namespace gf

using namespace gf;

extern "C" int64_t gf_sample_ancestors_noalloc_max_n(void) { return kNoAllocMaxN; }

extern "C" gf_status gf_sample_ancestors_noalloc(int32_t resampler, int32_t convention, int64_t n,
                                                 const double* weights_dev,
                                                 const double* uniforms_dev,
                                                 int64_t* ancestors_dev, void* stream) {
  if (!weights_dev || !uniforms_dev || !ancestors_dev || n < 1) return GF_ERR_ARG;
  if (resampler < 0 || resampler > 2 || convention < 0 || convention > 1) return GF_ERR_ARG;
  if (n > kNoAllocMaxN) return GF_ERR_DIM;  // beyond the fixed scratch: use gf_sample_ancestors
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return GF_ERR_CUDA;
  NoAllocScratch* S = nullptr;
  if (noalloc_scratch(device, &S) != cudaSuccess) return GF_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const int nst = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
  PfJob J;
  std::memset(&J, 0, sizeof J);
  J.N = n;
  J.T = 1;
  J.nstiles = nst;
  J.resampler = resampler;
  J.conv = convention;
  J.key = S->key;
  J.flags = S->flags;
  J.sc = &S->sc;
  J.unif = uniforms_dev;
  J.wraw = weights_dev;
  J.lw = (void*)weights_dev;  // not read when wraw is set
  na_write_job<<<1, 1, 0, s>>>(J, &S->job);
  if (cudaMemsetAsync(S->flags, 0, sizeof(unsigned long long) * 2 * nst, s) != cudaSuccess) return GF_ERR_CUDA;
  sa_partial_sum<<<kNoAllocParts, 256, 0, s>>>(weights_dev, n, S->part);
  sa_setup<<<1, 256, 0, s>>>(S->part, kNoAllocParts, &S->sc, uniforms_dev, resampler);
  pf_scan_kernel<float><<<nst, SCAN_THREADS, 0, s>>>(&S->job, 1);
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)dev_sms * 8) blocks = (int64_t)dev_sms * 8;
  sa_search<<<(int)blocks, 256, 0, s>>>(&S->job, ancestors_dev);
  if (cudaGetLastError() != cudaSuccess) return GF_ERR_CUDA;
  int32_t status = 0;
  if (cudaMemcpyAsync(&status, &S->sc.status, sizeof status, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return GF_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return GF_ERR_CUDA;
  return status;
}
