// gf_resample.cu -- standalone resampling primitives of the C ABI:
// sample_ancestors on device weights (resamplers.jl:206-238, ext/CUDAExt.jl:31-78),
// offspring <-> ancestors conversion (ext/CUDAExt.jl:90-142) and the exported
// in-kernel noise stream.
#include <cmath>
#include <cstring>
#include <vector>

#include "gf_internal.hpp"
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"

namespace gf {

// Deterministic two-level sum of the raw weights -> sc->wtotal; also seeds the
// scalars the shared scan / search read.
__global__ void sa_partial_sum(const double* __restrict__ w, int64_t n, double* __restrict__ part) {
  __shared__ double red[32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += w[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void sa_setup(const double* __restrict__ part, int nparts, PfScalars* sc,
                         const double* __restrict__ unif, int kind) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    sc->wtotal = s;
    sc->lse = 0.0;
    sc->ll = 0.0;
    sc->ess = 0.0;
    sc->u0 = kind == GF_RS_SYSTEMATIC ? unif[0] : 0.0;
    sc->wn = 1.0;
    sc->t = 0;
    sc->resample = 1;
    sc->uniform = 0;
    sc->status = s > 0.0 ? 0 : GF_ERR_ARG;
    sc->counter = 0;
    sc->scan_tile = 0;
    sc->lse_aux = 0.0;
    sc->base_adj = 0.0;
    sc->clamps = 0;
    sc->mcounter = 0;
  }
}

// Per-slot ancestor search over the scanned cumulative weights (1-based int64).
__global__ void sa_search(const PfJob* __restrict__ jobs, int64_t* __restrict__ anc) {
  const PfJob& J = jobs[0];
  PfScalars* sc = J.sc;
  if (sc->status != 0) return;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < J.N;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = find_ancestor(J, sc, 1, j, 0, J.N);
    anc[j] = a + 1;
  }
}

// offspring_to_ancestors with one binary search per output slot (balanced even
// when one particle has many offspring): ancestor of slot j = first i with
// offspring[i] > j.  Slots past offspring[n-1] are left 0.
__global__ void o2a_kernel(const int64_t* __restrict__ off, int64_t n, int64_t* __restrict__ anc) {
  const int64_t total = off[n - 1];
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    if (j >= total) {
      anc[j] = 0;
      continue;
    }
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = lo + ((hi - lo) >> 1);
      if (off[mid] > j) hi = mid;
      else lo = mid + 1;
    }
    anc[j] = lo + 1;
  }
}

__global__ void a2o_kernel(const int64_t* __restrict__ anc, int64_t n, unsigned long long* __restrict__ off) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = anc[i];
    if (a >= 1 && a <= n) atomicAdd(off + (a - 1), 1ull);
  }
}

template <typename Real>
__global__ void rng_normals_kernel(uint64_t seed, int t, int dx, int64_t n, Real* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (dx == 1) {  // 1-D layout: normal i % 4 of call i / 4
      Real tmp[4];
      philox_normals4<Real>(seed, (uint32_t)(i >> 2), (uint32_t)t, 0u, tmp);
      out[i] = tmp[i & 3];
      continue;
    }
    for (int q = 0; q * 4 < dx; ++q) {
      Real tmp[4];
      philox_normals4<Real>(seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, tmp);
      for (int r = 0; r < 4 && 4 * q + r < dx; ++r) out[(size_t)(4 * q + r) * n + i] = tmp[r];
    }
  }
}

static int grid_for(gf_ctx* ctx, int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = (int64_t)ctx->num_sms * 8;
  return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace gf

using namespace gf;

extern "C" gf_status gf_sample_ancestors(gf_ctx* ctx, int32_t resampler, int32_t convention, int64_t n,
                                         const double* weights_dev, const double* uniforms_dev,
                                         int64_t* ancestors_dev) {
  if (!ctx || !weights_dev || !uniforms_dev || !ancestors_dev || n < 1)
    return ctx ? set_err(ctx, GF_ERR_ARG, "bad arguments") : GF_ERR_ARG;
  if (resampler < 0 || resampler > 2 || convention < 0 || convention > 1)
    return set_err(ctx, GF_ERR_ARG, "unknown resampler / convention");
  if (n > (int64_t(1) << 31) - 1) return set_err(ctx, GF_ERR_ARG, "n must be < 2^31");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int nst = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
  const int nparts = 256;
  std::vector<DevBuf> bufs;
  struct Cleanup {
    gf_ctx* c;
    std::vector<DevBuf>* v;
    ~Cleanup() {
      cudaStreamSynchronize(c->stream);
      for (auto& b : *v) dev_free(c, b.p, b.bytes);
    }
  } cleanup{ctx, &bufs};
  auto get = [&](size_t bytes, void** d) -> gf_status {
    gf_status s2 = dev_alloc(ctx, bytes, d);
    if (!s2 && *d) bufs.push_back({*d, bytes});
    return s2;
  };
  gf_status st;
  void *key, *flags, *scv, *part, *jobv;
  if ((st = get(sizeof(double) * n, &key))) return st;
  if ((st = get(sizeof(unsigned long long) * 2 * nst, &flags))) return st;
  if ((st = get(sizeof(PfScalars), &scv))) return st;
  if ((st = get(sizeof(double) * nparts, &part))) return st;
  if ((st = get(sizeof(PfJob), &jobv))) return st;
  PfJob J;
  std::memset(&J, 0, sizeof J);
  J.N = n;
  J.T = 1;
  J.nstiles = nst;
  J.resampler = resampler;
  J.conv = convention;
  J.key = (double*)key;
  J.flags = (unsigned long long*)flags;
  J.sc = (PfScalars*)scv;
  J.unif = uniforms_dev;
  J.wraw = weights_dev;
  J.lw = (void*)weights_dev;  // not read when wraw is set
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(jobv, &J, sizeof J, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(flags, 0, sizeof(unsigned long long) * 2 * nst, s));
  sa_partial_sum<<<nparts, 256, 0, s>>>(weights_dev, n, (double*)part);
  sa_setup<<<1, 256, 0, s>>>((const double*)part, nparts, (PfScalars*)scv, uniforms_dev, resampler);
  // the scan runs for "step 0 -> 1" (t = 0 < T = 1, resample = 1)
  launch_scan(ctx, false, (const PfJob*)jobv, 1, nst);
  sa_search<<<grid_for(ctx, n), 256, 0, s>>>((const PfJob*)jobv, ancestors_dev);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  PfScalars sc;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(&sc, scv, sizeof sc, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (sc.status == GF_ERR_TIMEOUT) return set_err(ctx, GF_ERR_TIMEOUT, "lookback scan wait timed out");
  if (sc.status) return set_err(ctx, sc.status, "weights must have a positive sum");
  return GF_OK;
}

extern "C" gf_status gf_offspring_to_ancestors(gf_ctx* ctx, int64_t n, const int64_t* offspring_dev,
                                               int64_t* ancestors_dev) {
  if (!ctx || n < 1 || !offspring_dev || !ancestors_dev) return ctx ? set_err(ctx, GF_ERR_ARG, "bad arguments") : GF_ERR_ARG;
  cudaSetDevice(ctx->device);
  o2a_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(offspring_dev, n, ancestors_dev);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

extern "C" gf_status gf_ancestors_to_offspring(gf_ctx* ctx, int64_t n, const int64_t* ancestors_dev,
                                               int64_t* offspring_dev) {
  if (!ctx || n < 1 || !ancestors_dev || !offspring_dev) return ctx ? set_err(ctx, GF_ERR_ARG, "bad arguments") : GF_ERR_ARG;
  cudaSetDevice(ctx->device);
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(offspring_dev, 0, sizeof(int64_t) * n, ctx->stream));
  a2o_kernel<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(ancestors_dev, n, (unsigned long long*)offspring_dev);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

extern "C" gf_status gf_rng_normals(gf_ctx* ctx, uint64_t seed, int32_t t, int32_t dx, int64_t n,
                                    int32_t precision, void* out_dev) {
  if (!ctx || !out_dev || n < 1 || dx < 1) return ctx ? set_err(ctx, GF_ERR_ARG, "bad arguments") : GF_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (precision == GF_PREC_F64)
    rng_normals_kernel<double><<<grid_for(ctx, n), 256, 0, ctx->stream>>>(seed, t, dx, n, (double*)out_dev);
  else
    rng_normals_kernel<float><<<grid_for(ctx, n), 256, 0, ctx->stream>>>(seed, t, dx, n, (float*)out_dev);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}
