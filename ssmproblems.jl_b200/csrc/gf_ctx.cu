// gf_ctx.cu -- context, errors, HBM budget accounting and per-kernel timing.
#include <cmath>
#include <cstring>

#include "gf_internal.hpp"

namespace gf {

gf_status set_err(gf_ctx* ctx, gf_status code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

gf_status cuda_err(gf_ctx* ctx, cudaError_t e, const char* where) {
  return set_err(ctx, GF_ERR_CUDA, "CUDA error %s (%s) at %s", cudaGetErrorName(e),
                 cudaGetErrorString(e), where);
}

gf_status dev_alloc(gf_ctx* ctx, size_t bytes, void** p) {
  *p = nullptr;
  if (bytes == 0) return GF_OK;
  if (ctx->used + bytes > ctx->budget)
    return set_err(ctx, GF_ERR_OOM_BUDGET, "HBM budget exceeded: need %zu more bytes, %zu of %zu used",
                   bytes, ctx->used, ctx->budget);
  cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream)
                            : cudaMalloc(p, bytes);
  if (e != cudaSuccess) return cuda_err(ctx, e, "device allocation");
  ctx->used += bytes;
  return GF_OK;
}

void dev_free(gf_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  if (ctx->pool) cudaFreeAsync(p, ctx->stream);
  else cudaFree(p);
  ctx->used = ctx->used >= bytes ? ctx->used - bytes : 0;
}

static cudaEvent_t take_event(gf_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

ProfScope::ProfScope(gf_ctx* c, int k) : ctx(c), cls(k) {
  if (!ctx->profiling) return;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(ctx->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
    return;  // events inside a capture are not timestamps
  b = take_event(ctx);
  cudaEventRecord(b, ctx->stream);
}

ProfScope::~ProfScope() {
  if (!b) return;
  cudaEvent_t a = take_event(ctx);
  cudaEventRecord(a, ctx->stream);
  ctx->pending.push_back({cls, b, a});
}

int chol_lower(int n, const double* A, double* L) {
  for (int i = 0; i < n * n; ++i) L[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    double s = A[j + j * n];
    for (int k = 0; k < j; ++k) s -= L[j + k * n] * L[j + k * n];
    if (!(s > 0.0)) return 1;
    double d = std::sqrt(s);
    L[j + j * n] = d;
    for (int i = j + 1; i < n; ++i) {
      double t = A[j + i * n];
      for (int k = 0; k < j; ++k) t -= L[i + k * n] * L[j + k * n];
      L[i + j * n] = t / d;
    }
  }
  return 0;
}

void tri_inv_lower(int n, const double* L, double* X) {
  for (int i = 0; i < n * n; ++i) X[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    X[j + j * n] = 1.0 / L[j + j * n];
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s += L[i + k * n] * X[k + j * n];
      X[i + j * n] = -s / L[i + i * n];
    }
  }
}

void matmul(int m, int k, int n, const double* A, const double* B, double* C) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += A[i + p * m] * B[p + j * k];
      C[i + j * m] = s;
    }
}

}  // namespace gf

using namespace gf;

extern "C" {

int32_t gf_version(void) { return 100; }

gf_status gf_ctx_create(int32_t device, size_t hbm_budget_bytes, gf_ctx** out) {
  if (!out) return GF_ERR_ARG;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return GF_ERR_CUDA;
  if (device < 0 || device >= n) return GF_ERR_ARG;
  gf_ctx* ctx = new gf_ctx();
  ctx->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    delete ctx;
    return GF_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  ctx->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.9 * (double)fr);
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete ctx;
    return GF_ERR_CUDA;
  }
  ctx->own_stream = true;
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;  // keep freed blocks for reuse until the context goes
      cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
      ctx->pool = nullptr;  // fall back to cudaMalloc / cudaFree
      cudaGetLastError();
    }
  }
  *out = ctx;
  return GF_OK;
}

gf_status gf_ctx_destroy(gf_ctx* ctx) {
  if (!ctx) return GF_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  gf::pf_plan_cache_release(ctx);
  for (auto& p : ctx->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->pool) {
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolDestroy(ctx->pool);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GF_OK;
}

const char* gf_last_error(const gf_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

gf_status gf_ctx_set_stream(gf_ctx* ctx, void* stream) {
  if (!ctx) return GF_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->own_stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    ctx->own_stream = false;
  }
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    ctx->own_stream = true;
  }
  return GF_OK;
}

void* gf_ctx_get_stream(gf_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

gf_status gf_ctx_synchronize(gf_ctx* ctx) {
  if (!ctx) return GF_ERR_ARG;
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

gf_status gf_ctx_memory(const gf_ctx* ctx, size_t* used, size_t* budget) {
  if (!ctx) return GF_ERR_ARG;
  if (used) *used = ctx->used;
  if (budget) *budget = ctx->budget;
  return GF_OK;
}

gf_status gf_ctx_profile(gf_ctx* ctx, int32_t enable) {
  if (!ctx) return GF_ERR_ARG;
  ctx->profiling = enable != 0;
  if (enable) {
    for (int i = 0; i < 8; ++i) {
      ctx->prof_ms[i] = 0;
      ctx->prof_n[i] = 0;
    }
  }
  return GF_OK;
}

gf_status gf_ctx_profile_read(gf_ctx* ctx, int32_t cls, double* total_ms, int64_t* launches) {
  if (!ctx || cls < 0 || cls >= 8) return GF_ERR_ARG;
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto& p : ctx->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    ctx->prof_ms[p.cls] += ms;
    ctx->prof_n[p.cls] += 1;
    ctx->event_pool.push_back(p.a);
    ctx->event_pool.push_back(p.b);
  }
  ctx->pending.clear();
  if (total_ms) *total_ms = ctx->prof_ms[cls];
  if (launches) *launches = ctx->prof_n[cls];
  return GF_OK;
}

}  // extern "C"
