// gf_internal.hpp -- host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/gf_b200.h"

struct gf_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // private stream-ordered pool for scratch and plan buffers (freed memory stays
  // cached in the pool, so repeated one-shot calls do not synchronise the device)
  cudaMemPool_t pool = nullptr;
  size_t budget = 0;
  size_t used = 0;
  std::string err;
  // per-kernel-class event timing
  bool profiling = false;
  struct Pending {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  double prof_ms[8] = {0};
  long long prof_n[8] = {0};
  // plans kept by the one-shot particle-filter calls (gf_pf_run, gf_pf_run_tv),
  // most recently used first: (model / configuration key, gf_pf_plan*)
  std::vector<std::pair<std::vector<char>, void*>> pf_plans;
};

namespace gf {

enum KernelClass { KC_PROPAGATE = 0, KC_SCAN = 1, KC_KF = 2, KC_RBPF = 3, KC_PREP = 4, KC_FILL = 5 };

gf_status set_err(gf_ctx* ctx, gf_status code, const char* fmt, ...);
void pf_plan_cache_release(gf_ctx* ctx);  // frees the plans kept in ctx->pf_plans
gf_status cuda_err(gf_ctx* ctx, cudaError_t e, const char* where);
gf_status dev_alloc(gf_ctx* ctx, size_t bytes, void** p);
void dev_free(gf_ctx* ctx, void* p, size_t bytes);

// RAII event pair around a launch when profiling is on.
struct ProfScope {
  gf_ctx* ctx;
  int cls;
  cudaEvent_t b = nullptr;
  ProfScope(gf_ctx* c, int k);
  ~ProfScope();
};

// Device allocation owned by a plan; freed with the plan.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Small host-side dense helpers (FP64, column-major) used to precompute
// model factors once per plan.
int chol_lower(int n, const double* A, double* L);  // from the upper triangle
void tri_inv_lower(int n, const double* L, double* Linv);
void matmul(int m, int k, int n, const double* A, const double* B, double* C);

#define GF_CHECK_CUDA(ctx, expr)                              \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) return gf::cuda_err(ctx, _e, #expr); \
  } while (0)

}  // namespace gf
