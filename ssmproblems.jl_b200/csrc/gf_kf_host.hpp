// gf_kf_host.hpp -- Kalman-bank descriptors and launch helpers shared by the
// batched plans (gf_kf.cu) and the serving loop (gf_serve.cu).
#pragma once
#include <cstdint>
#include <vector>

#include "gf_internal.hpp"

namespace gf {

// Result record of one served filter, in host-mapped pinned memory.  The
// kernel writes ll, status, the final mean / covariance and the per-step
// log-likelihoods, issues a system-scope fence and sets `done` last, so a
// host thread that reads done == 1 sees everything else.
struct KfSrvRec {
  double ll;
  int32_t status;
  volatile int32_t done;
};

struct KfDesc {
  // pstep: floats per step of a time-varying model's parameter blocks (0: one
  // block for every step); p0: float offset of the prior (mu0, Sigma0) from the
  // filter's first block (0: right after the single block)
  int32_t dx, dy, T, pstep;
  int64_t poff;    // float offset into the parameter pool
  int64_t yoff;    // double offset into ys
  int64_t soff;    // step offset (ll_steps)
  int64_t moff;    // float offset of means
  int64_t coff;    // float offset of covs
  int32_t index;   // caller's filter index
  int32_t p0;
  // serving only (null in plans): host-mapped destinations of this filter
  KfSrvRec* srv;
  float* srv_mu;       // [dx] final filtered mean
  float* srv_cov;      // [dx*dx] final filtered covariance, column-major
  double* srv_steps;   // nullable [T] per-step log-likelihoods
};

struct KfRun {
  const KfDesc* desc;
  const int32_t* order;     // bucket work list (indices into desc)
  int32_t count;
  uint32_t* counter;        // persistent work ticket
  const float* params;
  const double* ys;
  double* ll;               // [B]
  double* ll_steps;
  float* means;
  float* covs;
  int32_t* status;          // [B]
  double jitter;
  int32_t use_jitter;
  int32_t algo;
};

// parameter pool layout per filter (column-major, unpadded):
//   A dx*dx | b dx | Q dx*dx | H dy*dx | c dy | R dy*dy | mu0 dx | S0 dx*dx |
//   UQ dx*dx | UR dy*dy | U0 dx*dx     (upper Cholesky factors, used by the SRKF)
// A time-varying model holds T step blocks followed by the prior: for the KF
// (A b Q H c R) then mu0 | S0; for the SRKF (A b H c UQ UR) then mu0 | U0.
__host__ __device__ inline int64_t kf_param_len(int dx, int dy) {
  return (int64_t)5 * dx * dx + 2 * dx + dy * dx + dy + 2 * dy * dy;
}
__host__ __device__ inline int32_t kf_step_block_len(int dx, int dy) {
  return 2 * dx * dx + dx + dy * dx + dy + dy * dy;
}
__host__ __device__ inline int32_t sr_step_block_len(int dx, int dy) {
  return 2 * dx * dx + dx + dy * dx + dy + dy * dy;
}

// Dimension buckets: index of the smallest compiled (DXP, DYP) holding (dx, dy),
// -1 if none (dx, dy <= 32).
int kf_bucket_for(int dx, int dy);
int kf_bucket_count();
int kf_bucket_dxp(int kidx);
int kf_default_group(int kidx);
// Sets the dynamic shared-memory limit of a bucket's kernel (idempotent).
gf_status kf_prepare_bucket(gf_ctx* ctx, int algo, int kidx);
// Persistent blocks per SM of a bucket kernel at `group` threads.
int kf_blocks_per_sm(int algo, int kidx, int group);
void kf_launch(int algo, int kidx, int group, int grid, const KfRun& r, cudaStream_t s);
// Appends one filter's parameters (and, for the SRKF, its Cholesky factors) to
// the FP32 pool; returns GF_ERR_NOT_PD if the SRKF factors do not exist.
gf_status kf_pack_model(gf_ctx* ctx, int algo, const gf_lg_model& m, int f, std::vector<float>& pool);

}  // namespace gf
