// gf_common.cuh -- shared device helpers for the B200 filtering library.
//
// Philox4x32-10 (Salmon et al., SC'11) counter-based RNG, warp/block
// reductions, and the per-job scalar block the particle-filter kernels share.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gf_b200.h"

#define GF_LOG2PI 1.8378770664093454835606594728112

namespace gf {

// ---------------------------------------------------------------- Philox ---
// Counter layout (shared with the FP64 oracle so it can regenerate the noise):
//   normals : ctr = (particle i, step t, block q, 'NORM'), 4 normals per call;
//             a one-dimensional linear-Gaussian state takes normal i % 4 of the
//             call (i / 4, t, 0, 'NORM'), so no draw is discarded

//   uniforms: ctr = (slot j, step t, 0, 'UNIF'), one FP64 uniform per call
constexpr uint32_t kTagNormal = 0x4E4F524Du;
constexpr uint32_t kTagUnif = 0x554E4946u;
constexpr uint32_t kTagLookahead = 0x4C4B4844u;  // DrawPredictive draws of the auxiliary filter

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                       uint32_t c3, uint32_t k0, uint32_t k1,
                                                       uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Four N(0,1) draws: Box-Muller on 24-bit uniforms u1 in (0,1], u2 in [0,1),
// angle 2*pi*u2 - pi (keeps the fast sin/cos argument inside [-pi, pi]).
template <typename Real>
__device__ __forceinline__ void philox_normals4(uint64_t seed, uint32_t i, uint32_t t, uint32_t q,
                                                Real out[4], uint32_t tag = kTagNormal) {
  uint32_t w[4];
  philox4x32_10(i, t, q, tag, (uint32_t)seed, (uint32_t)(seed >> 32), w);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if constexpr (sizeof(Real) == 4) {
      float u1 = (float)((w[2 * p] >> 8) + 1u) * (1.0f / 16777216.0f);
      float u2 = (float)(w[2 * p + 1] >> 8) * (1.0f / 16777216.0f);
      float r = sqrtf(-2.0f * __logf(u1));
      float s, c;
      __sincosf(6.2831853071795865f * u2 - 3.1415926535897932f, &s, &c);
      out[2 * p] = r * c;
      out[2 * p + 1] = r * s;
    } else {
      double u1 = (double)((w[2 * p] >> 8) + 1u) * (1.0 / 16777216.0);
      double u2 = (double)(w[2 * p + 1] >> 8) * (1.0 / 16777216.0);
      double r = sqrt(-2.0 * log(u1));
      double s, c;
      sincos(6.283185307179586 * u2 - 3.141592653589793, &s, &c);
      out[2 * p] = r * c;
      out[2 * p + 1] = r * s;
    }
  }
}

__host__ __device__ __forceinline__ double philox_uniform(uint64_t seed, uint32_t j, uint32_t t) {
  uint32_t w[4];
  philox4x32_10(j, t, 0u, kTagUnif, (uint32_t)seed, (uint32_t)(seed >> 32), w);
  uint64_t bits = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------- reductions ---
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// The threads that reduce and synchronise together (the block); the
// reductions and the step finalise are written against this interface.
struct BlockSync {
  __device__ __forceinline__ int tid() const { return (int)threadIdx.x; }
  __device__ __forceinline__ int size() const { return (int)blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Reductions over the threads of S (a multiple of 32, <= 1024). `sh` is shared
// scratch of >= 32 doubles owned by S; every thread ends holding the result.
template <class S>
__device__ __forceinline__ double sync_max(const S& g, double v, double* sh) {
  const int lane = g.tid() & 31, wid = g.tid() >> 5, nw = g.size() >> 5;
  v = warp_max(v);
  g.sync();
  if (lane == 0) sh[wid] = v;
  g.sync();
  v = lane < nw ? sh[lane] : -INFINITY;
  return warp_max(v);
}
template <class S>
__device__ __forceinline__ double sync_sum(const S& g, double v, double* sh) {
  const int lane = g.tid() & 31, wid = g.tid() >> 5, nw = g.size() >> 5;
  v = warp_sum(v);
  g.sync();
  if (lane == 0) sh[wid] = v;
  g.sync();
  v = lane < nw ? sh[lane] : 0.0;
  return warp_sum(v);
}
__device__ __forceinline__ double block_max(double v, double* sh) { return sync_max(BlockSync(), v, sh); }
__device__ __forceinline__ double block_sum(double v, double* sh) { return sync_sum(BlockSync(), v, sh); }

// ---------------------------------------------------------- job scalars ----
// Device-resident per-filter scalars of a particle filter.  The last block of
// each propagate launch folds the per-block partials into these.
struct PfScalars {
  double lse;         // LSE of the stored log-weights after the last update
  double ll;          // accumulated log-evidence
  double ess;         // ESS of the current weights (decides the next resample)
  double u0;          // systematic uniform of the pending resample
  double wn;          // total normalised weight (fixed-point sum / 2^62)
  double wtotal;      // sum of raw weights (standalone sample_ancestors)
  double lse_aux;     // auxiliary filter: LSE(logw + log eta) of the pending resample
  double base_adj;    // auxiliary filter: shift of the post-resample baseline log N
  int32_t t;          // last completed step (0 after initialisation)
  int32_t resample;   // 1 if step t+1 starts with a resample
  int32_t uniform;    // 1 while the weights are the initial TypelessZero ones
  int32_t status;     // gf_status of the job (sticky)
  uint32_t counter;   // last-block-done counter of the propagate launch
  uint32_t scan_tile; // dynamic tile ticket of the lookback scan
  int32_t clamps;     // slots clamped to N by the search (reference has no clamp)
  uint32_t mcounter;  // last-block-done counter of the weighted-means launch
};

}  // namespace gf
