// gf_kf.cu -- batched Kalman and square-root Kalman filters.
//
// One thread block per filter; the filter's matrices live in shared memory
// (row-major, padded stride) for the whole time loop.  FP32 storage and
// arithmetic for the bulk, FP64 for the innovation covariance S, its Cholesky
// factor, the gain solve and the log-likelihood.
//
// KF step restates kalman.jl:42-66 and kalman_gradient.jl:12-23:
//   mu^ = A mu + b, Sigma^ = A Sigma A' + Q
//   z = y - H mu^ - c, S = H Sigma^ H' + R, K = Sigma^ H' S^-1
//   Sigma = (I - K H) Sigma^ (I - K H)' + K R K'   (Joseph form, upper triangle
//   mirrored as PDMat(Symmetric(.)) does), mu = mu^ + K z,
//   ll = -1/2 (z' S^-1 z + log|S| + dy log 2 pi).
// SRKF step restates srkf.jl:93-176 with Householder QR.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "gf_common.cuh"
#include "gf_internal.hpp"
#include "gf_kf_host.hpp"

namespace gf {

template <int DXP, int DYP>
struct KfSmem {
  // Float matrices are row-major with 16-byte rows (stride a multiple of 4 and
  // at least 4 past the width): the products read four k at a time, so every
  // row an operand of a product is zero in its columns [k, ceil4(k)).
  static constexpr int LD = DXP + 4;   // row stride of dx-wide matrices
  static constexpr int LY = DYP + 4;   // row stride of dy-wide matrices
  static constexpr int LS = DYP + 1;   // row stride of S (FP64)
  static constexpr int LW = DXP + 1;   // row stride of the FP64 solve buffer (dx RHS + z)
  double S[DYP * LS], dinv[DYP], z[DYP], w[DYP], red[32];
  // Buffers shared by values whose lifetimes within a step do not overlap:
  //   Sig : filtered covariance; from phase 2 to 8 it holds the prediction Sp
  //   T1  : A Sig (phases 1-2), then I - K H (phases 7-9)
  //   W2  : (I - K H) Sp | K R (phases 7-9); the FP64 solve buffer Wm (5-6)
  alignas(16) float A[DXP * LD];
  alignas(16) float Q[DXP * LD];
  alignas(16) float Sig[DXP * LD];
  alignas(16) float T1[DXP * LD];
  alignas(16) float H[DYP * LD];
  alignas(16) float HS[DYP * LD];  // H Sp (phases 3-6)
  alignas(16) float K[DXP * LY];
  alignas(16) float R[DYP * LY];
  alignas(16) float W2[DXP * LD + DXP * LY];
  float mu[DXP], mup[DXP], b[DXP], c[DYP];
  int fid, fail;
  static_assert(DYP * LW * sizeof(double) <= sizeof(W2), "Wm must fit in W2");
};

__device__ __forceinline__ void group_sync() { __syncthreads(); }

// One step's parameters (A b Q H c R, column-major) into shared memory (the
// valid entries only: padding stays as kf_load left it).
template <int DXP, int DYP>
__device__ void kf_load_step(KfSmem<DXP, DYP>& s, const float* P, int dx, int dy) {
  const int G = blockDim.x;
  const float* pA = P;
  const float* pb = pA + dx * dx;
  const float* pQ = pb + dx;
  const float* pH = pQ + dx * dx;
  const float* pc = pH + dy * dx;
  const float* pR = pc + dy;
  constexpr int LD = KfSmem<DXP, DYP>::LD, LY = KfSmem<DXP, DYP>::LY;
  for (int e = threadIdx.x; e < dx * dx; e += G) {
    int i = e % dx, j = e / dx;  // column-major source
    s.A[i * LD + j] = pA[e];
    s.Q[i * LD + j] = pQ[e];
  }
  for (int e = threadIdx.x; e < dy * dx; e += G) {
    int i = e % dy, j = e / dy;
    s.H[i * LD + j] = pH[e];
  }
  for (int e = threadIdx.x; e < dy * dy; e += G) {
    int i = e % dy, j = e / dy;
    s.R[i * LY + j] = pR[e];
  }
  for (int e = threadIdx.x; e < dx; e += G) s.b[e] = pb[e];
  for (int e = threadIdx.x; e < dy; e += G) s.c[e] = pc[e];
}

// A filter's first-step parameters from P and its prior (mu0, Sigma0) from P0.
template <int DXP, int DYP>
__device__ void kf_load(KfSmem<DXP, DYP>& s, const float* P, const float* P0, int dx, int dy) {
  const int G = blockDim.x;
  constexpr int LD = KfSmem<DXP, DYP>::LD;
  // zero every float matrix first: the product operands' k-padding must be 0
  using SM = KfSmem<DXP, DYP>;
  constexpr int nzero = (int)((offsetof(SM, mu) - offsetof(SM, A)) / sizeof(float));
  for (int e = threadIdx.x; e < nzero; e += G) s.A[e] = 0.f;
  __syncthreads();
  kf_load_step<DXP, DYP>(s, P, dx, dy);
  const float* pm = P0;
  const float* pS = pm + dx;
  for (int e = threadIdx.x; e < dx * dx; e += G) s.Sig[(e % dx) * LD + e / dx] = pS[e];
  for (int e = threadIdx.x; e < dx; e += G) s.mu[e] = pm[e];
}

// ------------------------------------------------------------ small products
// C(i, j) = init(i, j) + sum_k A[i][k] B[j][k] for i < m, j < n (both operands
// row-major with k contiguous, 16-byte rows, zero in columns [kk, ceil4(kk))).
// Each thread of the block takes 2x2 outputs and reads four k per 128-bit
// shared-memory load (two A rows, two B rows: 16 FMAs per 4 loads).  Every
// output accumulates its FMAs in k order, so the result does not depend on
// the block size.  SYM: only tiles on or above the diagonal, each output with
// j >= i written to (i, j) and (j, i).  A second operand pair (A2, B2, kk2) is
// accumulated after the first into the same sums.  Acc = float or double
// (double: FP64 FMAs of the FP32 products' operands).
template <typename Acc, bool SYM, typename Init, typename Store>
__device__ __forceinline__ void mm_abt(const float* A, int lda, const float* B, int ldb, int kk,
                                       const float* A2, int lda2, const float* B2, int ldb2, int kk2,
                                       int m, int n, Init init, Store store) {
  const int tm = (m + 1) >> 1, tn = (n + 1) >> 1;
  for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
    const int ti = t / tn, tj = t - ti * tn;
    if (SYM && tj < ti) continue;
    const int i0 = 2 * ti, j0 = 2 * tj;
    const int i1 = min(i0 + 1, m - 1), j1 = min(j0 + 1, n - 1);
    Acc c00 = init(i0, j0), c01 = init(i0, j1), c10 = init(i1, j0), c11 = init(i1, j1);
    auto run = [&](const float* X, int ldx, const float* Y, int ldy, int k) {
      const float4* a0 = reinterpret_cast<const float4*>(X + i0 * ldx);
      const float4* a1 = reinterpret_cast<const float4*>(X + i1 * ldx);
      const float4* b0 = reinterpret_cast<const float4*>(Y + j0 * ldy);
      const float4* b1 = reinterpret_cast<const float4*>(Y + j1 * ldy);
      const int k4 = (k + 3) >> 2;
#pragma unroll 1
      for (int q = 0; q < k4; ++q) {
        const float4 x0 = a0[q], x1 = a1[q], y0 = b0[q], y1 = b1[q];
        auto step = [&](float u0, float u1, float v0, float v1) {
          c00 = fma((Acc)u0, (Acc)v0, c00);
          c01 = fma((Acc)u0, (Acc)v1, c01);
          c10 = fma((Acc)u1, (Acc)v0, c10);
          c11 = fma((Acc)u1, (Acc)v1, c11);
        };
        step(x0.x, x1.x, y0.x, y1.x);
        step(x0.y, x1.y, y0.y, y1.y);
        step(x0.z, x1.z, y0.z, y1.z);
        step(x0.w, x1.w, y0.w, y1.w);
      }
    };
    run(A, lda, B, ldb, kk);
    if (A2) run(A2, lda2, B2, ldb2, kk2);
    if (!SYM || j0 >= i0) store(i0, j0, c00);
    if (j1 > j0 && (!SYM || j1 >= i0)) store(i0, j1, c01);
    if (i1 > i0 && (!SYM || j0 >= i1)) store(i1, j0, c10);
    if (i1 > i0 && j1 > j0 && (!SYM || j1 >= i1)) store(i1, j1, c11);
  }
}

// C(i, j) = init(i, j) - sum_{k < kk} A[i][k] B[k][j] (B row-major, j contiguous,
// rows 8-byte aligned), 2x2 outputs per thread, FMAs in k order.
template <typename Init, typename Store>
__device__ __forceinline__ void mm_ab_neg(const float* A, int lda, const float* B, int ldb, int kk,
                                          int m, int n, Init init, Store store) {
  const int tm = (m + 1) >> 1, tn = (n + 1) >> 1;
  for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
    const int ti = t / tn, tj = t - ti * tn;
    const int i0 = 2 * ti, j0 = 2 * tj;
    const int i1 = min(i0 + 1, m - 1);
    float c00 = init(i0, j0), c01 = init(i0, j0 + 1), c10 = init(i1, j0), c11 = init(i1, j0 + 1);
    for (int k = 0; k < kk; ++k) {
      const float a0 = -A[i0 * lda + k], a1 = -A[i1 * lda + k];
      const float2 y = *reinterpret_cast<const float2*>(B + k * ldb + j0);
      c00 = fmaf(a0, y.x, c00);
      c01 = fmaf(a0, y.y, c01);
      c10 = fmaf(a1, y.x, c10);
      c11 = fmaf(a1, y.y, c11);
    }
    store(i0, j0, c00);
    if (j0 + 1 < n) store(i0, j0 + 1, c01);
    if (i1 > i0) {
      store(i1, j0, c10);
      if (j0 + 1 < n) store(i1, j0 + 1, c11);
    }
  }
}

// Zeroes columns [n, ceil4(n)) of rows [0, m) (k-padding of a product operand
// written into a buffer that held other data).
__device__ __forceinline__ void zero_pad(float* C, int ldc, int m, int n) {
  const int p = ((n + 3) & ~3) - n;
  for (int e = threadIdx.x; e < m * p; e += blockDim.x) C[(e / p) * ldc + n + e % p] = 0.f;
}

// FP64 Cholesky of s.S (dy x dy, lower triangle, in place) by warp 0 with one
// lane per row (right-looking; dy <= 32), plus the reciprocal diagonal.
// Returns false if S is not positive definite.
template <int DXP, int DYP>
__device__ bool kf_chol(KfSmem<DXP, DYP>& s, int dy) {
  constexpr int LS = KfSmem<DXP, DYP>::LS;
  if (threadIdx.x < 32) {
    const int r = threadIdx.x;
    for (int j = 0; j < dy; ++j) {
      const double djj = s.S[j * LS + j];
      if (!(djj > 0.0)) {
        if (r == 0) s.fail = 1;
        break;
      }
      const double d = sqrt(djj), inv = 1.0 / d;
      double lrj = 0.0;
      if (r > j && r < dy) {
        lrj = s.S[r * LS + j] * inv;
        s.S[r * LS + j] = lrj;
      }
      if (r == j) {
        s.S[j * LS + j] = d;
        s.dinv[j] = inv;
      }
      __syncwarp();
      if (r > j && r < dy)
        for (int k = j + 1; k <= r; ++k) s.S[r * LS + k] -= lrj * s.S[k * LS + j];
      __syncwarp();
    }
  }
  __syncthreads();
  return !s.fail;
}

// Triangular solves on the RHS buffer Wm (dy rows): forward L Y = Wm over
// columns [0, nf), then back L' X = Y over columns [0, nb).  Lane = row, warps
// take interleaved column sets; dy <= 32.
template <int DXP, int DYP>
__device__ void kf_solves(KfSmem<DXP, DYP>& s, double* Wm, int dy, int nf, int nb) {
  constexpr int LS = KfSmem<DXP, DYP>::LS, LW = KfSmem<DXP, DYP>::LW;
  const int r = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = 0; i < dy; ++i) {
    if (r == i)
      for (int c = w; c < nf; c += nw) Wm[i * LW + c] *= s.dinv[i];
    __syncwarp();
    if (r > i && r < dy) {
      const double l = s.S[r * LS + i];
      for (int c = w; c < nf; c += nw) Wm[r * LW + c] -= l * Wm[i * LW + c];
    }
    __syncwarp();
  }
  for (int i = dy - 1; i >= 0; --i) {
    if (r == i)
      for (int c = w; c < nb; c += nw) Wm[i * LW + c] *= s.dinv[i];
    __syncwarp();
    if (r < i) {
      const double l = s.S[i * LS + r];
      for (int c = w; c < nb; c += nw) Wm[r * LW + c] -= l * Wm[i * LW + c];
    }
    __syncwarp();
  }
  __syncthreads();
}

// Serving: publishes the final mean, covariance (cov(i, j)), ll and status of a
// filter to its host-mapped record; `done` is written after a system-scope fence.
template <typename CovF>
__device__ void kf_srv_publish(const KfDesc& D, const float* mu, CovF cov, double ll, int status) {
  const int dx = D.dx;
  for (int i = threadIdx.x; i < dx; i += blockDim.x) D.srv_mu[i] = mu[i];
  for (int e = threadIdx.x; e < dx * dx; e += blockDim.x) D.srv_cov[e] = cov(e % dx, e / dx);
  __threadfence_system();
  __syncthreads();
  if (threadIdx.x == 0) {
    D.srv->ll = ll;
    D.srv->status = status;
    __threadfence_system();
    D.srv->done = 1;
  }
}

// 64 registers: four blocks of 256 threads (the dx <= 32 bucket's shared memory
// also allows four)
template <int DXP, int DYP>
__global__ void __launch_bounds__(256, 4) kf_batch_kernel(KfRun run) {
  using SM = KfSmem<DXP, DYP>;
  constexpr int LD = SM::LD, LY = SM::LY, LS = SM::LS, LW = SM::LW;
  extern __shared__ __align__(16) unsigned char smraw[];
  SM& s = *reinterpret_cast<SM*>(smraw);
  const int G = blockDim.x;
  float* const Sp = s.Sig;        // predicted covariance (phases 2-8)
  float* const IKH = s.T1;        // I - K H (phases 7-9)
  float* const T2 = s.W2;         // (I - K H) Sp (phases 8-9)
  float* const KR = s.W2 + DXP * LD;  // K R (phases 7-9)
  double* const Wm = reinterpret_cast<double*>(s.W2);
  const float* const nul = nullptr;
  auto zero = [](int, int) { return 0.f; };
  while (true) {
    if (threadIdx.x == 0) {
      unsigned k = atomicAdd(run.counter, 1u);
      s.fid = k < (unsigned)run.count ? run.order[k] : -1;
      s.fail = 0;
    }
    group_sync();
    const int f = s.fid;
    if (f < 0) return;
    const KfDesc D = run.desc[f];
    const int dx = D.dx, dy = D.dy;
    const float* P = run.params + D.poff;
    kf_load<DXP, DYP>(s, P, P + (D.p0 ? D.p0 : kf_step_block_len(dx, dy)), dx, dy);
    group_sync();
    double lltot = 0.0;
    int status = GF_OK;
    for (int t = 0; t < D.T; ++t) {
      const double* y = run.ys + D.yoff + (int64_t)t * dy;
      // 0. time-varying model: this step's A, b, Q, H, c, R (calc_params(dyn, t),
      //    calc_params(obs, t), models/linear_gaussian.jl:44-63)
      if (D.pstep && t > 0) {
        kf_load_step<DXP, DYP>(s, P + (int64_t)t * D.pstep, dx, dy);
        group_sync();
      }
      // 1. T1 = A Sigma (Sigma symmetric: rows of Sigma are its columns) ; mup = A mu + b
      mm_abt<float, false>(s.A, LD, s.Sig, LD, dx, nul, 0, nul, 0, 0, dx, dx, zero,
                                  [&](int i, int j, float v) { s.T1[i * LD + j] = v; });
      for (int i = threadIdx.x; i < dx; i += G) {
        float acc = s.b[i];
        for (int k = 0; k < dx; ++k) acc = fmaf(s.A[i * LD + k], s.mu[k], acc);
        s.mup[i] = acc;
      }
      group_sync();
      // 2. Sp = T1 A' + Q (upper triangle, mirrored)
      mm_abt<float, true>(s.T1, LD, s.A, LD, dx, nul, 0, nul, 0, 0, dx, dx,
                                 [&](int i, int j) { return s.Q[i * LD + j]; },
                                 [&](int i, int j, float v) {
                                   Sp[i * LD + j] = v;
                                   Sp[j * LD + i] = v;
                                 });
      group_sync();
      // 3. HS = H Sp (= (Sp H')') ; z = y - H mup - c
      mm_abt<float, false>(s.H, LD, Sp, LD, dx, nul, 0, nul, 0, 0, dy, dx, zero,
                                  [&](int i, int j, float v) { s.HS[i * LD + j] = v; });
      for (int i = threadIdx.x; i < dy; i += G) {
        double acc = y[i] - (double)s.c[i];
        for (int k = 0; k < dx; ++k) acc -= (double)s.H[i * LD + k] * (double)s.mup[k];
        s.z[i] = acc;
      }
      group_sync();
      // 4. S = H HS' + R in FP64 (lower triangle is all the Cholesky reads)
      mm_abt<double, false>(s.H, LD, s.HS, LD, dx, nul, 0, nul, 0, 0, dy, dy,
                                   [&](int i, int j) { return (double)s.R[i * LY + j]; },
                                   [&](int i, int j, double v) {
                                     if (j <= i) s.S[i * LS + j] = v;
                                   });
      group_sync();
      // 5. Cholesky of S (FP64)
      if (!kf_chol<DXP, DYP>(s, dy)) {
        status = GF_ERR_NOT_PD;
        break;
      }
      // 6. RHS = [HS | z]; forward solve gives w = L^-1 z (last column),
      //    back solve of the first dx columns gives K' = S^-1 HS
      for (int e = threadIdx.x; e < dy * (dx + 1); e += G) {
        const int i = e / (dx + 1), cc = e - i * (dx + 1);
        Wm[i * LW + cc] = cc < dx ? (double)s.HS[i * LD + cc] : s.z[i];
      }
      __syncthreads();
      kf_solves<DXP, DYP>(s, Wm, dy, dx + 1, dx);
      for (int i = threadIdx.x; i < dy; i += G) s.w[i] = Wm[i * LW + dx];
      for (int e = threadIdx.x; e < dx * dy; e += G) {
        const int i = e / dy, j = e - i * dy;
        s.K[i * LY + j] = (float)Wm[j * LW + i];
      }
      group_sync();
      // 7. mu = mup + K z ; IKH = I - K H ; KR = K R (R symmetric)
      for (int i = threadIdx.x; i < dx; i += G) {
        double acc = (double)s.mup[i];
        for (int k = 0; k < dy; ++k) acc += (double)s.K[i * LY + k] * s.z[k];
        s.mu[i] = (float)acc;
      }
      mm_ab_neg(s.K, LY, s.H, LD, dy, dx, dx, [](int i, int j) { return i == j ? 1.f : 0.f; },
                [&](int i, int j, float v) { IKH[i * LD + j] = v; });
      mm_abt<float, false>(s.K, LY, s.R, LY, dy, nul, 0, nul, 0, 0, dx, dy, zero,
                                  [&](int i, int j, float v) { KR[i * LY + j] = v; });
      zero_pad(KR, LY, dx, dy);
      group_sync();
      // 8. T2 = IKH Sp
      mm_abt<float, false>(IKH, LD, Sp, LD, dx, nul, 0, nul, 0, 0, dx, dx, zero,
                                  [&](int i, int j, float v) { T2[i * LD + j] = v; });
      zero_pad(T2, LD, dx, dx);
      group_sync();
      // 9. Sig = T2 IKH' + KR K' (+ jitter I), upper triangle mirrored
      const float jit = run.use_jitter ? (float)run.jitter : 0.f;
      mm_abt<float, true>(T2, LD, IKH, LD, dx, KR, LY, s.K, LY, dy, dx, dx, zero,
                                 [&](int i, int j, float v) {
                                   if (run.use_jitter && i == j) v += jit;
                                   s.Sig[i * LD + j] = v;
                                   s.Sig[j * LD + i] = v;
                                 });
      group_sync();
      // 10. outputs
      float* cov_out = run.covs ? run.covs + D.coff + (int64_t)t * dx * dx : nullptr;
      if (cov_out)
        for (int e = threadIdx.x; e < dx * dx; e += G) {
          const int j = e / dx, i = e - j * dx;
          cov_out[e] = s.Sig[i * LD + j];
        }
      if (run.means)
        for (int i = threadIdx.x; i < dx; i += G) run.means[D.moff + (int64_t)t * dx + i] = s.mu[i];
      if (threadIdx.x < 32) {
        double q = 0.0, ld = 0.0;
        for (int i = threadIdx.x; i < dy; i += 32) {
          q += s.w[i] * s.w[i];
          ld += log(s.S[i * LS + i]);
        }
        q = warp_sum(q);
        ld = warp_sum(ld);
        double l = -0.5 * (q + 2.0 * ld + dy * GF_LOG2PI);
        lltot += l;
        if (threadIdx.x == 0 && run.ll_steps) run.ll_steps[D.soff + t] = l;
        if (threadIdx.x == 0 && D.srv_steps) D.srv_steps[t] = l;
      }
      group_sync();
    }
    if (D.srv)
      kf_srv_publish(D, s.mu, [&](int i, int j) { return s.Sig[i * LD + j]; }, lltot, status);
    if (threadIdx.x == 0 && run.ll) {
      run.ll[D.index] = lltot;
      run.status[D.index] = status;
    }
    group_sync();
  }
}

// ---------------------------------------------------------------- SRKF
template <int DXP, int DYP>
struct SrSmem {
  static constexpr int NN = DXP + DYP;
  static constexpr int LM = NN + 1;
  float M[(2 * DXP + DYP) * LM];   // QR work matrix, row-major
  float A[DXP * (DXP + 1)], H[DYP * (DXP + 1)];
  float U[DXP * (DXP + 1)], UQ[DXP * (DXP + 1)], UR[DYP * (DYP + 1)];
  float mu[DXP], b[DXP], c[DYP];
  double z[DYP], w[DYP], colscale[NN];
  double red[32];
  int fid;
};

// In-place Householder QR of M (m x n, row-major, stride LM); leaves R in the
// upper triangle with rows sign-corrected so diag(R) >= 0 (srkf.jl:83).
template <int LM>
__device__ void householder_qr(float* M, int m, int n, double* colscale, double* red) {
  for (int k = 0; k < n; ++k) {
    double part = 0.0;
    for (int i = k + threadIdx.x; i < m; i += blockDim.x) part += (double)M[i * LM + k] * M[i * LM + k];
    double nrm2 = block_sum(part, red);
    double nrm = sqrt(nrm2);
    double x0 = M[k * LM + k];
    double alpha = x0 >= 0 ? -nrm : nrm;
    double v0 = x0 - alpha;
    double vv = nrm2 - x0 * x0 + v0 * v0;
    __syncthreads();
    if (nrm > 0.0 && vv > 0.0) {
      // column scales s_j = 2 v'M[:,j] / v'v for j > k (v = [v0, M[k+1:,k]])
      for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
        double acc = v0 * M[k * LM + j];
        for (int i = k + 1; i < m; ++i) acc += (double)M[i * LM + k] * M[i * LM + j];
        colscale[j] = 2.0 * acc / vv;
      }
      __syncthreads();
      for (int i = k + (threadIdx.x >> 5); i < m; i += (blockDim.x >> 5)) {
        const double vi = i == k ? v0 : (double)M[i * LM + k];
        for (int j = k + 1 + (threadIdx.x & 31); j < n; j += 32)
          M[i * LM + j] = (float)((double)M[i * LM + j] - colscale[j] * vi);
      }
      __syncthreads();
      if (threadIdx.x == 0) M[k * LM + k] = (float)alpha;
    }
    __syncthreads();
  }
  // sign correction
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (M[i * LM + i] < 0.f)
      for (int j = i; j < n; ++j) M[i * LM + j] = -M[i * LM + j];
  }
  __syncthreads();
}

template <int DXP, int DYP>
__global__ void __launch_bounds__(256) srkf_batch_kernel(KfRun run) {
  using SM = SrSmem<DXP, DYP>;
  constexpr int LM = SM::LM, LD = DXP + 1, LY = DYP + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  SM& s = *reinterpret_cast<SM*>(smraw);
  const int G = blockDim.x;
  while (true) {
    if (threadIdx.x == 0) {
      unsigned k = atomicAdd(run.counter, 1u);
      s.fid = k < (unsigned)run.count ? run.order[k] : -1;
    }
    __syncthreads();
    const int f = s.fid;
    if (f < 0) return;
    const KfDesc D = run.desc[f];
    const int dx = D.dx, dy = D.dy;
    const float* P = run.params + D.poff;
    // homogeneous: A | b | Q | H | c | R | mu0 | S0 | UQ | UR | U0; time-varying:
    // step blocks A | b | H | c | UQ | UR (calc_params(., t + 1)), then mu0 | U0
    struct StepPtrs {
      const float *A, *b, *H, *c, *UQ, *UR;
    };
    auto step_ptrs = [&](int t) {
      StepPtrs q;
      if (D.pstep) {
        q.A = P + (int64_t)t * D.pstep;
        q.b = q.A + dx * dx;
        q.H = q.b + dx;
        q.c = q.H + dy * dx;
        q.UQ = q.c + dy;
        q.UR = q.UQ + dx * dx;
      } else {
        q.A = P;
        q.b = q.A + dx * dx;
        q.H = q.b + dx + dx * dx;
        q.c = q.H + dy * dx;
        q.UQ = q.c + dy + dy * dy + dx + dx * dx;
        q.UR = q.UQ + dx * dx;
      }
      return q;
    };
    auto load_step = [&](int t) {  // this step's A, b, H, c and the factors of Q and R
      const StepPtrs q = step_ptrs(t);
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        int i = e % dx, j = e / dx;
        s.A[i * LD + j] = q.A[e];
        s.UQ[i * LD + j] = q.UQ[e];
      }
      for (int e = threadIdx.x; e < dy * dx; e += G) s.H[(e % dy) * LD + e / dy] = q.H[e];
      for (int e = threadIdx.x; e < dy * dy; e += G) s.UR[(e % dy) * LY + e / dy] = q.UR[e];
      for (int e = threadIdx.x; e < dx; e += G) s.b[e] = q.b[e];
      for (int e = threadIdx.x; e < dy; e += G) s.c[e] = q.c[e];
    };
    const float* pm = D.pstep ? P + D.p0 : step_ptrs(0).c + dy + dy * dy;
    const float* pU0 = D.pstep ? pm + dx : step_ptrs(0).UR + dy * dy;
    load_step(0);
    for (int e = threadIdx.x; e < dx * dx; e += G) s.U[(e % dx) * LD + e / dx] = pU0[e];
    for (int e = threadIdx.x; e < dx; e += G) s.mu[e] = pm[e];
    __syncthreads();
    double lltot = 0.0;
    int status = GF_OK;
    for (int t = 0; t < D.T; ++t) {
      const double* y = run.ys + D.yoff + (int64_t)t * dy;
      if (D.pstep && t > 0) {  // time-varying model: step t's parameters
        load_step(t);
        __syncthreads();
      }
      // predict: mu = A mu + b ; U = R(qr([UQ; U A']))
      float mnew = 0.f;
      if (threadIdx.x < dx) {
        int i = threadIdx.x;
        float acc = s.b[i];
        for (int k = 0; k < dx; ++k) acc = fmaf(s.A[i * LD + k], s.mu[k], acc);
        mnew = acc;
      }
      for (int e = threadIdx.x; e < 2 * dx * dx; e += G) {
        int i = e / dx, j = e % dx;
        float v;
        if (i < dx) v = s.UQ[i * LD + j];
        else {
          int r = i - dx;
          float acc = 0.f;
          for (int k = r; k < dx; ++k) acc = fmaf(s.U[r * LD + k], s.A[j * LD + k], acc);
          v = acc;
        }
        s.M[i * LM + j] = v;
      }
      __syncthreads();
      if (threadIdx.x < dx) s.mu[threadIdx.x] = mnew;
      householder_qr<LM>(s.M, 2 * dx, dx, s.colscale, s.red);
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        int i = e / dx, j = e % dx;
        s.U[i * LD + j] = j >= i ? s.M[i * LM + j] : 0.f;
      }
      __syncthreads();
      // update: M = [[UR, 0], [U H', U]]
      const int nn = dx + dy;
      for (int e = threadIdx.x; e < nn * nn; e += G) {
        int i = e / nn, j = e % nn;
        float v = 0.f;
        if (i < dy) v = j < dy ? s.UR[i * LY + j] : 0.f;
        else {
          int r = i - dy;
          if (j < dy) {
            float acc = 0.f;
            for (int k = r; k < dx; ++k) acc = fmaf(s.U[r * LD + k], s.H[j * LD + k], acc);
            v = acc;
          } else {
            v = s.U[r * LD + (j - dy)];
          }
        }
        s.M[i * LM + j] = v;
      }
      for (int i = threadIdx.x; i < dy; i += G) {
        double acc = y[i] - (double)s.c[i];
        for (int k = 0; k < dx; ++k) acc -= (double)s.H[i * LD + k] * (double)s.mu[k];
        s.z[i] = acc;
      }
      __syncthreads();
      householder_qr<LM>(s.M, nn, nn, s.colscale, s.red);
      // w = U_S' \ z (U_S' lower), FP64, warp 0
      if (threadIdx.x == 0) {
        for (int i = 0; i < dy; ++i) {
          double acc = s.z[i];
          for (int k = 0; k < i; ++k) acc -= (double)s.M[k * LM + i] * s.w[k];
          double d = (double)s.M[i * LM + i];
          if (!(d > 0.0)) {
            status = GF_ERR_NOT_PD;
            s.fid = -2;
            break;
          }
          s.w[i] = acc / d;
        }
      }
      __syncthreads();
      if (s.fid == -2) {
        status = GF_ERR_NOT_PD;
        break;
      }
      // mu += PHt w (PHt = R[0:dy, dy:]') ; U = R[dy:, dy:] (+ jitter)
      for (int i = threadIdx.x; i < dx; i += G) {
        double acc = (double)s.mu[i];
        for (int k = 0; k < dy; ++k) acc += (double)s.M[k * LM + dy + i] * s.w[k];
        s.mu[i] = (float)acc;
      }
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        int i = e / dx, j = e % dx;
        float v = j >= i ? s.M[(dy + i) * LM + dy + j] : 0.f;
        if (run.use_jitter && i == j) v += (float)run.jitter;
        s.U[i * LD + j] = v;
      }
      __syncthreads();
      if (run.covs) {
        float* co = run.covs + D.coff + (int64_t)t * dx * dx;
        for (int e = threadIdx.x; e < dx * dx; e += G) {
          int i = e % dx, j = e / dx;  // column-major output of U'U
          float acc = 0.f;
          for (int k = 0; k <= min(i, j); ++k) acc = fmaf(s.U[k * LD + i], s.U[k * LD + j], acc);
          co[e] = acc;
        }
      }
      if (run.means)
        for (int i = threadIdx.x; i < dx; i += G) run.means[D.moff + (int64_t)t * dx + i] = s.mu[i];
      if (threadIdx.x < 32) {
        double q = 0.0, ld = 0.0;
        for (int i = threadIdx.x; i < dy; i += 32) {
          q += s.w[i] * s.w[i];
          ld += log((double)s.M[i * LM + i]);
        }
        q = warp_sum(q);
        ld = warp_sum(ld);
        double l = -0.5 * (q + 2.0 * ld + dy * GF_LOG2PI);
        lltot += l;
        if (threadIdx.x == 0 && run.ll_steps) run.ll_steps[D.soff + t] = l;
        if (threadIdx.x == 0 && D.srv_steps) D.srv_steps[t] = l;
      }
      __syncthreads();
    }
    if (D.srv)
      kf_srv_publish(D, s.mu, [&](int i, int j) {
        float acc = 0.f;
        for (int k = 0; k <= min(i, j); ++k) acc = fmaf(s.U[k * LD + i], s.U[k * LD + j], acc);
        return acc;
      }, lltot, status);
    if (threadIdx.x == 0 && run.ll) {
      run.ll[D.index] = lltot;
      run.status[D.index] = status;
    }
    __syncthreads();
  }
}


// ------------------------------------------------------------ RTS smoother
// smooth(model, KalmanSmoother(), ys) (kalman.jl:206-234): after the forward
// bank wrote the filtered means / covariances of every step (run.means,
// run.covs), one block per filter walks t = T-1 .. 1 and overwrites step t
// with the smoothed distribution (backward_smooth, kalman.jl:89-126):
//   mu_pred = A mu_f + b, Sigma_pred = A Sigma_f A' + Q,
//   G' = Sigma_pred^-1 (A Sigma_f)          (FP64 Cholesky and solves),
//   mu_s = mu_f + G (mu_s' - mu_pred),
//   Sigma_s = Sigma_f + G (Sigma_s' - Sigma_pred) G'   (upper triangle mirrored).
template <int DXP>
struct RtsSmem {
  static constexpr int LD = DXP + 1;
  double Lc[DXP * LD];  // Sigma_pred, then its Cholesky factor (lower)
  double X[DXP * LD];   // right-hand sides A Sigma_f, then G' (row k, column i = G[i][k])
  double dinv[DXP];
  float A[DXP * LD], Q[DXP * LD], Sf[DXP * LD], Sn[DXP * LD], T1[DXP * LD], D[DXP * LD];
  float b[DXP], mf[DXP], mn[DXP], mp[DXP], dd[DXP];
  int fid, fail;
};

template <int DXP>
__global__ void __launch_bounds__(256) rts_smooth_kernel(KfRun run) {
  using SM = RtsSmem<DXP>;
  constexpr int LD = SM::LD;
  extern __shared__ __align__(16) unsigned char smraw[];
  SM& s = *reinterpret_cast<SM*>(smraw);
  const int G = blockDim.x;
  while (true) {
    if (threadIdx.x == 0) {
      unsigned k = atomicAdd(run.counter, 1u);
      s.fid = k < (unsigned)run.count ? run.order[k] : -1;
      s.fail = 0;
    }
    __syncthreads();
    const int f = s.fid;
    if (f < 0) return;
    const KfDesc D = run.desc[f];
    const int dx = D.dx, T = D.T;
    if (run.status[D.index] != GF_OK || T < 2) {
      __syncthreads();
      continue;
    }
    const float* P = run.params + D.poff;  // A dx*dx | b dx | Q dx*dx | ...
    // the parameters of 0-based step k (a time-varying model's block k)
    auto load_params = [&](int k) {
      const float* Pk = P + (int64_t)k * D.pstep;
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        const int i = e % dx, j = e / dx;  // column-major source
        s.A[i * LD + j] = Pk[e];
        s.Q[i * LD + j] = Pk[dx * dx + dx + e];
      }
      for (int e = threadIdx.x; e < dx; e += G) s.b[e] = Pk[dx * dx + e];
    };
    load_params(0);
    for (int e = threadIdx.x; e < dx * dx; e += G)
      s.Sn[(e % dx) * LD + e / dx] = run.covs[D.coff + (int64_t)(T - 1) * dx * dx + e];
    for (int e = threadIdx.x; e < dx; e += G) s.mn[e] = run.means[D.moff + (int64_t)(T - 1) * dx + e];
    __syncthreads();
    for (int t = T - 2; t >= 0; --t) {
      float* cov = run.covs + D.coff + (int64_t)t * dx * dx;
      float* mean = run.means + D.moff + (int64_t)t * dx;
      // the prediction from t to t + 1 uses the parameters of step t + 1
      if (D.pstep) load_params(t + 1);
      for (int e = threadIdx.x; e < dx * dx; e += G) s.Sf[(e % dx) * LD + e / dx] = cov[e];
      for (int e = threadIdx.x; e < dx; e += G) s.mf[e] = mean[e];
      __syncthreads();
      // T1 = A Sigma_f ; mu_pred = A mu_f + b
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        const int i = e / dx, j = e - i * dx;
        float acc = 0.f;
        for (int k = 0; k < dx; ++k) acc = fmaf(s.A[i * LD + k], s.Sf[k * LD + j], acc);
        s.T1[i * LD + j] = acc;
      }
      for (int i = threadIdx.x; i < dx; i += G) {
        float acc = s.b[i];
        for (int k = 0; k < dx; ++k) acc = fmaf(s.A[i * LD + k], s.mf[k], acc);
        s.mp[i] = acc;
      }
      __syncthreads();
      // Sigma_pred = T1 A' + Q (FP64 copy for the Cholesky), D = Sigma_s' - Sigma_pred,
      // right-hand sides X = T1 ; dd = mu_s' - mu_pred
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        const int i = e / dx, j = e - i * dx;
        const int lo = i < j ? i : j, hi = i < j ? j : i;  // upper triangle, mirrored
        float acc = s.Q[lo * LD + hi];
        for (int k = 0; k < dx; ++k) acc = fmaf(s.T1[lo * LD + k], s.A[hi * LD + k], acc);
        s.Lc[i * LD + j] = (double)acc;
        s.D[i * LD + j] = s.Sn[i * LD + j] - acc;
        s.X[i * LD + j] = (double)s.T1[i * LD + j];
      }
      for (int i = threadIdx.x; i < dx; i += G) s.dd[i] = s.mn[i] - s.mp[i];
      __syncthreads();
      // FP64 Cholesky, warp 0, one lane per row (right-looking)
      if (threadIdx.x < 32) {
        const int r = threadIdx.x;
        for (int j = 0; j < dx; ++j) {
          const double djj = s.Lc[j * LD + j];
          if (!(djj > 0.0)) {
            if (r == 0) s.fail = 1;
            break;
          }
          const double dj = sqrt(djj), inv = 1.0 / dj;
          double lrj = 0.0;
          if (r > j && r < dx) {
            lrj = s.Lc[r * LD + j] * inv;
            s.Lc[r * LD + j] = lrj;
          }
          if (r == j) {
            s.Lc[j * LD + j] = dj;
            s.dinv[j] = inv;
          }
          __syncwarp();
          if (r > j && r < dx)
            for (int k = j + 1; k <= r; ++k) s.Lc[r * LD + k] -= lrj * s.Lc[k * LD + j];
          __syncwarp();
        }
      }
      __syncthreads();
      if (s.fail) break;
      // X = Sigma_pred^-1 X: lane = row, warps take interleaved columns
      {
        const int r = threadIdx.x & 31, w = threadIdx.x >> 5, nw = G >> 5;
        for (int i = 0; i < dx; ++i) {
          if (r == i)
            for (int c = w; c < dx; c += nw) s.X[i * LD + c] *= s.dinv[i];
          __syncwarp();
          if (r > i && r < dx) {
            const double l = s.Lc[r * LD + i];
            for (int c = w; c < dx; c += nw) s.X[r * LD + c] -= l * s.X[i * LD + c];
          }
          __syncwarp();
        }
        for (int i = dx - 1; i >= 0; --i) {
          if (r == i)
            for (int c = w; c < dx; c += nw) s.X[i * LD + c] *= s.dinv[i];
          __syncwarp();
          if (r < i) {
            const double l = s.Lc[i * LD + r];
            for (int c = w; c < dx; c += nw) s.X[r * LD + c] -= l * s.X[i * LD + c];
          }
          __syncwarp();
        }
      }
      __syncthreads();
      // mu_s = mu_f + G dd (G[i][k] = X[k][i]) ; T1 = G D
      for (int i = threadIdx.x; i < dx; i += G) {
        double acc = (double)s.mf[i];
        for (int k = 0; k < dx; ++k) acc += s.X[k * LD + i] * (double)s.dd[k];
        s.mn[i] = (float)acc;
      }
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        const int i = e / dx, j = e - i * dx;
        float acc = 0.f;
        for (int k = 0; k < dx; ++k) acc = fmaf((float)s.X[k * LD + i], s.D[k * LD + j], acc);
        s.T1[i * LD + j] = acc;
      }
      __syncthreads();
      // Sigma_s = Sigma_f + T1 G' (upper triangle, mirrored) -> next and output
      for (int e = threadIdx.x; e < dx * dx; e += G) {
        const int i = e / dx, j = e - i * dx;
        if (j < i) continue;
        float acc = s.Sf[i * LD + j];
        for (int k = 0; k < dx; ++k) acc = fmaf(s.T1[i * LD + k], (float)s.X[k * LD + j], acc);
        s.Sn[i * LD + j] = acc;
        s.Sn[j * LD + i] = acc;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < dx * dx; e += G) cov[e] = s.Sn[(e % dx) * LD + e / dx];
      for (int e = threadIdx.x; e < dx; e += G) mean[e] = s.mn[e];
      __syncthreads();
    }
    if (threadIdx.x == 0 && s.fail) run.status[D.index] = GF_ERR_NOT_PD;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- buckets
struct KfBucketKernels {
  int dxp, dyp;
  void (*kf)(KfRun);
  void (*sr)(KfRun);
  size_t kf_smem, sr_smem;
  void (*rts)(KfRun);
  size_t rts_smem;
};

template <int DXP, int DYP>
static KfBucketKernels make_bucket() {
  return {DXP, DYP, kf_batch_kernel<DXP, DYP>, srkf_batch_kernel<DXP, DYP>, sizeof(KfSmem<DXP, DYP>),
          sizeof(SrSmem<DXP, DYP>), rts_smooth_kernel<DXP>, sizeof(RtsSmem<DXP>)};
}

static const std::vector<KfBucketKernels>& kf_buckets() {
  static std::vector<KfBucketKernels> v = {make_bucket<4, 4>(), make_bucket<8, 8>(),
                                           make_bucket<16, 16>(), make_bucket<32, 32>()};
  return v;
}

int kf_bucket_count() { return (int)kf_buckets().size(); }
int kf_bucket_dxp(int kidx) { return kf_buckets()[kidx].dxp; }

int kf_bucket_for(int dx, int dy) {
  const auto& b = kf_buckets();
  for (size_t k = 0; k < b.size(); ++k)
    if (b[k].dxp >= dx && b[k].dyp >= dy) return (int)k;
  return -1;
}

int kf_default_group(int kidx) {
  const int dxp = kf_buckets()[kidx].dxp;
  return dxp <= 8 ? 32 : (dxp <= 16 ? 128 : 256);
}

static const void* kf_fn(int algo, int kidx, size_t* smem) {
  const KfBucketKernels& K = kf_buckets()[kidx];
  *smem = algo == GF_ALGO_KF ? K.kf_smem : K.sr_smem;
  return algo == GF_ALGO_KF ? (const void*)K.kf : (const void*)K.sr;
}

gf_status kf_prepare_bucket(gf_ctx* ctx, int algo, int kidx) {
  size_t smem;
  const void* fn = kf_fn(algo, kidx, &smem);
  GF_CHECK_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return GF_OK;
}

int kf_blocks_per_sm(int algo, int kidx, int group) {
  size_t smem;
  const void* fn = kf_fn(algo, kidx, &smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, group, smem) != cudaSuccess) per_sm = 1;
  return std::max(1, per_sm);
}

void kf_launch(int algo, int kidx, int group, int grid, const KfRun& r, cudaStream_t s) {
  const KfBucketKernels& K = kf_buckets()[kidx];
  if (algo == GF_ALGO_KF) K.kf<<<grid, group, K.kf_smem, s>>>(r);
  else K.sr<<<grid, group, K.sr_smem, s>>>(r);
}

gf_status kf_pack_model(gf_ctx* ctx, int algo, const gf_lg_model& m, int f, std::vector<float>& pool) {
  const int dx = m.dx, dy = m.dy;
  std::vector<double> LQ(dx * dx), LR(dy * dy), L0(dx * dx);
  bool bad = chol_lower(dx, m.Q, LQ.data()) || chol_lower(dy, m.R, LR.data()) ||
             chol_lower(dx, m.Sigma0, L0.data());
  if (bad && algo == GF_ALGO_SRKF) return set_err(ctx, GF_ERR_NOT_PD, "filter %d: Q, R or Sigma0 not PD", f);
  auto put = [&](const double* a, int n) {
    for (int i = 0; i < n; ++i) pool.push_back((float)a[i]);
  };
  auto putT = [&](const std::vector<double>& L, int n) {  // upper factor U = L'
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) pool.push_back((float)L[j + i * n]);
  };
  put(m.A, dx * dx);
  put(m.b, dx);
  put(m.Q, dx * dx);
  put(m.H, dy * dx);
  put(m.c, dy);
  put(m.R, dy * dy);
  put(m.mu0, dx);
  put(m.Sigma0, dx * dx);
  putT(LQ, dx);
  putT(LR, dy);
  putT(L0, dx);
  return GF_OK;
}

}  // namespace gf

using namespace gf;

struct gf_kf_plan {
  gf_ctx* ctx = nullptr;
  int algo = 0;
  int B = 0;
  double jitter = 0.0;
  int use_jitter = 0;
  bool plain = false, use_graph = true;
  std::vector<DevBuf> bufs;
  KfDesc* desc = nullptr;
  int32_t* order = nullptr;
  uint32_t* counters = nullptr;
  float* params = nullptr;
  std::vector<KfDesc> hdesc;
  struct Bucket {
    int kidx;
    int group;  // threads per filter block
    int grid;
    int start, count;  // range in `order`
  };
  std::vector<Bucket> buckets;
  std::vector<int32_t> horder;
  int64_t total_steps = 0, total_means = 0, total_covs = 0;
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> evs;
};

static gf_status kf_alloc(gf_kf_plan* p, size_t bytes, void** out) {
  gf_status st = dev_alloc(p->ctx, bytes, out);
  if (!st && *out) p->bufs.push_back({*out, bytes});
  return st;
}

static void kf_release(gf_kf_plan* p) {
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (auto s : p->side) cudaStreamDestroy(s);
  for (auto e : p->evs) cudaEventDestroy(e);
  for (auto& b : p->bufs) dev_free(p->ctx, b.p, b.bytes);
  p->bufs.clear();
}


static void kf_launch_bucket(gf_kf_plan* p, const gf_kf_plan::Bucket& bk, const KfRun& base,
                             cudaStream_t s) {
  const KfBucketKernels& K = kf_buckets()[bk.kidx];
  KfRun r = base;
  r.order = p->order + bk.start;
  r.count = bk.count;
  r.counter = p->counters + (&bk - p->buckets.data());
  size_t smem = p->algo == GF_ALGO_KF ? K.kf_smem : K.sr_smem;
  ProfScope ps(p->ctx, KC_KF);
  if (p->algo == GF_ALGO_KF) K.kf<<<bk.grid, bk.group, smem, s>>>(r);
  else K.sr<<<bk.grid, bk.group, smem, s>>>(r);
}

static gf_status kf_enqueue(gf_kf_plan* p, const double* ys, gf_kf_out* out) {
  gf_ctx* ctx = p->ctx;
  cudaStream_t s = ctx->stream;
  KfRun base{};
  base.desc = p->desc;
  base.params = p->params;
  base.ys = ys;
  base.ll = out->ll;
  base.ll_steps = out->ll_steps;
  base.means = out->means;
  base.covs = out->covs;
  base.status = out->status;
  base.jitter = p->jitter;
  base.use_jitter = p->use_jitter;
  base.algo = p->algo;
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(p->counters, 0, sizeof(uint32_t) * 64, s));
  if (p->plain) {
    // plain per-filter form: one launch per filter, one block each
    for (auto& bk : p->buckets) {
      for (int q = 0; q < bk.count; ++q) {
        gf_kf_plan::Bucket one = bk;
        one.start = bk.start + q;
        one.count = 1;
        one.grid = 1;
        KfRun r = base;
        r.order = p->order + one.start;
        r.count = 1;
        r.counter = p->counters + 63;
        GF_CHECK_CUDA(ctx, cudaMemsetAsync(p->counters + 63, 0, sizeof(uint32_t), s));
        const KfBucketKernels& K = kf_buckets()[bk.kidx];
        size_t smem = p->algo == GF_ALGO_KF ? K.kf_smem : K.sr_smem;
        ProfScope ps(ctx, KC_KF);
        if (p->algo == GF_ALGO_KF) K.kf<<<1, bk.group, smem, s>>>(r);
        else K.sr<<<1, bk.group, smem, s>>>(r);
      }
    }
    return GF_OK;
  }
  // fork buckets onto side streams so their persistent launches overlap
  const int nb = (int)p->buckets.size();
  if ((int)p->side.size() < nb) {
    while ((int)p->side.size() < nb) {
      cudaStream_t ss;
      cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking);
      p->side.push_back(ss);
    }
    while ((int)p->evs.size() < nb + 1) {
      cudaEvent_t e;
      cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      p->evs.push_back(e);
    }
  }
  GF_CHECK_CUDA(ctx, cudaEventRecord(p->evs[nb], s));
  for (int b = 0; b < nb; ++b) {
    GF_CHECK_CUDA(ctx, cudaStreamWaitEvent(p->side[b], p->evs[nb], 0));
    kf_launch_bucket(p, p->buckets[b], base, b == 0 ? s : p->side[b]);
  }
  for (int b = 1; b < nb; ++b) {
    GF_CHECK_CUDA(ctx, cudaEventRecord(p->evs[b], p->side[b]));
    GF_CHECK_CUDA(ctx, cudaStreamWaitEvent(s, p->evs[b], 0));
  }
  return GF_OK;
}

// ------------------------------------------------------------- autotuner
// Picks the block size (threads per filter) of each dimension bucket by timing
// the candidates on a sample of the bucket (its longest filters, T clipped to
// 64 steps, outputs off); results are cached per (GPU, algorithm, bucket) in
// the file named by GF_AUTOTUNE_CACHE (default ~/.cache/gfb200/kf_autotune.txt).
static std::string autotune_path() {
  const char* e = std::getenv("GF_AUTOTUNE_CACHE");
  if (e && *e) return e;
  const char* h = std::getenv("HOME");
  return std::string(h ? h : "/tmp") + "/.cache/gfb200/kf_autotune.txt";
}
static std::string autotune_key(gf_ctx* ctx, int algo, int dxp) {
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, ctx->device);
  std::string name = prop.name;
  for (auto& c : name)
    if (c == ' ') c = '_';
  return name + "|" + (algo == GF_ALGO_KF ? "kf" : "srkf") + "|" + std::to_string(dxp);
}
static int autotune_lookup(gf_ctx* ctx, int algo, int dxp) {
  std::ifstream f(autotune_path());
  std::string k, want = autotune_key(ctx, algo, dxp);
  int g;
  int found = 0;
  while (f >> k >> g)
    if (k == want && (g == 32 || g == 64 || g == 128 || g == 256)) found = g;
  return found;
}
static void autotune_store(gf_ctx* ctx, int algo, int dxp, int group) {
  std::string path = autotune_path();
  std::string dir = path.substr(0, path.find_last_of('/'));
  std::string cmd = "mkdir -p '" + dir + "'";
  if (std::system(cmd.c_str()) != 0) return;
  std::ofstream f(path, std::ios::app);
  if (f) f << autotune_key(ctx, algo, dxp) << " " << group << "\n";
}

static gf_status kf_autotune_bucket(gf_kf_plan* p, gf_kf_plan::Bucket& bk) {
  gf_ctx* ctx = p->ctx;
  const KfBucketKernels& K = kf_buckets()[bk.kidx];
  const size_t smem = p->algo == GF_ALGO_KF ? K.kf_smem : K.sr_smem;
  const void* fn = p->algo == GF_ALGO_KF ? (const void*)K.kf : (const void*)K.sr;
  const int sample = std::min(bk.count, 2 * ctx->num_sms * 4);
  std::vector<KfDesc> td(sample);
  std::vector<int32_t> ord(sample);
  int maxdy = 1;
  for (int q = 0; q < sample; ++q) {
    td[q] = p->hdesc[p->horder[bk.start + q]];
    td[q].T = std::min(td[q].T, 64);
    td[q].yoff = 0;
    td[q].soff = td[q].moff = td[q].coff = 0;
    td[q].index = q;
    ord[q] = q;
    maxdy = std::max(maxdy, td[q].dy);
  }
  void *ddesc = nullptr, *dord = nullptr, *dys = nullptr, *dll = nullptr, *dst = nullptr, *dcnt = nullptr;
  std::vector<DevBuf> tmp;
  auto get = [&](size_t b, void** d) -> gf_status {
    gf_status s2 = dev_alloc(ctx, b, d);
    if (!s2 && *d) tmp.push_back({*d, b});
    return s2;
  };
  struct Free {
    gf_ctx* c;
    std::vector<DevBuf>* v;
    ~Free() {
      cudaStreamSynchronize(c->stream);
      for (auto& b : *v) dev_free(c, b.p, b.bytes);
    }
  } fr{ctx, &tmp};
  gf_status st;
  if ((st = get(sizeof(KfDesc) * sample, &ddesc)) || (st = get(sizeof(int32_t) * sample, &dord)) ||
      (st = get(sizeof(double) * 64 * maxdy, &dys)) || (st = get(sizeof(double) * sample, &dll)) ||
      (st = get(sizeof(int32_t) * sample, &dst)) || (st = get(sizeof(uint32_t), &dcnt)))
    return st;
  cudaStream_t s = ctx->stream;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(ddesc, td.data(), sizeof(KfDesc) * sample, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dord, ord.data(), sizeof(int32_t) * sample, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(dys, 0, sizeof(double) * 64 * maxdy, s));
  KfRun r{};
  r.desc = (const KfDesc*)ddesc;
  r.order = (const int32_t*)dord;
  r.count = sample;
  r.counter = (uint32_t*)dcnt;
  r.params = p->params;
  r.ys = (const double*)dys;
  r.ll = (double*)dll;
  r.status = (int32_t*)dst;
  r.algo = p->algo;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_g = bk.group;
  for (int g : {32, 64, 128, 256}) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, g, smem);
    if (per_sm < 1) continue;
    const int grid = std::max(1, std::min(sample, per_sm * ctx->num_sms));
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      cudaMemsetAsync(dcnt, 0, sizeof(uint32_t), s);
      cudaEventRecord(e0, s);
      if (p->algo == GF_ALGO_KF) K.kf<<<grid, g, smem, s>>>(r);
      else K.sr<<<grid, g, smem, s>>>(r);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
    }
    if (cudaGetLastError() != cudaSuccess) continue;
    if (ms < best) {
      best = ms;
      best_g = g;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  bk.group = best_g;
  return GF_OK;
}

// A time-varying model's pool entry: T step blocks (A b Q H c R) then mu0, S0;
// for the SRKF T blocks (A b H c UQ UR) then mu0, U0 (upper Cholesky factors).
static gf_status kf_pack_model_tv(gf_ctx* ctx, int algo, const gf_lg_model& m, int f, int T,
                                  std::vector<float>& pool) {
  const int dx = m.dx, dy = m.dy;
  std::vector<double> L(std::max(dx, dy) * std::max(dx, dy));
  if (chol_lower(dx, m.Sigma0, L.data())) return set_err(ctx, GF_ERR_NOT_PD, "filter %d: Sigma0 not PD", f);
  auto put = [&](const double* a, int64_t n) {
    for (int64_t i = 0; i < n; ++i) pool.push_back((float)a[i]);
  };
  auto putU = [&](int n) {  // upper factor U = L' of the last chol_lower, column-major
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) pool.push_back((float)L[j + i * n]);
  };
  if (algo == GF_ALGO_SRKF) {
    for (int t = 0; t < T; ++t) {
      put(m.A + (size_t)t * dx * dx, (int64_t)dx * dx);
      put(m.b + (size_t)t * dx, dx);
      put(m.H + (size_t)t * dy * dx, (int64_t)dy * dx);
      put(m.c + (size_t)t * dy, dy);
      if (chol_lower(dx, m.Q + (size_t)t * dx * dx, L.data()))
        return set_err(ctx, GF_ERR_NOT_PD, "filter %d: Q of step %d not PD", f, t + 1);
      putU(dx);
      if (chol_lower(dy, m.R + (size_t)t * dy * dy, L.data()))
        return set_err(ctx, GF_ERR_NOT_PD, "filter %d: R of step %d not PD", f, t + 1);
      putU(dy);
    }
    put(m.mu0, dx);
    chol_lower(dx, m.Sigma0, L.data());
    putU(dx);
    return GF_OK;
  }
  for (int t = 0; t < T; ++t) {
    if (chol_lower(dy, m.R + (size_t)t * dy * dy, L.data()))
      return set_err(ctx, GF_ERR_NOT_PD, "filter %d: R of step %d not PD", f, t + 1);
    put(m.A + (size_t)t * dx * dx, (int64_t)dx * dx);
    put(m.b + (size_t)t * dx, dx);
    put(m.Q + (size_t)t * dx * dx, (int64_t)dx * dx);
    put(m.H + (size_t)t * dy * dx, (int64_t)dy * dx);
    put(m.c + (size_t)t * dy, dy);
    put(m.R + (size_t)t * dy * dy, (int64_t)dy * dy);
  }
  put(m.mu0, dx);
  put(m.Sigma0, (int64_t)dx * dx);
  return GF_OK;
}

static gf_status kf_plan_create_impl(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                                     const int32_t* T, const int32_t* param_steps, double jitter,
                                     int32_t use_jitter, int32_t flags, gf_kf_plan** out) {
  if (!ctx || !out || !models || !T || B < 1) return ctx ? set_err(ctx, GF_ERR_ARG, "bad arguments") : GF_ERR_ARG;
  if (algo != GF_ALGO_KF && algo != GF_ALGO_SRKF) return set_err(ctx, GF_ERR_ARG, "unknown algo");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  auto p = std::make_unique<gf_kf_plan>();
  p->ctx = ctx;
  p->algo = algo;
  p->B = B;
  p->jitter = jitter;
  p->use_jitter = use_jitter;
  p->plain = (flags & GF_PLAN_PLAIN) != 0;
  p->use_graph = !(flags & GF_PLAN_NO_GRAPH) && !p->plain;
  const auto& bks = kf_buckets();
  // descriptors + parameter pool (FP32)
  std::vector<float> pool;
  std::vector<std::vector<int32_t>> members(bks.size());
  p->hdesc.resize(B);
  int64_t poff = 0, yoff = 0, soff = 0, moff = 0, coff = 0;
  for (int f = 0; f < B; ++f) {
    const gf_lg_model& m = models[f];
    if (m.dx < 1 || m.dy < 1 || T[f] < 1) return set_err(ctx, GF_ERR_DIM, "filter %d: bad dims/T", f);
    const int kidx = kf_bucket_for(m.dx, m.dy);
    if (kidx < 0) return set_err(ctx, GF_ERR_DIM, "filter %d: dx=%d dy=%d exceeds 32", f, m.dx, m.dy);
    members[kidx].push_back(f);
    KfDesc& d = p->hdesc[f];
    std::memset(&d, 0, sizeof d);
    d.dx = m.dx;
    d.dy = m.dy;
    d.T = T[f];
    d.poff = poff;
    d.yoff = yoff;
    d.soff = soff;
    d.moff = moff;
    d.coff = coff;
    d.index = f;
    const int dx = m.dx, dy = m.dy;
    const int ps = param_steps ? param_steps[f] : 1;
    if (ps != 1 && ps < T[f])
      return set_err(ctx, GF_ERR_ARG, "filter %d: %d parameter steps for T = %d", f, ps, T[f]);
    if (ps != 1) {
      gf_status pst = kf_pack_model_tv(ctx, algo, m, f, T[f], pool);
      if (pst) return pst;
      d.pstep = algo == GF_ALGO_SRKF ? sr_step_block_len(dx, dy) : kf_step_block_len(dx, dy);
      d.p0 = T[f] * d.pstep;
      poff += (int64_t)d.p0 + dx + (int64_t)dx * dx;
    } else {
      gf_status pst = kf_pack_model(ctx, algo, m, f, pool);
      if (pst) return pst;
      poff += kf_param_len(dx, dy);
    }
    yoff += (int64_t)T[f] * dy;
    soff += T[f];
    moff += (int64_t)T[f] * dx;
    coff += (int64_t)T[f] * dx * dx;
  }
  p->total_steps = soff;
  p->total_means = moff;
  p->total_covs = coff;
  // buckets: longest filters first (largest T*dx^3 first keeps the tail short)
  for (size_t k = 0; k < bks.size(); ++k) {
    auto& mem = members[k];
    if (mem.empty()) continue;
    std::stable_sort(mem.begin(), mem.end(), [&](int a, int b) {
      const KfDesc &da = p->hdesc[a], &db = p->hdesc[b];
      double ca = (double)da.T * da.dx * da.dx * (da.dx + da.dy);
      double cb = (double)db.T * db.dx * db.dx * (db.dx + db.dy);
      return ca > cb;
    });
    gf_kf_plan::Bucket bk;
    bk.kidx = (int)k;
    bk.group = kf_default_group((int)k);
    bk.start = (int)p->horder.size();
    bk.count = (int)mem.size();
    p->horder.insert(p->horder.end(), mem.begin(), mem.end());
    p->buckets.push_back(bk);
  }
  gf_status st;
  void* v;
  if ((st = kf_alloc(p.get(), sizeof(KfDesc) * B, &v))) { kf_release(p.get()); return st; }
  p->desc = (KfDesc*)v;
  if ((st = kf_alloc(p.get(), sizeof(int32_t) * B, &v))) { kf_release(p.get()); return st; }
  p->order = (int32_t*)v;
  if ((st = kf_alloc(p.get(), sizeof(uint32_t) * 64, &v))) { kf_release(p.get()); return st; }
  p->counters = (uint32_t*)v;
  if ((st = kf_alloc(p.get(), sizeof(float) * pool.size(), &v))) { kf_release(p.get()); return st; }
  p->params = (float*)v;
  cudaStream_t s = ctx->stream;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->desc, p->hdesc.data(), sizeof(KfDesc) * B, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->order, p->horder.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->params, pool.data(), sizeof(float) * pool.size(), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  for (auto& bk : p->buckets) {
    const KfBucketKernels& K = bks[bk.kidx];
    size_t smem = algo == GF_ALGO_KF ? K.kf_smem : K.sr_smem;
    const void* fn = algo == GF_ALGO_KF ? (const void*)K.kf : (const void*)K.sr;
    GF_CHECK_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int cached = (flags & GF_PLAN_AUTOTUNE) ? autotune_lookup(ctx, algo, bks[bk.kidx].dxp) : 0;
    if (cached) bk.group = cached;
    else if (flags & GF_PLAN_AUTOTUNE) {
      if ((st = kf_autotune_bucket(p.get(), bk))) {
        kf_release(p.get());
        return st;
      }
      autotune_store(ctx, algo, bks[bk.kidx].dxp, bk.group);
    }
    int per_sm = 0;
    GF_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bk.group, smem));
    bk.grid = std::max(1, std::min(bk.count, per_sm * ctx->num_sms));
  }
  *out = p.release();
  return GF_OK;
}

extern "C" gf_status gf_kf_plan_create(gf_ctx* ctx, int32_t algo, const gf_lg_model* models,
                                       int32_t B, const int32_t* T, double jitter,
                                       int32_t use_jitter, int32_t flags, gf_kf_plan** out) {
  return kf_plan_create_impl(ctx, algo, models, B, T, nullptr, jitter, use_jitter, flags, out);
}

extern "C" gf_status gf_kf_plan_create_tv(gf_ctx* ctx, int32_t algo, const gf_lg_model* models,
                                          int32_t B, const int32_t* T, const int32_t* param_steps,
                                          double jitter, int32_t use_jitter, int32_t flags,
                                          gf_kf_plan** out) {
  return kf_plan_create_impl(ctx, algo, models, B, T, param_steps, jitter, use_jitter, flags, out);
}

extern "C" gf_status gf_kf_plan_run(gf_kf_plan* p, const double* ys_dev, gf_kf_out* out) {
  if (!p || !ys_dev || !out || !out->ll || !out->status)
    return p ? set_err(p->ctx, GF_ERR_ARG, "ys, out->ll and out->status are required") : GF_ERR_ARG;
  gf_ctx* ctx = p->ctx;
  cudaSetDevice(ctx->device);
  const void* key[5] = {ys_dev, out->ll, out->ll_steps, out->means, out->covs};
  if (p->use_graph && !ctx->profiling) {
    bool same = p->graph && std::equal(key, key + 5, p->graph_key);
    same = same && out->status == nullptr ? false : same;
    if (!p->graph || !std::equal(key, key + 5, p->graph_key)) {
      if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
      }
      cudaGraph_t g;
      GF_CHECK_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      gf_status st = kf_enqueue(p, ys_dev, out);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      if (st) return st;
      if (e != cudaSuccess) return cuda_err(ctx, e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&p->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_err(ctx, e, "cudaGraphInstantiate");
      std::copy(key, key + 5, p->graph_key);
    }
    GF_CHECK_CUDA(ctx, cudaGraphLaunch(p->graph, ctx->stream));
    return GF_OK;
  }
  gf_status st = kf_enqueue(p, ys_dev, out);
  if (st) return st;
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  return GF_OK;
}

extern "C" gf_status gf_kf_plan_destroy(gf_kf_plan* p) {
  if (!p) return GF_OK;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  kf_release(p);
  delete p;
  return GF_OK;
}

// RTS backward pass of every bucket over the filtered outputs in `out` (device).
static gf_status kf_smooth_enqueue(gf_kf_plan* p, const gf_kf_out* out) {
  gf_ctx* ctx = p->ctx;
  cudaStream_t s = ctx->stream;
  KfRun r{};
  r.desc = p->desc;
  r.params = p->params;
  r.means = out->means;
  r.covs = out->covs;
  r.status = out->status;
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(p->counters, 0, sizeof(uint32_t) * 64, s));
  for (size_t b = 0; b < p->buckets.size(); ++b) {
    const auto& bk = p->buckets[b];
    const KfBucketKernels& K = kf_buckets()[bk.kidx];
    GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)K.rts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)K.rts_smem));
    KfRun rb = r;
    rb.order = p->order + bk.start;
    rb.count = bk.count;
    rb.counter = p->counters + b;
    const int group = K.dxp <= 8 ? 32 : 128;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)K.rts, group, K.rts_smem);
    const int grid = std::max(1, std::min(bk.count, std::max(1, per_sm) * ctx->num_sms));
    ProfScope ps(ctx, KC_KF);
    K.rts<<<grid, group, K.rts_smem, s>>>(rb);
  }
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  return GF_OK;
}

static gf_status kf_batch_impl(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                               const int32_t* T, const int32_t* param_steps, const double* ys,
                               double jitter, int32_t use_jitter, int32_t memspace, gf_kf_out* out,
                               bool smooth) {
  if (!ctx || !out || !ys) return ctx ? set_err(ctx, GF_ERR_ARG, "null argument") : GF_ERR_ARG;
  if (smooth && (!out->means || !out->covs))
    return set_err(ctx, GF_ERR_ARG, "smoothing needs out->means and out->covs");
  gf_kf_plan* p = nullptr;
  gf_status st = kf_plan_create_impl(ctx, algo, models, B, T, param_steps, jitter, use_jitter,
                                     GF_PLAN_NO_GRAPH, &p);
  if (st) return st;
  std::unique_ptr<gf_kf_plan, gf_status (*)(gf_kf_plan*)> guard(p, gf_kf_plan_destroy);
  if (memspace == GF_MEM_DEVICE) {
    if (!out->status) return set_err(ctx, GF_ERR_ARG, "out->status is required");
    if ((st = gf_kf_plan_run(p, ys, out))) return st;
    return smooth ? kf_smooth_enqueue(p, out) : GF_OK;
  }
  // stage host buffers
  int64_t ny = 0;
  for (int f = 0; f < B; ++f) ny += (int64_t)T[f] * models[f].dy;
  cudaStream_t s = ctx->stream;
  std::vector<DevBuf> tmp;
  auto get = [&](size_t bytes, void** d) -> gf_status {
    gf_status s2 = dev_alloc(ctx, bytes, d);
    if (!s2 && *d) tmp.push_back({*d, bytes});
    return s2;
  };
  struct Cleanup {
    gf_ctx* c;
    std::vector<DevBuf>* v;
    ~Cleanup() {
      cudaStreamSynchronize(c->stream);
      for (auto& b : *v) dev_free(c, b.p, b.bytes);
    }
  } cleanup{ctx, &tmp};
  void *d_ys, *d_ll, *d_steps = nullptr, *d_means = nullptr, *d_covs = nullptr, *d_status;
  if ((st = get(sizeof(double) * ny, &d_ys))) return st;
  if ((st = get(sizeof(double) * B, &d_ll))) return st;
  if ((st = get(sizeof(int32_t) * B, &d_status))) return st;
  if (out->ll_steps && (st = get(sizeof(double) * p->total_steps, &d_steps))) return st;
  if (out->means && (st = get(sizeof(float) * p->total_means, &d_means))) return st;
  if (out->covs && (st = get(sizeof(float) * p->total_covs, &d_covs))) return st;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(d_ys, ys, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
  gf_kf_out d{(double*)d_ll, (double*)d_steps, (float*)d_means, (float*)d_covs, (int32_t*)d_status};
  if ((st = gf_kf_plan_run(p, (const double*)d_ys, &d))) return st;
  if (smooth && (st = kf_smooth_enqueue(p, &d))) return st;
  if (out->ll) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->ll, d_ll, sizeof(double) * B, cudaMemcpyDeviceToHost, s));
  std::vector<int32_t> hs(B);
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(hs.data(), d_status, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, s));
  if (d_steps) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->ll_steps, d_steps, sizeof(double) * p->total_steps, cudaMemcpyDeviceToHost, s));
  if (d_means) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->means, d_means, sizeof(float) * p->total_means, cudaMemcpyDeviceToHost, s));
  if (d_covs) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->covs, d_covs, sizeof(float) * p->total_covs, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (out->status) std::memcpy(out->status, hs.data(), sizeof(int32_t) * B);
  for (int f = 0; f < B; ++f)
    if (hs[f] != GF_OK) return set_err(ctx, hs[f], "filter %d failed with status %d (S not positive definite)", f, hs[f]);
  return GF_OK;
}

extern "C" gf_status gf_kf_batch(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                                 const int32_t* T, const double* ys, double jitter,
                                 int32_t use_jitter, int32_t memspace, gf_kf_out* out) {
  return kf_batch_impl(ctx, algo, models, B, T, nullptr, ys, jitter, use_jitter, memspace, out, false);
}

extern "C" gf_status gf_kf_smooth(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                                  const double* ys, int32_t memspace, gf_kf_out* out) {
  return kf_batch_impl(ctx, GF_ALGO_KF, models, B, T, nullptr, ys, 0.0, 0, memspace, out, true);
}

extern "C" gf_status gf_kf_batch_tv(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                                    const int32_t* T, const int32_t* param_steps, const double* ys,
                                    double jitter, int32_t use_jitter, int32_t memspace,
                                    gf_kf_out* out) {
  return kf_batch_impl(ctx, algo, models, B, T, param_steps, ys, jitter, use_jitter, memspace, out, false);
}

extern "C" gf_status gf_kf_smooth_tv(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                                     const int32_t* param_steps, const double* ys, int32_t memspace,
                                     gf_kf_out* out) {
  return kf_batch_impl(ctx, GF_ALGO_KF, models, B, T, param_steps, ys, 0.0, 0, memspace, out, true);
}

extern "C" gf_status gf_kf_plan_smooth(gf_kf_plan* p, const double* ys_dev, gf_kf_out* out) {
  if (!p || !ys_dev || !out || !out->ll || !out->status || !out->means || !out->covs)
    return p ? set_err(p->ctx, GF_ERR_ARG, "ys, out->ll, status, means and covs are required") : GF_ERR_ARG;
  if (p->algo != GF_ALGO_KF || p->use_jitter)
    return set_err(p->ctx, GF_ERR_ARG, "smoothing runs on a KalmanFilter() plan without jitter");
  gf_status st = gf_kf_plan_run(p, ys_dev, out);
  if (st) return st;
  return kf_smooth_enqueue(p, out);
}
