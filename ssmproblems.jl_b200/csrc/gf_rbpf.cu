// gf_rbpf.cu -- Rao-Blackwellised particle filter: per-particle Kalman banks.
//
// Restates rbpf.jl:16-84 on a conditionally linear-Gaussian HierarchicalSSM
// (models/hierarchical.jl:4-50).  Each thread owns one particle: the outer
// sample x (dxo), and the inner Gaussian N(mu, Sigma) (dz, Sigma packed upper).
// Per step: [ancestor gather] -> outer propagate (BF or overdispersed
// proposal, particles.jl:175-245) -> inner KF predict with prev_outer/new_outer
// (kalman.jl:42-49) -> inner KF update (kalman_gradient.jl:12-23, Joseph form)
// whose ll is the particle's log-weight increment.  The resampling, LSE/ESS
// reduction and lookback scan are the shared particle-filter kernels.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "gf_internal.hpp"
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"

namespace gf {

template <int DXO, int DZ, int DY>
struct RbLayout {
  static constexpr int NS = DZ * (DZ + 1) / 2;  // packed upper triangle
  static constexpr int WIDTH = DXO + DZ + NS;
  // params (float): Ao | bo | Lo | Lq | LQi | Az | bz | Cz | Qz(packed) | H | c | R | mu_o | L0o | mu_z | S0z(packed)
  static constexpr int Ao = 0, bo = Ao + DXO * DXO, Lo = bo + DXO, Lq = Lo + DXO * DXO,
                       LQi = Lq + DXO * DXO, Az = LQi + DXO * DXO, bz = Az + DZ * DZ,
                       Cz = bz + DZ, Qz = Cz + DZ * DXO, H = Qz + NS, c = H + DY * DZ,
                       R = c + DY, muo = R + DY * DY, L0o = muo + DXO, muz = L0o + DXO * DXO,
                       S0z = muz + DZ, total = S0z + NS;
};

__host__ __device__ constexpr int pk(int i, int j, int n) {  // packed upper index, i <= j
  return i * n - i * (i - 1) / 2 + (j - i);
}

static_assert(RB_SPLIT * RB_THREADS == PF_TILE, "RBPF blocks must tile a propagate tile exactly");
static_assert(RB_SPLIT <= PF_MAX_SPLIT, "part buffers hold PF_MAX_SPLIT partials per tile");

// Inner KF predict of one particle (kalman.jl:42-49 with prev_outer x and
// new_outer xn, rbpf.jl:45-55): mp = Az mu + bz + Cz x and the packed upper
// Sp = Az S Az' + Qz exp(gamma xn[q_index]).
template <int DXO, int DZ, int DY>
__device__ __forceinline__ void rb_inner_predict(const float* sp, const float (&x)[DXO], const float (&xn)[DXO],
                                                 float q_gamma, int q_index, const float (&mu)[DZ],
                                                 const float (&S)[DZ * (DZ + 1) / 2], float (&mp)[DZ],
                                                 float (&Sp)[DZ * (DZ + 1) / 2]) {
  using L = RbLayout<DXO, DZ, DY>;
#pragma unroll
  for (int r = 0; r < DZ; ++r) {
    float v = sp[L::bz + r];
#pragma unroll
    for (int c = 0; c < DXO; ++c) v = fmaf(sp[L::Cz + c * DZ + r], x[c], v);
#pragma unroll
    for (int c = 0; c < DZ; ++c) v = fmaf(sp[L::Az + c * DZ + r], mu[c], v);
    mp[r] = v;
  }
  const float qs = q_gamma != 0.f ? __expf(q_gamma * xn[q_index]) : 1.f;
  // T = Az S (row r), then Sp[r][j] = T_r . Az[j,:] for j >= r
#pragma unroll
  for (int r = 0; r < DZ; ++r) {
    float Tr[DZ];
#pragma unroll
    for (int k = 0; k < DZ; ++k) {
      float v = 0.f;
#pragma unroll
      for (int m = 0; m < DZ; ++m) {
        const float Smk = m <= k ? S[pk(m, k, DZ)] : S[pk(k, m, DZ)];
        v = fmaf(sp[L::Az + m * DZ + r], Smk, v);
      }
      Tr[k] = v;
    }
#pragma unroll
    for (int j = r; j < DZ; ++j) {
      float v = sp[L::Qz + pk(r, j, DZ)] * qs;
#pragma unroll
      for (int k = 0; k < DZ; ++k) v = fmaf(Tr[k], sp[L::Az + k * DZ + j], v);
      Sp[pk(r, j, DZ)] = v;
    }
  }
}

// Innovation of the inner update (kalman_gradient.jl:12-23): PHt = Sp H' and
// the FP64 Cholesky factor (lower, in place) of S = H Sp H' + R.  Returns
// false if S is not positive definite.
template <int DXO, int DZ, int DY>
__device__ __forceinline__ bool rb_innovation(const float* sp, const float (&Sp)[DZ * (DZ + 1) / 2],
                                              float (&PHt)[DZ][DY], double (&Sd)[DY][DY]) {
  using L = RbLayout<DXO, DZ, DY>;
#pragma unroll
  for (int r = 0; r < DZ; ++r)
#pragma unroll
    for (int j = 0; j < DY; ++j) {
      float v = 0.f;
#pragma unroll
      for (int k = 0; k < DZ; ++k) {
        const float Srk = r <= k ? Sp[pk(r, k, DZ)] : Sp[pk(k, r, DZ)];
        v = fmaf(Srk, sp[L::H + k * DY + j], v);
      }
      PHt[r][j] = v;
    }
#pragma unroll
  for (int i2 = 0; i2 < DY; ++i2)
#pragma unroll
    for (int j = 0; j <= i2; ++j) {
      double v = (double)sp[L::R + j * DY + i2];
#pragma unroll
      for (int k = 0; k < DZ; ++k) v += (double)sp[L::H + k * DY + i2] * (double)PHt[k][j];
      Sd[i2][j] = v;
    }
  bool pd = true;
#pragma unroll
  for (int j = 0; j < DY; ++j) {
    double d = Sd[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= Sd[j][k] * Sd[j][k];
    pd = pd && (d > 0.0);
    d = sqrt(fmax(d, 1e-300));
    Sd[j][j] = d;
#pragma unroll
    for (int i2 = j + 1; i2 < DY; ++i2) {
      double v = Sd[i2][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= Sd[i2][k] * Sd[j][k];
      Sd[i2][j] = v / d;
    }
  }
  return pd;
}

// Whitened innovation w = L^-1 (y - H mp - c), its squared norm and
// log det L: the update's log-likelihood is -(qf + 2 ldet + dy log 2 pi) / 2.
template <int DXO, int DZ, int DY>
__device__ __forceinline__ void rb_whiten(const float* sp, const double* sy, const float (&mp)[DZ],
                                          const double (&Sd)[DY][DY], double (&w)[DY], double& qf,
                                          double& ldet) {
  using L = RbLayout<DXO, DZ, DY>;
  qf = 0.0;
  ldet = 0.0;
#pragma unroll
  for (int i2 = 0; i2 < DY; ++i2) {
    double v = sy[i2] - (double)sp[L::c + i2];
#pragma unroll
    for (int k = 0; k < DZ; ++k) v -= (double)sp[L::H + k * DY + i2] * (double)mp[k];
#pragma unroll
    for (int k = 0; k < i2; ++k) v -= Sd[i2][k] * w[k];
    w[i2] = v / Sd[i2][i2];
    qf += w[i2] * w[i2];
    ldet += log(Sd[i2][i2]);
  }
}

// One particle per thread: a particle's Kalman update needs ~250 registers, so
// a 1024-particle tile is spread over RB_SPLIT blocks of RB_THREADS threads
// (grid = RB_SPLIT * tiles) to keep every SM busy at moderate N.
template <int DXO, int DZ, int DY>
__global__ void __launch_bounds__(RB_THREADS) rbpf_propagate(const PfJob* __restrict__ jobs, int njobs,
                                                            float q_gamma, int q_index, int guided) {
  using L = RbLayout<DXO, DZ, DY>;
  constexpr int NS = L::NS;
  __shared__ float sp[L::total];
  __shared__ double sy[DY];
  __shared__ double red[32];
  const int jb = find_job(jobs, njobs, blockIdx.x / RB_SPLIT, false);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const int tile = blockIdx.x / RB_SPLIT - J.tile0;
  const int part = blockIdx.x % RB_SPLIT;
  const bool resamp = sc->resample != 0;
  const bool fresh = resamp || sc->uniform != 0;
  const double lse_prev = sc->lse;
  const bool searched = J.resampler == GF_RS_MULTINOMIAL;
  // step t's parameter block (time-varying models: calc_params(., t)), else the one block
  const float* P = reinterpret_cast<const float*>(J.params) + (size_t)(t - 1) * J.pstride;
  for (int k = threadIdx.x; k < L::total; k += RB_THREADS) sp[k] = P[k];
  if (threadIdx.x < DY) sy[threadIdx.x] = J.ys[(size_t)(t - 1) * DY + threadIdx.x];
  __syncthreads();
  const int64_t N = J.N;
  const float* Xs = reinterpret_cast<const float*>(J.X[(t - 1) & 1]);
  float* Xd = reinterpret_cast<float*>(J.X[t & 1]);
  float* lw = reinterpret_cast<float*>(J.lw);
  const float* noise = J.noise ? reinterpret_cast<const float*>(J.noise) + (size_t)t * DXO * N : nullptr;
  // auxiliary filter: after a resample the new weights are -log eta[a]
  const float* eta = reinterpret_cast<const float*>(J.eta);
  const bool apf = resamp && eta != nullptr;
  LseAcc acc;
  int fail = 0;
  for (int p = 0; p < 1; ++p) {
    const int64_t i = (int64_t)tile * PF_TILE + part * RB_THREADS + threadIdx.x;
    if (i >= N) break;
    int64_t a = i;
    if (resamp) a = searched ? find_ancestor(J, sc, t, i, 0, N) : (int64_t)J.anc[i];
    float x[DXO], mu[DZ], S[NS];
#pragma unroll
    for (int d = 0; d < DXO; ++d) x[d] = Xs[(size_t)d * N + a];
#pragma unroll
    for (int d = 0; d < DZ; ++d) mu[d] = Xs[(size_t)(DXO + d) * N + a];
#pragma unroll
    for (int d = 0; d < NS; ++d) S[d] = Xs[(size_t)(DXO + DZ + d) * N + a];
    const double lin = !fresh ? (double)lw[i] - lse_prev : apf ? -(double)eta[a] : 0.0;
    // ---- outer propagate
    float e[DXO];
    if (noise) {
#pragma unroll
      for (int d = 0; d < DXO; ++d) e[d] = noise[(size_t)d * N + i];
    } else {
#pragma unroll
      for (int q = 0; q < (DXO + 3) / 4; ++q) {
        float tmp[4];
        philox_normals4<float>(J.seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, tmp);
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (4 * q + r < DXO) e[4 * q + r] = tmp[r];
      }
    }
    float xn[DXO];
    const float* Lf = guided ? sp + L::Lq : sp + L::Lo;
#pragma unroll
    for (int r = 0; r < DXO; ++r) {
      float v = sp[L::bo + r];
#pragma unroll
      for (int c = 0; c < DXO; ++c) v = fmaf(sp[L::Ao + c * DXO + r], x[c], v);
#pragma unroll
      for (int c = 0; c <= r; ++c) v = fmaf(Lf[c * DXO + r], e[c], v);
      xn[r] = v;
    }
    double inc = 0.0;
    if (guided) {
      // log p(x'|x) - log q(x'|x) with x' - (A x + b) = Lq e (particles.jl:175-195)
      float res[DXO], qz = 0.f, qe = 0.f;
#pragma unroll
      for (int r = 0; r < DXO; ++r) {
        float d = 0.f;
#pragma unroll
        for (int c = 0; c <= r; ++c) d = fmaf(sp[L::Lq + c * DXO + r], e[c], d);
        res[r] = d;
        qe = fmaf(e[r], e[r], qe);
      }
#pragma unroll
      for (int r = 0; r < DXO; ++r) {
        float z = 0.f;
#pragma unroll
        for (int c = 0; c <= r; ++c) z = fmaf(sp[L::LQi + c * DXO + r], res[c], z);
        qz = fmaf(z, z, qz);
      }
      inc = -0.5 * (double)qz + 0.5 * (double)qe + J.prop_const;
    }
    // ---- inner predict, then the update's innovation and log-likelihood
    float mp[DZ], Sp[NS];
    rb_inner_predict<DXO, DZ, DY>(sp, x, xn, q_gamma, q_index, mu, S, mp, Sp);
    float PHt[DZ][DY];
    double Sd[DY][DY];
    if (!rb_innovation<DXO, DZ, DY>(sp, Sp, PHt, Sd)) fail = 1;
    double w[DY], ldet, qf;
    rb_whiten<DXO, DZ, DY>(sp, sy, mp, Sd, w, qf, ldet);
    // K = PHt S^-1: rows solve L L' k' = PHt_r'
    float K[DZ][DY];
#pragma unroll
    for (int r = 0; r < DZ; ++r) {
      double v[DY];
#pragma unroll
      for (int i2 = 0; i2 < DY; ++i2) {
        double s2 = (double)PHt[r][i2];
#pragma unroll
        for (int k = 0; k < i2; ++k) s2 -= Sd[i2][k] * v[k];
        v[i2] = s2 / Sd[i2][i2];
      }
#pragma unroll
      for (int i2 = DY - 1; i2 >= 0; --i2) {
        double s2 = v[i2];
#pragma unroll
        for (int k = i2 + 1; k < DY; ++k) s2 -= Sd[k][i2] * v[k];
        v[i2] = s2 / Sd[i2][i2];
      }
#pragma unroll
      for (int i2 = 0; i2 < DY; ++i2) K[r][i2] = (float)v[i2];
    }
    // mu = mp + K z
    {
      double z[DY];
#pragma unroll
      for (int i2 = 0; i2 < DY; ++i2) {
        double zi = sy[i2] - (double)sp[L::c + i2];
#pragma unroll
        for (int k = 0; k < DZ; ++k) zi -= (double)sp[L::H + k * DY + i2] * (double)mp[k];
        z[i2] = zi;
      }
#pragma unroll
      for (int r = 0; r < DZ; ++r) {
        double v = (double)mp[r];
#pragma unroll
        for (int i2 = 0; i2 < DY; ++i2) v += (double)K[r][i2] * z[i2];
        mu[r] = (float)v;
      }
    }
    // Joseph form S = (I-KH) Sp (I-KH)' + K R K' (upper triangle), without
    // forming I - KH: row r of (I-KH) Sp is T_r = Sp_r - K_r (H Sp), where
    // H Sp = PHt' (Sp symmetric), and then
    //   S_rc = T_rc + sum_j (K R)_rj K_cj - sum_j (T_r H')_j K_cj.
#pragma unroll
    for (int r = 0; r < DZ; ++r) {
      float Tr[DZ], Cr[DY];
#pragma unroll
      for (int k = 0; k < DZ; ++k) {
        float v = r <= k ? Sp[pk(r, k, DZ)] : Sp[pk(k, r, DZ)];
#pragma unroll
        for (int j = 0; j < DY; ++j) v = fmaf(-K[r][j], PHt[k][j], v);
        Tr[k] = v;
      }
#pragma unroll
      for (int j = 0; j < DY; ++j) {
        float kr = 0.f, th = 0.f;
#pragma unroll
        for (int m = 0; m < DY; ++m) kr = fmaf(K[r][m], sp[L::R + j * DY + m], kr);
#pragma unroll
        for (int k = 0; k < DZ; ++k) th = fmaf(Tr[k], sp[L::H + k * DY + j], th);
        Cr[j] = kr - th;
      }
#pragma unroll
      for (int c = r; c < DZ; ++c) {
        float v = Tr[c];
#pragma unroll
        for (int j = 0; j < DY; ++j) v = fmaf(Cr[j], K[c][j], v);
        S[pk(r, c, DZ)] = v;
      }
    }
    const double lin_obs = -0.5 * (qf + 2.0 * ldet + DY * GF_LOG2PI);
    const double lout = lin + inc + lin_obs;
    const float lst = (float)lout;
    lw[i] = lst;
#pragma unroll
    for (int d = 0; d < DXO; ++d) Xd[(size_t)d * N + i] = xn[d];
#pragma unroll
    for (int d = 0; d < DZ; ++d) Xd[(size_t)(DXO + d) * N + i] = mu[d];
#pragma unroll
    for (int d = 0; d < NS; ++d) Xd[(size_t)(DXO + DZ + d) * N + i] = S[d];
    if (J.anc_out) J.anc_out[(size_t)(t - 1) * N + i] = (int32_t)(a + 1);
    acc.add((double)lst);
  }
  if (fail) sc->status = GF_ERR_NOT_PD;
  block_finish(J, tile, t, fresh, acc, red, part, RB_SPLIT);
}

// Auxiliary RBPF, first stage of step t (rbpf.jl:86-124 through compute_logeta,
// particles.jl:283-296): each particle's representative outer state x* is the
// mean (MeanPredictive, ModePredictive) of its outer transition, A_o x + b_o, or
// one draw A_o x + b_o + chol(Q_o) e' from it (DrawPredictive; e' from the
// Philox stream tagged kTagLookahead, counters (i, t, 0)); its inner Gaussian is
// predicted with (prev_outer x, new_outer x*) and log eta_i is that prediction's
// update log-likelihood of y_t (predictive_loglik, rbpf.jl:113-124).  The last
// block takes the resampling decision on softmax(logw + log eta) (apf_finish).
template <int DXO, int DZ, int DY>
__global__ void __launch_bounds__(RB_THREADS) rbpf_lookahead(const PfJob* __restrict__ jobs, int njobs,
                                                            float q_gamma, int q_index) {
  using L = RbLayout<DXO, DZ, DY>;
  constexpr int NS = L::NS;
  static_assert(DXO <= 4, "one Philox block draws the outer state");
  __shared__ float sp[L::total];
  __shared__ double sy[DY];
  __shared__ double red[32];
  const int jb = find_job(jobs, njobs, blockIdx.x / RB_SPLIT, false);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const int tile = blockIdx.x / RB_SPLIT - J.tile0;
  const int part = blockIdx.x % RB_SPLIT;
  // step t's parameter block (time-varying models: calc_params(., t)), else the one block
  const float* P = reinterpret_cast<const float*>(J.params) + (size_t)(t - 1) * J.pstride;
  for (int k = threadIdx.x; k < L::total; k += RB_THREADS) sp[k] = P[k];
  if (threadIdx.x < DY) sy[threadIdx.x] = J.ys[(size_t)(t - 1) * DY + threadIdx.x];
  __syncthreads();
  const int64_t N = J.N;
  const float* Xs = reinterpret_cast<const float*>(J.X[(t - 1) & 1]);
  const float* lw = reinterpret_cast<const float*>(J.lw);
  float* eta = reinterpret_cast<float*>(J.eta);
  LseAcc acc;
  int fail = 0;
  const int64_t i = (int64_t)tile * PF_TILE + part * RB_THREADS + threadIdx.x;
  if (i < N) {
    float x[DXO], mu[DZ], S[NS];
#pragma unroll
    for (int d = 0; d < DXO; ++d) x[d] = Xs[(size_t)d * N + i];
#pragma unroll
    for (int d = 0; d < DZ; ++d) mu[d] = Xs[(size_t)(DXO + d) * N + i];
#pragma unroll
    for (int d = 0; d < NS; ++d) S[d] = Xs[(size_t)(DXO + DZ + d) * N + i];
    float e[4] = {0.f, 0.f, 0.f, 0.f};
    if (J.lookahead_draw) philox_normals4<float>(J.seed, (uint32_t)i, (uint32_t)t, 0u, e, kTagLookahead);
    float xs[DXO];
#pragma unroll
    for (int r = 0; r < DXO; ++r) {
      float v = sp[L::bo + r];
#pragma unroll
      for (int c = 0; c < DXO; ++c) v = fmaf(sp[L::Ao + c * DXO + r], x[c], v);
#pragma unroll
      for (int c = 0; c <= r; ++c) v = fmaf(sp[L::Lo + c * DXO + r], e[c], v);
      xs[r] = v;
    }
    float mp[DZ], Sp[NS];
    rb_inner_predict<DXO, DZ, DY>(sp, x, xs, q_gamma, q_index, mu, S, mp, Sp);
    float PHt[DZ][DY];
    double Sd[DY][DY];
    if (!rb_innovation<DXO, DZ, DY>(sp, Sp, PHt, Sd)) fail = 1;
    double w[DY], ldet, qf;
    rb_whiten<DXO, DZ, DY>(sp, sy, mp, Sd, w, qf, ldet);
    const float le = (float)(-0.5 * (qf + 2.0 * ldet + DY * GF_LOG2PI));
    eta[i] = le;
    acc.add((double)lw[i] + (double)le);
  }
  if (fail) sc->status = GF_ERR_NOT_PD;
  apf_finish(J, tile, t, acc, red, part, RB_SPLIT);
}

template <int DXO, int DZ, int DY>
__global__ void __launch_bounds__(PF_THREADS) rbpf_init(const PfJob* __restrict__ jobs, int njobs) {
  using L = RbLayout<DXO, DZ, DY>;
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  const int tile = blockIdx.x - J.tile0;
  const int64_t N = J.N;
  const float* P = reinterpret_cast<const float*>(J.params);
  float* X = reinterpret_cast<float*>(J.X[0]);
  float* lw = reinterpret_cast<float*>(J.lw);
  const float* noise = reinterpret_cast<const float*>(J.noise);
  for (int p = 0; p < PF_PPT; ++p) {
    const int64_t i = (int64_t)tile * PF_TILE + p * PF_THREADS + threadIdx.x;
    if (i >= N) break;
    float e[DXO];
    if (noise) {
      for (int d = 0; d < DXO; ++d) e[d] = noise[(size_t)d * N + i];
    } else {
      for (int q = 0; q < (DXO + 3) / 4; ++q) {
        float tmp[4];
        philox_normals4<float>(J.seed, (uint32_t)i, 0u, (uint32_t)q, tmp);
        for (int r = 0; r < 4; ++r)
          if (4 * q + r < DXO) e[4 * q + r] = tmp[r];
      }
    }
    for (int r = 0; r < DXO; ++r) {
      float v = P[L::muo + r];
      for (int c = 0; c <= r; ++c) v = fmaf(P[L::L0o + c * DXO + r], e[c], v);
      X[(size_t)r * N + i] = v;
    }
    for (int d = 0; d < DZ; ++d) X[(size_t)(DXO + d) * N + i] = P[L::muz + d];
    for (int d = 0; d < L::NS; ++d) X[(size_t)(DXO + DZ + d) * N + i] = P[L::S0z + d];
    lw[i] = 0.f;
  }
  if (threadIdx.x == 0) {
    J.tprefix[tile] = (double)((int64_t)tile * PF_TILE) / (double)N;
    if (tile == J.ntiles - 1) J.tprefix[J.ntiles] = 1.0;
  }
}

template <int A, int B, int C>
static RbKernels make_rb() {
  return {A, B, C, rbpf_propagate<A, B, C>, rbpf_init<A, B, C>, rbpf_lookahead<A, B, C>};
}

bool pick_rb(int dxo, int dz, int dy, RbKernels* out) {
  static const RbKernels tab[] = {make_rb<1, 1, 1>(), make_rb<1, 2, 1>(), make_rb<2, 2, 2>(),
                                  make_rb<2, 4, 2>(), make_rb<2, 8, 4>()};
  for (const auto& k : tab)
    if (k.dxo == dxo && k.dz == dz && k.dy == dy) {
      *out = k;
      return true;
    }
  return false;
}


// Parameters (float) in RbLayout order, with the outer Cholesky factors and the
// proposal's log-normaliser difference.
gf_status rb_pack_params(gf_ctx* ctx, const gf_rb_model* m, const gf_pf_config* cfg,
                         std::vector<float>& P, double* prop_const_out) {
  const int dxo = m->dxo, dz = m->dz, dy = m->dy;
  std::vector<double> Lo(dxo * dxo), L0o(dxo * dxo), LQi(dxo * dxo), Lq(dxo * dxo);
  if (chol_lower(dxo, m->Q_o, Lo.data()) || chol_lower(dxo, m->Sigma_o, L0o.data()))
    return set_err(ctx, GF_ERR_NOT_PD, "outer Q or Sigma not positive definite");
  tri_inv_lower(dxo, Lo.data(), LQi.data());
  double kk = cfg->proposal == GF_PROP_OVERDISPERSED ? cfg->proposal_k : 1.0;
  for (int i = 0; i < dxo * dxo; ++i) Lq[i] = std::sqrt(kk) * Lo[i];
  double prop_const = 0.0;
  for (int i = 0; i < dxo; ++i) prop_const += std::log(Lq[i + i * dxo]) - std::log(Lo[i + i * dxo]);
  auto put = [&](const double* a, int n) {
    for (int i = 0; i < n; ++i) P.push_back((float)a[i]);
  };
  auto put_packed = [&](const double* a, int n) {
    for (int i = 0; i < n; ++i)
      for (int j = i; j < n; ++j) P.push_back((float)a[i + j * n]);
  };
  put(m->A_o, dxo * dxo);
  put(m->b_o, dxo);
  put(Lo.data(), dxo * dxo);
  put(Lq.data(), dxo * dxo);
  put(LQi.data(), dxo * dxo);
  put(m->A_z, dz * dz);
  put(m->b_z, dz);
  put(m->C_z, dz * dxo);
  put_packed(m->Q_z, dz);
  // H stored [k][j] = H[j][k] (dz-major) for the kernel's sp[H + k*DY + j]
  for (int k = 0; k < dz; ++k)
    for (int j = 0; j < dy; ++j) P.push_back((float)m->H[j + k * dy]);
  put(m->c, dy);
  put(m->R, dy * dy);
  put(m->mu_o, dxo);
  put(L0o.data(), dxo * dxo);
  put(m->mu_z, dz);
  put_packed(m->Sigma_z, dz);

  *prop_const_out = prop_const;
  return GF_OK;
}

}  // namespace gf

using namespace gf;

static gf_status rbpf_run_impl(gf_ctx* ctx, const gf_rb_model* m, int32_t param_steps,
                               const gf_pf_config* cfg, int32_t T, const double* ys, const void* noise,
                               const double* uniforms, int32_t memspace, gf_pf_out* out, double* zmeans) {
  if (!ctx || !m || !cfg || !out || !ys || !out->ll)
    return ctx ? set_err(ctx, GF_ERR_ARG, "null argument") : GF_ERR_ARG;
  if (cfg->precision != GF_PREC_F32) return set_err(ctx, GF_ERR_UNSUPPORTED, "RBPF runs in FP32 only");
  if (cfg->lookahead < GF_LOOKAHEAD_NONE || cfg->lookahead > GF_LOOKAHEAD_DRAW)
    return set_err(ctx, GF_ERR_ARG, "unknown lookahead");
  if (cfg->proposal == GF_PROP_OPTIMAL)
    return set_err(ctx, GF_ERR_UNSUPPORTED, "RBPF supports bootstrap and overdispersed outer proposals");
  if (cfg->n_particles < 1 || T < 1) return set_err(ctx, GF_ERR_ARG, "bad N or T");
  RbKernels K;
  if (!pick_rb(m->dxo, m->dz, m->dy, &K))
    return set_err(ctx, GF_ERR_DIM, "no RBPF kernel for (dxo, dz, dy) = (%d, %d, %d)", m->dxo, m->dz, m->dy);
  cudaSetDevice(ctx->device);
  const int dxo = m->dxo, dz = m->dz, dy = m->dy;
  const int NS = dz * (dz + 1) / 2, width = dxo + dz + NS;
  // one parameter block per step of a time-varying model (calc_params(., t)),
  // else one; each block also carries the priors, which the initialisation
  // reads from block 0
  const bool tv = param_steps != 1;
  if (tv && param_steps < T) return set_err(ctx, GF_ERR_ARG, "%d parameter steps for T = %d", param_steps, T);
  const int nblk = tv ? T : 1;
  std::vector<float> P;
  double prop_const = 0.0;
  gf_status st;
  for (int k = 0; k < nblk; ++k) {
    gf_rb_model mk = *m;
    if (tv) {
      mk.A_o = m->A_o + (size_t)k * dxo * dxo;
      mk.b_o = m->b_o + (size_t)k * dxo;
      mk.Q_o = m->Q_o + (size_t)k * dxo * dxo;
      mk.A_z = m->A_z + (size_t)k * dz * dz;
      mk.b_z = m->b_z + (size_t)k * dz;
      mk.C_z = m->C_z + (size_t)k * dz * dxo;
      mk.Q_z = m->Q_z + (size_t)k * dz * dz;
      mk.H = m->H + (size_t)k * dy * dz;
      mk.c = m->c + (size_t)k * dy;
      mk.R = m->R + (size_t)k * dy * dy;
    }
    // the proposal's log-normaliser difference, sum log sqrt(k), is the same every step
    if ((st = rb_pack_params(ctx, &mk, cfg, P, &prop_const))) return st;
  }
  const int64_t pstride = tv ? (int64_t)(P.size() / nblk) : 0;
  const int64_t N = cfg->n_particles;
  const int ntiles = (int)((N + PF_TILE - 1) / PF_TILE);
  const int nstiles = (int)((N + SCAN_TILE - 1) / SCAN_TILE);
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
  void *d_params, *X0, *X1, *lw, *key, *part, *mpart, *flags, *scv, *ess1, *res1, *jobv, *schedv = nullptr;
  void *ancv, *tprev, *mpkv, *fillv;
  if ((st = get(sizeof(float) * P.size(), &d_params))) return st;
  if ((st = get(sizeof(float) * (size_t)N * width, &X0))) return st;
  if ((st = get(sizeof(float) * (size_t)N * width, &X1))) return st;
  if ((st = get(sizeof(float) * (size_t)N, &lw))) return st;
  if ((st = get(sizeof(double) * (size_t)N, &key))) return st;
  if ((st = get(sizeof(int32_t) * (size_t)N, &ancv))) return st;
  if ((st = get(sizeof(double) * (size_t)(ntiles + 1), &tprev))) return st;
  if ((st = get(sizeof(int32_t) * (size_t)(ntiles + 1), &mpkv))) return st;
  if ((st = get(sizeof(int32_t) * (size_t)N, &fillv))) return st;
  if ((st = get(sizeof(double) * PF_PW * ntiles * PF_MAX_SPLIT, &part))) return st;
  if ((st = get(sizeof(double) * ntiles * (dxo + dz), &mpart))) return st;
  if ((st = get(sizeof(unsigned long long) * 2 * nstiles, &flags))) return st;
  if ((st = get(sizeof(PfScalars), &scv))) return st;
  if ((st = get(sizeof(double), &ess1))) return st;
  if ((st = get(8, &res1))) return st;
  if ((st = get(sizeof(PfJob), &jobv))) return st;
  if (cfg->schedule && (st = get((size_t)T, &schedv))) return st;
  void* etav = nullptr;  // auxiliary filter: first-stage log eta [N]
  if (cfg->lookahead != GF_LOOKAHEAD_NONE && (st = get(sizeof(float) * (size_t)N, &etav))) return st;
  cudaStream_t s = ctx->stream;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(d_params, P.data(), sizeof(float) * P.size(), cudaMemcpyHostToDevice, s));
  if (schedv) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(schedv, cfg->schedule, (size_t)T, cudaMemcpyHostToDevice, s));
  double e1 = uniform_ess(N);
  int sch0 = cfg->schedule ? cfg->schedule[0] : -1;
  int8_t r1 = (int8_t)(sch0 >= 0 ? (sch0 != 0) : (cfg->threshold * (double)N >= e1));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(ess1, &e1, sizeof(double), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(res1, &r1, 1, cudaMemcpyHostToDevice, s));
  // ---- inputs / outputs in device memory
  const bool host = memspace == GF_MEM_HOST;
  const double* d_ys = ys;
  const void* d_noise = noise;
  const double* d_unif = uniforms;
  gf_pf_out d = *out;
  double* d_means = nullptr;
  if (host) {
    void* v;
    if ((st = get(sizeof(double) * (size_t)T * dy, &v))) return st;
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(v, ys, sizeof(double) * (size_t)T * dy, cudaMemcpyHostToDevice, s));
    d_ys = (const double*)v;
    if (noise) {
      size_t nb = sizeof(float) * (size_t)(T + 1) * dxo * N;
      if ((st = get(nb, &v))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(v, noise, nb, cudaMemcpyHostToDevice, s));
      d_noise = v;
    }
    if (uniforms) {
      size_t ub = sizeof(double) * (size_t)T * (cfg->resampler == GF_RS_SYSTEMATIC ? 1 : N);
      if ((st = get(ub, &v))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(v, uniforms, ub, cudaMemcpyHostToDevice, s));
      d_unif = (const double*)v;
    }
    auto mk = [&](void* h, void** dp, size_t bytes) -> gf_status {
      if (!h) {
        *dp = nullptr;
        return GF_OK;
      }
      return get(bytes, dp);
    };
    if ((st = mk(out->ll, (void**)&d.ll, sizeof(double)))) return st;
    if ((st = mk(out->ll_steps, (void**)&d.ll_steps, sizeof(double) * T))) return st;
    if ((st = mk(out->ess_steps, (void**)&d.ess_steps, sizeof(double) * T))) return st;
    if ((st = mk(out->resampled, (void**)&d.resampled, (size_t)T))) return st;
    if ((st = mk(out->ancestors, (void**)&d.ancestors, sizeof(int32_t) * (size_t)T * N))) return st;
    if ((st = mk(out->states, (void**)&d.states, sizeof(float) * (size_t)N * width))) return st;
    if ((st = mk(out->log_weights, (void**)&d.log_weights, sizeof(double) * (size_t)N))) return st;
    if ((st = mk(out->clamps, (void**)&d.clamps, sizeof(int32_t)))) return st;
    if ((st = mk(out->paths, (void**)&d.paths, sizeof(float) * (size_t)(T + 1) * width * N))) return st;
    if ((st = mk(out->history, (void**)&d.history, sizeof(float) * (size_t)(T + 1) * width * N))) return st;
    if ((st = mk(out->log_weight_history, (void**)&d.log_weight_history, sizeof(double) * (size_t)T * N)))
      return st;
  }
  const bool want_means = out->means || zmeans;
  if (want_means && !host)
    return set_err(ctx, GF_ERR_UNSUPPORTED, "RBPF means are returned through host buffers only");
  if (want_means) {
    void* v;
    if ((st = get(sizeof(double) * (size_t)T * (dxo + dz), &v))) return st;
    d_means = (double*)v;
  }
  PfJob J;
  std::memset(&J, 0, sizeof J);
  J.N = N;
  J.dx = dxo;
  J.dy = dy;
  J.T = T;
  J.width = width;
  J.ntiles = ntiles;
  J.nstiles = nstiles;
  J.resampler = cfg->resampler;
  J.conv = cfg->convention;
  J.prop = cfg->proposal;
  J.threshold = cfg->threshold;
  J.log_n = std::log((double)N);
  J.prop_const = prop_const;
  J.seed = cfg->seed;
  J.params = d_params;
  J.pstride = pstride;
  J.X[0] = X0;
  J.X[1] = X1;
  J.lw = lw;
  J.key = (double*)key;
  J.part = (double*)part;
  J.flags = (unsigned long long*)flags;
  J.sc = (PfScalars*)scv;
  J.ocum = (int32_t*)ancv;
  J.mpk = (int32_t*)mpkv;
  J.anc = (int32_t*)fillv;
  J.tprefix = (double*)tprev;
  J.noise = d_noise;
  J.unif = d_unif;
  J.schedule = (const int8_t*)schedv;
  J.ll_steps = d.ll_steps;
  J.ess_steps = d.ess_steps;
  J.res_steps = d.resampled;
  J.anc_out = d.ancestors;
  J.ys = d_ys;
  J.ll_out = d.ll;
  J.logw_out = d.log_weights;
  J.states_out = d.states;
  J.clamps_out = d.clamps;
  J.means_out = d_means;
  J.hist = d.history;
  J.lwh = d.log_weight_history;
  J.eta = etav;
  J.lookahead_draw = cfg->lookahead == GF_LOOKAHEAD_DRAW ? 1 : 0;
  PfJob* jd = (PfJob*)jobv;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(jd, &J, sizeof J, cudaMemcpyHostToDevice, s));
  launch_init_scalars(ctx, jd, 1, (const double*)ess1, (const int8_t*)res1);
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(flags, 0, sizeof(unsigned long long) * 2 * nstiles, s));
  K.init<<<ntiles, PF_THREADS, 0, s>>>(jd, 1);
  // ancestry: the device path storage (AncestorCallback) and the dense history
  // (DenseAncestorCallback) over the packed device state [x | mu | Sigma upper]
  const bool paths = d.paths != nullptr, record = d.history || d.log_weight_history;
  TreeHost th;
  struct TreeGuard {
    TreeHost* h;
    ~TreeGuard() {
      if (h->ctx) {
        cudaStreamSynchronize(h->ctx->stream);
        tree_host_release(*h);
      }
    }
  } tree_guard{&th};
  if (paths) {
    th.ctx = ctx;
    th.N = N;
    th.width = width;
    th.rsize = sizeof(float);
    if ((st = tree_host_prepare(th))) return st;
    tree_launch_init(ctx, false, jd, N, th.tree);
  }
  if (record) launch_record(ctx, false, jd, N);
  // auxiliary filter: first-stage scores and the resampling decision of the
  // coming step, before its resample
  auto lookahead = [&]() {
    if (!etav) return;
    ProfScope ps(ctx, KC_SCAN);
    K.lookahead<<<ntiles * RB_SPLIT, RB_THREADS, 0, s>>>(jd, 1, (float)m->q_gamma, m->q_index);
  };
  lookahead();
  launch_resample(ctx, false, jd, 1, ntiles);
  const int guided = cfg->proposal == GF_PROP_OVERDISPERSED;
  for (int t = 1; t <= T; ++t) {
    if (paths) {
      if ((t - 1) % kTreeChunk == 0) {
        const int64_t steps = std::min<int64_t>(kTreeChunk, T - t + 1);
        if ((st = tree_host_reserve(th, steps * N))) return st;
      }
      tree_launch_step_pre(ctx, jd, N, th.tree, cfg->resampler != GF_RS_MULTINOMIAL);
    }
    {
      ProfScope ps(ctx, KC_RBPF);
      K.prop<<<ntiles * RB_SPLIT, RB_THREADS, 0, s>>>(jd, 1, (float)m->q_gamma, m->q_index, guided);
    }
    if (paths) tree_launch_insert(ctx, false, jd, N, th.tree, t);
    if (want_means) launch_means(ctx, false, jd, 1, ntiles, (double*)mpart, dxo + dz);
    if (record) launch_record(ctx, false, jd, N);
    if (t < T) {
      lookahead();
      launch_resample(ctx, false, jd, 1, ntiles);
    }
  }
  launch_finish(ctx, false, jd, N);
  if (paths) tree_launch_paths(ctx, false, jd, N, th.tree, T, d.paths);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  // ---- outputs
  std::vector<double> hm;
  if (want_means) {
    hm.resize((size_t)T * (dxo + dz));
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(hm.data(), d_means, sizeof(double) * hm.size(), cudaMemcpyDeviceToHost, s));
  }
  if (host) {
    auto back = [&](void* h, const void* dv, size_t bytes) -> gf_status {
      if (h && dv) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(h, dv, bytes, cudaMemcpyDeviceToHost, s));
      return GF_OK;
    };
    back(out->ll, d.ll, sizeof(double));
    back(out->ll_steps, d.ll_steps, sizeof(double) * T);
    back(out->ess_steps, d.ess_steps, sizeof(double) * T);
    back(out->resampled, d.resampled, (size_t)T);
    back(out->ancestors, d.ancestors, sizeof(int32_t) * (size_t)T * N);
    back(out->log_weights, d.log_weights, sizeof(double) * (size_t)N);
    back(out->clamps, d.clamps, sizeof(int32_t));
    back(out->paths, d.paths, sizeof(float) * (size_t)(T + 1) * width * N);
    back(out->history, d.history, sizeof(float) * (size_t)(T + 1) * width * N);
    back(out->log_weight_history, d.log_weight_history, sizeof(double) * (size_t)T * N);
    if (out->states) {
      // unpack: [x | mu | Sigma packed] -> [x | mu | Sigma column-major]
      std::vector<float> hs((size_t)N * width);
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(hs.data(), d.states, sizeof(float) * hs.size(), cudaMemcpyDeviceToHost, s));
      GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
      float* o = (float*)out->states;
      for (int c = 0; c < dxo + dz; ++c) std::memcpy(o + (size_t)c * N, hs.data() + (size_t)c * N, sizeof(float) * N);
      for (int i2 = 0; i2 < dz; ++i2)
        for (int j = i2; j < dz; ++j) {
          const float* src = hs.data() + (size_t)(dxo + dz + pk(i2, j, dz)) * N;
          std::memcpy(o + (size_t)(dxo + dz + i2 + j * dz) * N, src, sizeof(float) * N);
          std::memcpy(o + (size_t)(dxo + dz + j + i2 * dz) * N, src, sizeof(float) * N);
        }
    }
  }
  PfScalars sc;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(&sc, scv, sizeof sc, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (want_means) {
    for (int t = 0; t < T; ++t) {
      if (out->means && host)
        for (int d2 = 0; d2 < dxo; ++d2) out->means[(size_t)t * dxo + d2] = hm[(size_t)t * (dxo + dz) + d2];
      if (zmeans && host)
        for (int d2 = 0; d2 < dz; ++d2) zmeans[(size_t)t * dz + d2] = hm[(size_t)t * (dxo + dz) + dxo + d2];
    }
  }
  if (sc.status == GF_ERR_NOT_PD) return set_err(ctx, GF_ERR_NOT_PD, "inner innovation covariance not PD at step %d", sc.t + 1);
  if (sc.status) return set_err(ctx, sc.status, "RBPF failed at step %d (status %d)", sc.t + 1, sc.status);
  return GF_OK;
}

extern "C" gf_status gf_rbpf_run(gf_ctx* ctx, const gf_rb_model* m, const gf_pf_config* cfg, int32_t T,
                                 const double* ys, const void* noise, const double* uniforms,
                                 int32_t memspace, gf_pf_out* out, double* zmeans) {
  return rbpf_run_impl(ctx, m, 1, cfg, T, ys, noise, uniforms, memspace, out, zmeans);
}

extern "C" gf_status gf_rbpf_run_tv(gf_ctx* ctx, const gf_rb_model* m, int32_t param_steps,
                                    const gf_pf_config* cfg, int32_t T, const double* ys, const void* noise,
                                    const double* uniforms, int32_t memspace, gf_pf_out* out,
                                    double* zmeans) {
  return rbpf_run_impl(ctx, m, param_steps, cfg, T, ys, noise, uniforms, memspace, out, zmeans);
}
