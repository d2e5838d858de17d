// gf_pf_lg.cuh -- linear-Gaussian particle-filter kernel templates.
//
// Restates GeneralisedFilters' PF (particles.jl:36-90,147-245) for
// LinearGaussianStateSpaceModel: state x_t = A x_{t-1} + b + L_Q e (BF) or the
// linear-Gaussian proposal x_t = M x_{t-1} + v_t + L_q e with weight increment
// log p(x_t|x_{t-1}) - log q(x_t|x_{t-1},y_t) (GFTest OptimalProposal /
// OverdispersedProposal).  Observation log-density uses the whitened form
// -1/2 |L_R^{-1}(y - c) - (L_R^{-1}H) x|^2 + const, the same quantity as
// logpdf(MvNormal(Hx + c, R), y) (models/linear_gaussian.jl:85-90).
#pragma once
#include <type_traits>
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"
#include "gf_umma.cuh"

namespace gf {

// ------------------------------------------------------------------ layout
// params (Real, column-major, padded to DXP/DYP):
//   A[DXP*DXP] | L[DXP*DXP] | b[DXP] | Ht[DYP*DXP] | M[DXP*DXP] | Qi[DXP*DXP] |
//   mu0[DXP] | L0[DXP*DXP]
// ystep[t] (Real): ytil[DYP] | v[DXP]
template <int DXP, int DYP>
struct LgLayout {
  static constexpr int A = 0, L = DXP * DXP, b = 2 * DXP * DXP, H = 2 * DXP * DXP + DXP;
  static constexpr int M = H + DYP * DXP, Qi = M + DXP * DXP, mu0 = Qi + DXP * DXP;
  static constexpr int L0 = mu0 + DXP, total = L0 + DXP * DXP;
  static constexpr int smem_boot = H + DYP * DXP + DYP + DXP;  // A,L,b,H + ystep
  static constexpr int smem_guided = smem_boot + 2 * DXP * DXP;
};

template <typename Real, int DXP>
__device__ __forceinline__ void draw_noise(const PfJob& J, const Real* noise, int64_t i, int t,
                                           int dx, int64_t N, Real* e) {
  if (noise) {
#pragma unroll
    for (int d = 0; d < DXP; ++d) e[d] = d < dx ? noise[(size_t)d * N + i] : Real(0);
  } else if (DXP == 1) {
    Real tmp[4];  // 1-D: particle i takes normal i % 4 of call i / 4
    philox_normals4<Real>(J.seed, (uint32_t)(i >> 2), (uint32_t)t, 0u, tmp);
    e[0] = tmp[i & 3];
  } else {
#pragma unroll
    for (int q = 0; q < (DXP + 3) / 4; ++q) {
      Real tmp[4];
      philox_normals4<Real>(J.seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, tmp);
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (4 * q + r < DXP) e[4 * q + r] = tmp[r];
    }
  }
}

// 1-D noise of a thread's PF_PPT particles (i = tile * PF_TILE + p * PF_THREADS
// + threadIdx.x): lane l of each warp runs Philox call (i / 4) for the group of
// four consecutive particles at p = l / 8, slot l % 8, and the warp hands each
// particle normal i % 4 by shuffles -- one call per four particles.  All 32
// lanes take part (calls beyond N are unused).
template <typename Real>
__device__ __forceinline__ void noise_1d_tile(uint64_t seed, int tile, int t, Real* ep) {
  static_assert(PF_PPT * PF_THREADS == PF_TILE && PF_PPT == 4, "four particles per thread");
  const int lane = threadIdx.x & 31;
  const int64_t wbase = (int64_t)tile * PF_TILE + (threadIdx.x & ~31);
  const int64_t mine = wbase + (lane >> 3) * PF_THREADS + 4 * (lane & 7);
  Real r4[4];
  philox_normals4<Real>(seed, (uint32_t)(mine >> 2), (uint32_t)t, 0u, r4);
#pragma unroll
  for (int p = 0; p < PF_PPT; ++p) {
    const int src = p * 8 + (lane >> 2);
    const Real v0 = __shfl_sync(0xffffffffu, r4[0], src), v1 = __shfl_sync(0xffffffffu, r4[1], src);
    const Real v2 = __shfl_sync(0xffffffffu, r4[2], src), v3 = __shfl_sync(0xffffffffu, r4[3], src);
    const int k = lane & 3;
    ep[p] = k == 0 ? v0 : (k == 1 ? v1 : (k == 2 ? v2 : v3));
  }
}

// One 1024-particle tile of the propagate (a whole filter when N <= 1024).
// COHERENT: read the ancestors through L2, for a caller that wrote them earlier
// in the same kernel.
template <typename Real, int DXP, int DYP, bool GUIDED, bool COHERENT>
__device__ __forceinline__ void lg_propagate_tile(const PfJob& J, int tile) {
  using Lay = LgLayout<DXP, DYP>;
  extern __shared__ __align__(16) unsigned char smraw[];
  Real* sA = reinterpret_cast<Real*>(smraw);
  Real* sL = sA + Lay::L;
  Real* sb = sA + Lay::b;
  Real* sH = sA + Lay::H;
  Real* sy = sH + DYP * DXP;  // ytil[DYP] then v[DXP]
  Real* sv = sy + DYP;
  Real* sM = sv + DXP;
  Real* sQi = sM + DXP * DXP;
  __shared__ double red[32];

  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const bool resamp = sc->resample != 0;
  const bool fresh = resamp || sc->uniform != 0;
  const double lse_prev = sc->lse;
  const bool searched = J.resampler == GF_RS_MULTINOMIAL;

  const Real* P = reinterpret_cast<const Real*>(J.params) + (size_t)(t - 1) * J.pstride;
  for (int k = threadIdx.x; k < Lay::H + DYP * DXP; k += PF_THREADS) sA[k] = P[k];
  const Real* Y = reinterpret_cast<const Real*>(J.ystep) + (size_t)(t - 1) * J.ystride;
  for (int k = threadIdx.x; k < DYP + DXP; k += PF_THREADS) sy[k] = Y[k];
  if constexpr (GUIDED) {
    for (int k = threadIdx.x; k < 2 * DXP * DXP; k += PF_THREADS) sM[k] = P[Lay::M + k];
  }
  __syncthreads();

  const int64_t N = J.N;
  const int dx = J.dx;
  const Real* Xs = reinterpret_cast<const Real*>(J.X[(t - 1) & 1]);
  Real* Xd = reinterpret_cast<Real*>(J.X[t & 1]);
  Real* lw = reinterpret_cast<Real*>(J.lw);
  const Real* noise = J.noise ? reinterpret_cast<const Real*>(J.noise) + (size_t)t * dx * N : nullptr;
  const int32_t* __restrict__ ancv = J.anc;
  int32_t* __restrict__ anc_out = J.anc_out;
  const uint64_t seed = J.seed;
  const bool diag = J.diag_l != 0;
  const double obs_const = step_obs_const(J, t), prop_const = step_prop_const(J, t);
  const Real* eta = reinterpret_cast<const Real*>(J.eta);
  const bool apf = resamp && eta != nullptr;
  LseAcc acc;
  Real ep1[DXP == 1 ? PF_PPT : 1];
  if constexpr (DXP == 1) {
    if (!noise) noise_1d_tile<Real>(seed, tile, t, ep1);
  }

  for (int p = 0; p < PF_PPT; ++p) {
    const int64_t i = (int64_t)tile * PF_TILE + p * PF_THREADS + threadIdx.x;
    if (i >= N) break;
    int64_t a = i;
    if (resamp) a = searched ? find_ancestor(J, sc, t, i, 0, N) : (int64_t)(COHERENT ? __ldcg(ancv + i) : ancv[i]);
    Real x[DXP];
#pragma unroll
    for (int d = 0; d < DXP; ++d) x[d] = d < dx ? Xs[(size_t)d * N + a] : Real(0);
    // after an auxiliary resample the particle starts from -log eta of its ancestor
    const double lin = fresh ? (apf ? -(double)eta[a] : 0.0) : (double)lw[i] - lse_prev;
    // mean part: x' = A x + b (bootstrap, simulate(dyn) = rand(MvNormal(A x + b, Q)))
    // or M x + v_t (guided), with ma = A x + b kept for log p(x'|x)
    Real xn[DXP];
    Real ma[GUIDED ? DXP : 1];
#pragma unroll
    for (int r = 0; r < DXP; ++r) xn[r] = GUIDED ? sv[r] : sb[r];
    if constexpr (GUIDED) {
#pragma unroll
      for (int r = 0; r < DXP; ++r) ma[r] = sb[r];
    }
#pragma unroll
    for (int c = 0; c < DXP; ++c) {
      const Real xc = x[c];
#pragma unroll
      for (int r = 0; r < DXP; ++r) {
        if constexpr (GUIDED) {
          xn[r] = fma(sM[c * DXP + r], xc, xn[r]);
          ma[r] = fma(sA[c * DXP + r], xc, ma[r]);
        } else {
          xn[r] = fma(sA[c * DXP + r], xc, xn[r]);
        }
      }
    }
    // noise part: + L e, with e drawn four at a time and consumed at once
    Real qe = 0;
#pragma unroll
    for (int q = 0; q < (DXP + 3) / 4; ++q) {
      Real e4[4];
      if (noise) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int c = 4 * q + cc;
          e4[cc] = (c < DXP && c < dx) ? noise[(size_t)c * N + i] : Real(0);
        }
      } else if constexpr (DXP == 1) {
        e4[0] = ep1[p];
      } else {
        philox_normals4<Real>(seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, e4);
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const int c = 4 * q + cc;
        if (c < DXP) {
          const Real ec = e4[cc];
          if constexpr (GUIDED) qe = fma(ec, ec, qe);
          if (diag) {
            xn[c] = fma(sL[c * DXP + c], ec, xn[c]);
          } else {
#pragma unroll
            for (int r = c; r < DXP; ++r) xn[r] = fma(sL[c * DXP + r], ec, xn[r]);
          }
        }
      }
    }
    double inc = 0.0;
    if constexpr (GUIDED) {
      // inc = log N(x'; A x + b, Q) - log N(x'; M x + v_t, Lq Lq')
      Real qz = 0;
#pragma unroll
      for (int r = 0; r < DXP; ++r) ma[r] = xn[r] - ma[r];
#pragma unroll
      for (int r = 0; r < DXP; ++r) {
        Real z = 0;
#pragma unroll
        for (int c = 0; c <= r; ++c) z = fma(sQi[c * DXP + r], ma[c], z);
        qz = fma(z, z, qz);
      }
      inc = -0.5 * (double)qz + 0.5 * (double)qe + prop_const;
    }
    // observation: -1/2 |ytil - Ht x'|^2 + const
    Real q = 0;
#pragma unroll
    for (int k = 0; k < DYP; ++k) {
      Real r = sy[k];
#pragma unroll
      for (int c = 0; c < DXP; ++c) r = fma(-sH[c * DYP + k], xn[c], r);
      q = fma(r, r, q);
    }
    const double lout = lin + inc + (obs_const - 0.5 * (double)q);
    const Real lst = (Real)lout;
    lw[i] = lst;
#pragma unroll
    for (int d = 0; d < DXP; ++d)
      if (d < dx) Xd[(size_t)d * N + i] = xn[d];
    if (anc_out) anc_out[(size_t)(t - 1) * N + i] = (int32_t)(a + 1);
    acc.add((double)lst);
  }
  block_finish(J, tile, t, fresh, acc, red);
}

template <typename Real, int DXP, int DYP, bool GUIDED>
__global__ void __launch_bounds__(PF_THREADS, 3) pf_lg_propagate(const PfJob* __restrict__ jobs,
                                                             int njobs) {
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  lg_propagate_tile<Real, DXP, DYP, GUIDED, false>(J, blockIdx.x - J.tile0);
}

// x_0 ~ MvNormal(mu0, Sigma0) (particles.jl:36-50, models/linear_gaussian.jl:23-29)
template <typename Real, int DXP>
__device__ __forceinline__ void lg_init_tile(const PfJob& J, int tile, int mu_off, int l0_off) {
  const int64_t N = J.N;
  const int dx = J.dx;
  const Real* P = reinterpret_cast<const Real*>(J.params);
  Real* X = reinterpret_cast<Real*>(J.X[0]);
  Real* lw = reinterpret_cast<Real*>(J.lw);
  const Real* noise = reinterpret_cast<const Real*>(J.noise);
  for (int p = 0; p < PF_PPT; ++p) {
    const int64_t i = (int64_t)tile * PF_TILE + p * PF_THREADS + threadIdx.x;
    if (i >= N) break;
    Real e[DXP];
    draw_noise<Real, DXP>(J, noise, i, 0, dx, N, e);
#pragma unroll
    for (int r = 0; r < DXP; ++r) {
      if (r >= dx) break;
      Real v = P[mu_off + r];
#pragma unroll
      for (int c = 0; c <= r; ++c) v = fma(P[l0_off + c * DXP + r], e[c], v);
      X[(size_t)r * N + i] = v;
    }
    lw[i] = Real(0);
  }
  // cumulative weight at each tile start for the uniform initial weights
  if (threadIdx.x == 0) {
    J.tprefix[tile] = (double)((int64_t)tile * PF_TILE) / (double)N;
    if (tile == J.ntiles - 1) J.tprefix[J.ntiles] = 1.0;
  }
}

template <typename Real, int DXP>
__global__ void __launch_bounds__(PF_THREADS) pf_lg_init(const PfJob* __restrict__ jobs, int njobs,
                                                        int mu_off, int l0_off) {
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  lg_init_tile<Real, DXP>(J, blockIdx.x - J.tile0, mu_off, l0_off);
}

// A whole filter of N <= 1024 particles (one tile) in one block: the
// initialisation, then per step the propagate with its finalise, the resample
// and the ancestor fill of the multi-kernel run, separated by block barriers
// instead of kernel boundaries, and the final outputs.  Same arithmetic in the
// same order as the multi-kernel run, so the same ancestors and log-likelihood.
// Systematic and stratified rules (the multinomial search reads its keys
// through the read-only cache, which a kernel must not write); weighted means
// as the per-step means kernel computes them.
template <typename Real, int DXP, int DYP, bool GUIDED, bool MEANS>
__global__ void __launch_bounds__(PF_THREADS) pf_lg_small_filter(const PfJob* __restrict__ jobs, int mu_off,
                                                                int l0_off, double* __restrict__ mpart) {
  const PfJob& J = jobs[0];
  // loop-invariant job fields in registers (the job lives in global memory)
  const int T = J.T, dx = J.dx;
  double* const means_out = J.means_out;
  lg_init_tile<Real, DXP>(J, 0, mu_off, l0_off);
  __syncthreads();
  resample_tile<Real>(J, 0);
  __syncthreads();
  fill_block<true>(J, 0);
  __syncthreads();
  for (int t = 1; t <= T; ++t) {
    lg_propagate_tile<Real, DXP, DYP, GUIDED, true>(J, 0);
    __syncthreads();
    if (MEANS) {
      pf_means_kernel<Real>(jobs, 1, mpart, means_out, dx);
      __syncthreads();
    }
    if (t < T) {
      resample_tile<Real>(J, 0);
      __syncthreads();
      fill_block<true>(J, 0);
      __syncthreads();
    }
  }
  pf_finish_block<Real>(J);
}


// ------------------------------------------------- tensor-core propagation
// Bootstrap propagation + observation for state dimension >= 16 on the tcgen05
// tensor cores.  Per 128-particle sub-tile, one MMA chain computes
//   [x' - b | H~x' - H~b] = [x | e] * [[A, L], [H~A, H~L]]^T
// in kind::tf32 with the 3xTF32 split (A_hi B_hi + A_hi B_lo + A_lo B_hi), so
// the result carries FP32-level accuracy; the FP32 accumulator lives in TMEM
// (one lane per particle) and is read back for the weight and the state store.
constexpr int TC_THREADS = 128;
constexpr int TC_SUB = PF_TILE / TC_THREADS;
static_assert(TC_SUB == TC_SUB_UNITS && TC_SUB <= PF_MAX_SPLIT, "unit partials per tile");
// Blocks per tile (each TC_SUB / TC_SPLIT sub-tiles, partials kept per block).
// One: the per-block prologue (operand-B staging, TMEM allocation) and the
// partial reduction cost more than shorter waves save (at Dx=16, N=2^20 the
// propagate took 1.16x, 1.5x and 2.5x as long with 2, 4 and 8 blocks per tile).
constexpr int TC_SPLIT = 1;
constexpr int TC_SUB_BLOCK = TC_SUB / TC_SPLIT;
static_assert(TC_SUB % TC_SPLIT == 0 && TC_SPLIT <= PF_MAX_SPLIT, "tensor-core tile split");
constexpr uint32_t TC_WAIT = 1u << 22;  // bounded mbarrier polls

template <int DXP, int DYP>
struct TcLayout {
  static constexpr int K = 2 * DXP;
  static constexpr int NM = ((DXP + DYP + 15) / 16) * 16;
  static constexpr uint32_t NCOLS = NM <= 32 ? 32 : (NM <= 64 ? 64 : 128);
  // params appendix (float): B [NM][K] row-major, H~b [DYP]
  static constexpr int B_off = LgLayout<DXP, DYP>::total;
  static constexpr int Hb_off = B_off + NM * K;
  static constexpr int total = Hb_off + DYP;
  static constexpr size_t smem_bytes = sizeof(float) * (2 * 128 * K + 2 * NM * K + DXP + 2 * DYP);
  // Resident blocks per SM that shared memory allows (228 KB per SM, 1 KB
  // reserved per block, ~1 KB of static shared arrays), at most 5: the launch
  // bound caps registers to match (Dx=16: 91 instead of 156 registers, 5 blocks
  // per SM instead of 3, propagate 1.2x faster at N=2^20).
  static constexpr int by_smem = (int)((228u * 1024u) / (smem_bytes + 2048u));
  static constexpr int min_blocks = by_smem < 1 ? 1 : (by_smem > 5 ? 5 : by_smem);
};

// Staged ancestor gather (STAGED instances of pf_lg_propagate_tc): while the
// MMA and epilogue of sub-tile s run, one thread copies the contiguous source
// range [a_first, a_last] of sub-tile s+1 (sorted ancestors: the CPU-rule
// systematic and stratified resamplers, or a = i without a resample) from every
// state dimension into shared memory with cp.async.bulk (16-byte aligned, size
// a multiple of 16), completing on an mbarrier; the threads then read their
// gathered states from shared memory.  Ranges longer than TC_GCAP particles,
// the multinomial search and N % 4 != 0 take the per-thread gather.
constexpr int TC_GCAP = 192;
template <int DXP, int DYP, bool STAGED>
struct TcSmem {
  static constexpr size_t gather_off = (TcLayout<DXP, DYP>::smem_bytes + 127) / 128 * 128;
  static constexpr size_t bytes = STAGED ? gather_off + sizeof(float) * DXP * TC_GCAP
                                         : TcLayout<DXP, DYP>::smem_bytes;
  static constexpr int by_smem = (int)((228u * 1024u) / (bytes + 2048u));
  static constexpr int min_blocks = by_smem < 1 ? 1 : (by_smem > 5 ? 5 : by_smem);
};

template <int DXP, int DYP, bool STAGED = false>
__global__ void __launch_bounds__(TC_THREADS, (TcSmem<DXP, DYP, STAGED>::min_blocks)) pf_lg_propagate_tc(const PfJob* __restrict__ jobs,
                                                               int njobs) {
  using Lay = LgLayout<DXP, DYP>;
  using TL = TcLayout<DXP, DYP>;
  constexpr int K = TL::K, NM = TL::NM;
  extern __shared__ __align__(128) unsigned char smraw[];
  float* sAh = reinterpret_cast<float*>(smraw);
  float* sAl = sAh + 128 * K;
  float* sBh = sAl + 128 * K;
  float* sBl = sBh + NM * K;
  float* sb = sBl + NM * K;
  float* sHb = sb + DXP;
  float* sy = sHb + DYP;
  float* sG = reinterpret_cast<float*>(smraw + TcSmem<DXP, DYP, STAGED>::gather_off);  // [DXP][TC_GCAP]
  __shared__ double red[32];
  __shared__ uint64_t mbar, gbar;
  __shared__ int64_t glo[2];  // staged sub-tile: first copied source particle, -1 = per-thread gather
  __shared__ uint32_t tmem_slot;

  const int jb = find_job(jobs, njobs, blockIdx.x / TC_SPLIT, false);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const int tile = blockIdx.x / TC_SPLIT - J.tile0;
  const int part = blockIdx.x % TC_SPLIT;
  const int tid = threadIdx.x;
  const bool resamp = sc->resample != 0;
  const bool fresh = resamp || sc->uniform != 0;
  const double lse_prev = sc->lse;
  const bool searched = J.resampler == GF_RS_MULTINOMIAL;

  const float* P = reinterpret_cast<const float*>(J.params) + (size_t)(t - 1) * J.pstride;
  for (int e = tid; e < NM * K; e += TC_THREADS) {
    const int n = e / K, k = e - n * K;
    const float v = P[TL::B_off + e];
    const float h = umma::to_tf32(v);
    const uint32_t off = umma::kmajor_offset(n, k, K) >> 2;
    sBh[off] = h;
    sBl[off] = umma::to_tf32(v - h);
  }
  for (int e = tid; e < DXP; e += TC_THREADS) sb[e] = P[Lay::b + e];
  const float* Y = reinterpret_cast<const float*>(J.ystep) + (size_t)(t - 1) * J.ystride;
  for (int e = tid; e < DYP; e += TC_THREADS) {
    sHb[e] = P[TL::Hb_off + e];
    sy[e] = Y[e];
  }
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    if (STAGED) umma::mbar_init(&gbar, 1);
    umma::fence_mbar_init();
  }
  if (tid < 32) umma::tmem_alloc(&tmem_slot, TL::NCOLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_slot;
  const uint32_t tlane = tbase + ((uint32_t)(32 * (tid >> 5)) << 16);

  const int64_t N = J.N;
  const int dx = J.dx;
  const float* Xs = reinterpret_cast<const float*>(J.X[(t - 1) & 1]);
  float* Xd = reinterpret_cast<float*>(J.X[t & 1]);
  float* lw = reinterpret_cast<float*>(J.lw);
  const float* noise = J.noise ? reinterpret_cast<const float*>(J.noise) + (size_t)t * dx * N : nullptr;
  const int32_t* __restrict__ ancv = J.anc;
  int32_t* __restrict__ anc_out = J.anc_out;
  const uint64_t seed = J.seed;
  const double obs_const = step_obs_const(J, t);
  const float* eta = reinterpret_cast<const float*>(J.eta);
  const bool apf = resamp && eta != nullptr;
  const uint32_t idesc = umma::idesc_tf32(128, NM);
  const uint32_t kstride = 128, mstride = (uint32_t)(K / 4) * 128;
  LseAcc acc;
  bool ok = true;

  // the next sub-tile's ancestor index is loaded one sub-tile ahead, so only the
  // state gather stays on each sub-tile's critical path (2% at Dx=16, N=2^20)
  const int64_t ib = (int64_t)tile * PF_TILE + part * TC_SUB_BLOCK * TC_THREADS + tid;
  const bool pref = resamp && !searched;
  int32_t a_nx = (pref && ib < N) ? ancv[ib] : 0;
  // staged gather of sub-tile s (thread 0): bulk copies of the source range,
  // or glo = -1 (per-thread gather); the gbar phase completes either way
  const bool can_stage = STAGED && !searched && (N & 3) == 0;
  auto stage = [&](int s) {
    const int64_t f = ib - tid + (int64_t)s * TC_THREADS;
    const int64_t l = min(f + TC_THREADS - 1, N - 1);
    int64_t lo = -1, cnt = 0;
    if (can_stage && f < N) {
      const int64_t a0 = resamp ? (int64_t)ancv[f] : f, a1 = resamp ? (int64_t)ancv[l] : l;
      lo = a0 & ~(int64_t)3;
      cnt = min((a1 | 3) + 1, N) - lo;
      if (cnt > TC_GCAP) lo = -1;
    }
    glo[s & 1] = lo;
    if (lo >= 0) {
      umma::mbar_arrive_expect_tx(&gbar, (uint32_t)(dx * cnt * 4));
      for (int d = 0; d < dx; ++d)
        umma::bulk_copy_g2s(sG + d * TC_GCAP, Xs + (size_t)d * N + lo, (uint32_t)(cnt * 4), &gbar);
    } else {
      umma::mbar_arrive(&gbar);
    }
  };
  if (STAGED && tid == 0) stage(0);
  for (int s = 0; s < TC_SUB_BLOCK; ++s) {
    const int64_t i = ib + (int64_t)s * TC_THREADS;
    const bool valid = i < N;
    int64_t a = i;
    if (valid && resamp) a = searched ? find_ancestor(J, sc, t, i, 0, N) : (int64_t)a_nx;
    if (pref && s + 1 < TC_SUB_BLOCK) a_nx = i + TC_THREADS < N ? ancv[i + TC_THREADS] : 0;
    float xe[K];
    int64_t g0 = -1;
    if (STAGED) {
      ok = umma::mbar_wait(&gbar, (uint32_t)(s & 1), TC_WAIT) && ok;
      g0 = glo[s & 1];
    }
    if (g0 >= 0) {
      const float* src = sG + (a - g0);
#pragma unroll
      for (int d = 0; d < DXP; ++d) xe[d] = (valid && d < dx) ? src[d * TC_GCAP] : 0.f;
    } else {
#pragma unroll
      for (int d = 0; d < DXP; ++d) xe[d] = (valid && d < dx) ? Xs[(size_t)d * N + a] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < DXP / 4; ++q) {
      float e4[4];
      if (noise) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int c = 4 * q + cc;
          e4[cc] = (valid && c < dx) ? noise[(size_t)c * N + i] : 0.f;
        }
      } else {
        philox_normals4<float>(seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, e4);
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) xe[DXP + 4 * q + cc] = e4[cc];
    }
    const double lin = !valid ? 0.0 : fresh ? (apf ? -(double)eta[a] : 0.0) : (double)lw[i] - lse_prev;
    // this particle's row of the A operand, split hi / lo, 16-byte chunks
#pragma unroll
    for (int k4 = 0; k4 < K / 4; ++k4) {
      float4 h, l;
      umma::split_tf32(xe[4 * k4 + 0], h.x, l.x);
      umma::split_tf32(xe[4 * k4 + 1], h.y, l.y);
      umma::split_tf32(xe[4 * k4 + 2], h.z, l.z);
      umma::split_tf32(xe[4 * k4 + 3], h.w, l.w);
      const uint32_t off = umma::kmajor_offset(tid, 4 * k4, K) >> 2;
      *reinterpret_cast<float4*>(sAh + off) = h;
      *reinterpret_cast<float4*>(sAl + off) = l;
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      // every thread has read sub-tile s's staged states: stage s + 1
      if (STAGED && s + 1 < TC_SUB_BLOCK) stage(s + 1);
      umma::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < K / 8; ++ks) {
        const uint32_t koff = (uint32_t)ks * 2 * kstride;
        const uint64_t ah = umma::desc(umma::smem_u32(sAh) + koff, kstride, mstride);
        const uint64_t al = umma::desc(umma::smem_u32(sAl) + koff, kstride, mstride);
        const uint64_t bh = umma::desc(umma::smem_u32(sBh) + koff, kstride, mstride);
        const uint64_t bl = umma::desc(umma::smem_u32(sBl) + koff, kstride, mstride);
        umma::mma_tf32(tbase, ah, bh, idesc, ks > 0 ? 1u : 0u);
        umma::mma_tf32(tbase, ah, bl, idesc, 1u);
        umma::mma_tf32(tbase, al, bh, idesc, 1u);
      }
      umma::mma_commit(&mbar);
    }
    ok = umma::mbar_wait(&mbar, (uint32_t)(s & 1), TC_WAIT) && ok;
    umma::fence_after_sync();
    float accv[NM];
#pragma unroll
    for (int c = 0; c < NM; c += 16) umma::tmem_ld16(tlane + (uint32_t)c, accv + c);
    umma::tmem_wait_ld();
    if (valid) {
      float q = 0.f;
#pragma unroll
      for (int k = 0; k < DYP; ++k) {
        const float r = sy[k] - accv[DXP + k] - sHb[k];
        q = fmaf(r, r, q);
      }
      const double lout = lin + (obs_const - 0.5 * (double)q);
      const float lst = (float)lout;
      lw[i] = lst;
#pragma unroll
      for (int d = 0; d < DXP; ++d)
        if (d < dx) Xd[(size_t)d * N + i] = accv[d] + sb[d];
      if (anc_out) anc_out[(size_t)(t - 1) * N + i] = (int32_t)(a + 1);
      acc.add((double)lst);
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  if (!ok && tid == 0) sc->status = GF_ERR_TIMEOUT;
  if (STAGED && !ok) umma::mbar_wait(&gbar, (uint32_t)((TC_SUB_BLOCK - 1) & 1), TC_WAIT);  // copies in flight
  if (tid < 32) umma::tmem_dealloc(tbase, TL::NCOLS);
  // the operand buffers are free now (every MMA has completed): in the job's
  // last block they cache the partials' exponentials for the finalise
  const bool fits = (size_t)J.ntiles * TC_SPLIT * sizeof(double) <= TL::smem_bytes;
  block_finish(J, tile, t, fresh, acc, red, part, TC_SPLIT, fits ? reinterpret_cast<double*>(smraw) : nullptr);
}

// The same propagation over 128-particle units instead of whole tiles: a grid
// of resident blocks (5 per SM at Dx=16) strides over the units of every job,
// each unit exactly one sub-tile of pf_lg_propagate_tc, and writes one partial
// per unit (TC_SUB per tile, in unit order, so the fold and tile prefixes do
// not depend on the grid).  The step's finalise runs in pf_finish_units_kernel
// after this launch, so no unit pays a device-wide fence or a counter atomic.
// With 8192 units at N = 2^20 the last round of the grid is 92% full, against
// 38% for the last wave of 1024 tile blocks; the operand-B staging and TMEM
// allocation are paid once per block (again only when the job changes).
template <int DXP, int DYP>
__global__ void __launch_bounds__(TC_THREADS, (TcLayout<DXP, DYP>::min_blocks)) pf_lg_propagate_tc_units(
    const PfJob* __restrict__ jobs, int njobs) {
  using Lay = LgLayout<DXP, DYP>;
  using TL = TcLayout<DXP, DYP>;
  constexpr int K = TL::K, NM = TL::NM;
  extern __shared__ __align__(128) unsigned char smraw[];
  float* sAh = reinterpret_cast<float*>(smraw);
  float* sAl = sAh + 128 * K;
  float* sBh = sAl + 128 * K;
  float* sBl = sBh + NM * K;
  float* sb = sBl + NM * K;
  float* sHb = sb + DXP;
  float* sy = sHb + DYP;
  __shared__ double red[32];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x;
  const PfJob& JL = jobs[njobs - 1];
  const int64_t nunits = (int64_t)TC_SUB * (JL.tile0 + JL.ntiles);
  if ((int64_t)blockIdx.x >= nunits) return;
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::fence_mbar_init();
  }
  if (tid < 32) umma::tmem_alloc(&tmem_slot, TL::NCOLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_slot;
  const uint32_t tlane = tbase + ((uint32_t)(32 * (tid >> 5)) << 16);
  const uint32_t idesc = umma::idesc_tf32(128, NM);
  const uint32_t kstride = 128, mstride = (uint32_t)(K / 4) * 128;
  bool ok = true;
  uint32_t nmma = 0;
  int jcur = -1;
  // the current job's step state (reloaded when a unit belongs to another job)
  const PfJob* J = nullptr;
  PfScalars* sc = nullptr;
  int t = 0;
  bool active = false, resamp = false, fresh = false, searched = false, apf = false;
  double lse_prev = 0.0, obs_const = 0.0;
  int64_t N = 0;
  int dx = 0;
  const float* Xs = nullptr;
  float* Xd = nullptr;
  float* lw = nullptr;
  const float* noise = nullptr;
  const int32_t* ancv = nullptr;
  int32_t* anc_out = nullptr;
  const float* eta = nullptr;
  for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int gt = (int)(u / TC_SUB);
    const int jb = find_job(jobs, njobs, gt, false);
    if (jb != jcur) {
      jcur = jb;
      J = &jobs[jb];
      sc = J->sc;
      t = sc->t + 1;
      active = t <= J->T && sc->status == 0;
      if (active) {
        resamp = sc->resample != 0;
        fresh = resamp || sc->uniform != 0;
        lse_prev = sc->lse;
        searched = J->resampler == GF_RS_MULTINOMIAL;
        N = J->N;
        dx = J->dx;
        Xs = reinterpret_cast<const float*>(J->X[(t - 1) & 1]);
        Xd = reinterpret_cast<float*>(J->X[t & 1]);
        lw = reinterpret_cast<float*>(J->lw);
        noise = J->noise ? reinterpret_cast<const float*>(J->noise) + (size_t)t * dx * N : nullptr;
        ancv = J->anc;
        anc_out = J->anc_out;
        obs_const = step_obs_const(*J, t);
        eta = reinterpret_cast<const float*>(J->eta);
        apf = resamp && eta != nullptr;
        const float* P = reinterpret_cast<const float*>(J->params) + (size_t)(t - 1) * J->pstride;
        for (int e = tid; e < NM * K; e += TC_THREADS) {
          const int n = e / K, k = e - n * K;
          const float v = P[TL::B_off + e];
          const float h = umma::to_tf32(v);
          const uint32_t off = umma::kmajor_offset(n, k, K) >> 2;
          sBh[off] = h;
          sBl[off] = umma::to_tf32(v - h);
        }
        for (int e = tid; e < DXP; e += TC_THREADS) sb[e] = P[Lay::b + e];
        const float* Y = reinterpret_cast<const float*>(J->ystep) + (size_t)(t - 1) * J->ystride;
        for (int e = tid; e < DYP; e += TC_THREADS) {
          sHb[e] = P[TL::Hb_off + e];
          sy[e] = Y[e];
        }
      }
      __syncthreads();
    }
    if (!active) continue;
    const int tile = gt - J->tile0;
    const int sub = (int)(u % TC_SUB);
    const int64_t i = (int64_t)tile * PF_TILE + sub * TC_THREADS + tid;
    const bool valid = i < N;
    int64_t a = i;
    if (valid && resamp) a = searched ? find_ancestor(*J, sc, t, i, 0, N) : (int64_t)ancv[i];
    float xe[K];
#pragma unroll
    for (int d = 0; d < DXP; ++d) xe[d] = (valid && d < dx) ? Xs[(size_t)d * N + a] : 0.f;
#pragma unroll
    for (int q = 0; q < DXP / 4; ++q) {
      float e4[4];
      if (noise) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int c = 4 * q + cc;
          e4[cc] = (valid && c < dx) ? noise[(size_t)c * N + i] : 0.f;
        }
      } else {
        philox_normals4<float>(J->seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, e4);
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) xe[DXP + 4 * q + cc] = e4[cc];
    }
    const double lin = !valid ? 0.0 : fresh ? (apf ? -(double)eta[a] : 0.0) : (double)lw[i] - lse_prev;
#pragma unroll
    for (int k4 = 0; k4 < K / 4; ++k4) {
      float4 h, l;
      umma::split_tf32(xe[4 * k4 + 0], h.x, l.x);
      umma::split_tf32(xe[4 * k4 + 1], h.y, l.y);
      umma::split_tf32(xe[4 * k4 + 2], h.z, l.z);
      umma::split_tf32(xe[4 * k4 + 3], h.w, l.w);
      const uint32_t off = umma::kmajor_offset(tid, 4 * k4, K) >> 2;
      *reinterpret_cast<float4*>(sAh + off) = h;
      *reinterpret_cast<float4*>(sAl + off) = l;
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < K / 8; ++ks) {
        const uint32_t koff = (uint32_t)ks * 2 * kstride;
        const uint64_t ah = umma::desc(umma::smem_u32(sAh) + koff, kstride, mstride);
        const uint64_t al = umma::desc(umma::smem_u32(sAl) + koff, kstride, mstride);
        const uint64_t bh = umma::desc(umma::smem_u32(sBh) + koff, kstride, mstride);
        const uint64_t bl = umma::desc(umma::smem_u32(sBl) + koff, kstride, mstride);
        umma::mma_tf32(tbase, ah, bh, idesc, ks > 0 ? 1u : 0u);
        umma::mma_tf32(tbase, ah, bl, idesc, 1u);
        umma::mma_tf32(tbase, al, bh, idesc, 1u);
      }
      umma::mma_commit(&mbar);
    }
    ok = umma::mbar_wait(&mbar, nmma & 1u, TC_WAIT) && ok;
    ++nmma;
    umma::fence_after_sync();
    float accv[NM];
#pragma unroll
    for (int c = 0; c < NM; c += 16) umma::tmem_ld16(tlane + (uint32_t)c, accv + c);
    umma::tmem_wait_ld();
    LseAcc acc;
    if (valid) {
      float q = 0.f;
#pragma unroll
      for (int k = 0; k < DYP; ++k) {
        const float r = sy[k] - accv[DXP + k] - sHb[k];
        q = fmaf(r, r, q);
      }
      const double lout = lin + (obs_const - 0.5 * (double)q);
      const float lst = (float)lout;
      lw[i] = lst;
#pragma unroll
      for (int d = 0; d < DXP; ++d)
        if (d < dx) Xd[(size_t)d * N + i] = accv[d] + sb[d];
      if (anc_out) anc_out[(size_t)(t - 1) * N + i] = (int32_t)(a + 1);
      acc.add((double)lst);
    }
    umma::fence_before_sync();
    if (!ok && tid == 0) sc->status = GF_ERR_TIMEOUT;
    // the unit's (max, sum e, sum e^2); pf_finish_units_kernel folds them
    const double M = block_max(acc.m, red);
    const double f = acc.m > -INFINITY ? exp(acc.m - M) : 0.0;
    const double S1 = block_sum(acc.s1 * f, red);
    const double S2 = block_sum(acc.s2 * f * f, red);
    if (tid == 0) {
      const size_t ps = part_stride(*J);
      double* pp = J->part + (size_t)tile * TC_SUB + sub;
      pp[0] = M;
      pp[ps] = S1;
      pp[2 * ps] = S2;
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (tid < 32) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tbase, TL::NCOLS);
  }
}

// Auxiliary particle filter, first stage of step t (particles.jl:273-357):
// log eta_i = log p(y_t | x*_i) with x*_i = A x_i + b, the mean and the mode of
// the transition MvNormal(A x + b, Q) (MeanPredictive, ModePredictive), or a
// draw A x_i + b + chol(Q) e' from it (DrawPredictive, :377-384; e' from the
// Philox stream tagged kTagLookahead, counters (i, t, q) as the propagation's),
// then the resampling decision on softmax(logw + log eta) in apf_finish.
template <typename Real, int DXP, int DYP>
__global__ void __launch_bounds__(PF_THREADS) pf_apf_lookahead(const PfJob* __restrict__ jobs, int njobs) {
  using Lay = LgLayout<DXP, DYP>;
  __shared__ Real sA[DXP * DXP], sb[DXP], sH[DYP * DXP], sy[DYP], sL[DXP * DXP];
  __shared__ double red[32];
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const int tile = blockIdx.x - J.tile0;
  const Real* P = reinterpret_cast<const Real*>(J.params) + (size_t)(t - 1) * J.pstride;
  for (int k = threadIdx.x; k < DXP * DXP; k += PF_THREADS) {
    sA[k] = P[Lay::A + k];
    sL[k] = P[Lay::L + k];
  }
  for (int k = threadIdx.x; k < DYP * DXP; k += PF_THREADS) sH[k] = P[Lay::H + k];
  for (int k = threadIdx.x; k < DXP; k += PF_THREADS) sb[k] = P[Lay::b + k];
  const Real* Y = reinterpret_cast<const Real*>(J.ystep) + (size_t)(t - 1) * J.ystride;
  for (int k = threadIdx.x; k < DYP; k += PF_THREADS) sy[k] = Y[k];
  __syncthreads();
  const int64_t N = J.N;
  const int dx = J.dx;
  const Real* Xs = reinterpret_cast<const Real*>(J.X[(t - 1) & 1]);
  const Real* lw = reinterpret_cast<const Real*>(J.lw);
  Real* eta = reinterpret_cast<Real*>(J.eta);
  const double obs_const = step_obs_const(J, t);
  const bool draw = J.lookahead_draw != 0;
  LseAcc acc;
  for (int p = 0; p < PF_PPT; ++p) {
    const int64_t i = (int64_t)tile * PF_TILE + p * PF_THREADS + threadIdx.x;
    if (i >= N) break;
    Real m[DXP];
#pragma unroll
    for (int r = 0; r < DXP; ++r) m[r] = sb[r];
#pragma unroll
    for (int c = 0; c < DXP; ++c) {
      const Real xc = c < dx ? Xs[(size_t)c * N + i] : Real(0);
#pragma unroll
      for (int r = 0; r < DXP; ++r) m[r] = fma(sA[c * DXP + r], xc, m[r]);
    }
    if (draw) {
#pragma unroll
      for (int qq = 0; qq < (DXP + 3) / 4; ++qq) {
        Real e4[4];
        philox_normals4<Real>(J.seed, (uint32_t)i, (uint32_t)t, (uint32_t)qq, e4, kTagLookahead);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int c = 4 * qq + cc;
          if (c < DXP && c < dx)
#pragma unroll
            for (int r = c; r < DXP; ++r) m[r] = fma(sL[c * DXP + r], e4[cc], m[r]);
        }
      }
    }
    Real q = 0;
#pragma unroll
    for (int k = 0; k < DYP; ++k) {
      Real r = sy[k];
#pragma unroll
      for (int c = 0; c < DXP; ++c) r = fma(-sH[c * DYP + k], m[c], r);
      q = fma(r, r, q);
    }
    const Real le = (Real)(obs_const - 0.5 * (double)q);
    eta[i] = le;
    acc.add((double)lw[i] + (double)le);
  }
  apf_finish(J, tile, t, acc, red);
}

template <typename Real, int DXP, int DYP, bool G>
PfLgKernels make_lg() {
  PfLgKernels k;
  k.dxp = DXP;
  k.dyp = DYP;
  k.prop = pf_lg_propagate<Real, DXP, DYP, G>;
  k.init = pf_lg_init<Real, DXP>;
  k.small = pf_lg_small_filter<Real, DXP, DYP, G, false>;
  k.small_means = pf_lg_small_filter<Real, DXP, DYP, G, true>;
  k.lookahead = pf_apf_lookahead<Real, DXP, DYP>;
  k.smem = sizeof(Real) * (G ? LgLayout<DXP, DYP>::smem_guided : LgLayout<DXP, DYP>::smem_boot);
  k.params_len = LgLayout<DXP, DYP>::total;
  k.off_mu0 = LgLayout<DXP, DYP>::mu0;
  k.off_L0 = LgLayout<DXP, DYP>::L0;
  if constexpr (std::is_same<Real, float>::value && !G && DXP >= 16) {
    k.prop_tc = pf_lg_propagate_tc<DXP, DYP>;
    k.tc_smem = TcLayout<DXP, DYP>::smem_bytes;
    k.tc_nm = TcLayout<DXP, DYP>::NM;
    k.tc_split = TC_SPLIT;
    k.prop_tc_units = pf_lg_propagate_tc_units<DXP, DYP>;
    k.tc_units_blocks = TcLayout<DXP, DYP>::min_blocks;
    if constexpr (DXP == 16) {
      k.prop_tc_staged = pf_lg_propagate_tc<DXP, DYP, true>;
      k.tc_staged_smem = TcSmem<DXP, DYP, true>::bytes;
    }
  }
  return k;
}

}  // namespace gf
