// gf_csmc.cu -- conditional SMC sweeps (particle Gibbs), one CTA per chain.
//
// Restates ConditionalSMC (csmc.jl:44-462) on a linear-Gaussian model with the
// bootstrap proposal.  One sweep is
//   initialise (particles.jl:36-50)         particle 1 <- ref[0], others ~ prior
//   for t = 1..T (particles.jl:147-162)
//     [ancestor sampling, csmc.jl:250-258]  a* ~ softmax(logw_i + log p(ref_t | x_i))
//     maybe_resample (resamplers.jl:155-196) ESS rule, or always (csmc.jl:261)
//     _set_ref_index! (resamplers.jl:51)    ancestor of particle 1 <- 1 (or a*)
//     propagate + update (particles.jl:228-245, 76-90): x_1 <- ref[t]
//     marginalise! (containers.jl:160-173)  ll += LSE(logw) - baseline
//   next reference: get_ancestry of a particle drawn by its final weight
//   (csmc.jl:103-113) or backward simulation (csmc.jl:378-434).
// A chain's sweeps are sequential, so the whole chain runs inside one CTA:
// particles over threads, block reductions for LSE/ESS, block scans for the
// cumulative weights, and the per-step history (states, log-weights,
// ancestors) in global memory, where the path walk and the backward pass read
// it.  Many chains run at once, one CTA each.
#include <cmath>
#include <vector>

#include "gf_common.cuh"
#include "gf_internal.hpp"

namespace gf {
namespace {

constexpr int CS_MAXN = 1024;  // particles per sweep (12-bit counter field below)
constexpr int CS_MAXD = 16;
constexpr int CS_MAXT = (1 << 20) - 1;
constexpr uint32_t kTagCsNormal = 0x43534E4Du;
constexpr uint32_t kTagCsUnif = 0x43535546u;

struct CsmcArgs {
  int dx, dy, N, T, iters, burnin, refresh, resampler, ref_given;
  double threshold, obs_const, trans_const, log_n;
  uint64_t seed;
  const double* P;      // A | b | LQ | LQi | Ht | mu0 | L0, column-major (one block per step if pstride)
  int64_t pstride;      // time-varying model: block of step t at P + (t-1) * pstride; 0: one block
  const double* consts; // time-varying: [T][2] (transition, observation) log-normalisers; else null
  const double* yt;     // [T][dy] whitened observations L_R^{-1} (y_t - c)
  const double* noise;  // nullable [chains][iters][T+1][N][dx]
  const double* unif;   // nullable [chains][iters][T+1][N+1]
  double* X;            // [chains][T+1][N][dx] states of the current sweep
  double* LW;           // [chains][T+1][N] log-weights after each update
  int32_t* ANC;         // [chains][T][N] 0-based ancestors
  double* ref;          // [chains][T+1][dx] reference trajectory (in/out)
  double* traj_out;     // nullable [chains][iters-burnin][T+1][dx]
  double* ll_out;       // nullable [chains][iters-burnin]
  int32_t* status;      // nullable [chains]
};

__host__ __device__ inline int cs_param_count(int dx, int dy) { return 4 * dx * dx + 2 * dx + dy * dx; }

// Philox counters: (sweep, chain, t << 12 | slot, tag); slot = 4 i + q for
// normals (i < 1024, q < 4) and the uniform slot (<= 1024) for uniforms.
__device__ __forceinline__ double cs_uniform(const CsmcArgs& a, int chain, int it, int t, int slot) {
  if (a.unif) return a.unif[(((size_t)chain * a.iters + it) * (a.T + 1) + t) * (a.N + 1) + slot];
  uint32_t w[4];
  philox4x32_10((uint32_t)it, (uint32_t)chain, ((uint32_t)t << 12) | (uint32_t)slot, kTagCsUnif,
                (uint32_t)a.seed, (uint32_t)(a.seed >> 32), w);
  const uint64_t bits = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}

template <int DXP>
__device__ __forceinline__ void cs_normals(const CsmcArgs& a, int chain, int it, int t, int i, double* e) {
  if (a.noise) {
    const double* p = a.noise + ((((size_t)chain * a.iters + it) * (a.T + 1) + t) * a.N + i) * a.dx;
#pragma unroll
    for (int d = 0; d < DXP; ++d) e[d] = d < a.dx ? p[d] : 0.0;
    return;
  }
#pragma unroll
  for (int q = 0; q < (DXP + 3) / 4; ++q) {
    uint32_t w[4];
    philox4x32_10((uint32_t)it, (uint32_t)chain, ((uint32_t)t << 12) | (uint32_t)(4 * i + q), kTagCsNormal,
                  (uint32_t)a.seed, (uint32_t)(a.seed >> 32), w);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      // Box-Muller on 32-bit uniforms u1 in (0,1], u2 in [0,1)
      const double u1 = ((double)w[2 * p] + 1.0) * (1.0 / 4294967296.0);
      const double u2 = (double)w[2 * p + 1] * (1.0 / 4294967296.0);
      const double r = sqrt(-2.0 * log(u1));
      double s, c;
      sincospi(2.0 * u2, &s, &c);
      if (4 * q + 2 * p < DXP) e[4 * q + 2 * p] = r * c;
      if (4 * q + 2 * p + 1 < DXP) e[4 * q + 2 * p + 1] = r * s;
    }
  }
}

// Exclusive block scan of one double per thread; `sh` holds >= 33 doubles.
__device__ __forceinline__ double cs_block_excl_scan(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  __syncthreads();
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const double s = lane < nw ? sh[lane] : 0.0;
    double si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    if (lane < nw) sh[lane] = si - s;
  }
  __syncthreads();
  return sh[wid] + inc - v;
}

// In-place inclusive cumulative sum of W[0..N) (each thread owns one run).
__device__ __forceinline__ void cs_cumsum(double* W, int N, double* sh) {
  __syncthreads();
  const int per = (N + blockDim.x - 1) / blockDim.x;
  const int k0 = min(N, (int)threadIdx.x * per), k1 = min(N, k0 + per);
  double s = 0.0;
  for (int k = k0; k < k1; ++k) s += W[k];
  double run = cs_block_excl_scan(s, sh);
  for (int k = k0; k < k1; ++k) {
    run += W[k];
    W[k] = run;
  }
  __syncthreads();
}

// StatsBase.sample(rng, Weights(w)): the first k with cumsum(w)_k >= u * sum(w).
__device__ __forceinline__ int cs_draw(const double* W, int N, double u, double* red) {
  const double target = u * W[N - 1];
  double cnt = 0.0;
  for (int k = threadIdx.x; k < N; k += blockDim.x) cnt += W[k] < target ? 1.0 : 0.0;
  const int k = (int)block_sum(cnt, red);
  return k < N ? k : N - 1;
}

// Exponentiates log-weights held in W (shifted by their maximum), then scans.
__device__ __forceinline__ void cs_exp_cumsum(double* W, int N, double* red) {
  double m = -INFINITY;
  for (int i = threadIdx.x; i < N; i += blockDim.x) m = fmax(m, W[i]);
  m = block_max(m, red);
  for (int i = threadIdx.x; i < N; i += blockDim.x) W[i] = exp(W[i] - m);
  cs_cumsum(W, N, red);
}

// log N(xn; A x + b, Q) with Q = LQ LQ^T
template <int DXP>
__device__ __forceinline__ double cs_trans_logpdf(const CsmcArgs& a, double trans_const, const double* A,
                                                  const double* b, const double* LQi, const double* xn,
                                                  const double* x) {
  const int dx = a.dx;
  double r[DXP];
#pragma unroll
  for (int i = 0; i < DXP; ++i) {
    double s = 0.0;
    if (i < dx) {
      s = xn[i] - b[i];
#pragma unroll
      for (int k = 0; k < DXP; ++k)
        if (k < dx) s -= A[i + k * dx] * x[k];
    }
    r[i] = s;
  }
  double q = 0.0;
#pragma unroll
  for (int i = 0; i < DXP; ++i) {
    double z = 0.0;
#pragma unroll
    for (int k = 0; k <= i; ++k)
      if (i < dx) z += LQi[i + k * dx] * r[k];
    q += z * z;
  }
  return trans_const - 0.5 * q;
}

// Up to dx = 4 four 256-thread chains fit on an SM (<= 64 registers).
template <int DXP>
__global__ void __launch_bounds__(256, DXP <= 4 ? 4 : 1) csmc_kernel(CsmcArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = a.N, T = a.T, dx = a.dx, dy = a.dy;
  double* W = reinterpret_cast<double*>(smraw);  // [N] weights, then cumulative weights
  double* LWP = W + N;                           // [N] log-weights after the resampling step
  int32_t* AN = reinterpret_cast<int32_t*>(LWP + N);  // [N] ancestors of the step
  __shared__ double sP[4 * CS_MAXD * CS_MAXD + 2 * CS_MAXD + CS_MAXD * CS_MAXD];
  __shared__ double red[33];
  const int chain = blockIdx.x, tid = threadIdx.x, bd = blockDim.x;
  // the model of step t (time-varying: block t-1; every block also holds the prior)
  auto load_step = [&](int t) {
    const double* src = a.P + (size_t)(t - 1) * a.pstride;
    for (int e = tid; e < cs_param_count(dx, dy); e += bd) sP[e] = src[e];
  };
  auto trans_const = [&](int t) { return a.consts ? a.consts[2 * (t - 1)] : a.trans_const; };
  auto obs_const = [&](int t) { return a.consts ? a.consts[2 * (t - 1) + 1] : a.obs_const; };
  load_step(1);
  const double* A = sP;
  const double* b = A + dx * dx;
  const double* LQ = b + dx;
  const double* LQi = LQ + dx * dx;
  const double* Ht = LQi + dx * dx;
  const double* mu0 = Ht + dy * dx;
  const double* L0 = mu0 + dx;
  double* X = a.X + (size_t)chain * (T + 1) * N * dx;
  double* LW = a.LW + (size_t)chain * (T + 1) * N;
  int32_t* ANC = a.ANC + (size_t)chain * T * N;
  double* REF = a.ref + (size_t)chain * (T + 1) * dx;
  __syncthreads();

  int status = 0;
  for (int it = 0; it < a.iters && status == 0; ++it) {
    const bool has_ref = it > 0 || a.ref_given;
    // initialise: particle 1 takes the reference state, the rest the prior
    for (int i = tid; i < N; i += bd) {
      double x[DXP];
      if (has_ref && i == 0) {
#pragma unroll
        for (int d = 0; d < DXP; ++d) x[d] = d < dx ? REF[d] : 0.0;
      } else {
        double e[DXP];
        cs_normals<DXP>(a, chain, it, 0, i, e);
#pragma unroll
        for (int r = 0; r < DXP; ++r) {
          double s = r < dx ? mu0[r] : 0.0;
#pragma unroll
          for (int k = 0; k <= r; ++k)
            if (r < dx) s += L0[r + k * dx] * e[k];
          x[r] = s;
        }
      }
#pragma unroll
      for (int d = 0; d < DXP; ++d)
        if (d < dx) X[(size_t)i * dx + d] = x[d];
      LW[i] = 0.0;  // TypelessZero weights
    }
    double ll = 0.0;
    __syncthreads();
    for (int t = 1; t <= T && status == 0; ++t) {
      const double* Xp = X + (size_t)(t - 1) * N * dx;
      const double* LWp = LW + (size_t)(t - 1) * N;
      if (a.pstride) {  // step t's model (the previous step's readers are past a barrier)
        __syncthreads();
        load_step(t);
        __syncthreads();
      }
      // LSE and ESS of the weights entering the step (resamplers.jl:179-183)
      double m = -INFINITY;
      for (int i = tid; i < N; i += bd) m = fmax(m, LWp[i]);
      m = block_max(m, red);
      double s1 = 0.0, s2 = 0.0;
      for (int i = tid; i < N; i += bd) {
        const double w = exp(LWp[i] - m);
        s1 += w;
        s2 += w * w;
      }
      s1 = block_sum(s1, red);
      s2 = block_sum(s2, red);
      const double lse = m + log(s1);
      const double ess = s1 * s1 / s2;
      const bool resamp = a.refresh == GF_CSMC_ANCESTOR || a.threshold * (double)N >= ess;
      // ancestor sampling for the reference particle (csmc.jl:250-258)
      int as_idx = 0;
      if (a.refresh == GF_CSMC_ANCESTOR && has_ref) {
        const double* xr = REF + (size_t)t * dx;
        for (int i = tid; i < N; i += bd)
          W[i] = LWp[i] + cs_trans_logpdf<DXP>(a, trans_const(t), A, b, LQi, xr, Xp + (size_t)i * dx);
        cs_exp_cumsum(W, N, red);
        as_idx = cs_draw(W, N, cs_uniform(a, chain, it, t, N), red);
      }
      if (resamp) {
        __syncthreads();
        for (int i = tid; i < N; i += bd) W[i] = exp(LWp[i] - lse);
        cs_cumsum(W, N, red);
        const double nd = (double)N, wn = W[N - 1];
        for (int i = tid; i < N; i += bd) {
          // resamplers.jl:214-238 rule: first k with n W_k > u_i (systematic,
          // stratified), first W_k >= U_i W_n (multinomial)
          double uu;
          if (a.resampler == GF_RS_SYSTEMATIC) uu = cs_uniform(a, chain, it, t, 0) + (double)i;
          else if (a.resampler == GF_RS_STRATIFIED) uu = (double)i + cs_uniform(a, chain, it, t, i);
          else uu = cs_uniform(a, chain, it, t, i) * wn;
          const bool mult = a.resampler == GF_RS_MULTINOMIAL;
          int lo = 0, hi = N;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const bool right = mult ? (W[mid] >= uu) : (W[mid] * nd > uu);
            if (right) hi = mid;
            else lo = mid + 1;
          }
          AN[i] = lo < N ? lo : N - 1;
          LWP[i] = 0.0;
        }
      } else {
        for (int i = tid; i < N; i += bd) {
          AN[i] = i;
          LWP[i] = LWp[i];
        }
      }
      const double base = resamp ? a.log_n : lse;
      __syncthreads();
      if (tid == 0 && has_ref) AN[0] = as_idx;  // _set_ref_index!, or the sampled ancestor
      __syncthreads();
      // propagate and weight
      const double* y = a.yt + (size_t)(t - 1) * dy;
      double* Xt = X + (size_t)t * N * dx;
      double* LWt = LW + (size_t)t * N;
      double mloc = -INFINITY;
      for (int i = tid; i < N; i += bd) {
        double x[DXP];
        if (has_ref && i == 0) {
#pragma unroll
          for (int d = 0; d < DXP; ++d) x[d] = d < dx ? REF[(size_t)t * dx + d] : 0.0;
        } else {
          const double* xp = Xp + (size_t)AN[i] * dx;
          double xa[DXP], e[DXP];
#pragma unroll
          for (int d = 0; d < DXP; ++d) xa[d] = d < dx ? xp[d] : 0.0;
          cs_normals<DXP>(a, chain, it, t, i, e);
#pragma unroll
          for (int r = 0; r < DXP; ++r) {
            double s = 0.0;
            if (r < dx) {
              s = b[r];
#pragma unroll
              for (int k = 0; k < DXP; ++k)
                if (k < dx) s += A[r + k * dx] * xa[k];
#pragma unroll
              for (int k = 0; k <= r; ++k) s += LQ[r + k * dx] * e[k];
            }
            x[r] = s;
          }
        }
        double q = 0.0;
        for (int j = 0; j < dy; ++j) {
          double r = y[j];
#pragma unroll
          for (int k = 0; k < DXP; ++k)
            if (k < dx) r -= Ht[j + k * dy] * x[k];
          q += r * r;
        }
        const double lw = LWP[i] + obs_const(t) - 0.5 * q;
#pragma unroll
        for (int d = 0; d < DXP; ++d)
          if (d < dx) Xt[(size_t)i * dx + d] = x[d];
        LWt[i] = lw;
        ANC[(size_t)(t - 1) * N + i] = AN[i];
        mloc = fmax(mloc, lw);
      }
      const double M = block_max(mloc, red);
      double s = 0.0;
      for (int i = tid; i < N; i += bd) s += exp(LWt[i] - M);
      s = block_sum(s, red);
      const double lse_new = M + log(s);
      if (!(lse_new > -INFINITY) || isnan(lse_new)) status = GF_ERR_ARG;  // weights vanished
      ll += lse_new - base;
      __syncthreads();
    }
    if (status) break;
    // next reference trajectory
    for (int i = tid; i < N; i += bd) W[i] = LW[(size_t)T * N + i];
    cs_exp_cumsum(W, N, red);
    int k = cs_draw(W, N, cs_uniform(a, chain, it, 0, N), red);
    __syncthreads();
    if (a.refresh != GF_CSMC_BACKWARD) {
      // get_ancestry (containers.jl:587-611 / 421-440): walk the ancestors back
      if (tid == 0)
        for (int t = T; t >= 0; --t) {
          for (int d = 0; d < dx; ++d) REF[(size_t)t * dx + d] = X[((size_t)t * N + k) * dx + d];
          if (t > 0) k = ANC[(size_t)(t - 1) * N + k];
        }
      __syncthreads();
    } else {
      // backward simulation (csmc.jl:398-431)
      if (tid < dx) REF[(size_t)T * dx + tid] = X[((size_t)T * N + k) * dx + tid];
      __syncthreads();
      for (int t = T - 1; t >= 0; --t) {
        const double* xn = REF + (size_t)(t + 1) * dx;
        if (a.pstride) {  // the transition from x_t to x_{t+1} is step t+1's
          __syncthreads();
          load_step(t + 1);
          __syncthreads();
        }
        for (int i = tid; i < N; i += bd)
          W[i] = LW[(size_t)t * N + i] +
                 cs_trans_logpdf<DXP>(a, trans_const(t + 1), A, b, LQi, xn, X + ((size_t)t * N + i) * dx);
        cs_exp_cumsum(W, N, red);
        k = cs_draw(W, N, cs_uniform(a, chain, it, t + 1, N), red);
        if (tid < dx) REF[(size_t)t * dx + tid] = X[((size_t)t * N + k) * dx + tid];
        __syncthreads();
      }
    }
    if (it >= a.burnin) {
      const size_t kk = (size_t)chain * (a.iters - a.burnin) + (it - a.burnin);
      if (a.traj_out)
        for (int e = tid; e < (T + 1) * dx; e += bd) a.traj_out[kk * (T + 1) * dx + e] = REF[e];
      if (a.ll_out && tid == 0) a.ll_out[kk] = ll;
    }
    __syncthreads();
  }
  if (tid == 0 && a.status) a.status[chain] = status;
}

template <int DXP>
void launch_csmc(const CsmcArgs& a, int chains, int threads, size_t smem, cudaStream_t s) {
  csmc_kernel<DXP><<<chains, threads, smem, s>>>(a);
}

}  // namespace

extern "C" int32_t gf_csmc_max_particles(void) { return CS_MAXN; }

static gf_status csmc_run_impl(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                               const gf_csmc_config* cfg, int32_t T, const double* ys, int32_t chains,
                               int32_t iters, int32_t burnin, int32_t ref_given, const double* noise,
                               const double* uniforms, int32_t memspace, gf_csmc_out* out) {
  if (!ctx) return GF_ERR_ARG;
  if (!m || !cfg || !ys || !out || !out->ref) return set_err(ctx, GF_ERR_ARG, "null argument");
  const int dx = m->dx, dy = m->dy, N = cfg->N;
  if (dx < 1 || dy < 1 || dx > CS_MAXD || dy > CS_MAXD)
    return set_err(ctx, GF_ERR_DIM, "CSMC supports 1 <= dx, dy <= %d (got %d, %d)", CS_MAXD, dx, dy);
  if (N < 1 || N > CS_MAXN) return set_err(ctx, GF_ERR_ARG, "CSMC needs 1 <= N <= %d (got %d)", CS_MAXN, N);
  if (T < 1 || T > CS_MAXT) return set_err(ctx, GF_ERR_ARG, "CSMC needs 1 <= T <= %d", CS_MAXT);
  if (chains < 1 || iters < 1 || burnin < 0 || burnin >= iters)
    return set_err(ctx, GF_ERR_ARG, "need chains >= 1, iters >= 1 and 0 <= burnin < iters");
  if (cfg->refresh < GF_CSMC_NONE || cfg->refresh > GF_CSMC_BACKWARD)
    return set_err(ctx, GF_ERR_ARG, "unknown refresh %d", cfg->refresh);
  if (cfg->resampler < GF_RS_SYSTEMATIC || cfg->resampler > GF_RS_MULTINOMIAL)
    return set_err(ctx, GF_ERR_ARG, "unknown resampler %d", cfg->resampler);
  if (!std::isfinite(cfg->threshold)) return set_err(ctx, GF_ERR_ARG, "threshold must be finite");
  if (memspace != GF_MEM_HOST && memspace != GF_MEM_DEVICE) return set_err(ctx, GF_ERR_ARG, "bad memspace");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;

  const bool tv = param_steps != 1;
  if (tv && param_steps < T) return set_err(ctx, GF_ERR_ARG, "%d parameter steps for T = %d", param_steps, T);
  const int nblk = tv ? T : 1;
  // model factors (FP64, host), one block per step of a time-varying model
  // (calc_params(dyn, t), calc_params(obs, t)); each block repeats the prior
  std::vector<double> L0(dx * dx);
  if (chol_lower(dx, m->Sigma0, L0.data())) return set_err(ctx, GF_ERR_NOT_PD, "Sigma0 is not positive definite");
  std::vector<double> yh((size_t)T * dy), yt((size_t)T * dy);
  if (memspace == GF_MEM_DEVICE) {
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(yh.data(), ys, sizeof(double) * yh.size(), cudaMemcpyDeviceToHost, s));
    GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  } else {
    std::copy(ys, ys + yh.size(), yh.begin());
  }
  std::vector<double> P, consts;
  P.reserve((size_t)nblk * cs_param_count(dx, dy));
  double ldr = 0.0, ldq = 0.0;
  for (int k = 0; k < nblk; ++k) {
    const double *mA = m->A + (size_t)k * dx * dx, *mb = m->b + (size_t)k * dx, *mQ = m->Q + (size_t)k * dx * dx;
    const double *mH = m->H + (size_t)k * dy * dx, *mc = m->c + (size_t)k * dy, *mR = m->R + (size_t)k * dy * dy;
    std::vector<double> LQ(dx * dx), LQi(dx * dx), LR(dy * dy), LRi(dy * dy), Ht(dy * dx);
    if (chol_lower(dx, mQ, LQ.data())) return set_err(ctx, GF_ERR_NOT_PD, "Q of step %d is not positive definite", k + 1);
    if (chol_lower(dy, mR, LR.data())) return set_err(ctx, GF_ERR_NOT_PD, "R of step %d is not positive definite", k + 1);
    tri_inv_lower(dx, LQ.data(), LQi.data());
    tri_inv_lower(dy, LR.data(), LRi.data());
    matmul(dy, dy, dx, LRi.data(), mH, Ht.data());
    P.insert(P.end(), mA, mA + dx * dx);
    P.insert(P.end(), mb, mb + dx);
    P.insert(P.end(), LQ.begin(), LQ.end());
    P.insert(P.end(), LQi.begin(), LQi.end());
    P.insert(P.end(), Ht.begin(), Ht.end());
    P.insert(P.end(), m->mu0, m->mu0 + dx);
    P.insert(P.end(), L0.begin(), L0.end());
    // whitened observations of the steps this block serves
    for (int t = (tv ? k : 0); t < (tv ? k + 1 : T); ++t)
      for (int r = 0; r < dy; ++r) {
        double v = 0.0;
        for (int j = 0; j <= r; ++j) v += LRi[r + j * dy] * (yh[(size_t)t * dy + j] - mc[j]);
        yt[(size_t)t * dy + r] = v;
      }
    ldr = 0.0;
    ldq = 0.0;
    for (int i = 0; i < dy; ++i) ldr += std::log(LR[i + i * dy]);
    for (int i = 0; i < dx; ++i) ldq += std::log(LQ[i + i * dx]);
    if (tv) {
      consts.push_back(-ldq - 0.5 * dx * GF_LOG2PI);
      consts.push_back(-ldr - 0.5 * dy * GF_LOG2PI);
    }
  }

  // device buffers
  std::vector<DevBuf> bufs;
  struct Cleanup {
    gf_ctx* c;
    std::vector<DevBuf>* v;
    ~Cleanup() {
      cudaStreamSynchronize(c->stream);
      for (auto& b : *v) dev_free(c, b.p, b.bytes);
    }
  } cleanup{ctx, &bufs};
  auto get = [&](size_t bytes, void** p) -> gf_status {
    gf_status st = dev_alloc(ctx, bytes, p);
    if (!st) bufs.push_back({*p, bytes});
    return st;
  };
  const size_t steps = (size_t)T + 1, keep = (size_t)(iters - burnin);
  const size_t refb = sizeof(double) * chains * steps * dx;
  const size_t nz = sizeof(double) * chains * (size_t)iters * steps * N * dx;
  const size_t nu = sizeof(double) * chains * (size_t)iters * steps * (N + 1);
  gf_status st;
  void *dP, *dyt, *dX, *dLW, *dANC, *dC = nullptr;
  if (tv && (st = get(sizeof(double) * consts.size(), &dC))) return st;
  if ((st = get(sizeof(double) * P.size(), &dP)) || (st = get(sizeof(double) * yt.size(), &dyt)) ||
      (st = get(sizeof(double) * chains * steps * N * dx, &dX)) ||
      (st = get(sizeof(double) * chains * steps * N, &dLW)) ||
      (st = get(sizeof(int32_t) * chains * (size_t)T * N, &dANC)))
    return st;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dP, P.data(), sizeof(double) * P.size(), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dyt, yt.data(), sizeof(double) * yt.size(), cudaMemcpyHostToDevice, s));
  if (dC) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dC, consts.data(), sizeof(double) * consts.size(), cudaMemcpyHostToDevice, s));
  CsmcArgs a{};
  a.pstride = tv ? cs_param_count(dx, dy) : 0;
  a.consts = (const double*)dC;
  a.dx = dx;
  a.dy = dy;
  a.N = N;
  a.T = T;
  a.iters = iters;
  a.burnin = burnin;
  a.refresh = cfg->refresh;
  a.resampler = cfg->resampler;
  a.ref_given = ref_given != 0;
  a.threshold = cfg->threshold;
  a.obs_const = -ldr - 0.5 * dy * GF_LOG2PI;
  a.trans_const = -ldq - 0.5 * dx * GF_LOG2PI;
  a.log_n = std::log((double)N);
  a.seed = cfg->seed;
  a.P = (const double*)dP;
  a.yt = (const double*)dyt;
  a.X = (double*)dX;
  a.LW = (double*)dLW;
  a.ANC = (int32_t*)dANC;
  if (memspace == GF_MEM_DEVICE) {
    a.noise = noise;
    a.unif = uniforms;
    a.ref = out->ref;
    a.traj_out = out->trajectories;
    a.ll_out = out->ll;
    a.status = out->status;
  } else {
    void* p;
    if (noise) {
      if ((st = get(nz, &p))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, noise, nz, cudaMemcpyHostToDevice, s));
      a.noise = (const double*)p;
    }
    if (uniforms) {
      if ((st = get(nu, &p))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, uniforms, nu, cudaMemcpyHostToDevice, s));
      a.unif = (const double*)p;
    }
    if ((st = get(refb, &p))) return st;
    if (ref_given) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, out->ref, refb, cudaMemcpyHostToDevice, s));
    a.ref = (double*)p;
    if (out->trajectories) {
      if ((st = get(sizeof(double) * chains * keep * steps * dx, &p))) return st;
      a.traj_out = (double*)p;
    }
    if (out->ll) {
      if ((st = get(sizeof(double) * chains * keep, &p))) return st;
      a.ll_out = (double*)p;
    }
  }
  int32_t* dstatus = a.status;
  if (!dstatus) {
    void* p;
    if ((st = get(sizeof(int32_t) * chains, &p))) return st;
    dstatus = (int32_t*)p;
    a.status = dstatus;
  }
  const int threads = std::min(256, std::max(32, (N + 31) / 32 * 32));
  const size_t smem = (size_t)N * (2 * sizeof(double) + sizeof(int32_t));
  const int dxp = dx <= 1 ? 1 : dx <= 2 ? 2 : dx <= 4 ? 4 : dx <= 8 ? 8 : 16;
  switch (dxp) {
    case 1: launch_csmc<1>(a, chains, threads, smem, s); break;
    case 2: launch_csmc<2>(a, chains, threads, smem, s); break;
    case 4: launch_csmc<4>(a, chains, threads, smem, s); break;
    case 8: launch_csmc<8>(a, chains, threads, smem, s); break;
    default: launch_csmc<16>(a, chains, threads, smem, s); break;
  }
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  std::vector<int32_t> hs(chains);
  if (memspace == GF_MEM_HOST) {
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->ref, a.ref, refb, cudaMemcpyDeviceToHost, s));
    if (out->trajectories)
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->trajectories, a.traj_out, sizeof(double) * chains * keep * steps * dx,
                                         cudaMemcpyDeviceToHost, s));
    if (out->ll)
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->ll, a.ll_out, sizeof(double) * chains * keep, cudaMemcpyDeviceToHost, s));
  }
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(hs.data(), dstatus, sizeof(int32_t) * chains, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (memspace == GF_MEM_HOST && out->status) std::copy(hs.begin(), hs.end(), out->status);
  for (int c = 0; c < chains; ++c)
    if (hs[c]) return set_err(ctx, hs[c], "chain %d: particle weights degenerated (all zero or NaN)", c);
  return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" gf_status gf_csmc_run(gf_ctx* ctx, const gf_lg_model* m, const gf_csmc_config* cfg, int32_t T,
                                 const double* ys, int32_t chains, int32_t iters, int32_t burnin,
                                 int32_t ref_given, const double* noise, const double* uniforms,
                                 int32_t memspace, gf_csmc_out* out) {
  return csmc_run_impl(ctx, m, 1, cfg, T, ys, chains, iters, burnin, ref_given, noise, uniforms, memspace, out);
}

extern "C" gf_status gf_csmc_run_tv(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                                    const gf_csmc_config* cfg, int32_t T, const double* ys, int32_t chains,
                                    int32_t iters, int32_t burnin, int32_t ref_given, const double* noise,
                                    const double* uniforms, int32_t memspace, gf_csmc_out* out) {
  return csmc_run_impl(ctx, m, param_steps, cfg, T, ys, chains, iters, burnin, ref_given, noise, uniforms,
                       memspace, out);
}
