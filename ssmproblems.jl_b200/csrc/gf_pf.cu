// gf_pf.cu -- particle-filter host helpers: kernel registry, model factors, launches.
//
// Restates GeneralisedFilters' PF (particles.jl:36-90,147-245) for
// LinearGaussianStateSpaceModel: state x_t = A x_{t-1} + b + L_Q e (BF) or the
// linear-Gaussian proposal x_t = M x_{t-1} + v_t + L_q e with weight increment
// log p(x_t|x_{t-1}) - log q(x_t|x_{t-1},y_t) (GFTest OptimalProposal /
// OverdispersedProposal).  Observation log-density uses the whitened form
// -1/2 |L_R^{-1}(y - c) - (L_R^{-1}H) x|^2 + const, the same quantity as
// logpdf(MvNormal(Hx + c, R), y) (models/linear_gaussian.jl:85-90).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>

#include "gf_internal.hpp"
#include "gf_pf_lg.cuh"

namespace gf {

// Per-step vectors: ytil_t = L_R^{-1}(y_t - c), v_t = K (y_t - c) + vb.
template <typename Real>
__global__ void pf_prep_ystep(const PfJob* __restrict__ job, int T, int dx, int dy, int dxp,
                              int dyp, const double* __restrict__ pp, Real* __restrict__ out) {
  // pp: LRinv[dy*dy] | c[dy] | K[dx*dy] | vb[dx]
  const double* ys = job->ys;
  const int32_t pps = job->ppstride;  // time-varying model: per-step factor blocks
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    const double* LRi = pp + (size_t)t * pps;
    const double* c = LRi + dy * dy;
    const double* K = c + dy;
    const double* vb = K + dx * dy;
    const double* y = ys + (size_t)t * dy;
    Real* o = out + (size_t)t * (dyp + dxp);
    for (int k = 0; k < dyp; ++k) {
      double s = 0.0;
      if (k < dy)
        for (int j = 0; j <= k; ++j) s += LRi[k + j * dy] * (y[j] - c[j]);
      o[k] = (Real)s;
    }
    for (int r = 0; r < dxp; ++r) {
      double s = 0.0;
      if (r < dx) {
        s = vb[r];
        for (int j = 0; j < dy; ++j) s += K[r + j * dx] * (y[j] - c[j]);
      }
      o[dyp + r] = (Real)s;
    }
  }
}

// Initial scalars + step-1 decision outputs (uniform TypelessZero weights).
__global__ void pf_init_scalars(PfJob* jobs, int njobs, const double* ess1, const int8_t* res1) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  PfJob& J = jobs[j];
  PfScalars* sc = J.sc;
  sc->lse = J.log_n;
  sc->ll = 0.0;
  sc->ess = ess1[j];
  sc->u0 = J.unif ? J.unif[0] : philox_uniform(J.seed, 0u, 1u);
  sc->wn = 1.0;
  sc->t = 0;
  sc->resample = res1[j];
  sc->uniform = 1;
  sc->status = 0;
  sc->counter = 0;
  sc->scan_tile = 0;
  sc->clamps = 0;
  sc->mcounter = 0;
  sc->lse_aux = 0.0;
  sc->base_adj = 0.0;
  if (J.ess_steps) J.ess_steps[0] = ess1[j];
  if (J.res_steps) J.res_steps[0] = res1[j];
}

// Final outputs: normalised log-weights (lw - LSE), states, ll and clamps.
template <typename Real>
__global__ void pf_finish_kernel(const PfJob* __restrict__ jobs) {
  const PfJob& J = jobs[0];
  const Real* lw = reinterpret_cast<const Real*>(J.lw);
  const double lse = J.sc->lse;
  const int tcur = J.sc->t;
  const Real* X = reinterpret_cast<const Real*>(J.X[tcur & 1]);
  Real* so = reinterpret_cast<Real*>(J.states_out);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < J.N;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (J.logw_out) J.logw_out[i] = (double)lw[i] - lse;
    if (so)
      for (int d = 0; d < J.width; ++d) so[(size_t)d * J.N + i] = X[(size_t)d * J.N + i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (J.ll_out) *J.ll_out = J.sc->ll;
    if (J.clamps_out) *J.clamps_out = J.sc->clamps;
  }
}

// DenseAncestorCallback (callbacks.jl:47-81): after initialisation (t = 0)
// and after every update, the states of step t and, for t >= 1, the
// normalised log-weights the PostUpdate callback sees (marginalise! has
// subtracted the LSE, containers.jl:160-173).
template <typename Real>
__global__ void pf_record_kernel(const PfJob* __restrict__ jobs) {
  const PfJob& J = jobs[0];
  const PfScalars* sc = J.sc;
  if (sc->status != 0) return;
  const int t = sc->t;
  const int64_t N = J.N;
  const Real* X = reinterpret_cast<const Real*>(J.X[t & 1]);
  const Real* lw = reinterpret_cast<const Real*>(J.lw);
  Real* H = J.hist ? reinterpret_cast<Real*>(J.hist) + (size_t)t * J.width * N : nullptr;
  const double lse = sc->lse;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    if (H)
      for (int d = 0; d < J.width; ++d) H[(size_t)d * N + i] = X[(size_t)d * N + i];
    if (J.lwh && t >= 1) J.lwh[(size_t)(t - 1) * N + i] = (double)lw[i] - lse;
  }
}

// get_ancestry(container, i) (containers.jl:421-440) for M final particles.
template <typename Real>
__global__ void pf_dense_ancestry_kernel(int T, int64_t N, int dx, const Real* __restrict__ hist,
                                         const int32_t* __restrict__ anc, int64_t M,
                                         const int32_t* __restrict__ idx, Real* __restrict__ out,
                                         int32_t* __restrict__ bad) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M; k += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = idx ? (int64_t)idx[k] - 1 : k;
    for (int t = T; t >= 0; --t) {
      if (a < 0 || a >= N) {  // an index outside 1..N: report it, write nothing more
        atomicExch(bad, 1);
        break;
      }
      for (int d = 0; d < dx; ++d) out[((size_t)t * dx + d) * M + k] = hist[((size_t)t * dx + d) * N + a];
      if (t > 0) a = (int64_t)anc[(size_t)(t - 1) * N + a] - 1;
    }
  }
}

// The step's finalise after pf_lg_propagate_tc_units: one block of 1024
// threads per job folds the job's unit partials (finish_step, as the last
// propagate block does in the tile kernels).
constexpr int UNITS_FINISH_THREADS = 1024;
__global__ void __launch_bounds__(UNITS_FINISH_THREADS) pf_finish_units_kernel(const PfJob* __restrict__ jobs,
                                                                               int njobs) {
  __shared__ double red[32];
  __shared__ unsigned long long s_wsum[32];
  __shared__ int s_res;
  const PfJob& J = jobs[blockIdx.x];
  PfScalars* sc = J.sc;
  const int t = sc->t + 1;
  if (t > J.T || sc->status != 0) return;
  const bool fresh = sc->resample != 0 || sc->uniform != 0;
  finish_step(BlockSync(), J, t, fresh, TC_SUB, red, s_wsum, &s_res);
}

void launch_finish_units(gf_ctx* ctx, const PfJob* jobs_dev, int njobs) {
  pf_finish_units_kernel<<<njobs, UNITS_FINISH_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
}

void launch_record(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int64_t N) {
  int blocks = (int)std::min<int64_t>((N + 255) / 256, 8 * (int64_t)ctx->num_sms);
  if (dbl) pf_record_kernel<double><<<blocks, 256, 0, ctx->stream>>>(jobs_dev);
  else pf_record_kernel<float><<<blocks, 256, 0, ctx->stream>>>(jobs_dev);
}

// -------------------------------------------------------- kernel registry
// Instantiations live in gf_pf_inst_*.cu so they compile in parallel.
void register_lg_f32_small(std::vector<PfLgKernels>& v, bool guided);
void register_lg_f32_16(std::vector<PfLgKernels>& v, bool guided);
void register_lg_f32_32(std::vector<PfLgKernels>& v, bool guided);
void register_lg_f32_64(std::vector<PfLgKernels>& v, bool guided);
void register_lg_f64(std::vector<PfLgKernels>& v, bool guided);

static std::vector<PfLgKernels> lg_table(bool dbl, bool guided) {
  std::vector<PfLgKernels> v;
  if (dbl) {
    register_lg_f64(v, guided);
  } else {
    register_lg_f32_small(v, guided);
    register_lg_f32_16(v, guided);
    register_lg_f32_32(v, guided);
    register_lg_f32_64(v, guided);
  }
  return v;
}

bool pick_lg_kernels(bool dbl, bool guided, int dx, int dy, PfLgKernels* out) {
  for (auto& k : lg_table(dbl, guided))
    if (k.dxp >= dx && k.dyp >= dy) {
      *out = k;
      return true;
    }
  return false;
}

// Julia's pairwise sum of N copies of (1/N)^2 (Base.mapreduce_impl, block
// 1024): the ESS the reference sees for uniform weights (resamplers.jl:181).
static double pairwise_sq_uniform(int64_t n, double v, std::map<int64_t, double>& memo) {
  auto it = memo.find(n);
  if (it != memo.end()) return it->second;
  double r;
  if (n == 1) r = v * v;
  else if (n - 1 < 1024) {
    r = v * v + v * v;
    for (int64_t i = 2; i < n; ++i) r += v * v;
  } else {
    int64_t left = ((n - 1) >> 1) + 1;
    r = pairwise_sq_uniform(left, v, memo) + pairwise_sq_uniform(n - left, v, memo);
  }
  memo[n] = r;
  return r;
}

double uniform_ess(int64_t n) {
  std::map<int64_t, double> memo;
  return 1.0 / pairwise_sq_uniform(n, 1.0 / (double)n, memo);
}

void launch_scan(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_stiles) {
  ProfScope ps(ctx, KC_SCAN);
  if (dbl) pf_scan_kernel<double><<<total_stiles, SCAN_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
  else pf_scan_kernel<float><<<total_stiles, SCAN_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
}

void launch_resample(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_tiles) {
  {
    ProfScope ps(ctx, KC_SCAN);
    if (dbl) pf_resample_kernel<double><<<total_tiles, PF_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
    else pf_resample_kernel<float><<<total_tiles, PF_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
  }
  ProfScope ps(ctx, KC_FILL);
  pf_fill_ancestors_kernel<<<total_tiles, PF_THREADS, 0, ctx->stream>>>(jobs_dev, njobs);
}

void launch_init_scalars(gf_ctx* ctx, PfJob* jobs_dev, int njobs, const double* ess1,
                         const int8_t* res1) {
  pf_init_scalars<<<(njobs + 127) / 128, 128, 0, ctx->stream>>>(jobs_dev, njobs, ess1, res1);
}


// Weighted means: the job's means_out is read inside the kernel through `jobs`.
template <typename Real>
__global__ void pf_means_entry(const PfJob* __restrict__ jobs, int njobs, double* mpart, int mdim) {
  if (jobs[0].means_out == nullptr) return;
  pf_means_kernel<Real>(jobs, njobs, mpart, jobs[0].means_out, mdim);
}

void launch_means(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_tiles,
                  double* mpart, int mdim) {
  if (dbl) pf_means_entry<double><<<total_tiles, PF_THREADS, 0, ctx->stream>>>(jobs_dev, njobs, mpart, mdim);
  else pf_means_entry<float><<<total_tiles, PF_THREADS, 0, ctx->stream>>>(jobs_dev, njobs, mpart, mdim);
}

void launch_finish(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int64_t N) {
  int blocks = (int)std::min<int64_t>((N + 255) / 256, 4 * 148);
  if (dbl) pf_finish_kernel<double><<<blocks, 256, 0, ctx->stream>>>(jobs_dev);
  else pf_finish_kernel<float><<<blocks, 256, 0, ctx->stream>>>(jobs_dev);
}

void launch_prep(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int T, int dx, int dy, int dxp,
                 int dyp, const double* pp, void* out) {
  ProfScope ps(ctx, KC_PREP);
  int blocks = std::max(1, std::min(148, (T + 127) / 128));
  if (dbl) pf_prep_ystep<double><<<blocks, 128, 0, ctx->stream>>>(job_dev, T, dx, dy, dxp, dyp, pp, (double*)out);
  else pf_prep_ystep<float><<<blocks, 128, 0, ctx->stream>>>(job_dev, T, dx, dy, dxp, dyp, pp, (float*)out);
}

// ---------------------------------------------------------------- the plan
// Model factors (FP64, host): L (noise factor of the proposal), Ht = L_R^{-1} H,
// M, Qi = L_Q^{-1}, L0 = chol(Sigma0), the prep block and the constants.
gf_status build_lg_factors(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg,
                           LgFactors* f) {
  const int dx = m->dx, dy = m->dy;
  f->dx = dx;
  f->dy = dy;
  std::vector<double> LQ(dx * dx), LR(dy * dy), L0(dx * dx);
  if (chol_lower(dx, m->Q, LQ.data())) return set_err(ctx, GF_ERR_NOT_PD, "Q is not positive definite");
  if (chol_lower(dy, m->R, LR.data())) return set_err(ctx, GF_ERR_NOT_PD, "R is not positive definite");
  if (chol_lower(dx, m->Sigma0, L0.data()))
    return set_err(ctx, GF_ERR_NOT_PD, "Sigma0 is not positive definite");
  std::vector<double> LRi(dy * dy), Ht(dy * dx);
  tri_inv_lower(dy, LR.data(), LRi.data());
  matmul(dy, dy, dx, LRi.data(), m->H, Ht.data());
  double ldr = 0.0;
  for (int i = 0; i < dy; ++i) ldr += std::log(LR[i + i * dy]);
  f->obs_const = -ldr - 0.5 * dy * GF_LOG2PI;
  f->A.assign(m->A, m->A + dx * dx);
  f->b.assign(m->b, m->b + dx);
  f->Ht = Ht;
  f->mu0.assign(m->mu0, m->mu0 + dx);
  f->L0 = L0;
  f->LRi = LRi;
  f->c.assign(m->c, m->c + dy);
  f->K.assign(dx * dy, 0.0);
  f->vb.assign(m->b, m->b + dx);
  f->M.assign(m->A, m->A + dx * dx);
  f->Qi.assign(dx * dx, 0.0);
  f->prop_const = 0.0;
  f->L = LQ;
  if (cfg->proposal == GF_PROP_BOOTSTRAP) return GF_OK;
  tri_inv_lower(dx, LQ.data(), f->Qi.data());
  std::vector<double> Lq(dx * dx);
  if (cfg->proposal == GF_PROP_OVERDISPERSED) {
    std::vector<double> kQ(dx * dx);
    for (int i = 0; i < dx * dx; ++i) kQ[i] = cfg->proposal_k * m->Q[i];
    if (chol_lower(dx, kQ.data(), Lq.data()))
      return set_err(ctx, GF_ERR_NOT_PD, "k*Q is not positive definite");
  } else if (cfg->proposal == GF_PROP_OPTIMAL) {
    // kalman_update(MvNormal(A x + b, Q), (H, c, R), y) (GFTest/proposals.jl:20-31,
    // kalman_gradient.jl:12-23): the gain and covariance do not depend on x.
    std::vector<double> HL(dy * dx), S(dy * dy), LS(dy * dy), QHt(dx * dy), K(dx * dy);
    matmul(dy, dx, dx, m->H, LQ.data(), HL.data());
    for (int i = 0; i < dy; ++i)
      for (int j = 0; j < dy; ++j) {
        double s = 0.0;
        for (int p = 0; p < dx; ++p) s += HL[i + p * dy] * HL[j + p * dy];
        S[i + j * dy] = s + m->R[i + j * dy];
      }
    if (chol_lower(dy, S.data(), LS.data()))
      return set_err(ctx, GF_ERR_NOT_PD, "innovation covariance not positive definite");
    for (int r = 0; r < dx; ++r) {
      std::vector<double> w(dy);
      for (int j = 0; j < dy; ++j) {
        double s = 0.0;
        for (int p = 0; p < dx; ++p) s += m->Q[r + p * dx] * m->H[j + p * dy];
        w[j] = s;
      }
      for (int i = 0; i < dy; ++i) {
        double s = w[i];
        for (int k = 0; k < i; ++k) s -= LS[i + k * dy] * w[k];
        w[i] = s / LS[i + i * dy];
      }
      for (int i = dy - 1; i >= 0; --i) {
        double s = w[i];
        for (int k = i + 1; k < dy; ++k) s -= LS[k + i * dy] * w[k];
        w[i] = s / LS[i + i * dy];
      }
      for (int j = 0; j < dy; ++j) K[r + j * dx] = w[j];
    }
    std::vector<double> IKH(dx * dx), T1(dx * dx), Sr(dx * dx), KL(dx * dy);
    matmul(dx, dy, dx, K.data(), m->H, IKH.data());
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i) IKH[i + j * dx] = (i == j ? 1.0 : 0.0) - IKH[i + j * dx];
    matmul(dx, dx, dx, IKH.data(), LQ.data(), T1.data());
    matmul(dx, dy, dy, K.data(), LR.data(), KL.data());
    for (int i = 0; i < dx; ++i)
      for (int j = 0; j < dx; ++j) {
        double s = 0.0;
        for (int p = 0; p < dx; ++p) s += T1[i + p * dx] * T1[j + p * dx];
        for (int p = 0; p < dy; ++p) s += KL[i + p * dx] * KL[j + p * dx];
        Sr[i + j * dx] = s;
      }
    for (int j = 0; j < dx; ++j)
      for (int i = j + 1; i < dx; ++i) Sr[i + j * dx] = Sr[j + i * dx];  // Symmetric(upper)
    if (chol_lower(dx, Sr.data(), Lq.data()))
      return set_err(ctx, GF_ERR_NOT_PD, "proposal covariance not positive definite");
    matmul(dx, dx, dx, IKH.data(), m->A, f->M.data());
    std::vector<double> vb(dx);
    for (int r = 0; r < dx; ++r) {
      double s = 0.0;
      for (int p = 0; p < dx; ++p) s += IKH[r + p * dx] * m->b[p];
      vb[r] = s;
    }
    f->vb = vb;
    f->K = K;
  } else {
    return set_err(ctx, GF_ERR_ARG, "unknown proposal %d", cfg->proposal);
  }
  double lq = 0.0, lQ = 0.0;
  for (int i = 0; i < dx; ++i) {
    lq += std::log(Lq[i + i * dx]);
    lQ += std::log(LQ[i + i * dx]);
  }
  f->prop_const = lq - lQ;
  f->L = Lq;
  return GF_OK;
}

template <typename Real>
static void pack_lg_params(const LgFactors& f, int DXP, int DYP, std::vector<char>& out) {
  // mirrors LgLayout
  const int dx = f.dx, dy = f.dy;
  const int oA = 0, oL = DXP * DXP, ob = 2 * DXP * DXP, oH = ob + DXP, oM = oH + DYP * DXP;
  const int oQi = oM + DXP * DXP, omu = oQi + DXP * DXP, oL0 = omu + DXP, tot = oL0 + DXP * DXP;
  std::vector<Real> v(tot, Real(0));
  for (int j = 0; j < dx; ++j)
    for (int i = 0; i < dx; ++i) {
      v[oA + j * DXP + i] = (Real)f.A[i + j * dx];
      v[oL + j * DXP + i] = (Real)f.L[i + j * dx];
      v[oM + j * DXP + i] = (Real)f.M[i + j * dx];
      v[oQi + j * DXP + i] = (Real)f.Qi[i + j * dx];
      v[oL0 + j * DXP + i] = (Real)f.L0[i + j * dx];
    }
  for (int i = 0; i < dx; ++i) {
    v[ob + i] = (Real)f.b[i];
    v[omu + i] = (Real)f.mu0[i];
  }
  for (int j = 0; j < dx; ++j)
    for (int k = 0; k < dy; ++k) v[oH + j * DYP + k] = (Real)f.Ht[k + j * dy];
  if (sizeof(Real) == 4 && DXP >= 16) {
    // tensor-core appendix: B = [[A, L], [H~A, H~L]] (NM x 2DXP, row-major), H~b
    const int K = 2 * DXP, NM = ((DXP + DYP + 15) / 16) * 16;
    std::vector<Real> B((size_t)NM * K, Real(0)), Hb(DYP, Real(0));
    for (int n = 0; n < dx; ++n)
      for (int k = 0; k < dx; ++k) {
        B[(size_t)n * K + k] = (Real)f.A[n + k * dx];
        B[(size_t)n * K + DXP + k] = (Real)f.L[n + k * dx];
      }
    for (int j = 0; j < dy; ++j) {
      double hb = 0.0;
      for (int p = 0; p < dx; ++p) hb += f.Ht[j + p * dy] * f.b[p];
      Hb[j] = (Real)hb;
      for (int k = 0; k < dx; ++k) {
        double ha = 0.0, hl = 0.0;
        for (int p = 0; p < dx; ++p) {
          ha += f.Ht[j + p * dy] * f.A[p + k * dx];
          hl += f.Ht[j + p * dy] * f.L[p + k * dx];
        }
        B[(size_t)(DXP + j) * K + k] = (Real)ha;
        B[(size_t)(DXP + j) * K + DXP + k] = (Real)hl;
      }
    }
    v.insert(v.end(), B.begin(), B.end());
    v.insert(v.end(), Hb.begin(), Hb.end());
  }
  // appended: a time-varying model packs one block per step
  const size_t off = out.size();
  out.resize(off + sizeof(Real) * v.size());
  std::memcpy(out.data() + off, v.data(), sizeof(Real) * v.size());
}

void pack_params(const LgFactors& f, bool dbl, int dxp, int dyp, std::vector<char>& out) {
  if (dbl) pack_lg_params<double>(f, dxp, dyp, out);
  else pack_lg_params<float>(f, dxp, dyp, out);
}

}  // namespace gf

extern "C" gf_status gf_pf_dense_ancestry(gf_ctx* ctx, int32_t T, int64_t N, int32_t dx, int32_t precision,
                                          const void* history, const int32_t* ancestors, int64_t M,
                                          const int32_t* indices, int32_t memspace, void* paths) {
  using namespace gf;
  if (!ctx) return GF_ERR_ARG;
  if (!history || !paths || (T > 0 && !ancestors)) return set_err(ctx, GF_ERR_ARG, "null argument");
  if (T < 0 || N < 1 || dx < 1) return set_err(ctx, GF_ERR_ARG, "need T >= 0, N >= 1, dx >= 1");
  if (precision != GF_PREC_F32 && precision != GF_PREC_F64) return set_err(ctx, GF_ERR_ARG, "unknown precision");
  if (memspace != GF_MEM_HOST && memspace != GF_MEM_DEVICE) return set_err(ctx, GF_ERR_ARG, "bad memspace");
  if (!indices) M = N;
  if (M < 1) return set_err(ctx, GF_ERR_ARG, "need M >= 1");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t rs = precision == GF_PREC_F64 ? 8 : 4;
  const size_t hb = rs * (size_t)(T + 1) * dx * N, ab = sizeof(int32_t) * (size_t)T * N;
  const size_t ob = rs * (size_t)(T + 1) * dx * M, ib = indices ? sizeof(int32_t) * (size_t)M : 0;
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
  gf_status st;
  const void* h = history;
  const int32_t* a = ancestors;
  const int32_t* ix = indices;
  void* o = paths;
  void* pbad;
  if ((st = get(sizeof(int32_t), &pbad))) return st;
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(pbad, 0, sizeof(int32_t), s));
  if (memspace == GF_MEM_HOST) {
    void* p;
    if ((st = get(hb, &p))) return st;
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, history, hb, cudaMemcpyHostToDevice, s));
    h = p;
    if (T > 0) {
      if ((st = get(ab, &p))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, ancestors, ab, cudaMemcpyHostToDevice, s));
      a = (const int32_t*)p;
    }
    if (indices) {
      if ((st = get(ib, &p))) return st;
      GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, indices, ib, cudaMemcpyHostToDevice, s));
      ix = (const int32_t*)p;
    }
    if ((st = get(ob, &o))) return st;
  }
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((M + 255) / 256, 8 * (int64_t)ctx->num_sms));
  if (precision == GF_PREC_F64)
    pf_dense_ancestry_kernel<double><<<blocks, 256, 0, s>>>(T, N, dx, (const double*)h, a, M, ix, (double*)o,
                                                            (int32_t*)pbad);
  else
    pf_dense_ancestry_kernel<float><<<blocks, 256, 0, s>>>(T, N, dx, (const float*)h, a, M, ix, (float*)o,
                                                           (int32_t*)pbad);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  if (memspace == GF_MEM_HOST) GF_CHECK_CUDA(ctx, cudaMemcpyAsync(paths, o, ob, cudaMemcpyDeviceToHost, s));
  int32_t bad = 0;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(&bad, pbad, sizeof bad, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (bad) return set_err(ctx, GF_ERR_ARG, "an index or ancestor lies outside 1..N");
  return GF_OK;
}
