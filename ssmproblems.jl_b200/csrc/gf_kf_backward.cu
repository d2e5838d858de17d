// gf_kf_backward.cu -- batched backward information filter and two-filter smoother.
//
// BackwardInformationPredictor (kalman.jl:236-334) for B homogeneous linear-
// Gaussian models at once, one CTA per model, FP64: the backward predictive
// likelihoods p(y_{t:T} | x_t) and p(y_{t+1:T} | x_t) in information form
// (exp(lam'x - x'Om x / 2)),
//   backward_initialise : lam = H'R^-1 (y_T - c), Om = H'R^-1 H (+ initial jitter)
//   backward_predict    : m = lam - Om b, Lam = F'Om F + I (F = chol(Q)),
//                         Om^ = A'(I - Om F Lam^-1 F') Om A, lam^ = A'(I - Om F Lam^-1 F') m
//   backward_update     : lam += H'R^-1 (y_t - c), Om += H'R^-1 H
// (each new Om kept symmetric from its upper triangle, as PDMat(Symmetric(.)))
// and, on request, two_filter_smooth (kalman.jl:336-370) at every time: the
// forward filtered N(mu_t, Sigma_t), computed first in the same CTA, combined
// with p(y_{t+1:T} | x_t) as a product of Gaussians in information form.
#include <cmath>
#include <vector>

#include "gf_common.cuh"
#include "gf_internal.hpp"
#include "gf_smallmat.cuh"

namespace gf {
namespace {

constexpr int BI_THREADS = 256;
constexpr int BI_MATS = 30;  // shared LD x LD matrices, vectors included

struct BiDesc {
  int32_t dx, dy, T;
  int32_t pstep;   // time-varying: doubles per step block (block k = calc_params(., k+1)); 0 = one block
  int64_t y_off;   // into ys: [T][dy]
  int64_t p_off;   // into params: blocks A | b | F | G = H'R^-1 | W = H'R^-1 H | Q | H | c | R, then mu0 | Sigma0
  int64_t ck_off;  // forward scratch: T * (dx + dx*dx)
  int64_t v_off;   // outputs: sum of T*dx
  int64_t m_off;   // sum of T*dx*dx
};

struct BiArgs {
  const BiDesc* desc;
  const double* ys;
  const double* params;
  double* ck;
  double initial_jitter, jitter;
  int use_initial_jitter, use_jitter;
  double *lam_pred, *Om_pred, *lam_upd, *Om_upd, *mu_s, *Sig_s;
  int32_t* status;
};

// M = its upper triangle mirrored (PDMat(Symmetric(M))).
__device__ void sym_upper(double* M, int n) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    if (i > j) M[i + j * LD] = M[j + i * LD];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(BI_THREADS) kf_backinfo_kernel(BiArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double s_logdet;
  __shared__ int s_ok;
  const BiDesc D = a.desc[blockIdx.x];
  const int dx = D.dx, dy = D.dy, T = D.T, tid = threadIdx.x, bd = blockDim.x;
  const int MS = LD * LD;
  double* M0 = sm;
  auto mat = [&](int k) { return M0 + k * MS; };
  double *A = mat(0), *F = mat(1), *G = mat(2), *W = mat(3), *Q = mat(4), *H = mat(5), *R = mat(6);
  double *Sig = mat(7), *Sp = mat(8), *S = mat(9), *Ls = mat(10), *Si = mat(11), *K = mat(12);
  double *IKH = mat(13), *W2 = mat(14), *T1 = mat(15), *T2 = mat(16), *T3 = mat(17);
  double *Om = mat(18), *Omh = mat(19), *Lam = mat(20), *Li = mat(21), *FLF = mat(22), *Im = mat(23);
  double *Sfi = mat(24), *Os = mat(25), *Ss = mat(26);
  double* V = mat(27);  // vectors, LD apart
  double *b = V, *c = V + LD, *mu = V + 2 * LD, *mp = V + 3 * LD, *z = V + 4 * LD, *u = V + 5 * LD;
  double *lam = V + 6 * LD, *lamh = V + 7 * LD, *mv_ = V + 8 * LD, *v = V + 9 * LD, *lf = V + 10 * LD;
  double *ym = V + 11 * LD;

  const double* P = a.params + D.p_off;
  // one step block: A | b | F | G | W | Q | H | c | R (time-varying models: T of
  // them, block k holding calc_params(dyn, k+1) and calc_params(obs, k+1))
  const int blen = 4 * dx * dx + dx + 2 * dx * dy + dy + dy * dy;
  const double* Pmu0 = P + (D.pstep ? (int64_t)T * D.pstep : (int64_t)blen);
  const double* PS0 = Pmu0 + dx;
  auto load_dyn = [&](int k) {  // A, b, F = chol(Q), Q of block k
    const double* B = P + (int64_t)k * D.pstep;
    for (int e = tid; e < dx * dx; e += bd) {
      const int o = e % dx + (e / dx) * LD;
      A[o] = B[e];
      F[o] = B[dx * dx + dx + e];
      Q[o] = B[3 * dx * dx + dx + dx * dy + e];
    }
    for (int i = tid; i < dx; i += bd) b[i] = B[dx * dx + i];
  };
  auto load_obs = [&](int k) {  // G = H'R^-1, W = H'R^-1 H, H, c, R of block k
    const double* B = P + (int64_t)k * D.pstep;
    const double* PG = B + 2 * dx * dx + dx;
    const double* PW = PG + dx * dy;
    const double* PH = PW + 2 * dx * dx;
    const double* Pc = PH + dy * dx;
    const double* PR = Pc + dy;
    for (int e = tid; e < dx * dx; e += bd) W[e % dx + (e / dx) * LD] = PW[e];
    for (int e = tid; e < dx * dy; e += bd) G[e % dx + (e / dx) * LD] = PG[e];
    for (int e = tid; e < dy * dx; e += bd) H[e % dy + (e / dy) * LD] = PH[e];
    for (int e = tid; e < dy * dy; e += bd) R[e % dy + (e / dy) * LD] = PR[e];
    for (int i = tid; i < dy; i += bd) c[i] = Pc[i];
  };
  for (int e = tid; e < MS * (BI_MATS - 2); e += bd) sm[e] = 0.0;
  __syncthreads();
  load_dyn(0);
  load_obs(0);
  for (int e = tid; e < dx * dx; e += bd) Sig[e % dx + (e / dx) * LD] = PS0[e];
  for (int i = tid; i < dx; i += bd) mu[i] = Pmu0[i];
  __syncthreads();
  const double* Y = a.ys + D.y_off;
  double* CK = a.ck + D.ck_off;
  const int ckw = dx + dx * dx;
  const bool smooth = a.mu_s || a.Sig_s;
  int status = 0;

  // ---- forward filter (kalman.jl:42-79, Joseph form) when smoothing: filtered moments to CK
  for (int t = 0; smooth && t < T; ++t) {
    const double* y = Y + (size_t)t * dy;
    if (D.pstep && t > 0) {  // step t's model
      load_dyn(t);
      load_obs(t);
      __syncthreads();
    }
    mv(mp, A, false, mu, dx, dx);
    for (int i = tid; i < dx; i += bd) mp[i] += b[i];
    mm(T1, A, false, Sig, false, dx, dx, dx, 1.0, 0.0);
    mm(Sp, T1, false, A, true, dx, dx, dx, 1.0, 0.0);
    for (int e = tid; e < dx * dx; e += bd) Sp[e % dx + (e / dx) * LD] += Q[e % dx + (e / dx) * LD];
    __syncthreads();
    symmetrize(Sp, dx);
    mv(u, H, false, mp, dy, dx);
    for (int i = tid; i < dy; i += bd) z[i] = y[i] - u[i] - c[i];
    mm(W2, H, false, Sp, false, dy, dx, dx, 1.0, 0.0);
    mm(S, W2, false, H, true, dy, dx, dy, 1.0, 0.0);
    for (int e = tid; e < dy * dy; e += bd) S[e % dy + (e / dy) * LD] += R[e % dy + (e / dy) * LD];
    __syncthreads();
    symmetrize(S, dy);
    if (!chol_inv(S, Ls, Si, dy, &s_logdet, &s_ok)) {
      status = GF_ERR_NOT_PD;
      break;
    }
    mm(K, W2, true, Si, false, dx, dy, dy, 1.0, 0.0);
    mm(IKH, K, false, H, false, dx, dy, dx, -1.0, 0.0);
    for (int i = tid; i < dx; i += bd) IKH[i + i * LD] += 1.0;
    __syncthreads();
    mm(T1, IKH, false, Sp, false, dx, dx, dx, 1.0, 0.0);
    mm(Sig, T1, false, IKH, true, dx, dx, dx, 1.0, 0.0);
    mm(T2, K, false, R, false, dx, dy, dy, 1.0, 0.0);
    mm(Sig, T2, false, K, true, dx, dy, dx, 1.0, 1.0);
    mv(u, K, false, z, dx, dy);
    for (int i = tid; i < dx; i += bd) mu[i] = mp[i] + u[i];
    __syncthreads();
    for (int e = tid; e < ckw; e += bd)
      CK[(size_t)t * ckw + e] = e < dx ? mu[e] : Sig[(e - dx) % dx + ((e - dx) / dx) * LD];
    __syncthreads();
  }

  auto put_v = [&](double* out, int t, const double* x) {
    if (out)
      for (int i = tid; i < dx; i += bd) out[D.v_off + (int64_t)t * dx + i] = x[i];
  };
  auto put_m = [&](double* out, int t, const double* M) {
    if (out)
      for (int e = tid; e < dx * dx; e += bd) out[D.m_off + (int64_t)t * dx * dx + e] = M[e % dx + (e / dx) * LD];
  };
  auto obs_info = [&](const double* y) {  // lam += G (y - c)
    for (int i = tid; i < dy; i += bd) ym[i] = y[i] - c[i];
    __syncthreads();
    mv(u, G, false, ym, dx, dy);
    for (int i = tid; i < dx; i += bd) lam[i] += u[i];
    __syncthreads();
  };

  // ---- backward_initialise at T (calc_params(obs, T))
  if (!status) {
    if (D.pstep) {
      load_obs(T - 1);
      __syncthreads();
    }
    for (int i = tid; i < dx; i += bd) lam[i] = 0.0;
    for (int e = tid; e < dx * dx; e += bd) {
      const int i = e % dx, j = e / dx;
      Om[i + j * LD] = W[i + j * LD] + (a.use_initial_jitter && i == j ? a.initial_jitter : 0.0);
      Omh[i + j * LD] = 0.0;
    }
    __syncthreads();
    obs_info(Y + (size_t)(T - 1) * dy);
    sym_upper(Om, dx);
    put_v(a.lam_upd, T - 1, lam);
    put_m(a.Om_upd, T - 1, Om);
    for (int i = tid; i < dx; i += bd) lamh[i] = 0.0;
    __syncthreads();
    put_v(a.lam_pred, T - 1, lamh);  // p(y_{T+1:T} | x_T) = 1
    put_m(a.Om_pred, T - 1, Omh);
    if (smooth) {  // nothing after T: the smoothed moments are the filtered ones
      for (int e = tid; e < ckw; e += bd) {
        const double val = CK[(size_t)(T - 1) * ckw + e];
        if (e < dx) {
          if (a.mu_s) a.mu_s[D.v_off + (int64_t)(T - 1) * dx + e] = val;
        } else if (a.Sig_s) {
          a.Sig_s[D.m_off + (int64_t)(T - 1) * dx * dx + (e - dx)] = val;
        }
      }
    }
    __syncthreads();
  }

  for (int t = T - 2; t >= 0 && !status; --t) {
    // ---- backward_predict: p(y_{t+2:T} | x_{t+1}) -> p(y_{t+2:T} | x_t) (0-based t),
    //      the transition x_t -> x_{t+1} of block t + 1 (calc_params(dyn, iter + 1))
    if (D.pstep) {
      __syncthreads();
      load_dyn(t + 1);
      __syncthreads();
    }
    mv(u, Om, false, b, dx, dx);
    for (int i = tid; i < dx; i += bd) mv_[i] = lam[i] - u[i];
    mm(T1, Om, false, F, false, dx, dx, dx, 1.0, 0.0);
    mm(Lam, F, true, T1, false, dx, dx, dx, 1.0, 0.0);
    for (int i = tid; i < dx; i += bd) Lam[i + i * LD] += 1.0;
    __syncthreads();
    if (!chol_inv(Lam, Ls, Li, dx, &s_logdet, &s_ok)) {
      status = GF_ERR_NOT_PD;
      break;
    }
    mm(T2, F, false, Li, false, dx, dx, dx, 1.0, 0.0);
    mm(FLF, T2, false, F, true, dx, dx, dx, 1.0, 0.0);
    mm(Im, Om, false, FLF, false, dx, dx, dx, -1.0, 0.0);
    for (int i = tid; i < dx; i += bd) Im[i + i * LD] += 1.0;
    __syncthreads();
    mm(T3, Om, false, A, false, dx, dx, dx, 1.0, 0.0);
    mm(T1, Im, false, T3, false, dx, dx, dx, 1.0, 0.0);
    mm(Omh, A, true, T1, false, dx, dx, dx, 1.0, 0.0);
    if (a.use_jitter)
      for (int i = tid; i < dx; i += bd) Omh[i + i * LD] += a.jitter;
    __syncthreads();
    sym_upper(Omh, dx);
    mv(v, Im, false, mv_, dx, dx);
    mv(lamh, A, true, v, dx, dx);
    put_v(a.lam_pred, t, lamh);
    put_m(a.Om_pred, t, Omh);
    // ---- two_filter_smooth at t: filtered N(mu, Sig) x exp(lamh'x - x'Omh x / 2)
    if (smooth) {
      for (int e = tid; e < ckw; e += bd) {
        const double val = CK[(size_t)t * ckw + e];
        if (e < dx) mu[e] = val;
        else Sig[(e - dx) % dx + ((e - dx) / dx) * LD] = val;
      }
      __syncthreads();
      if (!chol_inv(Sig, Ls, Sfi, dx, &s_logdet, &s_ok)) {
        status = GF_ERR_NOT_PD;
        break;
      }
      mv(lf, Sfi, false, mu, dx, dx);
      for (int e = tid; e < dx * dx; e += bd) {
        const int o = e % dx + (e / dx) * LD;
        Os[o] = Sfi[o] + Omh[o];
      }
      __syncthreads();
      if (!chol_inv(Os, Ls, Ss, dx, &s_logdet, &s_ok)) {
        status = GF_ERR_NOT_PD;
        break;
      }
      for (int i = tid; i < dx; i += bd) lf[i] += lamh[i];
      __syncthreads();
      mv(u, Ss, false, lf, dx, dx);
      if (a.mu_s)
        for (int i = tid; i < dx; i += bd) a.mu_s[D.v_off + (int64_t)t * dx + i] = u[i];
      if (a.Sig_s)
        for (int e = tid; e < dx * dx; e += bd)
          a.Sig_s[D.m_off + (int64_t)t * dx * dx + e] = Ss[e % dx + (e / dx) * LD];
      __syncthreads();
    }
    // ---- backward_update with y_t (calc_params(obs, t + 1), block t)
    if (D.pstep) {
      __syncthreads();
      load_obs(t);
      __syncthreads();
    }
    for (int i = tid; i < dx; i += bd) lam[i] = lamh[i];
    for (int e = tid; e < dx * dx; e += bd) {
      const int o = e % dx + (e / dx) * LD;
      Om[o] = Omh[o] + W[o];
    }
    __syncthreads();
    obs_info(Y + (size_t)t * dy);
    sym_upper(Om, dx);
    put_v(a.lam_upd, t, lam);
    put_m(a.Om_upd, t, Om);
    __syncthreads();
  }
  if (tid == 0 && a.status) a.status[blockIdx.x] = status;
}

}  // namespace
}  // namespace gf

static gf_status backward_impl(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                               const int32_t* param_steps, const double* ys, double initial_jitter,
                               int32_t use_initial_jitter, double jitter, int32_t use_jitter, int32_t memspace,
                               gf_kf_backward_out* out) {
  using namespace gf;
  if (!ctx) return GF_ERR_ARG;
  if (!models || !T || !ys || !out || B < 1) return set_err(ctx, GF_ERR_ARG, "null argument or B < 1");
  if (memspace != GF_MEM_HOST && memspace != GF_MEM_DEVICE) return set_err(ctx, GF_ERR_ARG, "bad memspace");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  std::vector<BiDesc> desc(B);
  std::vector<double> params;
  int64_t ny = 0, nck = 0, nv = 0, nm = 0;
  for (int f = 0; f < B; ++f) {
    const gf_lg_model& m = models[f];
    const int dx = m.dx, dy = m.dy;
    if (dx < 1 || dy < 1 || dx > SM_MAXD || dy > SM_MAXD)
      return set_err(ctx, GF_ERR_DIM, "model %d: the backward filter needs 1 <= dx, dy <= %d", f, SM_MAXD);
    if (T[f] < 1) return set_err(ctx, GF_ERR_ARG, "model %d: T must be >= 1", f);
    const int ps = param_steps ? param_steps[f] : 1;
    if (ps != 1 && ps < T[f])
      return set_err(ctx, GF_ERR_ARG, "model %d: %d parameter steps for T = %d", f, ps, T[f]);
    const int nblk = ps == 1 ? 1 : T[f];
    BiDesc& d = desc[f];
    d.dx = dx;
    d.dy = dy;
    d.T = T[f];
    d.pstep = ps == 1 ? 0 : 4 * dx * dx + dx + 2 * dx * dy + dy + dy * dy;
    d.y_off = ny;
    d.p_off = (int64_t)params.size();
    d.ck_off = nck;
    d.v_off = nv;
    d.m_off = nm;
    for (int k = 0; k < nblk; ++k) {  // step block k: calc_params(dyn, k+1), calc_params(obs, k+1)
      const double *mA = m.A + (size_t)k * dx * dx, *mb = m.b + (size_t)k * dx, *mQ = m.Q + (size_t)k * dx * dx;
      const double *mH = m.H + (size_t)k * dy * dx, *mc = m.c + (size_t)k * dy, *mR = m.R + (size_t)k * dy * dy;
      std::vector<double> LQ(dx * dx), LR(dy * dy), LRi(dy * dy), Ri(dy * dy), G(dx * dy), W(dx * dx);
      if (chol_lower(dx, mQ, LQ.data()))
        return set_err(ctx, GF_ERR_NOT_PD, "model %d: Q of step %d is not positive definite", f, k + 1);
      if (chol_lower(dy, mR, LR.data()))
        return set_err(ctx, GF_ERR_NOT_PD, "model %d: R of step %d is not positive definite", f, k + 1);
      tri_inv_lower(dy, LR.data(), LRi.data());
      for (int i = 0; i < dy; ++i)  // R^-1 = L^-T L^-1
        for (int j = 0; j < dy; ++j) {
          double acc = 0.0;
          for (int p = 0; p < dy; ++p) acc += LRi[p + i * dy] * LRi[p + j * dy];
          Ri[i + j * dy] = acc;
        }
      for (int i = 0; i < dx; ++i)  // G = H' R^-1
        for (int j = 0; j < dy; ++j) {
          double acc = 0.0;
          for (int p = 0; p < dy; ++p) acc += mH[p + i * dy] * Ri[p + j * dy];
          G[i + j * dx] = acc;
        }
      for (int i = 0; i < dx; ++i)  // W = G H
        for (int j = 0; j < dx; ++j) {
          double acc = 0.0;
          for (int p = 0; p < dy; ++p) acc += G[i + p * dx] * mH[p + j * dy];
          W[i + j * dx] = acc;
        }
      params.insert(params.end(), mA, mA + dx * dx);
      params.insert(params.end(), mb, mb + dx);
      params.insert(params.end(), LQ.begin(), LQ.end());
      params.insert(params.end(), G.begin(), G.end());
      params.insert(params.end(), W.begin(), W.end());
      params.insert(params.end(), mQ, mQ + dx * dx);
      params.insert(params.end(), mH, mH + dy * dx);
      params.insert(params.end(), mc, mc + dy);
      params.insert(params.end(), mR, mR + dy * dy);
    }
    params.insert(params.end(), m.mu0, m.mu0 + dx);
    params.insert(params.end(), m.Sigma0, m.Sigma0 + dx * dx);
    ny += (int64_t)T[f] * dy;
    nck += (int64_t)T[f] * (dx + dx * dx);
    nv += (int64_t)T[f] * dx;
    nm += (int64_t)T[f] * dx * dx;
  }
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
  const bool smooth = out->mu_smooth || out->Sigma_smooth;
  gf_status st;
  void *dd, *dp, *dck = nullptr, *dstatus;
  if ((st = get(sizeof(BiDesc) * B, &dd)) || (st = get(sizeof(double) * params.size(), &dp)) ||
      (smooth && (st = get(sizeof(double) * nck, &dck))) || (st = get(sizeof(int32_t) * B, &dstatus)))
    return st;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dd, desc.data(), sizeof(BiDesc) * B, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dp, params.data(), sizeof(double) * params.size(), cudaMemcpyHostToDevice, s));
  BiArgs a{};
  a.desc = (const BiDesc*)dd;
  a.params = (const double*)dp;
  a.ck = (double*)dck;
  a.initial_jitter = initial_jitter;
  a.jitter = jitter;
  a.use_initial_jitter = use_initial_jitter != 0;
  a.use_jitter = use_jitter != 0;
  a.status = (int32_t*)dstatus;
  struct Io {
    double* host;
    double** dev;
    int64_t n;
  };
  std::vector<Io> io = {{out->lam_pred, &a.lam_pred, nv}, {out->Om_pred, &a.Om_pred, nm},
                        {out->lam_upd, &a.lam_upd, nv},   {out->Om_upd, &a.Om_upd, nm},
                        {out->mu_smooth, &a.mu_s, nv},    {out->Sigma_smooth, &a.Sig_s, nm}};
  if (memspace == GF_MEM_DEVICE) {
    a.ys = ys;
    for (auto& x : io) *x.dev = x.host;
  } else {
    void* p;
    if ((st = get(sizeof(double) * ny, &p))) return st;
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p, ys, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
    a.ys = (const double*)p;
    for (auto& x : io)
      if (x.host) {
        if ((st = get(sizeof(double) * x.n, &p))) return st;
        *x.dev = (double*)p;
      }
  }
  const size_t smem = sizeof(double) * ((size_t)BI_MATS * LD * LD);
  GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)kf_backinfo_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kf_backinfo_kernel<<<B, BI_THREADS, smem, s>>>(a);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  if (memspace == GF_MEM_HOST)
    for (auto& x : io)
      if (x.host)
        GF_CHECK_CUDA(ctx, cudaMemcpyAsync(x.host, *x.dev, sizeof(double) * x.n, cudaMemcpyDeviceToHost, s));
  std::vector<int32_t> hs(B);
  if (out->status && memspace == GF_MEM_DEVICE)
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(out->status, dstatus, sizeof(int32_t) * B, cudaMemcpyDeviceToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(hs.data(), dstatus, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (out->status && memspace == GF_MEM_HOST) std::copy(hs.begin(), hs.end(), out->status);
  for (int f = 0; f < B; ++f)
    if (hs[f]) return set_err(ctx, hs[f], "model %d: a covariance or precision lost positive definiteness", f);
  return GF_OK;
}

extern "C" gf_status gf_kf_backward_information(gf_ctx* ctx, const gf_lg_model* models, int32_t B,
                                                const int32_t* T, const double* ys, double initial_jitter,
                                                int32_t use_initial_jitter, double jitter, int32_t use_jitter,
                                                int32_t memspace, gf_kf_backward_out* out) {
  return backward_impl(ctx, models, B, T, nullptr, ys, initial_jitter, use_initial_jitter, jitter, use_jitter,
                       memspace, out);
}

extern "C" gf_status gf_kf_backward_information_tv(gf_ctx* ctx, const gf_lg_model* models, int32_t B,
                                                   const int32_t* T, const int32_t* param_steps, const double* ys,
                                                   double initial_jitter, int32_t use_initial_jitter, double jitter,
                                                   int32_t use_jitter, int32_t memspace, gf_kf_backward_out* out) {
  return backward_impl(ctx, models, B, T, param_steps, ys, initial_jitter, use_initial_jitter, jitter, use_jitter,
                       memspace, out);
}
