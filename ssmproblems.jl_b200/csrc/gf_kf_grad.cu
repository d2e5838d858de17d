// gf_kf_grad.cu -- batched Kalman log-likelihood gradients.
//
// kf_loglikelihood with its ChainRules pullback (integrations/logdensity.jl:
// 136-161, integrations/kalman_rrule.jl:22-107) for B homogeneous linear-
// Gaussian models at once, one CTA per model, FP64 throughout:
//   forward : kalman_predict (kalman.jl:42-49) and _kalman_update_cached
//             (kalman_gradient.jl:12-23, Joseph form), with the filtered
//             moments of every step checkpointed in global memory;
//   backward: per step t = T..1 the cache (mu_pred, Sigma_pred, S, K, z, I-KH)
//             is recomputed from the checkpoint, then gradient_c / gradient_H /
//             gradient_R (kalman_gradient.jl:172-263), backward_gradient_update
//             (:97-120, Parellier et al. eqs 8-9), gradient_b / gradient_A /
//             gradient_Q (:150-205) and backward_gradient_predict (:138-143,
//             eqs 10-11).
// The outputs are the gradients of ll (the pullback with Delta ll = 1), summed
// over t for the time-invariant A, b, Q, H, c, R.
#include <cmath>
#include <vector>

#include "gf_common.cuh"
#include "gf_internal.hpp"
#include "gf_smallmat.cuh"

namespace gf {
namespace {

constexpr int KG_MAXD = SM_MAXD;
constexpr int KG_THREADS = 256;
constexpr int KG_MATS = 26;  // shared matrices of LD x LD doubles

struct KgDesc {
  int32_t dx, dy, T, pad;
  int64_t y_off;    // into ys: [T][dy]
  int64_t p_off;    // into params: A | b | Q | H | c | R | Rinv | mu0 | Sigma0
  int64_t ck_off;   // into the checkpoint scratch: (T+1) * (dx + dx*dx)
  int64_t gx_off;   // output offsets: sum of dx
  int64_t gxx_off;  // sum of dx*dx
  int64_t gyx_off;  // sum of dy*dx
  int64_t gy_off;   // sum of dy
  int64_t gyy_off;  // sum of dy*dy
};

struct KgArgs {
  const KgDesc* desc;
  const double* ys;
  const double* params;
  double* ck;
  double jitter;
  int use_jitter;
  double* ll;
  double *g_mu0, *g_Sigma0, *g_A, *g_b, *g_Q, *g_H, *g_c, *g_R;
  int32_t* status;
};

__global__ void __launch_bounds__(KG_THREADS) kf_grad_kernel(KgArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double s_logdet;
  __shared__ int s_ok;
  const KgDesc D = a.desc[blockIdx.x];
  const int dx = D.dx, dy = D.dy, T = D.T, tid = threadIdx.x, bd = blockDim.x;
  const int MS = LD * LD;
  double* A = sm;
  double* Q = A + MS;
  double* H = Q + MS;
  double* R = H + MS;
  double* Ri = R + MS;
  double* Sig = Ri + MS;  // filtered covariance of the step's start
  double* Sp = Sig + MS;
  double* S = Sp + MS;
  double* Ls = S + MS;
  double* Si = Ls + MS;
  double* K = Si + MS;
  double* IKH = K + MS;
  double* W = IKH + MS;   // H Sp (dy x dx)
  double* Pf = W + MS;
  double* dS = Pf + MS;
  double* dSp = dS + MS;
  double* T1 = dSp + MS;
  double* T2 = T1 + MS;
  double* T3 = T2 + MS;
  double* gA = T3 + MS;
  double* gQ = gA + MS;
  double* gH = gQ + MS;
  double* gR = gH + MS;
  double* V = gR + MS;  // vectors, LD apart: b c mu mp z mf Siz dmu dmp v u Kdmu gb gc
  double* b = V;
  double* c = V + LD;
  double* mu = V + 2 * LD;
  double* mp = V + 3 * LD;
  double* z = V + 4 * LD;
  double* mf = V + 5 * LD;
  double* Siz = V + 6 * LD;
  double* dmu = V + 7 * LD;
  double* dmp = V + 8 * LD;
  double* v = V + 9 * LD;
  double* u = V + 10 * LD;
  double* Kd = V + 11 * LD;
  double* gb = V + 12 * LD;
  double* gc = V + 13 * LD;

  const double* P = a.params + D.p_off;
  const double* Pb = P + dx * dx;
  const double* PQ = Pb + dx;
  const double* PH = PQ + dx * dx;
  const double* Pc = PH + dy * dx;
  const double* PR = Pc + dy;
  const double* PRi = PR + dy * dy;
  const double* Pmu0 = PRi + dy * dy;
  const double* PS0 = Pmu0 + dx;
  for (int e = tid; e < MS * (KG_MATS - 2); e += bd) sm[e] = 0.0;
  for (int e = tid; e < 16 * LD; e += bd) V[e] = 0.0;
  __syncthreads();
  for (int e = tid; e < dx * dx; e += bd) {
    const int i = e % dx, j = e / dx;
    A[i + j * LD] = P[e];
    Q[i + j * LD] = PQ[e];
    Sig[i + j * LD] = PS0[e];
  }
  for (int e = tid; e < dy * dx; e += bd) H[e % dy + (e / dy) * LD] = PH[e];
  for (int e = tid; e < dy * dy; e += bd) {
    R[e % dy + (e / dy) * LD] = PR[e];
    Ri[e % dy + (e / dy) * LD] = PRi[e];
  }
  for (int i = tid; i < dx; i += bd) {
    b[i] = Pb[i];
    mu[i] = Pmu0[i];
  }
  for (int i = tid; i < dy; i += bd) c[i] = Pc[i];
  __syncthreads();
  const double* Y = a.ys + D.y_off;
  double* CK = a.ck + D.ck_off;  // per t: mu (dx) then Sigma (dx*dx, column-major)
  const int ckw = dx + dx * dx;
  int status = 0;
  double ll = 0.0;

  // recomputes the step cache from the filtered (mu, Sig) of the step start
  auto step_cache = [&](const double* y) -> bool {
    mv(mp, A, false, mu, dx, dx);
    for (int i = tid; i < dx; i += bd) mp[i] += b[i];
    mm(T1, A, false, Sig, false, dx, dx, dx, 1.0, 0.0);
    mm(Sp, T1, false, A, true, dx, dx, dx, 1.0, 0.0);
    for (int e = tid; e < dx * dx; e += bd) Sp[e % dx + (e / dx) * LD] += Q[e % dx + (e / dx) * LD];
    __syncthreads();
    symmetrize(Sp, dx);
    mv(u, H, false, mp, dy, dx);
    for (int i = tid; i < dy; i += bd) z[i] = y[i] - u[i] - c[i];
    mm(W, H, false, Sp, false, dy, dx, dx, 1.0, 0.0);
    mm(S, W, false, H, true, dy, dx, dy, 1.0, 0.0);
    for (int e = tid; e < dy * dy; e += bd) S[e % dy + (e / dy) * LD] += R[e % dy + (e / dy) * LD];
    __syncthreads();
    symmetrize(S, dy);
    if (!chol_inv(S, Ls, Si, dy, &s_logdet, &s_ok)) return false;
    mm(K, W, true, Si, false, dx, dy, dy, 1.0, 0.0);  // Sp H' S^-1 = (H Sp)' S^-1
    mm(IKH, K, false, H, false, dx, dy, dx, -1.0, 0.0);
    for (int i = tid; i < dx; i += bd) IKH[i + i * LD] += 1.0;
    __syncthreads();
    return true;
  };

  // ---- forward pass with checkpoints
  for (int t = 0; t < T && !status; ++t) {
    for (int e = tid; e < ckw; e += bd)
      CK[(size_t)t * ckw + e] = e < dx ? mu[e] : Sig[(e - dx) % dx + ((e - dx) / dx) * LD];
    if (!step_cache(Y + (size_t)t * dy)) {
      status = GF_ERR_NOT_PD;
      break;
    }
    // Joseph form: Sf = (I-KH) Sp (I-KH)' + K R K'
    mm(T1, IKH, false, Sp, false, dx, dx, dx, 1.0, 0.0);
    mm(Sig, T1, false, IKH, true, dx, dx, dx, 1.0, 0.0);
    mm(T2, K, false, R, false, dx, dy, dy, 1.0, 0.0);
    mm(Sig, T2, false, K, true, dx, dy, dx, 1.0, 1.0);
    if (a.use_jitter)
      for (int i = tid; i < dx; i += bd) Sig[i + i * LD] += a.jitter;
    mv(u, K, false, z, dx, dy);
    for (int i = tid; i < dx; i += bd) mu[i] = mp[i] + u[i];
    mv(Siz, Si, false, z, dy, dy);
    double q = 0.0;
    for (int i = 0; i < dy; ++i) q += z[i] * Siz[i];
    ll += -0.5 * (dy * GF_LOG2PI + s_logdet + q);
    __syncthreads();
  }
  if (!status)
    for (int e = tid; e < ckw; e += bd)
      CK[(size_t)T * ckw + e] = e < dx ? mu[e] : Sig[(e - dx) % dx + ((e - dx) / dx) * LD];
  __syncthreads();

  // ---- backward pass (NLL convention of the reference; negated at the end)
  for (int t = T - 1; t >= 0 && !status; --t) {
    for (int e = tid; e < ckw; e += bd) {
      const double vv = CK[(size_t)t * ckw + e];
      if (e < dx) mu[e] = vv;
      else Sig[(e - dx) % dx + ((e - dx) / dx) * LD] = vv;
    }
    for (int i = tid; i < dx; i += bd) mf[i] = CK[(size_t)(t + 1) * ckw + i];
    __syncthreads();
    if (!step_cache(Y + (size_t)t * dy)) {
      status = GF_ERR_NOT_PD;
      break;
    }
    mv(Siz, Si, false, z, dy, dy);
    mv(Kd, K, true, dmu, dy, dx);  // K' dmu
    // gradient_c: -S^-1 z - K' dmu
    for (int i = tid; i < dy; i += bd) gc[i] += -Siz[i] - Kd[i];
    // gradient_H: S^-1 H Sp - Siz mp' - Siz Siz' H Sp + Siz dmu' Pf - K' dmu mf' - 2 K' dS Pf
    mm(Pf, IKH, false, Sp, false, dx, dx, dx, 1.0, 0.0);
    mv(v, W, true, Siz, dx, dy);   // (Siz' H Sp)' = Sp H' Siz
    mv(u, Pf, true, dmu, dx, dx);  // (dmu' Pf)'
    mm(T1, Si, false, W, false, dy, dy, dx, 1.0, 0.0);
    mm(T2, dS, false, Pf, false, dx, dx, dx, 1.0, 0.0);
    mm(T3, K, true, T2, false, dy, dx, dx, 1.0, 0.0);
    for (int e = tid; e < dy * dx; e += bd) {
      const int i = e % dy, j = e / dy;
      gH[i + j * LD] += T1[i + j * LD] - Siz[i] * mp[j] - Siz[i] * v[j] + Siz[i] * u[j] - Kd[i] * mf[j] -
                        2.0 * T3[i + j * LD];
    }
    __syncthreads();
    // gradient_R: K' dS K - (K'dmu Siz' + Siz dmu'K)/2 + (S^-1 - Siz Siz')/2
    mm(T1, dS, false, K, false, dx, dx, dy, 1.0, 0.0);
    mm(T2, K, true, T1, false, dy, dx, dy, 1.0, 0.0);
    for (int e = tid; e < dy * dy; e += bd) {
      const int i = e % dy, j = e / dy;
      gR[i + j * LD] += T2[i + j * LD] - 0.5 * (Kd[i] * Siz[j] + Siz[i] * Kd[j]) +
                        0.5 * (Si[i + j * LD] - Siz[i] * Siz[j]);
    }
    __syncthreads();
    // backward_gradient_update: dmp = (I-KH)' dmu - H' Siz
    mv(dmp, IKH, true, dmu, dx, dx);
    mv(u, H, true, Siz, dx, dy);  // H' Siz
    for (int i = tid; i < dx; i += bd) dmp[i] -= u[i];
    // cross = (dmu (H' R^-1 z)' + (H' R^-1 z) dmu') / 2 added to dS
    mv(Kd, Ri, false, z, dy, dy);  // R^-1 z (Kd reused)
    mv(v, H, true, Kd, dx, dy);    // H' R^-1 z
    for (int e = tid; e < dx * dx; e += bd) {
      const int i = e % dx, j = e / dx;
      T1[i + j * LD] = dS[i + j * LD] + 0.5 * (dmu[i] * v[j] + v[i] * dmu[j]);
    }
    __syncthreads();
    mm(T2, IKH, true, T1, false, dx, dx, dx, 1.0, 0.0);
    mm(dSp, T2, false, IKH, false, dx, dx, dx, 1.0, 0.0);
    // + (H' S^-1 H - (H' Siz)(H' Siz)') / 2
    mm(T1, Si, false, H, false, dy, dy, dx, 1.0, 0.0);
    mm(T2, H, true, T1, false, dx, dy, dx, 1.0, 0.0);
    for (int e = tid; e < dx * dx; e += bd) {
      const int i = e % dx, j = e / dx;
      dSp[i + j * LD] += 0.5 * (T2[i + j * LD] - u[i] * u[j]);
    }
    __syncthreads();
    // gradient_b, gradient_A, gradient_Q
    for (int i = tid; i < dx; i += bd) gb[i] += dmp[i];
    mm(T1, dSp, false, A, false, dx, dx, dx, 1.0, 0.0);
    mm(T2, T1, false, Sig, false, dx, dx, dx, 1.0, 0.0);
    for (int e = tid; e < dx * dx; e += bd) {
      const int i = e % dx, j = e / dx;
      gA[i + j * LD] += dmp[i] * mu[j] + 2.0 * T2[i + j * LD];
      gQ[i + j * LD] += dSp[i + j * LD];
    }
    __syncthreads();
    // backward_gradient_predict: dmu = A' dmp, dS = A' dSp A
    mv(dmu, A, true, dmp, dx, dx);
    mm(T2, A, true, T1, false, dx, dx, dx, 1.0, 0.0);  // A' (dSp A)
    for (int e = tid; e < dx * dx; e += bd) dS[e % dx + (e / dx) * LD] = T2[e % dx + (e / dx) * LD];
    __syncthreads();
  }

  // ---- outputs (gradients of ll = minus the NLL gradients)
  const int f = blockIdx.x;
  if (tid == 0) {
    if (a.ll) a.ll[f] = status ? NAN : ll;
    if (a.status) a.status[f] = status;
  }
  auto put = [&](double* out, int64_t off, const double* M, int rows, int cols) {
    if (!out) return;
    for (int e = tid; e < rows * cols; e += bd)
      out[off + e] = status ? NAN : -M[e % rows + (e / rows) * LD];
  };
  put(a.g_mu0, D.gx_off, dmu, dx, 1);
  put(a.g_Sigma0, D.gxx_off, dS, dx, dx);
  put(a.g_A, D.gxx_off, gA, dx, dx);
  put(a.g_b, D.gx_off, gb, dx, 1);
  put(a.g_Q, D.gxx_off, gQ, dx, dx);
  put(a.g_H, D.gyx_off, gH, dy, dx);
  put(a.g_c, D.gy_off, gc, dy, 1);
  put(a.g_R, D.gyy_off, gR, dy, dy);
}

}  // namespace
}  // namespace gf

extern "C" gf_status gf_kf_loglikelihood_grad(gf_ctx* ctx, const gf_lg_model* models, int32_t B,
                                              const int32_t* T, const double* ys, double jitter,
                                              int32_t use_jitter, int32_t memspace, gf_kf_grad_out* out) {
  using namespace gf;
  if (!ctx) return GF_ERR_ARG;
  if (!models || !T || !ys || !out || B < 1) return set_err(ctx, GF_ERR_ARG, "null argument or B < 1");
  if (memspace != GF_MEM_HOST && memspace != GF_MEM_DEVICE) return set_err(ctx, GF_ERR_ARG, "bad memspace");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  std::vector<KgDesc> desc(B);
  std::vector<double> params;
  int64_t ny = 0, nck = 0, gx = 0, gxx = 0, gyx = 0, gy = 0, gyy = 0;
  for (int f = 0; f < B; ++f) {
    const gf_lg_model& m = models[f];
    const int dx = m.dx, dy = m.dy;
    if (dx < 1 || dy < 1 || dx > KG_MAXD || dy > KG_MAXD)
      return set_err(ctx, GF_ERR_DIM, "model %d: gradients need 1 <= dx, dy <= %d", f, KG_MAXD);
    if (T[f] < 1) return set_err(ctx, GF_ERR_ARG, "model %d: T must be >= 1", f);
    std::vector<double> LR(dy * dy), LRi(dy * dy), Ri(dy * dy);
    if (chol_lower(dy, m.R, LR.data())) return set_err(ctx, GF_ERR_NOT_PD, "model %d: R is not positive definite", f);
    tri_inv_lower(dy, LR.data(), LRi.data());
    for (int i = 0; i < dy; ++i)  // R^-1 = L^-T L^-1
      for (int j = 0; j < dy; ++j) {
        double acc = 0.0;
        for (int p = 0; p < dy; ++p) acc += LRi[p + i * dy] * LRi[p + j * dy];
        Ri[i + j * dy] = acc;
      }
    KgDesc& d = desc[f];
    d.dx = dx;
    d.dy = dy;
    d.T = T[f];
    d.pad = 0;
    d.y_off = ny;
    d.p_off = (int64_t)params.size();
    d.ck_off = nck;
    d.gx_off = gx;
    d.gxx_off = gxx;
    d.gyx_off = gyx;
    d.gy_off = gy;
    d.gyy_off = gyy;
    params.insert(params.end(), m.A, m.A + dx * dx);
    params.insert(params.end(), m.b, m.b + dx);
    params.insert(params.end(), m.Q, m.Q + dx * dx);
    params.insert(params.end(), m.H, m.H + dy * dx);
    params.insert(params.end(), m.c, m.c + dy);
    params.insert(params.end(), m.R, m.R + dy * dy);
    params.insert(params.end(), Ri.begin(), Ri.end());
    params.insert(params.end(), m.mu0, m.mu0 + dx);
    params.insert(params.end(), m.Sigma0, m.Sigma0 + dx * dx);
    ny += (int64_t)T[f] * dy;
    nck += (int64_t)(T[f] + 1) * (dx + dx * dx);
    gx += dx;
    gxx += dx * dx;
    gyx += dy * dx;
    gy += dy;
    gyy += dy * dy;
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
  gf_status st;
  void *dd, *dp, *dck;
  if ((st = get(sizeof(KgDesc) * B, &dd)) || (st = get(sizeof(double) * params.size(), &dp)) ||
      (st = get(sizeof(double) * nck, &dck)))
    return st;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dd, desc.data(), sizeof(KgDesc) * B, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(dp, params.data(), sizeof(double) * params.size(), cudaMemcpyHostToDevice, s));
  KgArgs a{};
  a.desc = (const KgDesc*)dd;
  a.params = (const double*)dp;
  a.ck = (double*)dck;
  a.jitter = jitter;
  a.use_jitter = use_jitter != 0;
  struct Io {
    double* host;
    double** dev;
    int64_t n;
  };
  std::vector<Io> io = {{out->ll, &a.ll, B},          {out->d_mu0, &a.g_mu0, gx}, {out->d_Sigma0, &a.g_Sigma0, gxx},
                        {out->d_A, &a.g_A, gxx},      {out->d_b, &a.g_b, gx},     {out->d_Q, &a.g_Q, gxx},
                        {out->d_H, &a.g_H, gyx},      {out->d_c, &a.g_c, gy},     {out->d_R, &a.g_R, gyy}};
  void* dstatus;
  if ((st = get(sizeof(int32_t) * B, &dstatus))) return st;
  a.status = (int32_t*)dstatus;
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
  const size_t smem = sizeof(double) * ((size_t)KG_MATS * LD * LD);
  GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)kf_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
  kf_grad_kernel<<<B, KG_THREADS, smem, s>>>(a);
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
    if (hs[f]) return set_err(ctx, hs[f], "model %d: innovation covariance lost positive definiteness", f);
  return GF_OK;
}
