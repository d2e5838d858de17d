/*
 * gf_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of GeneralisedFilters' filtering hot path, used as the
 * parity checker for the CUDA library and as the timed CPU baseline.  Nothing
 * in the product links or calls this file: only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it.
 *
 * Parity pinning: the reference is pure Julia and cannot run here, so this
 * restatement is pinned by (1) the analytic joint-Gaussian conditioning the
 * reference's own KF test uses (GFTest/models/linear_gaussian.jl:171-215,
 * test/algorithms/kalman.jl:5-43), (2) SRKF == KF (test/algorithms/srkf.jl:3-26),
 * (3) the known-answer offspring/ancestor vectors
 * (test/components/resamplers.jl:76-92), and (4) PF -> KF convergence
 * (test/algorithms/particles.jl:5-53, test/algorithms/rbpf.jl:5-34).
 *
 * Conventions: matrices are column-major (Julia layout), M[i + j*ld].
 * Particle arrays are particle-major: x[i*dx + d].  Ancestors are 1-based.
 * Every function cites the reference lines it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LOG2PI 1.8378770664093454835606594728112

enum { OR_OK = 0, OR_NOT_PD = 1, OR_DIM = 2, OR_ARG = 6 };
enum { OR_SYSTEMATIC = 0, OR_STRATIFIED = 1, OR_MULTINOMIAL = 2 };
enum { OR_CONV_CPU = 0, OR_CONV_CUDAEXT = 1 };
enum { OR_PROP_BOOTSTRAP = 0, OR_PROP_OPTIMAL = 1, OR_PROP_OVERDISPERSED = 2 };

static int g_threads = 1; /* >1 only for the timed multi-core CPU baseline */
void or_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), restated from the paper.
 * The CUDA library draws its in-kernel noise from the same counter layout so
 * the oracle can regenerate it. */
static void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1,
                          uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
/* Exported for the published Random123 known-answer test. */
void or_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  philox4x32_10(ctr, k0, k1, out);
}
#define TAG_NORMAL 0x4E4F524Du
#define TAG_UNIF 0x554E4946u

/* 4 standard normals for (particle i, step t, block q) -- Box-Muller on
 * 24-bit uniforms u1 in (0,1], u2 in [0,1), angle 2*pi*u2 - pi. */
#define TAG_LOOKAHEAD 0x4C4B4844u /* DrawPredictive draws of the auxiliary filter */
static void philox_normals4_tag(uint64_t seed, uint32_t i, uint32_t t, uint32_t q, uint32_t tag,
                                double out[4]);
void or_philox_normals4(uint64_t seed, uint32_t i, uint32_t t, uint32_t q,
                        double out[4]) {
  philox_normals4_tag(seed, i, t, q, TAG_NORMAL, out);
}
static void philox_normals4_tag(uint64_t seed, uint32_t i, uint32_t t, uint32_t q, uint32_t tag,
                                double out[4]) {
  uint32_t ctr[4] = {i, t, q, tag}, w[4];
  philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), w);
  for (int p = 0; p < 2; ++p) {
    double u1 = ((double)(w[2 * p] >> 8) + 1.0) * (1.0 / 16777216.0);
    double u2 = (double)(w[2 * p + 1] >> 8) * (1.0 / 16777216.0);
    double r = sqrt(-2.0 * log(u1));
    double th = 6.283185307179586 * u2 - 3.141592653589793;
    out[2 * p] = r * cos(th);
    out[2 * p + 1] = r * sin(th);
  }
}
/* One FP64 uniform in [0,1) with 53 random bits for (slot j, step t). */
double or_philox_uniform(uint64_t seed, uint32_t j, uint32_t t) {
  uint32_t ctr[4] = {j, t, 0u, TAG_UNIF}, w[4];
  philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), w);
  uint64_t bits = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------------ */
/* Dense helpers (column-major). */
static void mm(int m, int k, int n, const double* A, const double* B, double* C) {
  /* C (m x n) = A (m x k) * B (k x n) */
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += A[i + p * m] * B[p + j * k];
      C[i + j * m] = s;
    }
}
static void mmT(int m, int k, int n, const double* A, const double* B, double* C) {
  /* C (m x n) = A (m x k) * B^T, B is (n x k) */
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += A[i + p * m] * B[j + p * n];
      C[i + j * m] = s;
    }
}
static void mv(int m, int n, const double* A, const double* x, double* y) {
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += A[i + j * m] * x[j];
    y[i] = s;
  }
}
/* Cholesky from the UPPER triangle (LAPACK potrf 'U', the convention of
 * Julia's cholesky(Hermitian(A))).  Writes the lower factor L = U^T, full
 * column-major with zeros above the diagonal. */
int or_chol_lower(int n, const double* A, double* L) {
  memset(L, 0, sizeof(double) * (size_t)n * n);
  for (int j = 0; j < n; ++j) {
    double s = A[j + j * n];
    for (int k = 0; k < j; ++k) s -= L[j + k * n] * L[j + k * n];
    if (!(s > 0.0)) return OR_NOT_PD;
    double d = sqrt(s);
    L[j + j * n] = d;
    for (int i = j + 1; i < n; ++i) {
      double t = A[j + i * n]; /* upper triangle element (j, i) */
      for (int k = 0; k < j; ++k) t -= L[i + k * n] * L[j + k * n];
      L[i + j * n] = t / d;
    }
  }
  return OR_OK;
}
/* solve L x = b in place (L lower) */
static void trsv_lower(int n, const double* L, double* x) {
  for (int i = 0; i < n; ++i) {
    double s = x[i];
    for (int k = 0; k < i; ++k) s -= L[i + k * n] * x[k];
    x[i] = s / L[i + i * n];
  }
}
/* solve L^T x = b in place */
static void trsv_lowerT(int n, const double* L, double* x) {
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= L[k + i * n] * x[k];
    x[i] = s / L[i + i * n];
  }
}
/* X_A_Xt(a::PDMat, X) = (X * L)(X * L)^T  (PDMats; kalman.jl:47,52,57) */
static void x_a_xt_chol(int m, int n, const double* X, const double* L, double* out,
                        double* tmp /* m*n */) {
  mm(m, n, n, X, L, tmp);
  mmT(m, n, m, tmp, tmp, out);
}
/* logpdf(MvNormal(mu, S), x) given L = chol(S): Distributions' -(d log2pi +
 * logdet + sqmahal)/2. */
static double logpdf_chol(int d, const double* L, const double* diff_in, double* tmp) {
  memcpy(tmp, diff_in, sizeof(double) * d);
  trsv_lower(d, L, tmp);
  double q = 0.0, ld = 0.0;
  for (int i = 0; i < d; ++i) {
    q += tmp[i] * tmp[i];
    ld += log(L[i + i * d]);
  }
  return -0.5 * (d * LOG2PI + 2.0 * ld + q);
}

/* Julia's pairwise reduction of a sum (Base.mapreduce_impl, block 1024). */
static double pairwise_sum(const double* a, long lo, long hi /* inclusive */,
                           int square) {
  if (lo == hi) return square ? a[lo] * a[lo] : a[lo];
  if (hi - lo < 1024) {
    double v = square ? a[lo] * a[lo] + a[lo + 1] * a[lo + 1] : a[lo] + a[lo + 1];
    for (long i = lo + 2; i <= hi; ++i) v += square ? a[i] * a[i] : a[i];
    return v;
  }
  long mid = lo + ((hi - lo) >> 1);
  return pairwise_sum(a, lo, mid, square) + pairwise_sum(a, mid + 1, hi, square);
}
/* LogExpFunctions.logsumexp (one-pass form: max + log1p(sum of the rest)). */
double or_logsumexp(const double* x, long n) {
  double m = x[0], r = 0.0;
  for (long i = 1; i < n; ++i) {
    if (x[i] <= m) r += exp(x[i] - m);
    else { r = (r + 1.0) * exp(m - x[i]); m = x[i]; }
  }
  return m + log1p(r);
}
/* LogExpFunctions.softmax: exp(x - max) / sum (pairwise sum). */
static void softmax(const double* x, long n, double* w) {
  double m = x[0];
  for (long i = 1; i < n; ++i) m = x[i] > m ? x[i] : m;
  for (long i = 0; i < n; ++i) w[i] = exp(x[i] - m);
  double s = pairwise_sum(w, 0, n - 1, 0);
  for (long i = 0; i < n; ++i) w[i] /= s;
}

/* ------------------------------------------------------------------------ */
/* Resampling (resamplers.jl:214-238; ext/CUDAExt.jl:31-117).
 * weights: normalised FP64 weights (N).  u: systematic -> u[0]; stratified /
 * multinomial -> u[0..N-1].  anc: 1-based output.  margin (nullable): per
 * slot, distance (in the units the comparison is made in) between the slot's
 * threshold and the nearest cumulative boundary -- the test harness treats
 * slots with a tiny margin as boundary cases.  Returns the number of slots that
 * had to be clamped to N (the reference's systematic walk has no clamp). */
long or_sample_ancestors(int kind, int conv, long n, const double* weights,
                         const double* u, int32_t* anc, double* margin) {
  double* W = (double*)malloc(sizeof(double) * n);
  double acc = 0.0;
  for (long k = 0; k < n; ++k) { acc += weights[k]; W[k] = acc; } /* serial cumsum */
  long clamps = 0;
  if (kind == OR_MULTINOMIAL) {
    /* CUDAExt.jl:31-39: us = U*W[n]; first k with W[k] >= us */
    double Wn = W[n - 1];
    for (long j = 0; j < n; ++j) {
      double us = u[j] * Wn;
      long lo = 0, hi = n; /* first k in [0,n) with W[k] >= us, else n */
      while (lo < hi) { long mid = (lo + hi) >> 1; if (W[mid] >= us) hi = mid; else lo = mid + 1; }
      if (lo >= n) { lo = n - 1; ++clamps; }
      anc[j] = (int32_t)(lo + 1);
      if (margin) {
        double m1 = W[lo] - us, m0 = lo > 0 ? us - W[lo - 1] : INFINITY;
        margin[j] = fabs(m1 < m0 ? m1 : m0) / (Wn > 0 ? Wn : 1.0) * n;
      }
    }
    free(W);
    return clamps;
  }
  if (conv == OR_CONV_CPU) {
    /* resamplers.jl:220-235: vs = cumsum(w) * n; a_i = min{k : vs_k > u_i}
     * with u_i = u0 + (i-1) (systematic) or (i-1) + U_i (stratified). */
    for (long k = 0; k < n; ++k) W[k] = W[k] * (double)n;
    long idx = 0;
    for (long j = 0; j < n; ++j) {
      double uu = (kind == OR_SYSTEMATIC) ? u[0] + (double)j : (double)j + u[j];
      while (idx < n && W[idx] <= uu) ++idx;
      long a = idx;
      if (a >= n) { a = n - 1; ++clamps; }
      anc[j] = (int32_t)(a + 1);
      if (margin) {
        double m1 = W[a] - uu, m0 = a > 0 ? uu - W[a - 1] : INFINITY;
        margin[j] = fabs(m1 < m0 ? m1 : m0);
      }
    }
    free(W);
    return clamps;
  }
  /* CUDAExt convention (CUDAExt.jl:49-78): cumulative offspring
   * O_k = min(n, floor(r_k + u)), r = n*W/W[n]; stratified picks
   * u[min(n, floor(r_k + 1))]; then offspring -> ancestors (:90-103). */
  double Wn = W[n - 1];
  long* O = (long*)malloc(sizeof(long) * n);
  double* rr = (double*)malloc(sizeof(double) * n);
  for (long k = 0; k < n; ++k) {
    double r = ((double)n * W[k]) / Wn;
    rr[k] = r;
    double uu;
    if (kind == OR_SYSTEMATIC) uu = u[0];
    else {
      double kk = floor(r + 1.0);
      long ki = kk < (double)n ? (long)kk : n; /* 1-based */
      uu = u[ki - 1];
    }
    double f = floor(r + uu);
    O[k] = f < (double)n ? (long)f : n;
  }
  long prev = 0;
  for (long k = 0; k < n; ++k) {
    for (long j = prev; j < O[k]; ++j) anc[j] = (int32_t)(k + 1);
    if (O[k] > prev) prev = O[k];
  }
  for (long j = prev; j < n; ++j) { anc[j] = (int32_t)n; ++clamps; }
  if (margin) {
    for (long j = 0; j < n; ++j) {
      long a = anc[j] - 1;
      double uu = (kind == OR_SYSTEMATIC) ? u[0] : u[(long)fmin(floor(rr[a] + 1.0), (double)n) - 1];
      double m1 = fabs(rr[a] + uu - (double)(j + 1));
      double m0 = a > 0 ? fabs(rr[a - 1] + uu - (double)(j + 1)) : INFINITY;
      margin[j] = m1 < m0 ? m1 : m0;
    }
  }
  free(rr);
  free(O);
  free(W);
  return clamps;
}

/* CUDAExt.jl:90-103: cumulative offspring (1-based semantics) -> ancestors. */
void or_offspring_to_ancestors(long n, const int64_t* offspring, int64_t* anc) {
  for (long i = 0; i < n; ++i) {
    int64_t start = i == 0 ? 0 : offspring[i - 1], finish = offspring[i];
    for (int64_t j = start; j < finish; ++j) anc[j] = i + 1;
  }
}
/* CUDAExt.jl:119-128: ancestors (1-based) -> offspring counts. */
void or_ancestors_to_offspring(long n, const int64_t* anc, int64_t* off) {
  for (long i = 0; i < n; ++i) off[i] = 0;
  for (long i = 0; i < n; ++i) off[anc[i] - 1] += 1;
}

/* ESS decision (resamplers.jl:179-183): threshold*n >= 1/sum(w^2). */
static double ess_of(const double* w, long n) { return 1.0 / pairwise_sum(w, 0, n - 1, 1); }

/* ------------------------------------------------------------------------ */
/* Kalman filter (kalman.jl:23-79, kalman_gradient.jl:12-29), FP64.         */
/* tv = 0: homogeneous (one A, b, Q, H, c, R).  tv = 1: non-homogeneous, the
 * parameters calc_params(dyn, t), calc_params(obs, t) of every step t = 1..T
 * (models/linear_gaussian.jl:44-63; GFTest NonHomogeneousLinearGaussian*,
 * GFTest/models/linear_gaussian.jl:42-95) stored step-major, block t-1 of
 * each array column-major. */
typedef struct {
  int dx, dy;
  const double *mu0, *Sigma0, *A, *b, *Q, *H, *c, *R;
  int tv;
} or_lg_model;

/* Parameters of 0-based step s (1-based step s + 1). */
typedef struct {
  const double *A, *b, *Q, *H, *c, *R;
} or_step_params;
static or_step_params step_params(const or_lg_model* m, int s) {
  const size_t k = m->tv ? (size_t)s : 0;
  const size_t dx = m->dx, dy = m->dy;
  or_step_params p = {m->A + k * dx * dx, m->b + k * dx, m->Q + k * dx * dx,
                      m->H + k * dy * dx, m->c + k * dy, m->R + k * dy * dy};
  return p;
}

typedef struct { /* workspace for one KF step */
  double *L, *Lp, *LR, *LS, *tmp, *tmp2, *Sp, *PHt, *S, *K, *IKH, *Sraw, *z, *w;
} kf_ws;
static kf_ws kf_ws_alloc(int dx, int dy) {
  kf_ws w;
  int m = dx > dy ? dx : dy;
  size_t mm2 = (size_t)m * m;
  w.L = calloc(mm2, 8); w.Lp = calloc(mm2, 8); w.LR = calloc(mm2, 8); w.LS = calloc(mm2, 8);
  w.tmp = calloc(mm2, 8); w.tmp2 = calloc(mm2, 8); w.Sp = calloc(mm2, 8); w.PHt = calloc(mm2, 8);
  w.S = calloc(mm2, 8); w.K = calloc(mm2, 8); w.IKH = calloc(mm2, 8); w.Sraw = calloc(mm2, 8);
  w.z = calloc(m, 8); w.w = calloc(m, 8);
  return w;
}
static void kf_ws_free(kf_ws* w) {
  free(w->L); free(w->Lp); free(w->LR); free(w->LS); free(w->tmp); free(w->tmp2);
  free(w->Sp); free(w->PHt); free(w->S); free(w->K); free(w->IKH); free(w->Sraw);
  free(w->z); free(w->w);
}

/* kalman_predict (kalman.jl:42-49): mu' = A mu + b; Sigma' = X_A_Xt(Sigma, A) + Q,
 * Sigma carried as a PDMat (matrix + lower factor). Returns status. */
static int kf_predict(int dx, const double* A, const double* b, const double* Q,
                      double* mu, double* Sig, double* L, kf_ws* ws) {
  double* m2 = ws->w;
  mv(dx, dx, A, mu, m2);
  for (int i = 0; i < dx; ++i) mu[i] = m2[i] + b[i];
  x_a_xt_chol(dx, dx, A, L, ws->Sp, ws->tmp);
  for (int i = 0; i < dx * dx; ++i) Sig[i] = ws->Sp[i] + Q[i];
  return or_chol_lower(dx, Sig, L); /* MvNormal(mu, Matrix) -> PDMat */
}

/* _kalman_update_cached (kalman_gradient.jl:12-23) with the Joseph form
 * (kalman.jl:55-66).  mu/Sig/L are the predicted PDMat on entry and the
 * filtered PDMat on exit; returns ll via *ll. */
static int kf_update(int dx, int dy, const double* H, const double* c, const double* R,
                     const double* LR, const double* y, double jitter, int use_jitter,
                     double* mu, double* Sig, double* L, double* ll, kf_ws* ws) {
  /* z = y - H mu - c */
  mv(dy, dx, H, mu, ws->z);
  for (int i = 0; i < dy; ++i) ws->z[i] = y[i] - ws->z[i] - c[i];
  /* S = PDMat(X_A_Xt(Sigma_pred, H) + R) */
  x_a_xt_chol(dy, dx, H, L, ws->S, ws->tmp);
  for (int i = 0; i < dy * dy; ++i) ws->S[i] += R[i];
  if (or_chol_lower(dy, ws->S, ws->LS)) return OR_NOT_PD;
  /* K = Sigma_pred * H' / S  ->  K^T = S \ (H Sigma_pred) */
  mmT(dx, dx, dy, Sig, H, ws->PHt); /* Sigma H^T (dx x dy) */
  for (int r = 0; r < dx; ++r) {
    for (int j = 0; j < dy; ++j) ws->w[j] = ws->PHt[r + j * dx];
    trsv_lower(dy, ws->LS, ws->w);
    trsv_lowerT(dy, ws->LS, ws->w);
    for (int j = 0; j < dy; ++j) ws->K[r + j * dx] = ws->w[j];
  }
  /* I_KH = I - K H ; Sigma_raw = X_A_Xt(Sigma_pred, I_KH) + X_A_Xt(R, K) */
  mm(dx, dy, dx, ws->K, H, ws->IKH);
  for (int j = 0; j < dx; ++j)
    for (int i = 0; i < dx; ++i) ws->IKH[i + j * dx] = (i == j ? 1.0 : 0.0) - ws->IKH[i + j * dx];
  x_a_xt_chol(dx, dx, ws->IKH, L, ws->Sraw, ws->tmp);
  x_a_xt_chol(dx, dy, ws->K, LR, ws->tmp2, ws->tmp);
  for (int i = 0; i < dx * dx; ++i) ws->Sraw[i] += ws->tmp2[i];
  /* mu_filt = mu_pred + K z */
  mv(dx, dy, ws->K, ws->z, ws->w);
  for (int i = 0; i < dx; ++i) mu[i] += ws->w[i];
  if (use_jitter)
    for (int i = 0; i < dx; ++i) ws->Sraw[i + i * dx] += jitter;
  /* PDMat(Symmetric(Sigma_raw)): upper triangle mirrored */
  for (int j = 0; j < dx; ++j)
    for (int i = 0; i < dx; ++i) Sig[i + j * dx] = i <= j ? ws->Sraw[i + j * dx] : ws->Sraw[j + i * dx];
  /* ll = logpdf(MvNormal(z, S), 0) */
  for (int i = 0; i < dy; ++i) ws->w[i] = -ws->z[i];
  *ll = logpdf_chol(dy, ws->LS, ws->w, ws->tmp);
  return or_chol_lower(dx, Sig, L);
}

/* filter(model, KalmanFilter(), ys) (GeneralisedFilters.jl:58-84).
 * ys: T*dy (ys[t*dy + i]).  Outputs (nullable): ll_steps[T], mus[T*dx],
 * Sigmas[T*dx*dx].  Returns status; *ll gets the total. */
int or_kf_filter(const or_lg_model* m, int T, const double* ys, double jitter, int use_jitter,
                 double* ll, double* ll_steps, double* mus, double* Sigmas) {
  int dx = m->dx, dy = m->dy, st = OR_OK;
  kf_ws ws = kf_ws_alloc(dx, dy);
  double* mu = calloc(dx, 8);
  double* Sig = calloc((size_t)dx * dx, 8);
  double* L = calloc((size_t)dx * dx, 8);
  double* LR = calloc((size_t)dy * dy, 8);
  memcpy(mu, m->mu0, 8 * dx);
  memcpy(Sig, m->Sigma0, 8 * (size_t)dx * dx);
  double tot = 0.0;
  if ((st = or_chol_lower(dx, Sig, L)) || (st = or_chol_lower(dy, m->R, LR))) goto done;
  for (int t = 0; t < T; ++t) {
    double l = 0.0;
    const or_step_params P = step_params(m, t);
    if (m->tv && t > 0 && (st = or_chol_lower(dy, P.R, LR))) break;
    if ((st = kf_predict(dx, P.A, P.b, P.Q, mu, Sig, L, &ws))) break;
    if ((st = kf_update(dx, dy, P.H, P.c, P.R, LR, ys + (size_t)t * dy, jitter, use_jitter,
                        mu, Sig, L, &l, &ws)))
      break;
    tot += l;
    if (ll_steps) ll_steps[t] = l;
    if (mus) memcpy(mus + (size_t)t * dx, mu, 8 * dx);
    if (Sigmas) memcpy(Sigmas + (size_t)t * dx * dx, Sig, 8 * (size_t)dx * dx);
  }
done:
  *ll = tot;
  free(mu); free(Sig); free(L); free(LR);
  kf_ws_free(&ws);
  return st;
}

/* smooth(model, KalmanSmoother(), ys) (kalman.jl:206-234) with the RTS step of
 * backward_smooth (kalman.jl:89-126): the forward filter(model, KalmanFilter(),
 * ys) without jitter, then for t = T-1 down to 1
 *   mu_pred = A mu_f + b, Sigma_pred = A Sigma_f A' + Q,
 *   G = Sigma_f A' Sigma_pred^-1 (Cholesky solve; Sigma_pred as PDMat),
 *   mu_s = mu_f + G (mu_s' - mu_pred), Sigma_s = Sigma_f + G (Sigma_s' - Sigma_pred) G',
 *   Sigma_s symmetrised from its upper triangle (PDMat(Symmetric(.))).
 * Outputs the smoothed mus[T*dx] and Sigmas[T*dx*dx] (column-major) for every t;
 * the last step is the filtered one.  *ll gets the forward log-likelihood. */
int or_rts_smooth(const or_lg_model* m, int T, const double* ys, double* ll, double* mus,
                  double* Sigmas) {
  const int dx = m->dx;
  int st = or_kf_filter(m, T, ys, 0.0, 0, ll, NULL, mus, Sigmas);
  if (st) return st;
  const size_t n2 = (size_t)dx * dx;
  double *mp = malloc(8 * dx), *d = malloc(8 * dx), *ms = malloc(8 * dx);
  double *T1 = malloc(8 * n2), *Sp = malloc(8 * n2), *L = malloc(8 * n2), *X = malloc(8 * n2);
  double *D = malloc(8 * n2), *T2 = malloc(8 * n2), *Ss = malloc(8 * n2);
  for (int t = T - 2; t >= 0 && !st; --t) {
    /* the prediction from t to t + 1 uses the parameters of step t + 1 */
    const or_step_params P = step_params(m, t + 1);
    const double *A = P.A, *b = P.b, *Q = P.Q;
    const double* mf = mus + (size_t)t * dx;
    const double* Sf = Sigmas + (size_t)t * n2;
    const double* mn = mus + (size_t)(t + 1) * dx;   /* smoothed at t+1 */
    const double* Sn = Sigmas + (size_t)(t + 1) * n2;
    for (int i = 0; i < dx; ++i) {
      double v = b[i];
      for (int k = 0; k < dx; ++k) v += A[i + k * dx] * mf[k];
      mp[i] = v;
    }
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i) {
        double v = 0.0;
        for (int k = 0; k < dx; ++k) v += A[i + k * dx] * Sf[k + j * dx];
        T1[i + j * dx] = v; /* A Sigma_f */
      }
    /* Sigma_pred = X_A_Xt(Sigma_f, A) + Q through the Cholesky factor of Sigma_f
     * (kalman_predict, kalman.jl:42-49) */
    if ((st = or_chol_lower(dx, Sf, L))) break;
    x_a_xt_chol(dx, dx, A, L, Sp, D);
    for (size_t e = 0; e < n2; ++e) Sp[e] += Q[e];
    if ((st = or_chol_lower(dx, Sp, L))) break;
    /* G' = Sigma_pred^-1 (A Sigma_f): column by column, L L' x = T1(:, j) */
    for (int j = 0; j < dx; ++j) {
      double* x = X + (size_t)j * dx;
      for (int i = 0; i < dx; ++i) x[i] = T1[i + j * dx];
      for (int i = 0; i < dx; ++i) { /* forward */
        double v = x[i];
        for (int k = 0; k < i; ++k) v -= L[i + k * dx] * x[k];
        x[i] = v / L[i + i * dx];
      }
      for (int i = dx - 1; i >= 0; --i) { /* back (L') */
        double v = x[i];
        for (int k = i + 1; k < dx; ++k) v -= L[k + i * dx] * x[k];
        x[i] = v / L[i + i * dx];
      }
    }
    /* X(:, j) = G'(:, j) = G(j, :), i.e. G[i][k] = X[k + i*dx] */
    for (int i = 0; i < dx; ++i) d[i] = mn[i] - mp[i];
    for (int i = 0; i < dx; ++i) {
      double v = mf[i];
      for (int k = 0; k < dx; ++k) v += X[k + i * dx] * d[k];
      ms[i] = v;
    }
    for (size_t e = 0; e < n2; ++e) D[e] = Sn[e] - Sp[e];
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i) {
        double v = 0.0;
        for (int k = 0; k < dx; ++k) v += X[k + i * dx] * D[k + j * dx];
        T2[i + j * dx] = v; /* G D */
      }
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i <= j; ++i) {
        double v = Sf[i + j * dx];
        for (int k = 0; k < dx; ++k) v += T2[i + k * dx] * X[k + j * dx];
        Ss[i + j * dx] = v;
        Ss[j + i * dx] = v;
      }
    memcpy(mus + (size_t)t * dx, ms, 8 * dx);
    memcpy(Sigmas + (size_t)t * n2, Ss, 8 * n2);
  }
  free(mp); free(d); free(ms); free(T1); free(Sp); free(L); free(X); free(D); free(T2); free(Ss);
  return st;
}

/* ------------------------------------------------------------------------ */
/* Square-root Kalman filter (srkf.jl:93-176).                               */
/* Householder QR of M (m x n, m >= n), returns R (n x n upper, col-major)
 * with rows sign-corrected so diag(R) >= 0 (srkf.jl:83). */
static void qr_r_signfix(int m, int n, double* M, double* R) {
  double* v = malloc(sizeof(double) * m);
  for (int k = 0; k < n; ++k) {
    double nrm = 0.0;
    for (int i = k; i < m; ++i) nrm += M[i + k * m] * M[i + k * m];
    nrm = sqrt(nrm);
    if (nrm == 0.0) continue;
    double x0 = M[k + k * m];
    double alpha = x0 >= 0 ? -nrm : nrm;
    for (int i = k; i < m; ++i) v[i] = M[i + k * m];
    v[k] -= alpha;
    double vv = 0.0;
    for (int i = k; i < m; ++i) vv += v[i] * v[i];
    if (vv == 0.0) continue;
    for (int j = k; j < n; ++j) {
      double s = 0.0;
      for (int i = k; i < m; ++i) s += v[i] * M[i + j * m];
      s = 2.0 * s / vv;
      for (int i = k; i < m; ++i) M[i + j * m] -= s * v[i];
    }
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) R[i + j * n] = i <= j ? M[i + j * m] : 0.0;
  for (int i = 0; i < n; ++i) {
    double d = R[i + i * n];
    double s = d > 0 ? 1.0 : (d < 0 ? -1.0 : 0.0);
    for (int j = 0; j < n; ++j) R[i + j * n] *= s;
  }
  free(v);
}

/* filter(model, SRKF(), ys).  U is the upper factor, Sigma = U^T U. */
int or_srkf_filter(const or_lg_model* m, int T, const double* ys, double jitter, int use_jitter,
                   double* ll, double* ll_steps, double* mus, double* Sigmas) {
  int dx = m->dx, dy = m->dy, st = OR_OK, nn = dx + dy;
  double *L = calloc((size_t)dx * dx, 8), *U = calloc((size_t)dx * dx, 8);
  double *LQ = calloc((size_t)dx * dx, 8), *LR = calloc((size_t)dy * dy, 8);
  double *M = calloc((size_t)2 * nn * nn, 8), *Rm = calloc((size_t)nn * nn, 8);
  double *mu = calloc(dx, 8), *tmp = calloc(nn, 8), *z = calloc(dy, 8), *w = calloc(dy, 8);
  double tot = 0.0;
  memcpy(mu, m->mu0, 8 * dx);
  if ((st = or_chol_lower(dx, m->Sigma0, L)) || (st = or_chol_lower(dx, m->Q, LQ)) ||
      (st = or_chol_lower(dy, m->R, LR)))
    goto done;
  for (int j = 0; j < dx; ++j)
    for (int i = 0; i < dx; ++i) U[i + j * dx] = L[j + i * dx]; /* U = L^T */
  for (int t = 0; t < T; ++t) {
    /* predict: mu = A mu + b; U = R(qr([U_Q; U A^T])) */
    mv(dx, dx, m->A, mu, tmp);
    for (int i = 0; i < dx; ++i) mu[i] = tmp[i] + m->b[i];
    int mr = 2 * dx;
    for (int j = 0; j < dx; ++j) {
      for (int i = 0; i < dx; ++i) M[i + j * mr] = LQ[j + i * dx]; /* U_Q = LQ^T */
      for (int i = 0; i < dx; ++i) {                            /* (U A^T)_{ij} */
        double s = 0.0;
        for (int p = 0; p < dx; ++p) s += U[i + p * dx] * m->A[j + p * dx];
        M[dx + i + j * mr] = s;
      }
    }
    qr_r_signfix(mr, dx, M, U);
    /* update: M = [[U_R, 0], [U H^T, U]] */
    for (int j = 0; j < nn; ++j)
      for (int i = 0; i < nn; ++i) M[i + j * nn] = 0.0;
    for (int j = 0; j < dy; ++j)
      for (int i = 0; i < dy; ++i) M[i + j * nn] = LR[j + i * dy];
    for (int j = 0; j < dy; ++j)
      for (int i = 0; i < dx; ++i) {
        double s = 0.0;
        for (int p = 0; p < dx; ++p) s += U[i + p * dx] * m->H[j + p * dy];
        M[dy + i + j * nn] = s;
      }
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i) M[dy + i + (dy + j) * nn] = U[i + j * dx];
    qr_r_signfix(nn, nn, M, Rm);
    /* U_S = R[1:dy,1:dy]; PHt = R[1:dy, dy+1:end]'; U = R[dy+1:end, dy+1:end] */
    mv(dy, dx, m->H, mu, z);
    for (int i = 0; i < dy; ++i) z[i] = ys[(size_t)t * dy + i] - z[i] - m->c[i];
    /* w = U_S' \ z : U_S' is lower */
    for (int i = 0; i < dy; ++i) {
      double s = z[i];
      for (int k = 0; k < i; ++k) s -= Rm[k + i * nn] * w[k];
      w[i] = s / Rm[i + i * nn];
    }
    for (int i = 0; i < dx; ++i) {
      double s = 0.0;
      for (int k = 0; k < dy; ++k) s += Rm[k + (dy + i) * nn] * w[k];
      mu[i] += s;
    }
    double ww = 0.0, ld = 0.0;
    for (int i = 0; i < dy; ++i) { ww += w[i] * w[i]; ld += log(Rm[i + i * nn]); }
    double l = -0.5 * (ww + 2.0 * ld + dy * LOG2PI);
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i) U[i + j * dx] = Rm[dy + i + (dy + j) * nn];
    if (use_jitter)
      for (int i = 0; i < dx; ++i) U[i + i * dx] += jitter;
    for (int i = 0; i < dx; ++i)
      if (!(U[i + i * dx] > 0.0)) { st = OR_NOT_PD; }
    if (st) break;
    tot += l;
    if (ll_steps) ll_steps[t] = l;
    if (mus) memcpy(mus + (size_t)t * dx, mu, 8 * dx);
    if (Sigmas) { /* Sigma = U^T U */
      double* S = Sigmas + (size_t)t * dx * dx;
      for (int j = 0; j < dx; ++j)
        for (int i = 0; i < dx; ++i) {
          double s = 0.0;
          for (int p = 0; p < dx; ++p) s += U[p + i * dx] * U[p + j * dx];
          S[i + j * dx] = s;
        }
    }
  }
done:
  *ll = tot;
  free(L); free(U); free(LQ); free(LR); free(M); free(Rm); free(mu); free(tmp); free(z); free(w);
  return st;
}

/* ------------------------------------------------------------------------ */
/* Particle filter (particles.jl:36-90,147-162,175-245; resamplers.jl;      */
/* containers.jl:140-173).                                                   */
typedef struct {
  int kind;          /* OR_SYSTEMATIC / OR_STRATIFIED / OR_MULTINOMIAL */
  int conv;          /* OR_CONV_CPU / OR_CONV_CUDAEXT */
  double threshold;  /* ESSResampler threshold */
  const int8_t* schedule; /* nullable: per step -1 = ESS rule, 0 = keep, 1 = resample */
} or_resample_cfg;

typedef struct {
  int kind;           /* OR_PROP_* */
  double k;           /* overdispersion factor */
  int lookahead;      /* AuxiliaryParticleFilter first stage: 1 MeanPredictive, 2 DrawPredictive */
} or_proposal;

typedef struct { /* nullable outputs */
  double* ll_steps;   /* T */
  double* ess;        /* T: ESS evaluated by the resampling decision at step t */
  int8_t* resampled;  /* T */
  int32_t* ancestors; /* T*N (1-based; identity when not resampled) */
  double* margins;    /* T*N boundary margins (0 when not resampled) */
  double* means;      /* T*dx weighted filtered means */
  double* x_final;    /* N*dx */
  double* logw_final; /* N (normalised) */
  long* clamps;       /* scalar */
  double* x_all;      /* (T+1)*N*dx: states after initialisation and after every step */
  double* logw_all;   /* T*N: normalised log-weights after every update (PostUpdate) */
} or_pf_out;

/* Noise source: injected (noise != NULL, layout [(T+1)][dx][N], step 0 = prior
 * draw) or Philox with `seed` (counter layout shared with the CUDA library). */
static void draw_normals(const double* noise, uint64_t seed, int dx, long N, int t, long i,
                         double* e) {
  if (noise) {
    for (int d = 0; d < dx; ++d) e[d] = noise[((size_t)t * dx + d) * N + i];
  } else {
    double buf[4];
    for (int q = 0; q * 4 < dx; ++q) {
      or_philox_normals4(seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, buf);
      for (int r = 0; r < 4 && q * 4 + r < dx; ++r) e[q * 4 + r] = buf[r];
    }
  }
}
/* The linear-Gaussian particle filter's noise: as draw_normals, except that a
 * one-dimensional state takes normal i % 4 of the call (i / 4, t, 0) (the
 * library's 1-D layout: one Philox call serves four particles). */
static void draw_normals_lg(const double* noise, uint64_t seed, int dx, long N, int t, long i,
                            double* e) {
  if (noise || dx != 1) {
    draw_normals(noise, seed, dx, N, t, i, e);
  } else {
    double buf[4];
    or_philox_normals4(seed, (uint32_t)(i >> 2), (uint32_t)t, 0u, buf);
    e[0] = buf[i & 3];
  }
}
static void draw_uniforms(const double* uniforms, uint64_t seed, int kind, long N, int t,
                          double* u) {
  /* t is 1-based step index; injected layout: systematic [T], else [T][N] */
  if (kind == OR_SYSTEMATIC) {
    u[0] = uniforms ? uniforms[t - 1] : or_philox_uniform(seed, 0u, (uint32_t)t);
  } else {
    for (long j = 0; j < N; ++j)
      u[j] = uniforms ? uniforms[(size_t)(t - 1) * N + j] : or_philox_uniform(seed, (uint32_t)j, (uint32_t)t);
  }
}

/* Resample-or-preserve (resamplers.jl:149-196, 53-79).  `uniform` marks the
 * TypelessZero initial weights (containers.jl:19-65).  Returns 1 if resampled. */
static int maybe_resample(const or_resample_cfg* rc, int t, long N, int width, double* x,
                          double* xtmp, double* logw, int* uniform, double* wbuf,
                          double* ubuf, const double* uniforms, uint64_t seed, int32_t* anc,
                          double* margins, double* ess_out, long* clamps) {
  if (*uniform) {
    for (long i = 0; i < N; ++i) wbuf[i] = 1.0 / (double)N; /* softmax(TypelessZero) */
  } else {
    softmax(logw, N, wbuf);
  }
  double ess = ess_of(wbuf, N);
  if (ess_out) *ess_out = ess;
  int sched = rc->schedule ? rc->schedule[t - 1] : -1;
  int doit = sched >= 0 ? sched : (rc->threshold * (double)N >= ess);
  if (!doit) {
    if (anc)
      for (long i = 0; i < N; ++i) anc[i] = (int32_t)(i + 1);
    if (margins)
      for (long i = 0; i < N; ++i) margins[i] = 0.0;
    return 0;
  }
  draw_uniforms(uniforms, seed, rc->kind, N, t, ubuf);
  int32_t* a = anc ? anc : (int32_t*)malloc(sizeof(int32_t) * N);
  *clamps += or_sample_ancestors(rc->kind, rc->conv, N, wbuf, ubuf, a, margins);
  memcpy(xtmp, x, sizeof(double) * N * width);
  for (long i = 0; i < N; ++i)
    memcpy(x + (size_t)i * width, xtmp + (size_t)(a[i] - 1) * width, sizeof(double) * width);
  for (long i = 0; i < N; ++i) logw[i] = 0.0;
  *uniform = 0;
  if (!anc) free(a);
  return 1;
}

/* A guided proposal's factors for one step's (Q, H, c, R): OverdispersedProposal
 * MvNormal(A x + b, k Q) (GFTest/proposals.jl:39-50) gives Lq = chol(k Q);
 * OptimalProposal kalman_update(MvNormal(A x + b, Q), (H, c, R), y)
 * (GFTest/proposals.jl:20-31) gives the gain Kq and covariance Sq = Lq Lq',
 * which do not depend on x and are computed with the arithmetic kf_update
 * applies to every particle.  Bootstrap: nothing. */
static int guided_factors(int dx, int dy, const or_proposal* prop, const double* Q, const double* LQ,
                          const double* H, const double* c, const double* R, const double* LR,
                          double* Kq, double* Sq, double* Lq) {
  int st = OR_OK;
  if (prop->kind == OR_PROP_OVERDISPERSED) {
    double* kQ = malloc(sizeof(double) * dx * dx);
    for (int i = 0; i < dx * dx; ++i) kQ[i] = prop->k * Q[i];
    st = or_chol_lower(dx, kQ, Lq);
    free(kQ);
  } else if (prop->kind == OR_PROP_OPTIMAL) {
    kf_ws ws = kf_ws_alloc(dx, dy);
    double* mu = calloc(dx, 8);
    double* Sg = malloc(sizeof(double) * dx * dx);
    double* Lg = malloc(sizeof(double) * dx * dx);
    double* yz = calloc(dy, 8);
    memcpy(Sg, Q, 8 * dx * dx);
    memcpy(Lg, LQ, 8 * dx * dx);
    double lldummy;
    /* with mu = 0 and y = c the innovation is 0; K and Sigma_q are what we need */
    memcpy(yz, c, 8 * dy);
    st = kf_update(dx, dy, H, c, R, LR, yz, 0.0, 0, mu, Sg, Lg, &lldummy, &ws);
    memcpy(Kq, ws.K, 8 * dx * dy);
    memcpy(Sq, Sg, 8 * dx * dx);
    memcpy(Lq, Lg, 8 * dx * dx);
    free(mu); free(Sg); free(Lg); free(yz);
    kf_ws_free(&ws);
  }
  return st;
}

/* filter(rng, model, ParticleFilter(N, proposal; threshold, resampler), ys).
 * Returns status; *ll is the log-evidence. */
int or_pf_run(const or_lg_model* m, const or_proposal* prop, const or_resample_cfg* rc,
              long N, int T, const double* ys, const double* noise, const double* uniforms,
              uint64_t seed, double* ll, or_pf_out* out) {
  int dx = m->dx, dy = m->dy;
  double* x = malloc(sizeof(double) * N * dx);
  double* xtmp = malloc(sizeof(double) * N * dx);
  double* logw = calloc(N, 8);
  double* wbuf = malloc(sizeof(double) * N);
  double* ubuf = malloc(sizeof(double) * N);
  double* eta = malloc(sizeof(double) * N);
  double* aux = malloc(sizeof(double) * N);
  double *L0 = calloc((size_t)dx * dx, 8), *LQ = calloc((size_t)dx * dx, 8);
  double *LR = calloc((size_t)dy * dy, 8), *Lq = calloc((size_t)dx * dx, 8);
  double *Kq = calloc((size_t)dx * dy, 8), *Sq = calloc((size_t)dx * dx, 8);
  int st = OR_OK, uniform = 1;
  long clamps = 0;
  double tot = 0.0;
  if ((st = or_chol_lower(dx, m->Sigma0, L0)) || (st = or_chol_lower(dx, m->Q, LQ)) ||
      (st = or_chol_lower(dy, m->R, LR)))
    goto done;
  if ((st = guided_factors(dx, dy, prop, m->Q, LQ, m->H, m->c, m->R, LR, Kq, Sq, Lq))) goto done;
  /* initialise (particles.jl:36-50): x ~ MvNormal(mu0, Sigma0) */
  for (long i = 0; i < N; ++i) {
    double e[64], v[64];
    draw_normals_lg(noise, seed, dx, N, 0, i, e);
    mv(dx, dx, L0, e, v);
    for (int d = 0; d < dx; ++d) x[(size_t)i * dx + d] = m->mu0[d] + v[d];
  }
  if (out && out->x_all) memcpy(out->x_all, x, sizeof(double) * N * dx);
  for (int t = 1; t <= T; ++t) {
    int32_t* anc_t = out && out->ancestors ? out->ancestors + (size_t)(t - 1) * N : NULL;
    double* mar_t = out && out->margins ? out->margins + (size_t)(t - 1) * N : NULL;
    double ess = 0.0, baseline;
    int res;
    /* this step's parameters (calc_params(dyn, t), calc_params(obs, t)) */
    const or_step_params SP = step_params(m, t - 1);
    if (m->tv && ((st = or_chol_lower(dx, SP.Q, LQ)) || (st = or_chol_lower(dy, SP.R, LR)) ||
                  (st = guided_factors(dx, dy, prop, SP.Q, LQ, SP.H, SP.c, SP.R, LR, Kq, Sq, Lq))))
      goto done;
    const double *mA = SP.A, *mb = SP.b, *mH = SP.H, *mc = SP.c;
    if (prop->lookahead) {
      /* AuxiliaryParticleFilter step (particles.jl:311-345): log eta_i =
       * logpdf(obs, A x_i + b, y_t) (MeanPredictive, :359-365; predictive_loglik
       * :386-394), then maybe_resample with AuxiliaryResampler (resamplers.jl:
       * 109-116): weights softmax(logw + log eta), ESS decision on them. */
      const double* yl = ys + (size_t)(t - 1) * dy;
      for (long i = 0; i < N; ++i) {
        double mx[64], hx[64], dif[64], tmpd[64];
        mv(dx, dx, mA, x + (size_t)i * dx, mx);
        for (int d = 0; d < dx; ++d) mx[d] += mb[d];
        if (prop->lookahead == 2) {
          /* DrawPredictive (particles.jl:377-384): x* ~ MvNormal(A x + b, Q), the draw
           * from the Philox stream tagged TAG_LOOKAHEAD with counters (i, t, q) */
          double e[64], v[64], buf[4];
          for (int q = 0; 4 * q < dx; ++q) {
            philox_normals4_tag(seed, (uint32_t)i, (uint32_t)t, (uint32_t)q, TAG_LOOKAHEAD, buf);
            for (int r = 0; r < 4 && 4 * q + r < dx; ++r) e[4 * q + r] = buf[r];
          }
          mv(dx, dx, LQ, e, v);
          for (int d = 0; d < dx; ++d) mx[d] += v[d];
        }
        mv(dy, dx, mH, mx, hx);
        for (int k = 0; k < dy; ++k) dif[k] = yl[k] - hx[k] - mc[k];
        eta[i] = logpdf_chol(dy, LR, dif, tmpd);
        aux[i] = (uniform ? 0.0 : logw[i]) + eta[i];
      }
      softmax(aux, N, wbuf);
      ess = ess_of(wbuf, N);
      int sched = rc->schedule ? rc->schedule[t - 1] : -1;
      res = sched >= 0 ? sched : (rc->threshold * (double)N >= ess);
      if (res) {
        /* construct_new_state with auxiliary weights (resamplers.jl:118-143):
         * log_w = -log eta[a]; ll_baseline = -((LSE_1 - LSE_2) + (LSE_3 - LSE_4)) */
        draw_uniforms(uniforms, seed, rc->kind, N, t, ubuf);
        int32_t* a = anc_t ? anc_t : (int32_t*)malloc(sizeof(int32_t) * N);
        clamps += or_sample_ancestors(rc->kind, rc->conv, N, wbuf, ubuf, a, mar_t);
        memcpy(xtmp, x, sizeof(double) * N * dx);
        for (long i = 0; i < N; ++i)
          memcpy(x + (size_t)i * dx, xtmp + (size_t)(a[i] - 1) * dx, sizeof(double) * dx);
        const double lse1 = or_logsumexp(aux, N);
        const double lse2 = uniform ? log((double)N) : or_logsumexp(logw, N);
        for (long i = 0; i < N; ++i) logw[i] = -eta[a[i] - 1];
        const double lse3 = or_logsumexp(logw, N), lse4 = log((double)N);
        const double llb = -((lse1 - lse2) + (lse3 - lse4));
        /* predict (particles.jl:70-73): logsumexp(log_weights) + ll_baseline */
        baseline = lse3 + llb;
        uniform = 0;
        if (!anc_t) free(a);
      } else {
        if (anc_t)
          for (long i = 0; i < N; ++i) anc_t[i] = (int32_t)(i + 1);
        if (mar_t)
          for (long i = 0; i < N; ++i) mar_t[i] = 0.0;
        baseline = uniform ? log((double)N) : or_logsumexp(logw, N);
      }
    } else {
      int was_uniform = uniform;
      res = maybe_resample(rc, t, N, dx, x, xtmp, logw, &uniform, wbuf, ubuf, uniforms, seed,
                           anc_t, mar_t, &ess, &clamps);
      /* predict (particles.jl:52-74): baseline = logsumexp(log_weights) */
      baseline = (was_uniform && !res) ? log((double)N) : or_logsumexp(logw, N);
    }
    if (out && out->ess) out->ess[t - 1] = ess;
    if (out && out->resampled) out->resampled[t - 1] = (int8_t)res;
    const double* y = ys + (size_t)(t - 1) * dy;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (long i = 0; i < N; ++i) {
      double e[64], mx[64], v[64], xn[64], tmpd[64], dif[64];
      double* xi = x + (size_t)i * dx;
      draw_normals_lg(noise, seed, dx, N, t, i, e);
      mv(dx, dx, mA, xi, mx);
      for (int d = 0; d < dx; ++d) mx[d] += mb[d]; /* A x + b */
      double inc = 0.0;
      if (prop->kind == OR_PROP_BOOTSTRAP) {
        mv(dx, dx, LQ, e, v);
        for (int d = 0; d < dx; ++d) xn[d] = mx[d] + v[d];
      } else {
        double mq[64];
        if (prop->kind == OR_PROP_OPTIMAL) {
          double z[64];
          mv(dy, dx, mH, mx, z);
          for (int k = 0; k < dy; ++k) z[k] = y[k] - z[k] - mc[k];
          mv(dx, dy, Kq, z, v);
          for (int d = 0; d < dx; ++d) mq[d] = mx[d] + v[d];
        } else {
          for (int d = 0; d < dx; ++d) mq[d] = mx[d];
        }
        mv(dx, dx, Lq, e, v);
        for (int d = 0; d < dx; ++d) xn[d] = mq[d] + v[d];
        /* propogate (particles.jl:175-195): log p(x'|x) - log q(x'|x,y) */
        for (int d = 0; d < dx; ++d) dif[d] = xn[d] - mx[d];
        double lp = logpdf_chol(dx, LQ, dif, tmpd);
        for (int d = 0; d < dx; ++d) dif[d] = xn[d] - mq[d];
        double lq = logpdf_chol(dx, Lq, dif, tmpd);
        inc = lp - lq;
      }
      memcpy(xi, xn, sizeof(double) * dx);
      /* update (particles.jl:133-145): += logpdf(MvNormal(H x + c, R), y) */
      double hx[64];
      mv(dy, dx, mH, xn, hx);
      for (int k = 0; k < dy; ++k) dif[k] = y[k] - hx[k] - mc[k];
      double lo = logpdf_chol(dy, LR, dif, tmpd);
      logw[i] = logw[i] + inc + lo;
    }
    uniform = 0;
    if (out && out->x_all) memcpy(out->x_all + (size_t)t * N * dx, x, sizeof(double) * N * dx);
    /* marginalise! (containers.jl:160-173) */
    double lse = or_logsumexp(logw, N);
    double inc = lse - baseline;
    for (long i = 0; i < N; ++i) logw[i] -= lse;
    tot += inc;
    if (out && out->ll_steps) out->ll_steps[t - 1] = inc;
    if (out && out->logw_all) memcpy(out->logw_all + (size_t)(t - 1) * N, logw, sizeof(double) * N);
    if (out && out->means) {
      double* mo = out->means + (size_t)(t - 1) * dx;
      for (int d = 0; d < dx; ++d) mo[d] = 0.0;
      for (long i = 0; i < N; ++i) {
        double wi = exp(logw[i]);
        for (int d = 0; d < dx; ++d) mo[d] += wi * x[(size_t)i * dx + d];
      }
    }
  }
  if (out && out->x_final) memcpy(out->x_final, x, sizeof(double) * N * dx);
  if (out && out->logw_final) memcpy(out->logw_final, logw, sizeof(double) * N);
done:
  if (out && out->clamps) *out->clamps = clamps;
  *ll = tot;
  free(x); free(xtmp); free(logw); free(wbuf); free(ubuf); free(eta); free(aux);
  free(L0); free(LQ); free(LR); free(Lq); free(Kq); free(Sq);
  return st;
}

/* One PF step from a given state (teacher forcing for FP32 parity checks).
 * x (N*dx), logw (N, normalised) are updated in place; `uniform` marks the
 * initial TypelessZero weights.  u: the resampling uniforms of this step
 * (systematic: 1 value, else N); noise: this step's [dx][N] block. */
int or_pf_step(const or_lg_model* m, const or_resample_cfg* rc, long N, int t, const double* y,
               const double* noise_t, const double* u, int uniform, double* x, double* logw,
               int32_t* anc, double* margins, double* ess, int8_t* resampled,
               double* ll_inc) {
  int dx = m->dx, dy = m->dy;
  double *LQ = calloc((size_t)dx * dx, 8), *LR = calloc((size_t)dy * dy, 8);
  double* xtmp = malloc(sizeof(double) * N * dx);
  double* wbuf = malloc(sizeof(double) * N);
  int st = OR_OK;
  long clamps = 0;
  if ((st = or_chol_lower(dx, m->Q, LQ)) || (st = or_chol_lower(dy, m->R, LR))) goto done;
  {
    or_resample_cfg rc1 = *rc;
    int8_t sch = rc->schedule ? rc->schedule[0] : -1;
    rc1.schedule = &sch;
    int was_uniform = uniform;
    double* ubuf = malloc(sizeof(double) * N);
    /* `u` holds this step's uniforms: inject them as step-1 data */
    int res = maybe_resample(&rc1, 1, N, dx, x, xtmp, logw, &uniform, wbuf, ubuf, u, 0, anc,
                             margins, ess, &clamps);
    free(ubuf);
    *resampled = (int8_t)res;
    double baseline = (was_uniform && !res) ? log((double)N) : or_logsumexp(logw, N);
    for (long i = 0; i < N; ++i) {
      double e[64], mx[64], v[64], dif[64], tmpd[64], hx[64];
      double* xi = x + (size_t)i * dx;
      for (int d = 0; d < dx; ++d) e[d] = noise_t[(size_t)d * N + i];
      mv(dx, dx, m->A, xi, mx);
      mv(dx, dx, LQ, e, v);
      for (int d = 0; d < dx; ++d) xi[d] = mx[d] + m->b[d] + v[d];
      mv(dy, dx, m->H, xi, hx);
      for (int k = 0; k < dy; ++k) dif[k] = y[k] - hx[k] - m->c[k];
      logw[i] += logpdf_chol(dy, LR, dif, tmpd);
    }
    double lse = or_logsumexp(logw, N);
    for (long i = 0; i < N; ++i) logw[i] -= lse;
    *ll_inc = lse - baseline;
  }
done:
  free(LQ); free(LR); free(xtmp); free(wbuf);
  (void)t;
  return st;
}

/* ------------------------------------------------------------------------ */
/* Rao-Blackwellised PF (rbpf.jl:16-84) on a conditionally linear-Gaussian   */
/* HierarchicalSSM (models/hierarchical.jl:4-50): outer LG dynamics, inner   */
/* LG dynamics with b_t = b + C*prev_outer (GFTest dummy model,              */
/* dummy_linear_gaussian.jl:25-46) and Q_t = Q0*exp(gamma*new_outer[qi])     */
/* (the stochastic-volatility shape of examples/trend-inflation).            */
typedef struct {
  int dxo, dz, dy;
  const double *mu_o, *Sigma_o, *A_o, *b_o, *Q_o;        /* outer */
  const double *mu_z, *Sigma_z, *A_z, *b_z, *C_z, *Q_z;  /* inner */
  double q_gamma; int q_index;
  const double *H, *c, *R;                               /* obs on inner */
  int tv; /* 1: A_o, b_o, Q_o, A_z, b_z, C_z, Q_z, H, c, R hold one block per step */
} or_rb_model;

/* The model of 1-based step t+1 (calc_params(., t+1)): block t of a
 * time-varying model, else the model itself. */
static or_rb_model rb_step_model(const or_rb_model* m, int t) {
  or_rb_model s = *m;
  if (!m->tv) return s;
  const int dxo = m->dxo, dz = m->dz, dy = m->dy;
  s.A_o = m->A_o + (size_t)t * dxo * dxo;
  s.b_o = m->b_o + (size_t)t * dxo;
  s.Q_o = m->Q_o + (size_t)t * dxo * dxo;
  s.A_z = m->A_z + (size_t)t * dz * dz;
  s.b_z = m->b_z + (size_t)t * dz;
  s.C_z = m->C_z + (size_t)t * dz * dxo;
  s.Q_z = m->Q_z + (size_t)t * dz * dz;
  s.H = m->H + (size_t)t * dy * dz;
  s.c = m->c + (size_t)t * dy;
  s.R = m->R + (size_t)t * dy * dy;
  s.tv = 0;
  return s;
}

/* One particle's RBPF move (rbpf.jl:24-84): outer propogate with noise e
 * (particles.jl:175-245), inner KF predict with (prev_outer, new_outer)
 * (rbpf.jl:45-55), inner KF update with y; p = [x | mu | Sigma | L] is updated
 * in place and *inc receives the log-weight increment (proposal ratio plus the
 * inner predictive log-likelihood).  Returns nonzero if a Cholesky failed. */
static int rb_particle_step(const or_rb_model* m, const or_proposal* prop, const double* LQo,
                            const double* Lqo, const double* LR, const double* y, const double* e,
                            double* p, double* Qt, kf_ws* ws, double* inc_out) {
  int dxo = m->dxo, dz = m->dz, dy = m->dy;
  double mx[64], v[64], xn[64], dif[64], tmpd[64], bt[64];
  double *xo = p, *mu = p + dxo, *Sig = p + dxo + dz, *L = p + dxo + dz + dz * dz;
  mv(dxo, dxo, m->A_o, xo, mx);
  for (int d = 0; d < dxo; ++d) mx[d] += m->b_o[d];
  double inc = 0.0;
  if (prop->kind == OR_PROP_BOOTSTRAP) {
    mv(dxo, dxo, LQo, e, v);
    for (int d = 0; d < dxo; ++d) xn[d] = mx[d] + v[d];
  } else {
    mv(dxo, dxo, Lqo, e, v);
    for (int d = 0; d < dxo; ++d) xn[d] = mx[d] + v[d];
    for (int d = 0; d < dxo; ++d) dif[d] = xn[d] - mx[d];
    double lp = logpdf_chol(dxo, LQo, dif, tmpd);
    double lq = logpdf_chol(dxo, Lqo, dif, tmpd);
    inc = lp - lq;
  }
  mv(dz, dxo, m->C_z, xo, bt);
  for (int d = 0; d < dz; ++d) bt[d] += m->b_z[d];
  double qs = exp(m->q_gamma * xn[m->q_index]);
  for (int k = 0; k < dz * dz; ++k) Qt[k] = m->Q_z[k] * qs;
  int s1 = kf_predict(dz, m->A_z, bt, Qt, mu, Sig, L, ws);
  double lin = 0.0;
  int s2 = s1 ? s1 : kf_update(dz, dy, m->H, m->c, m->R, LR, y, 0.0, 0, mu, Sig, L, &lin, ws);
  memcpy(xo, xn, 8 * dxo);
  *inc_out = inc + lin;
  return s2;
}

/* First-stage score of the auxiliary RBPF (rbpf.jl:86-124 through
 * compute_logeta, particles.jl:283-296): x* = A_o x + b_o, the mean / mode of
 * the outer transition, or (lookahead == 2, DrawPredictive) one draw
 * A_o x + b_o + chol(Q_o) e' with e' from the Philox stream tagged
 * TAG_LOOKAHEAD, counters (i, t, 0); the inner Gaussian predicted with
 * (prev_outer x, new_outer x*) and log eta = the update log-likelihood of y
 * (predictive_loglik).  p = [x | mu | Sigma | L] is left unchanged; q is
 * scratch of the same width. */
static int rb_logeta(const or_rb_model* m, int lookahead, const double* LQo, const double* LR,
                     const double* y, const double* p, uint64_t seed, long i, int t, double* q,
                     double* Qt, kf_ws* ws, double* eta) {
  int dxo = m->dxo, dz = m->dz, dy = m->dy;
  double xs[64], bt[64], e[64], v[64], buf[4];
  mv(dxo, dxo, m->A_o, p, xs);
  for (int d = 0; d < dxo; ++d) xs[d] += m->b_o[d];
  if (lookahead == 2) {
    philox_normals4_tag(seed, (uint32_t)i, (uint32_t)t, 0u, TAG_LOOKAHEAD, buf);
    for (int d = 0; d < dxo; ++d) e[d] = buf[d];
    mv(dxo, dxo, LQo, e, v);
    for (int d = 0; d < dxo; ++d) xs[d] += v[d];
  }
  mv(dz, dxo, m->C_z, p, bt);
  for (int d = 0; d < dz; ++d) bt[d] += m->b_z[d];
  double qs = exp(m->q_gamma * xs[m->q_index]);
  for (int k = 0; k < dz * dz; ++k) Qt[k] = m->Q_z[k] * qs;
  double *mu = q, *Sig = q + dz, *L = q + dz + dz * dz;
  memcpy(mu, p + dxo, sizeof(double) * dz);
  memcpy(Sig, p + dxo + dz, sizeof(double) * dz * dz);
  memcpy(L, p + dxo + dz + dz * dz, sizeof(double) * dz * dz);
  int st = kf_predict(dz, m->A_z, bt, Qt, mu, Sig, L, ws);
  return st ? st : kf_update(dz, dy, m->H, m->c, m->R, LR, y, 0.0, 0, mu, Sig, L, eta, ws);
}

int or_rbpf_run(const or_rb_model* m, const or_proposal* prop, const or_resample_cfg* rc, long N,
                int T, const double* ys, const double* noise, const double* uniforms,
                uint64_t seed, double* ll, or_pf_out* out, double* zmeans /* T*dz */) {
  int dxo = m->dxo, dz = m->dz, dy = m->dy;
  int width = dxo + dz + dz * dz + dz * dz; /* x, mu, Sigma, L */
  double* S = malloc(sizeof(double) * N * width);
  double* Stmp = malloc(sizeof(double) * N * width);
  double* logw = calloc(N, 8);
  double* wbuf = malloc(sizeof(double) * N);
  double* ubuf = malloc(sizeof(double) * N);
  double* eta = malloc(sizeof(double) * N);
  double* aux = malloc(sizeof(double) * N);
  double *Lo0 = calloc(dxo * dxo, 8), *LQo = calloc(dxo * dxo, 8), *Lqo = calloc(dxo * dxo, 8);
  double *LZ0 = calloc(dz * dz, 8), *LR = calloc(dy * dy, 8);
  int st = OR_OK, uniform = 1;
  long clamps = 0;
  double tot = 0.0;
  if ((st = or_chol_lower(dxo, m->Sigma_o, Lo0)) || (st = or_chol_lower(dxo, m->Q_o, LQo)) ||
      (st = or_chol_lower(dz, m->Sigma_z, LZ0)) || (st = or_chol_lower(dy, m->R, LR)))
    goto done;
  if (prop->kind == OR_PROP_OVERDISPERSED) {
    double* kQ = malloc(sizeof(double) * dxo * dxo);
    for (int i = 0; i < dxo * dxo; ++i) kQ[i] = prop->k * m->Q_o[i];
    st = or_chol_lower(dxo, kQ, Lqo);
    free(kQ);
    if (st) goto done;
  }
  /* initialise_particle (rbpf.jl:16-22) */
  for (long i = 0; i < N; ++i) {
    double e[64], v[64];
    double* p = S + (size_t)i * width;
    draw_normals(noise, seed, dxo, N, 0, i, e);
    mv(dxo, dxo, Lo0, e, v);
    for (int d = 0; d < dxo; ++d) p[d] = m->mu_o[d] + v[d];
    memcpy(p + dxo, m->mu_z, 8 * dz);
    memcpy(p + dxo + dz, m->Sigma_z, 8 * dz * dz);
    memcpy(p + dxo + dz + dz * dz, LZ0, 8 * dz * dz);
  }
  for (int t = 1; t <= T; ++t) {
    int32_t* anc_t = out && out->ancestors ? out->ancestors + (size_t)(t - 1) * N : NULL;
    double* mar_t = out && out->margins ? out->margins + (size_t)(t - 1) * N : NULL;
    double ess = 0.0, baseline;
    int res;
    const double* y = ys + (size_t)(t - 1) * dy;
    /* this step's model (time-varying: calc_params(., t)) and its factors */
    const or_rb_model ms = rb_step_model(m, t - 1);
    if (m->tv) {
      if ((st = or_chol_lower(dxo, ms.Q_o, LQo)) || (st = or_chol_lower(dy, ms.R, LR))) break;
      if (prop->kind == OR_PROP_OVERDISPERSED) {
        double kQ[64 * 64];
        for (int i = 0; i < dxo * dxo; ++i) kQ[i] = prop->k * ms.Q_o[i];
        if ((st = or_chol_lower(dxo, kQ, Lqo))) break;
      }
    }
    if (prop->lookahead) {
      /* AuxiliaryParticleFilter(RBPF(...), pp) step (particles.jl:311-345):
       * resample on softmax(logw + log eta) (resamplers.jl:109-116), new weights
       * -log eta[a] and the ll_baseline of construct_new_state (:118-143), as
       * in or_pf_run. */
      int bad = 0;
#pragma omp parallel num_threads(g_threads) reduction(| : bad)
      {
      kf_ws ws = kf_ws_alloc(dz, dy);
      double* Qt = malloc(sizeof(double) * dz * dz);
      double* q = malloc(sizeof(double) * width);
#pragma omp for schedule(static)
      for (long i = 0; i < N; ++i) {
        if (rb_logeta(&ms, prop->lookahead, LQo, LR, y, S + (size_t)i * width, seed, i, t, q, Qt, &ws,
                      &eta[i]))
          bad |= 1;
        aux[i] = (uniform ? 0.0 : logw[i]) + eta[i];
      }
      free(q); free(Qt);
      kf_ws_free(&ws);
      }
      if (bad) { st = OR_NOT_PD; break; }
      softmax(aux, N, wbuf);
      ess = ess_of(wbuf, N);
      int sched = rc->schedule ? rc->schedule[t - 1] : -1;
      res = sched >= 0 ? sched : (rc->threshold * (double)N >= ess);
      if (res) {
        draw_uniforms(uniforms, seed, rc->kind, N, t, ubuf);
        int32_t* a = anc_t ? anc_t : (int32_t*)malloc(sizeof(int32_t) * N);
        clamps += or_sample_ancestors(rc->kind, rc->conv, N, wbuf, ubuf, a, mar_t);
        memcpy(Stmp, S, sizeof(double) * N * width);
        for (long i = 0; i < N; ++i)
          memcpy(S + (size_t)i * width, Stmp + (size_t)(a[i] - 1) * width, sizeof(double) * width);
        const double lse1 = or_logsumexp(aux, N);
        const double lse2 = uniform ? log((double)N) : or_logsumexp(logw, N);
        for (long i = 0; i < N; ++i) logw[i] = -eta[a[i] - 1];
        const double lse3 = or_logsumexp(logw, N), lse4 = log((double)N);
        baseline = lse3 - ((lse1 - lse2) + (lse3 - lse4));
        uniform = 0;
        if (!anc_t) free(a);
      } else {
        if (anc_t)
          for (long i = 0; i < N; ++i) anc_t[i] = (int32_t)(i + 1);
        if (mar_t)
          for (long i = 0; i < N; ++i) mar_t[i] = 0.0;
        baseline = uniform ? log((double)N) : or_logsumexp(logw, N);
      }
    } else {
      int was_uniform = uniform;
      res = maybe_resample(rc, t, N, width, S, Stmp, logw, &uniform, wbuf, ubuf, uniforms,
                           seed, anc_t, mar_t, &ess, &clamps);
      baseline = (was_uniform && !res) ? log((double)N) : or_logsumexp(logw, N);
    }
    if (out && out->ess) out->ess[t - 1] = ess;
    if (out && out->resampled) out->resampled[t - 1] = (int8_t)res;
    int fail = 0;
#pragma omp parallel num_threads(g_threads) reduction(| : fail)
    {
    kf_ws ws = kf_ws_alloc(dz, dy);
    double* Qt = malloc(sizeof(double) * dz * dz);
#pragma omp for schedule(static)
    for (long i = 0; i < N; ++i) {
      double e[64];
      draw_normals(noise, seed, dxo, N, t, i, e);
      double inc = 0.0;
      if (rb_particle_step(&ms, prop, LQo, Lqo, LR, y, e, S + (size_t)i * width, Qt, &ws, &inc))
        fail |= 1;
      logw[i] = logw[i] + inc;
    }
    free(Qt);
    kf_ws_free(&ws);
    }
    if (fail) { st = OR_NOT_PD; break; }
    uniform = 0;
    double lse = or_logsumexp(logw, N);
    double inc = lse - baseline;
    for (long i = 0; i < N; ++i) logw[i] -= lse;
    tot += inc;
    if (out && out->ll_steps) out->ll_steps[t - 1] = inc;
    if (out && out->means) {
      double* mo = out->means + (size_t)(t - 1) * dxo;
      for (int d = 0; d < dxo; ++d) mo[d] = 0.0;
      for (long i = 0; i < N; ++i)
        for (int d = 0; d < dxo; ++d) mo[d] += exp(logw[i]) * S[(size_t)i * width + d];
    }
    if (zmeans) {
      double* mo = zmeans + (size_t)(t - 1) * dz;
      for (int d = 0; d < dz; ++d) mo[d] = 0.0;
      for (long i = 0; i < N; ++i)
        for (int d = 0; d < dz; ++d) mo[d] += exp(logw[i]) * S[(size_t)i * width + dxo + d];
    }
  }
  if (out && out->logw_final) memcpy(out->logw_final, logw, sizeof(double) * N);
  if (out && out->x_final)
    for (long i = 0; i < N; ++i)
      memcpy(out->x_final + (size_t)i * (dxo + dz + dz * dz), S + (size_t)i * width,
             sizeof(double) * (dxo + dz + dz * dz));
done:
  if (out && out->clamps) *out->clamps = clamps;
  *ll = tot;
  free(S); free(Stmp); free(logw); free(wbuf); free(ubuf); free(eta); free(aux);
  free(Lo0); free(LQo); free(Lqo); free(LZ0); free(LR);
  return st;
}

/* One bootstrap RBPF step from a given state (teacher forcing for the FP32
 * bank's parity checks): maybe_resample with this step's uniforms u, then
 * rb_particle_step for every particle with noise_t ([dxo][N]), the baseline and
 * LSE accounting of or_rbpf_run.  state: [N][dxo + dz + dz*dz] (x, mu, Sigma
 * column-major) in and out; logw [N] normalised, in and out; `uniform` marks
 * the initial TypelessZero weights. */
int or_rbpf_step(const or_rb_model* m, const or_resample_cfg* rc, long N, const double* y,
                 const double* noise_t, const double* u, int uniform, double* state,
                 double* logw, int32_t* anc, double* margins, double* ess, int8_t* resampled,
                 double* ll_inc) {
  int dxo = m->dxo, dz = m->dz, dy = m->dy;
  int w_in = dxo + dz + dz * dz, width = w_in + dz * dz;
  double* S = malloc(sizeof(double) * N * width);
  double* Stmp = malloc(sizeof(double) * N * width);
  double* wbuf = malloc(sizeof(double) * N);
  double* ubuf = malloc(sizeof(double) * N);
  double *LQo = calloc(dxo * dxo, 8), *LR = calloc(dy * dy, 8);
  or_proposal boot = {OR_PROP_BOOTSTRAP, 1.0};
  int st = OR_OK, fail = 0;
  long clamps = 0;
  if ((st = or_chol_lower(dxo, m->Q_o, LQo)) || (st = or_chol_lower(dy, m->R, LR))) goto done;
  for (long i = 0; i < N && !st; ++i) {
    double* p = S + (size_t)i * width;
    memcpy(p, state + (size_t)i * w_in, sizeof(double) * w_in);
    st = or_chol_lower(dz, p + dxo + dz, p + w_in);
  }
  if (st) goto done;
  {
    or_resample_cfg rc1 = *rc;
    int8_t sch = rc->schedule ? rc->schedule[0] : -1;
    rc1.schedule = &sch;
    int was_uniform = uniform;
    int res = maybe_resample(&rc1, 1, N, width, S, Stmp, logw, &uniform, wbuf, ubuf, u, 0, anc,
                             margins, ess, &clamps);
    *resampled = (int8_t)res;
    double baseline = (was_uniform && !res) ? log((double)N) : or_logsumexp(logw, N);
    kf_ws ws = kf_ws_alloc(dz, dy);
    double* Qt = malloc(sizeof(double) * dz * dz);
    for (long i = 0; i < N; ++i) {
      double e[64], inc = 0.0;
      for (int d = 0; d < dxo; ++d) e[d] = noise_t[(size_t)d * N + i];
      if (rb_particle_step(m, &boot, LQo, NULL, LR, y, e, S + (size_t)i * width, Qt, &ws, &inc))
        fail = 1;
      logw[i] += inc;
    }
    free(Qt);
    kf_ws_free(&ws);
    if (fail) { st = OR_NOT_PD; goto done; }
    double lse = or_logsumexp(logw, N);
    for (long i = 0; i < N; ++i) logw[i] -= lse;
    *ll_inc = lse - baseline;
    for (long i = 0; i < N; ++i) memcpy(state + (size_t)i * w_in, S + (size_t)i * width, sizeof(double) * w_in);
  }
done:
  free(S); free(Stmp); free(wbuf); free(ubuf); free(LQo); free(LR);
  return st;
}

/* ------------------------------------------------------------------------ */
/* Conditional SMC sweeps (csmc.jl:231-434) on a linear-Gaussian model with the
 * bootstrap proposal, FP64, one chain after another (chains in parallel with
 * or_set_threads).  Restates, per sweep:
 *   initialise (particles.jl:36-50): particle 1 <- ref[0] when conditioned;
 *   per step t: [ancestor sampling, csmc.jl:250-258: a* drawn from
 *   logw_i + log p(ref_t | x_i)]; resample by the ESS rule (resamplers.jl:
 *   179-183) or always under ancestor sampling (csmc.jl:261 calls resample);
 *   _set_ref_index! (resamplers.jl:51) or a*; x_1 <- ref_t, the others
 *   A x_a + b + LQ e; logw = (0 if resampled else logw) + log p(y_t | x);
 *   ll += LSE(logw) - (log N if resampled else LSE of the previous weights);
 *   next reference: get_ancestry of a particle drawn by its final weight
 *   (csmc.jl:103-108, containers.jl:421-440) or backward simulation
 *   (csmc.jl:378-434, weights logw_t + log p(x*_{t+1} | x_t), logw_0 = 0).
 * Draws from weights take the first k with cumsum(w)_k >= u * sum(w)
 * (StatsBase.sample); resampling uses the resamplers.jl:214-238 rules.
 * Sums run in index order; the CUDA kernel's block reductions agree to
 * rounding.  Randomness: injected (noise [chains][iters][T+1][N][dx], uniforms
 * [chains][iters][T+1][N+1], the CUDA library's layout) or, when NULL, the
 * CUDA library's Philox counters (sweep, chain, t<<12 | slot, tag). */
#define TAG_CS_NORMAL 0x43534E4Du
#define TAG_CS_UNIF 0x43535546u
typedef struct {
  const double *noise, *unif;
  uint64_t seed;
  int iters, T, N, dx;
} cs_rng;
static double cs_uniform(const cs_rng* r, int chain, int it, int t, int slot) {
  if (r->unif) return r->unif[(((size_t)chain * r->iters + it) * (r->T + 1) + t) * (r->N + 1) + slot];
  uint32_t ctr[4] = {(uint32_t)it, (uint32_t)chain, ((uint32_t)t << 12) | (uint32_t)slot, TAG_CS_UNIF}, w[4];
  philox4x32_10(ctr, (uint32_t)r->seed, (uint32_t)(r->seed >> 32), w);
  uint64_t bits = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
  return (double)bits * (1.0 / 9007199254740992.0);
}
static void cs_normals(const cs_rng* r, int chain, int it, int t, int i, double* e) {
  if (r->noise) {
    memcpy(e, r->noise + ((((size_t)chain * r->iters + it) * (r->T + 1) + t) * r->N + i) * r->dx,
           sizeof(double) * r->dx);
    return;
  }
  for (int q = 0; 4 * q < r->dx; ++q) {
    uint32_t ctr[4] = {(uint32_t)it, (uint32_t)chain, ((uint32_t)t << 12) | (uint32_t)(4 * i + q),
                       TAG_CS_NORMAL}, w[4];
    philox4x32_10(ctr, (uint32_t)r->seed, (uint32_t)(r->seed >> 32), w);
    for (int p = 0; p < 2; ++p) {
      double u1 = ((double)w[2 * p] + 1.0) * (1.0 / 4294967296.0);
      double u2 = (double)w[2 * p + 1] * (1.0 / 4294967296.0);
      double rr = sqrt(-2.0 * log(u1));
      double th = 6.283185307179586 * u2;
      if (4 * q + 2 * p < r->dx) e[4 * q + 2 * p] = rr * cos(th);
      if (4 * q + 2 * p + 1 < r->dx) e[4 * q + 2 * p + 1] = rr * sin(th);
    }
  }
}
/* exp(v - max(v)) in place followed by the running sum; returns nothing. */
static void cs_exp_cumsum(double* W, int N) {
  double m = -INFINITY;
  for (int i = 0; i < N; ++i) m = W[i] > m ? W[i] : m;
  double acc = 0.0;
  for (int i = 0; i < N; ++i) { acc += exp(W[i] - m); W[i] = acc; }
}
static int cs_draw(const double* W, int N, double u) {
  double target = u * W[N - 1];
  int k = 0;
  while (k < N && W[k] < target) ++k;
  return k < N ? k : N - 1;
}
static double cs_trans_logpdf(int dx, const double* A, const double* b, const double* LQ,
                              double trans_const, const double* xn, const double* x, double* r) {
  for (int i = 0; i < dx; ++i) {
    double s = xn[i] - b[i];
    for (int k = 0; k < dx; ++k) s -= A[i + k * dx] * x[k];
    r[i] = s;
  }
  trsv_lower(dx, LQ, r);
  double q = 0.0;
  for (int i = 0; i < dx; ++i) q += r[i] * r[i];
  return trans_const - 0.5 * q;
}

int or_csmc_run(const or_lg_model* m, int N, double threshold, int resampler, int refresh,
                int T, const double* ys, int chains, int iters, int burnin, int ref_given,
                const double* noise, const double* uniforms, uint64_t seed, double* ref,
                double* traj_out, double* ll_out) {
  const int dx = m->dx, dy = m->dy;
  /* factors of every step's model (time-varying: calc_params(., t) for t = 1..T) */
  const int nb = m->tv ? T : 1;
  double *LQs = calloc((size_t)nb * dx * dx, 8), *LRs = calloc((size_t)nb * dy * dy, 8);
  double *tcs = calloc(nb, 8), *ocs = calloc(nb, 8), *L0 = calloc((size_t)dx * dx, 8);
  int st = or_chol_lower(dx, m->Sigma0, L0);
  for (int k = 0; k < nb && !st; ++k) {
    const or_step_params SP = step_params(m, k);
    double *LQk = LQs + (size_t)k * dx * dx, *LRk = LRs + (size_t)k * dy * dy;
    if ((st = or_chol_lower(dx, SP.Q, LQk)) || (st = or_chol_lower(dy, SP.R, LRk))) break;
    double ldq = 0.0, ldr = 0.0;
    for (int i = 0; i < dx; ++i) ldq += log(LQk[i + i * dx]);
    for (int i = 0; i < dy; ++i) ldr += log(LRk[i + i * dy]);
    tcs[k] = -ldq - 0.5 * dx * LOG2PI;
    ocs[k] = -ldr - 0.5 * dy * LOG2PI;
  }
  if (st) {
    free(LQs); free(LRs); free(tcs); free(ocs); free(L0);
    return st;
  }
#define CS_BLK(t) (m->tv ? (t) - 1 : 0) /* block of 1-based step t */
  const cs_rng rng = {noise, uniforms, seed, iters, T, N, dx};
  int fail = 0;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic) reduction(| : fail)
  for (int c = 0; c < chains; ++c) {
    double* X = malloc(sizeof(double) * (size_t)(T + 1) * N * dx);
    double* LW = malloc(sizeof(double) * (size_t)(T + 1) * N);
    int* ANC = malloc(sizeof(int) * (size_t)T * N);
    double *W = malloc(sizeof(double) * N), *LWP = malloc(sizeof(double) * N);
    int* AN = malloc(sizeof(int) * N);
    double e[16], xa[16], x[16], r[16], z[16];
    double* REF = ref + (size_t)c * (T + 1) * dx;
    for (int it = 0; it < iters && !fail; ++it) {
      const int has_ref = it > 0 || ref_given;
      for (int i = 0; i < N; ++i) {
        double* xo = X + (size_t)i * dx;
        if (has_ref && i == 0) { memcpy(xo, REF, sizeof(double) * dx); }
        else {
          cs_normals(&rng, c, it, 0, i, e);
          for (int rr = 0; rr < dx; ++rr) {
            double s = m->mu0[rr];
            for (int k = 0; k <= rr; ++k) s += L0[rr + k * dx] * e[k];
            xo[rr] = s;
          }
        }
        LW[i] = 0.0;
      }
      double ll = 0.0;
      for (int t = 1; t <= T; ++t) {
        const double* Xp = X + (size_t)(t - 1) * N * dx;
        const double* LWp = LW + (size_t)(t - 1) * N;
        double mx = -INFINITY, s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < N; ++i) mx = LWp[i] > mx ? LWp[i] : mx;
        for (int i = 0; i < N; ++i) { double w = exp(LWp[i] - mx); s1 += w; s2 += w * w; }
        const double lse = mx + log(s1), ess = s1 * s1 / s2;
        const int resamp = refresh == 1 || threshold * (double)N >= ess;
        int as_idx = 0;
        /* this step's model */
        const int kb = CS_BLK(t);
        const or_step_params SP = step_params(m, kb);
        const double *LQ = LQs + (size_t)kb * dx * dx, *LR = LRs + (size_t)kb * dy * dy;
        if (refresh == 1 && has_ref) {
          for (int i = 0; i < N; ++i)
            W[i] = LWp[i] + cs_trans_logpdf(dx, SP.A, SP.b, LQ, tcs[kb], REF + (size_t)t * dx,
                                            Xp + (size_t)i * dx, r);
          cs_exp_cumsum(W, N);
          as_idx = cs_draw(W, N, cs_uniform(&rng, c, it, t, N));
        }
        if (resamp) {
          double acc = 0.0;
          for (int i = 0; i < N; ++i) { acc += exp(LWp[i] - lse); W[i] = acc; }
          const double nd = (double)N, wn = W[N - 1];
          for (int i = 0; i < N; ++i) {
            double uu;
            if (resampler == OR_SYSTEMATIC) uu = cs_uniform(&rng, c, it, t, 0) + (double)i;
            else if (resampler == OR_STRATIFIED) uu = (double)i + cs_uniform(&rng, c, it, t, i);
            else uu = cs_uniform(&rng, c, it, t, i) * wn;
            int k = 0;
            if (resampler == OR_MULTINOMIAL) while (k < N && !(W[k] >= uu)) ++k;
            else while (k < N && !(W[k] * nd > uu)) ++k;
            AN[i] = k < N ? k : N - 1;
            LWP[i] = 0.0;
          }
        } else {
          for (int i = 0; i < N; ++i) { AN[i] = i; LWP[i] = LWp[i]; }
        }
        const double base = resamp ? log((double)N) : lse;
        if (has_ref) AN[0] = as_idx;
        const double* y = ys + (size_t)(t - 1) * dy;
        double* Xt = X + (size_t)t * N * dx;
        double* LWt = LW + (size_t)t * N;
        for (int i = 0; i < N; ++i) {
          if (has_ref && i == 0) memcpy(x, REF + (size_t)t * dx, sizeof(double) * dx);
          else {
            memcpy(xa, Xp + (size_t)AN[i] * dx, sizeof(double) * dx);
            cs_normals(&rng, c, it, t, i, e);
            for (int rr = 0; rr < dx; ++rr) {
              double s = SP.b[rr];
              for (int k = 0; k < dx; ++k) s += SP.A[rr + k * dx] * xa[k];
              for (int k = 0; k <= rr; ++k) s += LQ[rr + k * dx] * e[k];
              x[rr] = s;
            }
          }
          for (int j = 0; j < dy; ++j) {
            double s = y[j] - SP.c[j];
            for (int k = 0; k < dx; ++k) s -= SP.H[j + k * dy] * x[k];
            z[j] = s;
          }
          trsv_lower(dy, LR, z);
          double q = 0.0;
          for (int j = 0; j < dy; ++j) q += z[j] * z[j];
          memcpy(Xt + (size_t)i * dx, x, sizeof(double) * dx);
          LWt[i] = LWP[i] + ocs[kb] - 0.5 * q;
          ANC[(size_t)(t - 1) * N + i] = AN[i];
        }
        double M = -INFINITY, s = 0.0;
        for (int i = 0; i < N; ++i) M = LWt[i] > M ? LWt[i] : M;
        for (int i = 0; i < N; ++i) s += exp(LWt[i] - M);
        const double lse_new = M + log(s);
        if (!(lse_new > -INFINITY) || isnan(lse_new)) { fail = 1; break; }
        ll += lse_new - base;
      }
      if (fail) break;
      for (int i = 0; i < N; ++i) W[i] = LW[(size_t)T * N + i];
      cs_exp_cumsum(W, N);
      int k = cs_draw(W, N, cs_uniform(&rng, c, it, 0, N));
      if (refresh != 2) {
        for (int t = T; t >= 0; --t) {
          memcpy(REF + (size_t)t * dx, X + ((size_t)t * N + k) * dx, sizeof(double) * dx);
          if (t > 0) k = ANC[(size_t)(t - 1) * N + k];
        }
      } else {
        memcpy(REF + (size_t)T * dx, X + ((size_t)T * N + k) * dx, sizeof(double) * dx);
        for (int t = T - 1; t >= 0; --t) {
          /* the transition from x_t to x_{t+1} is step t+1's */
          const int kb = CS_BLK(t + 1);
          const or_step_params SP = step_params(m, kb);
          for (int i = 0; i < N; ++i)
            W[i] = LW[(size_t)t * N + i] + cs_trans_logpdf(dx, SP.A, SP.b, LQs + (size_t)kb * dx * dx, tcs[kb],
                                                           REF + (size_t)(t + 1) * dx,
                                                           X + ((size_t)t * N + i) * dx, r);
          cs_exp_cumsum(W, N);
          k = cs_draw(W, N, cs_uniform(&rng, c, it, t + 1, N));
          memcpy(REF + (size_t)t * dx, X + ((size_t)t * N + k) * dx, sizeof(double) * dx);
        }
      }
      if (it >= burnin) {
        size_t kk = (size_t)c * (iters - burnin) + (it - burnin);
        if (traj_out) memcpy(traj_out + kk * (T + 1) * dx, REF, sizeof(double) * (T + 1) * dx);
        if (ll_out) ll_out[kk] = ll;
      }
    }
    free(X); free(LW); free(ANC); free(W); free(LWP); free(AN);
  }
#undef CS_BLK
  free(LQs); free(LRs); free(tcs); free(ocs); free(L0);
  return fail ? OR_ARG : OR_OK;
}
