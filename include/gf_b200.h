/*
 * gf_b200.h -- C ABI of the B200 filtering library (libgfb200.so).
 *
 * Drop-in boundary for GeneralisedFilters' filtering hot path.  Every entry
 * point is `extern "C"`, takes plain pointers and sizes, and names the Julia
 * function of TuringLang/SSMProblems.jl it replaces (paths are relative to the
 * reference project root).  A Julia caller binds these with `ccall`; the
 * Python host layer (gfb200) binds them with ctypes.
 *
 * Conventions
 *   - Matrices are FP64, column-major (Julia's layout): M[i + j*rows].
 *   - Particle state buffers are structure-of-arrays: X[d*N + i] (a Julia
 *     Matrix{T}(N, width)).
 *   - Ancestor indices crossing the ABI are 1-based, like the reference.
 *   - `memspace` says where every buffer argument of the call lives:
 *     GF_MEM_HOST (pageable or pinned host memory; the call copies) or
 *     GF_MEM_DEVICE (device memory of the context's GPU).
 *   - A gf_ctx is not thread-safe: use one per host thread.  Calls are
 *     ordered on the context's stream; calls taking GF_MEM_HOST buffers
 *     return after the results are in host memory.
 *   - Errors are returned as gf_status; gf_last_error() gives the message.
 */
#ifndef GF_B200_H
#define GF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gf_status;
enum {
  GF_OK = 0,
  GF_ERR_NOT_PD = 1,      /* a covariance lost positive definiteness (PosDefException) */
  GF_ERR_DIM = 2,         /* unsupported or inconsistent dimensions (DimensionMismatch) */
  GF_ERR_OOM_BUDGET = 3,  /* request exceeds the context's HBM budget */
  GF_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  GF_ERR_CUDA = 5,        /* CUDA runtime error */
  GF_ERR_ARG = 6,         /* invalid argument (ArgumentError) */
  GF_ERR_UNSUPPORTED = 7, /* feature not supported by this build */
  GF_ERR_BUSY = 8         /* serving queue full */
};

enum { GF_MEM_HOST = 0, GF_MEM_DEVICE = 1 };
enum { GF_RS_SYSTEMATIC = 0, GF_RS_STRATIFIED = 1, GF_RS_MULTINOMIAL = 2 };
/* GF_CONV_CPU: resamplers.jl:214-238 rule a_i = min{k : n*W_k > u_i}, extended
 * to stratified u_i = (i-1) + U_i and multinomial (first W_k >= U_i*W_n).
 * GF_CONV_CUDAEXT: the cumulative-offspring rule of ext/CUDAExt.jl:49-78. */
enum { GF_CONV_CPU = 0, GF_CONV_CUDAEXT = 1 };
enum { GF_PREC_F32 = 0, GF_PREC_F64 = 1 };
/* Proposals: BootstrapFilter (particles.jl:197-245); GFTest OptimalProposal
 * (GFTest/proposals.jl:11-31); GFTest OverdispersedProposal (:33-50). */
enum { GF_PROP_BOOTSTRAP = 0, GF_PROP_OPTIMAL = 1, GF_PROP_OVERDISPERSED = 2 };
enum { GF_ALGO_KF = 0, GF_ALGO_SRKF = 1 };
/* AuxiliaryParticleFilter(pf, RepresentativeStateLookAhead(pp)) (particles.jl:
 * 247-384): GF_LOOKAHEAD_MEAN scores each particle by log p(y_t | A x + b), the
 * mean and mode of its transition (MeanPredictive, ModePredictive);
 * GF_LOOKAHEAD_DRAW by log p(y_t | x*) with x* one draw from the transition
 * (DrawPredictive; bootstrap proposal; the draws come from their own Philox
 * stream even when the propagation noise is injected). */
enum { GF_LOOKAHEAD_NONE = 0, GF_LOOKAHEAD_MEAN = 1, GF_LOOKAHEAD_DRAW = 2 };

typedef struct gf_ctx gf_ctx;

/* Homogeneous linear-Gaussian SSM: create_homogeneous_linear_gaussian_model
 * (models/linear_gaussian.jl:125-131). */
typedef struct {
  int32_t dx, dy;
  const double* mu0;    /* dx */
  const double* Sigma0; /* dx*dx */
  const double* A;      /* dx*dx */
  const double* b;      /* dx */
  const double* Q;      /* dx*dx */
  const double* H;      /* dy*dx */
  const double* c;      /* dy */
  const double* R;      /* dy*dy */
} gf_lg_model;

/* Conditionally linear-Gaussian HierarchicalSSM (models/hierarchical.jl:4-50):
 * outer x_t = A_o x_{t-1} + b_o + N(0, Q_o); inner z_t = A_z z_{t-1} + b_z +
 * C_z x_{t-1} + N(0, Q_z * exp(q_gamma * x_t[q_index])); y_t = H z_t + c + N(0, R).
 * C_z (dz*dxo) follows GFTest's InnerDynamics (dummy_linear_gaussian.jl:25-46);
 * the exp(.) scale is the stochastic-volatility shape of the trend-inflation
 * example (examples/trend-inflation/script.jl:93-165). */
typedef struct {
  int32_t dxo, dz, dy;
  const double *mu_o, *Sigma_o, *A_o, *b_o, *Q_o;
  const double *mu_z, *Sigma_z, *A_z, *b_z, *C_z, *Q_z;
  double q_gamma;
  int32_t q_index;
  const double *H, *c, *R;
} gf_rb_model;

/* ParticleFilter(N, proposal; threshold, resampler) (particles.jl:92-108)
 * wrapped in ESSResampler (resamplers.jl:171-183). */
typedef struct {
  int64_t n_particles;
  int32_t resampler;      /* GF_RS_* */
  int32_t convention;     /* GF_CONV_* */
  double threshold;       /* resample iff threshold*N >= ESS (inclusive) */
  int32_t precision;      /* GF_PREC_F32 (FP32 state, FP64 normaliser) or GF_PREC_F64 */
  int32_t proposal;       /* GF_PROP_* */
  double proposal_k;      /* overdispersion factor for GF_PROP_OVERDISPERSED */
  uint64_t seed;          /* Philox key for in-kernel noise / uniforms */
  const int8_t* schedule; /* nullable, host [T]: -1 ESS rule, 0 keep, 1 resample
                             (GFTest AlternatingResampler-style forcing) */
  int32_t lookahead;      /* GF_LOOKAHEAD_*: AuxiliaryParticleFilter(pf, ...) first stage */
} gf_pf_config;

/* Outputs of one particle-filter run; every pointer but `ll` is nullable. */
typedef struct {
  double* ll;          /* [1]  log-evidence returned by filter() */
  double* ll_steps;    /* [T]  per-step increments (GeneralisedFilters.jl:76-81) */
  double* ess_steps;   /* [T]  ESS seen by the resampling decision of step t */
  int8_t* resampled;   /* [T]  1 if step t resampled */
  int32_t* ancestors;  /* [T][N] 1-based; identity on steps that did not resample */
  double* means;       /* [T][dx] weighted filtered means (outer means for RBPF) */
  void* states;        /* [width][N] final particle states (precision of the run) */
  double* log_weights; /* [N] final normalised log-weights */
  int32_t* clamps;     /* [1] slots clamped to N by the ancestor search */
  /* [T+1][dx][N] ancestral trajectory of every final particle, in the run's
   * precision: get_ancestry of AncestorCallback / ParticleTree (callbacks.jl:
   * 90-111, containers.jl:466-631), kept on the device as sparse path storage
   * with pruning (ext/CUDAExt.jl:146-298).  RBPF runs give the packed device
   * state [dxo + dz + dz*(dz+1)/2] per particle (x, mu, Sigma upper by rows). */
  void* paths;
  /* Dense particle history of DenseAncestorCallback / DenseParticleContainer
   * (callbacks.jl:47-81, containers.jl:296-419): [T+1][dx][N] the states after
   * initialisation and after every step, in the run's precision, and [T][N]
   * the normalised log-weights after every update (the PostUpdate weights).
   * With `ancestors` they are the container; gf_pf_dense_ancestry walks it.
   * RBPF runs use the packed device state, as for `paths`. */
  void* history;
  double* log_weight_history;
} gf_pf_out;

/* Outputs of a Kalman batch (per-step arrays are packed filter after filter). */
typedef struct {
  double* ll;        /* [B] total log-likelihood per filter */
  double* ll_steps;  /* [sum_f T_f] */
  float* means;      /* [sum_f T_f*dx_f] filtered means */
  float* covs;       /* [sum_f T_f*dx_f*dx_f] filtered covariances, column-major */
  int32_t* status;   /* [B] per-filter gf_status */
} gf_kf_out;

/* ------------------------------------------------------------------ context */
/* Creates a context on `device` with an HBM budget (0 = 90% of free memory). */
gf_status gf_ctx_create(int32_t device, size_t hbm_budget_bytes, gf_ctx** out);
gf_status gf_ctx_destroy(gf_ctx* ctx);
const char* gf_last_error(const gf_ctx* ctx);
/* Use `stream` (a cudaStream_t) for all work of this context (NULL = own stream). */
gf_status gf_ctx_set_stream(gf_ctx* ctx, void* stream);
void* gf_ctx_get_stream(gf_ctx* ctx);
gf_status gf_ctx_synchronize(gf_ctx* ctx);
/* Bytes of HBM the context currently holds / may hold. */
gf_status gf_ctx_memory(const gf_ctx* ctx, size_t* used, size_t* budget);
/* Per-kernel timing with CUDA events on the context stream (0 = off). */
gf_status gf_ctx_profile(gf_ctx* ctx, int32_t enable);
/* Kernel classes: 0 propagate/weight, 1 resample (cumulative weights and
 * offspring counts), 2 KF batch, 3 RBPF, 4 init/prep, 5 ancestor fill.
 * Resolves pending events (synchronises the stream). */
gf_status gf_ctx_profile_read(gf_ctx* ctx, int32_t kernel_class, double* total_ms,
                              int64_t* launches);
int32_t gf_version(void);

/* ---------------------------------------------------------- Kalman filters */
/* filter(model, KalmanFilter(; jitter), ys) / filter(model, SRKF(; jitter), ys)
 * for B independent models at once (kalman.jl:23-79, kalman_gradient.jl:12-29,
 * srkf.jl:41-176).  ys: concatenated [sum_f T_f*dy_f] FP64, step-major.
 * jitter is applied iff use_jitter != 0 (KalmanFilter(jitter=nothing) default). */
gf_status gf_kf_batch(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                      const int32_t* T, const double* ys, double jitter, int32_t use_jitter,
                      int32_t memspace, gf_kf_out* out);

/* Time-varying (non-homogeneous) models: calc_params(dyn, t) and
 * calc_params(obs, t) of models/linear_gaussian.jl:44-63 changing with t, as
 * GFTest's NonHomogeneousLinearGaussianLatentDynamics / ObservationProcess
 * (GFTest/models/linear_gaussian.jl:42-95).  param_steps[f] = 1 runs model f as
 * gf_kf_batch does; param_steps[f] >= T[f] means the A, b, Q, H, c, R pointers
 * of models[f] each hold param_steps[f] consecutive per-step blocks (block t-1
 * = step t, each column-major) and step t uses block t-1, with GF_ALGO_KF or
 * GF_ALGO_SRKF (whose step blocks carry the Cholesky factors of Q_t and R_t);
 * the smoother's prediction from t to t+1 uses step t+1's parameters
 * (kalman.jl:89-126). */
gf_status gf_kf_batch_tv(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                         const int32_t* T, const int32_t* param_steps, const double* ys,
                         double jitter, int32_t use_jitter, int32_t memspace, gf_kf_out* out);
gf_status gf_kf_smooth_tv(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                          const int32_t* param_steps, const double* ys, int32_t memspace,
                          gf_kf_out* out);

/* Gradients of kf_loglikelihood (integrations/logdensity.jl:136-161) for B
 * homogeneous models: the ChainRules pullback (integrations/kalman_rrule.jl:
 * 22-107, step rules kalman_gradient.jl:89-263) with Delta ll = 1, summed over
 * time for A, b, Q, H, c, R.  Matrices column-major, packed model after model.
 * Every pointer but ll is nullable. */
typedef struct {
  double* ll;       /* [B] */
  double* d_mu0;    /* [sum dx] */
  double* d_Sigma0; /* [sum dx*dx] */
  double* d_A;      /* [sum dx*dx] */
  double* d_b;      /* [sum dx] */
  double* d_Q;      /* [sum dx*dx] */
  double* d_H;      /* [sum dy*dx] */
  double* d_c;      /* [sum dy] */
  double* d_R;      /* [sum dy*dy] */
  int32_t* status;  /* [B] per-model gf_status */
} gf_kf_grad_out;
/* FP64, one CTA per model, dx, dy <= 16; jitter as in gf_kf_batch. */
gf_status gf_kf_loglikelihood_grad(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                                   const double* ys, double jitter, int32_t use_jitter, int32_t memspace,
                                   gf_kf_grad_out* out);

/* BackwardInformationPredictor(; initial_jitter, jitter) (kalman.jl:236-334) for
 * B homogeneous models: every backward predictive likelihood in information
 * form exp(lam'x - x'Om x / 2), packed model after model, row t = time t+1:
 * *_upd = p(y_{t:T} | x_t) (backward_initialise at T, then backward_update),
 * *_pred = p(y_{t+1:T} | x_t) (backward_predict; zero at T).  mu_smooth /
 * Sigma_smooth: two_filter_smooth (kalman.jl:336-370) of the forward filter
 * with *_pred at every t, i.e. p(x_t | y_1:T).  Every pointer is nullable;
 * FP64, one CTA per model, dx, dy <= 16. */
typedef struct {
  double* lam_pred;     /* [sum T*dx] */
  double* Om_pred;      /* [sum T*dx*dx] column-major */
  double* lam_upd;      /* [sum T*dx] */
  double* Om_upd;       /* [sum T*dx*dx] */
  double* mu_smooth;    /* [sum T*dx] */
  double* Sigma_smooth; /* [sum T*dx*dx] */
  int32_t* status;      /* [B] */
} gf_kf_backward_out;
gf_status gf_kf_backward_information(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                                     const double* ys, double initial_jitter, int32_t use_initial_jitter,
                                     double jitter, int32_t use_jitter, int32_t memspace,
                                     gf_kf_backward_out* out);
/* The same for time-varying models (test/algorithms/kalman.jl:139-190 runs the
 * backward predictor on a non-homogeneous model): param_steps[f] = 1 for a
 * homogeneous model, else >= T[f] stacked step blocks as for gf_kf_batch_tv;
 * backward_predict from x_{t+1} to x_t uses the dynamics of step t+1
 * (calc_params(dyn, iter + 1), kalman.jl:294-320) and backward_update /
 * backward_initialise the observation model of step t. */
gf_status gf_kf_backward_information_tv(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                                        const int32_t* param_steps, const double* ys, double initial_jitter,
                                        int32_t use_initial_jitter, double jitter, int32_t use_jitter,
                                        int32_t memspace, gf_kf_backward_out* out);

/* smooth(model, KalmanSmoother(), ys) for B models (kalman.jl:206-234): the
 * forward Kalman filter (no jitter), then the Rauch-Tung-Striebel pass of
 * backward_smooth (kalman.jl:89-126) from T-1 down to 1.  out->means and
 * out->covs (required) receive the SMOOTHED p(x_t | y_1:T) of every step,
 * packed like gf_kf_batch's outputs (the reference returns the one at t_smooth;
 * every t is given here).  out->ll / ll_steps are the forward log-likelihoods. */
gf_status gf_kf_smooth(gf_ctx* ctx, const gf_lg_model* models, int32_t B, const int32_t* T,
                       const double* ys, int32_t memspace, gf_kf_out* out);

/* Batched plan: uploads the models once, buckets filters by dimension,
 * autotunes the per-bucket group shape and captures one CUDA graph of
 * persistent launches.  Run with device-resident ys and outputs. */
typedef struct gf_kf_plan gf_kf_plan;
gf_status gf_kf_plan_create(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                            const int32_t* T, double jitter, int32_t use_jitter,
                            int32_t flags, gf_kf_plan** out);
/* The same over time-varying models (param_steps as in gf_kf_batch_tv). */
gf_status gf_kf_plan_create_tv(gf_ctx* ctx, int32_t algo, const gf_lg_model* models, int32_t B,
                               const int32_t* T, const int32_t* param_steps, double jitter,
                               int32_t use_jitter, int32_t flags, gf_kf_plan** out);
gf_status gf_kf_plan_run(gf_kf_plan* plan, const double* ys_dev, gf_kf_out* out_dev);
/* Forward run plus the RTS pass (as gf_kf_smooth) on a KalmanFilter() plan
 * without jitter; out_dev->means and covs receive the smoothed moments. */
gf_status gf_kf_plan_smooth(gf_kf_plan* plan, const double* ys_dev, gf_kf_out* out_dev);
gf_status gf_kf_plan_destroy(gf_kf_plan* plan);
/* plan flags: AUTOTUNE (KF: time each bucket's block shapes and keep the
 * fastest), NO_GRAPH (launch eagerly instead of replaying a CUDA graph), PLAIN
 * (KF: one launch per filter, the unbatched baseline form), SIMT (PF: keep the
 * CUDA-core propagation even where the tensor-core path applies), NO_FUSE (PF:
 * run filters of N <= 1024 as separate kernels per step instead of one block
 * for the whole filter), STAGED_GATHER (PF, Dx <= 16 on the tensor-core path:
 * copy each 128-particle sub-tile's sorted ancestor range into shared memory
 * with bulk async copies, one sub-tile ahead, instead of per-thread loads),
 * UNITS (PF, tensor-core path: a grid of resident blocks striding over
 * 128-particle units instead of one block per 1024-particle tile; the default
 * for Dx > 32, where it is the faster form), TILES (PF: one block per tile
 * even where UNITS is the default). */
enum { GF_PLAN_AUTOTUNE = 1, GF_PLAN_NO_GRAPH = 2, GF_PLAN_PLAIN = 4, GF_PLAN_SIMT = 8, GF_PLAN_NO_FUSE = 16,
       GF_PLAN_STAGED_GATHER = 32, GF_PLAN_UNITS = 64, GF_PLAN_TILES = 128 };

/* -------------------------------------------------------- particle filters */
/* filter(rng, model, ParticleFilter(N, proposal; threshold, resampler), ys)
 * (GeneralisedFilters.jl:58-84; particles.jl:36-90,147-245; resamplers.jl:
 * 33-238; containers.jl:140-173).  ys: [T][dy] FP64.
 * noise: nullable [(T+1)][dx][N] standard normals in the run's precision
 *   (step 0 = prior draw); NULL draws them in-kernel from Philox(seed).
 * uniforms: nullable FP64, systematic [T], stratified/multinomial [T][N];
 *   NULL draws them from Philox(seed). */
gf_status gf_pf_run(gf_ctx* ctx, const gf_lg_model* model, const gf_pf_config* cfg, int32_t T,
                    const double* ys, const void* noise, const double* uniforms,
                    int32_t memspace, gf_pf_out* out);
/* The same for a time-varying model (calc_params(dyn, t), calc_params(obs, t),
 * models/linear_gaussian.jl:44-63): param_steps = 1 is gf_pf_run; param_steps
 * >= T means the A, b, Q, H, c, R pointers of `model` each hold param_steps
 * per-step blocks (block t-1 = step t, column-major).  Every proposal; a
 * guided proposal's factors (OptimalProposal's gain and covariance,
 * OverdispersedProposal's k Q_t) are those of step t, as is the auxiliary
 * lookahead. */
gf_status gf_pf_run_tv(gf_ctx* ctx, const gf_lg_model* model, int32_t param_steps,
                       const gf_pf_config* cfg, int32_t T, const double* ys, const void* noise,
                       const double* uniforms, int32_t memspace, gf_pf_out* out);

/* Reusable PF plan: device buffers sized once, the T-step loop captured in a
 * CUDA graph; gf_pf_plan_run takes device-resident inputs and outputs. */
typedef struct gf_pf_plan gf_pf_plan;
gf_status gf_pf_plan_create(gf_ctx* ctx, const gf_lg_model* model, const gf_pf_config* cfg,
                            int32_t T, int32_t flags, gf_pf_plan** out);
gf_status gf_pf_plan_create_tv(gf_ctx* ctx, const gf_lg_model* model, int32_t param_steps,
                               const gf_pf_config* cfg, int32_t T, int32_t flags, gf_pf_plan** out);
gf_status gf_pf_plan_run(gf_pf_plan* plan, const double* ys_dev, const void* noise_dev,
                         const double* uniforms_dev, gf_pf_out* out_dev);
gf_status gf_pf_plan_destroy(gf_pf_plan* plan);

/* get_ancestry(container, i) for a DenseParticleContainer (containers.jl:
 * 421-440): for each requested final particle, the trajectory read from the
 * dense history by walking the 1-based ancestors back from time T.
 * history [T+1][dx][N] and paths [T+1][dx][M] in `precision`
 * (GF_PREC_F32 / GF_PREC_F64); ancestors [T][N] int32, 1-based; indices
 * (nullable = all N particles, M = N) [M] 1-based final-particle indices. */
gf_status gf_pf_dense_ancestry(gf_ctx* ctx, int32_t T, int64_t N, int32_t dx, int32_t precision,
                               const void* history, const int32_t* ancestors, int64_t M,
                               const int32_t* indices, int32_t memspace, void* paths);

/* filter(rng, hier_model, RBPF(PF(N, ...), KalmanFilter()), ys) (rbpf.jl:8-84).
 * Supports GF_PROP_BOOTSTRAP and GF_PROP_OVERDISPERSED outer proposals.
 * cfg->lookahead != GF_LOOKAHEAD_NONE runs AuxiliaryParticleFilter(RBPF(...),
 * pp) (rbpf.jl:86-124): log eta_i is the inner update log-likelihood of y_t
 * after predicting particle i's inner Gaussian to x*, the mean of its outer
 * transition (GF_LOOKAHEAD_MEAN) or one draw from it (GF_LOOKAHEAD_DRAW, from
 * the lookahead Philox stream with counters (i, t, 0)).
 * noise: nullable [(T+1)][dxo][N] FP32.  states out: GF_MEM_HOST gives
 * [dxo + dz + dz*dz][N] (x, mu, Sigma column-major); GF_MEM_DEVICE gives the
 * device layout [dxo + dz + dz*(dz+1)/2][N] (Sigma packed upper, row by row).
 * means / zmeans ([T][dz] weighted inner means) need GF_MEM_HOST. */
gf_status gf_rbpf_run(gf_ctx* ctx, const gf_rb_model* model, const gf_pf_config* cfg, int32_t T,
                      const double* ys, const void* noise, const double* uniforms,
                      int32_t memspace, gf_pf_out* out, double* zmeans);
/* The same for a time-varying hierarchical model: param_steps = 1 is
 * gf_rbpf_run; param_steps >= T means A_o, b_o, Q_o, A_z, b_z, C_z, Q_z, H, c
 * and R each hold param_steps per-step blocks (block t-1 = calc_params(., t),
 * column-major); the priors and q_gamma, q_index are shared by all steps. */
gf_status gf_rbpf_run_tv(gf_ctx* ctx, const gf_rb_model* model, int32_t param_steps,
                         const gf_pf_config* cfg, int32_t T, const double* ys, const void* noise,
                         const double* uniforms, int32_t memspace, gf_pf_out* out, double* zmeans);

/* ---------------------------------------------------- resampling primitives */
/* sample_ancestors(rng, resampler, weights) (resamplers.jl:206-238;
 * ext/CUDAExt.jl:31-78) on device buffers: weights [n] FP64 (need not be
 * normalised), uniforms [1] (systematic) or [n], ancestors out [n] int64,
 * 1-based. */
gf_status gf_sample_ancestors(gf_ctx* ctx, int32_t resampler, int32_t convention, int64_t n,
                              const double* weights_dev, const double* uniforms_dev,
                              int64_t* ancestors_dev);
/* offspring_to_ancestors (ext/CUDAExt.jl:90-117): cumulative offspring ->
 * 1-based ancestors, device int64 buffers of length n. */
gf_status gf_offspring_to_ancestors(gf_ctx* ctx, int64_t n, const int64_t* offspring_dev,
                                    int64_t* ancestors_dev);
/* ancestors_to_offspring (ext/CUDAExt.jl:119-142): 1-based ancestors ->
 * offspring counts. */
gf_status gf_ancestors_to_offspring(gf_ctx* ctx, int64_t n, const int64_t* ancestors_dev,
                                    int64_t* offspring_dev);
/* gf_sample_ancestors without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc where they
 * resample (a memory-pool-managed host framework that forbids foreign
 * allocations, a real-time loop that must not take the allocator's locks or
 * synchronise the device, code sized up front that must not fail with
 * out-of-memory mid-run).  Same arguments and results as gf_sample_ancestors,
 * on the caller's `stream` (a cudaStream_t, NULL = default stream) of the
 * current device; returns once the ancestors are written.
 * Limit: n <= gf_sample_ancestors_noalloc_max_n() (2^18); larger n returns
 * GF_ERR_DIM.  All scratch lives in one fixed device array (about 2.1 MB) that
 * every device loading the library holds until the process exits.  The first
 * call on a device resolves that array's address (cudaGetSymbolAddress), so
 * make the first call before any stream capture.  The address is cached for
 * the life of the process: no call may follow a cudaDeviceReset of that
 * device.  Every call reads its status back and waits for `stream`
 * (cudaStreamSynchronize) before it returns.  Calls share the array: calls
 * that overlap on the GPU (other streams, other host threads on the same
 * device) race and must be serialised by the caller. */
gf_status gf_sample_ancestors_noalloc(int32_t resampler, int32_t convention, int64_t n,
                                      const double* weights_dev, const double* uniforms_dev,
                                      int64_t* ancestors_dev, void* stream);
int64_t gf_sample_ancestors_noalloc_max_n(void);
/* The noise the PF kernels draw in-kernel for step t: out [dx][n] in the given
 * precision (no reference counterpart: exported so tests can inject it). */
gf_status gf_rng_normals(gf_ctx* ctx, uint64_t seed, int32_t t, int32_t dx, int64_t n,
                         int32_t precision, void* out_dev);

/* ------------------------------------------------- conditional SMC (PMCMC) */
/* Trajectory refreshment of ConditionalSMC (csmc.jl:10-40). */
enum { GF_CSMC_NONE = 0, GF_CSMC_ANCESTOR = 1, GF_CSMC_BACKWARD = 2 };

typedef struct {
  int32_t N;          /* particles per sweep, 1..gf_csmc_max_particles() */
  double threshold;   /* BF(N; threshold): resample iff threshold*N >= ESS.  Ancestor
                         sampling resamples at every step, as csmc.jl:261 does */
  int32_t resampler;  /* GF_RS_*, GF_CONV_CPU rule (resamplers.jl:214-238) */
  int32_t refresh;    /* GF_CSMC_* */
  uint64_t seed;      /* Philox key for in-kernel noise and uniforms */
} gf_csmc_config;

typedef struct {
  /* [chains][iters-burnin][T+1][dx] the trajectory each kept sweep returned */
  double* trajectories;
  double* ll;       /* [chains][iters-burnin] log-likelihood estimate of each kept sweep */
  /* [chains][T+1][dx], in and out: the reference trajectory the first sweep is
   * conditioned on (when ref_given) and, on return, the last sampled one.
   * Required. */
  double* ref;
  int32_t* status;  /* [chains] per-chain gf_status (nullable) */
} gf_csmc_out;

/* `iters` sweeps of ConditionalSMC(BF(N; threshold, resampler), refresh) per
 * chain (_csmc_sample, csmc.jl:231-434, driven by AbstractMCMC.step :438-450)
 * on a linear-Gaussian model, for `chains` independent chains at once.  Each
 * sweep conditions on the previous sweep's trajectory (the first on `ref` when
 * ref_given, else none) and samples a new one: by the final weights from the
 * ancestry (NONE, ANCESTOR: get_ancestry of the path store) or by backward
 * simulation over the dense history (BACKWARD).  Single draws from weights
 * take the first k with cumsum(w)_k >= u*sum(w) (StatsBase.sample).
 * ys: [T][dy] FP64.  noise (nullable): [chains][iters][T+1][N][dx] N(0,1),
 * row 0 the prior draw; uniforms (nullable): [chains][iters][T+1][N+1]: in row
 * t >= 1, slots 0..N-1 are the resampling uniforms of step t and slot N the
 * ancestor-sampling draw of step t (ANCESTOR) or the backward draw of time
 * t-1 (BACKWARD); row 0 slot N is the final draw.  Bootstrap proposal, FP64.
 * Limits: dx, dy <= 16, T < 2^20. */
gf_status gf_csmc_run(gf_ctx* ctx, const gf_lg_model* model, const gf_csmc_config* cfg, int32_t T,
                      const double* ys, int32_t chains, int32_t iters, int32_t burnin,
                      int32_t ref_given, const double* noise, const double* uniforms,
                      int32_t memspace, gf_csmc_out* out);
/* The same for a time-varying model: param_steps = 1 is gf_csmc_run;
 * param_steps >= T means A, b, Q, H, c, R each hold param_steps per-step blocks
 * (block t-1 = calc_params(., t), column-major).  Ancestor sampling at step t
 * and the backward-simulation weight from x_{t-1} to x_t use step t's
 * transition. */
gf_status gf_csmc_run_tv(gf_ctx* ctx, const gf_lg_model* model, int32_t param_steps,
                         const gf_csmc_config* cfg, int32_t T, const double* ys, int32_t chains,
                         int32_t iters, int32_t burnin, int32_t ref_given, const double* noise,
                         const double* uniforms, int32_t memspace, gf_csmc_out* out);
int32_t gf_csmc_max_particles(void);

/* ------------------------------------------------------------------ serving */
/* No reference counterpart: the reference runs one synchronous filter() call
 * at a time (GeneralisedFilters.jl:58-84).  A server owns one GPU through a
 * worker thread and runs many independent requests at once: Kalman requests
 * as persistent batched launches, particle-filter requests continuously
 * batched into shared per-step launches.  Admission is first-come-first-served
 * against a fixed HBM arena (hbm_budget_bytes) and a pinned host arena.
 * Submitting, polling and statistics are thread-safe.  A served request
 * returns exactly what gf_kf_batch / gf_pf_run / gf_rbpf_run return for the
 * same inputs (with in-kernel Philox draws). */
typedef struct gf_srv gf_srv;
enum { GF_REQ_KF = 0, GF_REQ_SRKF = 1, GF_REQ_PF = 2, GF_REQ_RBPF = 3 };
typedef struct {
  int32_t device;
  size_t hbm_budget_bytes;  /* device arena (0 = half of the free memory) */
  size_t host_budget_bytes; /* pinned host arena for staging and results (0 = 1 GiB) */
  int32_t max_pending;      /* submitted, not yet admitted requests before GF_ERR_BUSY (0 = 65536) */
  int32_t pf_chunk;         /* steps per particle-filter batch iteration (0 = 16) */
  int32_t kf_streams;       /* streams for concurrent Kalman batches (0 = 64) */
  int32_t max_active_pf;    /* particle-filter jobs running at once (0 = 4096) */
} gf_srv_config;
typedef struct {
  int32_t kind;             /* GF_REQ_* */
  int32_t T;
  const gf_lg_model* lg;    /* KF, SRKF, PF */
  const gf_rb_model* rb;    /* RBPF */
  const gf_pf_config* pf;   /* PF, RBPF (noise and uniforms are drawn in-kernel) */
  const double* ys;         /* host [T][dy]; copied by gf_srv_submit */
  double jitter;            /* KF, SRKF */
  int32_t use_jitter;
  int32_t param_steps;      /* PF: >= T for a time-varying model laid out as for
                               gf_pf_run_tv; 0 or 1 = homogeneous (KF, SRKF, RBPF:
                               homogeneous only) */
  /* Optional host destinations, written before the result is reported; they
   * must stay valid until then. */
  double* ll_steps;         /* [T] per-step log-likelihood increments */
  double* mean;             /* KF/SRKF/PF: final filtered (weighted) mean [dx];
                               RBPF: [dxo + dz] weighted outer then inner means */
  double* cov;              /* KF/SRKF: final filtered covariance [dx*dx], column-major */
  uint64_t tag;             /* returned in the result */
} gf_srv_request;
typedef struct {
  uint64_t id, tag;
  gf_status status;
  int32_t kind;
  double ll;                /* log-evidence (filter()'s second return value) */
  double submit_ms, start_ms, done_ms; /* since gf_srv_create; start = admission (-1 if never) */
} gf_srv_result;
typedef struct {
  int64_t submitted, completed, failed, rejected, pending, running;
  double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> result latency of completed requests */
  double kf_steps, particle_steps;        /* work of completed requests */
  double elapsed_ms;                      /* first submit -> last result */
  size_t hbm_budget, hbm_used, hbm_peak;
  int64_t pf_iterations, kf_batches, launches;
} gf_srv_metrics;
gf_status gf_srv_create(const gf_srv_config* cfg, gf_srv** out);
/* Validates and copies the request (inputs need not outlive the call); returns
 * GF_ERR_BUSY when max_pending requests wait for admission. */
gf_status gf_srv_submit(gf_srv* srv, const gf_srv_request* req, uint64_t* id);
/* Moves up to `max` finished results to `out`, waiting up to wait_ms for the
 * first; returns how many were written. */
int32_t gf_srv_poll(gf_srv* srv, gf_srv_result* out, int32_t max, int32_t wait_ms);
/* Waits until every submitted request has a result (timeout_ms < 0: forever). */
gf_status gf_srv_drain(gf_srv* srv, int32_t timeout_ms);
gf_status gf_srv_stats(gf_srv* srv, gf_srv_metrics* out);
/* Forgets finished requests' latencies and work (for a fresh measurement window). */
gf_status gf_srv_reset_stats(gf_srv* srv);
const char* gf_srv_last_error(gf_srv* srv);
/* Cancels requests not yet admitted, waits for the running ones, frees the arenas. */
gf_status gf_srv_destroy(gf_srv* srv);

#ifdef __cplusplus
}
#endif
#endif /* GF_B200_H */
