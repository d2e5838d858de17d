// gf_pf_plan.cu -- PF plans (device buffers + captured T-step graph) and the
// particle-filter entry points of the C ABI.
#include <cmath>
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "gf_internal.hpp"
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"

using namespace gf;

struct gf_pf_plan {
  gf_ctx* ctx = nullptr;
  bool dbl = false;
  int dx = 0, dy = 0, T = 0;
  int64_t N = 0;
  gf_pf_config cfg{};
  std::vector<int8_t> sched;
  PfLgKernels k;
  int ntiles = 0, nstiles = 0;
  size_t rsize = 4;
  std::vector<DevBuf> bufs;
  void *params = nullptr, *ystep = nullptr, *X0 = nullptr, *X1 = nullptr, *lw = nullptr;
  double *pp = nullptr, *key = nullptr, *part = nullptr, *mpart = nullptr, *ess1 = nullptr;
  double* tprefix = nullptr;
  int32_t *ocum = nullptr, *mpk = nullptr, *anc = nullptr;
  void* eta = nullptr;  // auxiliary filter: lookahead log eta [N]
  double* obs_consts = nullptr;  // time-varying model: observation and proposal constants per step
  unsigned long long* flags = nullptr;
  PfScalars* sc = nullptr;
  int8_t *sched_dev = nullptr, *res1 = nullptr;
  PfJob* job_dev = nullptr;
  PfJob job{};
  void (*prop_fn)(const PfJob*, int) = nullptr;  // chosen propagate kernel
  int prop_threads = 0;
  int prop_split = 1;
  int prop_grid = 0;
  bool units = false;  // unit-grid propagation: the step's finalise is a separate launch
  size_t prop_smem = 0;
  cudaGraphExec_t graph = nullptr;
  bool graph_means = false;
  bool small = false;  // N <= 1024 filters run in one block (pf_lg_small_filter)
  bool graph_record = false;
  bool use_graph = true;
  // path storage (allocated on the first run that asks for paths)
  TreeHost tree;
};

static gf_status plan_alloc(gf_pf_plan* p, size_t bytes, void** out) {
  gf_status st = dev_alloc(p->ctx, bytes, out);
  if (st == GF_OK && *out) p->bufs.push_back({*out, bytes});
  return st;
}

static void plan_release(gf_pf_plan* p) {
  if (!p) return;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (auto& b : p->bufs) dev_free(p->ctx, b.p, b.bytes);
  p->bufs.clear();
  tree_host_release(p->tree);
}

static gf_status validate_cfg(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg, int T) {
  if (!m || !cfg) return set_err(ctx, GF_ERR_ARG, "null model or config");
  if (m->dx < 1 || m->dy < 1) return set_err(ctx, GF_ERR_DIM, "dx, dy must be >= 1");
  if (cfg->n_particles < 1 || cfg->n_particles > (int64_t(1) << 31) - 1)
    return set_err(ctx, GF_ERR_ARG, "n_particles must be in [1, 2^31)");
  if (T < 1) return set_err(ctx, GF_ERR_ARG, "T must be >= 1");
  if (cfg->resampler < 0 || cfg->resampler > 2) return set_err(ctx, GF_ERR_ARG, "unknown resampler");
  if (cfg->convention < 0 || cfg->convention > 1) return set_err(ctx, GF_ERR_ARG, "unknown convention");
  if (cfg->precision != GF_PREC_F32 && cfg->precision != GF_PREC_F64)
    return set_err(ctx, GF_ERR_ARG, "unknown precision");
  if (cfg->lookahead < GF_LOOKAHEAD_NONE || cfg->lookahead > GF_LOOKAHEAD_DRAW)
    return set_err(ctx, GF_ERR_ARG, "unknown lookahead");
  if (cfg->lookahead == GF_LOOKAHEAD_DRAW && cfg->proposal != GF_PROP_BOOTSTRAP)
    return set_err(ctx, GF_ERR_UNSUPPORTED, "DrawPredictive lookahead is built for the bootstrap proposal");
  return GF_OK;
}

namespace gf {

gf_status lg_job_setup(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg, int32_t T,
                       int32_t flags, LgJobSetup* o, int32_t param_steps) {
  gf_status st = validate_cfg(ctx, m, cfg, T);
  if (st) return st;
  o->dbl = cfg->precision == GF_PREC_F64;
  const bool guided = cfg->proposal != GF_PROP_BOOTSTRAP;
  const bool tv = param_steps != 1;
  if (tv && param_steps < T)
    return set_err(ctx, GF_ERR_ARG, "%d parameter steps for T = %d", param_steps, T);
  if (!pick_lg_kernels(o->dbl, guided, m->dx, m->dy, &o->k))
    return set_err(ctx, GF_ERR_DIM, "no kernel for dx=%d dy=%d in %s", m->dx, m->dy,
                   o->dbl ? "FP64 (max 16)" : "FP32 (max 64)");
  // one parameter block (and observation-prep block) per step of a
  // time-varying model (calc_params(dyn, t), calc_params(obs, t)), else one
  const int nblk = tv ? T : 1;
  const int dx = m->dx, dy = m->dy;
  o->params.clear();
  o->pp.clear();
  o->obs_consts.clear();
  bool diag = true;
  LgFactors f;
  for (int sblk = 0; sblk < nblk; ++sblk) {
    gf_lg_model ms = *m;
    if (tv) {
      ms.A = m->A + (size_t)sblk * dx * dx;
      ms.b = m->b + (size_t)sblk * dx;
      ms.Q = m->Q + (size_t)sblk * dx * dx;
      ms.H = m->H + (size_t)sblk * dy * dx;
      ms.c = m->c + (size_t)sblk * dy;
      ms.R = m->R + (size_t)sblk * dy * dy;
    }
    if ((st = build_lg_factors(ctx, &ms, cfg, &f))) return st;
    pack_params(f, o->dbl, o->k.dxp, o->k.dyp, o->params);
    o->pp.insert(o->pp.end(), f.LRi.begin(), f.LRi.end());
    o->pp.insert(o->pp.end(), f.c.begin(), f.c.end());
    o->pp.insert(o->pp.end(), f.K.begin(), f.K.end());
    o->pp.insert(o->pp.end(), f.vb.begin(), f.vb.end());
    if (tv) {  // step constants: observation, proposal
      o->obs_consts.push_back(f.obs_const);
      o->obs_consts.push_back(f.prop_const);
    }
    for (int j = 0; j < dx; ++j)
      for (int i = 0; i < dx; ++i)
        if (i != j && f.L[i + j * dx] != 0.0) diag = false;
  }
  o->pstride = tv ? (int64_t)(o->params.size() / nblk) / (o->dbl ? 8 : 4) : 0;
  o->ppstride = tv ? (int32_t)(o->pp.size() / nblk) : 0;
  o->units_blocks = 0;
  if (o->k.prop_tc && !(flags & GF_PLAN_SIMT)) {
    const bool staged = (flags & GF_PLAN_STAGED_GATHER) && o->k.prop_tc_staged;
    const bool units = (flags & GF_PLAN_UNITS) && o->k.prop_tc_units && !staged;
    o->prop = staged ? o->k.prop_tc_staged : (units ? o->k.prop_tc_units : o->k.prop_tc);
    o->threads = 128;
    o->smem = staged ? o->k.tc_staged_smem : o->k.tc_smem;
    o->split = o->k.tc_split;
    if (units) o->units_blocks = o->k.tc_units_blocks;
  } else {
    o->prop = o->k.prop;
    o->threads = PF_THREADS;
    o->smem = o->k.smem;
    o->split = 1;
  }
  const int64_t N = cfg->n_particles;
  // step-1 decision with the reference's uniform-weight ESS
  o->ess1 = uniform_ess(N);
  const int sch0 = cfg->schedule ? cfg->schedule[0] : -1;
  o->res1 = (int8_t)(sch0 >= 0 ? (sch0 != 0) : (cfg->threshold * (double)N >= o->ess1));
  PfJob& J = o->J;
  std::memset(&J, 0, sizeof J);
  J.N = N;
  J.dx = m->dx;
  J.dy = m->dy;
  J.T = T;
  J.width = m->dx;
  J.ntiles = (int)((N + PF_TILE - 1) / PF_TILE);
  J.nstiles = (int)((N + SCAN_TILE - 1) / SCAN_TILE);
  J.resampler = cfg->resampler;
  J.conv = cfg->convention;
  J.prop = cfg->proposal;
  J.diag_l = diag ? 1 : 0;
  J.threshold = cfg->threshold;
  J.log_n = std::log((double)N);
  J.obs_const = f.obs_const;
  J.prop_const = f.prop_const;
  J.seed = cfg->seed;
  J.ystride = o->k.dyp + o->k.dxp;
  J.pstride = o->pstride;
  J.ppstride = o->ppstride;
  J.lookahead_draw = cfg->lookahead == GF_LOOKAHEAD_DRAW ? 1 : 0;
  return GF_OK;
}

}  // namespace gf

static gf_status pf_plan_create_impl(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                                     const gf_pf_config* cfg, int32_t T, int32_t flags, gf_pf_plan** out) {
  if (!ctx || !out) return GF_ERR_ARG;
  *out = nullptr;
  // the unit grid is the default for the widest states (Dx > 32, FP32 bootstrap):
  // there one tile block per SM leaves the last wave partly empty and the unit
  // grid's separate finalise costs less than that wave
  if (m && cfg && !(flags & (GF_PLAN_TILES | GF_PLAN_STAGED_GATHER | GF_PLAN_SIMT)) && m->dx > 32 &&
      cfg->precision == GF_PREC_F32 && cfg->proposal == GF_PROP_BOOTSTRAP)
    flags |= GF_PLAN_UNITS;
  LgJobSetup L;
  gf_status st = lg_job_setup(ctx, m, cfg, T, flags, &L, param_steps);
  if (st) return st;
  cudaSetDevice(ctx->device);
  auto p = std::make_unique<gf_pf_plan>();
  p->ctx = ctx;
  p->dbl = L.dbl;
  p->dx = m->dx;
  p->dy = m->dy;
  p->T = T;
  p->N = cfg->n_particles;
  p->cfg = *cfg;
  p->use_graph = !(flags & GF_PLAN_NO_GRAPH);
  if (cfg->schedule) p->sched.assign(cfg->schedule, cfg->schedule + T);
  p->cfg.schedule = nullptr;
  p->k = L.k;
  p->rsize = p->dbl ? 8 : 4;
  const int64_t N = p->N;
  p->ntiles = L.J.ntiles;
  p->nstiles = L.J.nstiles;
  const int ystride = L.J.ystride;
  void* v;
#define ALLOC(field, bytes)                                              \
  if ((st = plan_alloc(p.get(), (bytes), &v))) { plan_release(p.get()); return st; } \
  p->field = decltype(p->field)(v);
  ALLOC(params, L.params.size());
  ALLOC(pp, sizeof(double) * L.pp.size());
  ALLOC(ystep, p->rsize * (size_t)T * ystride);
  ALLOC(X0, p->rsize * (size_t)N * m->dx);
  ALLOC(X1, p->rsize * (size_t)N * m->dx);
  ALLOC(lw, p->rsize * (size_t)N);
  ALLOC(key, sizeof(double) * (size_t)N);
  ALLOC(ocum, sizeof(int32_t) * (size_t)N);
  ALLOC(mpk, sizeof(int32_t) * (size_t)(p->ntiles + 1));
  ALLOC(anc, sizeof(int32_t) * (size_t)N);
  if (cfg->lookahead != GF_LOOKAHEAD_NONE) { ALLOC(eta, p->rsize * (size_t)N); }
  ALLOC(tprefix, sizeof(double) * (size_t)(p->ntiles + 1));
  ALLOC(part, sizeof(double) * PF_PW * (size_t)p->ntiles * PF_MAX_SPLIT);
  ALLOC(mpart, sizeof(double) * (size_t)p->ntiles * m->dx);
  ALLOC(flags, sizeof(unsigned long long) * 2 * (size_t)p->nstiles);
  ALLOC(sc, sizeof(PfScalars));
  ALLOC(ess1, sizeof(double));
  ALLOC(res1, 8);
  ALLOC(job_dev, sizeof(PfJob));
  if (!p->sched.empty()) { ALLOC(sched_dev, (size_t)T); }
  if (!L.obs_consts.empty()) { ALLOC(obs_consts, sizeof(double) * L.obs_consts.size()); }
#undef ALLOC
  cudaStream_t s = ctx->stream;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->params, L.params.data(), L.params.size(), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->pp, L.pp.data(), sizeof(double) * L.pp.size(), cudaMemcpyHostToDevice, s));
  if (p->sched_dev)
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->sched_dev, p->sched.data(), (size_t)T, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->ess1, &L.ess1, sizeof(double), cudaMemcpyHostToDevice, s));
  if (p->obs_consts)
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->obs_consts, L.obs_consts.data(), sizeof(double) * L.obs_consts.size(),
                                       cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->res1, &L.res1, 1, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  p->small = p->N <= PF_TILE && cfg->resampler != GF_RS_MULTINOMIAL && p->k.small && !(flags & GF_PLAN_NO_FUSE);
  if (p->small)
    for (auto f : {p->k.small, p->k.small_means})
      GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)p->k.smem));
  p->prop_fn = L.prop;
  p->prop_threads = L.threads;
  p->prop_split = L.split;
  p->prop_smem = L.smem;
  p->units = L.units_blocks > 0;
  p->prop_grid = L.units_blocks ? (int)std::min<int64_t>((int64_t)p->ntiles * TC_SUB_UNITS,
                                                        (int64_t)ctx->num_sms * L.units_blocks)
                                : p->ntiles * L.split;
  GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)p->prop_fn,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->prop_smem));
  // all of the SM's shared memory, so the tensor-core propagate reaches its
  // register-bound residency (5 blocks per SM at Dx=16)
  GF_CHECK_CUDA(ctx, cudaFuncSetAttribute((const void*)p->prop_fn,
                                          cudaFuncAttributePreferredSharedMemoryCarveout,
                                          (int)cudaSharedmemCarveoutMaxShared));
  PfJob& J = p->job;
  J = L.J;
  J.params = p->params;
  J.ystep = p->ystep;
  J.X[0] = p->X0;
  J.X[1] = p->X1;
  J.lw = p->lw;
  J.key = p->key;
  J.part = p->part;
  J.flags = p->flags;
  J.sc = p->sc;
  J.ocum = p->ocum;
  J.mpk = p->mpk;
  J.anc = p->anc;
  J.tprefix = p->tprefix;
  J.eta = p->eta;
  J.schedule = p->sched_dev;
  J.obs_consts = p->obs_consts;
  *out = p.release();
  return GF_OK;
}

extern "C" gf_status gf_pf_plan_create(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg,
                                       int32_t T, int32_t flags, gf_pf_plan** out) {
  return pf_plan_create_impl(ctx, m, 1, cfg, T, flags, out);
}

extern "C" gf_status gf_pf_plan_create_tv(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                                          const gf_pf_config* cfg, int32_t T, int32_t flags,
                                          gf_pf_plan** out) {
  return pf_plan_create_impl(ctx, m, param_steps, cfg, T, flags, out);
}

// Enqueues one full filter run (prep, init, T steps, outputs) on the stream.
// Auxiliary filter: the first-stage scores and the resampling decision of the
// coming step, between a propagate and the resample.
static void launch_lookahead(gf_pf_plan* p) {
  if (!p->eta) return;
  ProfScope ps(p->ctx, KC_SCAN);
  p->k.lookahead<<<p->ntiles, PF_THREADS, 0, p->ctx->stream>>>(p->job_dev, 1);
}

static void enqueue_run(gf_pf_plan* p, bool means, bool record) {
  gf_ctx* ctx = p->ctx;
  cudaStream_t s = ctx->stream;
  launch_prep(ctx, p->dbl, p->job_dev, p->T, p->dx, p->dy, p->k.dxp, p->k.dyp, p->pp, p->ystep);
  launch_init_scalars(ctx, p->job_dev, 1, p->ess1, p->res1);
  if (p->small && !record && !p->eta) {
    // the whole filter in one block (N <= 1024): no per-step launches
    ProfScope ps(ctx, KC_PROPAGATE);
    (means ? p->k.small_means : p->k.small)<<<1, PF_THREADS, p->k.smem, s>>>(p->job_dev, p->k.off_mu0,
                                                                          p->k.off_L0, p->mpart);
    return;
  }
  cudaMemsetAsync(p->flags, 0, sizeof(unsigned long long) * 2 * p->nstiles, s);
  {
    ProfScope ps(ctx, KC_PREP);
    p->k.init<<<p->ntiles, PF_THREADS, 0, s>>>(p->job_dev, 1, p->k.off_mu0, p->k.off_L0);
  }
  if (record) launch_record(ctx, p->dbl, p->job_dev, p->N);
  launch_lookahead(p);
  launch_resample(ctx, p->dbl, p->job_dev, 1, p->ntiles);
  for (int t = 1; t <= p->T; ++t) {
    {
      ProfScope ps(ctx, KC_PROPAGATE);
      p->prop_fn<<<p->prop_grid, p->prop_threads, p->prop_smem, s>>>(p->job_dev, 1);
    }
    if (p->units) launch_finish_units(ctx, p->job_dev, 1);
    if (means) launch_means(ctx, p->dbl, p->job_dev, 1, p->ntiles, p->mpart, p->dx);
    if (record) launch_record(ctx, p->dbl, p->job_dev, p->N);
    if (t < p->T) {
      launch_lookahead(p);
      launch_resample(ctx, p->dbl, p->job_dev, 1, p->ntiles);
    }
  }
  launch_finish(ctx, p->dbl, p->job_dev, p->N);
}

// ---------------------------------------------------------- path storage
// One run with path storage (eager launches: the pool is sized between chunks).
static gf_status enqueue_run_paths(gf_pf_plan* p, bool means, bool record, void* paths) {
  gf_ctx* ctx = p->ctx;
  cudaStream_t s = ctx->stream;
  p->tree.ctx = ctx;
  p->tree.N = p->N;
  p->tree.width = p->dx;
  p->tree.rsize = p->rsize;
  gf_status st = tree_host_prepare(p->tree);
  if (st) return st;
  launch_prep(ctx, p->dbl, p->job_dev, p->T, p->dx, p->dy, p->k.dxp, p->k.dyp, p->pp, p->ystep);
  launch_init_scalars(ctx, p->job_dev, 1, p->ess1, p->res1);
  GF_CHECK_CUDA(ctx, cudaMemsetAsync(p->flags, 0, sizeof(unsigned long long) * 2 * p->nstiles, s));
  p->k.init<<<p->ntiles, PF_THREADS, 0, s>>>(p->job_dev, 1, p->k.off_mu0, p->k.off_L0);
  tree_launch_init(ctx, p->dbl, p->job_dev, p->N, p->tree.tree);
  if (record) launch_record(ctx, p->dbl, p->job_dev, p->N);
  launch_lookahead(p);
  launch_resample(ctx, p->dbl, p->job_dev, 1, p->ntiles);
  for (int t = 1; t <= p->T; ++t) {
    if ((t - 1) % kTreeChunk == 0) {
      const int64_t steps = std::min<int64_t>(kTreeChunk, p->T - t + 1);
      if ((st = tree_host_reserve(p->tree, steps * p->N))) return st;
    }
    tree_launch_step_pre(ctx, p->job_dev, p->N, p->tree.tree, p->cfg.resampler != GF_RS_MULTINOMIAL);
    p->prop_fn<<<p->prop_grid, p->prop_threads, p->prop_smem, s>>>(p->job_dev, 1);
    if (p->units) launch_finish_units(ctx, p->job_dev, 1);
    tree_launch_insert(ctx, p->dbl, p->job_dev, p->N, p->tree.tree, t);
    if (means) launch_means(ctx, p->dbl, p->job_dev, 1, p->ntiles, p->mpart, p->dx);
    if (record) launch_record(ctx, p->dbl, p->job_dev, p->N);
    if (t < p->T) {
      launch_lookahead(p);
      launch_resample(ctx, p->dbl, p->job_dev, 1, p->ntiles);
    }
  }
  launch_finish(ctx, p->dbl, p->job_dev, p->N);
  tree_launch_paths(ctx, p->dbl, p->job_dev, p->N, p->tree.tree, p->T, paths);
  GF_CHECK_CUDA(ctx, cudaGetLastError());
  return GF_OK;
}

extern "C" gf_status gf_pf_plan_run(gf_pf_plan* p, const double* ys_dev, const void* noise_dev,
                                    const double* uniforms_dev, gf_pf_out* out) {
  if (!p || !out || !ys_dev) return GF_ERR_ARG;
  gf_ctx* ctx = p->ctx;
  cudaSetDevice(ctx->device);
  PfJob& J = p->job;
  J.ys = ys_dev;
  J.noise = noise_dev;
  J.unif = uniforms_dev;
  J.ll_steps = out->ll_steps;
  J.ess_steps = out->ess_steps;
  J.res_steps = out->resampled;
  J.anc_out = out->ancestors;
  J.ll_out = out->ll;
  J.logw_out = out->log_weights;
  J.states_out = out->states;
  J.clamps_out = out->clamps;
  J.means_out = out->means;
  J.hist = out->history;
  J.lwh = out->log_weight_history;
  cudaStream_t s = ctx->stream;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(p->job_dev, &J, sizeof(PfJob), cudaMemcpyHostToDevice, s));
  const bool means = out->means != nullptr;
  const bool record = out->history || out->log_weight_history;
  if (out->paths) return enqueue_run_paths(p, means, record, out->paths);
  if (p->use_graph && !ctx->profiling) {
    if (!p->graph || p->graph_means != means || p->graph_record != record) {
      if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
      }
      cudaGraph_t g;
      GF_CHECK_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      enqueue_run(p, means, record);
      GF_CHECK_CUDA(ctx, cudaStreamEndCapture(s, &g));
      cudaError_t e = cudaGraphInstantiate(&p->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_err(ctx, e, "cudaGraphInstantiate");
      p->graph_means = means;
      p->graph_record = record;
    }
    GF_CHECK_CUDA(ctx, cudaGraphLaunch(p->graph, s));
  } else {
    enqueue_run(p, means, record);
    GF_CHECK_CUDA(ctx, cudaGetLastError());
  }
  return GF_OK;
}

extern "C" gf_status gf_pf_plan_destroy(gf_pf_plan* p) {
  if (!p) return GF_OK;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  plan_release(p);
  delete p;
  return GF_OK;
}

// Reads the job status after a run (synchronises the stream).
static gf_status plan_status(gf_pf_plan* p) {
  gf_ctx* ctx = p->ctx;
  PfScalars sc;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(&sc, p->sc, sizeof sc, cudaMemcpyDeviceToHost, ctx->stream));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (sc.status == GF_ERR_TIMEOUT) return set_err(ctx, GF_ERR_TIMEOUT, "lookback scan wait timed out");
  if (sc.status != 0)
    return set_err(ctx, sc.status, "particle weights degenerated at step %d (all zero or NaN)", sc.t + 1);
  return GF_OK;
}

// ------------------------------------------------------------- gf_pf_run
namespace {
struct TmpDev {
  gf_ctx* ctx;
  std::vector<DevBuf> v;
  explicit TmpDev(gf_ctx* c) : ctx(c) {}
  ~TmpDev() {
    for (auto& b : v) dev_free(ctx, b.p, b.bytes);
  }
  gf_status get(size_t bytes, void** p) {
    gf_status st = dev_alloc(ctx, bytes, p);
    if (!st && *p) v.push_back({*p, bytes});
    return st;
  }
};
}  // namespace

// One-shot calls keep their plans in the context: a call with the same model,
// configuration (all but the seed), T and parameter steps as a kept plan reuses
// its device buffers and its captured CUDA graph instead of building them again
// (PF_PLAN_CACHE plans per context, least recently used dropped; models whose
// key exceeds PF_PLAN_KEY_MAX bytes are not kept).
constexpr size_t PF_PLAN_CACHE = 4;
constexpr size_t PF_PLAN_KEY_MAX = 1 << 20;

namespace gf {
void pf_plan_cache_release(gf_ctx* ctx) {
  for (auto& e : ctx->pf_plans) gf_pf_plan_destroy(static_cast<gf_pf_plan*>(e.second));
  ctx->pf_plans.clear();
}
}  // namespace gf

static bool pf_plan_key(const gf_lg_model* m, int32_t param_steps, const gf_pf_config* cfg, int32_t T,
                        std::vector<char>& key) {
  if (!m || !cfg || m->dx < 1 || m->dy < 1 || T < 1) return false;
  const size_t dx = m->dx, dy = m->dy, nb = param_steps > 1 ? (size_t)param_steps : 1;
  const size_t bytes = 8 * (dx + dx * dx + nb * (2 * dx * dx + dx + dy * dx + dy + dy * dy)) + T + 128;
  if (bytes > PF_PLAN_KEY_MAX) return false;
  key.clear();
  key.reserve(bytes);
  auto put = [&](const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    key.insert(key.end(), c, c + n);
  };
  gf_pf_config c = *cfg;
  c.seed = 0;
  c.schedule = nullptr;
  const int32_t hdr[4] = {m->dx, m->dy, T, param_steps};
  put(hdr, sizeof hdr);
  put(&c, sizeof c);
  const int8_t has_sched = cfg->schedule ? 1 : 0;
  put(&has_sched, 1);
  if (cfg->schedule) put(cfg->schedule, (size_t)T);
  put(m->mu0, 8 * dx);
  put(m->Sigma0, 8 * dx * dx);
  put(m->A, 8 * nb * dx * dx);
  put(m->b, 8 * nb * dx);
  put(m->Q, 8 * nb * dx * dx);
  put(m->H, 8 * nb * dy * dx);
  put(m->c, 8 * nb * dy);
  put(m->R, 8 * nb * dy * dy);
  return true;
}

static gf_status pf_run_impl(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                             const gf_pf_config* cfg, int32_t T, const double* ys, const void* noise,
                             const double* uniforms, int32_t memspace, gf_pf_out* out) {
  if (!ctx || !out || !ys) return ctx ? set_err(ctx, GF_ERR_ARG, "null argument") : GF_ERR_ARG;
  if (!out->ll) return set_err(ctx, GF_ERR_ARG, "out->ll is required");
  gf_pf_plan* p = nullptr;
  gf_status st = GF_OK;
  std::vector<char> key;
  const bool keep = pf_plan_key(m, param_steps, cfg, T, key);
  for (size_t k = 0; keep && k < ctx->pf_plans.size(); ++k)
    if (ctx->pf_plans[k].first == key) {
      p = static_cast<gf_pf_plan*>(ctx->pf_plans[k].second);
      std::rotate(ctx->pf_plans.begin(), ctx->pf_plans.begin() + k, ctx->pf_plans.begin() + k + 1);
      break;
    }
  std::unique_ptr<gf_pf_plan, gf_status (*)(gf_pf_plan*)> guard(nullptr, gf_pf_plan_destroy);
  if (!p) {
    st = pf_plan_create_impl(ctx, m, param_steps, cfg, T, keep ? 0 : GF_PLAN_NO_GRAPH, &p);
    if (st && !ctx->pf_plans.empty() && (st == GF_ERR_OOM_BUDGET || st == GF_ERR_CUDA)) {
      // the kept plans hold device memory: drop them and try once more
      pf_plan_cache_release(ctx);
      cudaGetLastError();
      st = pf_plan_create_impl(ctx, m, param_steps, cfg, T, keep ? 0 : GF_PLAN_NO_GRAPH, &p);
    }
    if (st) return st;
    if (keep) {
      ctx->pf_plans.insert(ctx->pf_plans.begin(), {std::move(key), p});
      while (ctx->pf_plans.size() > PF_PLAN_CACHE) {
        gf_pf_plan_destroy(static_cast<gf_pf_plan*>(ctx->pf_plans.back().second));
        ctx->pf_plans.pop_back();
      }
    } else {
      guard.reset(p);
    }
  }
  p->cfg.seed = cfg->seed;
  p->job.seed = cfg->seed;
  if (memspace == GF_MEM_DEVICE) {
    if ((st = gf_pf_plan_run(p, ys, noise, uniforms, out))) return st;
    return plan_status(p);
  }
  // host buffers: stage through device memory
  TmpDev tmp(ctx);
  cudaStream_t s = ctx->stream;
  const int64_t N = p->N;
  const size_t rs = p->rsize;
  void *d_ys, *d_noise = nullptr, *d_unif = nullptr;
  if ((st = tmp.get(sizeof(double) * (size_t)T * m->dy, &d_ys))) return st;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(d_ys, ys, sizeof(double) * (size_t)T * m->dy, cudaMemcpyHostToDevice, s));
  if (noise) {
    size_t nb = rs * (size_t)(T + 1) * m->dx * N;
    if ((st = tmp.get(nb, &d_noise))) return st;
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(d_noise, noise, nb, cudaMemcpyHostToDevice, s));
  }
  if (uniforms) {
    size_t ub = sizeof(double) * (size_t)T * (cfg->resampler == GF_RS_SYSTEMATIC ? 1 : N);
    if ((st = tmp.get(ub, &d_unif))) return st;
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(d_unif, uniforms, ub, cudaMemcpyHostToDevice, s));
  }
  gf_pf_out d{};
  struct Map {
    void* host;
    void** dev;
    size_t bytes;
  };
  std::vector<Map> maps;
  auto mk = [&](void* hptr, void** dptr, size_t bytes) -> gf_status {
    if (!hptr) return GF_OK;
    gf_status s2 = tmp.get(bytes, dptr);
    if (!s2) maps.push_back({hptr, dptr, bytes});
    return s2;
  };
  if ((st = mk(out->ll, (void**)&d.ll, sizeof(double)))) return st;
  if ((st = mk(out->ll_steps, (void**)&d.ll_steps, sizeof(double) * T))) return st;
  if ((st = mk(out->ess_steps, (void**)&d.ess_steps, sizeof(double) * T))) return st;
  if ((st = mk(out->resampled, (void**)&d.resampled, (size_t)T))) return st;
  if ((st = mk(out->ancestors, (void**)&d.ancestors, sizeof(int32_t) * (size_t)T * N))) return st;
  if ((st = mk(out->means, (void**)&d.means, sizeof(double) * (size_t)T * m->dx))) return st;
  if ((st = mk(out->states, (void**)&d.states, rs * (size_t)N * m->dx))) return st;
  if ((st = mk(out->log_weights, (void**)&d.log_weights, sizeof(double) * (size_t)N))) return st;
  if ((st = mk(out->clamps, (void**)&d.clamps, sizeof(int32_t)))) return st;
  if ((st = mk(out->paths, (void**)&d.paths, rs * (size_t)(T + 1) * m->dx * N))) return st;
  if ((st = mk(out->history, (void**)&d.history, rs * (size_t)(T + 1) * m->dx * N))) return st;
  if ((st = mk(out->log_weight_history, (void**)&d.log_weight_history, sizeof(double) * (size_t)T * N)))
    return st;
  if ((st = gf_pf_plan_run(p, (const double*)d_ys, d_noise, (const double*)d_unif, &d))) return st;
  for (auto& mp : maps)
    GF_CHECK_CUDA(ctx, cudaMemcpyAsync(mp.host, *mp.dev, mp.bytes, cudaMemcpyDeviceToHost, s));
  return plan_status(p);
}

extern "C" gf_status gf_pf_run(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg,
                               int32_t T, const double* ys, const void* noise,
                               const double* uniforms, int32_t memspace, gf_pf_out* out) {
  return pf_run_impl(ctx, m, 1, cfg, T, ys, noise, uniforms, memspace, out);
}

extern "C" gf_status gf_pf_run_tv(gf_ctx* ctx, const gf_lg_model* m, int32_t param_steps,
                                  const gf_pf_config* cfg, int32_t T, const double* ys,
                                  const void* noise, const double* uniforms, int32_t memspace,
                                  gf_pf_out* out) {
  return pf_run_impl(ctx, m, param_steps, cfg, T, ys, noise, uniforms, memspace, out);
}
