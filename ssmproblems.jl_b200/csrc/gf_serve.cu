// gf_serve.cu -- the serving loop: many independent filter requests on one GPU.
//
// No reference counterpart: GeneralisedFilters runs one synchronous `filter`
// call at a time (GeneralisedFilters.jl:58-84).  Here a worker thread owns the
// GPU and runs every admitted request concurrently:
//
//  * Admission is first-come-first-served against two fixed arenas carved out
//    once at start-up: device memory (the HBM budget) and pinned, device-mapped
//    host memory for staging and results.  A request whose blocks do not fit
//    waits; one larger than an arena is rejected with GF_ERR_OOM_BUDGET.
//    Carving from fixed slabs keeps cudaMalloc / cudaFree (which synchronise
//    the device) out of the loop.
//  * Kalman requests (KF, SRKF) admitted in the same loop iteration form one
//    batch: one persistent launch per dimension bucket, each on an idle stream
//    of a small pool.  Every filter publishes its ll, final mean / covariance
//    and per-step log-likelihoods to host-mapped memory and then sets a done
//    flag behind a system-scope fence, so a short filter completes while the
//    rest of its batch still runs.
//  * Particle-filter requests (LG PF, RBPF) are continuously batched: all
//    running jobs of one kernel variant share each propagate / resample /
//    ancestor-fill launch (blocks map to jobs through the job table), in
//    chunks of `pf_chunk` steps.  New jobs join and finished jobs leave at
//    chunk boundaries; at most two chunks are in flight.
//
// A served request computes exactly what the standalone entry point computes
// on the same inputs (gf_kf_batch, gf_pf_run, gf_rbpf_run with in-kernel
// Philox draws): the same kernels, per-job tiling and reductions.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "gf_internal.hpp"
#include "gf_kf_host.hpp"
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"

namespace gf {
namespace {

constexpr size_t kAlign = 256;
inline size_t round_up(size_t x) { return (std::max<size_t>(x, 1) + kAlign - 1) / kAlign * kAlign; }

// Best-fit offset allocator over one slab; adjacent free blocks coalesce.
class Arena {
 public:
  void reset(size_t cap) {
    cap_ = cap;
    used_ = peak_ = 0;
    free_.clear();
    if (cap) free_[0] = cap;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = round_up(bytes);
    auto best = free_.end();
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= bytes && (best == free_.end() || it->second < best->second)) best = it;
    if (best == free_.end()) return false;
    const size_t o = best->first, rest = best->second - bytes;
    free_.erase(best);
    if (rest) free_[o + bytes] = rest;
    *off = o;
    used_ += bytes;
    peak_ = std::max(peak_, used_);
    return true;
  }
  void release(size_t off, size_t bytes) {
    bytes = round_up(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t cap() const { return cap_; }
  size_t used() const { return used_; }
  size_t peak() const { return peak_; }
  size_t free_blocks() const { return free_.size(); }

 private:
  size_t cap_ = 0, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;
};

// Sequential sub-allocation of one block into 256-byte aligned pieces.
struct Layout {
  size_t size = 0;
  size_t take(size_t bytes) {
    size_t o = size;
    size += round_up(bytes);
    return o;
  }
};

enum { REQ_KF = GF_REQ_KF, REQ_SRKF = GF_REQ_SRKF, REQ_PF = GF_REQ_PF, REQ_RBPF = GF_REQ_RBPF };

struct Req {
  uint64_t id = 0, tag = 0;
  int kind = 0, T = 0;
  int64_t obs_off = 0;  // PF: offset (doubles) of the per-step constants in the prep buffer
  int dx = 0, dy = 0, mdim = 0;  // mdim: length of the mean result
  int64_t N = 0;
  double jitter = 0.0;
  int use_jitter = 0;
  double *out_steps = nullptr, *out_mean = nullptr, *out_cov = nullptr;
  std::vector<double> ys;
  std::vector<int8_t> sched;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // packed inputs
  std::vector<float> kf_params;      // KF / SRKF pool entry; RBPF parameters
  std::unique_ptr<LgJobSetup> lg;    // LG PF
  RbKernels rk{};
  float q_gamma = 0.f;
  int q_index = 0, guided = 0;
  double rb_prop_const = 0.0;
  double ess1 = 0.0;
  int8_t res1 = 0;
  int64_t kf_plen = 0;
  // blocks
  Layout dl, pl;                     // device / pinned layouts
  size_t doff = 0, poff = 0;
  bool have_dev = false, have_pin = false;
  // device piece offsets (relative to the block)
  size_t d_params = 0, d_pp = 0, d_ys = 0, d_ystep = 0, d_X0 = 0, d_X1 = 0, d_lw = 0, d_key = 0,
         d_ocum = 0, d_anc = 0, d_mpk = 0, d_tpre = 0, d_part = 0, d_mpart = 0, d_flags = 0,
         d_sc = 0, d_ess1 = 0, d_res1 = 0, d_job = 0, d_sched = 0, d_steps = 0, d_means = 0;
  // pinned piece offsets
  size_t p_params = 0, p_pp = 0, p_ys = 0, p_sched = 0, p_job = 0, p_e1 = 0, p_rec = 0, p_mu = 0,
         p_cov = 0, p_steps = 0, p_sc = 0, p_mean = 0;
  // particle-filter state
  PfJob job{};
  PfJob* job_dev = nullptr;
  int group = -1;
  int launched = 0;  // steps enqueued
  cudaEvent_t ev = nullptr;
  gf_status status = GF_OK;
  double ll = 0.0;
};

struct Group {
  bool rb = false, dbl = false;
  void (*prop)(const PfJob*, int) = nullptr;
  int threads = 0, split = 1;
  size_t smem = 0;
  RbKernels rk{};
  float q_gamma = 0.f;
  int q_index = 0, guided = 0;
  std::vector<Req*> active;
  PfJob* dev[2] = {nullptr, nullptr};
  PfJob* host[2] = {nullptr, nullptr};
  size_t doff = 0, poff = 0;
};

struct KfBatch {
  std::vector<Req*> reqs;
  std::vector<cudaEvent_t> evs;
  size_t doff = 0, dbytes = 0, poff = 0, pbytes = 0;
};

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace gf

using namespace gf;

struct gf_srv {
  gf_srv_config cfg{};
  int device = 0, num_sms = 148;
  gf_ctx pfx;  // internal context: the particle-filter stream for the launch helpers
  unsigned char* dbase = nullptr;  // device slab
  unsigned char* pbase = nullptr;  // pinned, mapped host slab
  unsigned char* pdev = nullptr;   // device view of the pinned slab
  Arena darena, parena;
  std::vector<cudaStream_t> kf_streams;
  std::vector<cudaEvent_t> kf_last;  // last event recorded on each KF stream (or null)
  std::vector<char> kf_busy;         // claimed by the batch being formed
  int kf_per_sm[2][8] = {};          // resident blocks per SM of each bucket kernel
  std::vector<cudaEvent_t> ev_pool;
  std::deque<cudaEvent_t> chunk_evs;
  uint64_t chunk_no = 0;
  std::vector<std::unique_ptr<Group>> groups;
  std::vector<Req*> kf_ready[2];
  std::vector<Req*> kf_running;
  std::vector<std::unique_ptr<KfBatch>> batches;
  std::vector<Req*> pf_finishing;
  int active_pf = 0;

  // shared with submitting / polling threads
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> inbox;
  std::deque<gf_srv_result> outbox;
  std::string err;
  bool stop = false;
  uint64_t next_id = 1;
  int64_t n_submitted = 0, n_completed = 0, n_failed = 0, n_rejected = 0;
  std::atomic<int64_t> n_pending{0}, n_running{0};
  std::vector<double> lat;  // completed latencies (ms)
  double kf_steps = 0, particle_steps = 0;
  double t0 = 0, t_first = -1, t_last = 0;
  std::atomic<int64_t> pf_iters{0}, kf_batches{0}, launches{0};
  std::atomic<size_t> hbm_used{0}, hbm_peak{0};

  // worker-only
  std::deque<Req*> pending;
  std::thread worker;
  std::string werr;

  void* dptr(size_t off) { return dbase + off; }
  void* pptr(size_t off) { return pbase + off; }
  void* pdptr(size_t off) { return pdev + off; }

  cudaEvent_t take_ev() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }
  void give_ev(cudaEvent_t e) {
    if (e) ev_pool.push_back(e);
  }

  void loop();
  bool admit();
  gf_status start_pf(Req* r);
  bool launch_kf();
  bool pf_iterate();
  bool reap();
  void finish(Req* r, gf_status st);
  void release(Req* r);
  Group* group_for(Req* r);
  cudaStream_t idle_kf_stream(int* idx);
};

// ------------------------------------------------------------- request setup
namespace {

gf_status copy_lg(const gf_lg_model* m, std::vector<double>& store, gf_lg_model* out) {
  const int dx = m->dx, dy = m->dy;
  const size_t n = (size_t)dx + 3 * dx * dx + dx + dy * dx + dy + dy * dy;
  store.resize(n);
  double* p = store.data();
  auto cp = [&](const double* src, size_t k) -> const double* {
    double* d = p;
    std::memcpy(d, src, sizeof(double) * k);
    p += k;
    return d;
  };
  *out = *m;
  out->mu0 = cp(m->mu0, dx);
  out->Sigma0 = cp(m->Sigma0, (size_t)dx * dx);
  out->A = cp(m->A, (size_t)dx * dx);
  out->b = cp(m->b, dx);
  out->Q = cp(m->Q, (size_t)dx * dx);
  out->H = cp(m->H, (size_t)dy * dx);
  out->c = cp(m->c, dy);
  out->R = cp(m->R, (size_t)dy * dy);
  return GF_OK;
}

// Device and pinned layouts of a particle-filter request (LG or RBPF).
void pf_layout(Req* r, size_t param_bytes, size_t pp_bytes, size_t rsize, int width, int ystride) {
  const int64_t N = r->N;
  const int T = r->T;
  const int ntiles = (int)((N + PF_TILE - 1) / PF_TILE);
  const int nstiles = (int)((N + SCAN_TILE - 1) / SCAN_TILE);
  Layout& d = r->dl;
  r->d_params = d.take(param_bytes);
  r->d_pp = pp_bytes ? d.take(pp_bytes) : 0;
  r->d_ys = d.take(sizeof(double) * (size_t)T * r->dy);
  r->d_ystep = ystride ? d.take(rsize * (size_t)T * ystride) : 0;
  r->d_X0 = d.take(rsize * (size_t)N * width);
  r->d_X1 = d.take(rsize * (size_t)N * width);
  r->d_lw = d.take(rsize * (size_t)N);
  r->d_key = d.take(sizeof(double) * (size_t)N);
  r->d_ocum = d.take(sizeof(int32_t) * (size_t)N);
  r->d_anc = d.take(sizeof(int32_t) * (size_t)N);
  r->d_mpk = d.take(sizeof(int32_t) * (size_t)(ntiles + 1));
  r->d_tpre = d.take(sizeof(double) * (size_t)(ntiles + 1));
  r->d_part = d.take(sizeof(double) * PF_PW * (size_t)ntiles * PF_MAX_SPLIT);  // per-block partials
  r->d_mpart = d.take(sizeof(double) * (size_t)ntiles * std::max(1, r->mdim));
  r->d_flags = d.take(sizeof(unsigned long long) * 2 * (size_t)nstiles);
  r->d_sc = d.take(sizeof(PfScalars));
  r->d_ess1 = d.take(sizeof(double));
  r->d_res1 = d.take(8);
  r->d_job = d.take(sizeof(PfJob));
  if (!r->sched.empty()) r->d_sched = d.take((size_t)T);
  if (r->out_steps) r->d_steps = d.take(sizeof(double) * (size_t)T);
  if (r->out_mean) r->d_means = d.take(sizeof(double) * (size_t)T * r->mdim);
  Layout& p = r->pl;
  r->p_params = p.take(param_bytes);
  r->p_pp = pp_bytes ? p.take(pp_bytes) : 0;
  r->p_ys = p.take(sizeof(double) * (size_t)T * r->dy);
  if (!r->sched.empty()) r->p_sched = p.take((size_t)T);
  r->p_job = p.take(sizeof(PfJob));
  r->p_e1 = p.take(16);
  r->p_sc = p.take(sizeof(PfScalars));
  if (r->out_steps) r->p_steps = p.take(sizeof(double) * (size_t)T);
  if (r->out_mean) r->p_mean = p.take(sizeof(double) * (size_t)r->mdim);
}

}  // namespace

static gf_status prepare(gf_ctx* ectx, const gf_srv_request* q, Req* r) {
  if (!q) return set_err(ectx, GF_ERR_ARG, "null request");
  if (q->T < 1) return set_err(ectx, GF_ERR_ARG, "T must be >= 1");
  if (!q->ys) return set_err(ectx, GF_ERR_ARG, "ys is required");
  r->kind = q->kind;
  if (q->kind != REQ_PF && q->param_steps > 1)
    return set_err(ectx, GF_ERR_UNSUPPORTED, "served time-varying models run with the particle filter");
  r->T = q->T;
  r->tag = q->tag;
  r->out_steps = q->ll_steps;
  r->out_mean = q->mean;
  r->out_cov = q->cov;
  std::vector<double> store;
  if (q->kind == REQ_KF || q->kind == REQ_SRKF) {
    if (!q->lg) return set_err(ectx, GF_ERR_ARG, "Kalman request needs lg");
    const gf_lg_model& m = *q->lg;
    if (m.dx < 1 || m.dy < 1) return set_err(ectx, GF_ERR_DIM, "dx, dy must be >= 1");
    if (kf_bucket_for(m.dx, m.dy) < 0) return set_err(ectx, GF_ERR_DIM, "dx=%d dy=%d exceeds 32", m.dx, m.dy);
    r->dx = m.dx;
    r->dy = m.dy;
    r->mdim = m.dx;
    r->jitter = q->jitter;
    r->use_jitter = q->use_jitter;
    gf_status st = kf_pack_model(ectx, q->kind == REQ_KF ? GF_ALGO_KF : GF_ALGO_SRKF, m, 0, r->kf_params);
    if (st) return st;
    r->kf_plen = (int64_t)r->kf_params.size();
    r->ys.assign(q->ys, q->ys + (size_t)r->T * r->dy);
    Layout& d = r->dl;
    r->d_params = d.take(sizeof(float) * r->kf_params.size());
    r->d_ys = d.take(sizeof(double) * r->ys.size());
    Layout& p = r->pl;
    r->p_params = p.take(sizeof(float) * r->kf_params.size());
    r->p_ys = p.take(sizeof(double) * r->ys.size());
    r->p_rec = p.take(sizeof(KfSrvRec));
    r->p_mu = p.take(sizeof(float) * r->dx);
    r->p_cov = p.take(sizeof(float) * r->dx * r->dx);
    if (r->out_steps) r->p_steps = p.take(sizeof(double) * r->T);
    return GF_OK;
  }
  if (!q->pf) return set_err(ectx, GF_ERR_ARG, "particle-filter request needs pf");
  const gf_pf_config& cfg = *q->pf;
  if (cfg.lookahead != GF_LOOKAHEAD_NONE)
    return set_err(ectx, GF_ERR_UNSUPPORTED, "the serving loop runs bootstrap and guided filters, not the auxiliary filter");
  if (cfg.n_particles < 1 || cfg.n_particles > (int64_t(1) << 31) - 1)
    return set_err(ectx, GF_ERR_ARG, "n_particles must be in [1, 2^31)");
  r->N = cfg.n_particles;
  if (cfg.schedule) r->sched.assign(cfg.schedule, cfg.schedule + r->T);
  const int sch0 = cfg.schedule ? cfg.schedule[0] : -1;
  if (q->kind == REQ_PF) {
    if (!q->lg) return set_err(ectx, GF_ERR_ARG, "PF request needs lg");
    r->lg.reset(new LgJobSetup);
    gf_status st = lg_job_setup(ectx, q->lg, &cfg, r->T, 0, r->lg.get(), q->param_steps > 1 ? q->param_steps : 1);
    if (st) return st;
    // a time-varying model's per-step observation and proposal constants ride at
    // the end of the observation-prep buffer
    r->obs_off = (int64_t)r->lg->pp.size();
    r->lg->pp.insert(r->lg->pp.end(), r->lg->obs_consts.begin(), r->lg->obs_consts.end());
    r->dx = q->lg->dx;
    r->dy = q->lg->dy;
    r->mdim = r->dx;
    r->ess1 = r->lg->ess1;
    r->res1 = r->lg->res1;
    r->ys.assign(q->ys, q->ys + (size_t)r->T * r->dy);
    pf_layout(r, r->lg->params.size(), sizeof(double) * r->lg->pp.size(), r->lg->dbl ? 8 : 4, r->dx,
              r->lg->J.ystride);
    return GF_OK;
  }
  if (q->kind != REQ_RBPF) return set_err(ectx, GF_ERR_ARG, "unknown request kind %d", q->kind);
  if (!q->rb) return set_err(ectx, GF_ERR_ARG, "RBPF request needs rb");
  const gf_rb_model& m = *q->rb;
  if (cfg.precision != GF_PREC_F32) return set_err(ectx, GF_ERR_UNSUPPORTED, "RBPF runs in FP32 only");
  if (cfg.proposal == GF_PROP_OPTIMAL)
    return set_err(ectx, GF_ERR_UNSUPPORTED, "RBPF supports bootstrap and overdispersed outer proposals");
  if (cfg.resampler < 0 || cfg.resampler > 2 || cfg.convention < 0 || cfg.convention > 1)
    return set_err(ectx, GF_ERR_ARG, "unknown resampler or convention");
  if (!pick_rb(m.dxo, m.dz, m.dy, &r->rk))
    return set_err(ectx, GF_ERR_DIM, "no RBPF kernel for (dxo, dz, dy) = (%d, %d, %d)", m.dxo, m.dz, m.dy);
  gf_status st = rb_pack_params(ectx, &m, &cfg, r->kf_params, &r->rb_prop_const);
  if (st) return st;
  r->dx = m.dxo;
  r->dy = m.dy;
  r->mdim = m.dxo + m.dz;
  r->q_gamma = (float)m.q_gamma;
  r->q_index = m.q_index;
  r->guided = cfg.proposal == GF_PROP_OVERDISPERSED;
  r->ess1 = uniform_ess(r->N);
  r->res1 = (int8_t)(sch0 >= 0 ? (sch0 != 0) : (cfg.threshold * (double)r->N >= r->ess1));
  r->ys.assign(q->ys, q->ys + (size_t)r->T * r->dy);
  const int width = m.dxo + m.dz + m.dz * (m.dz + 1) / 2;
  pf_layout(r, sizeof(float) * r->kf_params.size(), 0, 4, width, 0);
  // job template (RBPF fields as gf_rbpf_run sets them)
  PfJob& J = r->job;
  std::memset(&J, 0, sizeof J);
  J.N = r->N;
  J.dx = m.dxo;
  J.dy = m.dy;
  J.T = r->T;
  J.width = width;
  J.ntiles = (int)((r->N + PF_TILE - 1) / PF_TILE);
  J.nstiles = (int)((r->N + SCAN_TILE - 1) / SCAN_TILE);
  J.resampler = cfg.resampler;
  J.conv = cfg.convention;
  J.prop = cfg.proposal;
  J.threshold = cfg.threshold;
  J.log_n = std::log((double)r->N);
  J.prop_const = r->rb_prop_const;
  J.seed = cfg.seed;
  return GF_OK;
}

// ------------------------------------------------------------------ worker
Group* gf_srv::group_for(Req* r) {
  for (auto& g : groups) {
    if (r->kind == REQ_PF && !g->rb && g->prop == r->lg->prop && g->dbl == r->lg->dbl) return g.get();
    if (r->kind == REQ_RBPF && g->rb && g->rk.prop == r->rk.prop && g->q_gamma == r->q_gamma &&
        g->q_index == r->q_index && g->guided == r->guided)
      return g.get();
  }
  auto g = std::make_unique<Group>();
  const size_t cap = (size_t)cfg.max_active_pf;
  // job tables live in the arenas for the server's lifetime
  size_t bytes = 2 * sizeof(PfJob) * cap;
  if (!darena.alloc(bytes, &g->doff)) return nullptr;
  if (!parena.alloc(bytes, &g->poff)) {
    darena.release(g->doff, bytes);
    return nullptr;
  }
  g->dev[0] = (PfJob*)dptr(g->doff);
  g->dev[1] = g->dev[0] + cap;
  g->host[0] = (PfJob*)pptr(g->poff);
  g->host[1] = g->host[0] + cap;
  if (r->kind == REQ_PF) {
    g->dbl = r->lg->dbl;
    g->prop = r->lg->prop;
    g->threads = r->lg->threads;
    g->split = r->lg->split;
    g->smem = r->lg->smem;
    cudaFuncSetAttribute((const void*)g->prop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g->smem);
  } else {
    g->rb = true;
    g->rk = r->rk;
    g->q_gamma = r->q_gamma;
    g->q_index = r->q_index;
    g->guided = r->guided;
  }
  groups.push_back(std::move(g));
  return groups.back().get();
}

// Uploads a particle-filter request and runs its initialisation (prior draw and
// the step-1 resample) on the particle-filter stream; it joins the running
// batch at the next chunk.
gf_status gf_srv::start_pf(Req* r) {
  cudaStream_t s = pfx.stream;
  Group* g = group_for(r);
  if (!g) return set_err(&pfx, GF_ERR_OOM_BUDGET, "no arena room for a job table");
  r->group = (int)(std::find_if(groups.begin(), groups.end(), [&](auto& x) { return x.get() == g; }) -
                   groups.begin());
  auto D = [&](size_t o) { return dptr(r->doff + o); };
  auto P = [&](size_t o) { return pptr(r->poff + o); };
  PfJob J = r->kind == REQ_PF ? r->lg->J : r->job;
  J.params = D(r->d_params);
  J.ystep = r->kind == REQ_PF ? D(r->d_ystep) : nullptr;
  J.X[0] = D(r->d_X0);
  J.X[1] = D(r->d_X1);
  J.lw = D(r->d_lw);
  J.key = (double*)D(r->d_key);
  J.part = (double*)D(r->d_part);
  J.flags = (unsigned long long*)D(r->d_flags);
  J.sc = (PfScalars*)D(r->d_sc);
  J.ocum = (int32_t*)D(r->d_ocum);
  J.mpk = (int32_t*)D(r->d_mpk);
  J.anc = (int32_t*)D(r->d_anc);
  J.tprefix = (double*)D(r->d_tpre);
  J.schedule = r->sched.empty() ? nullptr : (const int8_t*)D(r->d_sched);
  J.ys = (const double*)D(r->d_ys);
  J.ll_steps = r->out_steps ? (double*)D(r->d_steps) : nullptr;
  J.means_out = r->out_mean ? (double*)D(r->d_means) : nullptr;
  if (r->kind == REQ_PF)
    J.obs_consts = r->lg->obs_consts.empty() ? nullptr : (const double*)D(r->d_pp) + r->obs_off;
  r->job = J;
  r->job_dev = (PfJob*)D(r->d_job);
  // staging
  const size_t pbytes = r->kind == REQ_PF ? r->lg->params.size() : sizeof(float) * r->kf_params.size();
  std::memcpy(P(r->p_params), r->kind == REQ_PF ? (const void*)r->lg->params.data() : (const void*)r->kf_params.data(),
              pbytes);
  std::memcpy(P(r->p_ys), r->ys.data(), sizeof(double) * r->ys.size());
  std::memcpy(P(r->p_job), &J, sizeof J);
  double* e1 = (double*)P(r->p_e1);
  e1[0] = r->ess1;
  ((int8_t*)(e1 + 1))[0] = r->res1;
  GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_params), P(r->p_params), pbytes, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_ys), P(r->p_ys), sizeof(double) * r->ys.size(), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(r->job_dev, P(r->p_job), sizeof J, cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_ess1), e1, sizeof(double), cudaMemcpyHostToDevice, s));
  GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_res1), e1 + 1, 1, cudaMemcpyHostToDevice, s));
  if (!r->sched.empty()) {
    std::memcpy(P(r->p_sched), r->sched.data(), r->sched.size());
    GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_sched), P(r->p_sched), r->sched.size(), cudaMemcpyHostToDevice, s));
  }
  const int ntiles = J.ntiles;
  if (r->kind == REQ_PF) {
    const LgJobSetup& L = *r->lg;
    std::memcpy(P(r->p_pp), L.pp.data(), sizeof(double) * L.pp.size());
    GF_CHECK_CUDA(&pfx, cudaMemcpyAsync(D(r->d_pp), P(r->p_pp), sizeof(double) * L.pp.size(), cudaMemcpyHostToDevice, s));
    launch_prep(&pfx, L.dbl, r->job_dev, r->T, r->dx, r->dy, L.k.dxp, L.k.dyp, (const double*)D(r->d_pp),
                D(r->d_ystep));
    launch_init_scalars(&pfx, r->job_dev, 1, (const double*)D(r->d_ess1), (const int8_t*)D(r->d_res1));
    GF_CHECK_CUDA(&pfx, cudaMemsetAsync(J.flags, 0, sizeof(unsigned long long) * 2 * J.nstiles, s));
    L.k.init<<<ntiles, PF_THREADS, 0, s>>>(r->job_dev, 1, L.k.off_mu0, L.k.off_L0);
    launch_resample(&pfx, L.dbl, r->job_dev, 1, ntiles);
  } else {
    launch_init_scalars(&pfx, r->job_dev, 1, (const double*)D(r->d_ess1), (const int8_t*)D(r->d_res1));
    GF_CHECK_CUDA(&pfx, cudaMemsetAsync(J.flags, 0, sizeof(unsigned long long) * 2 * J.nstiles, s));
    r->rk.init<<<ntiles, PF_THREADS, 0, s>>>(r->job_dev, 1);
    launch_resample(&pfx, false, r->job_dev, 1, ntiles);
  }
  launches += 5;
  GF_CHECK_CUDA(&pfx, cudaGetLastError());
  g->active.push_back(r);
  ++active_pf;
  return GF_OK;
}

bool gf_srv::admit() {
  bool any = false;
  while (!pending.empty()) {
    Req* r = pending.front();
    if (round_up(r->dl.size) > darena.cap() || round_up(r->pl.size) > parena.cap()) {
      pending.pop_front();
      n_pending--;
      finish(r, set_err(&pfx, GF_ERR_OOM_BUDGET, "request %llu needs %zu device / %zu pinned bytes, more than the arenas",
                        (unsigned long long)r->id, r->dl.size, r->pl.size));
      any = true;
      continue;
    }
    const bool pf = r->kind == REQ_PF || r->kind == REQ_RBPF;
    if (pf && active_pf >= cfg.max_active_pf) break;
    if (!darena.alloc(r->dl.size, &r->doff)) break;
    if (!parena.alloc(r->pl.size, &r->poff)) {
      darena.release(r->doff, r->dl.size);
      break;
    }
    r->have_dev = r->have_pin = true;
    pending.pop_front();
    n_pending--;
    n_running++;
    r->t_admit = now_ms();
    any = true;
    if (pf) {
      gf_status st = start_pf(r);
      if (st) finish(r, st);
    } else {
      kf_ready[r->kind == REQ_KF ? 0 : 1].push_back(r);
    }
  }
  return any;
}

// An idle stream of the Kalman pool (its last launch finished), creating one
// while the pool is below its size; null when every stream is busy.  A batch
// never queues behind a running one: it waits on the host and grows instead.
cudaStream_t gf_srv::idle_kf_stream(int* idx) {
  for (size_t i = 0; i < kf_streams.size(); ++i)
    if (!kf_busy[i] && (!kf_last[i] || cudaEventQuery(kf_last[i]) == cudaSuccess)) {
      *idx = (int)i;
      return kf_streams[i];
    }
  if ((int)kf_streams.size() < cfg.kf_streams) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    kf_streams.push_back(s);
    kf_last.push_back(nullptr);
    kf_busy.push_back(0);
    *idx = (int)kf_streams.size() - 1;
    return s;
  }
  return nullptr;
}

// Forms one batch per Kalman algorithm from the requests admitted since the
// last call: uploads their inputs and descriptors, then one persistent launch
// per dimension bucket on idle streams.
bool gf_srv::launch_kf() {
  bool any = false;
  for (int a = 0; a < 2; ++a) {
   while (!kf_ready[a].empty()) {
    // one batch per jitter setting: jitter is a launch argument
    std::vector<Req*> ready, rest;
    for (Req* r : kf_ready[a]) {
      const Req* h = kf_ready[a][0];
      (r->use_jitter == h->use_jitter && (!r->use_jitter || r->jitter == h->jitter) ? ready : rest).push_back(r);
    }
    const int algo = a == 0 ? GF_ALGO_KF : GF_ALGO_SRKF;
    const int B = (int)ready.size();
    const int nb = kf_bucket_count();
    // one idle stream per non-empty dimension bucket, or wait and coalesce
    std::vector<int> bstream(nb, -1);
    bool have = true;
    for (Req* r : ready) {
      const int k = kf_bucket_for(r->dx, r->dy);
      if (bstream[k] >= 0) continue;
      int idx = -1;
      if (!idle_kf_stream(&idx)) {
        have = false;
        break;
      }
      bstream[k] = idx;
      kf_busy[idx] = 1;
    }
    for (int k = 0; k < nb; ++k)
      if (bstream[k] >= 0) kf_busy[bstream[k]] = 0;
    if (!have) return any;
    auto bt = std::make_unique<KfBatch>();
    Layout dl, pl;
    const size_t d_desc = dl.take(sizeof(KfDesc) * B), d_order = dl.take(sizeof(int32_t) * B),
                 d_cnt = dl.take(sizeof(uint32_t) * nb);
    const size_t p_desc = pl.take(sizeof(KfDesc) * B), p_order = pl.take(sizeof(int32_t) * B);
    bt->dbytes = dl.size;
    bt->pbytes = pl.size;
    if (!darena.alloc(dl.size, &bt->doff)) return any;
    if (!parena.alloc(pl.size, &bt->poff)) {
      darena.release(bt->doff, dl.size);
      return any;
    }
    kf_ready[a].swap(rest);
    KfDesc* hd = (KfDesc*)pptr(bt->poff + p_desc);
    int32_t* ho = (int32_t*)pptr(bt->poff + p_order);
    std::vector<std::vector<int32_t>> members(nb);
    for (int i = 0; i < B; ++i) {
      Req* r = ready[i];
      KfDesc& d = hd[i];
      std::memset(&d, 0, sizeof d);
      d.dx = r->dx;
      d.dy = r->dy;
      d.T = r->T;
      d.poff = (int64_t)((r->doff + r->d_params) / sizeof(float));
      d.yoff = (int64_t)((r->doff + r->d_ys) / sizeof(double));
      d.index = i;
      d.srv = (KfSrvRec*)pdptr(r->poff + r->p_rec);
      d.srv_mu = (float*)pdptr(r->poff + r->p_mu);
      d.srv_cov = (float*)pdptr(r->poff + r->p_cov);
      d.srv_steps = r->out_steps ? (double*)pdptr(r->poff + r->p_steps) : nullptr;
      KfSrvRec* rec = (KfSrvRec*)pptr(r->poff + r->p_rec);
      rec->ll = 0.0;
      rec->status = 0;
      rec->done = 0;
      std::memcpy(pptr(r->poff + r->p_params), r->kf_params.data(), sizeof(float) * r->kf_params.size());
      std::memcpy(pptr(r->poff + r->p_ys), r->ys.data(), sizeof(double) * r->ys.size());
      members[kf_bucket_for(r->dx, r->dy)].push_back(i);
    }
    int n = 0;
    std::vector<std::pair<int, int>> ranges(nb);
    for (int k = 0; k < nb; ++k) {
      auto& mem = members[k];
      std::stable_sort(mem.begin(), mem.end(), [&](int x, int y) {
        const KfDesc &u = hd[x], &v = hd[y];
        return (double)u.T * u.dx * u.dx * (u.dx + u.dy) > (double)v.T * v.dx * v.dx * (v.dx + v.dy);
      });
      ranges[k] = {n, (int)mem.size()};
      for (int f : mem) ho[n++] = f;
    }
    int si = -1;
    for (int k = 0; k < nb && si < 0; ++k) si = bstream[k];
    cudaStream_t up = kf_streams[si];
    cudaError_t e = cudaSuccess;
    for (Req* r : ready) {
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dptr(r->doff + r->d_params), pptr(r->poff + r->p_params),
                            sizeof(float) * r->kf_params.size(), cudaMemcpyHostToDevice, up);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dptr(r->doff + r->d_ys), pptr(r->poff + r->p_ys), sizeof(double) * r->ys.size(),
                            cudaMemcpyHostToDevice, up);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dptr(bt->doff + d_desc), hd, sizeof(KfDesc) * B, cudaMemcpyHostToDevice, up);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dptr(bt->doff + d_order), ho, sizeof(int32_t) * B, cudaMemcpyHostToDevice, up);
    if (e == cudaSuccess) e = cudaMemsetAsync(dptr(bt->doff + d_cnt), 0, sizeof(uint32_t) * nb, up);
    cudaEvent_t uploaded = take_ev();
    if (e == cudaSuccess) e = cudaEventRecord(uploaded, up);
    KfRun run{};
    run.desc = (const KfDesc*)dptr(bt->doff + d_desc);
    run.params = (const float*)dbase;
    run.ys = (const double*)dbase;
    run.jitter = ready[0]->jitter;
    run.use_jitter = ready[0]->use_jitter;
    run.algo = algo;
    for (int k = 0; k < nb && e == cudaSuccess; ++k) {
      if (ranges[k].second == 0) continue;
      const int idx = bstream[k];
      cudaStream_t s = kf_streams[idx];
      if (idx != si) e = cudaStreamWaitEvent(s, uploaded, 0);
      KfRun rk = run;
      rk.order = (const int32_t*)dptr(bt->doff + d_order) + ranges[k].first;
      rk.count = ranges[k].second;
      rk.counter = (uint32_t*)dptr(bt->doff + d_cnt) + k;
      const int group = kf_default_group(k);
      int& per_sm = kf_per_sm[a][k];
      if (per_sm == 0) per_sm = kf_blocks_per_sm(algo, k, group);
      const int grid = std::max(1, std::min(rk.count, per_sm * num_sms));
      kf_launch(algo, k, group, grid, rk, s);
      e = cudaGetLastError();
      cudaEvent_t done = take_ev();
      if (e == cudaSuccess) e = cudaEventRecord(done, s);
      bt->evs.push_back(done);
      kf_last[idx] = done;
      ++launches;
    }
    give_ev(uploaded);  // re-recording a pooled event later is ordered after its waits
    for (Req* r : ready) {
      if (e != cudaSuccess) {
        finish(r, cuda_err(&pfx, e, "serving Kalman batch launch"));
        continue;
      }
      kf_running.push_back(r);
    }
    for (Req* r : ready) r->group = -1;
    bt->reqs = ready;
    batches.push_back(std::move(bt));
    ++kf_batches;
    any = true;
   }
  }
  return any;
}

// One chunk of steps for every running particle-filter job.
bool gf_srv::pf_iterate() {
  while (!chunk_evs.empty() && cudaEventQuery(chunk_evs.front()) == cudaSuccess) {
    give_ev(chunk_evs.front());
    chunk_evs.pop_front();
  }
  if (chunk_evs.size() >= 2) return false;
  bool any = false;
  for (auto& g : groups) any = any || !g->active.empty();
  if (!any) return false;
  cudaStream_t s = pfx.stream;
  const int slot = (int)(chunk_no & 1);
  for (auto& gp : groups) {
    Group& g = *gp;
    if (g.active.empty()) continue;
    int steps = 0, tiles = 0;
    const int nj = (int)g.active.size();
    for (int i = 0; i < nj; ++i) {
      Req* r = g.active[i];
      steps = std::max(steps, std::min(cfg.pf_chunk, r->T - r->launched));
      PfJob J = r->job;
      J.tile0 = tiles;
      tiles += J.ntiles;
      g.host[slot][i] = J;
    }
    cudaMemcpyAsync(g.dev[slot], g.host[slot], sizeof(PfJob) * nj, cudaMemcpyHostToDevice, s);
    for (int k = 0; k < steps; ++k) {
      if (g.rb) g.rk.prop<<<tiles * RB_SPLIT, RB_THREADS, 0, s>>>(g.dev[slot], nj, g.q_gamma, g.q_index, g.guided);
      else g.prop<<<tiles * g.split, g.threads, g.smem, s>>>(g.dev[slot], nj);
      launch_resample(&pfx, g.dbl, g.dev[slot], nj, tiles);
      launches += 3;
    }
    std::vector<Req*> keep;
    for (Req* r : g.active) {
      r->launched = std::min(r->T, r->launched + steps);
      if (r->launched < r->T) {
        keep.push_back(r);
        continue;
      }
      // results: final weighted mean, scalars and per-step ll to pinned memory
      const int ntiles = r->job.ntiles;
      if (r->out_mean) {
        launch_means(&pfx, g.dbl, r->job_dev, 1, ntiles, (double*)dptr(r->doff + r->d_mpart), r->mdim);
        ++launches;
        cudaMemcpyAsync(pptr(r->poff + r->p_mean), dptr(r->doff + r->d_means + sizeof(double) * (size_t)(r->T - 1) * r->mdim),
                        sizeof(double) * r->mdim, cudaMemcpyDeviceToHost, s);
      }
      cudaMemcpyAsync(pptr(r->poff + r->p_sc), dptr(r->doff + r->d_sc), sizeof(PfScalars), cudaMemcpyDeviceToHost, s);
      if (r->out_steps)
        cudaMemcpyAsync(pptr(r->poff + r->p_steps), dptr(r->doff + r->d_steps), sizeof(double) * r->T,
                        cudaMemcpyDeviceToHost, s);
      r->ev = take_ev();
      cudaEventRecord(r->ev, s);
      pf_finishing.push_back(r);
      --active_pf;
    }
    g.active.swap(keep);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) werr = std::string("particle-filter chunk: ") + cudaGetErrorString(e);
  cudaEvent_t ce = take_ev();
  cudaEventRecord(ce, s);
  chunk_evs.push_back(ce);
  ++chunk_no;
  ++pf_iters;
  return true;
}

void gf_srv::release(Req* r) {
  if (r->have_dev) darena.release(r->doff, r->dl.size);
  if (r->have_pin) parena.release(r->poff, r->pl.size);
  r->have_dev = r->have_pin = false;
  if (r->ev) {
    give_ev(r->ev);
    r->ev = nullptr;
  }
}

// Delivers a request's result (status st) and frees its blocks.
void gf_srv::finish(Req* r, gf_status st) {
  r->t_done = now_ms();
  r->status = st;
  const bool ran = r->t_admit > 0;
  release(r);
  gf_srv_result res{};
  res.id = r->id;
  res.tag = r->tag;
  res.status = st;
  res.kind = r->kind;
  res.ll = r->ll;
  res.submit_ms = r->t_submit - t0;
  res.start_ms = ran ? r->t_admit - t0 : -1.0;
  res.done_ms = r->t_done - t0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (ran) n_running--;
    if (st == GF_OK) {
      ++n_completed;
      lat.push_back(r->t_done - r->t_submit);
      if (r->kind == REQ_KF || r->kind == REQ_SRKF) kf_steps += r->T;
      else particle_steps += (double)r->N * r->T;
    } else if (st == GF_ERR_OOM_BUDGET && !ran) {
      ++n_rejected;
    } else {
      ++n_failed;
      if (!pfx.err.empty()) err = pfx.err;
    }
    t_last = r->t_done;
    outbox.push_back(res);
  }
  cv_done.notify_all();
  delete r;
}

bool gf_srv::reap() {
  bool any = false;
  // Kalman filters: host-mapped done flags
  std::vector<Req*> still;
  for (Req* r : kf_running) {
    KfSrvRec* rec = (KfSrvRec*)pptr(r->poff + r->p_rec);
    if (rec->done == 0) {
      still.push_back(r);
      continue;
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    r->ll = rec->ll;
    gf_status st = rec->status;
    const float* m = (const float*)pptr(r->poff + r->p_mu);
    const float* c = (const float*)pptr(r->poff + r->p_cov);
    if (r->out_mean)
      for (int i = 0; i < r->dx; ++i) r->out_mean[i] = m[i];
    if (r->out_cov)
      for (int i = 0; i < r->dx * r->dx; ++i) r->out_cov[i] = c[i];
    if (r->out_steps) std::memcpy(r->out_steps, pptr(r->poff + r->p_steps), sizeof(double) * r->T);
    if (st == GF_ERR_NOT_PD) set_err(&pfx, st, "request %llu: innovation covariance not positive definite",
                                     (unsigned long long)r->id);
    finish(r, st);
    any = true;
  }
  kf_running.swap(still);
  // Kalman batches: descriptor blocks are freed once every launch is done
  for (size_t i = 0; i < batches.size();) {
    KfBatch& b = *batches[i];
    bool done = true;
    for (cudaEvent_t e : b.evs) done = done && cudaEventQuery(e) == cudaSuccess;
    if (!done) {
      ++i;
      continue;
    }
    for (cudaEvent_t e : b.evs) {
      for (auto& l : kf_last)
        if (l == e) l = nullptr;
      give_ev(e);
    }
    darena.release(b.doff, b.dbytes);
    parena.release(b.poff, b.pbytes);
    batches.erase(batches.begin() + i);
    any = true;
  }
  // particle filters: result copies
  std::vector<Req*> fin;
  for (Req* r : pf_finishing) {
    cudaError_t q = cudaEventQuery(r->ev);
    if (q == cudaErrorNotReady) {
      fin.push_back(r);
      continue;
    }
    gf_status st = GF_OK;
    if (q != cudaSuccess) {
      st = cuda_err(&pfx, q, "particle-filter request");
    } else {
      const PfScalars* sc = (const PfScalars*)pptr(r->poff + r->p_sc);
      r->ll = sc->ll;
      st = sc->status;
      if (st == GF_ERR_TIMEOUT) set_err(&pfx, st, "request %llu: bounded device wait gave up", (unsigned long long)r->id);
      else if (st) set_err(&pfx, st, "request %llu: weights degenerated at step %d", (unsigned long long)r->id, sc->t + 1);
      if (r->out_steps) std::memcpy(r->out_steps, pptr(r->poff + r->p_steps), sizeof(double) * r->T);
      if (r->out_mean) std::memcpy(r->out_mean, pptr(r->poff + r->p_mean), sizeof(double) * r->mdim);
    }
    finish(r, st);
    any = true;
  }
  pf_finishing.swap(fin);
  return any;
}

void gf_srv::loop() {
  cudaSetDevice(device);
  while (true) {
    bool quit = false;
    {
      std::lock_guard<std::mutex> lk(mu);
      while (!inbox.empty()) {
        pending.push_back(inbox.front());
        inbox.pop_front();
      }
      quit = stop;
    }
    if (quit) {
      // cancel what was never admitted; let the running requests finish
      while (!pending.empty()) {
        Req* r = pending.front();
        pending.pop_front();
        n_pending--;
        finish(r, set_err(&pfx, GF_ERR_BUSY, "server stopped before admission"));
      }
      for (int a = 0; a < 2; ++a) {
        for (Req* r : kf_ready[a]) finish(r, set_err(&pfx, GF_ERR_BUSY, "server stopped before launch"));
        kf_ready[a].clear();
      }
    }
    bool busy = admit();
    busy = launch_kf() || busy;
    busy = pf_iterate() || busy;
    busy = reap() || busy;
    hbm_used = darena.used();
    hbm_peak = darena.peak();
    const bool running = !kf_running.empty() || !batches.empty() || !pf_finishing.empty() || active_pf > 0 ||
                         !chunk_evs.empty();
    if (quit && !running && pending.empty()) break;
    if (!busy) {
      std::unique_lock<std::mutex> lk(mu);
      if (inbox.empty() && !stop) {
        if (running) cv_work.wait_for(lk, std::chrono::microseconds(20));
        else cv_work.wait_for(lk, std::chrono::milliseconds(5));
      }
    }
  }
}

// --------------------------------------------------------------- C ABI
extern "C" {

gf_status gf_srv_create(const gf_srv_config* cfg_in, gf_srv** out) {
  if (!out) return GF_ERR_ARG;
  *out = nullptr;
  auto s = std::make_unique<gf_srv>();
  if (cfg_in) s->cfg = *cfg_in;
  gf_srv_config& c = s->cfg;
  if (c.max_pending <= 0) c.max_pending = 65536;
  if (c.pf_chunk <= 0) c.pf_chunk = 16;
  if (c.kf_streams <= 0) c.kf_streams = 64;
  if (c.max_active_pf <= 0) c.max_active_pf = 4096;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || c.device < 0 || c.device >= n) return GF_ERR_CUDA;
  s->device = c.device;
  if (cudaSetDevice(c.device) != cudaSuccess) return GF_ERR_CUDA;
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, c.device);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  if (c.hbm_budget_bytes == 0) c.hbm_budget_bytes = fr / 2;
  if (c.host_budget_bytes == 0) c.host_budget_bytes = (size_t)1 << 30;
  c.hbm_budget_bytes = c.hbm_budget_bytes / kAlign * kAlign;
  c.host_budget_bytes = c.host_budget_bytes / kAlign * kAlign;
  if (cudaMalloc((void**)&s->dbase, c.hbm_budget_bytes) != cudaSuccess) return GF_ERR_OOM_BUDGET;
  if (cudaHostAlloc((void**)&s->pbase, c.host_budget_bytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
    cudaFree(s->dbase);
    return GF_ERR_OOM_BUDGET;
  }
  cudaHostGetDevicePointer((void**)&s->pdev, s->pbase, 0);
  s->darena.reset(c.hbm_budget_bytes);
  s->parena.reset(c.host_budget_bytes);
  s->pfx.device = c.device;
  s->pfx.num_sms = s->num_sms;
  cudaStreamCreateWithFlags(&s->pfx.stream, cudaStreamNonBlocking);
  s->pfx.own_stream = true;
  s->pfx.budget = c.hbm_budget_bytes;
  for (int k = 0; k < kf_bucket_count(); ++k) {
    if (kf_prepare_bucket(&s->pfx, GF_ALGO_KF, k) || kf_prepare_bucket(&s->pfx, GF_ALGO_SRKF, k)) {
      cudaFree(s->dbase);
      cudaFreeHost(s->pbase);
      return GF_ERR_CUDA;
    }
  }
  s->t0 = now_ms();
  gf_srv* raw = s.release();
  raw->worker = std::thread([raw] { raw->loop(); });
  *out = raw;
  return GF_OK;
}

gf_status gf_srv_submit(gf_srv* s, const gf_srv_request* q, uint64_t* id) {
  if (!s) return GF_ERR_ARG;
  auto r = std::make_unique<Req>();
  gf_ctx ectx;
  gf_status st = prepare(&ectx, q, r.get());
  std::lock_guard<std::mutex> lk(s->mu);
  if (st) {
    s->err = ectx.err;
    return st;
  }
  if (s->stop) {
    s->err = "server is stopping";
    return GF_ERR_BUSY;
  }
  if (s->n_pending.load() >= s->cfg.max_pending) {
    s->err = "pending queue full";
    return GF_ERR_BUSY;
  }
  r->id = s->next_id++;
  r->t_submit = now_ms();
  if (s->t_first < 0) s->t_first = r->t_submit;
  if (id) *id = r->id;
  ++s->n_submitted;
  s->n_pending++;
  s->inbox.push_back(r.release());
  s->cv_work.notify_one();
  return GF_OK;
}

int32_t gf_srv_poll(gf_srv* s, gf_srv_result* out, int32_t max, int32_t wait_ms) {
  if (!s || !out || max < 1) return 0;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->outbox.empty() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->outbox.empty(); });
  int32_t n = 0;
  while (n < max && !s->outbox.empty()) {
    out[n++] = s->outbox.front();
    s->outbox.pop_front();
  }
  return n;
}

gf_status gf_srv_drain(gf_srv* s, int32_t timeout_ms) {
  if (!s) return GF_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto all_done = [&] { return s->n_completed + s->n_failed + s->n_rejected >= s->n_submitted; };
  if (timeout_ms < 0) s->cv_done.wait(lk, all_done);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), all_done)) return GF_ERR_TIMEOUT;
  return GF_OK;
}

gf_status gf_srv_stats(gf_srv* s, gf_srv_metrics* m) {
  if (!s || !m) return GF_ERR_ARG;
  std::memset(m, 0, sizeof *m);
  std::vector<double> l;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    m->submitted = s->n_submitted;
    m->completed = s->n_completed;
    m->failed = s->n_failed;
    m->rejected = s->n_rejected;
    m->kf_steps = s->kf_steps;
    m->particle_steps = s->particle_steps;
    m->elapsed_ms = s->t_first < 0 ? 0.0 : s->t_last - s->t_first;
    l = s->lat;
  }
  m->pending = s->n_pending.load();
  m->running = s->n_running.load();
  m->hbm_budget = s->cfg.hbm_budget_bytes;
  m->hbm_used = s->hbm_used.load();
  m->hbm_peak = s->hbm_peak.load();
  m->pf_iterations = s->pf_iters.load();
  m->kf_batches = s->kf_batches.load();
  m->launches = s->launches.load();
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double p) {
      size_t i = (size_t)std::min<double>((double)l.size() - 1, std::ceil(p * l.size()) - 1);
      return l[i];
    };
    m->p50_ms = q(0.50);
    m->p99_ms = q(0.99);
    m->max_ms = l.back();
    double sum = 0;
    for (double v : l) sum += v;
    m->mean_ms = sum / l.size();
  }
  return GF_OK;
}

gf_status gf_srv_reset_stats(gf_srv* s) {
  if (!s) return GF_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat.clear();
  s->kf_steps = s->particle_steps = 0;
  s->t_first = -1;
  s->n_submitted -= s->n_completed + s->n_failed + s->n_rejected;
  s->n_completed = s->n_failed = s->n_rejected = 0;
  return GF_OK;
}

const char* gf_srv_last_error(gf_srv* s) {
  if (!s) return "null server";
  std::lock_guard<std::mutex> lk(s->mu);
  return s->err.c_str();
}

gf_status gf_srv_destroy(gf_srv* s) {
  if (!s) return GF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->pfx.stream);
  for (auto st : s->kf_streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  cudaStreamDestroy(s->pfx.stream);
  for (auto e : s->ev_pool) cudaEventDestroy(e);
  for (auto e : s->chunk_evs) cudaEventDestroy(e);
  cudaFree(s->dbase);
  cudaFreeHost(s->pbase);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (Req* r : s->inbox) delete r;
    s->inbox.clear();
  }
  delete s;
  return GF_OK;
}

}  // extern "C"
