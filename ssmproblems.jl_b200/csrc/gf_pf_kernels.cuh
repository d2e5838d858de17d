// gf_pf_kernels.cuh -- particle-filter device code shared by the LG and RBPF paths.
//
// One filtering step of GeneralisedFilters' particle filter (particles.jl:147-162)
// is two launches:
//   1. propagate  : [ancestor search + gather if resampling] -> propagate ->
//                   weight -> per-block (max, sum exp, sum exp^2) partials ->
//                   the last block folds them into the job scalars
//                   (LSE, ll increment, ESS and the next resample decision).
//   2. lookback scan (only when the next step resamples): cumulative
//                   normalised weights, summed exactly in 64-bit fixed point.
// Several independent jobs (filters) can share one launch: blocks map to jobs
// through each job's first tile index.
#pragma once
#include "gf_common.cuh"

namespace gf {

constexpr int PF_THREADS = 256;
constexpr int PF_PPT = 4;                      // particles per thread
constexpr int PF_TILE = PF_THREADS * PF_PPT;   // particles per propagate block
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_IPT = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;
constexpr int PF_PW = 3;                       // doubles per block partial (M, S1, S2)
constexpr int PF_MAX_SPLIT = 8;                // largest number of partials per tile (sizes `part`)
constexpr int FILL_D = 2 * PF_TILE;            // merge items (particles + slots) per fill block
constexpr int FILL_IPT = FILL_D / PF_THREADS;  // merge items per fill thread
constexpr unsigned long long kReady = 1ull << 63;
constexpr double kFix = 4611686018427387904.0; // 2^62
constexpr double kInvFix = 1.0 / 4611686018427387904.0;
constexpr long long kSpinLimit = 1ll << 20;    // bounded lookback wait (~1 s)

struct PfJob {
  int64_t N;
  int32_t dx, dy, T, width;
  int32_t tile0, ntiles, stile0, nstiles;
  int32_t resampler, conv, prop, diag_l;  // diag_l: proposal noise factor is diagonal
  double threshold, log_n, obs_const, prop_const;
  uint64_t seed;
  const void* params;        // model parameters in the run's precision
  const void* ystep;         // per-step vectors [T][ystride]
  int32_t ystride;
  int32_t lookahead_draw;    // auxiliary filter: DrawPredictive (x* drawn from the transition)
  // time-varying model: step t's parameter block is params + (t-1) * pstride
  // elements, its observation and proposal constants obs_consts[2(t-1)] and
  // obs_consts[2(t-1) + 1]; the observation prep reads its factors
  // pp + t * ppstride (0 / null: one block for all steps)
  int64_t pstride;
  const double* obs_consts;
  int32_t ppstride;
  int32_t pad_tv;
  void* X[2];                // SoA state ping-pong [width][N]
  void* lw;                  // stored log-weights [N]
  double* key;               // cumulative normalised weights [N]
  double* part;              // [PF_PW][ntiles * PF_MAX_SPLIT] partial fields, one array each
  unsigned long long* flags; // [2][nstiles] lookback aggregate / inclusive prefix
  PfScalars* sc;
  const void* noise;         // nullable [(T+1)][nz][N]
  const double* unif;        // nullable
  const int8_t* schedule;    // nullable [T]
  double* ll_steps;          // nullable [T]
  double* ess_steps;         // nullable [T]
  int8_t* res_steps;         // nullable [T]
  int32_t* anc_out;          // nullable [T][N]
  const double* ys;          // observations [T][dy] (device)
  double* ll_out;            // nullable [1]
  double* logw_out;          // nullable [N] final normalised log-weights
  void* states_out;          // nullable [width][N] final states
  int32_t* clamps_out;       // nullable [1]
  double* means_out;         // nullable [T][mdim]
  const double* wraw;        // nullable: scan raw weights wraw[k] / sc->wtotal instead of exp(lw - LSE)
  double* tprefix;           // [ntiles + 1] cumulative normalised weight at each tile start
  int32_t* ocum;             // [N] cumulative offspring counts of the pending resample
  int32_t* mpk;              // [ntiles + 1] merge-path start particle of each fill block
  int32_t* anc;              // [N] 0-based ancestors of the pending resample
  void* eta;                 // auxiliary filter: [N] lookahead log eta of the current particles (else null)
  void* hist;                // nullable [T+1][dx][N] dense state history
  double* lwh;               // nullable [T][N] normalised log-weight history
};

// Observation constant of step t (time-varying models carry one per step).
__device__ __forceinline__ double step_obs_const(const PfJob& J, int t) {
  return J.obs_consts ? J.obs_consts[2 * (t - 1)] : J.obs_const;
}
// log-normaliser difference of a guided proposal at step t (proposal vs transition)
__device__ __forceinline__ double step_prop_const(const PfJob& J, int t) {
  return J.obs_consts ? J.obs_consts[2 * (t - 1) + 1] : J.prop_const;
}

__device__ __forceinline__ int find_job(const PfJob* jobs, int njobs, int block, bool scan) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    int t0 = scan ? jobs[mid].stile0 : jobs[mid].tile0;
    if (t0 <= block) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Per-slot uniform of step t: injected [T][N] or Philox(seed; j, t).
__device__ __forceinline__ double slot_uniform(const PfJob& J, int64_t j, int t) {
  return J.unif ? J.unif[(size_t)(t - 1) * J.N + j] : philox_uniform(J.seed, (uint32_t)j, (uint32_t)t);
}

// Monotone predicate "particle k is at or past slot j's ancestor"; the
// ancestor of slot j is the first k where it holds.
//  CPU convention (resamplers.jl:220-235): n*W_k > u0 + j  |  n*W_k > j + U_j
//  multinomial (CUDAExt.jl:34-37):         W_k >= U_j * W_n
//  CUDAExt systematic  (CUDAExt.jl:52-57): floor(n*W_k/W_n + u0) >= j + 1
//  CUDAExt stratified  (CUDAExt.jl:71-76): floor(r_k + U[min(n, floor(r_k+1))]) >= j + 1
struct SlotSearch {
  const double* key;
  int64_t n;
  double dn, wn, thr;
  int kind, conv, t;
  int64_t j;
  const PfJob* J;
  __device__ __forceinline__ bool pred(int64_t k) const {
    double W = __ldg(key + k);
    if (kind == GF_RS_MULTINOMIAL) return W >= thr;
    if (conv == GF_CONV_CPU) return dn * W > thr;
    double r = (dn * W) / wn;
    double u;
    if (kind == GF_RS_SYSTEMATIC) {
      u = thr;
    } else {
      double kk = floor(r + 1.0);
      int64_t ki = kk < dn ? (int64_t)kk : n;
      u = slot_uniform(*J, ki - 1, t);
    }
    return floor(r + u) >= (double)(j + 1);
  }
  // first k in [lo, hi) with pred(k); hi if none
  __device__ __forceinline__ int64_t first(int64_t lo, int64_t hi) const {
    while (lo < hi) {
      int64_t mid = lo + ((hi - lo) >> 1);
      if (pred(mid)) hi = mid;
      else lo = mid + 1;
    }
    return lo;
  }
};

__device__ __forceinline__ SlotSearch make_search(const PfJob& J, const PfScalars* sc, int t,
                                                  int64_t j) {
  SlotSearch s;
  s.key = J.key;
  s.n = J.N;
  s.dn = (double)J.N;
  s.wn = sc->wn;
  s.kind = J.resampler;
  s.conv = J.conv;
  s.t = t;
  s.j = j;
  s.J = &J;
  if (J.resampler == GF_RS_MULTINOMIAL) s.thr = slot_uniform(J, j, t) * s.wn;
  else if (J.resampler == GF_RS_SYSTEMATIC) s.thr = J.conv == GF_CONV_CPU ? sc->u0 + (double)j : sc->u0;
  else s.thr = J.conv == GF_CONV_CPU ? (double)j + slot_uniform(J, j, t) : 0.0;
  return s;
}

// Ancestor (0-based) of slot j within [lo, hi); counts clamps.
__device__ __forceinline__ int64_t find_ancestor(const PfJob& J, PfScalars* sc, int t, int64_t j,
                                                 int64_t lo, int64_t hi) {
  SlotSearch s = make_search(J, sc, t, j);
  int64_t a = s.first(lo, hi);
  if (a >= J.N) {
    a = J.N - 1;
    atomicAdd(&sc->clamps, 1);
  }
  return a;
}

// Offspring count: the number of slots j in [0, N) assigned to particles whose
// cumulative normalised weight is <= W, i.e. O_k for W = W_k.  Exact and O(1):
//  CPU rule (resamplers.jl:220-235) with thresholds t_j = u0 + j (systematic)
//  or j + U_j (stratified), both in [j, j+1]: every j < floor(n W) - 1 counts,
//  the two candidates at floor(n W) - 1 and floor(n W) are compared exactly.
//  CUDAExt rule (CUDAExt.jl:55-57,74-76): O = min(n, floor(n W / W_n + u)).
// The rule's inputs are copied into registers once per block.
struct OffspringRule {
  int64_t N;
  double dn, u0, wn;
  const double* unif;  // injected uniforms of this step (nullable)
  uint64_t seed;
  int kind, conv, t;
  __device__ __forceinline__ double uniform(int64_t j) const {
    return unif ? unif[j] : philox_uniform(seed, (uint32_t)j, (uint32_t)t);
  }
  __device__ __forceinline__ int64_t count(double W) const {
    if (conv == GF_CONV_CPU) {
      const double vs = dn * W;
      const double f = floor(vs) - 1.0;
      const int64_t g = f <= 0.0 ? 0 : (f >= dn ? N : (int64_t)f);
      int64_t cnt = g;
      for (int64_t j = g; j <= g + 1 && j < N; ++j) {
        const double thr = kind == GF_RS_SYSTEMATIC ? u0 + (double)j : (double)j + uniform(j);
        if (thr < vs) cnt = j + 1;
      }
      return cnt;
    }
    const double r = (dn * W) / wn;
    double u;
    if (kind == GF_RS_SYSTEMATIC) {
      u = u0;
    } else {
      const double kk = floor(r + 1.0);
      const int64_t ki = kk < dn ? (kk < 1.0 ? 1 : (int64_t)kk) : N;
      u = uniform(ki - 1);
    }
    const double f = floor(r + u);
    return f < dn ? (f < 0.0 ? 0 : (int64_t)f) : N;
  }
};

__device__ __forceinline__ OffspringRule make_rule(const PfJob& J, const PfScalars* sc, int t) {
  OffspringRule R;
  R.N = J.N;
  R.dn = (double)J.N;
  R.u0 = sc->u0;
  R.wn = sc->wn;
  R.unif = (J.unif && J.resampler != GF_RS_SYSTEMATIC) ? J.unif + (size_t)(t - 1) * J.N : nullptr;
  R.seed = J.seed;
  R.kind = J.resampler;
  R.conv = J.conv;
  R.t = t;
  return R;
}


// Exclusive scan of unsigned 64-bit values over the threads of S (exact,
// associative); returns the exclusive prefix of this thread's value, *total
// gets the sum.  `sh` holds >= 32 values owned by S.
template <class S>
__device__ __forceinline__ unsigned long long sync_excl_scan_u64(const S& g, unsigned long long v,
                                                                 unsigned long long* sh,
                                                                 unsigned long long* total) {
  const int lane = g.tid() & 31, wid = g.tid() >> 5, nw = g.size() >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  g.sync();
  if (lane == 31) sh[wid] = x;
  g.sync();
  unsigned long long pre = 0ull, tot = 0ull;
  for (int w = 0; w < nw; ++w) {
    const unsigned long long tw = sh[w];
    if (w < wid) pre += tw;
    tot += tw;
  }
  *total = tot;
  return pre + x - v;
}
__device__ __forceinline__ unsigned long long block_excl_scan_u64(unsigned long long v,
                                                                  unsigned long long* sh,
                                                                  unsigned long long* total) {
  return sync_excl_scan_u64(BlockSync(), v, sh, total);
}

// Per-thread online accumulation of (max, sum exp, sum exp^2) in FP64.
struct LseAcc {
  double m = -INFINITY, s1 = 0.0, s2 = 0.0;
  __device__ __forceinline__ void add(double v) {
    if (!(v > -INFINITY)) return;
    if (v > m) {
      double f = exp(m - v);
      s1 = s1 * f + 1.0;
      s2 = s2 * f * f + 1.0;
      m = v;
    } else {
      double w = exp(v - m);
      s1 += w;
      s2 += w * w;
    }
  }
};

// The block partials are kept field by field (structure of arrays): M, S1
// and S2 of partial b at part[f * part_stride(J) + b], so the last block's
// reads of one field are contiguous across its threads.
__host__ __device__ __forceinline__ size_t part_stride(const PfJob& J) {
  return (size_t)J.ntiles * PF_MAX_SPLIT;
}

// Folds the block's accumulators into partial tile * nparts + part; true in
// the job's last block to arrive (which then folds every partial).
static __device__ bool fold_partials(const PfJob& J, int tile, LseAcc a, double* red, int part,
                                     int nparts) {
  PfScalars* sc = J.sc;
  __shared__ int s_last;
  const int nall = J.ntiles * nparts;
  double M = block_max(a.m, red);
  double f = a.m > -INFINITY ? exp(a.m - M) : 0.0;
  double S1 = block_sum(a.s1 * f, red);
  double S2 = block_sum(a.s2 * f * f, red);
  if (threadIdx.x == 0) {
    const size_t ps = part_stride(J);
    double* p = J.part + (size_t)tile * nparts + part;
    p[0] = M;
    p[ps] = S1;
    p[2 * ps] = S2;
    __threadfence();
    unsigned prev = atomicAdd(&sc->counter, 1u);
    s_last = (prev == (unsigned)(nall - 1));
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  return true;
}

// Last block: (max, sum e, sum e^2) over every partial, in a fixed order.
// ecache (nullable, shared, nall entries): keeps exp(M_b - GM) of every
// partial for write_tile_prefixes.
template <class S>
static __device__ void global_stats(const S& g, const PfJob& J, int nparts, double* red,
                                    double* GM_out, double* GS1_out, double* GS2_out,
                                    double* ecache = nullptr) {
  // job fields are read once: a store through ecache (or any pointer) may
  // alias the job table, and every later J.x would be another L2 round trip
  const int nall = J.ntiles * nparts;
  const size_t ps = part_stride(J);
  const double* __restrict__ part = J.part;
  // each thread's partials are read in batches of independent loads (one L2
  // round trip per batch, not per partial); the per-thread order of the sums
  // is the partial order, as in an unbatched loop
  const int G = g.size();
  constexpr int kMaxB = 8, kSumB = 4;
  double m = -INFINITY;
  for (int b0 = g.tid(); b0 < nall; b0 += kMaxB * G) {
    double v[kMaxB];
#pragma unroll
    for (int k = 0; k < kMaxB; ++k) v[k] = b0 + k * G < nall ? __ldcg(part + b0 + k * G) : -INFINITY;
#pragma unroll
    for (int k = 0; k < kMaxB; ++k) m = fmax(m, v[k]);
  }
  double GM = sync_max(g, m, red);
  double s1 = 0.0, s2 = 0.0;
  for (int b0 = g.tid(); b0 < nall; b0 += kSumB * G) {
    double mb[kSumB], p1[kSumB], p2[kSumB];
#pragma unroll
    for (int k = 0; k < kSumB; ++k) {
      const int bb = b0 + k * G;
      const double* p = part + (bb < nall ? bb : 0);
      mb[k] = bb < nall ? __ldcg(p) : -INFINITY;
      p1[k] = __ldcg(p + ps);
      p2[k] = __ldcg(p + 2 * ps);
    }
#pragma unroll
    for (int k = 0; k < kSumB; ++k) {
      const int bb = b0 + k * G;
      double ff = 0.0;
      if (mb[k] > -INFINITY) {
        ff = exp(mb[k] - GM);
        s1 += p1[k] * ff;
        s2 += p2[k] * ff * ff;
      }
      if (ecache && bb < nall) ecache[bb] = ff;
    }
  }
  *GM_out = GM;
  *GS1_out = sync_sum(g, s1, red);
  *GS2_out = sync_sum(g, s2, red);
}

// Last block: cumulative normalised weight at every tile start,
// P_b = sum_{b'<b} S1_b' e^{M_b' - lse}, summed in 64-bit fixed point (2^-62
// units): integer sums are exact, so the parallel scan gives the same monotone
// prefixes in any order.  `wsum` is shared scratch of >= 32 values owned by S.
// ecache (nullable): global_stats' exp(M_b - GM) of every partial, with
// inv_gs1 = 1 / sum: exp(M_b - lse) is then ecache[b] * inv_gs1.
template <class S>
static __device__ void write_tile_prefixes(const S& g, const PfJob& J, int nparts, double lse,
                                           unsigned long long* wsum, const double* ecache = nullptr,
                                           double inv_gs1 = 0.0) {
  // job fields in registers (the tprefix stores may alias the job table)
  PfScalars* const sc = J.sc;
  const int ntiles = J.ntiles;
  const double* __restrict__ part = J.part;
  const size_t ps = part_stride(J);
  double* __restrict__ tprefix = J.tprefix;
  const int per = (ntiles + g.size() - 1) / g.size();
  const int b0 = min(g.tid() * per, ntiles), b1 = min(b0 + per, ntiles);
  // this thread's tiles own the contiguous partials [q0, q1), nparts per tile,
  // read in batches of independent loads
  constexpr int kB = 8;
  const int q0 = b0 * nparts, q1 = b1 * nparts;
  auto batch = [&](int j0, unsigned long long (&w)[kB]) {  // fixed-point weights of j0 .. j0+kB-1
    double mb[kB], p1[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) {
      const double* p = part + (j0 + k < q1 ? j0 + k : 0);
      mb[k] = j0 + k < q1 ? __ldcg(p) : -INFINITY;
      p1[k] = __ldcg(p + ps);
    }
#pragma unroll
    for (int k = 0; k < kB; ++k) {
      w[k] = 0ull;
      if (mb[k] > -INFINITY) {
        const double e = ecache ? ecache[j0 + k] * inv_gs1 : exp(mb[k] - lse);
        w[k] = __double2ull_rn(p1[k] * e * kFix);
      }
    }
  };
  unsigned long long tot = 0ull;
  for (int j0 = q0; j0 < q1; j0 += kB) {
    unsigned long long w[kB];
    batch(j0, w);
#pragma unroll
    for (int k = 0; k < kB; ++k) tot += w[k];
  }
  unsigned long long all = 0ull;
  unsigned long long run = sync_excl_scan_u64(g, tot, wsum, &all);
  for (int j0 = q0; j0 < q1; j0 += kB) {
    unsigned long long w[kB];
    batch(j0, w);
#pragma unroll
    for (int k = 0; k < kB; ++k) {
      const int j = j0 + k;
      if (j < q1) {
        if ((j - q0) % nparts == 0) tprefix[j / nparts] = (double)run * kInvFix;  // tile start
        run += w[k];
      }
    }
  }
  if (g.tid() == 0) {
    tprefix[ntiles] = (double)all * kInvFix;
    sc->wn = (double)all * kInvFix;
  }
}

// The step's finalise, run by the threads of S in the job's last block (or
// group) once every partial of the step is in J.part (containers.jl:160-173
// marginalise!, particles.jl:70-73 baseline, resamplers.jl:179-183 ESS
// decision).  Baseline: log N after a resample or for the initial
// TypelessZero weights (plus the auxiliary filter's first-stage shift
// sc->base_adj after one of its resamples, resamplers.jl:118-138); otherwise
// logsumexp of the normalised log-weights, which is 0 up to the rounding of the
// normalisation (below 1e-15), so it is taken as 0.  `red`, `wsum` and `s_res`
// are shared scratch owned by S.
template <class S>
static __device__ void finish_step(const S& g, const PfJob& J, int t, bool fresh, int nparts,
                                   double* red, unsigned long long* wsum, int* s_res,
                                   double* ecache = nullptr) {
  PfScalars* const sc = J.sc;
  const bool aux = J.eta != nullptr;
  // the job's fields and this step's schedule / uniform entries are read before
  // the fold, so their L2 round trips overlap it (the later stores through sc
  // and the output pointers may alias the job table and would order each read
  // after the previous store)
  const int T = J.T;
  const int64_t N = J.N;
  const double threshold = J.threshold, log_n = J.log_n;
  const int8_t* const schedule = J.schedule;
  double* const ll_steps = J.ll_steps;
  double* const ess_steps = J.ess_steps;
  int8_t* const res_steps = J.res_steps;
  const double* const unif = J.unif;
  const uint64_t seed = J.seed;
  const int sch = (t < T && schedule) ? (int)schedule[t] : -1;
  const double u_next = (t < T && unif) ? unif[t] : 0.0;
  const double ll_prev = sc->ll, base_adj = sc->base_adj;
  // fold all partials in a fixed order (deterministic)
  double GM, GS1, GS2;
  global_stats(g, J, nparts, red, &GM, &GS1, &GS2, ecache);
  const double base = fresh ? log_n + base_adj : 0.0;
  const double lse = GM + log(GS1);
  if (g.tid() == 0) {
    double inc = lse - base;
    double ess = GS1 * GS1 / GS2;
    if (!(lse > -INFINITY) || isnan(lse)) sc->status = GF_ERR_ARG;  // all weights vanished
    sc->ll = ll_prev + inc;
    if (ll_steps) ll_steps[t - 1] = inc;
    int res = 0;
    if (t < T) {
      res = sch >= 0 ? (sch != 0) : (threshold * (double)N >= ess);
      if (ess_steps) ess_steps[t] = ess;
      if (res_steps) res_steps[t] = (int8_t)res;
      sc->u0 = unif ? u_next : philox_uniform(seed, 0u, (uint32_t)(t + 1));
    }
    sc->lse = lse;
    sc->ess = ess;
    sc->resample = res;
    sc->base_adj = 0.0;
    *s_res = res;
  }
  g.sync();
  // the auxiliary filter decides in its lookahead kernel instead
  if (*s_res && !aux) write_tile_prefixes(g, J, nparts, lse, wsum, ecache, 1.0 / GS1);
  g.sync();
  if (g.tid() == 0) {
    sc->uniform = 0;
    sc->scan_tile = 0u;
    sc->counter = 0u;
    __threadfence();
    sc->t = t;
  }
}

// Folds the block's accumulators into part[tile] and lets the last block of
// the job finalise the step (finish_step).  A tile may be covered by `nparts`
// blocks (block `part` of tile `tile`); the partials are then kept per part,
// folded in part order and summed per tile for the tile prefixes.
// ecache (nullable): shared memory for one double per partial, which keeps each
// partial's exponential from the fold for the tile prefixes (one exponential
// per partial instead of three on the last block's serial path).
static __device__ void block_finish(const PfJob& J, int tile, int t, bool fresh, LseAcc a,
                                    double* red, int part = 0, int nparts = 1, double* ecache = nullptr) {
  if (!fold_partials(J, tile, a, red, part, nparts)) return;
  __shared__ unsigned long long s_wsum[32];
  __shared__ int s_res;
  finish_step(BlockSync(), J, t, fresh, nparts, red, s_wsum, &s_res, ecache);
}

// Auxiliary particle filter, last block of the lookahead launch of step t:
// the ESS decision on softmax(logw + log eta) (AuxiliaryResampler,
// resamplers.jl:109-116, 179-183), and after a resample the tile prefixes of
// those weights and the baseline shift LSE(logw) - LSE(logw + log eta) that
// construct_new_state folds into ll_baseline (resamplers.jl:118-138; with the
// particles' new log-weights -log eta[a], LSE_3 cancels in predict).  A tile
// may be scored by `nparts` blocks (block `part` of tile `tile`).
static __device__ void apf_finish(const PfJob& J, int tile, int t, LseAcc a, double* red, int part = 0,
                                  int nparts = 1) {
  PfScalars* sc = J.sc;
  if (!fold_partials(J, tile, a, red, part, nparts)) return;
  double GM, GS1, GS2;
  global_stats(BlockSync(), J, nparts, red, &GM, &GS1, &GS2);
  const double lse1 = GM + log(GS1);
  __shared__ int s_res;
  __shared__ unsigned long long s_wsum[32];
  if (threadIdx.x == 0) {
    const double ess = GS1 * GS1 / GS2;
    const int s = J.schedule ? (int)J.schedule[t - 1] : -1;
    const int res = s >= 0 ? (s != 0) : (J.threshold * (double)J.N >= ess);
    if (!(lse1 > -INFINITY) || isnan(lse1)) sc->status = GF_ERR_ARG;
    if (J.ess_steps) J.ess_steps[t - 1] = ess;
    if (J.res_steps) J.res_steps[t - 1] = (int8_t)res;
    sc->resample = res;
    sc->lse_aux = lse1;
    sc->base_adj = res ? sc->lse - lse1 : 0.0;
    s_res = res;
  }
  __syncthreads();
  if (s_res) write_tile_prefixes(BlockSync(), J, nparts, lse1, s_wsum);
  __syncthreads();
  if (threadIdx.x == 0) {
    sc->counter = 0u;
    __threadfence();
  }
}

// Weighted filtered means sum_i exp(lw_i - LSE) x_i after step t (optional output).
template <typename Real>
__device__ __forceinline__ void pf_means_kernel(const PfJob* __restrict__ jobs, int njobs, double* __restrict__ mpart,
                                double* __restrict__ means, int mdim) {
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  const int t = sc->t;
  if (t < 1 || sc->status != 0) return;
  const int tile = blockIdx.x - J.tile0;
  const int64_t N = J.N;
  const Real* X = reinterpret_cast<const Real*>(J.X[t & 1]);
  const Real* lw = reinterpret_cast<const Real*>(J.lw);
  const double lse = sc->lse;
  __shared__ double red[32];
  __shared__ int s_last;
  for (int d = 0; d < mdim; ++d) {
    double s = 0.0;
    for (int p = 0; p < PF_PPT; ++p) {
      const int64_t i = (int64_t)tile * PF_TILE + p * PF_THREADS + threadIdx.x;
      if (i < N) s += exp((double)lw[i] - lse) * (double)X[(size_t)d * N + i];
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) mpart[(size_t)tile * mdim + d] = s;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&sc->mcounter, 1u) == (unsigned)(J.ntiles - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int d = 0; d < mdim; ++d) {
    double s = 0.0;
    for (int b = threadIdx.x; b < J.ntiles; b += blockDim.x) s += __ldcg(mpart + (size_t)b * mdim + d);
    s = block_sum(s, red);
    if (threadIdx.x == 0) means[(size_t)(t - 1) * mdim + d] = s;
  }
  if (threadIdx.x == 0) sc->mcounter = 0;
}

// Final outputs of a filter run by one block: normalised log-weights
// (lw - LSE), states, ll and clamps.
template <typename Real>
__device__ __forceinline__ void pf_finish_block(const PfJob& J) {
  const Real* lw = reinterpret_cast<const Real*>(J.lw);
  const double lse = J.sc->lse;
  const int tcur = J.sc->t;
  const Real* X = reinterpret_cast<const Real*>(J.X[tcur & 1]);
  Real* so = reinterpret_cast<Real*>(J.states_out);
  for (int64_t i = threadIdx.x; i < J.N; i += blockDim.x) {
    if (J.logw_out) J.logw_out[i] = (double)lw[i] - lse;
    if (so)
      for (int d = 0; d < J.width; ++d) so[(size_t)d * J.N + i] = X[(size_t)d * J.N + i];
  }
  if (threadIdx.x == 0) {
    if (J.ll_out) *J.ll_out = J.sc->ll;
    if (J.clamps_out) *J.clamps_out = J.sc->clamps;
  }
}

// ---------------------------------------------------------- resample kernel
// Runs after a propagate whose finalise decided to resample: per propagate
// tile, the cumulative normalised weights W_k = P_b + (running sum inside the
// tile) and each particle's cumulative offspring count O(W_k) (exact per
// rule) and the merge-path start points of the fill kernel, which turns the
// counts into ancestors.
// Multinomial ancestors (unsorted uniforms) instead take W_k to the per-slot
// search of the next propagate.
template <typename Real>
__device__ __forceinline__ void resample_tile(const PfJob& J, int tile) {
  PfScalars* sc = J.sc;
  if (!sc->resample || sc->status != 0 || sc->t >= J.T) return;
  __shared__ unsigned long long s_wsum[32];
  __shared__ int32_t s_last[PF_THREADS / 32];
  __shared__ int32_t s_O0;
  const int tstep = sc->t + 1;
  const int64_t N = J.N, i0 = (int64_t)tile * PF_TILE;
  const int nloc = (int)min((int64_t)PF_TILE, N - i0);
  // auxiliary filter: weights softmax(logw + log eta) (resamplers.jl:109-116)
  const bool aux = J.eta != nullptr;
  const double lse = aux ? sc->lse_aux : sc->lse;
  const double P0 = J.tprefix[tile], P1 = J.tprefix[tile + 1];
  // this thread's PF_PPT consecutive particles (vector loads; tiles start 16-byte aligned)
  const int l0 = PF_PPT * threadIdx.x;
  const Real* lw = reinterpret_cast<const Real*>(J.lw) + i0 + l0;
  Real x[PF_PPT];
  if (l0 + PF_PPT <= nloc) {
    if constexpr (sizeof(Real) == 4) {
      const float4 v = *reinterpret_cast<const float4*>(lw);
      x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
    } else {
      const double2 a = reinterpret_cast<const double2*>(lw)[0], b = reinterpret_cast<const double2*>(lw)[1];
      x[0] = a.x, x[1] = a.y, x[2] = b.x, x[3] = b.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < PF_PPT; ++q) x[q] = l0 + q < nloc ? lw[q] : (Real)0;
  }
  double xv[PF_PPT];
#pragma unroll
  for (int q = 0; q < PF_PPT; ++q) xv[q] = (double)x[q];
  if (aux) {
    const Real* eta = reinterpret_cast<const Real*>(J.eta) + i0 + l0;
#pragma unroll
    for (int q = 0; q < PF_PPT; ++q)
      if (l0 + q < nloc) xv[q] += (double)eta[q];
  }
  // W_k = P0 + (fixed-point running sum inside the tile), clamped to the tile's end
  unsigned long long loc[PF_PPT], acc = 0ull;
#pragma unroll
  for (int q = 0; q < PF_PPT; ++q) {
    if (l0 + q < nloc) acc += __double2ull_rn(exp(xv[q] - lse) * kFix);
    loc[q] = acc;
  }
  unsigned long long all;
  const unsigned long long excl = block_excl_scan_u64(acc, s_wsum, &all);
  auto cumw = [&](int q) {
    const double W = P0 + (double)(excl + loc[q]) * kInvFix;
    return (l0 + q == nloc - 1) ? P1 : (W < P1 ? W : P1);
  };
  if (J.resampler == GF_RS_MULTINOMIAL) {
    double* __restrict__ key = J.key + i0;
#pragma unroll
    for (int q = 0; q < PF_PPT; ++q)
      if (l0 + q < nloc) key[l0 + q] = cumw(q);
    return;
  }
  const OffspringRule rule = make_rule(J, sc, tstep);
  if (threadIdx.x == 0) s_O0 = (int32_t)rule.count(P0);
  int32_t c[PF_PPT];
#pragma unroll
  for (int q = 0; q < PF_PPT; ++q) {
    c[q] = 0;
    if (l0 + q >= nloc) continue;
    c[q] = (int32_t)rule.count(cumw(q));
    if (i0 + l0 + q == N - 1) {
      // slots past the last threshold below W_N (rounding) go to the last
      // particle; the reference's walk has no clamp, so they are counted
      if (c[q] < N) atomicAdd(&sc->clamps, (int32_t)(N - c[q]));
      c[q] = (int32_t)N;
    }
  }
  int32_t* __restrict__ ocum = J.ocum + i0 + l0;
  if (l0 + PF_PPT <= nloc) {
    *reinterpret_cast<int4*>(ocum) = make_int4(c[0], c[1], c[2], c[3]);
  } else {
#pragma unroll
    for (int q = 0; q < PF_PPT; ++q)
      if (l0 + q < nloc) ocum[q] = c[q];
  }
  // count of the particle before this thread's first one
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t cprev = __shfl_up_sync(0xffffffffu, c[PF_PPT - 1], 1);
  if (lane == 31) s_last[wid] = c[PF_PPT - 1];
  __syncthreads();
  if (lane == 0) cprev = wid == 0 ? s_O0 : s_last[wid - 1];
  // Merge-path partition of the fill: merging particles (consumed when all
  // their slots are out) with slots j (slot j belongs to the first k with
  // O_k > j), the state after d items has consumed the largest k with
  // f(k) = O_{k-1} + k <= d.  f(k+1) - f(k) = offspring_k + 1 >= 1, so the
  // diagonals d in [f(k), f(k+1)) start at particle k; fill block m starts at
  // diagonal m * FILL_D.
#pragma unroll
  for (int q = 0; q < PF_PPT; ++q) {
    if (l0 + q >= nloc) break;
    const int64_t k = i0 + l0 + q;
    const int64_t flo = (int64_t)(q == 0 ? cprev : c[q - 1]) + k;
    const int64_t fhi = (int64_t)c[q] + k + 1;
    for (int64_t d = (flo + FILL_D - 1) / FILL_D * FILL_D; d < fhi; d += FILL_D)
      J.mpk[d / FILL_D] = (int32_t)k;
  }
}

template <typename Real>
// 4 blocks per SM: 64 registers, no spills (a bound of 6 spilled at 40 registers
// and still needed two waves for 1,024 tiles)
__global__ void __launch_bounds__(PF_THREADS, 4) pf_resample_kernel(const PfJob* __restrict__ jobs,
                                                                   int njobs) {
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  resample_tile<Real>(J, blockIdx.x - J.tile0);
}

// Fill kernel: ancestors (0-based) of every slot from the cumulative offspring
// counts (slot j's ancestor is the first k with ocum[k] > j, the cumulative-
// offspring form of CUDAExt.jl:90-103), written to J.anc, which the next
// propagate reads coalesced.  Block m merges exactly FILL_D items (particles
// plus slots) starting at its merge-path point, so the work is balanced
// however the offspring are distributed: at most FILL_D + 1 counts are staged
// in shared memory, each thread binary-searches its own start and merges
// FILL_IPT items, and the block's slots are written out coalesced.
// COHERENT: read the counts through L2, for a caller that wrote them earlier
// in the same kernel.
template <bool COHERENT>
__device__ __forceinline__ void fill_block(const PfJob& J, int m) {
  const PfScalars* sc = J.sc;
  if (!sc->resample || sc->status != 0 || sc->t >= J.T || J.resampler == GF_RS_MULTINOMIAL) return;
  __shared__ int32_t s_oc[FILL_D + 1];
  __shared__ int32_t s_anc[FILL_D];
  const int64_t N = J.N;
  const int64_t d0 = (int64_t)m * FILL_D, d1 = min(d0 + FILL_D, 2 * N);
  const int64_t k0 = J.mpk[m];
  const int64_t k1 = m + 1 < J.ntiles ? (int64_t)J.mpk[m + 1] : N;
  const int64_t j0 = d0 - k0, j1 = d1 - k1;
  const int nk = (int)(min(k1, N - 1) - k0 + 1);  // counts ocum[k0 .. min(k1, N-1)]
  const int32_t* __restrict__ oc = J.ocum;
  int32_t* __restrict__ anc = J.anc;
  // all of a thread's counts are loaded before any is stored to shared memory:
  // one L2 round trip instead of one per count (nk <= FILL_D + 1)
  constexpr int kPer = (FILL_D + 1 + PF_THREADS - 1) / PF_THREADS;
  int32_t cv[kPer];
#pragma unroll
  for (int r = 0; r < kPer; ++r) {
    const int q = threadIdx.x + r * PF_THREADS;
    cv[r] = q < nk ? (COHERENT ? __ldcg(oc + k0 + q) : oc[k0 + q]) : 0;
  }
#pragma unroll
  for (int r = 0; r < kPer; ++r) {
    const int q = threadIdx.x + r * PF_THREADS;
    if (q < nk) s_oc[q] = cv[r];
  }
  __syncthreads();
  const int64_t d = d0 + (int64_t)threadIdx.x * FILL_IPT;
  if (d < d1) {
    // largest local k in [0, k1 - k0] with f(k0 + k) <= d (f(k0) <= d0 <= d)
    int lo = 0, hi = (int)(k1 - k0);
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((int64_t)s_oc[mid - 1] + k0 + mid <= d) lo = mid;
      else hi = mid - 1;
    }
    int64_t k = k0 + lo, j = d - k;
    const int64_t de = min(d + FILL_IPT, d1);
    for (int64_t e = d; e < de; ++e) {
      if (k < N && j < (int64_t)s_oc[k - k0]) {
        s_anc[j - j0] = (int32_t)k;
        ++j;
      } else {
        ++k;
      }
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < (int)(j1 - j0); q += PF_THREADS) anc[j0 + q] = s_anc[q];
}

template <int DUMMY = 0>
__global__ void __launch_bounds__(PF_THREADS, 8) pf_fill_ancestors_kernel(const PfJob* __restrict__ jobs,
                                                                      int njobs) {
  const int jb = find_job(jobs, njobs, blockIdx.x, false);
  const PfJob& J = jobs[jb];
  fill_block<false>(J, blockIdx.x - J.tile0);
}

// ------------------------------------------------------------ lookback scan
// Decoupled lookback of tile b, run by one full warp: publishes the tile's
// aggregate `tot` (fagg[b]), walks back over the predecessors' inclusive
// prefixes (finc) or aggregates 32 tiles at a time, publishes the inclusive
// prefix finc[b] and returns the exclusive prefix.  Every flag carries kReady
// once written.  A predecessor whose flag stays unset is polled at most
// `spin_limit` times; then *fail is set (all lanes), finc[b] stays
// unpublished and the return value is meaningless.
__device__ __forceinline__ unsigned long long lookback_exclusive(unsigned long long* fagg,
                                                                 unsigned long long* finc, int b,
                                                                 unsigned long long tot,
                                                                 long long spin_limit, bool* fail) {
  const int lane = threadIdx.x & 31;
  unsigned long long excl = 0ull;
  *fail = false;
  if (b == 0) {
    if (lane == 0) atomicExch(finc, kReady | tot);
    return 0ull;
  }
  if (lane == 0) atomicExch(fagg + b, kReady | tot);
  int j = b - 1;
  long long spins = 0;
  while (true) {
    const int k = j - lane;
    unsigned long long vi = 0ull, va = 0ull;
    if (k >= 0) {
      vi = *(volatile unsigned long long*)(finc + k);
      if (!(vi & kReady)) va = *(volatile unsigned long long*)(fagg + k);
    }
    const int st = k < 0 ? 3 : ((vi & kReady) ? 2 : ((va & kReady) ? 1 : 0));
    const unsigned prefix_mask = __ballot_sync(0xffffffffu, st >= 2);
    const int stop = prefix_mask ? __ffs(prefix_mask) - 1 : 32;  // first lane holding a prefix
    const unsigned notready = __ballot_sync(0xffffffffu, st == 0);
    const unsigned need = stop >= 32 ? 0xffffffffu : ((2u << stop) - 1u);
    if (notready & need) {
      if (++spins > spin_limit) {
        *fail = true;
        return 0ull;
      }
      continue;
    }
    unsigned long long val = 0ull;
    if (lane <= stop && st < 3) val = (st == 2 ? vi : va) & ~kReady;
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    excl += val;
    if (stop < 32) break;
    j -= 32;
  }
  if (lane == 0) atomicExch(finc + b, kReady | (excl + tot));
  return excl;
}

// Cumulative normalised weights W_k = sum_{i<=k} exp(lw_i - LSE) for the
// pending resample.  Each weight is rounded once to 64-bit fixed point (2^-62
// units); integer sums are associative, so the decoupled lookback's result is
// exact and does not depend on how far each tile looked back.
template <typename Real>
__global__ void __launch_bounds__(SCAN_THREADS) pf_scan_kernel(const PfJob* __restrict__ jobs,
                                                              int njobs) {
  const int jb = find_job(jobs, njobs, blockIdx.x, true);
  const PfJob& J = jobs[jb];
  PfScalars* sc = J.sc;
  if (!sc->resample || sc->status != 0 || sc->t >= J.T) return;
  __shared__ unsigned long long sv[SCAN_TILE + SCAN_TILE / 16];
  __shared__ unsigned long long wsum[SCAN_THREADS / 32];
  __shared__ int s_tile;
  __shared__ unsigned long long s_excl;
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_tile = (int)atomicAdd(&sc->scan_tile, 1u);
    s_fail = 0;
  }
  __syncthreads();
  const int b = s_tile;
  const int64_t base = (int64_t)b * SCAN_TILE;
  const int64_t N = J.N;
  const double lse = sc->lse;
  const Real* lw = (const Real*)J.lw;
  // striped coalesced loads -> fixed point -> shared (padded)
#pragma unroll 4
  for (int q = 0; q < SCAN_IPT; ++q) {
    int idx = q * SCAN_THREADS + threadIdx.x;
    int64_t k = base + idx;
    unsigned long long v = 0ull;
    if (k < N) {
      double w = J.wraw ? J.wraw[k] / sc->wtotal : exp((double)lw[k] - lse);
      v = __double2ull_rn(w * kFix);
    }
    sv[idx + (idx >> 4)] = v;
  }
  __syncthreads();
  // thread-serial inclusive scan over 16 contiguous items
  unsigned long long loc[SCAN_IPT];
  unsigned long long acc = 0ull;
#pragma unroll
  for (int q = 0; q < SCAN_IPT; ++q) {
    int idx = threadIdx.x * SCAN_IPT + q;
    acc += sv[idx + (idx >> 4)];
    loc[q] = acc;
  }
  // block exclusive scan of the thread totals
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long x = acc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  unsigned long long wpre = 0ull, tot = 0ull;
  for (int w = 0; w < SCAN_THREADS / 32; ++w) {
    if (w < wid) wpre += wsum[w];
    tot += wsum[w];
  }
  unsigned long long texcl = wpre + x - acc;
  // decoupled lookback (warp 0)
  if (wid == 0) {
    bool fail = false;
    const unsigned long long excl = lookback_exclusive(J.flags, J.flags + J.nstiles, b, tot,
                                                       kSpinLimit, &fail);
    if (lane == 0) {
      if (fail) {
        sc->status = GF_ERR_TIMEOUT;
        s_fail = 1;
      }
      s_excl = excl;
    }
  }
  __syncthreads();
  if (s_fail) return;
  const unsigned long long off = s_excl + texcl;
  // back through shared for coalesced stores of W_k
  double* sw = reinterpret_cast<double*>(sv);
  __syncthreads();
#pragma unroll
  for (int q = 0; q < SCAN_IPT; ++q) {
    int idx = threadIdx.x * SCAN_IPT + q;
    sw[idx + (idx >> 4)] = (double)(off + loc[q]) * kInvFix;
  }
  __syncthreads();
#pragma unroll 4
  for (int q = 0; q < SCAN_IPT; ++q) {
    int idx = q * SCAN_THREADS + threadIdx.x;
    int64_t k = base + idx;
    if (k < N) J.key[k] = sw[idx + (idx >> 4)];
  }
  if (b == J.nstiles - 1 && threadIdx.x == 0) sc->wn = (double)(s_excl + tot) * kInvFix;
}

}  // namespace gf
