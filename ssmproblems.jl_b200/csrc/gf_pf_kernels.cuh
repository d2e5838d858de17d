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
constexpr int PF_PW = 6;                       // doubles per block partial
constexpr unsigned long long kReady = 1ull << 63;
constexpr double kFix = 4611686018427387904.0; // 2^62
constexpr double kInvFix = 1.0 / 4611686018427387904.0;
constexpr long long kSpinLimit = 1ll << 20;    // bounded lookback wait (~1 s)

struct PfJob {
  int64_t N;
  int32_t dx, dy, T, width;
  int32_t tile0, ntiles, stile0, nstiles;
  int32_t resampler, conv, prop, pad0;
  double threshold, log_n, obs_const, prop_const;
  uint64_t seed;
  const void* params;        // model parameters in the run's precision
  const void* ystep;         // per-step vectors [T][ystride]
  int32_t ystride, pad1;
  void* X[2];                // SoA state ping-pong [width][N]
  void* lw;                  // stored log-weights [N]
  double* key;               // cumulative normalised weights [N]
  double* part;              // [ntiles][PF_PW]
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
};

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

// Boundary ancestors of the block's slot chunks (monotone resamplers): thread
// 2p / 2p+1 searches the first / last slot of chunk p over the whole range.
__device__ __forceinline__ void chunk_bounds(const PfJob& J, PfScalars* sc, int t, int tile,
                                             int64_t* sb) {
  if (threadIdx.x < 2 * PF_PPT) {
    int p = threadIdx.x >> 1;
    int64_t first = (int64_t)tile * PF_TILE + (int64_t)p * PF_THREADS;
    int64_t j = (threadIdx.x & 1) ? first + PF_THREADS - 1 : first;
    if (j > J.N - 1) j = J.N - 1;
    if (first > J.N - 1) {
      sb[threadIdx.x] = 0;
    } else {
      SlotSearch s = make_search(J, sc, t, j);
      int64_t a = s.first(0, J.N);
      sb[threadIdx.x] = a >= J.N ? J.N - 1 : a;
    }
  }
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

// Folds the block's accumulators into part[tile] and lets the last block of
// the job finalise the step (containers.jl:160-173 marginalise!,
// particles.jl:70-73 baseline, resamplers.jl:179-183 ESS decision).
static __device__ void block_finish(const PfJob& J, int tile, int t, bool fresh, LseAcc a, LseAcc b0,
                             double* red) {
  PfScalars* sc = J.sc;
  __shared__ int s_last;
  double M = block_max(a.m, red);
  double f = a.m > -INFINITY ? exp(a.m - M) : 0.0;
  double S1 = block_sum(a.s1 * f, red);
  double S2 = block_sum(a.s2 * f * f, red);
  double M0 = -INFINITY, S0 = 0.0;
  if (!fresh) {
    M0 = block_max(b0.m, red);
    double f0 = b0.m > -INFINITY ? exp(b0.m - M0) : 0.0;
    S0 = block_sum(b0.s1 * f0, red);
  }
  if (threadIdx.x == 0) {
    double* p = J.part + (size_t)tile * PF_PW;
    p[0] = M;
    p[1] = S1;
    p[2] = S2;
    p[3] = M0;
    p[4] = S0;
    __threadfence();
    unsigned prev = atomicAdd(&sc->counter, 1u);
    s_last = (prev == (unsigned)(J.ntiles - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // ---- last block: fold all partials in a fixed order (deterministic) ----
  double m = -INFINITY;
  for (int bb = threadIdx.x; bb < J.ntiles; bb += blockDim.x) m = fmax(m, __ldcg(J.part + (size_t)bb * PF_PW));
  double GM = block_max(m, red);
  double s1 = 0.0, s2 = 0.0, m0 = -INFINITY;
  for (int bb = threadIdx.x; bb < J.ntiles; bb += blockDim.x) {
    const double* p = J.part + (size_t)bb * PF_PW;
    double mb = __ldcg(p);
    if (mb > -INFINITY) {
      double ff = exp(mb - GM);
      s1 += __ldcg(p + 1) * ff;
      s2 += __ldcg(p + 2) * ff * ff;
    }
    if (!fresh) m0 = fmax(m0, __ldcg(p + 3));
  }
  double GS1 = block_sum(s1, red);
  double GS2 = block_sum(s2, red);
  double base = J.log_n;
  if (!fresh) {
    double GM0 = block_max(m0, red);
    double s0 = 0.0;
    for (int bb = threadIdx.x; bb < J.ntiles; bb += blockDim.x) {
      const double* p = J.part + (size_t)bb * PF_PW;
      double mb = __ldcg(p + 3);
      if (mb > -INFINITY) s0 += __ldcg(p + 4) * exp(mb - GM0);
    }
    double GS0 = block_sum(s0, red);
    base = GM0 + log(GS0);
  }
  // clear the lookback flags for the scan that may follow
  for (int bb = threadIdx.x; bb < 2 * J.nstiles; bb += blockDim.x) J.flags[bb] = 0ull;
  if (threadIdx.x == 0) {
    double lse = GM + log(GS1);
    double inc = lse - base;
    double ess = GS1 * GS1 / GS2;
    if (!(lse > -INFINITY) || isnan(lse)) sc->status = GF_ERR_ARG;  // all weights vanished
    sc->ll += inc;
    if (J.ll_steps) J.ll_steps[t - 1] = inc;
    int res = 0;
    if (t < J.T) {
      int s = J.schedule ? (int)J.schedule[t] : -1;
      res = s >= 0 ? (s != 0) : (J.threshold * (double)J.N >= ess);
      if (J.ess_steps) J.ess_steps[t] = ess;
      if (J.res_steps) J.res_steps[t] = (int8_t)res;
      sc->u0 = J.unif ? J.unif[t] : philox_uniform(J.seed, 0u, (uint32_t)(t + 1));
    }
    sc->lse = lse;
    sc->ess = ess;
    sc->resample = res;
    sc->uniform = 0;
    sc->scan_tile = 0u;
    sc->counter = 0u;
    __threadfence();
    sc->t = t;
  }
}

// ------------------------------------------------------------ lookback scan
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
    unsigned long long* fagg = J.flags;
    unsigned long long* finc = J.flags + J.nstiles;
    unsigned long long excl = 0ull;
    if (b == 0) {
      if (lane == 0) atomicExch(finc, kReady | tot);
    } else {
      if (lane == 0) atomicExch(fagg + b, kReady | tot);
      int j = b - 1;
      long long spins = 0;
      while (true) {
        int k = j - lane;
        unsigned long long vi = 0ull, va = 0ull;
        if (k >= 0) {
          vi = *(volatile unsigned long long*)(finc + k);
          if (!(vi & kReady)) va = *(volatile unsigned long long*)(fagg + k);
        }
        int st = k < 0 ? 3 : ((vi & kReady) ? 2 : ((va & kReady) ? 1 : 0));
        unsigned prefix_mask = __ballot_sync(0xffffffffu, st >= 2);
        int stop = prefix_mask ? __ffs(prefix_mask) - 1 : 32;  // first lane holding a prefix
        unsigned notready = __ballot_sync(0xffffffffu, st == 0);
        unsigned need = stop >= 32 ? 0xffffffffu : ((2u << stop) - 1u);
        if (notready & need) {
          if (++spins > kSpinLimit) {
            if (lane == 0) {
              sc->status = GF_ERR_TIMEOUT;
              s_fail = 1;
            }
            break;
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
      if (lane == 0 && !s_fail) atomicExch(finc + b, kReady | (excl + tot));
    }
    if (lane == 0) s_excl = excl;
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
