// gf_pf_tree.cu -- device path storage (ancestry tree) of a particle-filter run.
//
// Restates the sparse path storage of AncestorCallback / ParticleTree
// (callbacks.jl:90-111, containers.jl:466-631) and of the GPU
// ParallelParticleTree (ext/CUDAExt.jl:146-298), Jacob, Murray & Rubenthaler
// (2015): per step,
//   count : a_i = ancestor of new particle i, offspring counts of the current ones
//   prune : a current particle without offspring frees its slot, and each freed
//           slot decrements its parent's count; the thread whose atomic decrement
//           takes a count to zero frees that parent and walks on (so exactly one
//           thread continues up a dying lineage)
//   assign: new particle i takes a freed slot, parent = slot of its ancestor
//   insert: (after the propagate) copy the new states into their slots.
// The observable result is get_ancestry: the trajectory of every final particle.
#include <type_traits>

#include "gf_internal.hpp"
#include "gf_pf_host.hpp"
#include "gf_pf_kernels.cuh"

namespace gf {
namespace {

constexpr int TREE_THREADS = 256;
constexpr int kWalkLimit = 1 << 26;  // bound on a lineage walk (depth <= T + 1)

inline int tree_blocks(int64_t n, int sms) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + TREE_THREADS - 1) / TREE_THREADS, 8 * (int64_t)sms));
}

template <typename Real>
__global__ void tree_init_kernel(const PfJob* __restrict__ jobs, PfTree tr) {
  const PfJob& J = jobs[0];
  const int64_t N = J.N, M = tr.M;
  const Real* X = reinterpret_cast<const Real*>(J.X[0]);
  Real* S = reinterpret_cast<Real*>(tr.states);
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < M; s += (int64_t)gridDim.x * blockDim.x) {
    tr.offspring[s] = 0;
    tr.parents[s] = -1;
    if (s < N) {
      for (int d = 0; d < tr.width; ++d) S[(size_t)s * tr.width + d] = X[(size_t)d * N + s];
      tr.leaves[s] = (int32_t)s;
      tr.cnt[s] = 0;
    } else {
      tr.stack[M - 1 - s] = (int32_t)s;  // free slots N..M-1
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *tr.top = (int32_t)(M - N);
}

__device__ __forceinline__ bool tree_step_live(const PfJob& J, int* t) {
  const PfScalars* sc = J.sc;
  if (sc->status != 0) return false;
  *t = sc->t + 1;
  return *t <= J.T;
}

__global__ void tree_count_kernel(const PfJob* __restrict__ jobs, PfTree tr) {
  const PfJob& J = jobs[0];
  int t;
  if (!tree_step_live(J, &t)) return;
  PfScalars* sc = J.sc;
  const bool resamp = sc->resample != 0;
  const int64_t N = J.N;
  const bool multinomial = J.resampler == GF_RS_MULTINOMIAL;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = i;
    if (!resamp) {
      tr.cnt[i] = 1;
    } else if (multinomial) {
      a = make_search(J, sc, t, i).first(0, N);  // the propagate's search (clamps counted there)
      if (a >= N) a = N - 1;
      atomicAdd(&tr.cnt[a], 1);
    } else {
      a = J.anc[i];
      tr.cnt[i] = J.ocum[i] - (i > 0 ? J.ocum[i - 1] : 0);  // cumulative offspring counts
    }
    tr.anc[i] = (int32_t)a;
  }
}

// Freed slots are collected per block in shared memory and pushed with one
// reservation on the global free stack per block; a single stack counter would
// otherwise serialise one atomic per warp and per freed lineage node.
constexpr int PRUNE_BUF = 4096;

struct FreeList {
  int32_t* buf;
  int* n;
  __device__ __forceinline__ void push(const PfTree& tr, int32_t slot) const {
    const int pos = atomicAdd(n, 1);
    if (pos < PRUNE_BUF) buf[pos] = slot;
    else tr.stack[atomicAdd(tr.top, 1)] = slot;  // buffer full: push directly
  }
};

// SORTED: the rule keeps ancestors nondecreasing (systematic, stratified, or no
// resampling), so the children of one parent are consecutive particles; each
// warp sums its dead children per parent (segmented scan over equal parents)
// and issues one atomic per parent, where a weight collapse would otherwise
// serialise thousands of decrements on one count.
template <bool SORTED>
__global__ void tree_prune_kernel(const PfJob* __restrict__ jobs, PfTree tr) {
  const PfJob& J = jobs[0];
  int t;
  if (!tree_step_live(J, &t)) return;
  __shared__ int32_t s_buf[PRUNE_BUF];
  __shared__ int s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  const FreeList fl{s_buf, &s_n};
  const int64_t N = J.N;
  const int lane = threadIdx.x & 31;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s = tr.leaves[k];
    const int32_t c = tr.cnt[k];
    tr.offspring[s] = c;
    if (c == 0) fl.push(tr, s);
    int32_t walk = -1;  // a parent whose count this thread took to zero
    if constexpr (SORTED) {
      const unsigned act = __activemask();
      const int32_t key = tr.parents[s];
      int sum = c == 0 ? 1 : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(act, sum, o);
        const int32_t kk = __shfl_up_sync(act, key, o);
        if (lane >= o && ((act >> (lane - o)) & 1u) && kk == key) sum += v;
      }
      const int32_t next = __shfl_down_sync(act, key, 1);
      const bool tail = lane == 31 || !((act >> (lane + 1)) & 1u) || next != key;
      if (tail && sum > 0 && key >= 0 && atomicSub(&tr.offspring[key], sum) == sum) walk = key;
    } else if (c == 0) {
      const int32_t p = tr.parents[s];
      if (p >= 0 && atomicSub(&tr.offspring[p], 1) == 1) walk = p;
    }
    for (int it = 0; walk >= 0 && it < kWalkLimit; ++it) {
      fl.push(tr, walk);
      const int32_t p = tr.parents[walk];
      walk = (p >= 0 && atomicSub(&tr.offspring[p], 1) == 1) ? p : -1;
    }
  }
  __syncthreads();
  const int n = min(s_n, PRUNE_BUF);
  if (threadIdx.x == 0 && n > 0) s_base = atomicAdd(tr.top, n);
  __syncthreads();
  for (int q = threadIdx.x; q < n; q += blockDim.x) tr.stack[s_base + q] = s_buf[q];
}

__global__ void tree_assign_kernel(const PfJob* __restrict__ jobs, PfTree tr) {
  const PfJob& J = jobs[0];
  int t;
  if (!tree_step_live(J, &t)) return;
  const int64_t N = J.N;
  const int32_t top0 = *tr.top;
  if (top0 < N) {  // no room: the host sizes the pool before every chunk of steps
    if (blockIdx.x == 0 && threadIdx.x == 0) J.sc->status = GF_ERR_OOM_BUDGET;
    return;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t nl = tr.stack[top0 - N + i];
    tr.new_leaf[i] = nl;
    tr.parents[nl] = tr.leaves[tr.anc[i]];
    tr.offspring[nl] = 0;
  }
}

template <typename Real>
__global__ void tree_insert_kernel(const PfJob* __restrict__ jobs, PfTree tr, int t) {
  const PfJob& J = jobs[0];
  if (J.sc->status != 0) return;
  const int64_t N = J.N, M = tr.M;
  const Real* X = reinterpret_cast<const Real*>(J.X[t & 1]);
  Real* S = reinterpret_cast<Real*>(tr.states);
  constexpr int V = 16 / sizeof(Real);  // elements per 16-byte store
  using Vec = typename std::conditional<sizeof(Real) == 4, float4, double2>::type;
  const bool vec = tr.width % V == 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t nl = tr.new_leaf[i];
    Real* dst = S + (size_t)nl * tr.width;
    if (vec) {
      for (int d0 = 0; d0 < tr.width; d0 += V) {
        Real v[V];
#pragma unroll
        for (int q = 0; q < V; ++q) v[q] = X[(size_t)(d0 + q) * N + i];
        *reinterpret_cast<Vec*>(dst + d0) = *reinterpret_cast<const Vec*>(v);
      }
    } else {
      for (int d = 0; d < tr.width; ++d) dst[d] = X[(size_t)d * N + i];
    }
    tr.leaves[i] = nl;
    tr.cnt[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *tr.top -= (int32_t)N;
}

template <typename Real>
__global__ void tree_paths_kernel(const PfJob* __restrict__ jobs, PfTree tr, int T, Real* __restrict__ out) {
  const PfJob& J = jobs[0];
  const int64_t N = J.N, M = tr.M;
  const Real* S = reinterpret_cast<const Real*>(tr.states);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
    int32_t s = tr.leaves[k];
    for (int t = T; t >= 0 && s >= 0; --t) {
      for (int d = 0; d < tr.width; ++d) out[((size_t)t * tr.width + d) * N + k] = S[(size_t)s * tr.width + d];
      s = tr.parents[s];
    }
  }
}

// New slots M_old..M-1 join the free stack above the surviving entries.
__global__ void tree_grow_kernel(PfTree tr, int64_t M_old, int32_t top_old) {
  const int64_t add = tr.M - M_old;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < add; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = tr.M - 1 - k;
    tr.parents[s] = -1;
    tr.offspring[s] = 0;
    tr.stack[top_old + k] = (int32_t)s;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *tr.top = (int32_t)(top_old + add);
}

}  // namespace

void tree_launch_init(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr) {
  const int g = tree_blocks(tr.M, ctx->num_sms);
  if (dbl) tree_init_kernel<double><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
  else tree_init_kernel<float><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
}

void tree_launch_step_pre(gf_ctx* ctx, const PfJob* job_dev, int64_t N, const PfTree& tr,
                          bool sorted_ancestors) {
  const int g = tree_blocks(N, ctx->num_sms);
  tree_count_kernel<<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
  if (sorted_ancestors) tree_prune_kernel<true><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
  else tree_prune_kernel<false><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
  tree_assign_kernel<<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr);
}

void tree_launch_insert(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr, int t) {
  const int g = tree_blocks(N, ctx->num_sms);
  if (dbl) tree_insert_kernel<double><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr, t);
  else tree_insert_kernel<float><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr, t);
}

void tree_launch_paths(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr, int T,
                       void* out) {
  const int g = tree_blocks(N, ctx->num_sms);
  if (dbl) tree_paths_kernel<double><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr, T, (double*)out);
  else tree_paths_kernel<float><<<g, TREE_THREADS, 0, ctx->stream>>>(job_dev, tr, T, (float*)out);
}

void tree_launch_grow_init(gf_ctx* ctx, const PfTree& tr_new, int64_t M_old, int32_t top_old) {
  const int g = tree_blocks(tr_new.M - M_old, ctx->num_sms);
  tree_grow_kernel<<<g, TREE_THREADS, 0, ctx->stream>>>(tr_new, M_old, top_old);
}


// ------------------------------------------------------------ host side
// Pool arrays of M slots (states, parents, offspring, stack) into `bufs`.
static gf_status tree_pool_alloc(TreeHost& h, int64_t M, PfTree* tr, std::vector<DevBuf>* bufs) {
  gf_ctx* ctx = h.ctx;
  auto get = [&](size_t bytes, void** v) -> gf_status {
    gf_status st = dev_alloc(ctx, bytes, v);
    if (!st) bufs->push_back({*v, bytes});
    return st;
  };
  void* v;
  gf_status st;
  tr->M = M;
  if ((st = get(h.rsize * (size_t)h.width * M, &v))) return st;
  tr->states = v;
  if ((st = get(sizeof(int32_t) * (size_t)M, &v))) return st;
  tr->parents = (int32_t*)v;
  if ((st = get(sizeof(int32_t) * (size_t)M, &v))) return st;
  tr->offspring = (int32_t*)v;
  if ((st = get(sizeof(int32_t) * (size_t)M, &v))) return st;
  tr->stack = (int32_t*)v;
  return GF_OK;
}

// Per-particle arrays once, the pool at its default size N (2 + ceil(log2 N))
// (grown during the run as needed).
gf_status tree_host_prepare(TreeHost& h) {
  const int64_t N = h.N;
  PfTree& tr = h.tree;
  tr.width = h.width;
  if (!tr.leaves) {
    std::vector<DevBuf> bufs;
    void* v;
    gf_status st;
    for (int32_t** f : {&tr.leaves, &tr.new_leaf, &tr.anc, &tr.cnt}) {
      if ((st = dev_alloc(h.ctx, sizeof(int32_t) * (size_t)N, &v))) return st;
      bufs.push_back({v, sizeof(int32_t) * (size_t)N});
      *f = (int32_t*)v;
    }
    if ((st = dev_alloc(h.ctx, 256, &v))) return st;
    bufs.push_back({v, 256});
    tr.top = (int32_t*)v;
    h.bufs.insert(h.bufs.end(), bufs.begin(), bufs.end());
  }
  if (!tr.states) {
    int64_t lg = 1;
    while ((int64_t(1) << lg) < N) ++lg;
    const int64_t M = std::min<int64_t>(N * (2 + lg), INT32_MAX);
    std::vector<DevBuf> bufs;
    gf_status st = tree_pool_alloc(h, M, &tr, &bufs);
    h.bufs.insert(h.bufs.end(), bufs.begin(), bufs.end());
    if (st) return st;
  }
  return GF_OK;
}

// Makes room for `need` slots: doubles the pool (at least) when fewer are free.
gf_status tree_host_reserve(TreeHost& h, int64_t need) {
  gf_ctx* ctx = h.ctx;
  cudaStream_t s = ctx->stream;
  PfTree& tr = h.tree;
  int32_t top = 0;
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(&top, tr.top, sizeof top, cudaMemcpyDeviceToHost, s));
  GF_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
  if (top >= need) return GF_OK;
  const int64_t M_old = tr.M;
  const int64_t M_new = std::max<int64_t>(2 * M_old, M_old + need - top);
  if (M_new > INT32_MAX) return set_err(ctx, GF_ERR_OOM_BUDGET, "ancestry tree exceeds 2^31 slots");
  PfTree nt = tr;
  std::vector<DevBuf> bufs;
  gf_status st = tree_pool_alloc(h, M_new, &nt, &bufs);
  if (st) {
    for (auto& b : bufs) dev_free(ctx, b.p, b.bytes);
    return st;
  }
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(nt.states, tr.states, h.rsize * (size_t)h.width * M_old,
                                     cudaMemcpyDeviceToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(nt.parents, tr.parents, 4 * M_old, cudaMemcpyDeviceToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(nt.offspring, tr.offspring, 4 * M_old, cudaMemcpyDeviceToDevice, s));
  GF_CHECK_CUDA(ctx, cudaMemcpyAsync(nt.stack, tr.stack, 4 * (size_t)top, cudaMemcpyDeviceToDevice, s));
  tree_launch_grow_init(ctx, nt, M_old, top);
  // release the old pool arrays
  for (void* old : {tr.states, (void*)tr.parents, (void*)tr.offspring, (void*)tr.stack})
    for (size_t i = 0; i < h.bufs.size(); ++i)
      if (h.bufs[i].p == old) {
        dev_free(ctx, old, h.bufs[i].bytes);
        h.bufs.erase(h.bufs.begin() + i);
        break;
      }
  h.bufs.insert(h.bufs.end(), bufs.begin(), bufs.end());
  tr = nt;
  return GF_OK;
}

void tree_host_release(TreeHost& h) {
  for (auto& b : h.bufs) dev_free(h.ctx, b.p, b.bytes);
  h.bufs.clear();
  h.tree = PfTree();
}

}  // namespace gf
