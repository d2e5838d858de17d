// gf_pf_host.hpp -- host-side pieces of the particle-filter path.
#pragma once
#include <cstdint>
#include <vector>

#include "gf_internal.hpp"

namespace gf {

struct PfJob;

// One compiled (precision, padded dims, proposal) variant of the LG kernels.
struct PfLgKernels {
  int dxp = 0, dyp = 0;
  void (*prop)(const PfJob*, int) = nullptr;
  void (*init)(const PfJob*, int, int, int) = nullptr;
  void (*small)(const PfJob*, int, int, double*) = nullptr;  // whole filter in one block, N <= 1024
  void (*small_means)(const PfJob*, int, int, double*) = nullptr;  // the same with weighted means
  void (*lookahead)(const PfJob*, int) = nullptr;  // auxiliary filter first stage
  size_t smem = 0;
  int params_len = 0, off_mu0 = 0, off_L0 = 0;
  // tensor-core bootstrap propagation (FP32, state dim >= 16), null if none
  void (*prop_tc)(const PfJob*, int) = nullptr;
  size_t tc_smem = 0;
  int tc_nm = 0;
  int tc_split = 1;  // blocks per tile of the tensor-core kernel
  // the same with the staged (bulk-copy) ancestor gather, Dx = 16; null if none
  void (*prop_tc_staged)(const PfJob*, int) = nullptr;
  size_t tc_staged_smem = 0;
  // the same over 128-particle units with a grid of resident blocks
  void (*prop_tc_units)(const PfJob*, int) = nullptr;
  int tc_units_blocks = 0;  // resident blocks per SM
};

// FP64 model factors computed once per plan (column-major).
struct LgFactors {
  int dx = 0, dy = 0;
  std::vector<double> A, L, b, Ht, M, Qi, mu0, L0, LRi, c, K, vb;
  double obs_const = 0.0, prop_const = 0.0;
};

bool pick_lg_kernels(bool dbl, bool guided, int dx, int dy, PfLgKernels* out);
gf_status build_lg_factors(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg,
                           LgFactors* f);
void pack_params(const LgFactors& f, bool dbl, int dxp, int dyp, std::vector<char>& out);
double uniform_ess(int64_t n);

void launch_scan(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_stiles);
void launch_resample(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_tiles);
void launch_init_scalars(gf_ctx* ctx, PfJob* jobs_dev, int njobs, const double* ess1,
                         const int8_t* res1);
void launch_means(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int njobs, int total_tiles,
                  double* mpart, int mdim);
void launch_finish(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int64_t N);
void launch_record(gf_ctx* ctx, bool dbl, const PfJob* jobs_dev, int64_t N);
// the step's finalise after the unit-grid tensor-core propagation
void launch_finish_units(gf_ctx* ctx, const PfJob* jobs_dev, int njobs);
void launch_prep(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int T, int dx, int dy, int dxp,
                 int dyp, const double* pp, void* out);

}  // namespace gf

namespace gf {

// 128-particle units per 1024-particle tile (pf_lg_propagate_tc_units)
constexpr int TC_SUB_UNITS = 8;

// Rao-Blackwellised PF propagation: one particle per thread, RB_SPLIT blocks of
// RB_THREADS threads per 1024-particle tile (its log-sum-exp partials are kept
// per block, so the job's `part` buffer holds ntiles * RB_SPLIT entries).
constexpr int RB_THREADS = 128;
constexpr int RB_SPLIT = 1024 / RB_THREADS;

// Rao-Blackwellised PF kernels of one compiled (dxo, dz, dy).
struct RbKernels {
  int dxo, dz, dy;
  void (*prop)(const PfJob*, int, float, int, int);
  void (*init)(const PfJob*, int);
  void (*lookahead)(const PfJob*, int, float, int);  // auxiliary RBPF first stage
};
bool pick_rb(int dxo, int dz, int dy, RbKernels* out);
gf_status rb_pack_params(gf_ctx* ctx, const gf_rb_model* m, const gf_pf_config* cfg,
                         std::vector<float>& P, double* prop_const);

}  // namespace gf

#include "gf_pf_kernels.cuh"

namespace gf {

// Everything of one linear-Gaussian PF job that does not depend on its device
// buffers: kernels (the propagate variant a plan picks for `flags`), packed
// parameters, the observation-prep block, the step-1 decision and the job
// descriptor's scalar fields.  Plans and the serving loop share it, so a
// served filter computes exactly what a standalone run computes.
struct LgJobSetup {
  bool dbl = false;
  PfLgKernels k;
  void (*prop)(const PfJob*, int) = nullptr;
  int threads = 0;
  int split = 1;  // propagate blocks per tile (grid = tiles * split)
  int units_blocks = 0;  // > 0: unit kernel, grid = min(units, SMs * units_blocks)
  size_t smem = 0;
  std::vector<char> params;      // parameter blocks (one per step if time-varying)
  std::vector<double> pp;        // observation-prep factors (likewise)
  std::vector<double> obs_consts;  // time-varying: observation and proposal constants of every step
  int64_t pstride = 0;           // time-varying: elements between parameter blocks
  int32_t ppstride = 0;          // time-varying: doubles between prep blocks
  double ess1 = 0.0;
  int8_t res1 = 0;
  PfJob J;
};
// param_steps: 1 for a homogeneous model, >= T when the A, b, Q, H, c, R
// pointers of m hold one block per step (bootstrap proposal only).
gf_status lg_job_setup(gf_ctx* ctx, const gf_lg_model* m, const gf_pf_config* cfg, int32_t T,
                       int32_t flags, LgJobSetup* out, int32_t param_steps = 1);

}  // namespace gf

namespace gf {

// Device path storage of one particle-filter run (AncestorCallback /
// ParticleTree, callbacks.jl:90-111 and containers.jl:466-631; the GPU
// ParallelParticleTree of ext/CUDAExt.jl:146-298): a pool of M slots holding
// particle states with parent links and live-descendant counts.  Each step the
// lineages that left no offspring are freed (walking up while a parent's count
// drops to zero) and the new particles take freed slots.
struct PfTree {
  int64_t M = 0;              // slots
  int32_t width = 0;          // state dimensions
  void* states = nullptr;     // [M][width] (run precision; one particle's state contiguous)
  int32_t* parents = nullptr;    // [M] parent slot, -1 for time-0 states
  int32_t* offspring = nullptr;  // [M] live children
  int32_t* stack = nullptr;      // [M] free slots
  int32_t* top = nullptr;        // [1] number of free slots on the stack
  int32_t* leaves = nullptr;     // [N] slots of the current particles
  int32_t* new_leaf = nullptr;   // [N] slots taken by the next generation
  int32_t* anc = nullptr;        // [N] 0-based ancestors of the step being inserted
  int32_t* cnt = nullptr;        // [N] offspring counts of the current particles
};

// Host side of a run's path storage: the tree and the device buffers it holds.
// Set ctx, N, width and rsize (bytes per state element) before the first
// tree_host_prepare; the pool grows between chunks of steps.
struct TreeHost {
  gf_ctx* ctx = nullptr;
  int64_t N = 0;
  int width = 0;
  size_t rsize = 4;
  PfTree tree;
  std::vector<DevBuf> bufs;
};
constexpr int kTreeChunk = 32;  // steps between host checks of the free-slot count
gf_status tree_host_prepare(TreeHost& h);
gf_status tree_host_reserve(TreeHost& h, int64_t need);
void tree_host_release(TreeHost& h);

// Launchers (stream of ctx).  Before step t's propagate: count / prune / assign;
// after it: insert.  tree_paths writes [T+1][width][N].
void tree_launch_init(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr);
// sorted_ancestors: the rule keeps ancestors nondecreasing (systematic, stratified)
void tree_launch_step_pre(gf_ctx* ctx, const PfJob* job_dev, int64_t N, const PfTree& tr,
                          bool sorted_ancestors);
void tree_launch_insert(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr, int t);
void tree_launch_paths(gf_ctx* ctx, bool dbl, const PfJob* job_dev, int64_t N, const PfTree& tr, int T,
                       void* out);
// Grows the pool from tr.M to M_new slots (new arrays from `alloc`, old ones to `release`).
void tree_launch_grow_init(gf_ctx* ctx, const PfTree& tr_new, int64_t M_old, int32_t top_old);

}  // namespace gf
