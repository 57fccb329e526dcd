// fe_internal.h -- shared host/device definitions of the B200 fixed-effects
// LSMR library.  Nothing here is part of the C ABI (include/fe_b200.h is).
//
// Terminology follows FixedEffects.jl: an observation has one level ("ref")
// per fixed effect (FE); the design matrix A = D' diag(scale) has one column
// per level and one row per observation.
//   expand  (A x):  per observation, sum over FEs of cache * x[ref]
//                   (the reference's scatter!, src/SolverCPU.jl:29-34)
//   reduce  (A' u): per level, sum over its observations of cache * u
//                   (the reference's gather!, src/SolverCPU.jl:21-27)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace fe {

// cudaFuncSetAttribute applies to the device that is current when it is
// called, so a kernel's one-time attribute settings are recorded per device:
// one bit per device index below kDeviceSlots (higher indices make the
// setting on every launch).  Two threads may both make the same setting,
// which is harmless.
constexpr int kDeviceSlots = 64;
struct PerDeviceOnce {
  std::atomic<uint64_t> bits{0};
  bool needed(int dev) const {
    return dev < 0 || dev >= kDeviceSlots ||
           !((bits.load(std::memory_order_acquire) >> dev) & 1u);
  }
  void done(int dev) {
    if (dev >= 0 && dev < kDeviceSlots)
      bits.fetch_or(uint64_t(1) << dev, std::memory_order_acq_rel);
  }
};

// The device current on the calling host thread (0 if it cannot be read).
inline int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    (void)cudaGetLastError();
    d = 0;
  }
  return d;
}

constexpr int kMaxFE = 8;          // fixed effects per plan
constexpr int kWarps = 8;          // warps per CTA in the expand/reduce kernels
constexpr int kThreads = kWarps * 32;
constexpr int kScalarThreads = 256;
constexpr int kSentinel = 0x7fffffff;  // "no level" key
constexpr int kSmallRows = 32;         // rows of the row-sum pass's small-FE tables
constexpr int kRowSumSmallFE = 2;      // small FEs the row-sum pass reduces
constexpr int64_t kDemeanRows = 32;    // rows per demean item (whole primary levels)
constexpr int64_t kDemeanIpc = 128;    // demean items per CTA of a batch plan (16 per warp)

// A contiguous range of observations (sorted order) processed by one warp.
// Items hold whole levels of the primary FE (the FE that orders the
// observations), so the expand can also reduce that FE; split >= 0 marks one
// piece of a primary level too long for one warp.
struct ExpandItem {
  int64_t ib, ie;
  int32_t prob;
  int32_t split;
  int32_t piece;
  int32_t pad;
};

// A contiguous range of positions in one FE's level order processed by one
// warp.  split < 0: the range holds whole levels.  split >= 0: the range is one
// piece of a level too long for one warp; split is the global piece index.
struct ReduceItem {
  int64_t pb, pe;
  int32_t fe;
  int32_t prob;
  int32_t split;
  int32_t pad;
};

// A contiguous range of [P][C] slab rows (levels of one FE and one problem)
// streamed by one warp in the per-level epilogue.
struct PItem {
  int64_t rb, re;
  int32_t fe;
  int32_t prob;
};

// A level cut into pieces, combined in two deterministic stages: the pieces
// form blocks of kSplitBlock; the last piece of a block to finish sums the
// block's pieces in piece order, and the last block to finish sums the block
// partials in block order and stores the level.  (Integer counters decide who
// is last; the summation order does not depend on it.)
constexpr int kSplitBlock = 32;
struct SplitLevel {
  int32_t first_piece;
  int32_t npieces;
  int32_t fe;
  int32_t level;        // FE-local level id
  int32_t first_block;  // index of its first block in the block arrays
  int32_t nblocks;
};

// Scratch of the split-level combine (per launch list).
struct SplitArgs {
  const SplitLevel* splits;
  double* piece_part;   // [C][n_pieces]
  int64_t n_pieces;
  double* block_part;   // [C][n_blocks]
  int64_t n_blocks;
  int32_t* level_cnt;   // per split level
  int32_t* block_cnt;   // per block
};

// Device-side view of a plan (passed by value to kernels).
struct FeDev {
  int32_t K;
  int32_t C;  // column tile width the P-side slabs are laid out for
  int64_t N;
  int64_t P;  // total levels over all FEs (+ one null level per FE)
  const int32_t* refs[kMaxFE];   // sorted observation order -> FE-local level
  const int32_t* perm[kMaxFE];   // level-order position -> sorted observation
  const int32_t* key[kMaxFE];    // level-order position -> FE-local level
  const float* scale_f[kMaxFE];  // FE-local level -> Jacobi scale
  const double* scale_d[kMaxFE];
  const float* cw_f[kMaxFE];     // sorted order: interaction*sqrt(w), or null
  const double* cw_d[kMaxFE];
  const float* cwp_f[kMaxFE];    // level order: interaction*sqrt(w), or null
  const double* cwp_d[kMaxFE];
  int64_t lev_base[kMaxFE];      // first row of FE k in a [P][C] slab
  int32_t primary;               // FE whose levels order the observations
  // set inside the LSMR loop only: the number of instances still running
  // (written by the scalar kernel's beta phase, and by the refinement phase
  // that starts an inner solve); the reductions return at once when it is 0,
  // so the iterations that finish a replayed chunk after every instance has
  // stopped cost launches only
  const int32_t* active;
  // the same count for kernels that run before the beta phase (the demean
  // and the fused expand + demean of the absorbed loop): the alpha phase of
  // the previous iteration, or the refinement phase, has just written it
  const int32_t* active_pre;
  // absorbed-primary mode: the expand leaves out the primary FE (its effect is
  // projected out of the rows by the demean pass instead)
  int32_t absorb;
};

// LSMR state of one instance (problem p, column j).  Scalars are FP64 in every
// precision mode.  The recurrence restates src/utils/lsmr.jl:46-222.
struct Inst {
  double atol, btol, ctol;
  int64_t maxiter;
  // recurrence
  double alpha, beta, alphabar, rho, rhobar, cbar, sbar, zeta, zetabar;
  double betadd, betad, rhodold, tautildeold, thetatilde, d;
  double normA2, normA, condA, maxrbar, minrbar, normb, normr, normAr, normx;
  double u_scale;  // stored U = u * (1/u_scale)
  double s_v;      // stored V = v * (1/s_v)
  int64_t iter;
  int32_t istop;
  int32_t active;   // LSMR loop still running
  int32_t pending;  // test of iteration `iter` awaits ||x||
  int32_t do_v;     // reduce updates V this iteration
  int32_t upd_mode; // deferred h/hbar/x update: 0 none, 1 init, 2 normal
  int32_t pad0;
  // kernel coefficients
  double ex_av, ex_au;  // expand: U <- ex_av * (A V) + ex_au * U
  double rd_acc, rd_v;  // reduce: V <- rd_acc * (A'U) - rd_v * V
  double c1, c2, c3;    // deferred: hbar<-h+c1 hbar; x<-x+c2 hbar; h<-v+c3 h
  // mixed-precision refinement
  double normA2_prev;   // sum of normA^2 of earlier inner solves
  double normAr0;       // ||A'r|| at the start of this inner solve
  double inner_theta_tol; // stop when normAr <= theta*tol*normA_tot*normr
  double inner_rho;       // ... or when normAr <= rho*normAr0
  double normb0;        // ||b - A x0|| of the first residual (outer test1)
  double tol_a, tol_b;  // outer (FP64) tolerances of the mixed mode
  double last_test2;    // FP64 ||A'r|| / (||A|| ||r||) at the last outer test
  int64_t maxiter_total;
  int64_t iter_total;   // LSMR iterations over all inner solves
  int32_t outer_active; // refinement still running
  int32_t outer_rounds;
  int32_t max_rounds;
  int32_t converged;    // final verdict
  int32_t mode_inner;   // 1: inner solve of the mixed mode
  int32_t skip_lsmr;    // single FE in solve_residuals!: x = A'b is exact
};

struct ScalarArgs {
  Inst* inst;
  int32_t C;
  int32_t phase;
  int32_t init_mode;  // PH_INIT_ALPHA: 1 keep x, 3 zero x
  int32_t pad;
  const double* part0;  // expand slots
  const int64_t* off0;
  int64_t S0;
  const double* part1;  // P-side slots (||v||^2 or ||g||^2)
  const double* part2;  // P-side slots (||x||^2)
  const int64_t* off1;
  int64_t S1;
  int32_t* counters;    // [0] LSMR-active instances, [1] refinement-active
};

void launch_scalar(const ScalarArgs& a, int n_inst, cudaStream_t s);

enum ScalarPhase : int32_t {
  PH_INIT_BETA = 0,
  PH_INIT_ALPHA = 1,
  PH_BETA = 2,
  PH_ALPHA = 3,
  PH_INIT_MIXED = 4,
  PH_OUTER = 5,
  PH_FINISH_PLAIN = 6,
};

// Per-kernel launch statistics kept when profiling is on.
struct KernelStat {
  std::string name;
  int64_t launches = 0;
  double ms = 0.0;
  double bytes = 0.0;  // algorithmic bytes
  std::vector<float> times;  // CUDA-event milliseconds of every launch
};

}  // namespace fe
