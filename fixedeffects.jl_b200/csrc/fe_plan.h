// fe_plan.h -- the solver plan: the device-resident replacement of the
// reference's AbstractFixedEffectSolver{T}(fes, w, Val{:CUDA}) object
// (ext/CUDAExt.jl:86-121).  Internal; the C ABI is include/fe_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "fe_internal.h"

struct fe_plan;

namespace fe {

// thread-local last error (fe_last_error)
void set_error(const std::string& msg);
void set_error_cstr(const char* msg);
const char* last_error();

#define FE_CK(call)                                                                     \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      (void)cudaGetLastError();                                                         \
      ::fe::set_error(std::string("CUDA error ") + cudaGetErrorString(e_) + " at " +    \
                      __FILE__ + ":" + std::to_string(__LINE__) + " (" #call ")");      \
      return 2; /* FE_ERR_CUDA */                                                       \
    }                                                                                   \
  } while (0)

// The caller's current device, saved when an entry point starts and put back
// on every return path.  A host binding such as CUDA.jl tracks its own
// current device per task; the library switches to the plan's device for its
// work and must not leave that switch behind.  With no usable device nothing
// is saved and nothing is restored.
struct DeviceRestore {
  int saved = -1;
  DeviceRestore() {
    if (cudaGetDevice(&saved) != cudaSuccess) {
      (void)cudaGetLastError();
      saved = -1;
    }
  }
  ~DeviceRestore() {
    if (saved < 0) return;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != saved) {
      if (cudaSetDevice(saved) != cudaSuccess) (void)cudaGetLastError();
    }
  }
  DeviceRestore(const DeviceRestore&) = delete;
  DeviceRestore& operator=(const DeviceRestore&) = delete;
};

// fe_exchange_fn of include/fe_b200.h: in-place sum over ranks of `count`
// elements (0: FP64, 1: FP32) at device address `buf`, ordered on `stream`.
using ExchangeFn = int (*)(void* ctx, void* buf, int64_t count, int32_t dtype, void* stream);
// calls the plan's exchange (a no-op for plans that are not sharded)
int exchange(fe_plan* pl, void* buf, int64_t count, int elem_bytes, cudaStream_t s);

// An NVTX range around a host phase of the library (plan build, a solve,
// a column tile, a refinement round, an LSMR loop), visible on the timeline
// of a profiler (Nsight Systems); without a profiler attached the calls
// return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// A device allocation owned by the plan.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf();
  int ensure(size_t n);  // grows (contents not preserved)
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Work items for one column-tile width C.
struct ItemSet {
  int C = 0;
  std::vector<ExpandItem> ex;
  std::vector<ReduceItem> rd;
  std::vector<SplitLevel> splits;      // level pieces of the segsum items
  std::vector<SplitLevel> ex_splits;   // primary-level pieces of the expand items
  // segsum items are ordered [large non-primary FEs | small FEs | primary FE];
  // the row-sum pass (32-column tiles of single-problem plans) reduces the last two
  // groups itself, so the segsum then runs only the first rd_large items
  int64_t rd_large = 0;
  int64_t rd_np = 0;                   // items of non-primary FEs (first)
  uint32_t small_mask = 0;             // FEs reduced in the row-sum tables
  int32_t small_rows = 0;              // table rows (levels + null level)
  int32_t small_off[kMaxFE] = {};      // first table row of each small FE
  std::vector<int64_t> small_slab_row; // [P][C] slab row of each table row
  int sms = 148;                       // multiprocessors of the plan's device
  int64_t ex_n_pieces = 0;
  std::vector<PItem> pu;
  int64_t pu_np = 0;                   // leading P-side items of the non-primary FEs
  int64_t Sp_np = 0;                   // their norm slots
  std::vector<ExpandItem> dm;          // demean items (absorbed-primary mode)
  // batch plans (absorbed mode on narrow tiles): demean items padded per
  // problem to whole CTAs of dm_ipc items, one norm slot per CTA; the P-side
  // items of the non-primary FEs as a list of their own, padded likewise
  int64_t dm_ipc = 0;                  // 0: single problem, grid-stride walk
  int64_t Sdm = 0;                     // demean norm slots (batch plans)
  std::vector<int64_t> dm_slot_off;    // per problem (batch plans)
  std::vector<PItem> pu_abs;           // batch plans' non-primary P-side items
  std::vector<int64_t> pu_abs_slot_off;
  std::vector<int64_t> ex_slot_off;       // per problem, expand norm slots (CTAs)
  std::vector<int64_t> pu_slot_off;       // per problem, P-side norm slots (CTAs)
  int64_t n_pieces = 0, n_blocks = 0;
  int64_t ex_n_blocks = 0;
  int64_t Se = 0, Sp = 0;                 // slot counts
  DevBuf d_ex, d_rd, d_splits, d_pu, d_ex_off, d_pu_off, d_split_cnt, d_block_cnt;
  DevBuf d_ex_splits, d_ex_split_cnt, d_ex_block_cnt;
  DevBuf d_pu_off_np, d_dm;
  DevBuf d_dm_off, d_pu_abs;
};

struct Workspace {
  int C = 0;
  DevBuf B64, R64, U, V, H, Hb, X, X64, S;
  DevBuf VS;  // scale * v, the fused absorbed loop's coefficient table (FP32)
  DevBuf XS64;  // (x64 + dx32) * scale, the FP64 residual's coefficient table
  DevBuf part_e, part_a, part_b, piece_part, ex_piece_part, block_part, ex_block_part, inst,
      counters;
  DevBuf small_part;  // the row-sum CTA partials of the small FEs
  DevBuf coef;
  DevBuf ystage;  // device copy of host Y for host-buffer solves
  DevBuf xbuf;    // sharded plans: per-column norms exchanged over the ranks
  DevBuf off01;   // sharded plans: the slot range {0, 1} of xbuf
};

// A captured run of LSMR iterations (the inner loop of one tile shape).
struct LoopGraph {
  cudaGraphExec_t exec = nullptr;
  size_t key = 0;  // fingerprint of everything the captured launches use
};

struct Profile {
  bool on = false;
  std::map<std::string, KernelStat> stats;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> pool;
  std::map<std::string, double> bytes_per_launch;
};

}  // namespace fe

struct fe_plan {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  int64_t N = 0;
  int32_t K = 0;
  int32_t nprob = 1;
  int32_t primary = 0;
  // the primary FE can be projected out of every problem: one problem with
  // 2+ FEs, or a batch whose problems all hold the primary FE and another
  bool absorbable = false;
  bool weighted = false;
  std::vector<bool> interacted;
  std::vector<int64_t> nlev;           // per FE: total levels over problems
  std::vector<int64_t> prob_obs_off;   // nprob+1
  std::vector<int64_t> prob_lev_off;   // [(nprob+1) * K]: first global level of problem p in FE k
  std::vector<int32_t> prob_nfe;       // FEs present in each problem
  std::vector<int64_t> lev_base;       // per FE, row base in [P][C] slabs
  int64_t P = 0;                       // slab rows (levels + one null level per FE)
  std::vector<std::vector<int64_t>> seg_off;  // per FE: level-order offsets (host)
  std::vector<int64_t> seg_len;        // per FE: positions in level order

  // device integer plan
  fe::DevBuf d_obs_src, d_obs_dst;     // sorted -> original, original -> sorted
  std::vector<fe::DevBuf> d_refs, d_perm, d_key;
  std::vector<bool> perm_identity;
  // device weights/interaction/preconditioner
  fe::DevBuf d_sw_orig, d_sw_sorted;
  std::vector<fe::DevBuf> d_inter_sorted;
  std::vector<fe::DevBuf> d_scale_d, d_scale_f, d_cw_d, d_cw_f, d_cwp_d, d_cwp_f;
  // absorbed-primary mode: per non-primary FE, 1 / ||M a_l|| (the column norms
  // of the operator the absorbed LSMR runs on; empty for the primary FE)
  std::vector<fe::DevBuf> d_abs_scale_d, d_abs_scale_f;

  fe::FeDev dev{};                     // device view (C patched per launch)

  // options
  int32_t opt_tile = 0;        // 0 = automatic
  int32_t opt_check_every = 4; // iterations between host convergence checks
  int32_t opt_max_rounds = 8;  // mixed-precision refinement rounds
  int32_t opt_unroll = 0;      // reserved
  double opt_inner_rho = 1e-8;
  double opt_inner_theta = 0.5;
  int32_t opt_fuse = 1;        // row-sum pass: primary and small FEs reduced contiguously
  int32_t opt_ex_variant = -1; // expand kernel variant (-1: tuned default)
  int32_t opt_seg_variant = -1; // segsum kernel variant (-1: tuned default)
  int32_t opt_autotune = 1;     // time the variants on first use of a tile shape
  int32_t opt_mixed_warm = 1;   // mixed precision starts from x0 = A'b (else x0 = 0)
  int32_t opt_graph = 1;        // replay the LSMR iterations from a CUDA graph
  int32_t opt_rowsum_variant = -1; // row-sum pass: 0 shared-memory ring, 1 registers
  int32_t opt_absorb = 1;       // mixed residual solves project the primary FE out
  int32_t opt_exdm = 1;         // absorbed loop: fused expand + demean kernel
  int32_t opt_fused_resid = -1;  // absorbed refinement: FP64 residual + projection in one kernel
  int32_t opt_abs_scale = 1;    // absorbed loop: columns scaled by 1 / ||M a_l||
  int32_t opt_exdm_pipe = -1;   // absorbed loop: pipelined fused kernel (-1 default, 0 off, 1.. cfg)
  int32_t opt_firm_atomic = 0;  // absorbed loop: gathered FE's sums by reductions (-1 tuned, 0, 1)
  float last_firm_tune_ms[2] = {0.f, 0.f};  // the tuner's times: segmented sum, reductions
  std::map<std::pair<int, int>, fe::LoopGraph> graphs;  // by (C, precision)
  // tuned variants per (tile width C, element size): {expand, segsum}
  std::map<std::pair<int, int>, std::pair<int, int>> tuned;
  std::string tune_signature;   // plan shape, key of the persisted tuning cache

  std::map<int, std::unique_ptr<fe::ItemSet>> items;  // by C
  fe::Workspace ws;
  fe::Profile prof;
  void* host_pinned = nullptr;  // small pinned staging for counters
  // fe_plan_scales_noalloc on a caller stream: orders it after the plan's stream
  cudaEvent_t noalloc_order = nullptr;
  // pinned staging rings of pageable host-buffer solves (fe_staging.cu)
  void* ring_up = nullptr;
  void* ring_down = nullptr;
  size_t ring_slot_bytes = 0;
  // observation-sharded plans: the sum-over-ranks exchange (fe_exchange_fn)
  fe::ExchangeFn xchg = nullptr;
  void* xchg_ctx = nullptr;

  // results of the last solve (per column)
  std::vector<double> last_test2;
  std::vector<int32_t> last_rounds;
  std::vector<int64_t> last_iters_raw;
  std::vector<int64_t> last_prob_iters;
  std::vector<uint8_t> last_prob_conv;
};

namespace fe {
int plan_build(fe_plan* pl, int32_t nprob, const int64_t* n_obs, int32_t K,
               const int64_t* const* refs, const int64_t* n_levels,
               const double* const* interaction, const double* weights, int32_t device);
int plan_update_weights(fe_plan* pl, const double* weights);
// the integer plan and the interactions in sorted order, built on the device
int plan_build_device(fe_plan* pl, const int64_t* const* refs, const int64_t* n_levels,
                      const double* const* interaction);
int plan_items(fe_plan* pl, int C, ItemSet** out);
int plan_destroy(fe_plan* pl);
}  // namespace fe
