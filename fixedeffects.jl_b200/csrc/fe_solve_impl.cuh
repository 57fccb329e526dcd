// fe_solve_impl.cuh -- solve drivers of the fixed-effects LSMR hot path.
// Included by one translation unit per column-tile width (fe_tile_c*.cu),
// which instantiates solve_tile_C<C>; fe_solve.cu dispatches on C.
//
// Replaces, for one plan, the bodies of
//   solve_residuals!(r, feM)     src/AbstractFixedEffectSolver.jl:49-68
//   solve_residuals!(xs, feM)    src/AbstractFixedEffectSolver.jl:74-97
//   solve_coefficients!(r, feM)  src/AbstractFixedEffectSolver.jl:147-160
// with all columns of a tile (and all problems of a batch plan) advanced as
// one batched LSMR; every instance has its own FP64 scalars and stops on its
// own test.
//
// Precision modes:
//   FP64  : bulk FP64, the plain form of the reference's Float64 solver.
//   FP32  : bulk FP32 (FP64 scalars), no refinement.
//   MIXED : FP32 inner LSMR solves on correction problems; the residual
//           r = b - A x and g = A'r are recomputed in FP64 between them and
//           tested with the reference's tests (FP64 iterative refinement).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#pragma once
#include "fe_exdm_pipe.cuh"
#include "fe_kernels.cuh"
#include "fe_plan.h"
#include "fe_solve.h"

namespace fe {

// ---------------------------------------------------------------------------
// load / unload / coefficient kernels
// ---------------------------------------------------------------------------
// B[q][j] = y[i][col0 + j] * sqrt(w_i) with q the sorted position of i
// (src/AbstractFixedEffectSolver.jl:50-55).  A CTA stages load_rows<C>()
// observations x C columns (2048 elements, 8 per thread, for every tile
// width) in shared memory: the reads are coalesced along observations
// (column-major input), the writes are whole contiguous rows.  Every thread
// issues all its loads before the first shared-memory store, so 16 KB per CTA
// are in flight.  C is a compile-time power of two (index splits are shifts)
// and W says whether there are weights (without, no multiply or divide by
// sqrt(w) = 1).
constexpr int kLoadElems = 2048;  // elements per CTA
constexpr int kLoadPer = kLoadElems / 256;
template <int C> constexpr int load_rows() { return kLoadElems / C; }
// the row padding of the staged tile (none for one column, whose accesses
// run along rows in both phases)
template <int C> constexpr int load_pad() { return C == 1 ? 0 : 1; }
template <typename TY, int C, bool W>
__global__ void __launch_bounds__(256) k_load(const TY* __restrict__ Y, int64_t ld, int64_t col0,
                                              int ncols, const int32_t* __restrict__ dst,
                                              const double* __restrict__ sw,
                                              double* __restrict__ B, int64_t N) {
  constexpr int R = load_rows<C>();
  __shared__ double tile[R][C + load_pad<C>()];
  __shared__ int32_t rows[R];
  const int64_t i0 = (int64_t)blockIdx.x * R;
  // load phase: element e = t + 256 u in column-major order (column e / R,
  // row e % R)
  double v[kLoadPer];
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    const int j = e / R, r = e % R;
    const int64_t i = i0 + r;
    double x = 0.0;
    if (i < N && j < ncols) {
      x = (double)Y[i + (col0 + j) * ld];
      if (W) x *= sw[i];
    }
    v[u] = x;
  }
  for (int r = threadIdx.x; r < R; r += 256) rows[r] = (i0 + r < N) ? dst[i0 + r] : -1;
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    tile[e % R][e / R] = v[u];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    const int rr = e / C, j = e % C;
    const int32_t q = rows[rr];
    if (q >= 0) B[(int64_t)q * C + j] = tile[rr][j];
  }
}

// The same for tiles of 1 or 2 columns, whose sorted rows are shorter than a
// 32-byte sector: gathered through the inverse permutation (src: sorted
// position -> observation; sw_sorted: sqrt(w) in sorted order), so the rows
// are written whole and in order and the random reads of y fall in L2,
// instead of scattering partial-sector writes.
template <typename TY, int C, bool W>
__global__ void __launch_bounds__(256) k_load_gather(const TY* __restrict__ Y, int64_t ld,
                                                     int64_t col0, int ncols,
                                                     const int32_t* __restrict__ src,
                                                     const double* __restrict__ sw_sorted,
                                                     double* __restrict__ B, int64_t N) {
  static_assert(C <= 2, "narrow rows");
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const int64_t i = src[q];
  const double s = W ? sw_sorted[q] : 1.0;
#pragma unroll
  for (int j = 0; j < C; ++j) {
    const double x = j < ncols ? (double)Y[i + (col0 + j) * ld] : 0.0;
    B[q * C + j] = W ? x * s : x;
  }
}

// y[i][col0 + j] = R[q][j] / sqrt(w_i)  (src/AbstractFixedEffectSolver.jl:62-66):
// whole rows in (all of a thread's row loads issued before the first
// shared-memory store), coalesced columns out.
template <typename TY, int C, bool W>
__global__ void __launch_bounds__(256) k_unload(const double* __restrict__ Rw, int64_t ld,
                                                int64_t col0, int ncols,
                                                const int32_t* __restrict__ dst,
                                                const double* __restrict__ sw,
                                                TY* __restrict__ Y, int64_t N) {
  constexpr int R = load_rows<C>();
  __shared__ double tile[R][C + load_pad<C>()];
  const int64_t i0 = (int64_t)blockIdx.x * R;
  double v[kLoadPer];
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    const int rr = e / C, j = e % C;
    const int64_t i = i0 + rr;
    v[u] = i < N ? Rw[(int64_t)dst[i] * C + j] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    tile[e / C][e % C] = v[u];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < kLoadPer; ++u) {
    const int e = threadIdx.x + u * 256;
    const int j = e / R, r = e % R;
    const int64_t i = i0 + r;
    if (i < N && j < ncols) {
      const double x = tile[r][j];
      Y[i + (col0 + j) * ld] = (TY)(W ? x / sw[i] : x);
    }
  }
}

// coefficients in original units: x_k .* scale_k  (src/AbstractFixedEffectSolver.jl:155-157)
template <typename TX>
__global__ void k_coefs(const TX* __restrict__ X, int C, int j, int64_t base, int64_t n,
                        const double* __restrict__ scale, double* __restrict__ out) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n) out[l] = (double)X[(base + l) * C + j] * scale[l];
}

static inline unsigned grid1(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// ---------------------------------------------------------------------------
// profiling: CUDA events around launches on the plan's stream
// ---------------------------------------------------------------------------
struct ProfScope {
  fe_plan* pl;
  const char* name;
  double bytes;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(fe_plan* p, const char* n, double by) : pl(p), name(n), bytes(by) {
    if (!pl->prof.on) return;
    a = take();
    b = take();
    cudaEventRecord(a, pl->stream);
  }
  cudaEvent_t take() {
    if (!pl->prof.pool.empty()) {
      cudaEvent_t e = pl->prof.pool.back();
      pl->prof.pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  ~ProfScope() {
    if (!pl->prof.on) return;
    cudaEventRecord(b, pl->stream);
    pl->prof.pending.push_back({name, {a, b}});
    pl->prof.bytes_per_launch[name] = bytes;
  }
};


// ---------------------------------------------------------------------------
// solve context for one tile
// ---------------------------------------------------------------------------
struct Ctx {
  fe_plan* pl;
  ItemSet* its;
  FeDev d;
  int C;
  cudaStream_t s;
  Inst* inst;
  int32_t* counters;
  int32_t* h_counters;
  int n_inst;
  double* part_e;
  double* part_a;
  double* part_b;
  double* piece;
  double* ex_piece;
  void* S;
  SplitArgs seg_split() const {
    return SplitArgs{its->d_splits.as<SplitLevel>(), piece, its->n_pieces, block, its->n_blocks,
                     its->d_split_cnt.as<int32_t>(), its->d_block_cnt.as<int32_t>()};
  }
  SplitArgs ex_split() const {
    return SplitArgs{its->d_ex_splits.as<SplitLevel>(), ex_piece, its->ex_n_pieces, ex_block,
                     its->ex_n_blocks, its->d_ex_split_cnt.as<int32_t>(),
                     its->d_ex_block_cnt.as<int32_t>()};
  }
  double* block;
  double* ex_block;
  double* small_part;  // the row-sum pass's CTA partials of the small FEs
  bool rowsum;         // primary and small FEs reduced by the row-sum pass
  bool absorb = false; // primary FE projected out (demean pass; mixed residual solves)
  // absorbed loop: the gathered FE's level sums by vector reductions inside
  // the pipelined kernel (no level-order segmented sum)
  bool firm_atomic = false;
  // observation-sharded plans: per-column norms summed over the ranks, read
  // by the scalar phases as one slot per column
  double* xbuf = nullptr;
  const int64_t* off01 = nullptr;
};

// ---------------------------------------------------------------------------
// observation-sharded plans: the exchange steps (no-ops otherwise)
// ---------------------------------------------------------------------------
// per-column totals of the [C][S] norm slots, summed in slot order (one CTA
// per column, a fixed reduction tree)
static __global__ void __launch_bounds__(256) k_slot_totals(const double* __restrict__ part, int64_t S,
                                                     double* __restrict__ out) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  double t = 0.0;
  for (int64_t q = threadIdx.x; q < S; q += 256) t += part[(int64_t)j * S + q];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0];
}

// the norms of this rank's rows -> summed over the ranks (xbuf)
static int xchg_slots(Ctx& c, const double* part) {
  if (!c.pl->xchg) return 0;
  k_slot_totals<<<c.C, 256, 0, c.s>>>(part, c.its->Se, c.xbuf);
  FE_CK(cudaGetLastError());
  return exchange(c.pl, c.xbuf, c.C, 8, c.s);
}

// slab rows exchanged: every FE's, or the non-primary FEs' in the absorbed
// mode (the primary levels are this rank's own)
static void slab_ranges(const Ctx& c, std::vector<std::pair<int64_t, int64_t>>& out) {
  const fe_plan* pl = c.pl;
  out.clear();
  if (!c.absorb) {
    out.push_back({0, pl->P});
    return;
  }
  const int64_t pb = pl->lev_base[pl->primary], pe = pb + pl->nlev[pl->primary] + 1;
  if (pb > 0) out.push_back({0, pb});
  if (pe < pl->P) out.push_back({pe, pl->P});
}
// zeroed before the reductions (rows without local positions stay 0 instead
// of keeping the last exchanged sums) ...
static int zero_slab(Ctx& c, void* S, int elem) {
  if (!c.pl->xchg) return 0;
  std::vector<std::pair<int64_t, int64_t>> r;
  slab_ranges(c, r);
  for (const auto& q : r)
    FE_CK(cudaMemsetAsync(static_cast<char*>(S) + (size_t)q.first * c.C * elem, 0,
                          (size_t)(q.second - q.first) * c.C * elem, c.s));
  return 0;
}
// ... and summed over the ranks after them
static int xchg_slab(Ctx& c, void* S, int elem) {
  if (!c.pl->xchg) return 0;
  std::vector<std::pair<int64_t, int64_t>> r;
  slab_ranges(c, r);
  for (const auto& q : r) {
    const int st = exchange(c.pl, static_cast<char*>(S) + (size_t)q.first * c.C * elem,
                            (q.second - q.first) * c.C, elem, c.s);
    if (st) return st;
  }
  return 0;
}

// Kernel variants (unroll depth = row slots per lane group per step, and
// whether the next step's indices are prefetched).  Variant 0 is the default;
// fe_plan_set_option(FE_OPT_EXPAND_VARIANT / FE_OPT_SEGSUM_VARIANT) selects
// another, which is how the tuner compares them.
//   expand: 0 U=2 PF, 1 U=4 PF, 2 U=2 no-PF, 3 U=4 no-PF,
//           4 U=2 PF of refs and old rows, 5 U=4 PF of refs and old rows
//   segsum: 0 U=8 no-PF, 1 U=4 PF, 2 U=8 PF, 3 U=4 no-PF,
//           4 cp.async ring U=4 x 4 stages, 5 cp.async ring U=2 x 6 stages
constexpr int kVariants = 6;
constexpr int kSegVariants = 6;
template <int C> struct Tune {
  static constexpr int kPU = 4;
};
// tuning state of the tile being solved
// tuning state of the tile being solved, per element size (0: FP32, 1: FP64)
struct TuneSel {
  int ex[2] = {-1, -1}, seg[2] = {-1, -1};
};
inline TuneSel& cur_tune() {
  static thread_local TuneSel t;
  return t;
}
inline int pick_ex(const fe_plan* pl, size_t elem) {
  const int t = cur_tune().ex[elem == 8 ? 1 : 0];
  return pl->opt_ex_variant >= 0 ? pl->opt_ex_variant : (t >= 0 ? t : 0);
}
inline int pick_seg(const fe_plan* pl, size_t elem) {
  const int t = cur_tune().seg[elem == 8 ? 1 : 0];
  return pl->opt_seg_variant >= 0 ? pl->opt_seg_variant : (t >= 0 ? t : 0);
}
template <typename T, int C> constexpr int vec_of() { return Shape<T, C>::VEC; }

template <int KB, int U, int PF, typename TA, int C, class Tab, class Epi>
static int expand_kbu(Ctx& c, Tab tab, Epi epi, double* part) {
  const unsigned grid = (unsigned)(c.its->ex.size() / kWarps);
  const ExpandItem* items = c.its->d_ex.as<ExpandItem>();
  const int64_t n = (int64_t)c.its->ex.size();
  k_expand<TA, C, U, KB, PF, Tab, Epi><<<grid, kThreads, 0, c.s>>>(c.d, items, n, tab, epi, part,
                                                                   c.its->Se);
  FE_CK(cudaGetLastError());
  return 0;
}

template <int KB, typename TA, int C, class Tab, class Epi>
static int expand_kb(Ctx& c, Tab tab, Epi epi, double* part) {
  const int var = pick_ex(c.pl, sizeof(TA));
  switch (var) {
    case 1: return expand_kbu<KB, 4, 1, TA, C>(c, tab, epi, part);
    case 2: return expand_kbu<KB, 2, 0, TA, C>(c, tab, epi, part);
    case 3: return expand_kbu<KB, 4, 0, TA, C>(c, tab, epi, part);
    case 4: return expand_kbu<KB, 2, 2, TA, C>(c, tab, epi, part);
    case 5: return expand_kbu<KB, 4, 2, TA, C>(c, tab, epi, part);
    default: return expand_kbu<KB, 2, 1, TA, C>(c, tab, epi, part);
  }
}

// The FP64 residual's coefficient table: (x64 + dx32) .* scale for every FE
// the expand gathers (all but the primary when it is absorbed), once per
// refinement round.
static int launch_prescale64(Ctx& c, const double* x64, const float* x32, double* out,
                             bool absorb, double bytes) {
  ProfScope ps(c.pl, "prescale64", bytes);
  const fe_plan* pl = c.pl;
  for (int k = 0; k < pl->K; ++k) {
    if (absorb && k == pl->primary) continue;
    const int64_t n = pl->nlev[k] + 1;
    const int64_t o = pl->lev_base[k] * c.C;
    const int64_t pairs = n * ((c.C + 1) / 2);
    k_prescale64<<<grid1(pairs), 256, 0, c.s>>>(x64 + o, x32 + o, c.d.scale_d[k], out + o, n, c.C);
    FE_CK(cudaGetLastError());
  }
  return 0;
}

template <typename TA, int C, class Tab, class Epi>
static int launch_expand(Ctx& c, Tab tab, Epi epi, double* part, const char* name, double bytes) {
  ProfScope ps(c.pl, name, bytes);
  if (c.d.K <= 2) return expand_kb<2, TA, C>(c, tab, epi, part);
  if (c.d.K <= 4) return expand_kb<4, TA, C>(c, tab, epi, part);
  return expand_kb<kMaxFE, TA, C>(c, tab, epi, part);
}

// The contiguous row-sum pass (k_rowsum: primary and small FEs) and the
// combine of its small-FE partials.  32-column tiles only.
template <typename TA, int C, bool W, int NS>
static int rowsum_launch(Ctx& c, const TA* src, TA* out) {
  if constexpr (C == 32) {
    // default: rows in registers for FP32, the shared-memory ring for FP64
    const bool regs = c.pl->opt_rowsum_variant == 1 ||
                      (c.pl->opt_rowsum_variant < 0 && sizeof(TA) == 4);
    auto kern = regs ? k_rowsum_reg<TA, C, W, NS> : k_rowsum<TA, C, W, NS>;
    const int RING = regs ? 0 : RowSumStep<TA>::value * RowSumStep<TA>::NBUF;
    const size_t smem = (size_t)kWarps * (RING + c.its->small_rows) * C * sizeof(TA);
    // per instantiation: the opt-in shared-memory limit (set once per
    // device) and the resident CTAs per SM for the last shared-memory size seen
    static PerDeviceOnce attr_set[2];
    static size_t occ_smem[2] = {(size_t)-1, (size_t)-1};
    static int occ[2] = {1, 1};
    const int vi = regs ? 1 : 0;
    if (attr_set[vi].needed(c.pl->device)) {
      FE_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kWarps * (RING + kSmallRows) * C * sizeof(TA))));
      attr_set[vi].done(c.pl->device);
    }
    if (occ_smem[vi] != smem) {
      int o = 0;
      FE_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kThreads, smem));
      occ[vi] = std::max(o, 1);
      occ_smem[vi] = smem;
    }
    const int64_t n = (int64_t)c.its->ex.size();
    const int64_t grid =
        std::max<int64_t>(1, std::min<int64_t>(c.its->Se, (int64_t)occ[vi] * c.its->sms));
    RowSumArgs rs{};
    rs.sum = out;
    rs.sa = c.ex_split();
    rs.small_part = c.small_part;
    rs.small_rows = c.its->small_rows;
    for (int k = 0; k < c.d.K; ++k)
      if ((c.its->small_mask >> k) & 1u) {
        rs.small_fe[rs.n_small] = k;
        rs.small_off[rs.n_small] = c.its->small_off[k];
        ++rs.n_small;
      }
    kern<<<(unsigned)grid, kThreads, smem, c.s>>>(c.d, c.its->d_ex.as<ExpandItem>(), n, src, rs);
    FE_CK(cudaGetLastError());
    if (c.its->small_rows > 0) {
      SmallRows m{};
      for (int r = 0; r < c.its->small_rows; ++r) m.slab_row[r] = c.its->small_slab_row[(size_t)r];
      k_small_combine<TA, C><<<(unsigned)c.its->small_rows, kThreads, 0, c.s>>>(
          c.small_part, (int)grid, c.its->small_rows, m, out, c.d.active);
      FE_CK(cudaGetLastError());
    }
    return 0;
  } else {
    (void)c;
    (void)src;
    (void)out;
    set_error_cstr("row-sum pass requested for a tile narrower than 32 columns");
    return 1;
  }
}

template <typename TA, int C>
static int launch_rowsum(Ctx& c, const TA* src, TA* out) {
  const fe_plan* pl = c.pl;
  bool w = false;
  int ns = 0;
  for (int k = 0; k < pl->K; ++k) {
    const bool small = ((c.its->small_mask >> k) & 1u) != 0;
    if (small) ++ns;
    if ((small || k == pl->primary) && (pl->weighted || pl->interacted[k])) w = true;
  }
  switch (ns * 2 + (w ? 1 : 0)) {
    case 0: return rowsum_launch<TA, C, false, 0>(c, src, out);
    case 1: return rowsum_launch<TA, C, true, 0>(c, src, out);
    case 2: return rowsum_launch<TA, C, false, 1>(c, src, out);
    case 3: return rowsum_launch<TA, C, true, 1>(c, src, out);
    case 4: return rowsum_launch<TA, C, false, 2>(c, src, out);
    default: return rowsum_launch<TA, C, true, 2>(c, src, out);
  }
}

// The demean pass of the absorbed-primary mode (k_demean) and the combine of
// its small-FE partials.  rows: [N][32] of T, projected in place; rows32: an
// optional FP32 copy; out: the [P][C] sum slab (z rows of the primary FE,
// small-FE sums); ||rows||^2 goes to the expand norm slots.
template <typename T, int C, bool W, int NS, int NG = 0>
static int demean_launch(Ctx& c, const T* in, T* rows, float* rows32, T* out,
                         const T* xs = nullptr) {
  if constexpr (C == 32) {
    auto kern = k_demean<T, C, W, NS, NG>;
    const size_t smem = (size_t)kWarps * (kDemeanRows + c.its->small_rows) * C * sizeof(T);
    static PerDeviceOnce attr_set;  // per instantiation
    static size_t occ_smem = (size_t)-1;
    static int occ = 1;
    if (attr_set.needed(c.pl->device)) {
      FE_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kWarps * (kDemeanRows + kSmallRows) * C * sizeof(T))));
      attr_set.done(c.pl->device);
    }
    if (occ_smem != smem) {
      int o = 0;
      FE_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kThreads, smem));
      occ = std::max(o, 1);
      occ_smem = smem;
    }
    const int64_t n = (int64_t)c.its->dm.size();
    // norm slots are the expand's: the grid must not exceed their count
    const int64_t grid =
        std::max<int64_t>(1, std::min<int64_t>(c.its->Se, (int64_t)occ * c.its->sms));
    RowSumArgs rs{};
    rs.sum = out;
    rs.small_part = c.small_part;
    rs.small_rows = c.its->small_rows;
    for (int k = 0; k < c.d.K; ++k)
      if ((c.its->small_mask >> k) & 1u) {
        rs.small_fe[rs.n_small] = k;
        rs.small_off[rs.n_small] = c.its->small_off[k];
        ++rs.n_small;
      }
    kern<<<(unsigned)grid, kThreads, smem, c.s>>>(c.d, c.its->d_dm.as<ExpandItem>(), n, in, rows,
                                                  rows32, rs, c.part_e, c.its->Se, xs, c.inst);
    FE_CK(cudaGetLastError());
    if (c.its->small_rows > 0) {
      SmallRows m{};
      for (int r = 0; r < c.its->small_rows; ++r) m.slab_row[r] = c.its->small_slab_row[(size_t)r];
      k_small_combine<T, C><<<(unsigned)c.its->small_rows, kThreads, 0, c.s>>>(
          c.small_part, (int)grid, c.its->small_rows, m, out, c.d.active_pre);
      FE_CK(cudaGetLastError());
    }
    return 0;
  } else if constexpr (NS == 0 && NG == 0 && C < 32) {
    // narrow tiles (no small FEs, the residual computed apart)
    (void)out;
    (void)xs;
    const int64_t n = (int64_t)c.its->dm.size();
    if (c.its->dm_ipc > 0) {
      // batch plans: one CTA per kDemeanIpc items of one problem, one norm slot
      // each; the problems whose columns have stopped are skipped (the inner
      // loop's FP32 pass: its flag; the refinement's FP64 pass: the outer flag)
      const int act_mode = sizeof(T) == 4 ? 1 : 2;
      k_demean_narrow<T, C, W, true><<<(unsigned)c.its->Sdm, kThreads, 0, c.s>>>(
          c.d, c.its->d_dm.as<ExpandItem>(), n, in, rows, rows32, c.part_e, c.its->Sdm,
          c.its->dm_ipc, c.inst, act_mode);
      FE_CK(cudaGetLastError());
      return 0;
    }
    static int occ = 0;  // resident CTAs per SM, per instantiation
    if (occ == 0) {
      int o = 0;
      FE_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_demean_narrow<T, C, W>, kThreads, 0));
      occ = std::max(o, 1);
    }
    const int64_t grid =
        std::max<int64_t>(1, std::min<int64_t>(c.its->Se, (int64_t)occ * c.its->sms));
    k_demean_narrow<T, C, W><<<(unsigned)grid, kThreads, 0, c.s>>>(
        c.d, c.its->d_dm.as<ExpandItem>(), n, in, rows, rows32, c.part_e, c.its->Se, 0, nullptr,
        0);
    FE_CK(cudaGetLastError());
    return 0;
  } else {
    (void)c;
    (void)in;
    (void)rows;
    (void)rows32;
    (void)out;
    (void)xs;
    set_error_cstr("demean pass with small fixed effects requested for a narrow tile");
    return 1;
  }
}

// in: source rows (nullptr: rows, projected in place).  xs (FP64 only): the
// refinement's residual form, rows = M (in - A_r x) with xs the pre-scaled
// table of x (resid_demean_fits: at most kDemeanResidFE gathered FEs).
constexpr int kDemeanResidFE = 3;
inline bool resid_demean_fits(const fe_plan* pl) { return pl->K - 1 <= kDemeanResidFE; }
template <typename T, int C, int NG>
static int demean_sel(Ctx& c, const T* in, T* rows, float* rows32, T* out, const T* xs) {
  const fe_plan* pl = c.pl;
  bool w = false;
  int ns = 0;
  for (int k = 0; k < pl->K; ++k) {
    const bool small = ((c.its->small_mask >> k) & 1u) != 0;
    if (small) ++ns;
    if ((small || k == pl->primary) && (pl->weighted || pl->interacted[k])) w = true;
  }
  switch (ns * 2 + (w ? 1 : 0)) {
    case 0: return demean_launch<T, C, false, 0, NG>(c, in, rows, rows32, out, xs);
    case 1: return demean_launch<T, C, true, 0, NG>(c, in, rows, rows32, out, xs);
    case 2: return demean_launch<T, C, false, 1, NG>(c, in, rows, rows32, out, xs);
    case 3: return demean_launch<T, C, true, 1, NG>(c, in, rows, rows32, out, xs);
    case 4: return demean_launch<T, C, false, 2, NG>(c, in, rows, rows32, out, xs);
    default: return demean_launch<T, C, true, 2, NG>(c, in, rows, rows32, out, xs);
  }
}
template <typename T, int C>
static int launch_demean(Ctx& c, T* rows, float* rows32, T* out, const char* name, double bytes,
                         const T* in = nullptr, const T* xs = nullptr) {
  if (!in) in = rows;
  ProfScope ps(c.pl, name, bytes);
  if constexpr (std::is_same<T, double>::value) {
    if (xs) {
      switch (c.pl->K - 1) {
        case 1: return demean_sel<T, C, 1>(c, in, rows, rows32, out, xs);
        case 2: return demean_sel<T, C, 2>(c, in, rows, rows32, out, xs);
        case 3: return demean_sel<T, C, 3>(c, in, rows, rows32, out, xs);
        default:
          set_error_cstr("residual demean pass requested for more than 4 fixed effects");
          return 1;
      }
    }
  }
  return demean_sel<T, C, 0>(c, in, rows, rows32, out, nullptr);
}

// The fused expand + demean of the absorbed-primary loop (k_expand_demean):
// u = M (av A_r v + au u), in place on rows, ||u||^2 to the expand norm slots,
// small-FE sums to the slab (through the CTA partials).
// RESID (FP64): rows = M (B - A_r x) with tab holding scale * x, an FP32 copy
// into rows32; columns whose refinement has stopped (mask 2) keep their rows.
template <typename T, int C, int U, int KB, bool W, int NS, class Tab, bool RESID = false>
static int exdm_launch(Ctx& c, Tab tab, T* rows, const double* B = nullptr,
                       float* rows32 = nullptr, int mask = 0) {
  if constexpr (C == 32) {
    auto kern = k_expand_demean<T, C, U, KB, RESID, W, NS, Tab, true>;
    const size_t smem =
        (size_t)kWarps * ((2 * kDemeanRows + c.its->small_rows) * C * sizeof(T) + 32 * sizeof(int));
    static PerDeviceOnce attr_set;  // per instantiation
    static size_t occ_smem = (size_t)-1;
    static int occ = 1;
    if (attr_set.needed(c.pl->device)) {
      FE_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kWarps * ((2 * kDemeanRows + kSmallRows) * C * sizeof(T) +
                                                 32 * sizeof(int)))));
      attr_set.done(c.pl->device);
    }
    if (occ_smem != smem) {
      int o = 0;
      FE_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kThreads, smem));
      occ = std::max(o, 1);
      occ_smem = smem;
    }
    const int64_t n = (int64_t)c.its->dm.size();
    const int64_t grid =
        std::max<int64_t>(1, std::min<int64_t>(c.its->Se, (int64_t)occ * c.its->sms));
    RowSumArgs rs{};
    rs.sum = c.S;
    rs.small_part = c.small_part;
    rs.small_rows = c.its->small_rows;
    for (int k = 0; k < c.d.K; ++k)
      if ((c.its->small_mask >> k) & 1u) {
        rs.small_fe[rs.n_small] = k;
        rs.small_off[rs.n_small] = c.its->small_off[k];
        ++rs.n_small;
      }
    kern<<<(unsigned)grid, kThreads, smem, c.s>>>(c.d, c.its->d_dm.as<ExpandItem>(), n, tab, rows,
                                                  B, rows32, c.inst, mask, rs, c.part_e,
                                                  c.its->Se);
    FE_CK(cudaGetLastError());
    if (c.its->small_rows > 0) {
      SmallRows m{};
      for (int r = 0; r < c.its->small_rows; ++r) m.slab_row[r] = c.its->small_slab_row[(size_t)r];
      k_small_combine<T, C><<<(unsigned)c.its->small_rows, kThreads, 0, c.s>>>(
          c.small_part, (int)grid, c.its->small_rows, m, static_cast<T*>(c.S), c.d.active_pre);
      FE_CK(cudaGetLastError());
    }
    return 0;
  } else {
    (void)c;
    (void)tab;
    (void)rows;
    (void)B;
    (void)rows32;
    (void)mask;
    set_error_cstr("fused expand-demean requested for a tile narrower than 32 columns");
    return 1;
  }
}

template <typename T, int C, int U, class Tab, bool RESID = false>
static int exdm_u(Ctx& c, Tab tab, T* rows, const double* B = nullptr, float* rows32 = nullptr,
                  int mask = 0) {
  const fe_plan* pl = c.pl;
  bool w = false;
  int ns = 0;
  for (int k = 0; k < pl->K; ++k) {
    const bool small = ((c.its->small_mask >> k) & 1u) != 0;
    if (small) ++ns;
    if ((small || k == pl->primary) && (pl->weighted || pl->interacted[k])) w = true;
  }
  const int sel = ns * 2 + (w ? 1 : 0);
#define FE_EXDM_CASE(KB, W_, NS_) \
  return exdm_launch<T, C, U, KB, W_, NS_, Tab, RESID>(c, tab, rows, B, rows32, mask)
  if (c.d.K <= 4) {
    switch (sel) {
      case 0: FE_EXDM_CASE(4, false, 0);
      case 1: FE_EXDM_CASE(4, true, 0);
      case 2: FE_EXDM_CASE(4, false, 1);
      case 3: FE_EXDM_CASE(4, true, 1);
      case 4: FE_EXDM_CASE(4, false, 2);
      default: FE_EXDM_CASE(4, true, 2);
    }
  }
  switch (sel) {
    case 0: FE_EXDM_CASE(kMaxFE, false, 0);
    case 1: FE_EXDM_CASE(kMaxFE, true, 0);
    case 2: FE_EXDM_CASE(kMaxFE, false, 1);
    case 3: FE_EXDM_CASE(kMaxFE, true, 1);
    case 4: FE_EXDM_CASE(kMaxFE, false, 2);
    default: FE_EXDM_CASE(kMaxFE, true, 2);
  }
#undef FE_EXDM_CASE
}

// The refinement's residual of the absorbed mode in one pass (rounds after
// the first): R64 = M (B64 - A_r x) with x the pre-scaled FP64 table, its FP32
// copy U, ||R64||^2 and the small FEs' sums; columns whose refinement has
// stopped keep their rows.
template <int C>
static int launch_resid_demean(Ctx& c, const double* xs64, double* R64, const double* B64,
                               float* U, double bytes) {
  ProfScope ps(c.pl, "resid_demean64", bytes);
  return exdm_u<double, C, 4, TabPre64<vec_of<double, C>()>, true>(
      c, TabPre64<vec_of<double, C>()>{xs64}, R64, B64, U, 2);
}

// The pipelined fused kernel (k_exdm_pipe): FP32 rows of 32-column tiles, at
// most one gathered (large) non-primary FE, and staging that fits the
// shared-memory limit.  Sets *launched when it ran; otherwise the caller runs
// k_expand_demean.  FE_OPT_EXDM_PIPE: -1 the default configuration (the
// first of kExdmPrefer that fits), 1 or 2 one configuration, 0 off.
// The configuration of the pipelined kernel the plan's tile takes: ok = 0
// when it does not fit (the caller then runs k_expand_demean).
struct ExdmChoice {
  bool ok = false;
  int nl = 0, ns = 0, nsr = 0, cfg = -1;
  bool w = false;
  ExdmFEs lf{};
};
static int exdm_choose(const Ctx& c, ExdmChoice* ch) {
  static const int kExdmPrefer[] = {1, 2};
  *ch = ExdmChoice{};
  const fe_plan* pl = c.pl;
  if (pl->opt_exdm_pipe == 0) return 0;
  // opt-in shared memory per block of the plan's device (a host query, read
  // per call so that every device of the process answers for itself)
  int smem_max = 0;
  FE_CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, pl->device));
  for (int k = 0; k < pl->K; ++k) {
    const bool small = ((c.its->small_mask >> k) & 1u) != 0;
    if (pl->weighted || pl->interacted[k]) ch->w = true;
    if (k == pl->primary) continue;
    if (small) {
      ++ch->ns;
      continue;
    }
    if (ch->nl == 2) return 0;
    ch->lf.large[ch->nl] = k;
    ch->lf.large_base[ch->nl] = pl->lev_base[k];
    ++ch->nl;
  }
  if (ch->nl > 1) return 0;
  ch->nsr = ch->ns ? c.its->small_rows : 0;
  auto fits = [&](int cfg) {
    const ExdmCfg k = exdm_cfg(cfg);
    return exdm_pipe_smem(ch->nl, ch->nsr, k.stages, k.per_group, k.warps, k.vsm) <=
           (size_t)smem_max;
  };
  if (pl->opt_exdm_pipe > 0) {
    if (fits(pl->opt_exdm_pipe)) ch->cfg = pl->opt_exdm_pipe;
  } else {
    for (int k : kExdmPrefer)
      if (fits(k)) {
        ch->cfg = k;
        break;
      }
  }
  ch->ok = ch->cfg > 0;
  return 0;
}

// Whether the tile's gathered FE can take its level sums by vector
// reductions inside the pipelined kernel: configuration 1, one gathered FE,
// and no level of it with more than kAtomicMaxLevel positions.  The
// reductions of one level arrive in no fixed order, each rounded into one
// FP32 sum; over the ~1e5-1e6 rows of a Zipf head level that error stalled
// the FP32 inner LSMR (measured: non-convergence at maxiter), and the
// contention on the level's row made the fused kernel 5x slower.
constexpr int64_t kAtomicMaxLevel = 1024;
static bool exdm_atomic_eligible(const fe_plan* pl, const ExdmChoice& ch) {
  if (!(ch.ok && ch.cfg == 1 && ch.nl == 1)) return false;
  const int k = ch.lf.large[0];
  const std::vector<int64_t>& off = pl->seg_off[k];
  int64_t mx = 0;
  for (size_t l = 0; l + 1 < off.size(); ++l) mx = std::max(mx, off[l + 1] - off[l]);
  return mx <= kAtomicMaxLevel;
}

// The pipelined fused kernel; *launched = 1 when it ran (with the gathered
// FE's level sums by reductions when c.firm_atomic), else the caller runs
// k_expand_demean.
static int try_exdm_pipe(Ctx& c, const float* tab, float* rows, int* launched) {
  *launched = 0;
  ExdmChoice ch;
  int st0 = exdm_choose(c, &ch);
  if (st0 || !ch.ok) return st0;
  const int nl = ch.nl, ns = ch.ns, nsr = ch.nsr, cfg = ch.cfg;
  const bool w = ch.w;
  const ExdmFEs lf = ch.lf;
  const ExdmCfg kc = exdm_cfg(cfg);
  ExdmLaunch a{};
  a.d = c.d;
  a.items = c.its->d_dm.as<ExpandItem>();
  a.n_items = (int64_t)c.its->dm.size();
  a.tab = tab;
  a.rows = rows;
  a.inst = c.inst;
  a.rs.sum = c.S;
  a.rs.small_part = c.small_part;
  a.rs.small_rows = c.its->small_rows;
  for (int k = 0; k < c.d.K; ++k)
    if ((c.its->small_mask >> k) & 1u) {
      a.rs.small_fe[a.rs.n_small] = k;
      a.rs.small_off[a.rs.n_small] = c.its->small_off[k];
      ++a.rs.n_small;
    }
  for (int r = 0; r < c.its->small_rows; ++r) a.sr.slab_row[r] = c.its->small_slab_row[(size_t)r];
  a.lf = lf;
  a.part = c.part_e;
  a.S = c.its->Se;
  // as many CTAs as the shared memory of the SMs holds (one of 8 warps, or up
  // to three of 4 warps); the norm slots are the expand's, so the grid must
  // not exceed their count
  a.smem = exdm_pipe_smem(nl, nsr, kc.stages, kc.per_group, kc.warps, kc.vsm);
  // shared memory per SM and reserved per CTA on the plan's device
  int smem_sm = 0, smem_res = 0;
  FE_CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c.pl->device));
  FE_CK(cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, c.pl->device));
  const size_t per_cta = a.smem + (size_t)smem_res;  // no static shared memory
  const int per_sm = std::max(1, std::min(kc.warps < kWarps ? 3 : 1, (int)(smem_sm / per_cta)));
  a.grid = std::max<int64_t>(1, std::min<int64_t>(c.its->Se, (int64_t)per_sm * c.its->sms));
  a.stream = c.s;
  int st = launch_exdm_pipe(a, nl, ns, w, cfg, c.firm_atomic && exdm_atomic_eligible(c.pl, ch));
  if (st) return st;
  if (c.its->small_rows > 0) {
    k_small_combine<float, 32><<<(unsigned)c.its->small_rows, kThreads, 0, c.s>>>(
        c.small_part, (int)a.grid, c.its->small_rows, a.sr, static_cast<float*>(c.S),
        c.d.active_pre);
    FE_CK(cudaGetLastError());
  }
  *launched = 1;
  return 0;
}

template <typename T, int C, class Tab>
static int launch_expand_demean(Ctx& c, Tab tab, T* rows, const char* name, double bytes) {
  ProfScope ps(c.pl, name, bytes);
  if constexpr (C == 32 && std::is_same<T, float>::value) {
    int launched = 0;
    const int st = try_exdm_pipe(c, tab.tab, rows, &launched);
    if (st || launched) return st;
  }
  // unroll depth 4 (measured fastest on the worker/firm/year workload), or
  // that of a forced expand variant
  const int var = c.pl->opt_ex_variant >= 0 ? c.pl->opt_ex_variant : 3;
  if (var == 1 || var == 3 || var == 5) return exdm_u<T, C, 4>(c, tab, rows);
  return exdm_u<T, C, 2>(c, tab, rows);
}

// Rows of 32-column tiles: 32 bytes per lane (FP64: 4 elements, 4 rows per
// warp instruction; FP32: 8 elements, 8 rows), half the per-row work of
// 16-byte lanes, with half the row slots per lane group so that a stage
// holds the same rows
template <typename TA, int C, int U, int S, class Load>
static int launch_segsum_async(Ctx& c, Load ld, TA* out, const ReduceItem* items, int64_t n,
                               unsigned grid) {
  constexpr int VF = C == 32 ? 32 / (int)sizeof(TA) : 0;
  constexpr int UE = VF ? (U > 1 ? U / 2 : 1) : U;
  using L = AsyncSegLayout<TA, C, UE, S, VF>;
  const int smem = kWarps * L::kWarpBytes;
  static PerDeviceOnce attr_set;  // per instantiation (set once per device)
  if (attr_set.needed(c.pl->device)) {
    FE_CK(cudaFuncSetAttribute(k_segsum_async<TA, C, UE, S, Load, VF>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set.done(c.pl->device);
  }
  k_segsum_async<TA, C, UE, S, Load, VF><<<grid, kThreads, smem, c.s>>>(c.d, items, n, ld, out,
                                                                         c.seg_split());
  return 0;
}

// rowsum: the primary and small FEs go through the contiguous row-sum pass
// (32-column tiles of single-problem plans), the segsum gathers only the
// large non-primary FEs; otherwise the segsum reduces every FE.
template <typename TA, int C, class Load>
static int launch_segsum(Ctx& c, Load ld, TA* out, const char* name, double bytes,
                         bool rowsum = false, const char* rs_name = "rowsum", double rs_bytes = 0.0,
                         bool large_only = false) {
  if (large_only) rowsum = true;  // the segsum part of the row-sum mode only
  if constexpr (!Load::kSquareWeight) {
    if (rowsum && !large_only) {
      ProfScope ps(c.pl, rs_name, rs_bytes);
      static_assert(std::is_same<typename Load::InType, TA>::value, "rows are summed in their type");
      const int st = launch_rowsum<TA, C>(c, ld.in, out);
      if (st) return st;
    }
  }
  const int64_t n = rowsum ? c.its->rd_large : (int64_t)c.its->rd.size();
  if (n == 0) return 0;
  ProfScope ps(c.pl, name, bytes);
  const unsigned grid = (unsigned)((n + kWarps - 1) / kWarps);
  const ReduceItem* items = c.its->d_rd.as<ReduceItem>();
  const SplitArgs sa = c.seg_split();
  const int var = pick_seg(c.pl, sizeof(TA));
  if constexpr (Load::kAsyncable) {
    if (var == 4 || var == 5) {
      const int st = var == 4 ? launch_segsum_async<TA, C, 4, 4>(c, ld, out, items, n, grid)
                              : launch_segsum_async<TA, C, 2, 6>(c, ld, out, items, n, grid);
      if (st) return st;
      FE_CK(cudaGetLastError());
      return 0;
    }
  }
  switch (var) {
    case 1:
      k_segsum<TA, C, 4, true, Load><<<grid, kThreads, 0, c.s>>>(c.d, items, n, ld, out, sa);
      break;
    case 2:
      k_segsum<TA, C, 8, true, Load><<<grid, kThreads, 0, c.s>>>(c.d, items, n, ld, out, sa);
      break;
    case 3:
      k_segsum<TA, C, 4, false, Load><<<grid, kThreads, 0, c.s>>>(c.d, items, n, ld, out, sa);
      break;
    default:
      k_segsum<TA, C, 8, false, Load><<<grid, kThreads, 0, c.s>>>(c.d, items, n, ld, out, sa);
      break;
  }
  FE_CK(cudaGetLastError());
  return 0;
}

template <int C, class Epi>
static int launch_pupdate(Ctx& c, const typename Epi::TS* S, Epi epi, double* pa, double* pb,
                          const char* name, double bytes) {
  ProfScope ps(c.pl, name, bytes);
  // absorbed-primary mode: the non-primary levels only (the leading items)
  // (batch plans: a list of their own, per problem)
  const int64_t n = c.absorb ? c.its->pu_np : (int64_t)c.its->pu.size();
  const unsigned grid = (unsigned)(n / kWarps);
  const PItem* items = (c.absorb && c.its->dm_ipc > 0) ? c.its->d_pu_abs.as<PItem>()
                                                       : c.its->d_pu.as<PItem>();
  k_pupdate<C, Tune<C>::kPU, Epi><<<grid, kThreads, 0, c.s>>>(
      c.d, items, n, S, epi, pa, pb, c.absorb ? c.its->Sp_np : c.its->Sp);
  FE_CK(cudaGetLastError());
  return 0;
}

static int launch_scalar_phase(Ctx& c, int phase, int init_mode) {
  ProfScope ps(c.pl, "scalar", 0.0);
  ScalarArgs a;
  memset(&a, 0, sizeof(a));
  a.inst = c.inst;
  a.C = c.C;
  a.phase = phase;
  a.init_mode = init_mode;
  a.counters = c.counters;
  // the absorbed mode's norms of u come from the demean pass: per-problem
  // slots of their own in batch plans
  const bool dm_slots = c.absorb && c.its->dm_ipc > 0;
  a.off0 = dm_slots ? c.its->d_dm_off.as<int64_t>() : c.its->d_ex_off.as<int64_t>();
  a.S0 = dm_slots ? c.its->Sdm : c.its->Se;
  a.off1 = c.absorb ? c.its->d_pu_off_np.as<int64_t>() : c.its->d_pu_off.as<int64_t>();
  a.S1 = c.absorb ? c.its->Sp_np : c.its->Sp;
  switch (phase) {
    case PH_INIT_BETA:
    case PH_BETA:
      a.part0 = c.part_e;
      break;
    case PH_INIT_ALPHA:
    case PH_ALPHA:
      a.part1 = c.part_a;
      a.part2 = c.part_b;
      break;
    case PH_OUTER:
      a.part0 = c.part_e;
      a.part1 = c.part_a;
      a.part2 = c.part_b;
      break;
    default:
      break;
  }
  if (c.pl->xchg && a.part0) {
    // sharded plan: the exchanged per-column totals, one slot per column
    a.part0 = c.xbuf;
    a.off0 = c.off01;
    a.S0 = 1;
  }
  launch_scalar(a, c.n_inst, c.s);
  FE_CK(cudaGetLastError());
  return 0;
}

static int read_counter(Ctx& c, int idx, int32_t* out) {
  FE_CK(cudaMemcpyAsync(c.h_counters + idx, c.counters + idx, sizeof(int32_t),
                        cudaMemcpyDeviceToHost, c.s));
  FE_CK(cudaStreamSynchronize(c.s));
  *out = c.h_counters[idx];
  return 0;
}

// The row-sum pass serves 32-column tiles (its walk puts one column on each
// lane) of single-problem plans (its small-FE tables hold one problem).
static bool use_rowsum(const fe_plan* pl, int C) {
  return pl->opt_fuse != 0 && C == 32 && pl->nprob == 1;
}

// Absorbed-primary mode of the mixed-precision residual solve (plans with 2+
// FEs, and batches whose problems all hold the primary FE and another): the
// least-squares residual is
// that of the problem with the primary FE projected out,
//   min || M (b - A_r x_r) ||,  M u = u - sum_l a_l (a_l' u),
// a_l the unit columns of the primary FE (contiguous row segments).  LSMR then
// iterates over the other FEs' levels only, on a better-conditioned operator.
static bool use_absorb(const fe_plan* pl, const ItemSet* its, int C) {
  // tiles of every width: k_demean (32 columns) or k_demean_narrow; batch
  // plans have demean items on narrow tiles only
  (void)C;
  return pl->opt_absorb != 0 && pl->absorbable && !its->dm.empty();
}

// algorithmic bytes per launch (the roofline numerators): every index vector
// and observation row once, every coefficient-table row once
struct Bytes {
  double expand, segsum, pupdate, resid64, segsum64, grad64, rowsum, rowsum64;
  // absorbed-primary mode
  double expand_abs, resid64_abs, demean, demean64, pupdate_np, grad64_np, expand_demean;
  double segsum_abs, segsum64_abs;  // the gathered (neither primary nor small) FEs only
  double prescale64, prescale64_abs, resid_demean64, resid_dm64;
};
static Bytes alg_bytes(const fe_plan* pl, const ItemSet* its, int C, int sT) {
  Bytes b{};
  const bool fuse = use_rowsum(pl, C);
  const double N = (double)pl->N;
  // Pf: levels whose sums the row-sum pass writes (primary and small FEs)
  double P = 0, Pf = 0, pos = 0, posmeta = 0, cw = 0, cw64 = 0, cwp = 0, cwp64 = 0;
  for (int k = 0; k < pl->K; ++k) {
    P += (double)pl->nlev[k];
    const bool has_cw = pl->weighted || pl->interacted[k];
    if (has_cw) {
      cw += N * sT;
      cw64 += N * 8.0;
    }
    if (fuse && (k == pl->primary || ((its->small_mask >> k) & 1u))) {
      Pf += (double)pl->nlev[k];
      continue;  // reduced by the row-sum pass
    }
    pos += (double)pl->seg_len[k];
    posmeta += (double)pl->seg_len[k] * (4.0 + (pl->perm_identity[k] ? 0.0 : 4.0));
    if (has_cw) {
      cwp += (double)pl->seg_len[k] * sT;
      cwp64 += (double)pl->seg_len[k] * 8.0;
    }
  }
  const double refs = N * 4.0 * pl->K;
  // the row-sum pass: one contiguous read of the rows and of the fused FEs'
  // refs (and weights), the fused levels' sums written
  double rowsum = 0.0, rowsum64 = 0.0;
  if (fuse) {
    double meta = 0.0, meta64 = 0.0;
    for (int k = 0; k < pl->K; ++k)
      if (k == pl->primary || ((its->small_mask >> k) & 1u)) {
        const bool has_cw = pl->weighted || pl->interacted[k];
        meta += N * (4.0 + (has_cw ? sT : 0));
        meta64 += N * (4.0 + (has_cw ? 8.0 : 0.0));
      }
    rowsum = meta + N * C * sT + Pf * C * sT;
    rowsum64 = meta64 + N * C * 8.0 + Pf * C * 8.0;
  }
  b.expand = refs + cw + 2.0 * N * C * sT + P * C * sT;
  b.segsum = posmeta + cwp + pos * C * sT + (P - Pf) * C * sT;
  b.rowsum = rowsum;
  b.rowsum64 = rowsum64;
  {
    // absorbed-primary mode: the expand leaves out the primary FE; the demean
    // pass reads the primary (and small-FE) keys and scales and reads and
    // writes the rows once (z rows stay on chip except for levels longer than
    // kDemeanRows); the P side covers the other FEs
    const int kp = pl->primary;
    const bool cwp = pl->weighted || pl->interacted[kp];
    const double Pp = (double)pl->nlev[kp], Pnp = P - Pp;
    double keys = N * (4.0 + (cwp ? sT : 0)), keys64 = N * (4.0 + (cwp ? 8.0 : 0.0));
    for (int k = 0; k < pl->K; ++k)
      if ((its->small_mask >> k) & 1u) {
        const bool hc = pl->weighted || pl->interacted[k];
        keys += N * (4.0 + (hc ? sT : 0));
        keys64 += N * (4.0 + (hc ? 8.0 : 0.0));
      }
    const double cwnp = cw - (cwp ? N * sT : 0.0), cwnp64 = cw64 - (cwp ? N * 8.0 : 0.0);
    b.expand_abs = N * 4.0 * (pl->K - 1) + cwnp + 2.0 * N * C * sT + Pnp * C * sT;
    b.resid64_abs = N * 4.0 * (pl->K - 1) + cwnp64 + N * C * 16.0 + Pnp * C * 8.0;
    b.prescale64_abs = Pnp * (C * 20.0 + 8.0);
    b.demean = keys + 2.0 * N * C * sT + Pp * sT;
    b.demean64 = keys64 + 2.0 * N * C * 8.0 + N * C * 4.0 + Pp * 8.0;
    b.pupdate_np = 9.0 * Pnp * C * sT;
    // fused: the expand's bytes (which already hold every non-primary FE's
    // refs and weights, the small FEs' included) plus the primary FE's keys,
    // weights and scales
    b.expand_demean = b.expand_abs + N * (4.0 + (cwp ? sT : 0)) + Pp * sT;
    // fused FP64 residual + projection: the residual's bytes, the FP32 copy,
    // the primary FE's keys, weights and scales
    b.resid_demean64 = b.resid64_abs + N * C * 4.0 + N * (4.0 + (cwp ? 8.0 : 0.0)) + Pp * 8.0;
    // the demean kernel's residual form: the same bytes (the small FEs' keys
    // are among the K - 1 gathered FEs' refs, counted once)
    b.resid_dm64 = b.resid_demean64;
    b.grad64_np = Pnp * C * (8.0 + 4.0 + 8.0 + 4.0 + 8.0);
  }
  b.pupdate = 9.0 * P * C * sT;
  b.resid64 = refs + cw64 + N * C * (8.0 + 8.0 + 4.0) + P * C * 8.0;
  b.prescale64 = P * (C * 20.0 + 8.0);
  b.segsum64 = posmeta + cwp64 + pos * C * 8.0 + (P - Pf) * C * 8.0;
  b.grad64 = P * C * (8.0 + 4.0 + 8.0 + 4.0 + 8.0);
  {
    // the absorbed loop's segmented sums cover the FEs that are neither the
    // primary nor small (the same figures as above where the row-sum pass runs)
    double posA = 0, metaA = 0, cwA = 0, cwA64 = 0, PA = 0;
    for (int k = 0; k < pl->K; ++k) {
      if (k == pl->primary || ((its->small_mask >> k) & 1u)) continue;
      const double sl = (double)pl->seg_len[k];
      posA += sl;
      metaA += sl * (4.0 + (pl->perm_identity[k] ? 0.0 : 4.0));
      if (pl->weighted || pl->interacted[k]) {
        cwA += sl * sT;
        cwA64 += sl * 8.0;
      }
      PA += (double)pl->nlev[k];
    }
    b.segsum_abs = metaA + cwA + posA * C * sT + PA * C * sT;
    b.segsum64_abs = metaA + cwA64 + posA * C * 8.0 + PA * C * 8.0;
  }
  return b;
}

static int prepare(fe_plan* pl, int C, int sT, bool mixed, Ctx& c) {
  ItemSet* its = nullptr;
  int st = plan_items(pl, C, &its);
  if (st) return st;
  Workspace& w = pl->ws;
  const size_t N = (size_t)std::max<int64_t>(pl->N, 1), P = (size_t)pl->P;
  const size_t nC = (size_t)C;
  if ((st = w.B64.ensure(N * nC * 8))) return st;
  if ((st = w.R64.ensure(N * nC * 8))) return st;
  if ((st = w.U.ensure(N * nC * (size_t)sT))) return st;
  if ((st = w.V.ensure(P * nC * (size_t)sT))) return st;
  if (mixed && (st = w.VS.ensure(P * nC * 4))) return st;
  if ((st = w.H.ensure(P * nC * (size_t)sT))) return st;
  if ((st = w.Hb.ensure(P * nC * (size_t)sT))) return st;
  if ((st = w.X.ensure(P * nC * (size_t)sT))) return st;
  if (mixed && (st = w.X64.ensure(P * nC * 8))) return st;
  if (mixed && (st = w.XS64.ensure(P * nC * 8))) return st;
  if ((st = w.part_e.ensure((size_t)std::max<int64_t>(std::max(its->Se, its->Sdm), 1) * nC * 8)))
    return st;
  // (a batch plan's absorbed P-side list can hold more slots than the full one)
  const int64_t sp = std::max<int64_t>(std::max(its->Sp, its->Sp_np), 1);
  if ((st = w.part_a.ensure((size_t)sp * nC * 8))) return st;
  if ((st = w.part_b.ensure((size_t)sp * nC * 8))) return st;
  if ((st = w.S.ensure(P * nC * 8))) return st;
  if ((st = w.piece_part.ensure((size_t)std::max<int64_t>(its->n_pieces, 1) * nC * 8))) return st;
  if ((st = w.ex_piece_part.ensure((size_t)std::max<int64_t>(its->ex_n_pieces, 1) * nC * 8))) return st;
  if ((st = w.block_part.ensure((size_t)std::max<int64_t>(its->n_blocks, 1) * nC * 8))) return st;
  if ((st = w.ex_block_part.ensure((size_t)std::max<int64_t>(its->ex_n_blocks, 1) * nC * 8))) return st;
  if ((st = w.inst.ensure((size_t)pl->nprob * nC * sizeof(Inst)))) return st;
  // at most 8 resident CTAs of 256 threads per SM
  if ((st = w.small_part.ensure((size_t)its->sms * 8 * std::max(its->small_rows, 1) * nC * 8)))
    return st;
  if ((st = w.counters.ensure(64))) return st;
  if (pl->xchg) {
    if ((st = w.xbuf.ensure(nC * 8))) return st;
    if (!w.off01.p) {
      const int64_t off[2] = {0, 1};
      if ((st = w.off01.ensure(sizeof(off)))) return st;
      FE_CK(cudaMemcpyAsync(w.off01.p, off, sizeof(off), cudaMemcpyHostToDevice, pl->stream));
      FE_CK(cudaStreamSynchronize(pl->stream));
    }
  }
  if (!pl->host_pinned) FE_CK(cudaMallocHost(&pl->host_pinned, 64));
  c.pl = pl;
  c.its = its;
  c.d = pl->dev;
  c.d.C = C;
  c.C = C;
  c.s = pl->stream;
  c.inst = w.inst.as<Inst>();
  c.counters = w.counters.as<int32_t>();
  c.h_counters = static_cast<int32_t*>(pl->host_pinned);
  c.n_inst = pl->nprob * C;
  c.part_e = w.part_e.as<double>();
  c.part_a = w.part_a.as<double>();
  c.part_b = w.part_b.as<double>();
  c.piece = w.piece_part.as<double>();
  c.ex_piece = w.ex_piece_part.as<double>();
  c.block = w.block_part.as<double>();
  c.ex_block = w.ex_block_part.as<double>();
  c.S = w.S.p;
  c.small_part = w.small_part.as<double>();
  c.rowsum = use_rowsum(pl, C);
  c.xbuf = pl->xchg ? w.xbuf.as<double>() : nullptr;
  c.off01 = pl->xchg ? w.off01.as<int64_t>() : nullptr;
  // coefficient-side slabs start at zero (levels without observations and
  // the null levels are never written afterwards)
  FE_CK(cudaMemsetAsync(w.V.p, 0, P * nC * (size_t)sT, c.s));
  if (mixed) FE_CK(cudaMemsetAsync(w.VS.p, 0, P * nC * 4, c.s));
  FE_CK(cudaMemsetAsync(w.H.p, 0, P * nC * (size_t)sT, c.s));
  FE_CK(cudaMemsetAsync(w.Hb.p, 0, P * nC * (size_t)sT, c.s));
  FE_CK(cudaMemsetAsync(w.X.p, 0, P * nC * (size_t)sT, c.s));
  if (mixed) FE_CK(cudaMemsetAsync(w.X64.p, 0, P * nC * 8, c.s));
  FE_CK(cudaMemsetAsync(w.S.p, 0, P * nC * 8, c.s));
  FE_CK(cudaMemsetAsync(c.counters, 0, 64, c.s));
  return 0;
}

template <int C, typename TY, bool W>
static void launch_load(const fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  if constexpr (C <= 2) {
    k_load_gather<TY, C, W><<<grid1(pl->N), 256, 0, c.s>>>(
        (const TY*)rq.Y, rq.ld, col0, ncols, pl->d_obs_src.as<int32_t>(),
        W ? pl->d_sw_sorted.as<double>() : nullptr, pl->ws.B64.as<double>(), pl->N);
    return;
  }
  k_load<TY, C, W><<<grid1(pl->N, load_rows<C>()), 256, 0, c.s>>>(
      (const TY*)rq.Y, rq.ld, col0, ncols, pl->d_obs_dst.as<int32_t>(),
      W ? pl->d_sw_orig.as<double>() : nullptr, pl->ws.B64.as<double>(), pl->N);
}
template <int C, typename TY, bool W>
static void launch_unload(const fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  k_unload<TY, C, W><<<grid1(pl->N, load_rows<C>()), 256, 0, c.s>>>(
      pl->ws.R64.as<double>(), rq.ld, col0, ncols, pl->d_obs_dst.as<int32_t>(),
      W ? pl->d_sw_orig.as<double>() : nullptr, (TY*)rq.Y, pl->N);
}

template <int C>
static int load_tile(fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  NvtxRange nv("fe: load tile");
  if (pl->N == 0) return 0;
  ProfScope ps(pl, "load", (double)pl->N * ncols * (rq.dtype == 0 ? 8 : 4) + (double)pl->N * C * 8);
  if (rq.dtype == 0)
    pl->weighted ? launch_load<C, double, true>(pl, c, rq, col0, ncols)
                 : launch_load<C, double, false>(pl, c, rq, col0, ncols);
  else
    pl->weighted ? launch_load<C, float, true>(pl, c, rq, col0, ncols)
                 : launch_load<C, float, false>(pl, c, rq, col0, ncols);
  FE_CK(cudaGetLastError());
  return 0;
}

template <int C>
static int unload_tile(fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  NvtxRange nv("fe: unload tile");
  if (pl->N == 0) return 0;
  ProfScope ps(pl, "unload", (double)pl->N * ncols * (rq.dtype == 0 ? 8 : 4) + (double)pl->N * C * 8);
  if (rq.dtype == 0)
    pl->weighted ? launch_unload<C, double, true>(pl, c, rq, col0, ncols)
                 : launch_unload<C, double, false>(pl, c, rq, col0, ncols);
  else
    pl->weighted ? launch_unload<C, float, true>(pl, c, rq, col0, ncols)
                 : launch_unload<C, float, false>(pl, c, rq, col0, ncols);
  FE_CK(cudaGetLastError());
  return 0;
}

static void init_insts(fe_plan* pl, const SolveReq& rq, int C, int ncols, std::vector<Inst>& h) {
  h.assign((size_t)pl->nprob * C, Inst{});
  const bool mixed = rq.precision == 1;
  const int64_t mi = rq.residuals ? rq.maxiter - 1 : rq.maxiter;
  for (int p = 0; p < pl->nprob; ++p)
    for (int j = 0; j < C; ++j) {
      Inst& s = h[(size_t)p * C + j];
      memset(&s, 0, sizeof(s));
      s.ctol = 1e-8;  // 1/conlim, conlim = 1e8 (src/utils/lsmr.jl:47)
      s.skip_lsmr = (rq.residuals && pl->prob_nfe[p] <= 1) ? 1 : 0;
      if (mixed) {
        s.atol = 0.0;
        s.btol = 0.0;
        s.tol_a = rq.tol;
        s.tol_b = rq.tol;
        s.maxiter_total = mi;
        s.maxiter = mi;
        s.inner_theta_tol = pl->opt_inner_theta * rq.tol;
        s.inner_rho = pl->opt_inner_rho;
        s.outer_active = j < ncols ? 1 : 0;
        s.converged = j < ncols ? 0 : 1;
        s.max_rounds = pl->opt_max_rounds;
      } else {
        s.atol = rq.tol;
        s.btol = rq.tol;
        s.maxiter = mi;
      }
    }
}

// ---------------------------------------------------------------------------
// CUDA-graph replay of the LSMR loop: `body` enqueues one iteration; m of them
// are captured once per (tile width, precision) and workspace layout, then
// replayed between host convergence checks.  Every per-iteration quantity
// lives in device memory (the Inst array), so the launches are identical from
// one iteration to the next.  Profiling mode launches directly instead (its
// per-launch CUDA events cannot be read back from inside a graph).
// ---------------------------------------------------------------------------
template <class Body>
static int run_loop(fe_plan* pl, Ctx& c, int prec, int64_t cap, int32_t nact0, Body body,
                    int64_t* done_iters) {
  NvtxRange nv("fe: LSMR loop");
  int32_t nact = nact0;
  const int m = std::max(1, pl->opt_check_every);
  int64_t it = 0;
  // sharded plans exchange between launches: no graph replay
  const bool graph = pl->opt_graph != 0 && !pl->prof.on && !pl->xchg;
  LoopGraph* lg = nullptr;
  if (graph) {
    size_t key = (size_t)c.C * 1000003u ^ (size_t)m;
    const void* ptrs[] = {c.inst, c.part_e, c.part_a, c.part_b, c.piece, c.ex_piece, c.S,
                          c.block, c.ex_block, pl->ws.U.p, pl->ws.V.p, pl->ws.H.p, pl->ws.Hb.p,
                          pl->ws.X.p, c.its, c.counters, c.s, c.small_part, pl->ws.VS.p};
    for (const void* p : ptrs) key = key * 1315423911u + (size_t)p;
    // the variants the captured launches use (tuned, or forced by an option)
    for (size_t e : {(size_t)4, (size_t)8})
      key = key * 31 + (size_t)pick_ex(pl, e) * 7 + (size_t)pick_seg(pl, e);
    key = key * 3 + (c.rowsum ? 1u : 0u);
    key = key * 5 + (size_t)(pl->opt_rowsum_variant + 1);
    key = key * 3 + (c.absorb ? 1u : 0u);
    key = key * 3 + (size_t)pl->opt_exdm;
    key = key * 3 + (size_t)pl->opt_abs_scale;
    key = key * 7 + (size_t)(pl->opt_exdm_pipe + 1);
    key = key * 3 + (c.firm_atomic ? 1u : 0u);
    lg = &pl->graphs[{c.C, prec}];
    if (!lg->exec || lg->key != key) {
      if (lg->exec) {
        cudaGraphExecDestroy(lg->exec);
        lg->exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      FE_CK(cudaStreamBeginCapture(c.s, cudaStreamCaptureModeThreadLocal));
      int st = 0;
      for (int r = 0; r < m && !st; ++r) st = body();
      const cudaError_t e = cudaStreamEndCapture(c.s, &g);
      if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      FE_CK(e);
      const cudaError_t ei = cudaGraphInstantiate(&lg->exec, g, 0);
      cudaGraphDestroy(g);
      FE_CK(ei);
      lg->key = key;
    }
  }
  while (nact > 0 && it < cap) {
    if (graph) {
      FE_CK(cudaGraphLaunch(lg->exec, c.s));
      it += m;
    } else {
      for (int r = 0; r < m; ++r) {
        int st = body();
        if (st) return st;
      }
      it += m;
    }
    int st = read_counter(c, 0, &nact);
    if (st) return st;
  }
  if (done_iters) *done_iters = it;
  return 0;
}

// ---------------------------------------------------------------------------
// autotuner: the expand and segsum variants of the LSMR loop timed on this
// plan's own index data (values are irrelevant to the timing: U and V are
// zeroed scratch), best of two launches each; the winner is kept per (C, T)
// and persisted through tune_cache_{load,store} (fe_solve.cu).
// ---------------------------------------------------------------------------
bool tune_cache_load(fe_plan* pl, int C, int sT, int* ex, int* seg);
void tune_cache_store(fe_plan* pl, int C, int sT, int ex, int seg);

// rows: scratch of N x C elements of T; levels: P x C elements of T (their
// contents are irrelevant to the timing and are left as scratch values)
template <typename T, int C>
static int autotune(fe_plan* pl, Ctx& c, T* rows, T* levels, bool resid_form = false) {
  NvtxRange nv("fe: autotune");
  // tuning key: element size, + 100 for the mixed mode's FP64 refinement
  // kernels (a different expand epilogue than the plain FP64 loop)
  const int kind = (int)sizeof(T) + (resid_form ? 100 : 0);
  const std::pair<int, int> key(C, kind);
  const int ti = sizeof(T) == 8 ? 1 : 0;
  auto f = pl->tuned.find(key);
  if (f != pl->tuned.end()) {
    cur_tune().ex[ti] = f->second.first;
    cur_tune().seg[ti] = f->second.second;
    return 0;
  }
  int ex = 0, seg = 0;
  if (tune_cache_load(pl, C, kind, &ex, &seg)) {
    pl->tuned[key] = {ex, seg};
    cur_tune().ex[ti] = ex;
    cur_tune().seg[ti] = seg;
    return 0;
  }
  if (!pl->opt_autotune) {
    cur_tune().ex[ti] = 0;
    cur_tune().seg[ti] = 0;
    return 0;
  }
  const size_t N = (size_t)pl->N, P = (size_t)pl->P;
  FE_CK(cudaMemsetAsync(rows, 0, N * C * sizeof(T), c.s));
  std::vector<Inst> h((size_t)pl->nprob * C);
  for (Inst& s : h) {
    memset(&s, 0, sizeof(s));
    s.active = 1;
    s.ex_av = 1.0;
    s.ex_au = 0.5;
  }
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  (void)P;
  cudaEvent_t e0, e1;
  FE_CK(cudaEventCreate(&e0));
  FE_CK(cudaEventCreate(&e1));
  const bool prof = pl->prof.on;
  pl->prof.on = false;
  const int save_ex = pl->opt_ex_variant, save_seg = pl->opt_seg_variant;
  EpiExpandLsmr<T, vec_of<T, C>()> ee{};
  ee.U = rows;
  ee.inst = c.inst;
  float best_e = 1e30f, best_s = 1e30f;
  int st = 0;
  for (int v = 0; v < kVariants && !st; ++v) {
    pl->opt_ex_variant = v;
    float ms = 1e30f;
    for (int rep = 0; rep < 3 && !st; ++rep) {
      cudaEventRecord(e0, c.s);
      if constexpr (std::is_same<T, double>::value) {
        if (resid_form) {  // the refinement's r = b - A x (pre-scaled table), all columns
          Workspace& w = pl->ws;
          st = launch_expand<double, C>(
              c, TabPre64<vec_of<double, C>()>{levels},
              EpiBminusAx<double, double, vec_of<double, C>()>{w.B64.as<double>(), rows,
                                                                w.U.as<float>(), c.inst, 0},
              c.part_e, "tune", 0.0);
        } else {
          st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{levels}, ee, c.part_e, "tune", 0.0);
        }
      } else {
        st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{levels}, ee, c.part_e, "tune", 0.0);
      }
      cudaEventRecord(e1, c.s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = std::min(ms, t);
    }
    if (ms < best_e) {
      best_e = ms;
      ex = v;
    }
  }
  for (int v = 0; v < kSegVariants && !st; ++v) {
    pl->opt_seg_variant = v;
    float ms = 1e30f;
    for (int rep = 0; rep < 3 && !st; ++rep) {
      cudaEventRecord(e0, c.s);
      st = launch_segsum<T, C>(c, LoadIn<T, T, vec_of<T, C>()>{rows}, static_cast<T*>(c.S), "tune",
                               0.0, c.rowsum);
      cudaEventRecord(e1, c.s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = std::min(ms, t);
    }
    if (ms < best_s) {
      best_s = ms;
      seg = v;
    }
  }
  pl->opt_ex_variant = save_ex;
  pl->opt_seg_variant = save_seg;
  pl->prof.on = prof;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  // the tuning launches wrote scratch values into S and the item counters are
  // back at zero (every split level completed); clear S for the solve
  FE_CK(cudaMemsetAsync(c.S, 0, P * C * 8, c.s));
  pl->tuned[key] = {ex, seg};
  tune_cache_store(pl, C, kind, ex, seg);
  cur_tune().ex[ti] = ex;
  cur_tune().seg[ti] = seg;
  return 0;
}

// ---------------------------------------------------------------------------
// absorbed loop: the gathered FE's level sums by vector reductions inside the
// pipelined kernel, or by the deterministic level-order segmented sum.  With
// FE_OPT_FIRM_ATOMIC = -1 both are timed once per plan shape on the plan's
// own index data (best of two after a warm-up) and the faster is kept, in
// the plan and in the tuning cache (kind 300).
// ---------------------------------------------------------------------------
template <int C>
static int tune_firm_atomic(fe_plan* pl, Ctx& c, bool* out) {
  *out = false;
  if constexpr (C != 32) {
    (void)pl;
    (void)c;
    return 0;
  } else {
  ExdmChoice ch;
  int st = exdm_choose(c, &ch);
  if (st) return st;
  if (!c.absorb || !pl->opt_exdm || !exdm_atomic_eligible(pl, ch) || pl->opt_firm_atomic == 0)
    return 0;
  if (pl->opt_firm_atomic == 1) {
    *out = true;
    return 0;
  }
  const std::pair<int, int> key(c.C, 300);
  auto f = pl->tuned.find(key);
  if (f != pl->tuned.end()) {
    *out = f->second.first == 1;
    return 0;
  }
  int a = 0, b = 0;
  if (tune_cache_load(pl, c.C, 300, &a, &b)) {
    pl->tuned[key] = {a, 0};
    *out = a == 1;
    return 0;
  }
  if (!pl->opt_autotune) return 0;
  NvtxRange nv("fe: autotune (gathered-FE reduction)");
  Workspace& w = pl->ws;
  std::vector<Inst> h((size_t)pl->nprob * c.C);
  for (Inst& s0 : h) {
    memset(&s0, 0, sizeof(s0));
    s0.active = 1;
    s0.ex_av = 1.0;
    s0.ex_au = 0.5;
  }
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  const int k = ch.lf.large[0];
  float* S32 = static_cast<float*>(c.S);
  const size_t frow = (size_t)pl->lev_base[k] * c.C, fbytes = (size_t)(pl->nlev[k] + 1) * c.C * 4;
  cudaEvent_t e0, e1;
  FE_CK(cudaEventCreate(&e0));
  FE_CK(cudaEventCreate(&e1));
  const bool prof = pl->prof.on;
  pl->prof.on = false;
  float best[2] = {1e30f, 1e30f};
  for (int v = 0; v < 2 && !st; ++v) {
    c.firm_atomic = v == 1;
    for (int rep = 0; rep < 3 && !st; ++rep) {
      cudaEventRecord(e0, c.s);
      if (v == 1 && cudaMemsetAsync(S32 + frow, 0, fbytes, c.s) != cudaSuccess) st = 2;
      if (!st)
        st = launch_expand_demean<float, 32>(c, TabOne<float, float, vec_of<float, 32>()>{w.VS.as<float>()},
                                             w.U.as<float>(), "tune", 0.0);
      if (!st && v == 0)
        st = launch_segsum<float, 32>(c, LoadIn<float, float, vec_of<float, 32>()>{w.U.as<float>()}, S32,
                                      "tune", 0.0, true, "", 0.0, true);
      cudaEventRecord(e1, c.s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) best[v] = std::min(best[v], t);
    }
  }
  c.firm_atomic = false;
  pl->prof.on = prof;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  FE_CK(cudaMemsetAsync(c.S, 0, (size_t)pl->P * c.C * 8, c.s));
  const int choice = best[1] < best[0] ? 1 : 0;
  pl->tuned[key] = {choice, 0};
  tune_cache_store(pl, c.C, 300, choice, 0);
  pl->last_firm_tune_ms[0] = best[0];
  pl->last_firm_tune_ms[1] = best[1];
  *out = choice == 1;
  return 0;
  }
}

// ---------------------------------------------------------------------------
// coefficient download (solve_coefficients!)
// ---------------------------------------------------------------------------
template <typename TX>
static int download_coefs(fe_plan* pl, Ctx& c, const TX* X, const SolveReq& rq) {
  Workspace& w = pl->ws;
  for (int k = 0; k < pl->K; ++k) {
    const int64_t n = pl->nlev[k];
    if (!n) continue;
    int st = w.coef.ensure((size_t)n * 8);
    if (st) return st;
    k_coefs<TX><<<grid1(n), 256, 0, c.s>>>(X, c.C, 0, pl->lev_base[k], n,
                                             pl->d_scale_d[k].as<double>(), w.coef.as<double>());
    FE_CK(cudaGetLastError());
    FE_CK(cudaMemcpyAsync(rq.coefs[k], w.coef.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c.s));
    FE_CK(cudaStreamSynchronize(c.s));
  }
  return 0;
}

// ---------------------------------------------------------------------------
// plain LSMR (bulk type T) on one tile
// ---------------------------------------------------------------------------
template <typename T, int C>
static int solve_plain_tile(fe_plan* pl, const SolveReq& rq, int64_t col0, int ncols,
                            std::vector<Inst>& out) {
  NvtxRange nv("fe: tile (plain LSMR)");
  Ctx c;
  int st = prepare(pl, C, (int)sizeof(T), false, c);
  if (st) return st;
  if ((st = autotune<T, C>(pl, c, pl->ws.U.as<T>(), pl->ws.V.as<T>()))) return st;
  Workspace& w = pl->ws;
  const Bytes by = alg_bytes(pl, c.its, C, (int)sizeof(T));
  std::vector<Inst> h;
  init_insts(pl, rq, C, ncols, h);
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  if ((st = load_tile<C>(pl, c, rq, col0, ncols))) return st;
  T* U = w.U.as<T>();
  T* V = w.V.as<T>();
  T* X = w.X.as<T>();
  double* B64 = w.B64.as<double>();
  double* S64 = static_cast<double*>(c.S);
  T* ST = static_cast<T*>(c.S);
  // warm start x = A'b (src/AbstractFixedEffectSolver.jl:56); solve_coefficients! starts at 0
  if (rq.residuals) {
    if ((st = zero_slab(c, S64, 8))) return st;
    if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{B64}, S64, "segsum_warm", 0.0,
                                        c.rowsum, "rowsum_warm", 0.0)))
      return st;
    if ((st = xchg_slab(c, S64, 8))) return st;
    if ((st = launch_pupdate<C>(c, S64, PEpiStoreX<T, vec_of<double, C>()>{X, true}, nullptr, nullptr, "pupdate_warm", 0.0)))
      return st;
  }
  // u = b - A x, beta (lsmr.jl:63-64)
  const bool fuse = c.rowsum;
  if ((st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{X},
                                EpiBminusAx<T, T, vec_of<T, C>()>{B64, U, nullptr, c.inst, 0}, c.part_e,
                                "expand_init", by.expand)))
    return st;
  if ((st = xchg_slots(c, c.part_e))) return st;
  if ((st = launch_scalar_phase(c, PH_INIT_BETA, 0))) return st;
  PEpiLsmr<T, vec_of<T, C>()> pe{};
  pe.V = V;
  pe.H = w.H.as<T>();
  pe.Hb = w.Hb.as<T>();
  pe.X = X;
  pe.inst = c.inst;
  if ((st = zero_slab(c, ST, (int)sizeof(T)))) return st;
  if ((st = launch_segsum<T, C>(c, LoadIn<T, T, vec_of<T, C>()>{U}, ST, "segsum", by.segsum, fuse,
                                "rowsum", by.rowsum)))
    return st;
  if ((st = xchg_slab(c, ST, (int)sizeof(T)))) return st;
  if ((st = launch_pupdate<C>(c, ST, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return st;
  if ((st = launch_scalar_phase(c, PH_INIT_ALPHA, 1))) return st;
  int32_t nact = 0;
  if ((st = read_counter(c, 0, &nact))) return st;
  EpiExpandLsmr<T, vec_of<T, C>()> ee{};
  ee.U = U;
  ee.inst = c.inst;
  const int64_t cap = std::max<int64_t>(rq.maxiter, 1) + 2;
  auto body = [&]() -> int {
    int e;
    if ((e = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{V}, ee, c.part_e, "expand", by.expand)))
      return e;
    if ((e = xchg_slots(c, c.part_e))) return e;
    if ((e = launch_scalar_phase(c, PH_BETA, 0))) return e;
    if ((e = zero_slab(c, ST, (int)sizeof(T)))) return e;
    if ((e = launch_segsum<T, C>(c, LoadIn<T, T, vec_of<T, C>()>{U}, ST, "segsum", by.segsum, fuse,
                                 "rowsum", by.rowsum)))
      return e;
    if ((e = xchg_slab(c, ST, (int)sizeof(T)))) return e;
    if ((e = launch_pupdate<C>(c, ST, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return e;
    return launch_scalar_phase(c, PH_ALPHA, 0);
  };
  c.d.active = c.counters + 2;
  st = run_loop(pl, c, (int)sizeof(T), cap, nact, body, nullptr);
  c.d.active = nullptr;
  if (st) return st;
  if (rq.residuals) {
    // r = b - A x (src/AbstractFixedEffectSolver.jl:62)
    if ((st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{X},
                                  EpiBminusAx<double, T, vec_of<T, C>()>{B64, w.R64.as<double>(), nullptr, c.inst, 0},
                                  nullptr, "expand_final", by.expand)))
      return st;
    if ((st = unload_tile<C>(pl, c, rq, col0, ncols))) return st;
  }
  out.resize(h.size());
  FE_CK(cudaMemcpyAsync(out.data(), c.inst, h.size() * sizeof(Inst), cudaMemcpyDeviceToHost, c.s));
  FE_CK(cudaStreamSynchronize(c.s));
  if (!rq.residuals && rq.coefs) {
    if ((st = download_coefs<T>(pl, c, X, rq))) return st;
  }
  return prof_flush(pl);
}

// ---------------------------------------------------------------------------
// mixed precision: FP32 inner LSMR + FP64 iterative refinement, one tile
// ---------------------------------------------------------------------------
template <int C>
static int solve_mixed_tile(fe_plan* pl, const SolveReq& rq, int64_t col0, int ncols,
                            std::vector<Inst>& out) {
  NvtxRange nv("fe: tile (mixed precision)");
  Ctx c;
  int st = prepare(pl, C, 4, true, c);
  if (st) return st;
  // FP32 loop kernels on U/V; FP64 refinement kernels on R64/X64 (FP64-sized)
  if ((st = autotune<float, C>(pl, c, pl->ws.U.as<float>(), pl->ws.V.as<float>()))) return st;
  if ((st = autotune<double, C>(pl, c, pl->ws.R64.as<double>(), pl->ws.X64.as<double>(), true)))
    return st;
  Workspace& w = pl->ws;
  const Bytes by = alg_bytes(pl, c.its, C, 4);
  // absorbed-primary mode (residual solves): LSMR over the other FEs, from
  // x0 = 0 (the reference's warm start A'b belongs to the full problem)
  const bool absorb = rq.residuals && use_absorb(pl, c.its, C);
  c.absorb = absorb;
  c.d.absorb = absorb ? 1 : 0;
  // the absorbed LSMR runs on M A_r with its own column scales 1 / ||M a_l||
  // (the projection shrinks the columns unevenly); the primary FE keeps its
  // Jacobi scale, which the projection itself uses
  if (absorb && pl->opt_abs_scale)
    for (int k = 0; k < pl->K; ++k)
      if (k != pl->primary && pl->d_abs_scale_d[k].p) {
        c.d.scale_d[k] = pl->d_abs_scale_d[k].as<double>();
        c.d.scale_f[k] = pl->d_abs_scale_f[k].as<float>();
      }
  // the gathered FE's reduction (timed on scratch before the tile is loaded)
  if (absorb && (st = tune_firm_atomic<C>(pl, c, &c.firm_atomic))) return st;
  std::vector<Inst> h;
  init_insts(pl, rq, C, ncols, h);
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  if ((st = load_tile<C>(pl, c, rq, col0, ncols))) return st;
  float* U = w.U.as<float>();
  float* V = w.V.as<float>();
  float* X = w.X.as<float>();
  double* X64 = w.X64.as<double>();
  double* B64 = w.B64.as<double>();
  double* R64 = w.R64.as<double>();
  double* S64 = static_cast<double*>(c.S);
  float* S32 = static_cast<float*>(c.S);
  if (rq.residuals && pl->opt_mixed_warm && !absorb) {
    if ((st = zero_slab(c, S64, 8))) return st;
    if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{B64}, S64, "segsum_warm", 0.0,
                                        c.rowsum, "rowsum_warm", 0.0)))
      return st;
    if ((st = xchg_slab(c, S64, 8))) return st;
    if ((st = launch_pupdate<C>(c, S64, PEpiStoreX<double, vec_of<double, C>()>{X64, true}, nullptr, nullptr,
                                "pupdate_warm", 0.0)))
      return st;
  }
  PEpiLsmr<float, vec_of<float, C>()> pe{};
  pe.V = V;
  pe.H = w.H.as<float>();
  pe.Hb = w.Hb.as<float>();
  pe.X = X;
  pe.inst = c.inst;
  EpiExpandLsmr<float, vec_of<float, C>()> ee{};
  ee.U = U;
  ee.inst = c.inst;
  PEpiGrad64<vec_of<double, C>()> pg{};
  pg.V32 = V;
  pg.X64 = X64;
  pg.X32 = X;
  pg.inst = c.inst;
  // the fused absorbed loop gathers scale * v, kept beside v by both P-side
  // updates
  // (32-column tiles; narrower tiles run the expand, then the projection)
  const bool exdm = absorb && pl->opt_exdm && C == 32;
  float* VS = exdm ? w.VS.as<float>() : nullptr;
  pe.VS = VS;
  pg.VS32 = VS;
  const int64_t cap = std::max<int64_t>(rq.maxiter, 1) + 2;
  int64_t total_it = 0;
  const bool fuse = c.rowsum;
  for (int round = 0; round <= pl->opt_max_rounds + 1; ++round) {
    NvtxRange nvr("fe: FP64 refinement round");
    FE_CK(cudaMemsetAsync(c.counters, 0, 3 * sizeof(int32_t), c.s));
    // r = b - A (x64 + dx32) in FP64, with the FP32 copy as the next inner u
    // (absorbed: r = M (b - A_r x), projected and copied by the demean pass)
    // absorbed: round 0 starts from x = 0, so r0 = M b comes straight from b
    const bool from_b = absorb && round == 0;
    // absorbed rounds after the first, FE_OPT_FUSED_RESID: the residual and
    // its projection in one pass, by the demean kernel (2, and the default
    // where it fits) or by the staged fused kernel (1)
    const int fres = C != 32 ? 0
                     : pl->opt_fused_resid < 0 ? (resid_demean_fits(pl) ? 2 : 0)
                                               : (pl->opt_fused_resid == 2 && !resid_demean_fits(pl)
                                                      ? 0 : pl->opt_fused_resid);
    const bool fused_r = absorb && !from_b && fres != 0;
    if ((st = zero_slab(c, S64, 8))) return st;
    if (!from_b && (st = launch_prescale64(c, X64, X, w.XS64.as<double>(), absorb,
                                           absorb ? by.prescale64_abs : by.prescale64)))
      return st;
    if (!from_b && !fused_r &&
        (st = launch_expand<double, C>(
             c, TabPre64<vec_of<double, C>()>{w.XS64.as<double>()},
             EpiBminusAx<double, double, vec_of<double, C>()>{B64, R64, absorb ? nullptr : U, c.inst, 2},
             absorb ? nullptr : c.part_e, "resid64", absorb ? by.resid64_abs : by.resid64)))
      return st;
    // g = A'r in FP64 (the next inner v), x64 += dx32, ||x64||
    if (absorb) {
      if (fused_r && fres == 2) {
        if ((st = launch_demean<double, C>(c, R64, U, S64, "resid_demean64", by.resid_dm64, B64,
                                           w.XS64.as<double>())))
          return st;
      } else if (fused_r) {
        if ((st = launch_resid_demean<C>(c, w.XS64.as<double>(), R64, B64, U, by.resid_demean64)))
          return st;
      } else if ((st = launch_demean<double, C>(c, R64, U, S64, "demean64", by.demean64,
                                                from_b ? B64 : nullptr))) {
        return st;
      }
      if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{R64}, S64,
                                         "segsum64", by.segsum64_abs, true, "", 0.0, true)))
        return st;
    } else if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{R64}, S64,
                                              "segsum64", by.segsum64, fuse, "rowsum64", by.rowsum64))) {
      return st;
    }
    if ((st = xchg_slots(c, c.part_e))) return st;
    if ((st = xchg_slab(c, S64, 8))) return st;
    if ((st = launch_pupdate<C>(c, S64, pg, c.part_a, c.part_b, "grad64",
                                absorb ? by.grad64_np : by.grad64)))
      return st;
    if ((st = launch_scalar_phase(c, PH_OUTER, 0))) return st;
    int32_t nout = 0;
    if ((st = read_counter(c, 1, &nout))) return st;
    if (nout == 0) break;
    auto body = [&]() -> int {
      int e;
      if (absorb) {
        // u = M (av A_r v + au u): the expand without the primary FE, then the
        // projection (which also gives ||u|| and the small FEs' sums)
        if ((e = zero_slab(c, S32, 4))) return e;
        if (c.firm_atomic) {
          // the gathered FE's level sums are added by the fused kernel
          for (int k = 0; k < pl->K; ++k)
            if (k != pl->primary && !((c.its->small_mask >> k) & 1u))
              FE_CK(cudaMemsetAsync(S32 + (size_t)pl->lev_base[k] * C, 0,
                                    (size_t)(pl->nlev[k] + 1) * C * 4, c.s));
        }
        if (exdm) {
          if ((e = launch_expand_demean<float, C>(c, TabOne<float, float, vec_of<float, C>()>{VS}, U,
                                                  "expand_demean", by.expand_demean)))
            return e;
        } else {
          if ((e = launch_expand<float, C>(c, TabOne<float, float, vec_of<float, C>()>{V}, ee, nullptr,
                                           "expand", by.expand_abs)))
            return e;
          if ((e = launch_demean<float, C>(c, U, nullptr, S32, "demean", by.demean))) return e;
        }
        if ((e = xchg_slots(c, c.part_e))) return e;
        if ((e = launch_scalar_phase(c, PH_BETA, 0))) return e;
        if (!c.firm_atomic &&
            (e = launch_segsum<float, C>(c, LoadIn<float, float, vec_of<float, C>()>{U}, S32, "segsum",
                                         by.segsum_abs, true, "", 0.0, true)))
          return e;
        if ((e = xchg_slab(c, S32, 4))) return e;
        if ((e = launch_pupdate<C>(c, S32, pe, c.part_a, c.part_b, "pupdate", by.pupdate_np))) return e;
        return launch_scalar_phase(c, PH_ALPHA, 0);
      }
      if ((e = launch_expand<float, C>(c, TabOne<float, float, vec_of<float, C>()>{V}, ee, c.part_e,
                                       "expand", by.expand)))
        return e;
      if ((e = xchg_slots(c, c.part_e))) return e;
      if ((e = launch_scalar_phase(c, PH_BETA, 0))) return e;
      if ((e = zero_slab(c, S32, 4))) return e;
      if ((e = launch_segsum<float, C>(c, LoadIn<float, float, vec_of<float, C>()>{U}, S32, "segsum",
                                       by.segsum, fuse, "rowsum", by.rowsum)))
        return e;
      if ((e = xchg_slab(c, S32, 4))) return e;
      if ((e = launch_pupdate<C>(c, S32, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return e;
      return launch_scalar_phase(c, PH_ALPHA, 0);
    };
    int64_t done = 0;
    c.d.active = c.counters + 2;
    c.d.active_pre = c.counters;
    st = run_loop(pl, c, 1, cap - total_it, nout, body, &done);
    c.d.active = nullptr;
    c.d.active_pre = nullptr;
    if (st) return st;
    total_it += done;
  }
  if (rq.residuals) {
    if ((st = unload_tile<C>(pl, c, rq, col0, ncols))) return st;
  }
  out.resize(h.size());
  FE_CK(cudaMemcpyAsync(out.data(), c.inst, h.size() * sizeof(Inst), cudaMemcpyDeviceToHost, c.s));
  FE_CK(cudaStreamSynchronize(c.s));
  if (!rq.residuals && rq.coefs) {
    if ((st = download_coefs<double>(pl, c, X64, rq))) return st;
  }
  return prof_flush(pl);
}

template <int C>
int solve_tile_C(fe_plan* pl, const SolveReq& rq, int64_t col0, int ncols,
                        std::vector<Inst>& out) {
  switch (rq.precision) {
    case 0:
      return solve_plain_tile<double, C>(pl, rq, col0, ncols, out);
    case 2:
      return solve_plain_tile<float, C>(pl, rq, col0, ncols, out);
    default:
      return solve_mixed_tile<C>(pl, rq, col0, ncols, out);
  }
}

}  // namespace fe
