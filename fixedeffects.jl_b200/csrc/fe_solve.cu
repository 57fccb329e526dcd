// fe_solve.cu -- solve drivers of the fixed-effects LSMR hot path.
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

#include "fe_kernels.cuh"
#include "fe_plan.h"
#include "fe_solve.h"

namespace fe {

// ---------------------------------------------------------------------------
// load / unload / coefficient kernels
// ---------------------------------------------------------------------------
// B[q][j] = y[i][col0 + j] * sqrt(w_i) with q the sorted position of i
// (src/AbstractFixedEffectSolver.jl:50-55).  Reads are coalesced per column;
// each thread writes one whole row of B.
template <typename TY>
__global__ void k_load(const TY* __restrict__ Y, int64_t ld, int64_t col0, int ncols, int C,
                       const int32_t* __restrict__ dst, const double* __restrict__ sw,
                       double* __restrict__ B, int64_t N) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t q = dst[i];
  const double w = sw ? sw[i] : 1.0;
  for (int j = 0; j < C; ++j)
    B[q * C + j] = j < ncols ? (double)Y[i + (col0 + j) * ld] * w : 0.0;
}

// y[i][col0 + j] = R[q][j] / sqrt(w_i)  (src/AbstractFixedEffectSolver.jl:62-66)
template <typename TY>
__global__ void k_unload(const double* __restrict__ R, int64_t ld, int64_t col0, int ncols, int C,
                         const int32_t* __restrict__ dst, const double* __restrict__ sw,
                         TY* __restrict__ Y, int64_t N) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t q = dst[i];
  const double w = sw ? sw[i] : 1.0;
  for (int j = 0; j < ncols; ++j) Y[i + (col0 + j) * ld] = (TY)(R[q * C + j] / w);
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

int prof_flush(fe_plan* pl) {
  if (pl->prof.pending.empty()) return 0;
  FE_CK(cudaStreamSynchronize(pl->stream));
  for (auto& pr : pl->prof.pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pr.second.first, pr.second.second);
    KernelStat& st = pl->prof.stats[pr.first];
    st.name = pr.first;
    st.launches += 1;
    st.ms += ms;
    st.bytes += pl->prof.bytes_per_launch[pr.first];
    pl->prof.pool.push_back(pr.second.first);
    pl->prof.pool.push_back(pr.second.second);
  }
  pl->prof.pending.clear();
  return 0;
}

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
  void* S;
};

// unroll depths (row slots per lane group per step)
template <int C> struct Tune {
  static constexpr int kExpandU = 4;
  static constexpr int kSegU = 8;
  static constexpr int kPU = 4;
};
template <typename T, int C> constexpr int vec_of() { return Shape<T, C>::VEC; }

template <typename TA, int C, class Tab, class Epi>
static int launch_expand(Ctx& c, Tab tab, Epi epi, double* part, const char* name, double bytes) {
  ProfScope ps(c.pl, name, bytes);
  const unsigned grid = (unsigned)(c.its->ex.size() / kWarps);
  const ExpandItem* items = c.its->d_ex.as<ExpandItem>();
  const int64_t n = (int64_t)c.its->ex.size();
  constexpr int U = Tune<C>::kExpandU;
  if (c.d.K <= 2)
    k_expand<TA, C, U, 2, Tab, Epi><<<grid, kThreads, 0, c.s>>>(c.d, items, n, tab, epi, part, c.its->Se);
  else if (c.d.K <= 4)
    k_expand<TA, C, U, 4, Tab, Epi><<<grid, kThreads, 0, c.s>>>(c.d, items, n, tab, epi, part, c.its->Se);
  else
    k_expand<TA, C, U, kMaxFE, Tab, Epi><<<grid, kThreads, 0, c.s>>>(c.d, items, n, tab, epi, part, c.its->Se);
  FE_CK(cudaGetLastError());
  return 0;
}

template <typename TA, int C, class Load>
static int launch_segsum(Ctx& c, Load ld, TA* out, const char* name, double bytes) {
  if (c.its->rd.empty()) return 0;
  ProfScope ps(c.pl, name, bytes);
  const unsigned grid = (unsigned)((c.its->rd.size() + kWarps - 1) / kWarps);
  k_segsum<TA, C, Tune<C>::kSegU, Load><<<grid, kThreads, 0, c.s>>>(
      c.d, c.its->d_rd.as<ReduceItem>(), (int64_t)c.its->rd.size(), ld, out,
      c.its->d_splits.as<SplitLevel>(), c.piece, c.its->n_pieces, c.its->d_split_cnt.as<int32_t>());
  FE_CK(cudaGetLastError());
  return 0;
}

template <int C, class Epi>
static int launch_pupdate(Ctx& c, const typename Epi::TS* S, Epi epi, double* pa, double* pb,
                          const char* name, double bytes) {
  ProfScope ps(c.pl, name, bytes);
  const unsigned grid = (unsigned)(c.its->pu.size() / kWarps);
  k_pupdate<C, Tune<C>::kPU, Epi><<<grid, kThreads, 0, c.s>>>(
      c.d, c.its->d_pu.as<PItem>(), (int64_t)c.its->pu.size(), S, epi, pa, pb, c.its->Sp);
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
  a.off0 = c.its->d_ex_off.as<int64_t>();
  a.S0 = c.its->Se;
  a.off1 = c.its->d_pu_off.as<int64_t>();
  a.S1 = c.its->Sp;
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

// algorithmic bytes per launch (the roofline numerators): every index vector
// and observation row once, every coefficient-table row once
struct Bytes {
  double expand, segsum, pupdate, resid64, segsum64, grad64;
};
static Bytes alg_bytes(const fe_plan* pl, int C, int sT) {
  Bytes b{};
  const double N = (double)pl->N;
  double P = 0, pos = 0, posmeta = 0, cw = 0, cw64 = 0, cwp = 0, cwp64 = 0;
  for (int k = 0; k < pl->K; ++k) {
    P += (double)pl->nlev[k];
    pos += (double)pl->seg_len[k];
    posmeta += (double)pl->seg_len[k] * (4.0 + (pl->perm_identity[k] ? 0.0 : 4.0));
    const bool has_cw = pl->weighted || pl->interacted[k];
    if (has_cw) {
      cw += N * sT;
      cw64 += N * 8.0;
      cwp += (double)pl->seg_len[k] * sT;
      cwp64 += (double)pl->seg_len[k] * 8.0;
    }
  }
  const double refs = N * 4.0 * pl->K;
  b.expand = refs + cw + 2.0 * N * C * sT + P * C * sT;
  b.segsum = posmeta + cwp + pos * C * sT + P * C * sT;
  b.pupdate = 9.0 * P * C * sT;
  b.resid64 = refs + cw64 + N * C * (8.0 + 8.0 + 4.0) + P * C * 12.0;
  b.segsum64 = posmeta + cwp64 + pos * C * 8.0 + P * C * 8.0;
  b.grad64 = P * C * (8.0 + 4.0 + 8.0 + 4.0 + 8.0);
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
  if ((st = w.H.ensure(P * nC * (size_t)sT))) return st;
  if ((st = w.Hb.ensure(P * nC * (size_t)sT))) return st;
  if ((st = w.X.ensure(P * nC * (size_t)sT))) return st;
  if (mixed && (st = w.X64.ensure(P * nC * 8))) return st;
  if ((st = w.part_e.ensure((size_t)std::max<int64_t>(its->Se, 1) * nC * 8))) return st;
  if ((st = w.part_a.ensure((size_t)std::max<int64_t>(its->Sp, 1) * nC * 8))) return st;
  if ((st = w.part_b.ensure((size_t)std::max<int64_t>(its->Sp, 1) * nC * 8))) return st;
  if ((st = w.S.ensure(P * nC * 8))) return st;
  if ((st = w.piece_part.ensure((size_t)std::max<int64_t>(its->n_pieces, 1) * nC * 8))) return st;
  if ((st = w.inst.ensure((size_t)pl->nprob * nC * sizeof(Inst)))) return st;
  if ((st = w.counters.ensure(64))) return st;
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
  c.S = w.S.p;
  // coefficient-side slabs start at zero (levels without observations and
  // the null levels are never written afterwards)
  FE_CK(cudaMemsetAsync(w.V.p, 0, P * nC * (size_t)sT, c.s));
  FE_CK(cudaMemsetAsync(w.H.p, 0, P * nC * (size_t)sT, c.s));
  FE_CK(cudaMemsetAsync(w.Hb.p, 0, P * nC * (size_t)sT, c.s));
  FE_CK(cudaMemsetAsync(w.X.p, 0, P * nC * (size_t)sT, c.s));
  if (mixed) FE_CK(cudaMemsetAsync(w.X64.p, 0, P * nC * 8, c.s));
  FE_CK(cudaMemsetAsync(w.S.p, 0, P * nC * 8, c.s));
  FE_CK(cudaMemsetAsync(c.counters, 0, 64, c.s));
  return 0;
}

static int load_tile(fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  const int64_t N = pl->N;
  if (N == 0) return 0;
  const double* sw = pl->weighted ? pl->d_sw_orig.as<double>() : nullptr;
  ProfScope ps(pl, "load", (double)N * ncols * (rq.dtype == 0 ? 8 : 4) + (double)N * c.C * 8);
  if (rq.dtype == 0)
    k_load<double><<<grid1(N), 256, 0, c.s>>>((const double*)rq.Y, rq.ld, col0, ncols, c.C,
                                                pl->d_obs_dst.as<int32_t>(), sw,
                                                pl->ws.B64.as<double>(), N);
  else
    k_load<float><<<grid1(N), 256, 0, c.s>>>((const float*)rq.Y, rq.ld, col0, ncols, c.C,
                                               pl->d_obs_dst.as<int32_t>(), sw,
                                               pl->ws.B64.as<double>(), N);
  FE_CK(cudaGetLastError());
  return 0;
}

static int unload_tile(fe_plan* pl, Ctx& c, const SolveReq& rq, int64_t col0, int ncols) {
  const int64_t N = pl->N;
  if (N == 0) return 0;
  const double* sw = pl->weighted ? pl->d_sw_orig.as<double>() : nullptr;
  ProfScope ps(pl, "unload", (double)N * ncols * (rq.dtype == 0 ? 8 : 4) + (double)N * c.C * 8);
  if (rq.dtype == 0)
    k_unload<double><<<grid1(N), 256, 0, c.s>>>(pl->ws.R64.as<double>(), rq.ld, col0, ncols, c.C,
                                                  pl->d_obs_dst.as<int32_t>(), sw, (double*)rq.Y, N);
  else
    k_unload<float><<<grid1(N), 256, 0, c.s>>>(pl->ws.R64.as<double>(), rq.ld, col0, ncols, c.C,
                                                 pl->d_obs_dst.as<int32_t>(), sw, (float*)rq.Y, N);
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
  Ctx c;
  int st = prepare(pl, C, (int)sizeof(T), false, c);
  if (st) return st;
  Workspace& w = pl->ws;
  const Bytes by = alg_bytes(pl, C, (int)sizeof(T));
  std::vector<Inst> h;
  init_insts(pl, rq, C, ncols, h);
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  if ((st = load_tile(pl, c, rq, col0, ncols))) return st;
  T* U = w.U.as<T>();
  T* V = w.V.as<T>();
  T* X = w.X.as<T>();
  double* B64 = w.B64.as<double>();
  double* S64 = static_cast<double*>(c.S);
  T* ST = static_cast<T*>(c.S);
  // warm start x = A'b (src/AbstractFixedEffectSolver.jl:56); solve_coefficients! starts at 0
  if (rq.residuals) {
    if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{B64}, S64, "segsum_warm", 0.0)))
      return st;
    if ((st = launch_pupdate<C>(c, S64, PEpiStoreX<T, vec_of<double, C>()>{X, true}, nullptr, nullptr, "pupdate_warm", 0.0)))
      return st;
  }
  // u = b - A x, beta (lsmr.jl:63-64)
  if ((st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{X},
                                EpiBminusAx<T, T, vec_of<T, C>()>{B64, U, nullptr, c.inst, 0}, c.part_e,
                                "expand_init", by.expand)))
    return st;
  if ((st = launch_scalar_phase(c, PH_INIT_BETA, 0))) return st;
  PEpiLsmr<T, vec_of<T, C>()> pe{};
  pe.V = V;
  pe.H = w.H.as<T>();
  pe.Hb = w.Hb.as<T>();
  pe.X = X;
  pe.inst = c.inst;
  if ((st = launch_segsum<T, C>(c, LoadIn<T, T, vec_of<T, C>()>{U}, ST, "segsum", by.segsum))) return st;
  if ((st = launch_pupdate<C>(c, ST, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return st;
  if ((st = launch_scalar_phase(c, PH_INIT_ALPHA, 1))) return st;
  int32_t nact = 0;
  if ((st = read_counter(c, 0, &nact))) return st;
  EpiExpandLsmr<T, vec_of<T, C>()> ee{};
  ee.U = U;
  ee.inst = c.inst;
  const int64_t cap = std::max<int64_t>(rq.maxiter, 1) + 2;
  for (int64_t it = 1; nact > 0 && it <= cap; ++it) {
    if ((st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{V}, ee, c.part_e, "expand", by.expand))) return st;
    if ((st = launch_scalar_phase(c, PH_BETA, 0))) return st;
    if ((st = launch_segsum<T, C>(c, LoadIn<T, T, vec_of<T, C>()>{U}, ST, "segsum", by.segsum))) return st;
    if ((st = launch_pupdate<C>(c, ST, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return st;
    if ((st = launch_scalar_phase(c, PH_ALPHA, 0))) return st;
    if (it % pl->opt_check_every == 0 || it == cap) {
      if ((st = read_counter(c, 0, &nact))) return st;
    }
  }
  if (rq.residuals) {
    // r = b - A x (src/AbstractFixedEffectSolver.jl:62)
    if ((st = launch_expand<T, C>(c, TabOne<T, T, vec_of<T, C>()>{X},
                                  EpiBminusAx<double, T, vec_of<T, C>()>{B64, w.R64.as<double>(), nullptr, c.inst, 0},
                                  nullptr, "expand_final", by.expand)))
      return st;
    if ((st = unload_tile(pl, c, rq, col0, ncols))) return st;
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
  Ctx c;
  int st = prepare(pl, C, 4, true, c);
  if (st) return st;
  Workspace& w = pl->ws;
  const Bytes by = alg_bytes(pl, C, 4);
  std::vector<Inst> h;
  init_insts(pl, rq, C, ncols, h);
  FE_CK(cudaMemcpyAsync(c.inst, h.data(), h.size() * sizeof(Inst), cudaMemcpyHostToDevice, c.s));
  if ((st = load_tile(pl, c, rq, col0, ncols))) return st;
  float* U = w.U.as<float>();
  float* V = w.V.as<float>();
  float* X = w.X.as<float>();
  double* X64 = w.X64.as<double>();
  double* B64 = w.B64.as<double>();
  double* R64 = w.R64.as<double>();
  double* S64 = static_cast<double*>(c.S);
  float* S32 = static_cast<float*>(c.S);
  if (rq.residuals) {
    if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{B64}, S64, "segsum_warm", 0.0)))
      return st;
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
  const int64_t cap = std::max<int64_t>(rq.maxiter, 1) + 2;
  int64_t total_it = 0;
  for (int round = 0; round <= pl->opt_max_rounds + 1; ++round) {
    FE_CK(cudaMemsetAsync(c.counters + 1, 0, sizeof(int32_t), c.s));
    // r = b - A (x64 + dx32) in FP64, with the FP32 copy as the next inner u
    if ((st = launch_expand<double, C>(c, TabSum64<vec_of<double, C>()>{X64, X},
                                       EpiBminusAx<double, double, vec_of<double, C>()>{B64, R64, U, c.inst, 2},
                                       c.part_e, "resid64", by.resid64)))
      return st;
    // g = A'r in FP64 (the next inner v), x64 += dx32, ||x64||
    if ((st = launch_segsum<double, C>(c, LoadIn<double, double, vec_of<double, C>()>{R64}, S64, "segsum64", by.segsum64)))
      return st;
    if ((st = launch_pupdate<C>(c, S64, pg, c.part_a, c.part_b, "grad64", by.grad64))) return st;
    if ((st = launch_scalar_phase(c, PH_OUTER, 0))) return st;
    int32_t nout = 0;
    if ((st = read_counter(c, 1, &nout))) return st;
    if (nout == 0) break;
    int32_t nact = nout;
    for (int64_t it = 1; nact > 0 && total_it < cap; ++it, ++total_it) {
      if ((st = launch_expand<float, C>(c, TabOne<float, float, vec_of<float, C>()>{V}, ee, c.part_e, "expand", by.expand)))
        return st;
      if ((st = launch_scalar_phase(c, PH_BETA, 0))) return st;
      if ((st = launch_segsum<float, C>(c, LoadIn<float, float, vec_of<float, C>()>{U}, S32, "segsum", by.segsum))) return st;
      if ((st = launch_pupdate<C>(c, S32, pe, c.part_a, c.part_b, "pupdate", by.pupdate))) return st;
      if ((st = launch_scalar_phase(c, PH_ALPHA, 0))) return st;
      if (it % pl->opt_check_every == 0) {
        if ((st = read_counter(c, 0, &nact))) return st;
      }
    }
  }
  if (rq.residuals) {
    if ((st = unload_tile(pl, c, rq, col0, ncols))) return st;
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
static int solve_tile_C(fe_plan* pl, const SolveReq& rq, int64_t col0, int ncols,
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

static int tile_width(const fe_plan* pl, int64_t remaining) {
  int cmax = 32;
  if (pl->opt_tile > 0) cmax = pl->opt_tile;
  int64_t want = std::min<int64_t>(remaining, cmax);
  int C = 1;
  while (C < want) C <<= 1;
  return std::min(C, 32);
}

int solve(fe_plan* pl, const SolveReq& rq) {
  FE_CK(cudaSetDevice(pl->device));
  const int64_t ncols = rq.ncols;
  pl->last_test2.assign((size_t)ncols, 0.0);
  pl->last_rounds.assign((size_t)ncols, 0);
  pl->last_iters_raw.assign((size_t)ncols, 0);
  if (pl->N == 0) {
    for (int64_t j = 0; j < ncols; ++j) {
      if (rq.iters) rq.iters[j] = rq.residuals ? 1 : 0;
      if (rq.converged) rq.converged[j] = 1;
    }
    return 0;
  }
  std::vector<Inst> res;
  for (int64_t col0 = 0; col0 < ncols;) {
    const int C = tile_width(pl, ncols - col0);
    const int nc = (int)std::min<int64_t>(C, ncols - col0);
    int st;
    switch (C) {
      case 1: st = solve_tile_C<1>(pl, rq, col0, nc, res); break;
      case 2: st = solve_tile_C<2>(pl, rq, col0, nc, res); break;
      case 4: st = solve_tile_C<4>(pl, rq, col0, nc, res); break;
      case 8: st = solve_tile_C<8>(pl, rq, col0, nc, res); break;
      case 16: st = solve_tile_C<16>(pl, rq, col0, nc, res); break;
      default: st = solve_tile_C<32>(pl, rq, col0, nc, res); break;
    }
    if (st) return st;
    // per-column verdicts: a column's instances are (problem p, column j);
    // with several problems the column aggregates them (max iterations, all
    // converged).  Single-problem plans report the instance itself.
    for (int j = 0; j < nc; ++j) {
      int64_t itmax = 0, raw = 0;
      bool conv = true;
      double t2 = 0.0;
      int32_t rounds = 0;
      for (int p = 0; p < pl->nprob; ++p) {
        const Inst& s = res[(size_t)p * C + j];
        int64_t it;
        bool cv;
        if (rq.precision == 1) {
          raw = std::max<int64_t>(raw, s.iter_total);
          it = rq.residuals ? s.iter_total + 1 : s.iter_total / 2;
          cv = s.converged != 0;
          t2 = std::max(t2, s.last_test2);
          rounds = std::max(rounds, s.outer_rounds);
        } else {
          raw = std::max<int64_t>(raw, s.iter);
          it = rq.residuals ? (s.skip_lsmr ? 1 : s.iter + 1) : s.iter / 2;
          cv = !(s.istop == 3 || s.istop == 6 || s.istop == 7);
        }
        itmax = std::max(itmax, it);
        conv = conv && cv;
        if (rq.prob_iters) rq.prob_iters[(size_t)p * ncols + col0 + j] = it;
        if (rq.prob_converged) rq.prob_converged[(size_t)p * ncols + col0 + j] = cv ? 1 : 0;
      }
      if (rq.iters) rq.iters[col0 + j] = itmax;
      if (rq.converged) rq.converged[col0 + j] = conv ? 1 : 0;
      pl->last_test2[(size_t)(col0 + j)] = t2;
      pl->last_rounds[(size_t)(col0 + j)] = rounds;
      pl->last_iters_raw[(size_t)(col0 + j)] = raw;
    }
    col0 += nc;
  }
  return 0;
}

}  // namespace fe
