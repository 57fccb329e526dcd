// fe_plan.cu -- plan construction: argument checks, work items, and the
// Jacobi preconditioner on the device (the integer plan is built in
// fe_build.cu).
//
// Replaces the solver constructor and update_weights! of the reference's CUDA
// backend (ext/CUDAExt.jl:99-121) and of the CPU backend
// (src/SolverCPU.jl:55-95).
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "fe_kernels.cuh"
#include "fe_plan.h"

namespace fe {

namespace {
// fixed-size per-thread message buffer: reporting an error allocates nothing
thread_local char g_err[1024];
}
void set_error(const std::string& msg) { set_error_cstr(msg.c_str()); }
void set_error_cstr(const char* msg) {
  size_t n = 0;
  for (; msg[n] && n + 1 < sizeof(g_err); ++n) g_err[n] = msg[n];
  g_err[n] = '\0';
}
const char* last_error() { return g_err; }

DevBuf::~DevBuf() {
  if (p) cudaFree(p);
}

int exchange(fe_plan* pl, void* buf, int64_t count, int elem_bytes, cudaStream_t s) {
  if (!pl->xchg || count <= 0) return 0;
  const int rc = pl->xchg(pl->xchg_ctx, buf, count, elem_bytes == 8 ? 0 : 1, (void*)s);
  if (rc != 0) {
    set_error("the exchange over ranks failed (callback status " + std::to_string(rc) + ")");
    return 2;  // FE_ERR_CUDA
  }
  return 0;
}
// Host-side fault injection for the allocation-failure path: with
// FE_B200_FAIL_ALLOC_BYTES=b in the environment, every device allocation of at
// least b bytes fails as an out-of-memory cudaMalloc would (FE_ERR_ALLOC and
// a message), without touching the GPU.  Read on every allocation, so a test
// can set and clear it between calls.
static bool injected_alloc_failure(size_t n) {
  const char* v = getenv("FE_B200_FAIL_ALLOC_BYTES");
  if (!v || !*v) return false;
  char* end = nullptr;
  const unsigned long long b = strtoull(v, &end, 10);
  return end != v && (unsigned long long)n >= b;
}

int DevBuf::ensure(size_t n) {
  if (n <= bytes && p) return 0;
  if (p) {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  if (n == 0) n = 16;
  if (injected_alloc_failure(n)) {
    set_error(std::string("cudaMalloc of ") + std::to_string(n) +
              " bytes failed: injected by FE_B200_FAIL_ALLOC_BYTES");
    return 3;  // FE_ERR_ALLOC
  }
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    set_error(std::string("cudaMalloc of ") + std::to_string(n) + " bytes failed: " +
              cudaGetErrorString(e));
    (void)cudaGetLastError();
    return 3;  // FE_ERR_ALLOC
  }
  bytes = n;
  return 0;
}

template <typename T>
static int upload(DevBuf& b, const T* src, size_t n, cudaStream_t s) {
  int st = b.ensure((n > 0 ? n : 1) * sizeof(T));
  if (st) return st;
  if (n > 0 && src) FE_CK(cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return 0;
}

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
__global__ void k_sqrt_w(const double* __restrict__ w, double* __restrict__ sw, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sw[i] = sqrt(w[i]);
}
__global__ void k_gather_d(const double* __restrict__ src, const int32_t* __restrict__ idx,
                           double* __restrict__ dst, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}
// cw = interaction * sqrt(w) in sorted observation order (the per-observation
// part of the reference's cache!, src/SolverCPU.jl:91-95).
__global__ void k_cw(const double* __restrict__ inter, const double* __restrict__ sw,
                     double* __restrict__ cw_d, float* __restrict__ cw_f, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double c = 1.0;
    if (inter) c = inter[i];
    if (sw) c *= sw[i];
    cw_d[i] = c;
    cw_f[i] = (float)c;
  }
}
__global__ void k_cwp(const double* __restrict__ cw_d, const int32_t* __restrict__ perm,
                      double* __restrict__ cwp_d, float* __restrict__ cwp_f, int64_t n) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) {
    const double c = cw_d[perm ? perm[q] : q];
    cwp_d[q] = c;
    cwp_f[q] = (float)c;
  }
}

static inline unsigned grid1(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// Column scales of the absorbed operator M A_r: 1 / ||M a_l|| for level l of
// a non-primary FE, where M projects out the primary FE's columns e_w:
//   ||M a_l||^2 = ||a_l||^2 - sum_w (e_w' a_l)^2 / ||e_w||^2,
// e_w' a_l = sum over the rows of level l in primary level w of cw_i cw_p,i,
// ||a_l||^2 = 1 / scale_l^2 and 1 / ||e_w||^2 = scale_p,w^2 (the Jacobi
// scales).  Level l's positions in level order are in sorted-row order, and
// sorted rows are grouped by primary level, so the rows of one (w, l) pair
// form a run of consecutive positions.  Levels are cut into pieces of at most
// kAbsPiece positions: one thread per piece sums its runs and reports its
// first and last run separately (they may continue in the neighbouring
// pieces); one thread per level then joins the pieces in order.  The order is
// fixed, so the result does not depend on scheduling.  The ratio
// ||M a_l||^2 / ||a_l||^2 is floored at 1e-4, so a column that the projection
// (almost) removes is amplified at most 100-fold; an empty column keeps 0.
constexpr int64_t kAbsPiece = 1024;
struct AbsPiece {
  int64_t q0, q1;   // positions in level order
  int32_t nruns;    // runs (distinct primary levels) in the piece
  int32_t w0, w1;   // primary level of the first and of the last run
  double s0, s1;    // sums of cw cw_p over the first and the last run
  double mid;       // runs in between: sum of s^2 / ||e_w||^2
};
__device__ __forceinline__ double abs_run(double s, int32_t w, const double* scp) {
  return s * s * scp[w] * scp[w];
}
__global__ void k_abs_pieces(AbsPiece* __restrict__ pc, int64_t n, const int32_t* __restrict__ perm,
                             const int32_t* __restrict__ refp, const double* __restrict__ cwk,
                             const double* __restrict__ cwp, const double* __restrict__ scp) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  AbsPiece a = pc[i];
  a.nruns = 0;
  a.w0 = a.w1 = -1;
  a.s0 = a.s1 = a.mid = 0.0;
  int32_t wc = -1;
  double s = 0.0;
  for (int64_t q = a.q0; q < a.q1; ++q) {
    const int64_t p = perm ? (int64_t)perm[q] : q;
    const int32_t w = refp[p];
    if (w != wc) {
      if (a.nruns == 1) {
        a.w0 = wc;
        a.s0 = s;
      } else if (a.nruns > 1) {
        a.mid += abs_run(s, wc, scp);
      }
      ++a.nruns;
      s = 0.0;
      wc = w;
    }
    s += (cwk ? cwk[p] : 1.0) * (cwp ? cwp[p] : 1.0);
  }
  if (a.nruns == 1) {
    a.w0 = wc;
    a.s0 = s;
  } else if (a.nruns > 1) {
    a.w1 = wc;
    a.s1 = s;
  }
  pc[i] = a;
}
// partial: write the sum of squared projections `tot` of each level (the
// share of this rank's primary levels; the ranks' shares are summed by the
// exchange of a sharded plan and k_abs_final finishes), else the scale.
__global__ void k_abs_join(const AbsPiece* __restrict__ pc, const int64_t* __restrict__ first,
                           int64_t nl, const double* __restrict__ scp,
                           const double* __restrict__ sck, double* __restrict__ out_d,
                           float* __restrict__ out_f, int partial) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nl) return;
  const double sk = sck[l];
  double res = 0.0;
  if (sk > 0.0) {
    double tot = 0.0, sc = 0.0;
    int32_t wc = -1;  // the open run
    for (int64_t i = first[l]; i < first[l + 1]; ++i) {
      const AbsPiece& a = pc[i];
      if (a.nruns == 0) continue;
      if (a.w0 == wc) {
        sc += a.s0;  // the open run continues
      } else {
        if (wc >= 0) tot += abs_run(sc, wc, scp);
        wc = a.w0;
        sc = a.s0;
      }
      if (a.nruns > 1) {  // the first run ends inside the piece
        tot += abs_run(sc, wc, scp) + a.mid;
        wc = a.w1;
        sc = a.s1;
      }
    }
    if (wc >= 0) tot += abs_run(sc, wc, scp);
    if (partial) {
      res = tot;
    } else {
      const double a2 = 1.0 / (sk * sk);
      res = 1.0 / sqrt(fmax(a2 - tot, 1e-4 * a2));
    }
  }
  out_d[l] = res;
  if (!partial) out_f[l] = (float)res;
}
// the scales 1 / ||M a_l|| from the exchanged sums `tot` (in out_d)
__global__ void k_abs_final(int64_t nl, const double* __restrict__ sck, double* __restrict__ out_d,
                            float* __restrict__ out_f) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nl) return;
  const double sk = sck[l];
  double res = 0.0;
  if (sk > 0.0) {
    const double a2 = 1.0 / (sk * sk);
    res = 1.0 / sqrt(fmax(a2 - out_d[l], 1e-4 * a2));
  }
  out_d[l] = res;
  out_f[l] = (float)res;
}

// ---------------------------------------------------------------------------
// the solver constructor
// ---------------------------------------------------------------------------
int plan_build(fe_plan* pl, int32_t nprob, const int64_t* n_obs, int32_t K,
               const int64_t* const* refs, const int64_t* n_levels,
               const double* const* interaction, const double* weights, int32_t device) {
  NvtxRange nv("fe: plan build");
  if (nprob < 1 || !n_obs) {
    set_error("plan: need at least one problem");
    return 1;
  }
  if (K < 1 || K > kMaxFE) {
    set_error("plan: number of fixed effects must be in 1.." + std::to_string(kMaxFE));
    return 1;
  }
  if (!refs || !n_levels) {
    set_error("plan: refs and n_levels are required");
    return 1;
  }
  pl->K = K;
  pl->nprob = nprob;
  pl->device = device;
  pl->prob_obs_off.assign((size_t)nprob + 1, 0);
  for (int p = 0; p < nprob; ++p) {
    if (n_obs[p] < 0) {
      set_error("plan: negative observation count");
      return 1;
    }
    pl->prob_obs_off[p + 1] = pl->prob_obs_off[p] + n_obs[p];
  }
  const int64_t N = pl->prob_obs_off[nprob];
  if (N >= (int64_t)INT32_MAX) {
    set_error("plan: more than 2^31-1 observations is not supported");
    return 1;
  }
  pl->N = N;
  for (int k = 0; k < K; ++k)
    if (N > 0 && !refs[k]) {
      set_error("plan: refs[" + std::to_string(k) + "] is null");
      return 1;
    }
  // per-problem level offsets and validation (refs are 1-based; 0 marks an FE
  // absent from a problem, which requires n_levels == 0 there)
  pl->prob_lev_off.assign((size_t)(nprob + 1) * K, 0);
  pl->prob_nfe.assign(nprob, 0);
  pl->nlev.assign(K, 0);
  for (int p = 0; p < nprob; ++p)
    for (int k = 0; k < K; ++k) {
      const int64_t nl = n_levels[(int64_t)p * K + k];
      if (nl < 0) {
        set_error("plan: negative level count");
        return 1;
      }
      pl->prob_lev_off[(size_t)(p + 1) * K + k] = pl->prob_lev_off[(size_t)p * K + k] + nl;
      if (nl > 0) pl->prob_nfe[p] += 1;
    }
  for (int k = 0; k < K; ++k) {
    pl->nlev[k] = pl->prob_lev_off[(size_t)nprob * K + k];
    if (pl->nlev[k] >= (int64_t)INT32_MAX - 1) {
      set_error("plan: too many levels");
      return 1;
    }
  }
  // primary FE: the one with the most levels (its observations become
  // contiguous, so its expand and reduce stream through memory)
  pl->primary = 0;
  for (int k = 1; k < K; ++k)
    if (pl->nlev[k] > pl->nlev[pl->primary]) pl->primary = k;
  pl->absorbable = K >= 2;
  if (nprob > 1)
    for (int p = 0; p < nprob && pl->absorbable; ++p)
      if (n_obs[p] > 0 && (n_levels[(int64_t)p * K + pl->primary] == 0 || pl->prob_nfe[p] < 2))
        pl->absorbable = false;

  FE_CK(cudaSetDevice(device));
  if (!pl->stream) {
    FE_CK(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking));
    pl->own_stream = true;
  }

  // level ids are validated on the device (plan_build_device)
  pl->lev_base.assign(K, 0);
  pl->P = 0;
  for (int k = 0; k < K; ++k) {
    pl->lev_base[k] = pl->P;
    pl->P += pl->nlev[k] + 1;
  }
  int st = plan_build_device(pl, refs, n_levels, interaction);
  if (st) return st;
  pl->d_scale_d.resize(K);
  pl->d_scale_f.resize(K);
  pl->d_cw_d.resize(K);
  pl->d_cw_f.resize(K);
  pl->d_cwp_d.resize(K);
  pl->d_cwp_f.resize(K);

  // device view
  FeDev& d = pl->dev;
  memset(&d, 0, sizeof(d));
  d.K = K;
  d.N = N;
  d.P = pl->P;
  for (int k = 0; k < K; ++k) {
    d.refs[k] = pl->d_refs[k].as<int32_t>();
    d.perm[k] = pl->perm_identity[k] ? nullptr : pl->d_perm[k].as<int32_t>();
    d.key[k] = pl->d_key[k].as<int32_t>();
    d.lev_base[k] = pl->lev_base[k];
  }
  d.primary = pl->primary;
  return plan_update_weights(pl, weights);
}

// update_weights!: src/SolverCPU.jl:67-76, ext/CUDAExt.jl:112-121.
int plan_update_weights(fe_plan* pl, const double* weights) {
  NvtxRange nv("fe: weights and preconditioner");
  const int64_t N = pl->N;
  const int K = pl->K;
  cudaStream_t s = pl->stream;
  FE_CK(cudaSetDevice(pl->device));
  // captured LSMR loops hold the kernel instantiations and the weight
  // pointers of the old weights (unit weights select other kernels): drop
  // them, the next solve captures again
  FE_CK(cudaStreamSynchronize(s));
  for (auto& g : pl->graphs)
    if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  pl->graphs.clear();
  pl->weighted = weights != nullptr;
  if (weights) {
    DevBuf w;
    int st = upload(w, weights, (size_t)N, s);
    if (!st) st = pl->d_sw_orig.ensure((size_t)std::max<int64_t>(N, 1) * 8);
    if (!st) st = pl->d_sw_sorted.ensure((size_t)std::max<int64_t>(N, 1) * 8);
    if (st) return st;
    if (N) {
      k_sqrt_w<<<grid1(N), 256, 0, s>>>(w.as<double>(), pl->d_sw_orig.as<double>(), N);
      k_gather_d<<<grid1(N), 256, 0, s>>>(pl->d_sw_orig.as<double>(), pl->d_obs_src.as<int32_t>(),
                                          pl->d_sw_sorted.as<double>(), N);
      FE_CK(cudaGetLastError());
    }
    FE_CK(cudaStreamSynchronize(s));
  }
  FeDev& d = pl->dev;
  for (int k = 0; k < K; ++k) {
    const int64_t nl = pl->nlev[k] + 1;
    int st = pl->d_scale_d[k].ensure((size_t)nl * 8);
    if (!st) st = pl->d_scale_f[k].ensure((size_t)nl * 4);
    if (st) return st;
    FE_CK(cudaMemsetAsync(pl->d_scale_d[k].p, 0, (size_t)nl * 8, s));
    FE_CK(cudaMemsetAsync(pl->d_scale_f[k].p, 0, (size_t)nl * 4, s));
    d.scale_d[k] = pl->d_scale_d[k].as<double>();
    d.scale_f[k] = pl->d_scale_f[k].as<float>();
    const bool has_cw = pl->weighted || pl->interacted[k];
    if (has_cw) {
      const int64_t np = std::max<int64_t>(pl->seg_len[k], 1);
      st = pl->d_cw_d[k].ensure((size_t)std::max<int64_t>(N, 1) * 8);
      if (!st) st = pl->d_cw_f[k].ensure((size_t)std::max<int64_t>(N, 1) * 4);
      if (!st) st = pl->d_cwp_d[k].ensure((size_t)np * 8);
      if (!st) st = pl->d_cwp_f[k].ensure((size_t)np * 4);
      if (st) return st;
      if (N) {
        k_cw<<<grid1(N), 256, 0, s>>>(pl->interacted[k] ? pl->d_inter_sorted[k].as<double>() : nullptr,
                                      pl->weighted ? pl->d_sw_sorted.as<double>() : nullptr,
                                      pl->d_cw_d[k].as<double>(), pl->d_cw_f[k].as<float>(), N);
        if (pl->seg_len[k])
          k_cwp<<<grid1(pl->seg_len[k]), 256, 0, s>>>(pl->d_cw_d[k].as<double>(), d.perm[k],
                                                       pl->d_cwp_d[k].as<double>(),
                                                       pl->d_cwp_f[k].as<float>(), pl->seg_len[k]);
        FE_CK(cudaGetLastError());
      }
      d.cw_d[k] = pl->d_cw_d[k].as<double>();
      d.cw_f[k] = pl->d_cw_f[k].as<float>();
      d.cwp_d[k] = pl->d_cwp_d[k].as<double>();
      d.cwp_f[k] = pl->d_cwp_f[k].as<float>();
    } else {
      d.cw_d[k] = nullptr;
      d.cw_f[k] = nullptr;
      d.cwp_d[k] = nullptr;
      d.cwp_f[k] = nullptr;
    }
  }
  // Jacobi scales as a deterministic segmented reduction (C = 1 items)
  ItemSet* its = nullptr;
  int st = plan_items(pl, 1, &its);
  if (st) return st;
  FeDev dd = d;
  dd.C = 1;
  DevBuf sums, piece, block;
  st = sums.ensure((size_t)std::max<int64_t>(pl->P, 1) * 8);
  if (!st) st = piece.ensure((size_t)std::max<int64_t>(its->n_pieces, 1) * 8);
  if (!st) st = block.ensure((size_t)std::max<int64_t>(its->n_blocks, 1) * 8);
  if (st) return st;
  FE_CK(cudaMemsetAsync(sums.p, 0, (size_t)std::max<int64_t>(pl->P, 1) * 8, s));
  if (!its->rd.empty()) {
    const unsigned grid = (unsigned)((its->rd.size() + kWarps - 1) / kWarps);
    SplitArgs sa{its->d_splits.as<SplitLevel>(), piece.as<double>(), its->n_pieces,
                 block.as<double>(), its->n_blocks, its->d_split_cnt.as<int32_t>(),
                 its->d_block_cnt.as<int32_t>()};
    k_segsum<double, 1, 8, false, LoadScaleSq><<<grid, kThreads, 0, s>>>(
        dd, its->d_rd.as<ReduceItem>(), (int64_t)its->rd.size(), LoadScaleSq{}, sums.as<double>(), sa);
    FE_CK(cudaGetLastError());
  }
  // sharded plan: the sums of w * interaction^2 over every rank's rows
  st = exchange(pl, sums.p, pl->P, 8, s);
  if (st) return st;
  if (!its->pu.empty()) {
    PEpiScale epi;
    for (int k = 0; k < kMaxFE; ++k) {
      epi.sd[k] = k < K ? pl->d_scale_d[k].as<double>() : nullptr;
      epi.sf[k] = k < K ? pl->d_scale_f[k].as<float>() : nullptr;
    }
    const unsigned grid = (unsigned)(its->pu.size() / kWarps);
    k_pupdate<1, 4, PEpiScale><<<grid, kThreads, 0, s>>>(dd, its->d_pu.as<PItem>(),
                                                           (int64_t)its->pu.size(), sums.as<double>(),
                                                           epi, nullptr, nullptr, 0);
    FE_CK(cudaGetLastError());
  }
  // the absorbed operator's column scales (plans whose primary FE can be
  // projected out; a batch's levels belong to one problem each)
  pl->d_abs_scale_d.resize(K);
  pl->d_abs_scale_f.resize(K);
  if (pl->absorbable && N > 0) {
    const int kp = pl->primary;
    DevBuf pcs, first;
    std::vector<AbsPiece> hp;
    std::vector<int64_t> hf;
    for (int k = 0; k < K; ++k) {
      if (k == kp) continue;
      const int64_t nl = pl->nlev[k];
      const std::vector<int64_t>& so = pl->seg_off[k];
      hp.clear();
      hf.assign((size_t)nl + 1, 0);
      for (int64_t l = 0; l < nl; ++l) {
        hf[(size_t)l] = (int64_t)hp.size();
        for (int64_t q = so[(size_t)l]; q < so[(size_t)l + 1]; q += kAbsPiece) {
          AbsPiece a{};
          a.q0 = q;
          a.q1 = std::min(q + kAbsPiece, so[(size_t)l + 1]);
          hp.push_back(a);
        }
      }
      hf[(size_t)nl] = (int64_t)hp.size();
      st = pl->d_abs_scale_d[k].ensure((size_t)(nl + 1) * 8);
      if (!st) st = pl->d_abs_scale_f[k].ensure((size_t)(nl + 1) * 4);
      if (!st) st = upload(pcs, hp.data(), hp.size(), s);
      if (!st) st = upload(first, hf.data(), hf.size(), s);
      if (st) return st;
      FE_CK(cudaMemsetAsync(pl->d_abs_scale_d[k].p, 0, (size_t)(nl + 1) * 8, s));
      FE_CK(cudaMemsetAsync(pl->d_abs_scale_f[k].p, 0, (size_t)(nl + 1) * 4, s));
      if (!hp.empty()) {
        k_abs_pieces<<<grid1((int64_t)hp.size(), 128), 128, 0, s>>>(
            pcs.as<AbsPiece>(), (int64_t)hp.size(), d.perm[k], d.refs[kp], d.cw_d[k], d.cw_d[kp],
            d.scale_d[kp]);
        FE_CK(cudaGetLastError());
      }
      if (nl > 0) {
        const int partial = pl->xchg ? 1 : 0;
        k_abs_join<<<grid1(nl, 128), 128, 0, s>>>(
            pcs.as<AbsPiece>(), first.as<int64_t>(), nl, d.scale_d[kp], d.scale_d[k],
            pl->d_abs_scale_d[k].as<double>(), pl->d_abs_scale_f[k].as<float>(), partial);
        FE_CK(cudaGetLastError());
        if (partial) {
          // sharded plan: sum the ranks' shares, then finish the scales
          st = exchange(pl, pl->d_abs_scale_d[k].p, nl, 8, s);
          if (st) return st;
          k_abs_final<<<grid1(nl, 128), 128, 0, s>>>(nl, d.scale_d[k],
                                                      pl->d_abs_scale_d[k].as<double>(),
                                                      pl->d_abs_scale_f[k].as<float>());
          FE_CK(cudaGetLastError());
        }
      }
      FE_CK(cudaStreamSynchronize(s));  // the host piece lists are reused
    }
  }
  FE_CK(cudaStreamSynchronize(s));
  return 0;
}

// ---------------------------------------------------------------------------
// work items for a column tile width C
// ---------------------------------------------------------------------------
static int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

int plan_items(fe_plan* pl, int C, ItemSet** out) {
  auto itf = pl->items.find(C);
  if (itf != pl->items.end()) {
    *out = itf->second.get();
    return 0;
  }
  std::unique_ptr<ItemSet> its(new ItemSet());
  its->C = C;
  int sms = 148;
  {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, pl->device) == cudaSuccess && v > 0)
      sms = v;
  }
  // about 4 waves of resident warps; rows per item a multiple of 32
  const int64_t warps_target = (int64_t)sms * 64 * 4;
  const int64_t cap = std::max<int64_t>(32, 16384 / C);
  auto item_size = [&](int64_t total) {
    return std::min(cap, std::max<int64_t>(32, round_up((total + warps_target - 1) / warps_target, 32)));
  };
  const int64_t Te = item_size(pl->N);
  int64_t total_pos = 0;
  for (int k = 0; k < pl->K; ++k) total_pos += pl->seg_len[k];
  const int64_t Tr = item_size(total_pos);
  int64_t total_rows = 0;
  for (int k = 0; k < pl->K; ++k) total_rows += pl->nlev[k];
  const int64_t Tp = item_size(total_rows);
  // the non-primary FEs' levels alone (the absorbed loop's P side) are sized
  // on their own count, so that their items fill the GPU in whole waves
  const int64_t Tp_np = item_size(total_rows - (pl->absorbable ? pl->nlev[pl->primary] : 0));

  const int nprob = pl->nprob;
  const int K = pl->K;
  its->ex_slot_off.assign((size_t)nprob + 1, 0);
  its->pu_slot_off.assign((size_t)nprob + 1, 0);
  its->pu_abs_slot_off.assign(1, 0);
  std::vector<ReduceItem> rd_prim, rd_small;
  const int kp = pl->primary;
  its->sms = sms;
  // small FEs (32-column tiles of single-problem plans): the non-primary FEs
  // with the fewest levels whose tables (levels + null level) fit kSmallRows
  if (C == 32 && pl->nprob == 1) {
    std::vector<int> order;
    for (int k = 0; k < pl->K; ++k)
      if (k != pl->primary) order.push_back(k);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return pl->nlev[a] < pl->nlev[b]; });
    int nsmall = 0;
    for (int k : order) {
      const int64_t rows = pl->nlev[k] + 1;
      if (its->small_rows + rows > kSmallRows || nsmall == kRowSumSmallFE) break;
      ++nsmall;
      its->small_mask |= 1u << k;
      its->small_off[k] = its->small_rows;
      for (int64_t l = 0; l < rows; ++l) its->small_slab_row.push_back(pl->lev_base[k] + l);
      its->small_rows += (int32_t)rows;
    }
  }
  for (int p = 0; p < nprob; ++p) {
    // expand items: whole primary levels of the problem's sorted range packed
    // up to Te observations (a longer level is cut into pieces), padded so
    // that every CTA belongs to one problem (its norm slot is per problem)
    const int64_t o0 = pl->prob_obs_off[p], o1 = pl->prob_obs_off[p + 1];
    const size_t e0 = its->ex.size();
    const int64_t plb = pl->prob_lev_off[(size_t)p * K + kp];
    const int64_t ple = pl->prob_lev_off[(size_t)(p + 1) * K + kp];
    if (ple == plb) {
      for (int64_t b = o0; b < o1; b += Te) its->ex.push_back({b, std::min(o1, b + Te), p, -1, 0, 0});
    } else {
      const std::vector<int64_t>& off = pl->seg_off[kp];
      const int64_t base = o0 - off[(size_t)plb];  // sorted position of level-order position
      int64_t cur_b = -1, cur_e = -1;
      for (int64_t l = plb; l < ple; ++l) {
        const int64_t b = off[(size_t)l] + base, e = off[(size_t)l + 1] + base, cnt = e - b;
        if (cnt == 0) continue;
        if (cnt > Te) {
          if (cur_b >= 0) {
            its->ex.push_back({cur_b, cur_e, p, -1, 0, 0});
            cur_b = -1;
          }
          const int64_t npieces = (cnt + Te - 1) / Te;
          const int64_t psz = (cnt + npieces - 1) / npieces;
          SplitLevel sl;
          sl.first_piece = (int32_t)its->ex_n_pieces;
          sl.npieces = (int32_t)npieces;
          sl.fe = kp;
          sl.level = (int32_t)l;
          sl.nblocks = (int32_t)((npieces + kSplitBlock - 1) / kSplitBlock);
          sl.first_block = (int32_t)its->ex_n_blocks;
          its->ex_n_blocks += sl.nblocks;
          const int32_t sid = (int32_t)its->ex_splits.size();
          its->ex_splits.push_back(sl);
          for (int64_t q = 0; q < npieces; ++q) {
            const int64_t pb = b + q * psz, pe = std::min(e, pb + psz);
            its->ex.push_back({pb, pe, p, sid, (int32_t)q, 0});
          }
          its->ex_n_pieces += npieces;
          continue;
        }
        if (cur_b < 0) cur_b = b;
        cur_e = e;
        if (cur_e - cur_b >= Te) {
          its->ex.push_back({cur_b, cur_e, p, -1, 0, 0});
          cur_b = -1;
        }
      }
      if (cur_b >= 0) its->ex.push_back({cur_b, cur_e, p, -1, 0, 0});
    }
    while ((its->ex.size() - e0) % kWarps) its->ex.push_back({o1, o1, p, -1, 0, 0});
    if (its->ex.size() == e0)
      for (int w = 0; w < kWarps; ++w) its->ex.push_back({o1, o1, p, -1, 0, 0});
    its->ex_slot_off[p + 1] = (int64_t)(its->ex.size() / kWarps);
    // P-side items: chunks of the problem's slab rows, per FE, padded likewise.
    // Single-problem plans list the non-primary FEs first, padded on their
    // own, so that the absorbed-primary mode can run just that prefix.
    const size_t q0 = its->pu.size();
    auto pu_fe = [&](int k, int64_t T) {
      const int64_t rb = pl->lev_base[k] + pl->prob_lev_off[(size_t)p * K + k];
      const int64_t re = pl->lev_base[k] + pl->prob_lev_off[(size_t)(p + 1) * K + k];
      for (int64_t b = rb; b < re; b += T) its->pu.push_back({b, std::min(re, b + T), k, p});
    };
    if (nprob == 1) {
      for (int k = 0; k < K; ++k)
        if (k != kp) pu_fe(k, Tp_np);
      while ((its->pu.size() - q0) % kWarps) its->pu.push_back({0, 0, 0, p});
      if (its->pu.size() == q0)
        for (int w = 0; w < kWarps; ++w) its->pu.push_back({0, 0, 0, p});
      its->pu_np = (int64_t)its->pu.size();
      pu_fe(kp, Tp);
    } else {
      for (int k = 0; k < K; ++k) pu_fe(k, Tp);
      if (pl->absorbable && C < 32) {
        // the absorbed loop's P side: the problem's non-primary levels
        const size_t a0 = its->pu_abs.size();
        for (int k = 0; k < K; ++k) {
          if (k == kp) continue;
          const int64_t rb = pl->lev_base[k] + pl->prob_lev_off[(size_t)p * K + k];
          const int64_t re = pl->lev_base[k] + pl->prob_lev_off[(size_t)(p + 1) * K + k];
          for (int64_t b = rb; b < re; b += Tp_np) its->pu_abs.push_back({b, std::min(re, b + Tp_np), k, p});
        }
        while ((its->pu_abs.size() - a0) % kWarps) its->pu_abs.push_back({0, 0, 0, p});
        if (its->pu_abs.size() == a0)
          for (int w = 0; w < kWarps; ++w) its->pu_abs.push_back({0, 0, 0, p});
        its->pu_abs_slot_off.push_back((int64_t)(its->pu_abs.size() / kWarps));
      }
    }
    while ((its->pu.size() - q0) % kWarps) its->pu.push_back({0, 0, 0, p});
    if (its->pu.size() == q0)
      for (int w = 0; w < kWarps; ++w) its->pu.push_back({0, 0, 0, p});
    its->pu_slot_off[p + 1] = (int64_t)(its->pu.size() / kWarps);
    // segmented-sum items: whole levels packed up to Tr positions; a longer
    // level is cut into pieces.  Items of the primary FE go to a second list
    // (appended after all others): the fused expand reduces that FE itself.
    for (int k = 0; k < K; ++k) {
      std::vector<ReduceItem>& dst =
          (k == kp) ? rd_prim : (((its->small_mask >> k) & 1u) ? rd_small : its->rd);
      const int64_t lb = pl->prob_lev_off[(size_t)p * K + k];
      const int64_t le = pl->prob_lev_off[(size_t)(p + 1) * K + k];
      if (le == lb) continue;
      const std::vector<int64_t>& off = pl->seg_off[k];
      int64_t cur_b = -1, cur_e = -1;
      for (int64_t l = lb; l < le; ++l) {
        const int64_t b = off[(size_t)l], e = off[(size_t)l + 1], cnt = e - b;
        if (cnt == 0) continue;
        if (cnt > Tr) {
          if (cur_b >= 0) {
            dst.push_back({cur_b, cur_e, k, p, -1, 0});
            cur_b = -1;
          }
          const int64_t npieces = (cnt + Tr - 1) / Tr;
          const int64_t psz = (cnt + npieces - 1) / npieces;
          SplitLevel sl;
          sl.first_piece = (int32_t)its->n_pieces;
          sl.npieces = (int32_t)npieces;
          sl.fe = k;
          sl.level = (int32_t)l;
          sl.nblocks = (int32_t)((npieces + kSplitBlock - 1) / kSplitBlock);
          sl.first_block = (int32_t)its->n_blocks;
          its->n_blocks += sl.nblocks;
          const int32_t sid = (int32_t)its->splits.size();
          its->splits.push_back(sl);
          for (int64_t q = 0; q < npieces; ++q) {
            const int64_t pb = b + q * psz, pe = std::min(e, pb + psz);
            dst.push_back({pb, pe, k, p, sid, (int32_t)q});
          }
          its->n_pieces += npieces;
          continue;
        }
        if (cur_b < 0) cur_b = b;
        cur_e = e;
        if (cur_e - cur_b >= Tr) {
          dst.push_back({cur_b, cur_e, k, p, -1, 0});
          cur_b = -1;
        }
      }
      if (cur_b >= 0) dst.push_back({cur_b, cur_e, k, p, -1, 0});
    }
  }
  // demean items (absorbed-primary mode: one problem, 2+ FEs): whole primary
  // levels packed up to kDemeanRows rows; a longer level is one item of its
  // own (the pass walks each item twice, so short items keep the second read
  // in cache)
  if (nprob == 1 && K >= 2) {
    const std::vector<int64_t>& off = pl->seg_off[kp];
    const int64_t nl = pl->nlev[kp];
    int64_t cur_b = -1, cur_e = -1;
    for (int64_t l = 0; l < nl; ++l) {
      const int64_t b = off[(size_t)l], e = off[(size_t)l + 1];
      if (e == b) continue;
      if (cur_b >= 0 && e - cur_b > kDemeanRows) {
        its->dm.push_back({cur_b, cur_e, 0, -1, 0, 0});
        cur_b = -1;
      }
      if (cur_b < 0) cur_b = b;
      cur_e = e;
    }
    if (cur_b >= 0) its->dm.push_back({cur_b, cur_e, 0, -1, 0, 0});
  } else if (pl->absorbable && C < 32) {
    // batch plans: each problem's primary levels (its rows are one contiguous
    // range, in level order) packed alike, padded to whole CTAs of kDemeanIpc
    // items, so that each CTA's norm slot belongs to one problem
    its->dm_ipc = kDemeanIpc;
    its->dm_slot_off.assign((size_t)nprob + 1, 0);
    const std::vector<int64_t>& off = pl->seg_off[kp];
    for (int p = 0; p < nprob; ++p) {
      const size_t d0 = its->dm.size();
      const int64_t o0 = pl->prob_obs_off[p], o1 = pl->prob_obs_off[p + 1];
      const int64_t plb = pl->prob_lev_off[(size_t)p * K + kp];
      const int64_t ple = pl->prob_lev_off[(size_t)(p + 1) * K + kp];
      if (o1 > o0 && ple > plb) {
        const int64_t base = o0 - off[(size_t)plb];  // sorted row of level-order position
        int64_t cur_b = -1, cur_e = -1;
        for (int64_t l = plb; l < ple; ++l) {
          const int64_t b = off[(size_t)l] + base, e = off[(size_t)l + 1] + base;
          if (e == b) continue;
          if (cur_b >= 0 && e - cur_b > kDemeanRows) {
            its->dm.push_back({cur_b, cur_e, p, -1, 0, 0});
            cur_b = -1;
          }
          if (cur_b < 0) cur_b = b;
          cur_e = e;
        }
        if (cur_b >= 0) its->dm.push_back({cur_b, cur_e, p, -1, 0, 0});
      }
      while ((its->dm.size() - d0) % kDemeanIpc) its->dm.push_back({o1, o1, p, -1, 0, 0});
      if (its->dm.size() == d0)
        for (int64_t q = 0; q < kDemeanIpc; ++q) its->dm.push_back({o1, o1, p, -1, 0, 0});
      its->dm_slot_off[(size_t)p + 1] = (int64_t)(its->dm.size() / kDemeanIpc);
    }
    its->Sdm = its->dm_slot_off[(size_t)nprob];
  }
  its->rd_large = (int64_t)its->rd.size();
  its->rd.insert(its->rd.end(), rd_small.begin(), rd_small.end());
  its->rd_np = (int64_t)its->rd.size();
  its->rd.insert(its->rd.end(), rd_prim.begin(), rd_prim.end());
  for (int p = 0; p < nprob; ++p) {
    its->ex_slot_off[p + 1] = std::max(its->ex_slot_off[p + 1], its->ex_slot_off[p]);
    its->pu_slot_off[p + 1] = std::max(its->pu_slot_off[p + 1], its->pu_slot_off[p]);
  }
  its->Se = its->ex_slot_off[nprob];
  its->Sp = its->pu_slot_off[nprob];

  cudaStream_t s = pl->stream;
  int st = upload(its->d_ex, its->ex.data(), its->ex.size(), s);
  if (!st) st = upload(its->d_rd, its->rd.data(), its->rd.size(), s);
  if (!st) st = upload(its->d_splits, its->splits.data(), its->splits.size(), s);
  if (!st) st = upload(its->d_pu, its->pu.data(), its->pu.size(), s);
  if (!st) st = upload(its->d_ex_off, its->ex_slot_off.data(), its->ex_slot_off.size(), s);
  if (!st) st = upload(its->d_pu_off, its->pu_slot_off.data(), its->pu_slot_off.size(), s);
  if (its->dm_ipc == 0) {
    // single problem: the absorbed loop's P side is the leading items
    its->Sp_np = its->pu_np / kWarps;
    const int64_t off_np[2] = {0, its->Sp_np};
    if (!st) st = upload(its->d_pu_off_np, off_np, 2, s);
  } else {
    // batch plans: its own list, per-problem P-side and demean slots
    its->pu_np = (int64_t)its->pu_abs.size();
    its->Sp_np = its->pu_np / kWarps;
    if (!st) st = upload(its->d_pu_abs, its->pu_abs.data(), its->pu_abs.size(), s);
    if (!st) st = upload(its->d_pu_off_np, its->pu_abs_slot_off.data(), its->pu_abs_slot_off.size(), s);
    if (!st) st = upload(its->d_dm_off, its->dm_slot_off.data(), its->dm_slot_off.size(), s);
  }
  if (!st) st = upload(its->d_dm, its->dm.data(), its->dm.size(), s);
  if (!st) st = upload(its->d_ex_splits, its->ex_splits.data(), its->ex_splits.size(), s);
  const size_t nsc = std::max<size_t>(its->splits.size(), 1) * 4;
  const size_t nesc = std::max<size_t>(its->ex_splits.size(), 1) * 4;
  const size_t nbc = (size_t)std::max<int64_t>(its->n_blocks, 1) * 4;
  const size_t nebc = (size_t)std::max<int64_t>(its->ex_n_blocks, 1) * 4;
  if (!st) st = its->d_split_cnt.ensure(nsc);
  if (!st) st = its->d_ex_split_cnt.ensure(nesc);
  if (!st) st = its->d_block_cnt.ensure(nbc);
  if (!st) st = its->d_ex_block_cnt.ensure(nebc);
  if (st) return st;
  FE_CK(cudaMemsetAsync(its->d_split_cnt.p, 0, nsc, s));
  FE_CK(cudaMemsetAsync(its->d_ex_split_cnt.p, 0, nesc, s));
  FE_CK(cudaMemsetAsync(its->d_block_cnt.p, 0, nbc, s));
  FE_CK(cudaMemsetAsync(its->d_ex_block_cnt.p, 0, nebc, s));
  FE_CK(cudaStreamSynchronize(s));
  *out = its.get();
  pl->items[C] = std::move(its);
  return 0;
}

int plan_destroy(fe_plan* pl) {
  if (!pl) return 0;
  cudaSetDevice(pl->device);
  if (pl->stream) cudaStreamSynchronize(pl->stream);
  for (auto& e : pl->prof.pool) cudaEventDestroy(e);
  for (auto& pr : pl->prof.pending) {
    cudaEventDestroy(pr.second.first);
    cudaEventDestroy(pr.second.second);
  }
  if (pl->host_pinned) cudaFreeHost(pl->host_pinned);
  if (pl->noalloc_order) cudaEventDestroy(pl->noalloc_order);
  if (pl->ring_up) cudaFreeHost(pl->ring_up);
  if (pl->ring_down) cudaFreeHost(pl->ring_down);
  for (auto& g : pl->graphs)
    if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  cudaStream_t s = pl->stream;
  bool own = pl->own_stream;
  delete pl;
  if (own && s) cudaStreamDestroy(s);
  return 0;
}

}  // namespace fe
