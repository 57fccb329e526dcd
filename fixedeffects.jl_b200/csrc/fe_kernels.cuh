// fe_kernels.cuh -- sm_100a kernels of the fixed-effects LSMR hot path.
//
// Every kernel here is HBM-bound integer-indexed gather/segmented-reduction
// work; nothing is a dense contraction, so there are no tensor-core paths.
//
// Layout: a column tile of C right-hand sides is stored observation-major
// ([N][C], one row per observation) and level-major ([P][C]) on the
// coefficient side, so one warp-wide access touches C contiguous values of a
// row.  A warp is split into G = 32/C groups of C lanes: group g handles one
// observation (or one level-order position) at a time and lane j of the group
// handles column j.
//
// Determinism: no floating-point atomics anywhere.  The reduce (A'u, the
// reference's gather!, src/SolverCPU.jl:21-27) is a segmented reduction over
// a once-computed stable level order; each work item is summed by one warp in
// a fixed order, long levels are cut into pieces whose partials are summed in
// piece order by the last piece to finish, and norms are reduced per CTA into
// fixed slots that a scalar kernel sums in slot order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fe_internal.h"

namespace fe {

#define FE_FULL 0xffffffffu

template <typename T> __device__ __forceinline__ const T* scale_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* scale_of<float>(const FeDev& d, int k) { return d.scale_f[k]; }
template <> __device__ __forceinline__ const double* scale_of<double>(const FeDev& d, int k) { return d.scale_d[k]; }
template <typename T> __device__ __forceinline__ const T* cw_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* cw_of<float>(const FeDev& d, int k) { return d.cw_f[k]; }
template <> __device__ __forceinline__ const double* cw_of<double>(const FeDev& d, int k) { return d.cw_d[k]; }
template <typename T> __device__ __forceinline__ const T* cwp_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* cwp_of<float>(const FeDev& d, int k) { return d.cwp_f[k]; }
template <> __device__ __forceinline__ const double* cwp_of<double>(const FeDev& d, int k) { return d.cwp_d[k]; }

// Norm accumulators of the warps of one CTA -> one slot per CTA (fixed order).
template <int C>
__device__ __forceinline__ void cta_norm_to_slot(double na, double* __restrict__ part,
                                                 int64_t S, int64_t slot, double (*sm)[32]) {
#pragma unroll
  for (int o = C; o < 32; o <<= 1) na += __shfl_xor_sync(FE_FULL, na, o);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane < C) sm[wib][lane] = na;
  __syncthreads();
  if (threadIdx.x < C && part != nullptr && slot >= 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) t += sm[w][threadIdx.x];
    part[(int64_t)threadIdx.x * S + slot] = t;
  }
}

// ---------------------------------------------------------------------------
// Coefficient tables gathered by the expand.
// ---------------------------------------------------------------------------
template <typename T, typename TA>
struct TabOne {
  const T* __restrict__ tab;
  __device__ __forceinline__ TA load(int64_t off) const { return (TA)__ldg(tab + off); }
};
// x64 + x32: the FP64 accumulated solution plus the FP32 correction of the
// inner solve that just finished (the mixed-precision residual).
struct TabSum64 {
  const double* __restrict__ hi;
  const float* __restrict__ lo;
  __device__ __forceinline__ double load(int64_t off) const {
    return __ldg(hi + off) + (double)__ldg(lo + off);
  }
};

// ---------------------------------------------------------------------------
// Expand epilogues: given s = (A x)[i, j] for observation i, column j.
// ---------------------------------------------------------------------------
// LSMR u-update: U <- av * (A v) + au * U   (src/utils/lsmr.jl:104 with the
// normalisations of u and v folded into av, au).
template <typename T>
struct EpiExpandLsmr {
  T* __restrict__ U;
  const Inst* __restrict__ inst;
  T av, au;
  bool act;
  __device__ __forceinline__ void begin(int prob, int j, int C) {
    const Inst& s = inst[(int64_t)prob * C + j];
    act = s.active != 0;
    av = (T)s.ex_av;
    au = (T)s.ex_au;
  }
  __device__ __forceinline__ double apply(int64_t i, int j, int C, T s) {
    T* p = U + i * C + j;
    const T u = av * s + au * (*p);
    *p = u;
    return (double)u * (double)u;
  }
};

// out <- B - (A x): initial u of LSMR and the final residual
// (src/utils/lsmr.jl:63, src/AbstractFixedEffectSolver.jl:62).  mask: 0 all
// instances, 2 only instances whose refinement is still running.
template <typename TOut, typename TA>
struct EpiBminusAx {
  const double* __restrict__ B;
  TOut* __restrict__ out;
  float* __restrict__ out32;  // optional FP32 copy (mixed-precision u)
  const Inst* __restrict__ inst;
  int mask;
  bool act;
  __device__ __forceinline__ void begin(int prob, int j, int C) {
    act = true;
    if (mask == 2) act = inst[(int64_t)prob * C + j].outer_active != 0;
  }
  __device__ __forceinline__ double apply(int64_t i, int j, int C, TA s) {
    const int64_t o = i * C + j;
    const double r = __ldg(B + o) - (double)s;
    out[o] = (TOut)r;
    if (out32) out32[o] = (float)r;
    return r * r;
  }
};

// ---------------------------------------------------------------------------
// expand kernel: one warp per ExpandItem (a range of sorted observations).
// ---------------------------------------------------------------------------
template <typename TA, int C, int U, class Tab, class Epi>
__global__ void __launch_bounds__(kThreads)
k_expand(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items, Tab tab, Epi epi,
         double* __restrict__ part, int64_t S) {
  constexpr int G = 32 / C;
  __shared__ double sm[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int g = lane / C, j = lane - g * C;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  double nrm = 0.0;
  if (w < n_items) {
    const ExpandItem it = items[w];
    epi.begin(it.prob, j, C);
    const bool any = __any_sync(FE_FULL, epi.act);
    if (any) {
      for (int64_t base = it.ib; base < it.ie; base += (int64_t)G * U) {
        TA s[U];
        int64_t ii[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          ii[u] = base + u * G + g;
          s[u] = TA(0);
        }
#pragma unroll
        for (int k = 0; k < kMaxFE; ++k) {
          if (k >= d.K) break;
          const int32_t* __restrict__ refs = d.refs[k];
          const TA* __restrict__ sc = scale_of<TA>(d, k);
          const TA* __restrict__ cw = cw_of<TA>(d, k);
          const int64_t lb = d.lev_base[k];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (ii[u] < it.ie && epi.act) {
              const int r = __ldg(refs + ii[u]);
              TA c = __ldg(sc + r);
              if (cw) c *= __ldg(cw + ii[u]);
              s[u] += c * tab.load((lb + r) * C + j);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ii[u] < it.ie && epi.act) nrm += epi.apply(ii[u], j, C, s[u]);
      }
    }
  }
  cta_norm_to_slot<C>(nrm, part, S, (int64_t)blockIdx.x, sm);
}

// ---------------------------------------------------------------------------
// Reduce value loaders: the per-position term summed into a level.
// ---------------------------------------------------------------------------
template <typename TIn, typename TA>
struct LoadIn {
  const TIn* __restrict__ in;
  __device__ __forceinline__ TA load(int64_t p, int64_t i, int j, int C,
                                     const TA* __restrict__ cwp) const {
    const TA v = (TA)in[i * C + j];
    return cwp ? __ldg(cwp + p) * v : v;
  }
};
// sum of interaction^2 * w for the Jacobi scale (src/SolverCPU.jl:78-89)
struct LoadScaleSq {
  __device__ __forceinline__ double load(int64_t p, int64_t, int, int,
                                         const double* __restrict__ cwp) const {
    if (cwp) {
      const double c = __ldg(cwp + p);
      return c * c;
    }
    return 1.0;
  }
};

// ---------------------------------------------------------------------------
// Reduce epilogues: finalize(level l of FE k, column j, acc = sum over level).
// ---------------------------------------------------------------------------
// LSMR v-update fused with the deferred h/hbar/x update of the previous
// iteration (src/utils/lsmr.jl:108-110 and :138-142) and the norms ||v||^2,
// ||x||^2.
template <typename T>
struct EpiReduceLsmr {
  T* __restrict__ V;
  T* __restrict__ H;
  T* __restrict__ Hb;
  T* __restrict__ X;
  const Inst* __restrict__ inst;
  double rd_acc, rd_v, s_v, c1, c2, c3;
  int upd_mode;
  bool do_v, act;
  __device__ __forceinline__ void begin(int prob, int j, int C) {
    const Inst& s = inst[(int64_t)prob * C + j];
    act = s.active != 0;
    rd_acc = s.rd_acc;
    rd_v = s.rd_v;
    s_v = s.s_v;
    c1 = s.c1;
    c2 = s.c2;
    c3 = s.c3;
    upd_mode = s.upd_mode;
    do_v = s.do_v != 0;
  }
  __device__ __forceinline__ void finalize(const FeDev& d, int k, int l, int j, int C, double acc,
                                           double& na, double& nb) {
    if (!act) return;
    const int64_t idx = (d.lev_base[k] + l) * C + j;
    const double vold = (double)V[idx];
    if (upd_mode != 0) {
      const double vo = s_v * vold;
      double x;
      if (upd_mode == 2) {
        const double h = (double)H[idx];
        const double hb = h + c1 * (double)Hb[idx];
        x = (double)X[idx] + c2 * hb;
        Hb[idx] = (T)hb;
        X[idx] = (T)x;
        H[idx] = (T)(vo + c3 * h);
      } else {
        H[idx] = (T)vo;
        Hb[idx] = (T)0;
        if (upd_mode == 3) {
          X[idx] = (T)0;
          x = 0.0;
        } else {
          x = (double)X[idx];
        }
      }
      const double xr = (double)(T)x;
      nb += xr * xr;
    }
    if (do_v) {
      const double sc = (double)__ldg(scale_of<T>(d, k) + l);
      const T vn = (T)(acc * sc * rd_acc - rd_v * vold);
      V[idx] = vn;
      na += (double)vn * (double)vn;
    }
  }
};

// x <- A'b (the warm start of src/AbstractFixedEffectSolver.jl:56).
template <typename TOut>
struct EpiStoreX {
  TOut* __restrict__ X;
  bool act;
  __device__ __forceinline__ void begin(int, int, int) { act = true; }
  __device__ __forceinline__ void finalize(const FeDev& d, int k, int l, int j, int C, double acc,
                                           double&, double&) {
    const int64_t idx = (d.lev_base[k] + l) * C + j;
    X[idx] = (TOut)(acc * __ldg(d.scale_d[k] + l));
  }
};

// Mixed precision: g = A'r computed in FP64 from the FP64 residual, stored as
// the FP32 starting v of the next inner solve; x64 += x32 and ||x64||^2.
struct EpiGrad64 {
  float* __restrict__ V32;
  double* __restrict__ X64;
  const float* __restrict__ X32;
  const Inst* __restrict__ inst;
  bool act;
  __device__ __forceinline__ void begin(int prob, int j, int C) {
    act = inst[(int64_t)prob * C + j].outer_active != 0;
  }
  __device__ __forceinline__ void finalize(const FeDev& d, int k, int l, int j, int C, double acc,
                                           double& na, double& nb) {
    if (!act) return;
    const int64_t idx = (d.lev_base[k] + l) * C + j;
    const double g = acc * __ldg(d.scale_d[k] + l);
    V32[idx] = (float)g;
    na += g * g;
    const double x = X64[idx] + (double)X32[idx];
    X64[idx] = x;
    nb += x * x;
  }
};

// Jacobi scale: 1/sqrt(sum interaction^2 w), or 0 for an empty sum
// (src/SolverCPU.jl:84-88, issue #97 of the reference).
struct EpiScale {
  double* sd[kMaxFE];
  float* sf[kMaxFE];
  bool act;
  __device__ __forceinline__ void begin(int, int, int) { act = true; }
  __device__ __forceinline__ void finalize(const FeDev&, int k, int l, int, int, double acc,
                                           double&, double&) {
    const double s = acc > 0 ? 1.0 / sqrt(acc) : 0.0;
    sd[k][l] = s;
    sf[k][l] = (float)s;
  }
};

// ---------------------------------------------------------------------------
// reduce kernel: one warp per ReduceItem.  Positions are visited in level
// order in batches of G (one per lane group); an inclusive segmented scan over
// the groups (keys are sorted inside an item, so equal keys are contiguous)
// plus a carry across batches yields each level's sum; the group holding a
// level's last position finalizes it.
// ---------------------------------------------------------------------------
template <typename TA, int C, int U, class Load, class Epi>
__global__ void __launch_bounds__(kThreads)
k_reduce(const FeDev d, const ReduceItem* __restrict__ items, int64_t n_items, Load ld, Epi epi,
         const SplitLevel* __restrict__ splits, double* __restrict__ piece_part,
         int32_t* __restrict__ split_cnt, double* __restrict__ part_a, double* __restrict__ part_b,
         int64_t S, const int32_t* __restrict__ cta_slot) {
  constexpr int G = 32 / C;
  __shared__ double sm[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int g = lane / C, j = lane - g * C;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  double na = 0.0, nb = 0.0;
  if (w < n_items) {
    const ReduceItem it = items[w];
    epi.begin(it.prob, j, C);
    const bool any = __any_sync(FE_FULL, epi.act);
    if (any && it.pe > it.pb) {
      const int k = it.fe;
      const int32_t* __restrict__ perm = d.perm[k];
      const int32_t* __restrict__ key = d.key[k];
      const TA* __restrict__ cwp = cwp_of<TA>(d, k);
      int ckey = -1;
      TA carry = TA(0);
      for (int64_t base = it.pb; base < it.pe; base += (int64_t)G * U) {
        int kk[U];
        TA val[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t p = base + u * G + g;
          if (p < it.pe) {
            kk[u] = __ldg(key + p);
            const int64_t i = perm ? (int64_t)__ldg(perm + p) : p;
            val[u] = epi.act ? ld.load(p, i, j, C, cwp) : TA(0);
          } else {
            kk[u] = kSentinel;
            val[u] = TA(0);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t b0 = base + (int64_t)u * G;
          if (b0 >= it.pe) break;  // warp-uniform
          const int nvalid = (int)((it.pe - b0) < G ? (it.pe - b0) : G);
          const int k0 = __shfl_sync(FE_FULL, kk[u], j);
          if (ckey >= 0 && ckey != k0) {
            if (g == 0) epi.finalize(d, k, ckey, j, C, (double)carry, na, nb);
            ckey = -1;
            carry = TA(0);
          }
          TA v = val[u];
          const int km = kk[u];
#pragma unroll
          for (int dd = 1; dd < G; dd <<= 1) {
            const TA vo = __shfl_up_sync(FE_FULL, v, dd * C);
            const int ko = __shfl_up_sync(FE_FULL, km, dd * C);
            if (g >= dd && ko == km) v += vo;
          }
          if (km == ckey) v += carry;
          const int kn = __shfl_down_sync(FE_FULL, km, C);
          if (g < nvalid - 1 && kn != km) epi.finalize(d, k, km, j, C, (double)v, na, nb);
          const int src = (nvalid - 1) * C + j;
          ckey = __shfl_sync(FE_FULL, km, src);
          carry = __shfl_sync(FE_FULL, v, src);
        }
      }
      if (ckey >= 0) {
        if (it.split < 0) {
          if (g == 0) epi.finalize(d, k, ckey, j, C, (double)carry, na, nb);
        } else {
          const SplitLevel sl = splits[it.split];
          if (g == 0) piece_part[(int64_t)(sl.first_piece + it.pad) * C + j] = (double)carry;
          __threadfence();
          __syncwarp();
          int last = 0;
          if (lane == 0) last = (atomicAdd(split_cnt + it.split, 1) == sl.npieces - 1) ? 1 : 0;
          last = __shfl_sync(FE_FULL, last, 0);
          if (last) {
            __threadfence();
            if (g == 0) {
              double tot = 0.0;
              for (int q = 0; q < sl.npieces; ++q)
                tot += __ldcg(piece_part + (int64_t)(sl.first_piece + q) * C + j);
              double sa = 0.0, sb = 0.0;
              epi.finalize(d, k, ckey, j, C, tot, sa, sb);
              if (part_a) part_a[(int64_t)j * S + sl.norm_slot] = sa;
              if (part_b) part_b[(int64_t)j * S + sl.norm_slot] = sb;
            }
            if (lane == 0) split_cnt[it.split] = 0;
          }
        }
      }
    }
  }
  const int64_t slot = cta_slot ? (int64_t)cta_slot[blockIdx.x] : -1;
  cta_norm_to_slot<C>(na, part_a, S, slot, sm);
  __syncthreads();
  cta_norm_to_slot<C>(nb, part_b, S, slot, sm);
}

}  // namespace fe
