// fe_kernels.cuh -- sm_100a kernels of the fixed-effects LSMR hot path.
//
// Every kernel here is HBM-bound integer-indexed gather / segmented-reduction
// work; nothing is a dense contraction, so there are no tensor-core paths.
//
// Layout: a column tile of C right-hand sides is stored observation-major
// ([N][C], one row per observation) and level-major ([P][C]) on the
// coefficient side.  Each lane owns VEC consecutive columns of a row (16-byte
// vectors: 4 floats or 2 doubles), a row is CL = C/VEC lanes wide, and a warp
// instruction covers G = 32/CL rows.  Lane (g, jl) handles row slot g and
// columns jl*VEC .. jl*VEC+VEC-1.
//
// Three kernels make one matvec pair:
//   k_expand  u <- f(A v, u)             (the reference's scatter!, per FE)
//   k_segsum  S[l] = sum_{i in l} c_i u_i (the reference's gather!, per FE)
//   k_pupdate the per-level epilogue: v <- S*scale/beta - beta v, the deferred
//             LSMR h/hbar/x update, and the norms, streamed over levels.
// Index vectors (refs, level-order perms and keys, interaction*sqrt(w)) are
// read with coalesced warp-wide loads and broadcast with shuffles.
//
// Determinism: no floating-point atomics anywhere.  Each segsum work item is
// summed by one warp in a fixed order; long levels are cut into pieces whose
// partials are summed in piece order by the last piece to finish (an integer
// atomic counter decides who is last; the sum order does not depend on it);
// norms are reduced per CTA into fixed slots that a scalar kernel sums in
// slot order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "fe_internal.h"

namespace fe {

#define FE_FULL 0xffffffffu

// ---------------------------------------------------------------------------
// small vectors
// ---------------------------------------------------------------------------
template <typename T, int V>
struct VA {
  T v[V];
};

// Loads/stores of V contiguous elements as 16-, 8- or 4-byte accesses.  The
// offsets used below are multiples of V, and slabs are 256-byte aligned, so
// every access is naturally aligned.
template <int B> struct Carrier { };
template <> struct Carrier<16> { using type = float4; };
template <> struct Carrier<8> { using type = float2; };
template <> struct Carrier<4> { using type = float; };

template <typename T, int V>
struct VecIO {
  static constexpr int kBytes = (int)sizeof(T) * V;
  static constexpr int kChunk = kBytes >= 16 ? 16 : kBytes;
  static constexpr int kN = kBytes / kChunk;
  using Cr = typename Carrier<kChunk>::type;
};

template <typename T, int V>
__device__ __forceinline__ VA<T, V> vld(const T* p) {
  using IO = VecIO<T, V>;
  typename IO::Cr c[IO::kN];
#pragma unroll
  for (int q = 0; q < IO::kN; ++q) c[q] = reinterpret_cast<const typename IO::Cr*>(p)[q];
  VA<T, V> a;
  memcpy(&a, c, sizeof(a));
  return a;
}
template <typename T, int V>
__device__ __forceinline__ VA<T, V> vldg(const T* p) {
  using IO = VecIO<T, V>;
  typename IO::Cr c[IO::kN];
#pragma unroll
  for (int q = 0; q < IO::kN; ++q) c[q] = __ldg(reinterpret_cast<const typename IO::Cr*>(p) + q);
  VA<T, V> a;
  memcpy(&a, c, sizeof(a));
  return a;
}
template <typename T, int V>
__device__ __forceinline__ void vst(T* p, const VA<T, V>& a) {
  using IO = VecIO<T, V>;
  typename IO::Cr c[IO::kN];
  memcpy(c, &a, sizeof(a));
#pragma unroll
  for (int q = 0; q < IO::kN; ++q) reinterpret_cast<typename IO::Cr*>(p)[q] = c[q];
}

// Asynchronous global -> shared copies (cp.async, hand-written PTX).
__device__ __forceinline__ void cp_async_bytes16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_bytes8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_bytes4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
template <int B>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  if (B == 16) cp_async_bytes16(smem, gmem);
  else if (B == 8) cp_async_bytes8(smem, gmem);
  else cp_async_bytes4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Streaming (evict-first) variants for data touched once per kernel, so that
// it does not push reused coefficient rows out of L1/L2.
template <typename T, int V>
__device__ __forceinline__ VA<T, V> vld_cs(const T* p) {
  using IO = VecIO<T, V>;
  typename IO::Cr c[IO::kN];
#pragma unroll
  for (int q = 0; q < IO::kN; ++q) c[q] = __ldcs(reinterpret_cast<const typename IO::Cr*>(p) + q);
  VA<T, V> a;
  memcpy(&a, c, sizeof(a));
  return a;
}
template <typename T, int V>
__device__ __forceinline__ void vst_cs(T* p, const VA<T, V>& a) {
  using IO = VecIO<T, V>;
  typename IO::Cr c[IO::kN];
  memcpy(c, &a, sizeof(a));
#pragma unroll
  for (int q = 0; q < IO::kN; ++q) __stcs(reinterpret_cast<typename IO::Cr*>(p) + q, c[q]);
}

// lane shape for accumulation type TA and tile width C
template <typename TA, int C>
struct Shape {
  static constexpr int VEC = sizeof(TA) == 4 ? (C >= 4 ? 4 : C) : (C >= 2 ? 2 : 1);
  static constexpr int CL = C / VEC;  // lanes per row
  static constexpr int G = 32 / CL;   // rows per warp instruction
};

template <typename T> __device__ __forceinline__ const T* scale_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* scale_of<float>(const FeDev& d, int k) { return d.scale_f[k]; }
template <> __device__ __forceinline__ const double* scale_of<double>(const FeDev& d, int k) { return d.scale_d[k]; }
template <typename T> __device__ __forceinline__ const T* cw_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* cw_of<float>(const FeDev& d, int k) { return d.cw_f[k]; }
template <> __device__ __forceinline__ const double* cw_of<double>(const FeDev& d, int k) { return d.cw_d[k]; }
template <typename T> __device__ __forceinline__ const T* cwp_of(const FeDev& d, int k);
template <> __device__ __forceinline__ const float* cwp_of<float>(const FeDev& d, int k) { return d.cwp_f[k]; }
template <> __device__ __forceinline__ const double* cwp_of<double>(const FeDev& d, int k) { return d.cwp_d[k]; }

// Per-column norm accumulators of one CTA -> one slot per CTA (fixed order).
// nrm[v] is column jl*VEC+v of this lane.
template <int C, int VEC>
__device__ __forceinline__ void cta_norm_to_slot(const double (&nrm)[VEC], double* __restrict__ part,
                                                 int64_t S, int64_t slot, double (*sm)[32]) {
  constexpr int CL = C / VEC;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    double a = nrm[v];
#pragma unroll
    for (int o = CL; o < 32; o <<= 1) a += __shfl_xor_sync(FE_FULL, a, o);
    if (lane < CL) sm[wib][lane * VEC + v] = a;
  }
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
// kPrescaled: the table rows already hold scale_l * x_l, so the gather
// multiplies by the observation's weight only.
template <typename T, typename TA, int VEC>
struct TabOne {
  static constexpr bool kPrescaled = false;
  const T* __restrict__ tab;
  __device__ __forceinline__ VA<TA, VEC> load(int64_t off) const {
    const VA<T, VEC> a = vldg<T, VEC>(tab + off);
    VA<TA, VEC> r;
#pragma unroll
    for (int v = 0; v < VEC; ++v) r.v[v] = (TA)a.v[v];
    return r;
  }
};
// (x64 + dx32) .* scale, written once per refinement round by k_prescale64
// (the FP64 residual's table: one FP64 row per gathered level, no scale load).
template <int VEC>
struct TabPre64 {
  static constexpr bool kPrescaled = true;
  const double* __restrict__ tab;
  __device__ __forceinline__ VA<double, VEC> load(int64_t off) const {
    return vldg<double, VEC>(tab + off);
  }
};

// out[l][j] = (x64[l][j] + x32[l][j]) * scale[l] for the n levels of one FE
// (pointers already offset to the FE's first level); two columns per thread.
static __global__ void __launch_bounds__(256) k_prescale64(const double* __restrict__ x64,
                                                           const float* __restrict__ x32,
                                                           const double* __restrict__ scale,
                                                           double* __restrict__ out, int64_t n, int C) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // pair index
  const int half = (C + 1) / 2;
  if (e >= n * half) return;
  const int64_t l = e / half;
  const int j = (int)(e - l * half) * 2;
  const double sc = scale[l];
  const int64_t o = l * C + j;
  out[o] = (x64[o] + (double)x32[o]) * sc;
  if (j + 1 < C) out[o + 1] = (x64[o + 1] + (double)x32[o + 1]) * sc;
}

// ---------------------------------------------------------------------------
// Expand epilogues.  begin() loads the per-column coefficients of the lane's
// VEC columns; pre(o) loads the observation's old values; apply() gets
// s = (A x)[i, cols] and adds the squared new values to nrm.
// ---------------------------------------------------------------------------
// LSMR u-update: U <- av * (A v) + au * U   (src/utils/lsmr.jl:104 with the
// normalisations of u and v folded into av, au).  A stopped instance has
// av = 0, au = 1, so its U is left as it is (its norm is not used).
template <typename T, int VEC>
struct EpiExpandLsmr {
  using TP = T;
  using TN = T;  // norm accumulation within an item
  T* __restrict__ U;
  const Inst* __restrict__ inst;
  T av[VEC], au[VEC];
  bool act;
  __device__ __forceinline__ void begin(int prob, int jl, int C) {
    act = false;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const Inst& s = inst[(int64_t)prob * C + jl * VEC + v];
      av[v] = (T)s.ex_av;
      au[v] = (T)s.ex_au;
      act = act || s.active != 0;
    }
  }
  __device__ __forceinline__ VA<T, VEC> pre(int64_t o) const { return vld_cs<T, VEC>(U + o); }
  __device__ __forceinline__ VA<T, VEC> apply(int64_t o, const VA<T, VEC>& s,
                                               const VA<T, VEC>& old, TN (&nrm)[VEC]) {
    VA<T, VEC> u;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      u.v[v] = av[v] * s.v[v] + au[v] * old.v[v];
      nrm[v] += u.v[v] * u.v[v];
    }
    vst_cs<T, VEC>(U + o, u);
    return u;
  }
};

// out <- B - (A x): initial u of LSMR and the final residual
// (src/utils/lsmr.jl:63, src/AbstractFixedEffectSolver.jl:62).  mask: 0 all
// instances, 2 only instances whose refinement is still running (the others
// keep their stored residual).
template <typename TOut, typename TA, int VEC>
struct EpiBminusAx {
  using TP = double;
  using TN = double;
  const double* __restrict__ B;
  TOut* __restrict__ out;
  float* __restrict__ out32;  // optional FP32 copy (mixed-precision u)
  const Inst* __restrict__ inst;
  int mask;
  bool actv[VEC];
  bool act, all;
  __device__ __forceinline__ void begin(int prob, int jl, int C) {
    act = false;
    all = true;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      actv[v] = mask == 2 ? inst[(int64_t)prob * C + jl * VEC + v].outer_active != 0 : true;
      act = act || actv[v];
      all = all && actv[v];
    }
  }
  __device__ __forceinline__ VA<double, VEC> pre(int64_t o) const { return vldg<double, VEC>(B + o); }
  __device__ __forceinline__ VA<TA, VEC> apply(int64_t o, const VA<TA, VEC>& s,
                                                const VA<double, VEC>& b, TN (&nrm)[VEC]) {
    VA<TOut, VEC> r;
    VA<TA, VEC> ret;
    VA<float, VEC> r32;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const double x = b.v[v] - (double)s.v[v];
      r.v[v] = (TOut)x;
      r32.v[v] = (float)x;
      ret.v[v] = (TA)r.v[v];
      if (actv[v]) nrm[v] += x * x;
    }
    if (all) {
      vst<TOut, VEC>(out + o, r);
      if (out32) vst<float, VEC>(out32 + o, r32);
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        if (actv[v]) {
          out[o + v] = r.v[v];
          if (out32) out32[o + v] = r32.v[v];
        }
    }
    return ret;
  }
};

// ---------------------------------------------------------------------------
// Segmented run accumulation shared by k_segsum and the fused k_expand.
// Rows arrive G at a time (one per lane group) in key order; equal keys are
// contiguous.  An inclusive segmented scan over the groups plus a carry across
// steps yields each key's sum; the group holding a key's last row stores it.
// ---------------------------------------------------------------------------
template <typename TA, int VEC, int CL, int G>
struct SegRun {
  int ckey;
  VA<TA, VEC> carry;  // running sum of key ckey (the same in every group)
  VA<TA, VEC> acc;    // per-group partial of ckey from fast-path steps
  bool pend;          // acc holds something (warp-uniform)
  __device__ __forceinline__ void init() {
    ckey = -1;
    pend = false;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      carry.v[v] = TA(0);
      acc.v[v] = TA(0);
    }
  }
  // carry += sum over groups of acc (fixed xor tree)
  __device__ __forceinline__ void fold() {
    if (!pend) return;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      TA t = acc.v[v];
#pragma unroll
      for (int o = CL; o < 32; o <<= 1) t += __shfl_xor_sync(FE_FULL, t, o);
      carry.v[v] += t;
      acc.v[v] = TA(0);
    }
    pend = false;
  }
  // one warp instruction worth of rows: key km and value x of this lane's
  // group; nvalid groups hold real rows.  Sk points at the lane's column block
  // of row 0 of the FE's [levels][C] sum slab.
  __device__ __forceinline__ void push(int km, VA<TA, VEC> x, int nvalid, int g, int jl, int C,
                                       TA* __restrict__ Sk) {
    // fast path: every group continues the current run (long levels)
    if (G > 1 && ckey >= 0 && __all_sync(FE_FULL, km == ckey)) {
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc.v[v] += x.v[v];
      pend = true;
      return;
    }
    fold();
    const int k0 = __shfl_sync(FE_FULL, km, jl);
    if (ckey >= 0 && ckey != k0) {
      if (g == 0) vst<TA, VEC>(Sk + (int64_t)ckey * C, carry);
      ckey = -1;
#pragma unroll
      for (int v = 0; v < VEC; ++v) carry.v[v] = TA(0);
    }
#pragma unroll
    for (int dd = 1; dd < G; dd <<= 1) {
      const int ko = __shfl_up_sync(FE_FULL, km, dd * CL);
      const bool take = g >= dd && ko == km;
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        const TA xo = __shfl_up_sync(FE_FULL, x.v[v], dd * CL);
        if (take) x.v[v] += xo;
      }
    }
    if (km == ckey) {
#pragma unroll
      for (int v = 0; v < VEC; ++v) x.v[v] += carry.v[v];
    }
    const int kn = __shfl_down_sync(FE_FULL, km, CL);
    if (g < nvalid - 1 && kn != km) vst<TA, VEC>(Sk + (int64_t)km * C, x);
    const int srcl = (nvalid - 1) * CL + jl;
    ckey = __shfl_sync(FE_FULL, km, srcl);
#pragma unroll
    for (int v = 0; v < VEC; ++v) carry.v[v] = __shfl_sync(FE_FULL, x.v[v], srcl);
  }
  // end of a work item.  split < 0: the last key is complete.  Otherwise the
  // item is piece `piece` of split level sa.splits[split], combined in two
  // deterministic stages (see SplitLevel).  smt: 32 doubles of shared scratch
  // owned by this warp.
  __device__ __forceinline__ void finish(int split, int piece, const SplitArgs& sa, int g, int jl,
                                         int C, TA* __restrict__ Sk, double* smt) {
    fold();
    if (ckey < 0) return;
    if (split < 0) {
      if (g == 0) vst<TA, VEC>(Sk + (int64_t)ckey * C, carry);
      return;
    }
    const int lane = threadIdx.x & 31;
    const SplitLevel sl = sa.splits[split];
    if (g == 0) {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        sa.piece_part[(int64_t)(jl * VEC + v) * sa.n_pieces + sl.first_piece + piece] =
            (double)carry.v[v];
    }
    // stage 1: the last piece of the block sums the block
    const int blk = piece / kSplitBlock;
    const int p0 = blk * kSplitBlock;
    const int np = min(kSplitBlock, sl.npieces - p0);
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane == 0) last = (atomicAdd(sa.block_cnt + sl.first_block + blk, 1) == np - 1) ? 1 : 0;
    last = __shfl_sync(FE_FULL, last, 0);
    if (!last) return;
    __threadfence();
    for (int jj = 0; jj < C; ++jj) {
      double acc = lane < np ? __ldcg(sa.piece_part + (int64_t)jj * sa.n_pieces + sl.first_piece + p0 + lane) : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FE_FULL, acc, o);
      if (lane == 0) sa.block_part[(int64_t)jj * sa.n_blocks + sl.first_block + blk] = acc;
    }
    if (lane == 0) sa.block_cnt[sl.first_block + blk] = 0;
    // stage 2: the last block sums the level
    __threadfence();
    __syncwarp();
    last = 0;
    if (lane == 0) last = (atomicAdd(sa.level_cnt + split, 1) == sl.nblocks - 1) ? 1 : 0;
    last = __shfl_sync(FE_FULL, last, 0);
    if (!last) return;
    __threadfence();
    for (int jj = 0; jj < C; ++jj) {
      const double* bp = sa.block_part + (int64_t)jj * sa.n_blocks + sl.first_block;
      double acc = 0.0;
      for (int q = lane; q < sl.nblocks; q += 32) acc += __ldcg(bp + q);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FE_FULL, acc, o);
      if (lane == 0) smt[jj] = acc;
    }
    __syncwarp();
    if (g == 0) {
      VA<TA, VEC> tot;
#pragma unroll
      for (int v = 0; v < VEC; ++v) tot.v[v] = (TA)smt[jl * VEC + v];
      vst<TA, VEC>(Sk + (int64_t)ckey * C, tot);
    }
    if (lane == 0) sa.level_cnt[split] = 0;
  }
};

// ---------------------------------------------------------------------------
// k_expand: one warp per ExpandItem (a range of sorted observations); U row
// slots per lane group per step, KB >= number of FEs (compile-time bound so
// that every index and row load of a step can be issued before the first is
// consumed).  PF = 1: the next step's refs and weights are prefetched while
// the current step's rows are in flight; PF = 2: its old rows as well, so a
// step waits only for its coefficient-row gathers.
// ---------------------------------------------------------------------------
template <typename TA, int C, int U, int KB, int PF, class Tab, class Epi>
__global__ void __launch_bounds__(kThreads)
k_expand(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items, Tab tab, Epi epi,
         double* __restrict__ part, int64_t S) {
  using Sh = Shape<TA, C>;
  constexpr int VEC = Sh::VEC, CL = Sh::CL, G = Sh::G;
  constexpr int STEP = G * U;                     // observations per step
  constexpr int NI = STEP >= 32 ? STEP / 32 : 1;  // index registers per lane
  static_assert(STEP <= 32 || STEP % 32 == 0, "a step's indices fill whole index registers");
  using TP = typename Epi::TP;
  using TN = typename Epi::TN;
  __shared__ double sm[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane / CL, jl = lane - g * CL;
  double nrm[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) nrm[v] = 0.0;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wib;
  if (w < n_items) {
    const ExpandItem it = items[w];
    epi.begin(it.prob, jl, C);
    if (__any_sync(FE_FULL, epi.act)) {
      const int K = d.K;
      TN nit[VEC];  // norms of this item (FP32 for the FP32 path), flushed below
#pragma unroll
      for (int v = 0; v < VEC; ++v) nit[v] = TN(0);
      int rl[KB][NI];
      TA cl[KB][NI];
      auto fetch = [&](int64_t base) {
#pragma unroll
        for (int k = 0; k < KB; ++k) {
#pragma unroll
          for (int r = 0; r < NI; ++r) {
            const int64_t p = base + r * 32 + lane;
            const bool ok = k < K && p < it.ie && (r * 32 + lane) < STEP;
            rl[k][r] = ok ? __ldcs(d.refs[k] + p) : kSentinel;
            const TA* __restrict__ cw = cw_of<TA>(d, k < K ? k : 0);
            cl[k][r] = (ok && cw) ? __ldg(cw + p) : TA(1);
          }
        }
      };
      if (PF) fetch(it.ib);
      VA<TP, VEC> oldn[U];  // PF == 2: the next step's old rows
      if (PF == 2) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t i = it.ib + u * G + g;
          if (i < it.ie && epi.act) oldn[u] = epi.pre(i * C + jl * VEC);
        }
      }
      for (int64_t base = it.ib; base < it.ie; base += STEP) {
        if (!PF) fetch(base);
        int rc[KB][NI];
        TA cc[KB][NI];
#pragma unroll
        for (int k = 0; k < KB; ++k)
#pragma unroll
          for (int r = 0; r < NI; ++r) {
            rc[k][r] = rl[k][r];
            cc[k][r] = cl[k][r];
          }
        if (PF && base + STEP < it.ie) fetch(base + STEP);
        VA<TP, VEC> old[U];
        VA<TA, VEC> s[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t i = base + u * G + g;
#pragma unroll
          for (int v = 0; v < VEC; ++v) s[u].v[v] = TA(0);
          if (PF == 2) {
            old[u] = oldn[u];
          } else if (i < it.ie && epi.act) {
            old[u] = epi.pre(i * C + jl * VEC);
          }
        }
        if (PF == 2 && base + STEP < it.ie) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int64_t i = base + STEP + u * G + g;
            if (i < it.ie && epi.act) oldn[u] = epi.pre(i * C + jl * VEC);
          }
        }
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          if (k < K && !(d.absorb && k == d.primary)) {
            const TA* __restrict__ sc = scale_of<TA>(d, k);
            const int64_t lb = d.lev_base[k];
            const bool wk = cw_of<TA>(d, k) != nullptr;  // uniform
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int q = u * G;  // + g: the same index register (G divides 32)
              const int ref = __shfl_sync(FE_FULL, rc[k][q >> 5], (q & 31) + g);
              const TA c = wk ? __shfl_sync(FE_FULL, cc[k][q >> 5], (q & 31) + g) : TA(1);
              const int64_t i = base + u * G + g;
              if (i < it.ie && epi.act) {
                TA cs;
                if constexpr (Tab::kPrescaled) {
                  cs = wk ? c : TA(1);
                } else {
                  const TA scl = __ldg(sc + ref);
                  cs = wk ? c * scl : scl;
                }
                const VA<TA, VEC> t = tab.load((lb + ref) * C + jl * VEC);
#pragma unroll
                for (int v = 0; v < VEC; ++v) s[u].v[v] += cs * t.v[v];
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t i = base + u * G + g;
          if (i < it.ie && epi.act) (void)epi.apply(i * C + jl * VEC, s[u], old[u], nit);
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) nrm[v] += (double)nit[v];
    }
  }
  __syncthreads();
  cta_norm_to_slot<C, VEC>(nrm, part, S, (int64_t)blockIdx.x, sm);
}

// ---------------------------------------------------------------------------
// k_rowsum: the reductions that need no gather (the reference's gather!,
// src/SolverCPU.jl:21-27, for those FEs) in one contiguous pass over the
// sorted observation rows of a 32-column tile:
//   - the primary FE: observations are sorted by it, so each of its levels is
//     a contiguous run of rows;
//   - small FEs (at most kSmallRows table rows in total, e.g. a year FE):
//     summed into a per-warp table in shared memory.
// One column per lane.  A step loads the keys (and weights) of STEP rows with
// one coalesced load per FE and the STEP rows themselves (STEP independent
// loads per lane, 4 KB per warp in flight), then walks them in order: a
// primary level is stored at each key change, and every row is added into the
// small-FE tables.  The segsum then gathers only the remaining (large) FEs.
//
// Work split: warp wib of CTA b takes the expand items (whole primary levels,
// or pieces of long ones) b*8 + wib + j*grid*8, so the warps in flight work
// on neighbouring rows and the tables' summation order depends only on the
// grid size.  At the end the 8
// warp tables are summed (warp order, FP64) into the CTA's partial slot;
// k_small_combine sums the slots in CTA order into the [P][C] slab.
// ---------------------------------------------------------------------------
struct RowSumArgs {
  void* sum;                  // [P][C] TA slab: primary level sums
  SplitArgs sa;               // pieces of long primary levels
  double* small_part;         // [grid][small_rows][C] CTA partials of the small FEs
  int32_t n_small;            // small FEs (<= kRowSumSmallFE)
  int32_t small_fe[kRowSumSmallFE];
  int32_t small_off[kRowSumSmallFE];  // first table row of each
  int32_t small_rows;         // table rows in use
};

// Row ring of one warp: NBUF buffers of STEP rows; NBUF-1 steps are in
// flight while one is walked.
template <typename TA> struct RowSumStep {
  static constexpr int value = 16;
  static constexpr int NBUF = sizeof(TA) == 4 ? 3 : 2;
};

// The walk of one step, in groups of 4 rows (r0 a compile-time multiple of 4
// in the unrolled full-step walk).  Primary FE: a running sum per lane,
// stored at each level change.  Small FEs: rows of a group with equal keys
// are added together first (into the group's first row with that key), so the
// remaining table rows are distinct and their 4 loads, adds and stores are
// independent: one shared-memory round trip per group instead of per row.
template <typename TA, int C, bool W>
__device__ __forceinline__ void rowsum_primary(int r, const TA x, TA& acc, uint32_t bmask,
                                               int kpr, TA cpv, TA* __restrict__ Sf) {
  acc += W ? x * __shfl_sync(FE_FULL, cpv, r) : x;
  if ((bmask >> r) & 1u) {
    const int kr = __shfl_sync(FE_FULL, kpr, r);
    Sf[(int64_t)kr * C] = acc;
    acc = TA(0);
  }
}

template <typename TA, int C, bool W>
__device__ __forceinline__ void rowsum_small4(int r0, TA v0, TA v1, TA v2, TA v3, int kt, TA ct,
                                              TA* __restrict__ tbl, int lane) {
  const int t0 = __shfl_sync(FE_FULL, kt, r0);
  const int t1 = __shfl_sync(FE_FULL, kt, r0 + 1);
  const int t2 = __shfl_sync(FE_FULL, kt, r0 + 2);
  const int t3 = __shfl_sync(FE_FULL, kt, r0 + 3);
  if (W) {
    v0 *= __shfl_sync(FE_FULL, ct, r0);
    v1 *= __shfl_sync(FE_FULL, ct, r0 + 1);
    v2 *= __shfl_sync(FE_FULL, ct, r0 + 2);
    v3 *= __shfl_sync(FE_FULL, ct, r0 + 3);
  }
  // a row whose key appeared earlier in the group is added into that row
  // (the first with the key); the rows left have distinct keys
  const bool s1 = t1 != t0;
  const bool s2 = t2 != t0 && t2 != t1;
  const bool s3 = t3 != t0 && t3 != t1 && t3 != t2;
  const int d3 = t3 == t0 ? 0 : (t3 == t1 ? 1 : 2);  // target of row 3 when !s3
  const int d2 = t2 == t0 ? 0 : 1;                    // target of row 2 when !s2
  if (!s3) {
    if (d3 == 0) v0 += v3;
    else if (d3 == 1) v1 += v3;
    else v2 += v3;
  }
  if (!s2) {
    if (d2 == 0) v0 += v2;
    else v1 += v2;
  }
  if (!s1) v0 += v1;
  TA* p0 = tbl + t0 * C + lane;
  TA* p1 = tbl + t1 * C + lane;
  TA* p2 = tbl + t2 * C + lane;
  TA* p3 = tbl + t3 * C + lane;
  TA a0 = *p0;
  TA a1 = s1 ? *p1 : TA(0);
  TA a2 = s2 ? *p2 : TA(0);
  TA a3 = s3 ? *p3 : TA(0);
  a0 += v0;
  a1 += v1;
  a2 += v2;
  a3 += v3;
  *p0 = a0;
  if (s1) *p1 = a1;
  if (s2) *p2 = a2;
  if (s3) *p3 = a3;
}

// one row at a time (partial steps)
template <typename TA, int C, bool W, int NS>
__device__ __forceinline__ void rowsum_row(int r, const TA x, TA& acc, uint32_t bmask, int kpr,
                                           TA cpv, int k0, TA c0, int k1, TA c1,
                                           TA* __restrict__ Sf, TA* __restrict__ tbl, int lane) {
  rowsum_primary<TA, C, W>(r, x, acc, bmask, kpr, cpv, Sf);
  if (NS > 0) {
    const int t0 = __shfl_sync(FE_FULL, k0, r);
    tbl[t0 * C + lane] += W ? x * __shfl_sync(FE_FULL, c0, r) : x;
  }
  if (NS > 1) {
    const int t1 = __shfl_sync(FE_FULL, k1, r);
    tbl[t1 * C + lane] += W ? x * __shfl_sync(FE_FULL, c1, r) : x;
  }
}

// a full step of STEP rows (a multiple of 4)
template <typename TA, int C, bool W, int NS, int STEP>
__device__ __forceinline__ void rowsum_full_step(const TA (&xs)[STEP], TA& acc, uint32_t bmask,
                                                 int kpr, TA cpv, int k0, TA c0, int k1, TA c1,
                                                 TA* __restrict__ Sf, TA* __restrict__ tbl,
                                                 int lane) {
  static_assert(STEP % 4 == 0, "groups of 4 rows");
#pragma unroll
  for (int r0 = 0; r0 < STEP; r0 += 4) {
    TA x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      x[j] = xs[r0 + j];
      rowsum_primary<TA, C, W>(r0 + j, x[j], acc, bmask, kpr, cpv, Sf);
    }
    if (NS > 0) rowsum_small4<TA, C, W>(r0, x[0], x[1], x[2], x[3], k0, c0, tbl, lane);
    if (NS > 1) rowsum_small4<TA, C, W>(r0, x[0], x[1], x[2], x[3], k1, c1, tbl, lane);
  }
}

// W: some reduced FE has weights (cw); NS: small FEs reduced in the tables.
template <typename TA, int C, bool W, int NS>
__global__ void __launch_bounds__(kThreads, sizeof(TA) == 4 ? 4 : 2)
k_rowsum(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items,
         const TA* __restrict__ src, RowSumArgs rs) {
  static_assert(C == 32, "the walk puts one column on each lane");
  constexpr int STEP = RowSumStep<TA>::value;
  constexpr int NBUF = RowSumStep<TA>::NBUF;
  constexpr int BUF = STEP * C;                               // elements per buffer
  constexpr int CHUNKS = BUF * (int)sizeof(TA) / 16 / 32;     // 16-byte copies per lane
  constexpr int ROWCH = C * (int)sizeof(TA) / 16;             // 16-byte chunks per row
  static_assert(CHUNKS * 32 * 16 == BUF * (int)sizeof(TA), "whole chunks per lane");
  __shared__ double smt[kWarps][32];
  extern __shared__ __align__(16) unsigned char rowsum_smem[];
  if (d.active && *d.active == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  TA* wbuf = reinterpret_cast<TA*>(rowsum_smem) + (size_t)wib * NBUF * BUF;     // row ring
  TA* tbl = reinterpret_cast<TA*>(rowsum_smem) + (size_t)kWarps * NBUF * BUF +  // small-FE table
            (size_t)wib * rs.small_rows * C;
  for (int e = lane; e < rs.small_rows * C; e += 32) tbl[e] = TA(0);
  __syncwarp();
  const int kp = d.primary;
  TA* __restrict__ Sf = reinterpret_cast<TA*>(rs.sum) + d.lev_base[kp] * C + lane;
  const int32_t* __restrict__ refp = d.refs[kp];
  const TA* __restrict__ cwp = cw_of<TA>(d, kp);
  const int32_t* __restrict__ ref0 = NS > 0 ? d.refs[rs.small_fe[0]] : nullptr;
  const int32_t* __restrict__ ref1 = NS > 1 ? d.refs[rs.small_fe[1]] : nullptr;
  const TA* __restrict__ cw0 = NS > 0 ? cw_of<TA>(d, rs.small_fe[0]) : nullptr;
  const TA* __restrict__ cw1 = NS > 1 ? cw_of<TA>(d, rs.small_fe[1]) : nullptr;
  const int off0 = rs.small_off[0], off1 = rs.small_off[1];
  const int64_t wstride = (int64_t)gridDim.x * kWarps;
  for (int64_t wi = (int64_t)blockIdx.x * kWarps + wib; wi < n_items; wi += wstride) {
    const ExpandItem it = items[wi];
    const int64_t ie = it.ie;
    if (ie <= it.ib) continue;
    // copy the rows of the step at `base` into buffer b (one commit group,
    // empty past the end of the item)
    auto issue = [=](int64_t base, int b) {
      const int64_t left = ie - base;
      const int nv = (int)(left < STEP ? (left > 0 ? left : 0) : STEP);
      const unsigned char* g = reinterpret_cast<const unsigned char*>(src + base * C);
      unsigned char* sp = reinterpret_cast<unsigned char*>(wbuf + b * BUF);
#pragma unroll
      for (int q = 0; q < CHUNKS; ++q) {
        const int ch = q * 32 + lane;
        if (ch < nv * ROWCH) cp_async_bytes16(sp + ch * 16, g + ch * 16);
      }
      cp_async_commit();
    };
    // keys and weights of the step at `base` (row base + lane); a missing
    // weight vector reads as 1
    int kpr_n = kSentinel, k0_n = 0, k1_n = 0;
    TA cp_n = TA(1), c0_n = TA(1), c1_n = TA(1);
    auto keys = [&kpr_n, &k0_n, &k1_n, &cp_n, &c0_n, &c1_n, ie, lane, refp, cwp, ref0, ref1, cw0,
                 cw1, off0, off1](int64_t base) {
      const int64_t p = base + lane;
      const bool ok = lane < STEP && p < ie;
      kpr_n = ok ? __ldg(refp + p) : kSentinel;
      if (W) cp_n = (ok && cwp) ? __ldg(cwp + p) : TA(1);
      if (NS > 0) {
        k0_n = ok ? off0 + __ldg(ref0 + p) : 0;
        if (W) c0_n = (ok && cw0) ? __ldg(cw0 + p) : TA(1);
      }
      if (NS > 1) {
        k1_n = ok ? off1 + __ldg(ref1 + p) : 0;
        if (W) c1_n = (ok && cw1) ? __ldg(cw1 + p) : TA(1);
      }
    };
#pragma unroll
    for (int q = 0; q < NBUF - 1; ++q) issue(it.ib + (int64_t)q * STEP, q);
    keys(it.ib);
    int ckey = -1;  // primary level of the open run (warp-uniform)
    TA acc = TA(0);
    int b = 0;
    for (int64_t base = it.ib; base < ie; base += STEP, b = (b + 1 == NBUF ? 0 : b + 1)) {
      const int kpr = kpr_n, k0 = k0_n, k1 = k1_n;
      const TA cpv = cp_n, c0 = c0_n, c1 = c1_n;
      const int nvalid = (int)((ie - base) < STEP ? (ie - base) : STEP);
      issue(base + (int64_t)(NBUF - 1) * STEP, b == 0 ? NBUF - 1 : b - 1);
      if (base + STEP < ie) keys(base + STEP);
      cp_async_wait<NBUF - 1>();  // this step's group is complete
      __syncwarp();               // every lane's copies of this step are visible
      const int kn = __shfl_down_sync(FE_FULL, kpr, 1);
      const uint32_t bmask = __ballot_sync(FE_FULL, lane + 1 < nvalid && kn != kpr);
      const int kfirst = __shfl_sync(FE_FULL, kpr, 0);
      if (ckey >= 0 && ckey != kfirst) {
        Sf[(int64_t)ckey * C] = acc;
        acc = TA(0);
      }
      const TA* __restrict__ rows = wbuf + b * BUF + lane;
      if (nvalid == STEP) {
        TA xs[STEP];
#pragma unroll
        for (int r = 0; r < STEP; ++r) xs[r] = rows[r * C];
        rowsum_full_step<TA, C, W, NS, STEP>(xs, acc, bmask, kpr, cpv, k0, c0, k1, c1, Sf, tbl,
                                             lane);
      } else {
#pragma unroll 1
        for (int r = 0; r < nvalid; ++r)
          rowsum_row<TA, C, W, NS>(r, rows[r * C], acc, bmask, kpr, cpv, k0, c0, k1, c1, Sf, tbl,
                                   lane);
      }
      ckey = __shfl_sync(FE_FULL, kpr, nvalid - 1);
      __syncwarp();  // buffer b is free for the copies of step + NBUF
    }
    // the open run: a whole level, or one piece of a long one
    SegRun<TA, 1, 32, 1> run;
    run.ckey = ckey;
    run.carry.v[0] = acc;
    run.acc.v[0] = TA(0);
    run.pend = false;
    run.finish(it.split, it.piece, rs.sa, 0, lane, C, Sf, smt[wib]);
  }
  if (NS > 0) {
    __syncthreads();
    const int n = rs.small_rows * C;
    double* __restrict__ out = rs.small_part + (int64_t)blockIdx.x * n;
    const TA* t0 = reinterpret_cast<const TA*>(rowsum_smem) + (size_t)kWarps * NBUF * BUF;
    for (int e = threadIdx.x; e < n; e += kThreads) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) t += (double)t0[(size_t)w * n + e];
      out[e] = t;
    }
  }
}

// The same pass with the rows staged in registers instead of shared memory:
// STEP loads per lane for the next step are issued before the current step is
// walked.  Shared memory then carries only the small-FE table traffic (two
// wavefronts per row instead of four), at the price of 2 x STEP registers.
template <typename TA, int C, bool W, int NS>
__global__ void __launch_bounds__(kThreads, sizeof(TA) == 4 ? 3 : 2)
k_rowsum_reg(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items,
             const TA* __restrict__ src, RowSumArgs rs) {
  static_assert(C == 32, "the walk puts one column on each lane");
  constexpr int STEP = sizeof(TA) == 4 ? 16 : 8;
  __shared__ double smt[kWarps][32];
  extern __shared__ __align__(16) unsigned char rowsum_smem[];
  if (d.active && *d.active == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  TA* tbl = reinterpret_cast<TA*>(rowsum_smem) + (size_t)wib * rs.small_rows * C;
  for (int e = lane; e < rs.small_rows * C; e += 32) tbl[e] = TA(0);
  __syncwarp();
  const int kp = d.primary;
  TA* __restrict__ Sf = reinterpret_cast<TA*>(rs.sum) + d.lev_base[kp] * C + lane;
  const int32_t* __restrict__ refp = d.refs[kp];
  const TA* __restrict__ cwp = cw_of<TA>(d, kp);
  const int32_t* __restrict__ ref0 = NS > 0 ? d.refs[rs.small_fe[0]] : nullptr;
  const int32_t* __restrict__ ref1 = NS > 1 ? d.refs[rs.small_fe[1]] : nullptr;
  const TA* __restrict__ cw0 = NS > 0 ? cw_of<TA>(d, rs.small_fe[0]) : nullptr;
  const TA* __restrict__ cw1 = NS > 1 ? cw_of<TA>(d, rs.small_fe[1]) : nullptr;
  const int off0 = rs.small_off[0], off1 = rs.small_off[1];
  const int64_t wstride = (int64_t)gridDim.x * kWarps;
  for (int64_t wi = (int64_t)blockIdx.x * kWarps + wib; wi < n_items; wi += wstride) {
    const ExpandItem it = items[wi];
    const int64_t ie = it.ie;
    if (ie <= it.ib) continue;
    TA xn[STEP];
    int kpr_n = kSentinel, k0_n = 0, k1_n = 0;
    TA cp_n = TA(1), c0_n = TA(1), c1_n = TA(1);
    auto fetch = [&](int64_t base) {
      const int64_t left = ie - base;
      const int nv = (int)(left < STEP ? left : STEP);
      const TA* __restrict__ row = src + base * C + lane;
#pragma unroll
      for (int r = 0; r < STEP; ++r) xn[r] = r < nv ? __ldcs(row + (int64_t)r * C) : TA(0);
      const int64_t p = base + lane;
      const bool ok = lane < nv;
      kpr_n = ok ? __ldg(refp + p) : kSentinel;
      if (W) cp_n = (ok && cwp) ? __ldg(cwp + p) : TA(1);
      if (NS > 0) {
        k0_n = ok ? off0 + __ldg(ref0 + p) : 0;
        if (W) c0_n = (ok && cw0) ? __ldg(cw0 + p) : TA(1);
      }
      if (NS > 1) {
        k1_n = ok ? off1 + __ldg(ref1 + p) : 0;
        if (W) c1_n = (ok && cw1) ? __ldg(cw1 + p) : TA(1);
      }
    };
    fetch(it.ib);
    int ckey = -1;  // primary level of the open run (warp-uniform)
    TA acc = TA(0);
    for (int64_t base = it.ib; base < ie; base += STEP) {
      TA x[STEP];
#pragma unroll
      for (int r = 0; r < STEP; ++r) x[r] = xn[r];
      const int kpr = kpr_n, k0 = k0_n, k1 = k1_n;
      const TA cpv = cp_n, c0 = c0_n, c1 = c1_n;
      const int nvalid = (int)((ie - base) < STEP ? (ie - base) : STEP);
      if (base + STEP < ie) fetch(base + STEP);
      const int kn = __shfl_down_sync(FE_FULL, kpr, 1);
      const uint32_t bmask = __ballot_sync(FE_FULL, lane + 1 < nvalid && kn != kpr);
      const int kfirst = __shfl_sync(FE_FULL, kpr, 0);
      if (ckey >= 0 && ckey != kfirst) {
        Sf[(int64_t)ckey * C] = acc;
        acc = TA(0);
      }
      if (nvalid == STEP) {
        rowsum_full_step<TA, C, W, NS, STEP>(x, acc, bmask, kpr, cpv, k0, c0, k1, c1, Sf, tbl,
                                             lane);
      } else {
#pragma unroll
        for (int r = 0; r < STEP; ++r)
          if (r < nvalid)  // warp-uniform
            rowsum_row<TA, C, W, NS>(r, x[r], acc, bmask, kpr, cpv, k0, c0, k1, c1, Sf, tbl, lane);
      }
      ckey = __shfl_sync(FE_FULL, kpr, nvalid - 1);
    }
    SegRun<TA, 1, 32, 1> run;
    run.ckey = ckey;
    run.carry.v[0] = acc;
    run.acc.v[0] = TA(0);
    run.pend = false;
    run.finish(it.split, it.piece, rs.sa, 0, lane, C, Sf, smt[wib]);
  }
  if (NS > 0) {
    __syncthreads();
    const int n = rs.small_rows * C;
    double* __restrict__ out = rs.small_part + (int64_t)blockIdx.x * n;
    const TA* t0 = reinterpret_cast<const TA*>(rowsum_smem);
    for (int e = threadIdx.x; e < n; e += kThreads) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) t += (double)t0[(size_t)w * n + e];
      out[e] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// k_demean: the projection of the absorbed-primary mode.  With the primary FE
// (whose levels are contiguous row segments, the observations being sorted by
// it) projected out of the least-squares problem, the solver works with
// M u = u - a_l (a_l' u) per primary level l, where a_l holds cw_i * scale_l on
// the rows of level l (a unit vector).  From rows `in` to rows `rows` ([N][32]
// of T; the same buffer for the in-place projection, every element being read
// before the same thread stores it):
//   pass 1 of an item: z_l = sum_{i in l} cw_i u_i per level -> sum slab
//                      (the primary FE's rows of the [P][C] slab, free here);
//   pass 2:            u_i -= cw_i scale_l^2 z_l, ||u||^2 per column into the
//                      norm slot of the CTA, the small FEs' sums of cw u into
//                      the per-warp tables (as k_rowsum), optional FP32 copy.
// Items are whole primary levels (dm list), short enough that the second
// read of an item's rows hits L1/L2.  Lane = column, STEP rows per step held
// in registers.  The only cross-lane dependency is the z row of a level,
// written by all lanes in pass 1 and read in pass 2 after a __syncwarp.
//
// NG > 0, the refinement's residual form: the rows are w = in - A_r x, with
// `in` the right-hand side B and x given by the pre-scaled table xs
// ([P][C], scale_l * x_l), the NG = K - 1 non-primary FEs gathered in FE
// order (one coalesced row per FE and row, an L2 hit), the same sums as the
// separate residual kernel; columns whose refinement has stopped
// (inst[j].outer_active == 0) project their stored rows instead.
// ---------------------------------------------------------------------------
template <typename T, int C, bool W, int NS, int NG = 0>
__global__ void __launch_bounds__(kThreads, 2)
k_demean(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items, const T* in,
         T* rows, float* __restrict__ rows32, RowSumArgs rs, double* __restrict__ part,
         int64_t S, const T* __restrict__ xs, const Inst* __restrict__ inst) {
  static_assert(C == 32, "one column per lane");
  constexpr int STEP = sizeof(T) == 4 ? 16 : 8;
  constexpr int RC = (int)kDemeanRows;  // rows of an item held in registers
  static_assert(RC == 32, "one item row per lane for the keys");
  __shared__ double sm[kWarps][32];
  extern __shared__ __align__(16) unsigned char demean_smem[];
  if (d.active_pre && *d.active_pre == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  // per warp: RC z rows (levels of a short item), then the small-FE table
  T* zs = reinterpret_cast<T*>(demean_smem) + (size_t)wib * (RC + rs.small_rows) * C;
  T* tbl = zs + RC * C;
  for (int e = lane; e < rs.small_rows * C; e += 32) tbl[e] = T(0);
  __syncwarp();
  const int kp = d.primary;
  T* __restrict__ Z = reinterpret_cast<T*>(rs.sum) + d.lev_base[kp] * C + lane;
  const int32_t* __restrict__ refp = d.refs[kp];
  const T* __restrict__ cwp = cw_of<T>(d, kp);
  const T* __restrict__ scp = scale_of<T>(d, kp);
  const int32_t* __restrict__ ref0 = NS > 0 ? d.refs[rs.small_fe[0]] : nullptr;
  const int32_t* __restrict__ ref1 = NS > 1 ? d.refs[rs.small_fe[1]] : nullptr;
  const T* __restrict__ cw0 = NS > 0 ? cw_of<T>(d, rs.small_fe[0]) : nullptr;
  const T* __restrict__ cw1 = NS > 1 ? cw_of<T>(d, rs.small_fe[1]) : nullptr;
  const int off0 = rs.small_off[0], off1 = rs.small_off[1];
  // residual form: the gathered FEs (every FE but the primary, in FE order),
  // and whether this lane's column is still refined
  const int32_t* __restrict__ gref[NG > 0 ? NG : 1];
  const T* __restrict__ gcw[NG > 0 ? NG : 1];
  const T* __restrict__ gtab[NG > 0 ? NG : 1];
  bool ract = true;
  if (NG > 0) {
    int j = 0;
    for (int k = 0; k < d.K && j < NG; ++k) {
      if (k == kp) continue;
      gref[j] = d.refs[k];
      gcw[j] = cw_of<T>(d, k);
      gtab[j] = xs + d.lev_base[k] * C + lane;
      ++j;
    }
    ract = inst[lane].outer_active != 0;
  }
  // row p of w into registers: (B - A_r x) for refined columns, the stored row
  // otherwise; ref/cw: the gathered FEs' refs and weights of row p
  auto w_row = [&](int64_t p, const int (&ref)[NG > 0 ? NG : 1], const T (&cw)[NG > 0 ? NG : 1]) {
    if (NG == 0) return in[p * C + lane];
    T acc = T(0);
    if (ract) {
#pragma unroll
      for (int j = 0; j < NG; ++j) {
        const T t = gtab[j][(int64_t)ref[j] * C];
        acc += gcw[j] ? cw[j] * t : t;
      }
      return in[p * C + lane] - acc;
    }
    return rows[p * C + lane];
  };
  double nrm = 0.0;
  const int64_t wstride = (int64_t)gridDim.x * kWarps;
  for (int64_t wi = (int64_t)blockIdx.x * kWarps + wib; wi < n_items; wi += wstride) {
    const ExpandItem it = items[wi];
    const int64_t ie = it.ie;
    if (ie <= it.ib) continue;
    if (ie - it.ib <= RC) {
      // ---- short item: rows in registers, z rows in shared memory ----
      const int n = (int)(ie - it.ib);
      const bool okl = lane < n;
      const int64_t p = it.ib + lane;
      const int kpr = okl ? __ldg(refp + p) : kSentinel;
      const T cwv = (W && okl && cwp) ? __ldg(cwp + p) : T(1);
      T f = T(0);  // cw_i scale_l^2 of row ib + lane
      if (okl) {
        const T sl = __ldg(scp + kpr);
        f = sl * sl * cwv;
      }
      int k0 = 0, k1 = 0;
      T c0 = T(1), c1 = T(1);
      if (NS > 0 && okl) {
        k0 = off0 + __ldg(ref0 + p);
        if (W && cw0) c0 = __ldg(cw0 + p);
      }
      if (NS > 1 && okl) {
        k1 = off1 + __ldg(ref1 + p);
        if (W && cw1) c1 = __ldg(cw1 + p);
      }
      T x[RC];
      {
        // the rows (residual form: the right-hand side, or the stored row of
        // a stopped column)
        const T* src = (NG > 0 && !ract ? rows : in) + it.ib * C + lane;
#pragma unroll
        for (int r = 0; r < RC; ++r) x[r] = r < n ? src[(int64_t)r * C] : T(0);
      }
      if (NG > 0) {
        // minus A_r x, GB rows at a time: the gathers of a group are
        // unconditional (padding rows read level 0), so they are in flight
        // together; the sums are the residual kernel's, in FE order
        int grl[NG > 0 ? NG : 1];
        T gcl[NG > 0 ? NG : 1];
#pragma unroll
        for (int j = 0; j < NG; ++j) {
          grl[j] = okl ? __ldg(gref[j] + p) : 0;
          gcl[j] = (okl && gcw[j]) ? __ldg(gcw[j] + p) : T(1);
        }
        constexpr int GB = (NG <= 2 && !W) ? 8 : 4;  // rows gathered together (no spills)
#pragma unroll
        for (int r0 = 0; r0 < RC; r0 += GB) {
          if (r0 < n) {  // warp-uniform
            T t[GB];
#pragma unroll
            for (int q = 0; q < GB; ++q) {
              t[q] = T(0);
#pragma unroll
              for (int j = 0; j < NG; ++j) {
                const int ref = __shfl_sync(FE_FULL, grl[j], r0 + q);
                const T cr = __shfl_sync(FE_FULL, gcl[j], r0 + q);
                const T v = gtab[j][(int64_t)ref * C];
                t[q] += gcw[j] ? cr * v : v;
              }
            }
#pragma unroll
            for (int q = 0; q < GB; ++q)
              if (ract && r0 + q < n) x[r0 + q] -= t[q];
          }
        }
      }
      const int kn = __shfl_down_sync(FE_FULL, kpr, 1);
      // level ends after row r: a key change, or the item's last row
      const uint32_t ends = __ballot_sync(FE_FULL, okl && (lane + 1 == n || kn != kpr));
      // pass 1: z of each level of the item, in level order
      T acc = T(0);
      int li = 0;
#pragma unroll
      for (int r = 0; r < RC; ++r) {
        if (r < n) {  // warp-uniform
          acc += W ? x[r] * __shfl_sync(FE_FULL, cwv, r) : x[r];
          if ((ends >> r) & 1u) {
            zs[li * C + lane] = acc;
            acc = T(0);
            ++li;
          }
        }
      }
      __syncwarp();
      // pass 2: u -= cw scale^2 z, stored, ||u||^2; padded rows stay 0
      T* dst = rows + it.ib * C + lane;
      li = 0;
#pragma unroll
      for (int r = 0; r < RC; ++r) {
        if (r < n) {
          const T u = x[r] - __shfl_sync(FE_FULL, f, r) * zs[li * C + lane];
          dst[(int64_t)r * C] = u;
          if (rows32) rows32[(it.ib + r) * C + lane] = (float)u;
          nrm += (double)u * (double)u;
          x[r] = u;
          if ((ends >> r) & 1u) ++li;
        }
      }
      __syncwarp();  // zs is rewritten by the next item
      // small FEs: tables += cw u, 4 rows at a time (padded rows add 0)
      if (NS > 0) {
#pragma unroll
        for (int r0 = 0; r0 < RC; r0 += 4) {
          if (r0 < n) {
            rowsum_small4<T, C, W>(r0, x[r0], x[r0 + 1], x[r0 + 2], x[r0 + 3], k0, c0, tbl, lane);
            if (NS > 1)
              rowsum_small4<T, C, W>(r0, x[r0], x[r0 + 1], x[r0 + 2], x[r0 + 3], k1, c1, tbl, lane);
          }
        }
      }
      continue;
    }
    // ---- long item (one level longer than RC rows): two passes over memory ----
    // pass 1: z_l = sum cw u over the level
    int ckey = -1;
    T acc = T(0);
    for (int64_t base = it.ib; base < ie; base += STEP) {
      const int nvalid = (int)((ie - base) < STEP ? (ie - base) : STEP);
      const bool okl = lane < nvalid;
      const int kpr = okl ? __ldg(refp + base + lane) : kSentinel;
      const T cpv = (W && okl && cwp) ? __ldg(cwp + base + lane) : T(1);
      int grl[NG > 0 ? NG : 1];
      T gcl[NG > 0 ? NG : 1];
#pragma unroll
      for (int j = 0; j < NG; ++j) {
        grl[j] = okl ? __ldg(gref[j] + base + lane) : 0;
        gcl[j] = (okl && gcw[j]) ? __ldg(gcw[j] + base + lane) : T(1);
      }
      T x[STEP];
#pragma unroll
      for (int r = 0; r < STEP; ++r) {
        int rr[NG > 0 ? NG : 1];
        T cr[NG > 0 ? NG : 1];
#pragma unroll
        for (int j = 0; j < NG; ++j) {
          rr[j] = __shfl_sync(FE_FULL, grl[j], r);
          cr[j] = __shfl_sync(FE_FULL, gcl[j], r);
        }
        x[r] = r < nvalid ? w_row(base + r, rr, cr) : T(0);
      }
      const int kn = __shfl_down_sync(FE_FULL, kpr, 1);
      const uint32_t bmask = __ballot_sync(FE_FULL, lane + 1 < nvalid && kn != kpr);
      const int kfirst = __shfl_sync(FE_FULL, kpr, 0);
      if (ckey >= 0 && ckey != kfirst) {
        Z[(int64_t)ckey * C] = acc;
        acc = T(0);
      }
#pragma unroll
      for (int r = 0; r < STEP; ++r)
        if (r < nvalid) rowsum_primary<T, C, W>(r, x[r], acc, bmask, kpr, cpv, Z);
      ckey = __shfl_sync(FE_FULL, kpr, nvalid - 1);
    }
    if (ckey >= 0) Z[(int64_t)ckey * C] = acc;  // items hold whole levels
    __syncwarp();  // z rows written by every lane are visible to every lane
    // pass 2: u -= cw scale^2 z, norms, small-FE sums, FP32 copy
    for (int64_t base = it.ib; base < ie; base += STEP) {
      const int nvalid = (int)((ie - base) < STEP ? (ie - base) : STEP);
      const bool okl = lane < nvalid;
      const int64_t p = base + lane;
      const int kpr = okl ? __ldg(refp + p) : 0;
      T f = T(0);  // cw_i scale_l^2 of row base + lane
      if (okl) {
        const T sl = __ldg(scp + kpr);
        f = sl * sl * ((W && cwp) ? __ldg(cwp + p) : T(1));
      }
      int k0 = 0, k1 = 0;
      T c0 = T(1), c1 = T(1);
      if (NS > 0 && okl) {
        k0 = off0 + __ldg(ref0 + p);
        if (W && cw0) c0 = __ldg(cw0 + p);
      }
      if (NS > 1 && okl) {
        k1 = off1 + __ldg(ref1 + p);
        if (W && cw1) c1 = __ldg(cw1 + p);
      }
      int grl[NG > 0 ? NG : 1];
      T gcl[NG > 0 ? NG : 1];
#pragma unroll
      for (int j = 0; j < NG; ++j) {
        grl[j] = okl ? __ldg(gref[j] + p) : 0;
        gcl[j] = (okl && gcw[j]) ? __ldg(gcw[j] + p) : T(1);
      }
      T x[STEP];
#pragma unroll
      for (int r = 0; r < STEP; ++r) {
        if (r < nvalid) {
          const int kr = __shfl_sync(FE_FULL, kpr, r);
          const T fr = __shfl_sync(FE_FULL, f, r);
          const int64_t o = (base + r) * C + lane;
          int rr[NG > 0 ? NG : 1];
          T cr[NG > 0 ? NG : 1];
#pragma unroll
          for (int j = 0; j < NG; ++j) {
            rr[j] = __shfl_sync(FE_FULL, grl[j], r);
            cr[j] = __shfl_sync(FE_FULL, gcl[j], r);
          }
          const T u = w_row(base + r, rr, cr) - fr * Z[(int64_t)kr * C];
          rows[o] = u;
          if (rows32) rows32[o] = (float)u;
          nrm += (double)u * (double)u;
          x[r] = u;
        } else {
          x[r] = T(0);
        }
      }
      if (NS > 0) {
#pragma unroll
        for (int r0 = 0; r0 < STEP; r0 += 4) {
          if (r0 < nvalid) {
            rowsum_small4<T, C, W>(r0, x[r0], x[r0 + 1], x[r0 + 2], x[r0 + 3], k0, c0, tbl, lane);
            if (NS > 1)
              rowsum_small4<T, C, W>(r0, x[r0], x[r0 + 1], x[r0 + 2], x[r0 + 3], k1, c1, tbl, lane);
          }
        }
      }
    }
  }
  // ||u||^2: warp -> CTA slot (fixed order); slots beyond the grid hold 0
  sm[wib][lane] = nrm;
  __syncthreads();
  if (part != nullptr && threadIdx.x < C) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) t += sm[w][threadIdx.x];
    part[(int64_t)threadIdx.x * S + blockIdx.x] = t;
    for (int64_t sl = (int64_t)blockIdx.x + gridDim.x; sl < S; sl += gridDim.x)
      part[(int64_t)threadIdx.x * S + sl] = 0.0;
  }
  if (NS > 0) {
    const int n = rs.small_rows * C;
    double* __restrict__ out = rs.small_part + (int64_t)blockIdx.x * n;
    const T* t0 = reinterpret_cast<const T*>(demean_smem) + (size_t)kDemeanRows * C;
    const size_t wstep = (size_t)(kDemeanRows + rs.small_rows) * C;
    for (int e = threadIdx.x; e < n; e += kThreads) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) t += (double)t0[(size_t)w * wstep + e];
      out[e] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// k_demean_narrow: the projection of the absorbed-primary mode (as k_demean)
// for tiles of C < 32 columns.  One warp per demean item.  An item's rows are
// contiguous C-element rows, so its element e = lane + 32 k lies in row e / C
// and column e % C = lane % C (32 is a multiple of C): every lane keeps one
// column.  A short item (at most kDemeanRows rows) is read in KC chunks of 32
// elements; in each chunk the level sums of cw x are scanned over the rows of
// each column (lanes C apart; the levels are contiguous rows, so a lane adds
// the partial d rows back only within its own level), the open level's partial
// carries into the next chunk, and each level's total is kept at its last row
// in shared memory; then u = x - cw scale_l^2 z_l.  A long item (one level) is
// summed per lane and reduced over the lanes of each column, then projected
// in a second pass over memory.  ||u||^2 per column goes to the CTA's norm
// slot.  `in` is the source (== rows for the in-place projection); rows
// (optional) and rows32 (optional FP32 copy) receive u.
// BATCH = false: the CTAs walk all items grid-stride (one problem).  BATCH
// (batch plans): CTA b takes items [b ipc, (b+1) ipc), all of one problem, and
// skips the items of a problem none of whose columns is active (act_mode 1:
// the inner loop's flag, 2: the refinement's); its rows are left as they are.
// (A compile-time switch: the batch walk costs the single-problem form
// registers, 64 -> 116 for FP64 8-column tiles.)
// ---------------------------------------------------------------------------
template <typename T, int C, bool W, bool BATCH = false>
__global__ void __launch_bounds__(kThreads)
k_demean_narrow(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items,
                const T* in, T* rows, float* __restrict__ rows32, double* __restrict__ part,
                int64_t S, int64_t ipc, const Inst* __restrict__ inst, int act_mode) {
  static_assert(C < 32 && 32 % C == 0, "tiles narrower than a warp");
  constexpr int RC = (int)kDemeanRows;
  static_assert(RC == 32, "one item row per lane for the keys");
  constexpr int KC = RC * C / 32;  // chunks of 32 elements in a short item
  constexpr int RPC = 32 / C;      // rows per chunk
  // FP32 with C >= 4 (TASKS): the item's rows, their weights and the level
  // sums z in shared memory; each lane sums the rows of one (level, column)
  // pair (measured at 8 columns: 2.69 -> 2.13 ms per launch on 100M rows).
  // Otherwise z from per-column segmented scans over the lanes (at 1 column
  // the pairs are too few to occupy the warp: 93 us against 115 us).
  constexpr bool TASKS = sizeof(T) == 4 && C >= 4;
  constexpr int WSH = TASKS ? 2 * RC * C + RC : RC * C;  // elements per warp
  __shared__ T wsh[kWarps][WSH];
  __shared__ int lends[kWarps][TASKS ? RC : 1];  // last row of each level
  __shared__ double sm[kWarps][32];
  if (d.active_pre && *d.active_pre == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int col = lane % C;
  const int kp = d.primary;
  const int32_t* __restrict__ refp = d.refs[kp];
  const T* __restrict__ cwp = cw_of<T>(d, kp);
  const T* __restrict__ scp = scale_of<T>(d, kp);
  T* zb = wsh[wib];                          // z (level, column)
  T* bx = TASKS ? wsh[wib] + RC * C : nullptr;   // staged rows
  T* cws = TASKS ? wsh[wib] + 2 * RC * C : nullptr;  // staged row weights
  double nrm = 0.0;
  // Items are walked with the next one's loads in flight: its descriptor,
  // row keys, weights and scales, and (at most 32 bytes per lane, where the
  // registers do not cost occupancy) its rows.
  constexpr bool PFX = KC * (int)sizeof(T) <= 32;
  struct Pre {
    int64_t ib, ne;  // first row; rows (0: none)
    int kpr;
    T cwv, sl;
    T x[PFX ? KC : 1];
  };
  const int64_t wstride = BATCH ? (int64_t)kWarps : (int64_t)gridDim.x * kWarps;
  int64_t wi = BATCH ? (int64_t)blockIdx.x * ipc + wib : (int64_t)blockIdx.x * kWarps + wib;
  const int64_t cta_end = ((int64_t)blockIdx.x + 1) * ipc;
  const int64_t wend = (BATCH && cta_end < n_items) ? cta_end : n_items;
  auto fetch = [&](int64_t wi, Pre& p) {
    p.ib = 0;
    p.ne = 0;
    p.kpr = kSentinel;
    p.cwv = T(1);
    p.sl = T(0);
    if (wi >= wend) return;
    const ExpandItem it = items[wi];
    p.ib = it.ib;
    p.ne = it.ie > it.ib ? it.ie - it.ib : 0;
    if (BATCH && p.ne > 0) {
      const Inst& s = inst[(int64_t)it.prob * C + col];
      if (!__any_sync(FE_FULL, (act_mode == 1 ? s.active : s.outer_active) != 0)) p.ne = 0;
    }
    if (p.ne == 0 || p.ne > RC) return;
    const int n = (int)p.ne;
    if (lane < n) {
      p.kpr = __ldg(refp + p.ib + lane);
      if (W && cwp) p.cwv = __ldg(cwp + p.ib + lane);
      p.sl = __ldg(scp + p.kpr);
    }
    if constexpr (PFX) {
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int e = lane + 32 * k;
        p.x[k] = e < n * C ? in[p.ib * C + e] : T(0);
      }
    }
  };
  Pre cur, nxt;
  fetch(wi, cur);
  for (; wi < wend; wi += wstride) {
    fetch(wi + wstride, nxt);
    const int64_t ib = cur.ib;
    const int64_t ne = cur.ne;
    if (ne == 0) {
      cur = nxt;
      continue;
    }
    if (ne <= RC) {
      const int n = (int)ne;
      const bool okl = lane < n;
      const int kpr = cur.kpr;
      const T cwv = cur.cwv;
      const T f = okl ? cur.sl * cur.sl * cwv : T(0);  // cw scale^2 of row `lane`
      const int kn = __shfl_down_sync(FE_FULL, kpr, 1);
      // level ends after row r: a key change, or the item's last row
      const uint32_t ends = __ballot_sync(FE_FULL, okl && (lane + 1 == n || kn != kpr));
      T x[KC];
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        if constexpr (PFX) {
          x[k] = cur.x[k];
        } else {
          const int e = lane + 32 * k;
          x[k] = e < n * C ? in[ib * C + e] : T(0);
        }
      }
      if constexpr (TASKS) {
        // level sums: lane t takes (level t / C, column t % C) and sums the
        // level's rows of its column in row order
#pragma unroll
        for (int k = 0; k < KC; ++k) bx[lane + 32 * k] = x[k];
        if (W) cws[lane] = cwv;
        const int nlev = __popc(ends);
        if (okl && ((ends >> lane) & 1u)) lends[wib][__popc(ends & ((1u << lane) - 1u))] = lane;
        __syncwarp();
        for (int t = lane; t < nlev * C; t += 32) {
          const int j = t / C, c = t - j * C;
          const int r1 = lends[wib][j];
          T acc = T(0);
          for (int r = j > 0 ? lends[wib][j - 1] + 1 : 0; r <= r1; ++r)
            acc += W ? cws[r] * bx[r * C + c] : bx[r * C + c];
          zb[j * C + c] = acc;
        }
      }
      T carry = T(0);   // the partial of the level open at the previous chunk's end
      int carry_lv = -1;
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        if (TASKS || RPC * k >= n) break;  // warp-uniform
        const int r = (lane + 32 * k) / C;
        const int lv = __popc(ends & ((1u << r) - 1u));
        const T cr = W ? __shfl_sync(FE_FULL, cwv, r) : T(1);
        T v = W ? cr * x[k] : x[k];
#pragma unroll
        for (int dd = C; dd < 32; dd <<= 1) {
          const T o = __shfl_up_sync(FE_FULL, v, dd);
          const int lo = __shfl_up_sync(FE_FULL, lv, dd);
          if (lane >= dd && lo == lv) v += o;
        }
        if (lv == carry_lv) v += carry;
        if (r < n && ((ends >> r) & 1u)) zb[lv * C + col] = v;
        carry = __shfl_sync(FE_FULL, v, 32 - C + col);
        carry_lv = __shfl_sync(FE_FULL, lv, 32 - C + col);
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int e = lane + 32 * k;
        const int r = e / C;  // < 32
        const T fr = __shfl_sync(FE_FULL, f, r);
        if (e < n * C) {
          const int lv = __popc(ends & ((1u << r) - 1u));
          const T u = x[k] - fr * zb[lv * C + col];
          if (rows) rows[ib * C + e] = u;
          if (rows32) rows32[ib * C + e] = (float)u;
          nrm += (double)u * (double)u;
        }
      }
      __syncwarp();  // zb is rewritten by the next item
      cur = nxt;
      continue;
    }
    // one level longer than RC rows: z per column over the whole level
    const T sl = __ldg(scp + __ldg(refp + ib));
    const int64_t nel = ne * C;
    T acc = T(0);
    for (int64_t e = lane; e < nel; e += 32) {
      const T v = in[ib * C + e];
      acc += (W && cwp) ? __ldg(cwp + ib + e / C) * v : v;
    }
#pragma unroll
    for (int o = C; o < 32; o <<= 1) acc += __shfl_xor_sync(FE_FULL, acc, o);
    for (int64_t e = lane; e < nel; e += 32) {
      const T cr = (W && cwp) ? __ldg(cwp + ib + e / C) : T(1);
      const T u = in[ib * C + e] - sl * sl * cr * acc;
      if (rows) rows[ib * C + e] = u;
      if (rows32) rows32[ib * C + e] = (float)u;
      nrm += (double)u * (double)u;
    }
    cur = nxt;
  }
  // ||u||^2 per column: the lanes of a column, then warps in order -> the
  // CTA's slot (slots beyond the grid hold 0)
#pragma unroll
  for (int o = C; o < 32; o <<= 1) nrm += __shfl_xor_sync(FE_FULL, nrm, o);
  if (lane < C) sm[wib][lane] = nrm;
  __syncthreads();
  if (part != nullptr && threadIdx.x < C) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) t += sm[w][threadIdx.x];
    part[(int64_t)threadIdx.x * S + blockIdx.x] = t;
    for (int64_t sl = (int64_t)blockIdx.x + gridDim.x; sl < S; sl += gridDim.x)
      part[(int64_t)threadIdx.x * S + sl] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// k_expand_demean: the expand and the demean of the absorbed-primary mode in
// one pass over the rows (32-column tiles).  Per demean item (whole primary
// levels, at most kDemeanRows rows):
//   phase A: the new rows without the primary FE, in the expand's lane layout
//            (Shape<T, 32>):  LSMR   w = av * (A_r v) + au * u_old
//                             RESID  w = b - A_r x            (FP64)
//            staged in a per-warp shared buffer;
//   phase B: B1 the level sums z_l = sum cw w (vector layout); B2
//            u = w - cw scale_l^2 z_l stored once (LSMR: u in place; RESID:
//            the FP64 residual and its FP32 copy) and ||u||^2 per column
//            into the CTA's norm slot; B3 the small FEs' sums of cw u into
//            the per-warp tables, one column per lane (as k_rowsum).
// A level longer than kDemeanRows rows is processed in chunks: phase A writes
// w to the row buffer and accumulates z, then a second walk finalizes it.
// RESID, mask: columns whose refinement has stopped keep their stored rows.
// PRE: tab holds scale_l * v_l (the P-side update stores that copy), so phase
// A skips the per-row load of the scale.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

template <typename T, int VEC>
struct ExDmCoef {
  T av[VEC], au[VEC];
  bool act[VEC];  // the column's rows may be written
};

template <typename T, int C, int U, int KB, bool RESID, bool W, int NS, class Tab, bool PRE>
__global__ void __launch_bounds__(kThreads, 2)
k_expand_demean(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items, Tab tab,
                T* __restrict__ rows, const double* __restrict__ B, float* __restrict__ rows32,
                const Inst* __restrict__ inst, int mask, RowSumArgs rs,
                double* __restrict__ part, int64_t S) {
  static_assert(C == 32, "one column per lane in phase B");
  using Sh = Shape<T, C>;
  constexpr int VEC = Sh::VEC, CL = Sh::CL, G = Sh::G;
  constexpr int STEP = G * U;
  constexpr int RC = (int)kDemeanRows;
  static_assert(STEP <= 32 && RC % STEP == 0, "steps tile an item's row buffer");
  __shared__ double sm[kWarps][32];
  extern __shared__ __align__(16) unsigned char exdm_smem[];
  if (d.active_pre && *d.active_pre == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane / CL, jl = lane - g * CL;
  // per warp: staged rows, level sums, small-FE table, end row of each level
  const size_t wstride_smem = (size_t)(2 * RC + rs.small_rows) * C + 32 * sizeof(int) / sizeof(T);
  T* ub = reinterpret_cast<T*>(exdm_smem) + (size_t)wib * wstride_smem;  // staged rows
  T* zs = ub + RC * C;                                                   // level sums
  T* tbl = zs + RC * C;                                                  // small-FE table
  int* lend = reinterpret_cast<int*>(tbl + rs.small_rows * C);           // last row of level j
  for (int e = lane; e < rs.small_rows * C; e += 32) tbl[e] = T(0);
  const int K = d.K;
  const int kp = d.primary;
  const int32_t* __restrict__ refp = d.refs[kp];
  const T* __restrict__ cwp = cw_of<T>(d, kp);
  const T* __restrict__ scp = scale_of<T>(d, kp);
  const int32_t* __restrict__ ref0 = NS > 0 ? d.refs[rs.small_fe[0]] : nullptr;
  const int32_t* __restrict__ ref1 = NS > 1 ? d.refs[rs.small_fe[1]] : nullptr;
  const T* __restrict__ cw0 = NS > 0 ? cw_of<T>(d, rs.small_fe[0]) : nullptr;
  const T* __restrict__ cw1 = NS > 1 ? cw_of<T>(d, rs.small_fe[1]) : nullptr;
  const int off0 = rs.small_off[0], off1 = rs.small_off[1];
  // per-column coefficients (phase A, lane group layout) and activity (phase B)
  ExDmCoef<T, VEC> cf;
  bool act_any = false;
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    const Inst& st = inst[jl * VEC + v];
    cf.av[v] = (T)st.ex_av;
    cf.au[v] = (T)st.ex_au;
    cf.act[v] = RESID ? (mask != 2 || st.outer_active != 0) : true;
    act_any = act_any || (RESID ? cf.act[v] : st.active != 0);
  }
  const bool col_act = RESID ? (mask != 2 || inst[lane].outer_active != 0) : inst[lane].active != 0;
  act_any = __any_sync(FE_FULL, act_any);
  double nrm = 0.0;      // ||u||^2 of column `lane` (long levels)
  double nrmv[VEC];      // ||u||^2 of this lane's VEC columns (short items)
#pragma unroll
  for (int v = 0; v < VEC; ++v) nrmv[v] = 0.0;
  __syncwarp();

  // phase A on rows [cb, cb + cn) (cn <= RC): w rows into ub (and, for a
  // chunk of a long level, into the row buffer)
  auto phase_a = [&](int64_t cb, int cn, bool to_global) {
    // refs and weights of the chunk's rows (row = lane), loaded once
    int rl[KB];
    T cl[KB];
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      const bool ok = k < K && k != kp && lane < cn;
      rl[k] = ok ? __ldg(d.refs[k] + cb + lane) : 0;
      const T* __restrict__ cw = cw_of<T>(d, k < K ? k : 0);
      cl[k] = (ok && cw) ? __ldg(cw + cb + lane) : T(1);
    }
    for (int b0 = 0; b0 < cn; b0 += STEP) {
      const int64_t base = cb + b0;
      VA<T, VEC> old[U];
      VA<T, VEC> sacc[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = b0 + u * G + g;
#pragma unroll
        for (int v = 0; v < VEC; ++v) sacc[u].v[v] = T(0);
        if (r < cn) {
          const int64_t o = (cb + r) * C + jl * VEC;
          if (RESID) {
            const VA<double, VEC> bb = vldg<double, VEC>(B + o);
#pragma unroll
            for (int v = 0; v < VEC; ++v) old[u].v[v] = (T)bb.v[v];
          } else {
            old[u] = vld<T, VEC>(rows + o);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < KB; ++k) {
        if (k < K && k != kp) {
          const T* __restrict__ sc = scale_of<T>(d, k);
          const int64_t lb = d.lev_base[k];
          const bool wk = cw_of<T>(d, k) != nullptr;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int q = u * G + g;
            const int ref = __shfl_sync(FE_FULL, rl[k], b0 + q);
            const T c = wk ? __shfl_sync(FE_FULL, cl[k], b0 + q) : T(1);
            if (b0 + q < cn) {
              const T scl = PRE ? T(1) : __ldg(sc + ref);
              const T cs = wk ? c * scl : scl;
              const VA<T, VEC> t = tab.load((lb + ref) * C + jl * VEC);
#pragma unroll
              for (int v = 0; v < VEC; ++v) sacc[u].v[v] += cs * t.v[v];
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = b0 + u * G + g;
        if (r < cn) {
          VA<T, VEC> w;
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            w.v[v] = RESID ? old[u].v[v] - sacc[u].v[v] : cf.av[v] * sacc[u].v[v] + cf.au[v] * old[u].v[v];
          vst<T, VEC>(ub + r * C + jl * VEC, w);
          if (to_global) {
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              if (cf.act[v]) rows[(cb + r) * C + jl * VEC + v] = w.v[v];
          }
        }
      }
    }
    __syncwarp();
  };
  // per-row data of rows [cb, cb + cn), one row per lane
  struct RowData {
    int kpr, k0, k1;
    T cwv, f, c0, c1;
  };
  auto row_data = [&](int64_t cb, int cn) {
    RowData rd;
    const bool okl = lane < cn;
    const int64_t p = cb + lane;
    rd.kpr = okl ? __ldg(refp + p) : kSentinel;
    rd.cwv = (W && okl && cwp) ? __ldg(cwp + p) : T(1);
    rd.f = T(0);
    if (okl) {
      const T sl = __ldg(scp + rd.kpr);
      rd.f = sl * sl * rd.cwv;
    }
    rd.k0 = 0;
    rd.k1 = 0;
    rd.c0 = T(1);
    rd.c1 = T(1);
    if (NS > 0 && okl) {
      rd.k0 = off0 + __ldg(ref0 + p);
      if (W && cw0) rd.c0 = __ldg(cw0 + p);
    }
    if (NS > 1 && okl) {
      rd.k1 = off1 + __ldg(ref1 + p);
      if (W && cw1) rd.c1 = __ldg(cw1 + p);
    }
    return rd;
  };
  // finalize rows [cb, cb + cn) whose w is in ub: u = w - f z (z of row r's
  // level: zrow(r)), stored, norms, small-FE tables
  auto finalize = [&](int64_t cb, int cn, const RowData& rd, uint32_t ends, bool zs_local, T zlong) {
    int li = 0;
#pragma unroll 8
    for (int r = 0; r < cn; ++r) {
      const T z = zs_local ? zs[li * C + lane] : zlong;
      const T u = ub[r * C + lane] - __shfl_sync(FE_FULL, rd.f, r) * z;
      ub[r * C + lane] = u;
      if (col_act) {
        const int64_t o = (cb + r) * C + lane;
        rows[o] = u;
        if (RESID && rows32) rows32[o] = (float)u;
        nrm += (double)u * (double)u;
      }
      if ((ends >> r) & 1u) ++li;
    }
    if (NS > 0) {
      for (int r0 = 0; r0 < cn; r0 += 4) {
        T x0 = ub[r0 * C + lane];
        T x1 = r0 + 1 < cn ? ub[(r0 + 1) * C + lane] : T(0);
        T x2 = r0 + 2 < cn ? ub[(r0 + 2) * C + lane] : T(0);
        T x3 = r0 + 3 < cn ? ub[(r0 + 3) * C + lane] : T(0);
        rowsum_small4<T, C, W>(r0, x0, x1, x2, x3, rd.k0, rd.c0, tbl, lane);
        if (NS > 1) rowsum_small4<T, C, W>(r0, x0, x1, x2, x3, rd.k1, rd.c1, tbl, lane);
      }
    }
    __syncwarp();  // ub and zs are rewritten next
  };

  const int64_t wstride = (int64_t)gridDim.x * kWarps;
  int64_t wi0 = (int64_t)blockIdx.x * kWarps + wib;
  ExpandItem nxt{};  // descriptor of the warp's next item (loaded one item ahead)
  if (wi0 < n_items) nxt = items[wi0];
  for (int64_t wi = wi0; wi < n_items; wi += wstride) {
    const ExpandItem it = nxt;
    if (wi + wstride < n_items) nxt = items[wi + wstride];
    const int64_t ie = it.ie;
    if (ie <= it.ib || !act_any) continue;
    // the warp's next item: its rows and index lines into L2 while this one
    // is processed
    if (wi + wstride < n_items) {
      const ExpandItem nx = nxt;
      const int64_t nn = nx.ie - nx.ib;
      if (lane < nn && lane < RC) {
        const int64_t o = (nx.ib + lane) * C;
        if (RESID) {
          prefetch_l2(B + o);
          if (C * sizeof(double) > 128) prefetch_l2(B + o + 128 / sizeof(double));
        } else {
          prefetch_l2(rows + o);
          if (C * sizeof(T) > 128) prefetch_l2(rows + o + 128 / sizeof(T));
        }
      }
#pragma unroll
      for (int k = 0; k < KB; ++k)
        if (k < K && lane == k) prefetch_l2(d.refs[k] + nx.ib);
    }
    if (ie - it.ib <= RC) {
      const int n = (int)(ie - it.ib);
      const RowData rd = row_data(it.ib, n);  // loads overlap phase A's
      phase_a(it.ib, n, false);
      const int kn = __shfl_down_sync(FE_FULL, rd.kpr, 1);
      const bool is_end = lane < n && (lane + 1 == n || kn != rd.kpr);
      const uint32_t ends = __ballot_sync(FE_FULL, is_end);
      const int nlev = __popc(ends);
      if (is_end) lend[__popc(ends & ((1u << lane) - 1u))] = lane;
      __syncwarp();
      // B1: level sums, vector layout; row group g sums levels g, g+G, ...
      for (int jb = 0; jb < nlev; jb += G) {
        const int j = jb + g;
        const bool okj = j < nlev;
        const int e = okj ? lend[j] : -1;
        const int st = (okj && j > 0) ? lend[j - 1] + 1 : 0;
        const int len = okj ? e - st + 1 : 0;
        const int maxlen = __reduce_max_sync(FE_FULL, (unsigned)len);
        VA<T, VEC> acc;
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc.v[v] = T(0);
        for (int t = 0; t < maxlen; ++t) {
          const bool ok = t < len;
          const int r = ok ? st + t : 0;
          const T cwr = W ? __shfl_sync(FE_FULL, rd.cwv, r) : T(1);
          if (ok) {
            const VA<T, VEC> w = vld<T, VEC>(ub + r * C + jl * VEC);
#pragma unroll
            for (int v = 0; v < VEC; ++v) acc.v[v] += cwr * w.v[v];
          }
        }
        if (okj) vst<T, VEC>(zs + j * C + jl * VEC, acc);
      }
      __syncwarp();
      // B2: u = w - cw scale^2 z, stored once; norms
      VA<T, VEC> nvi;
#pragma unroll
      for (int v = 0; v < VEC; ++v) nvi.v[v] = T(0);
      for (int t = 0; t * G < n; ++t) {
        const int r = t * G + g;
        const bool ok = r < n;
        const T fr = __shfl_sync(FE_FULL, rd.f, r);
        VA<T, VEC> u;
        if (ok) {
          const int li = __popc(ends & ((1u << r) - 1u));
          const VA<T, VEC> z = vld<T, VEC>(zs + li * C + jl * VEC);
          u = vld<T, VEC>(ub + r * C + jl * VEC);
#pragma unroll
          for (int v = 0; v < VEC; ++v) u.v[v] -= fr * z.v[v];
          const int64_t o = (it.ib + r) * C + jl * VEC;
          if (RESID) {
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              if (cf.act[v]) {
                rows[o + v] = u.v[v];
                if (rows32) rows32[o + v] = (float)u.v[v];
                nvi.v[v] += u.v[v] * u.v[v];
              }
          } else {
            vst<T, VEC>(rows + o, u);
#pragma unroll
            for (int v = 0; v < VEC; ++v) nvi.v[v] += u.v[v] * u.v[v];
          }
          if (NS > 0) vst<T, VEC>(ub + r * C + jl * VEC, u);  // for B3
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) nrmv[v] += (double)nvi.v[v];
      // B3: small-FE sums of cw u, one column per lane: a row's table key is
      // the same in every lane, so rows sharing a key are merged with uniform
      // branches before the table rows are updated
      if (NS > 0) {
        __syncwarp();  // u rows in ub
        for (int r0 = 0; r0 < n; r0 += 4) {
          const T x0 = ub[r0 * C + lane];
          const T x1 = r0 + 1 < n ? ub[(r0 + 1) * C + lane] : T(0);
          const T x2 = r0 + 2 < n ? ub[(r0 + 2) * C + lane] : T(0);
          const T x3 = r0 + 3 < n ? ub[(r0 + 3) * C + lane] : T(0);
          rowsum_small4<T, C, W>(r0, x0, x1, x2, x3, rd.k0, rd.c0, tbl, lane);
          if (NS > 1) rowsum_small4<T, C, W>(r0, x0, x1, x2, x3, rd.k1, rd.c1, tbl, lane);
        }
      }
      __syncwarp();  // ub, zs and lend are rewritten by the next item
      continue;
    }
    // one level longer than RC rows: w through the row buffer, then finalize
    T zl = T(0);
    for (int64_t cb = it.ib; cb < ie; cb += RC) {
      const int cn = (int)((ie - cb) < RC ? (ie - cb) : RC);
      phase_a(cb, cn, true);
      const T cwr = (W && lane < cn && cwp) ? __ldg(cwp + cb + lane) : T(1);
      for (int r = 0; r < cn; ++r) {
        const T w = ub[r * C + lane];
        zl += W ? w * __shfl_sync(FE_FULL, cwr, r) : w;
      }
      __syncwarp();
    }
    for (int64_t cb = it.ib; cb < ie; cb += RC) {
      const int cn = (int)((ie - cb) < RC ? (ie - cb) : RC);
      for (int r = 0; r < cn; ++r) ub[r * C + lane] = rows[(cb + r) * C + lane];
      __syncwarp();
      const RowData rd = row_data(cb, cn);
      finalize(cb, cn, rd, 0u, false, zl);
    }
  }
  // ||u||^2: the vector-layout sums folded into the per-column ones, then
  // warp -> CTA slot (fixed order); slots beyond the grid hold 0
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    double a = nrmv[v];
#pragma unroll
    for (int o = CL; o < 32; o <<= 1) a += __shfl_xor_sync(FE_FULL, a, o);
    if (g == 0) sm[wib][jl * VEC + v] = a;
  }
  __syncwarp();
  nrm += sm[wib][lane];
  __syncwarp();
  sm[wib][lane] = nrm;
  __syncthreads();
  if (part != nullptr && threadIdx.x < C) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) t += sm[w][threadIdx.x];
    part[(int64_t)threadIdx.x * S + blockIdx.x] = t;
    for (int64_t sl = (int64_t)blockIdx.x + gridDim.x; sl < S; sl += gridDim.x)
      part[(int64_t)threadIdx.x * S + sl] = 0.0;
  }
  if (NS > 0) {
    const int n = rs.small_rows * C;
    double* __restrict__ out = rs.small_part + (int64_t)blockIdx.x * n;
    const T* t0 = reinterpret_cast<const T*>(exdm_smem) + (size_t)2 * RC * C;
    for (int e = threadIdx.x; e < n; e += kThreads) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) t += (double)t0[(size_t)w * wstride_smem + e];
      out[e] = t;
    }
  }
}

// Small-FE level sums = the row-sum CTA partials summed in CTA order.  One
// CTA per table row; thread t sums the slots q, q + Q, ... of column t % C
// (Q = kThreads / C groups), and the groups are added in group order.
struct SmallRows {
  int64_t slab_row[kSmallRows];  // [P][C] slab row of each table row
};
template <typename TA, int C>
__global__ void __launch_bounds__(kThreads)
k_small_combine(const double* __restrict__ part, int nparts, int small_rows, SmallRows m,
                TA* __restrict__ out, const int32_t* __restrict__ active) {
  if (active && *active == 0) return;
  constexpr int Q = kThreads / C;
  __shared__ double sm[Q][C];
  const int row = blockIdx.x;
  const int c = threadIdx.x % C, q = threadIdx.x / C;
  double a = 0.0;
  for (int b = q; b < nparts; b += Q) a += __ldcg(part + ((int64_t)b * small_rows + row) * C + c);
  sm[q][c] = a;
  __syncthreads();
  if (threadIdx.x < C) {
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < Q; ++j) t += sm[j][threadIdx.x];
    out[m.slab_row[row] * C + threadIdx.x] = (TA)t;
  }
}

// ---------------------------------------------------------------------------
// Segmented-sum value loaders: the per-position vector summed into a level.
// ---------------------------------------------------------------------------
template <typename TIn, typename TA, int VEC>
struct LoadIn {
  using InType = TIn;
  const TIn* __restrict__ in;
  static constexpr bool kSquareWeight = false;
  static constexpr bool kAsyncable = std::is_same<TIn, TA>::value;  // raw rows can be copied
  __device__ __forceinline__ VA<TA, VEC> load(int64_t off) const {
    const VA<TIn, VEC> a = vld<TIn, VEC>(in + off);
    VA<TA, VEC> r;
#pragma unroll
    for (int v = 0; v < VEC; ++v) r.v[v] = (TA)a.v[v];
    return r;
  }
};
// sum of interaction^2 * w for the Jacobi scale (src/SolverCPU.jl:78-89):
// the per-position weight cw = interaction*sqrt(w) enters squared, the value
// is 1.  C = 1.
struct LoadScaleSq {
  static constexpr bool kSquareWeight = true;
  static constexpr bool kAsyncable = false;
  __device__ __forceinline__ VA<double, 1> load(int64_t) const {
    VA<double, 1> r;
    r.v[0] = 1.0;
    return r;
  }
};

// ---------------------------------------------------------------------------
// k_segsum: one warp per ReduceItem.  Positions are visited in level order,
// G per warp instruction (one per lane group); an inclusive segmented scan
// over the groups (keys are sorted inside an item, so equal keys are
// contiguous) plus a carry across steps yields each level's sum, stored to
// Sout[level] by the group holding the level's last position.  Split pieces
// hand their partial to the last piece of the level.
// ---------------------------------------------------------------------------
template <typename TA, int C, int U, bool PF, class Load>
__global__ void __launch_bounds__(kThreads)
k_segsum(const FeDev d, const ReduceItem* __restrict__ items, int64_t n_items, Load ld,
         TA* __restrict__ Sout, SplitArgs sa) {
  using Sh = Shape<TA, C>;
  constexpr int VEC = Sh::VEC, CL = Sh::CL, G = Sh::G;
  constexpr int STEP = G * U;
  constexpr int NI = STEP >= 32 ? STEP / 32 : 1;
  static_assert(STEP <= 32 || STEP % 32 == 0, "a step's indices fill whole index registers");
  __shared__ double smt[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int g = lane / CL, jl = lane - g * CL;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (w >= n_items) return;
  if (d.active && *d.active == 0) return;
  const ReduceItem it = items[w];
  if (it.pe <= it.pb) return;
  const int k = it.fe;
  const int32_t* __restrict__ perm = d.perm[k];
  const int32_t* __restrict__ key = d.key[k];
  const TA* __restrict__ cwp = cwp_of<TA>(d, k);
  TA* __restrict__ Sk = Sout + d.lev_base[k] * C + jl * VEC;
  SegRun<TA, VEC, CL, G> run;
  run.init();
  // index data of a step (level keys, sorted positions, weights), fetched one
  // step ahead so that the row gathers of a step do not wait for its indices
  int kl[NI], il[NI];
  TA cl[NI];
  auto fetch = [&](int64_t base) {
#pragma unroll
    for (int r = 0; r < NI; ++r) {
      const int64_t p = base + r * 32 + lane;
      const bool ok = p < it.pe && (r * 32 + lane) < STEP;
      kl[r] = ok ? __ldg(key + p) : kSentinel;
      il[r] = ok ? (perm ? __ldg(perm + p) : (int)p) : 0;
      TA c = TA(1);
      if (ok && cwp) c = __ldg(cwp + p);
      if (Load::kSquareWeight) c = c * c;
      cl[r] = c;
    }
  };
  if (PF) fetch(it.pb);
  for (int64_t base = it.pb; base < it.pe; base += STEP) {
    if (!PF) fetch(base);
    VA<TA, VEC> val[U];
    int kk[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = u * G;
      const int src = (q & 31) + g;
      kk[u] = __shfl_sync(FE_FULL, kl[q >> 5], src);
      const int i = __shfl_sync(FE_FULL, il[q >> 5], src);
      const TA c = __shfl_sync(FE_FULL, cl[q >> 5], src);
      if (kk[u] != kSentinel) {
        val[u] = ld.load((int64_t)i * C + jl * VEC);
#pragma unroll
        for (int v = 0; v < VEC; ++v) val[u].v[v] *= c;
      } else {
#pragma unroll
        for (int v = 0; v < VEC; ++v) val[u].v[v] = TA(0);
      }
    }
    if (PF && base + STEP < it.pe) fetch(base + STEP);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t b0 = base + (int64_t)u * G;
      if (b0 >= it.pe) break;  // warp-uniform
      const int nvalid = (int)((it.pe - b0) < G ? (it.pe - b0) : G);
      run.push(kk[u], val[u], nvalid, g, jl, C, Sk);
    }
  }
  run.finish(it.split, it.pad, sa, g, jl, C, Sk, smt[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------------------
// k_segsum_async: the same segmented sum with the level-order row gathers
// moved off the registers.  Each warp keeps an S-stage ring in shared memory;
// step t+S-1 is issued with cp.async (hand-written PTX) while step t is
// consumed, so S-1 steps of row gathers are in flight per warp whatever the
// register count.  Each lane copies exactly the row chunks it later reads
// (group g, column block jl), so a lane's own cp.async.wait_group makes its
// data visible; keys and weights are copied by lane jl = 0 of each group and
// shared through a __syncwarp.
// ---------------------------------------------------------------------------
// shared memory per warp of k_segsum_async.  VF > 0: VF elements per lane
// instead of the default 16 bytes (FP64 32-column tiles take 4: 8 lanes per
// row and 4 rows per warp instruction, as FP32 rows do).
template <typename TA, int C, int U, int S, int VF = 0>
struct AsyncSegLayout {
  using Sh = Shape<TA, C>;
  static constexpr int VEC = VF > 0 ? VF : Sh::VEC;
  static constexpr int G = 32 / (C / VEC);
  static constexpr int STEP = G * U;
  static constexpr int kRowBytes = C * (int)sizeof(TA);
  static constexpr int kStageRows = STEP * kRowBytes;
  static constexpr int kStage = kStageRows + STEP * (4 + (int)sizeof(TA));
  static constexpr int kWarpBytes = S * kStage;
};

template <typename TA, int C, int U, int S, class Load, int VF = 0>
__global__ void __launch_bounds__(kThreads)
k_segsum_async(const FeDev d, const ReduceItem* __restrict__ items, int64_t n_items, Load ld,
               TA* __restrict__ Sout, SplitArgs sa) {
  using L = AsyncSegLayout<TA, C, U, S, VF>;
  constexpr int VEC = L::VEC, CL = C / VEC, G = L::G;
  static_assert(CL * G == 32, "lane groups fill the warp");
  constexpr int STEP = L::STEP;
  constexpr int NI = STEP >= 32 ? STEP / 32 : 1;
  static_assert(STEP <= 32 || STEP % 32 == 0, "a step's indices fill whole index registers");
  constexpr int CHUNK = VEC * (int)sizeof(TA);  // bytes a lane copies per row
  constexpr int CP = CHUNK > 16 ? 16 : CHUNK;   // bytes per cp.async
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ double smt[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane / CL, jl = lane - g * CL;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wib;
  if (w >= n_items) return;
  if (d.active && *d.active == 0) return;
  const ReduceItem it = items[w];
  if (it.pe <= it.pb) return;
  unsigned char* ring = dyn_smem + (size_t)wib * L::kWarpBytes;
  const int k = it.fe;
  const int32_t* __restrict__ perm = d.perm[k];
  const int32_t* __restrict__ key = d.key[k];
  const TA* __restrict__ cwp = cwp_of<TA>(d, k);
  const TA* __restrict__ in = ld.in;
  TA* __restrict__ Sk = Sout + d.lev_base[k] * C + jl * VEC;
  const int64_t nsteps = (it.pe - it.pb + STEP - 1) / STEP;
  // sorted positions of the step to issue next (loaded one step early)
  int il[NI];
  auto load_idx = [&](int64_t step) {
#pragma unroll
    for (int r = 0; r < NI; ++r) {
      const int64_t p = it.pb + step * STEP + r * 32 + lane;
      const bool ok = step < nsteps && p < it.pe && (r * 32 + lane) < STEP;
      il[r] = ok ? (perm ? __ldg(perm + p) : (int)p) : -1;
    }
  };
  auto issue = [&](int64_t step) {
    if (step < nsteps) {
      unsigned char* st = ring + (int)(step % S) * L::kStage;
      int32_t* skey = reinterpret_cast<int32_t*>(st + L::kStageRows);
      TA* scw = reinterpret_cast<TA*>(st + L::kStageRows + STEP * 4);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int q = u * G;
        const int i = __shfl_sync(FE_FULL, il[q >> 5], (q & 31) + g);
        const int row = u * G + g;
        const int64_t p = it.pb + step * STEP + row;
        if (i >= 0) {
#pragma unroll
          for (int q = 0; q < CHUNK / CP; ++q)
            cp_async<CP>(st + row * L::kRowBytes + jl * CHUNK + q * CP,
                         reinterpret_cast<const char*>(in + (int64_t)i * C + jl * VEC) + q * CP);
          if (jl == 0) {
            cp_async_bytes4(skey + row, key + p);
            if (cwp) cp_async<(int)sizeof(TA)>(scw + row, cwp + p);
          }
        }
      }
    }
    cp_async_commit();  // one group per step, empty past the end
  };
  load_idx(0);
#pragma unroll
  for (int t = 0; t < S - 1; ++t) {
    issue(t);
    load_idx(t + 1);
  }
  SegRun<TA, VEC, CL, G> run;
  run.init();
  for (int64_t t = 0; t < nsteps; ++t) {
    issue(t + S - 1);
    load_idx(t + S);
    cp_async_wait<S - 1>();
    __syncwarp();
    const unsigned char* st = ring + (int)(t % S) * L::kStage;
    const int32_t* skey = reinterpret_cast<const int32_t*>(st + L::kStageRows);
    const TA* scw = reinterpret_cast<const TA*>(st + L::kStageRows + STEP * 4);
    const int64_t base = it.pb + t * STEP;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t b0 = base + (int64_t)u * G;
      if (b0 >= it.pe) break;  // warp-uniform
      const int row = u * G + g;
      const bool ok = b0 + g < it.pe;
      const int km = ok ? skey[row] : kSentinel;
      VA<TA, VEC> x;
      if (ok) {
        x = vld<TA, VEC>(reinterpret_cast<const TA*>(st + row * L::kRowBytes + jl * CHUNK));
        const TA c = cwp ? scw[row] : TA(1);
#pragma unroll
        for (int v = 0; v < VEC; ++v) x.v[v] *= c;
      } else {
#pragma unroll
        for (int v = 0; v < VEC; ++v) x.v[v] = TA(0);
      }
      const int nvalid = (int)((it.pe - b0) < G ? (it.pe - b0) : G);
      run.push(km, x, nvalid, g, jl, C, Sk);
    }
    __syncwarp();  // the stage is refilled by the next issue
  }
  cp_async_wait<0>();
  run.finish(it.split, it.pad, sa, g, jl, C, Sk, smt[wib]);
}

// ---------------------------------------------------------------------------
// P-side epilogues: update(k, lrow, o, sum, na, nb) for level lrow of FE k;
// o is the element offset of the lane's first column.
// ---------------------------------------------------------------------------
// LSMR v-update (src/utils/lsmr.jl:108-110) fused with the deferred h/hbar/x
// update of the previous iteration (lsmr.jl:138-142) and the norms ||v||^2,
// ||x||^2.  Columns whose LSMR has stopped are left untouched.  The
// elementwise arithmetic runs in T (the coefficients come from the FP64
// scalar recurrences, rounded once); the norms accumulate in FP64.
template <typename T, int VEC>
struct PEpiLsmr {
  using TS = T;
  using TN = T;  // norm accumulation within an item
  T* __restrict__ V;
  T* __restrict__ H;
  T* __restrict__ Hb;
  T* __restrict__ X;
  T* __restrict__ VS;  // optional: v scaled by the Jacobi scale (the fused loop's table)
  const Inst* __restrict__ inst;
  T rd_acc[VEC], rd_v[VEC], s_v[VEC], c1[VEC], c2[VEC], c3[VEC];
  uint32_t upd_bits;  // 2 bits per column: deferred update mode
  uint32_t v_bits;    // 1 bit per column: v is updated this iteration
  bool act;
  __device__ __forceinline__ void begin(int prob, int jl, int C) {
    act = false;
    upd_bits = 0;
    v_bits = 0;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const Inst& s = inst[(int64_t)prob * C + jl * VEC + v];
      const bool a = s.active != 0;
      rd_acc[v] = (T)s.rd_acc;
      rd_v[v] = (T)s.rd_v;
      s_v[v] = (T)s.s_v;
      c1[v] = (T)s.c1;
      c2[v] = (T)s.c2;
      c3[v] = (T)s.c3;
      if (a) upd_bits |= (uint32_t)(s.upd_mode & 3) << (2 * v);
      if (a && s.do_v) v_bits |= 1u << v;
      act = act || a;
    }
  }
  __device__ __forceinline__ void update(const FeDev& d, int k, int64_t l, int64_t o,
                                         const VA<T, VEC>& sum, TN (&na)[VEC], TN (&nb)[VEC]) {
    VA<T, VEC> vv = vld<T, VEC>(V + o);
    if (upd_bits) {
      VA<T, VEC> hh = vld<T, VEC>(H + o);
      VA<T, VEC> hb = vld<T, VEC>(Hb + o);
      VA<T, VEC> xx = vld<T, VEC>(X + o);
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        const uint32_t m = (upd_bits >> (2 * v)) & 3u;
        const T vo = s_v[v] * vv.v[v];
        if (m == 2) {
          const T h = hh.v[v];
          const T hbn = h + c1[v] * hb.v[v];
          hb.v[v] = hbn;
          xx.v[v] = xx.v[v] + c2[v] * hbn;
          hh.v[v] = vo + c3[v] * h;
        } else if (m != 0) {
          hh.v[v] = vo;
          hb.v[v] = T(0);
          if (m == 3) xx.v[v] = T(0);
        }
        if (m != 0) nb[v] += xx.v[v] * xx.v[v];
      }
      vst<T, VEC>(H + o, hh);
      vst<T, VEC>(Hb + o, hb);
      vst<T, VEC>(X + o, xx);
    }
    if (v_bits) {
      const T sc = __ldg(scale_of<T>(d, k) + l);
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        if ((v_bits >> v) & 1u) {
          const T vn = sum.v[v] * sc * rd_acc[v] - rd_v[v] * vv.v[v];
          vv.v[v] = vn;
          na[v] += vn * vn;
        }
      }
      vst<T, VEC>(V + o, vv);
      if (VS) {
        VA<T, VEC> vs;
#pragma unroll
        for (int v = 0; v < VEC; ++v) vs.v[v] = vv.v[v] * sc;
        vst<T, VEC>(VS + o, vs);
      }
    }
  }
};

// x <- A'b (the warm start of src/AbstractFixedEffectSolver.jl:56).
template <typename TOut, int VEC>
struct PEpiStoreX {
  using TS = double;
  using TN = double;
  TOut* __restrict__ X;
  bool act;
  __device__ __forceinline__ void begin(int, int, int) { act = true; }
  __device__ __forceinline__ void update(const FeDev& d, int k, int64_t l, int64_t o,
                                         const VA<double, VEC>& sum, double (&)[VEC],
                                         double (&)[VEC]) {
    const double sc = __ldg(d.scale_d[k] + l);
    VA<TOut, VEC> x;
#pragma unroll
    for (int v = 0; v < VEC; ++v) x.v[v] = (TOut)(sum.v[v] * sc);
    vst<TOut, VEC>(X + o, x);
  }
};

// Mixed precision: g = A'r computed in FP64 from the FP64 residual, stored as
// the FP32 starting v of the next inner solve; x64 += x32 and ||x64||^2.
template <int VEC>
struct PEpiGrad64 {
  using TS = double;
  using TN = double;
  float* __restrict__ V32;
  double* __restrict__ X64;
  const float* __restrict__ X32;
  float* __restrict__ VS32;  // optional: v scaled by the FP32 Jacobi scale
  const Inst* __restrict__ inst;
  bool actv[VEC];
  bool act;
  __device__ __forceinline__ void begin(int prob, int jl, int C) {
    act = false;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      actv[v] = inst[(int64_t)prob * C + jl * VEC + v].outer_active != 0;
      act = act || actv[v];
    }
  }
  __device__ __forceinline__ void update(const FeDev& d, int k, int64_t l, int64_t o,
                                         const VA<double, VEC>& sum, double (&na)[VEC],
                                         double (&nb)[VEC]) {
    const double sc = __ldg(d.scale_d[k] + l);
    VA<float, VEC> g32 = vld<float, VEC>(V32 + o);
    VA<double, VEC> x64 = vld<double, VEC>(X64 + o);
    const VA<float, VEC> x32 = vld<float, VEC>(X32 + o);
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      if (!actv[v]) continue;
      const double gv = sum.v[v] * sc;
      g32.v[v] = (float)gv;
      na[v] += gv * gv;
      const double x = x64.v[v] + (double)x32.v[v];
      x64.v[v] = x;
      nb[v] += x * x;
    }
    vst<float, VEC>(V32 + o, g32);
    vst<double, VEC>(X64 + o, x64);
    if (VS32) {
      const float sf = __ldg(d.scale_f[k] + l);
      VA<float, VEC> vs;
#pragma unroll
      for (int v = 0; v < VEC; ++v) vs.v[v] = g32.v[v] * sf;
      vst<float, VEC>(VS32 + o, vs);
    }
  }
};

// Jacobi scale: 1/sqrt(sum interaction^2 w), or 0 for an empty sum
// (src/SolverCPU.jl:84-88, issue #97 of the reference).  C = 1.
struct PEpiScale {
  using TS = double;
  using TN = double;
  double* sd[kMaxFE];
  float* sf[kMaxFE];
  bool act;
  __device__ __forceinline__ void begin(int, int, int) { act = true; }
  __device__ __forceinline__ void update(const FeDev&, int k, int64_t l, int64_t,
                                         const VA<double, 1>& sum, double (&)[1], double (&)[1]) {
    const double s = sum.v[0] > 0 ? 1.0 / sqrt(sum.v[0]) : 0.0;
    sd[k][l] = s;
    sf[k][l] = (float)s;
  }
};

// ---------------------------------------------------------------------------
// k_pupdate: one warp per PItem (a range of slab rows of one FE and problem),
// streaming.  Norms go to one slot per CTA.
// ---------------------------------------------------------------------------
template <int C, int U, class Epi>
__global__ void __launch_bounds__(kThreads)
k_pupdate(const FeDev d, const PItem* __restrict__ items, int64_t n_items,
          const typename Epi::TS* __restrict__ Sin, Epi epi, double* __restrict__ part_a,
          double* __restrict__ part_b, int64_t S) {
  using TS = typename Epi::TS;
  using Sh = Shape<TS, C>;
  constexpr int VEC = Sh::VEC, CL = Sh::CL, G = Sh::G;
  using TN = typename Epi::TN;
  __shared__ double sm[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int g = lane / CL, jl = lane - g * CL;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  double na[VEC], nb[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    na[v] = 0.0;
    nb[v] = 0.0;
  }
  if (w < n_items) {
    const PItem it = items[w];
    epi.begin(it.prob, jl, C);
    if (__any_sync(FE_FULL, epi.act)) {
      const int k = it.fe;
      const int64_t lb = d.lev_base[k];
      TN ia[VEC], ib[VEC];  // norms of this item, flushed below
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        ia[v] = TN(0);
        ib[v] = TN(0);
      }
      for (int64_t base = it.rb; base < it.re; base += (int64_t)G * U) {
        VA<TS, VEC> sv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t row = base + u * G + g;
          if (row < it.re) sv[u] = vld<TS, VEC>(Sin + row * C + jl * VEC);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t row = base + u * G + g;
          if (row < it.re && epi.act) epi.update(d, k, row - lb, row * C + jl * VEC, sv[u], ia, ib);
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        na[v] = (double)ia[v];
        nb[v] = (double)ib[v];
      }
    }
  }
  cta_norm_to_slot<C, VEC>(na, part_a, S, (int64_t)blockIdx.x, sm);
  __syncthreads();
  cta_norm_to_slot<C, VEC>(nb, part_b, S, (int64_t)blockIdx.x, sm);
}

}  // namespace fe
