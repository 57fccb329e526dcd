// fe_exdm_pipe.cuh -- the pipelined fused expand + demean of the absorbed
// loop (k_exdm_pipe): FP32 rows, 32-column tiles, the LSMR u-update.
//
// It computes what k_expand_demean computes in its LSMR form
//   u = M (av * A_r v + au * u),  ||u||^2,  small-FE sums of cw u
// (the reference's scatter! of the non-primary FEs with the rmul! of
// src/AbstractFixedEffectLinearMap.jl:26-44, then the projection of the
// absorbed primary FE and the gather! of the small FEs), with a different
// schedule:
//   - each warp walks its demean items (whole primary levels, at most 32
//     rows) with the NEXT item's rows and its gathered large-FE coefficient
//     rows already in flight: 16-byte cp.async copies into a two-stage
//     per-warp buffer, issued before the current item is computed, so the
//     DRAM reads of the rows and the L2 gathers of the coefficient rows
//     overlap the arithmetic of the item before;
//   - the item's refs and weights are loaded two items ahead into registers
//     (one row per lane), and its descriptor three items ahead, so the
//     gathers of the next item can be issued at once;
//   - the small FEs' pre-scaled coefficient rows (at most 32 table rows) are
//     held in shared memory by the CTA;
//   - the small-FE sums are added in the vector layout into one table per
//     lane group (4 groups of 8 lanes, one row each per warp instruction), so
//     rows of one instruction never update the same table row and no merging
//     of equal keys is needed.  The tables are summed in a fixed order
//     (warp, then group) into the CTA's partial, so the result is
//     deterministic for a given grid.
// A primary level longer than 32 rows is one item that takes a two-pass path
// with direct global loads (w written over u, level sum, then the
// projection).
#pragma once

#include "fe_kernels.cuh"

namespace fe {

// The non-primary FEs whose coefficient rows are gathered per row (the
// "large" FEs: neither the absorbed primary nor a small FE).
struct ExdmFEs {
  int32_t large[2];
  int64_t large_base[2];  // first slab row of each
};

template <int NL, int NS>
struct ExdmMeta {
  int64_t ib;
  int n;      // rows of the item (0: none; > 32: one long primary level)
  int kpr;    // primary level of row `lane`
  float cwp;  // primary interaction * sqrt(w) of row `lane`
  float sl;   // Jacobi scale of that level (loaded when the item's copies are issued)
  int rl[NL > 0 ? NL : 1];
  float cl[NL > 0 ? NL : 1];
  int ks[NS > 0 ? NS : 1];  // small-table row of row `lane`
  float cs[NS > 0 ? NS : 1];
};

// shared-memory bytes of one CTA of k_exdm_pipe with `stages` pipeline
// stages, per-group (pg) or per-warp small-FE tables, `warps` warps, and the
// small FEs' coefficient rows in shared memory (vsm) or read through L1
inline size_t exdm_pipe_smem(int NL, int small_rows, int stages, bool pg, int warps = kWarps,
                             bool vsm = true) {
  const size_t stage = (size_t)(1 + NL) * 32 * 32;
  const size_t per_warp = stages * stage + (NL == 0 ? 32 * 32 : 0) +
                          (pg ? 4 : 1) * (size_t)small_rows * 32 + 32;
  return ((vsm ? (size_t)small_rows * 32 : 0) + warps * per_warp) * sizeof(float);
}

__device__ __forceinline__ float4 f4_fma(float a, const float4 x, float4 y) {
  y.x = fmaf(a, x.x, y.x);
  y.y = fmaf(a, x.y, y.y);
  y.z = fmaf(a, x.z, y.z);
  y.w = fmaf(a, x.w, y.w);
  return y;
}

// W: some FE has interaction * sqrt(w) (per-FE pointers say which).
// STG: pipeline stages of the copies (2: the item computed and the next).
// PG: small-FE sums in one table per lane group, added in the vector layout
// (fast, 4x the shared memory); else one table per warp, added one column
// per lane after the rows are projected (rows of a group of 4 with equal
// keys merged first, as in the row-sum pass).
// Vector reduction of 4 floats into global memory (one 16-byte red).
__device__ __forceinline__ void red_add_v4(float* p, float a, float b, float c, float d) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

// ATOM (NL == 1 only): the gathered FE's level sums A'u are added here, row
// by row, with vector reductions into the [P][32] FP32 slab rs.sum (zeroed
// before the launch) instead of by the level-order segmented sum that
// follows; the order of the additions is not fixed, so the sums are not
// bitwise reproducible.
// WARPS < kWarps: small CTAs, three per SM; they read the small FEs'
// coefficient rows through L1 instead of holding a shared copy (VG), so that
// three CTAs' staging fits the shared memory of an SM.
template <int NL, int NS, bool W, int STG, bool PG, bool ATOM = false, int WARPS = kWarps>
__global__ void __launch_bounds__(WARPS * 32, WARPS < kWarps ? 3 : 1)
k_exdm_pipe(const FeDev d, const ExpandItem* __restrict__ items, int64_t n_items,
            const float* __restrict__ tab, float* __restrict__ rows,
            const Inst* __restrict__ inst, RowSumArgs rs, SmallRows sr, ExdmFEs lf,
            double* __restrict__ part, int64_t S) {
  constexpr int C = 32, G = 4, RC = 32;
  constexpr int STAGE = (1 + NL) * RC * C;  // floats per stage
  constexpr int NT = PG ? 4 : 1;            // small-FE tables per warp
  constexpr bool VG = WARPS < kWarps;       // small-FE rows through L1
  constexpr int NTH = WARPS * 32;
  static_assert(STG == 2, "two copy stages: the item computed and the next");
  using Meta = ExdmMeta<NL, NS>;
  extern __shared__ __align__(16) float xs_smem[];
  if (d.active_pre && *d.active_pre == 0) return;  // the whole CTA
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane >> 3, jl = lane & 7;
  const int nsr = NS > 0 ? rs.small_rows : 0;
  const int wstride_f = STG * STAGE + (NL == 0 ? RC * C : 0) + NT * nsr * C + 32;
  const int vsm_f = VG ? 0 : nsr * C;
  float* vsm = xs_smem;  // [nsr][32] the small FEs' pre-scaled coefficient rows
  float* wbase = xs_smem + vsm_f + (size_t)wib * wstride_f;
  float* zs_own = wbase + STG * STAGE;            // level sums when NL == 0
  float* tbl = zs_own + (NL == 0 ? RC * C : 0);   // [NT][nsr][32] small-FE sums
  int* lend = reinterpret_cast<int*>(tbl + NT * nsr * C);
  if (!VG)
    for (int e = threadIdx.x; e < nsr * C; e += NTH)
      vsm[e] = tab[sr.slab_row[e / C] * C + (e % C)];
  for (int e = lane; e < NT * nsr * C; e += 32) tbl[e] = 0.f;
  __syncthreads();
  // small-FE coefficient row k (table row k = small_off[j] + ref of FE j):
  // slab row lev_base[j's FE] + ref
  int64_t vgoff[NS > 0 ? NS : 1];
#pragma unroll
  for (int j = 0; j < NS; ++j)
    vgoff[j] = (int64_t)(d.lev_base[rs.small_fe[j]] - rs.small_off[j]) * C + jl * 4;
  auto small_row = [&](int j, int k) -> float4 {
    if (VG) return __ldg(reinterpret_cast<const float4*>(tab + vgoff[j] + (int64_t)k * C));
    return *reinterpret_cast<const float4*>(vsm + k * C + jl * 4);
  };

  const int kp = d.primary;
  const int32_t* __restrict__ refp = d.refs[kp];
  const float* __restrict__ cwpp = d.cw_f[kp];
  const float* __restrict__ scp = d.scale_f[kp];
  const int32_t* refL[NL > 0 ? NL : 1];
  const float* cwL[NL > 0 ? NL : 1];
#pragma unroll
  for (int j = 0; j < NL; ++j) {
    refL[j] = d.refs[lf.large[j]];
    cwL[j] = d.cw_f[lf.large[j]];
  }
  const int32_t* refS[NS > 0 ? NS : 1];
  const float* cwS[NS > 0 ? NS : 1];
  int offS[NS > 0 ? NS : 1];
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    refS[j] = d.refs[rs.small_fe[j]];
    cwS[j] = d.cw_f[rs.small_fe[j]];
    offS[j] = rs.small_off[j];
  }
  // the expand coefficients of this lane's 4 columns
  float av[4], au[4];
  bool act_any = false;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const Inst& st = inst[jl * 4 + v];
    av[v] = (float)st.ex_av;
    au[v] = (float)st.ex_au;
    act_any = act_any || st.active != 0;
  }
  act_any = __any_sync(FE_FULL, act_any);
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};

  // the descriptor of item wi (an empty item past the end)
  auto load_desc = [&](int64_t wi) {
    ExpandItem it{};
    if (wi < n_items) it = items[wi];
    return it;
  };
  // refs and weights of an item, one row per lane
  auto load_meta = [&](const ExpandItem& it) {
    Meta m;
    m.ib = 0;
    m.n = 0;
    m.kpr = 0;
    m.cwp = 1.f;
    m.sl = 0.f;
#pragma unroll
    for (int j = 0; j < (NL > 0 ? NL : 1); ++j) {
      m.rl[j] = 0;
      m.cl[j] = 1.f;
    }
#pragma unroll
    for (int j = 0; j < (NS > 0 ? NS : 1); ++j) {
      m.ks[j] = 0;
      m.cs[j] = 1.f;
    }
    {
      m.ib = it.ib;
      m.n = (int)(it.ie - it.ib);
      if (m.n > 0 && m.n <= RC && lane < m.n) {
        const int64_t p = m.ib + lane;
        m.kpr = __ldg(refp + p);
        if (W && cwpp) m.cwp = __ldg(cwpp + p);
#pragma unroll
        for (int j = 0; j < NL; ++j) {
          m.rl[j] = __ldg(refL[j] + p);
          if (W && cwL[j]) m.cl[j] = __ldg(cwL[j] + p);
        }
#pragma unroll
        for (int j = 0; j < NS; ++j) {
          m.ks[j] = offS[j] + __ldg(refS[j] + p);
          if (W && cwS[j]) m.cs[j] = __ldg(cwS[j] + p);
        }
      }
    }
    return m;
  };

  // asynchronous copies of an item's rows and gathered coefficient rows into
  // stage `st` (one cp.async group per item, possibly empty), and the load of
  // its rows' primary scales
  auto issue = [&](Meta& m, float* st) {
    if (m.n > 0 && m.n <= RC) {
      const float* src = rows + m.ib * C;
      for (int c = lane; c < m.n * 8; c += 32) cp_async_bytes16(st + c * 4, src + c * 4);
#pragma unroll
      for (int j = 0; j < NL; ++j) {
        for (int r0 = 0; r0 < m.n; r0 += G) {
          const int r = r0 + g;
          const int ref = __shfl_sync(FE_FULL, m.rl[j], r & 31);
          if (r < m.n)
            cp_async_bytes16(st + (1 + j) * RC * C + r * C + jl * 4,
                             tab + (lf.large_base[j] + ref) * C + jl * 4);
        }
      }
      if (lane < m.n) m.sl = __ldg(scp + m.kpr);
    }
    cp_async_commit();
  };

  // one item of at most 32 rows whose rows and gathered rows are in stage st
  auto compute_short = [&](const Meta& m, float* st) {
    constexpr int NT8 = RC / G;  // row steps of an item (8)
    const int n = m.n;
    float* ub = st;
    const float* lg = st + RC * C;
    float* zs = NL > 0 ? st + RC * C : zs_own;  // the gathered rows are dead after phase A
    // phase A: w = av * (A_r v) + au * u over the staged rows, all 8 row
    // steps unrolled (independent loads in flight); w kept in registers for
    // B2 and stored in place for B1
    float4 wv[NT8];
#pragma unroll
    for (int t = 0; t < NT8; ++t) {
      const int r = t * G + g;
      float cl[NL > 0 ? NL : 1], cs[NS > 0 ? NS : 1];
      int ks[NS > 0 ? NS : 1];
#pragma unroll
      for (int j = 0; j < NL; ++j) cl[j] = W ? __shfl_sync(FE_FULL, m.cl[j], r) : 1.f;
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        ks[j] = __shfl_sync(FE_FULL, m.ks[j], r);
        cs[j] = W ? __shfl_sync(FE_FULL, m.cs[j], r) : 1.f;
      }
      wv[t] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (r < n) {
        float4* up = reinterpret_cast<float4*>(ub + r * C + jl * 4);
        const float4 o = *up;
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < NL; ++j)
          a = f4_fma(cl[j], *reinterpret_cast<const float4*>(lg + j * RC * C + r * C + jl * 4), a);
#pragma unroll
        for (int j = 0; j < NS; ++j) a = f4_fma(cs[j], small_row(j, ks[j]), a);
        float4 w;
        w.x = av[0] * a.x + au[0] * o.x;
        w.y = av[1] * a.y + au[1] * o.y;
        w.z = av[2] * a.z + au[2] * o.z;
        w.w = av[3] * a.w + au[3] * o.w;
        *up = w;
        wv[t] = w;
      }
    }
    __syncwarp();
    // the primary levels of the item: the last row of each
    const int kn = __shfl_down_sync(FE_FULL, m.kpr, 1);
    const bool is_end = lane < n && (lane + 1 == n || kn != m.kpr);
    const uint32_t ends = __ballot_sync(FE_FULL, is_end);
    const int nlev = __popc(ends);
    if (is_end) lend[__popc(ends & ((1u << lane) - 1u))] = lane;
    __syncwarp();
    // B1: level sums z_l = sum cw w; group g sums levels g, g + 4, ..., four
    // rows at a time into independent partial sums
    for (int jb = 0; jb < nlev; jb += G) {
      const int j = jb + g;
      const bool okj = j < nlev;
      const int e = okj ? lend[j] : -1;
      const int s0 = (okj && j > 0) ? lend[j - 1] + 1 : 0;
      const int len = okj ? e - s0 + 1 : 0;
      const int maxlen = __reduce_max_sync(FE_FULL, (unsigned)len);
      float4 acc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int t0 = 0; t0 < maxlen; t0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int t = t0 + u;
          const bool ok = t < len;
          const int r = ok ? s0 + t : 0;
          const float c = W ? __shfl_sync(FE_FULL, m.cwp, r) : 1.f;
          if (ok) acc[u] = f4_fma(c, *reinterpret_cast<const float4*>(ub + r * C + jl * 4), acc[u]);
        }
      }
      float4 z;
      z.x = (acc[0].x + acc[1].x) + (acc[2].x + acc[3].x);
      z.y = (acc[0].y + acc[1].y) + (acc[2].y + acc[3].y);
      z.z = (acc[0].z + acc[1].z) + (acc[2].z + acc[3].z);
      z.w = (acc[0].w + acc[1].w) + (acc[2].w + acc[3].w);
      if (okj) *reinterpret_cast<float4*>(zs + j * C + jl * 4) = z;
    }
    __syncwarp();
    // B2: u = w - scale_l^2 cw z_l, stored once; ||u||^2; small-FE sums of
    // cw u into this group's tables (all 8 row steps unrolled)
    const float f = m.sl * m.sl * m.cwp;
    float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int t = 0; t < NT8; ++t) {
      const int r = t * G + g;
      const float fr = __shfl_sync(FE_FULL, f, r);
      const int fref = ATOM ? __shfl_sync(FE_FULL, m.rl[0], r) : 0;
      const float fcl = (ATOM && W) ? __shfl_sync(FE_FULL, m.cl[0], r) : 1.f;
      float cs[NS > 0 ? NS : 1];
      int ks[NS > 0 ? NS : 1];
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        ks[j] = __shfl_sync(FE_FULL, m.ks[j], r);
        cs[j] = W ? __shfl_sync(FE_FULL, m.cs[j], r) : 1.f;
      }
      if (r < n) {
        const int li = __popc(ends & ((1u << r) - 1u));
        const float4 z = *reinterpret_cast<const float4*>(zs + li * C + jl * 4);
        float4 u = wv[t];
        u.x -= fr * z.x;
        u.y -= fr * z.y;
        u.z -= fr * z.z;
        u.w -= fr * z.w;
        *reinterpret_cast<float4*>(rows + (m.ib + r) * C + jl * 4) = u;
        if (ATOM) {
          float* sl = static_cast<float*>(rs.sum) + (lf.large_base[0] + fref) * C + jl * 4;
          red_add_v4(sl, fcl * u.x, fcl * u.y, fcl * u.z, fcl * u.w);
        }
        nv.x += u.x * u.x;
        nv.y += u.y * u.y;
        nv.z += u.z * u.z;
        nv.w += u.w * u.w;
        if (PG) {
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            float4* tp = reinterpret_cast<float4*>(tbl + (g * nsr + ks[j]) * C + jl * 4);
            *tp = f4_fma(cs[j], u, *tp);
          }
        } else if (NS > 0) {
          *reinterpret_cast<float4*>(ub + r * C + jl * 4) = u;  // for B3
        }
      }
    }
    if (!PG && NS > 0) {
      // B3: small-FE sums of cw u, one column per lane (a row's table key is
      // the same in every lane)
      __syncwarp();
      for (int r0 = 0; r0 < n; r0 += 4) {
        const float x0 = ub[r0 * C + lane];
        const float x1 = r0 + 1 < n ? ub[(r0 + 1) * C + lane] : 0.f;
        const float x2 = r0 + 2 < n ? ub[(r0 + 2) * C + lane] : 0.f;
        const float x3 = r0 + 3 < n ? ub[(r0 + 3) * C + lane] : 0.f;
#pragma unroll
        for (int j = 0; j < NS; ++j)
          rowsum_small4<float, C, W>(r0, x0, x1, x2, x3, m.ks[j], m.cs[j], tbl, lane);
      }
    }
    nrm[0] += (double)nv.x;
    nrm[1] += (double)nv.y;
    nrm[2] += (double)nv.z;
    nrm[3] += (double)nv.w;
  };

  // one primary level longer than 32 rows: pass 1 writes w over u and sums
  // z = sum cw w; pass 2 projects.  Row r is handled by group r % 4 in both
  // passes, so every lane reads back what it wrote.
  auto compute_long = [&](const Meta& m) {
    const int64_t n = m.n;
    float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int64_t r = g; r < n; r += G) {
      const int64_t p = m.ib + r;
      float4* up = reinterpret_cast<float4*>(rows + p * C + jl * 4);
      const float4 o = *up;
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int j = 0; j < NL; ++j) {
        const int ref = __ldg(refL[j] + p);
        const float c = (W && cwL[j]) ? __ldg(cwL[j] + p) : 1.f;
        a = f4_fma(c, __ldg(reinterpret_cast<const float4*>(tab + (lf.large_base[j] + ref) * C + jl * 4)), a);
      }
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        const int k = offS[j] + __ldg(refS[j] + p);
        const float c = (W && cwS[j]) ? __ldg(cwS[j] + p) : 1.f;
        a = f4_fma(c, small_row(j, k), a);
      }
      float4 w;
      w.x = av[0] * a.x + au[0] * o.x;
      w.y = av[1] * a.y + au[1] * o.y;
      w.z = av[2] * a.z + au[2] * o.z;
      w.w = av[3] * a.w + au[3] * o.w;
      *up = w;
      const float cwr = (W && cwpp) ? __ldg(cwpp + p) : 1.f;
      z = f4_fma(cwr, w, z);
    }
    // the level sum over the 4 groups
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
      z.x += __shfl_xor_sync(FE_FULL, z.x, o);
      z.y += __shfl_xor_sync(FE_FULL, z.y, o);
      z.z += __shfl_xor_sync(FE_FULL, z.z, o);
      z.w += __shfl_xor_sync(FE_FULL, z.w, o);
    }
    const float sl = __ldg(scp + __ldg(refp + m.ib));
    float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
    // a warp-uniform loop: the per-warp table is updated by the groups in turn
    for (int64_t r0 = 0; r0 < n; r0 += G) {
      const int64_t r = r0 + g;
      const bool ok = r < n;
      const int64_t p = m.ib + (ok ? r : 0);
      float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
      if (ok) {
        const float cwr = (W && cwpp) ? __ldg(cwpp + p) : 1.f;
        const float fr = sl * sl * cwr;
        float4* up = reinterpret_cast<float4*>(rows + p * C + jl * 4);
        u = *up;
        u.x -= fr * z.x;
        u.y -= fr * z.y;
        u.z -= fr * z.z;
        u.w -= fr * z.w;
        *up = u;
        if (ATOM) {
          const int ref = __ldg(refL[0] + p);
          const float c = (W && cwL[0]) ? __ldg(cwL[0] + p) : 1.f;
          red_add_v4(static_cast<float*>(rs.sum) + (lf.large_base[0] + ref) * C + jl * 4, c * u.x,
                     c * u.y, c * u.z, c * u.w);
        }
        nv.x += u.x * u.x;
        nv.y += u.y * u.y;
        nv.z += u.z * u.z;
        nv.w += u.w * u.w;
      }
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        const int k = ok ? offS[j] + __ldg(refS[j] + p) : 0;
        const float c = (ok && W && cwS[j]) ? __ldg(cwS[j] + p) : 1.f;
        if (PG) {
          if (ok) {
            float4* tp = reinterpret_cast<float4*>(tbl + (g * nsr + k) * C + jl * 4);
            *tp = f4_fma(c, u, *tp);
          }
        } else {
          // one table per warp: the 4 groups add their rows in turn
          for (int gg = 0; gg < G; ++gg) {
            if (ok && g == gg) {
              float4* tp = reinterpret_cast<float4*>(tbl + k * C + jl * 4);
              *tp = f4_fma(c, u, *tp);
            }
            __syncwarp();
          }
        }
      }
    }
    nrm[0] += (double)nv.x;
    nrm[1] += (double)nv.y;
    nrm[2] += (double)nv.z;
    nrm[3] += (double)nv.w;
  };

  if (act_any) {
    // Software pipeline over the warp's items (stride wstride): while item i
    // is computed, the copies of item i+1 are in flight (stage s ^ 1), the
    // refs of item i+2 are being loaded into registers, and the descriptor of
    // item i+3; nothing loaded is used before the next step.
    const int64_t wstride = (int64_t)gridDim.x * WARPS;
    const int64_t w0 = (int64_t)blockIdx.x * WARPS + wib;
    ExpandItem d2 = load_desc(w0 + 2 * wstride);
    Meta m0 = load_meta(load_desc(w0));
    issue(m0, wbase);
    Meta m1 = load_meta(load_desc(w0 + wstride));
    int s = 0;
    for (int64_t wi = w0; wi < n_items; wi += wstride) {
      const ExpandItem d3 = load_desc(wi + 3 * wstride);
      const Meta m2 = load_meta(d2);
      issue(m1, wbase + (s ^ 1) * STAGE);  // the next item's copies, in flight
      cp_async_wait<1>();                    // this item's copies have landed
      __syncwarp();
      if (m0.n > RC) compute_long(m0);
      else if (m0.n > 0) compute_short(m0, wbase + s * STAGE);
      __syncwarp();  // the stage is refilled on the next step
      m0 = m1;
      m1 = m2;
      d2 = d3;
      s ^= 1;
    }
    cp_async_wait<0>();
  }
  // ||u||^2 per column: groups, then warps in order -> the CTA's slot.  The
  // scratch of the warp sums reuses the start of the dynamic shared memory
  // (staged rows and small-FE rows, dead once every warp is past its items),
  // so that the CTA holds no static shared memory.
  __syncthreads();
  double(*sm)[32] = reinterpret_cast<double(*)[32]>(xs_smem);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double a = nrm[v];
    a += __shfl_xor_sync(FE_FULL, a, 8);
    a += __shfl_xor_sync(FE_FULL, a, 16);
    if (g == 0) sm[wib][jl * 4 + v] = a;
  }
  __syncthreads();
  if (part != nullptr && threadIdx.x < C) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) t += sm[w][threadIdx.x];
    part[(int64_t)threadIdx.x * S + blockIdx.x] = t;
    for (int64_t sl = (int64_t)blockIdx.x + gridDim.x; sl < S; sl += gridDim.x)
      part[(int64_t)threadIdx.x * S + sl] = 0.0;
  }
  if (NS > 0) {
    // small-FE sums: warp tables in warp order, groups in group order
    const int n = nsr * C;
    double* __restrict__ out = rs.small_part + (int64_t)blockIdx.x * n;
    const float* t0 = xs_smem + vsm_f + STG * STAGE + (NL == 0 ? RC * C : 0);
    for (int e = threadIdx.x; e < n; e += NTH) {
      double t = 0.0;
      for (int w = 0; w < WARPS; ++w)
#pragma unroll
        for (int gg = 0; gg < NT; ++gg) t += (double)t0[(size_t)w * wstride_f + gg * n + e];
      out[e] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// host side: one launch of k_exdm_pipe (instantiated in fe_exdm_pipe.cu)
// ---------------------------------------------------------------------------
struct ExdmLaunch {
  FeDev d;
  const ExpandItem* items;
  int64_t n_items;
  const float* tab;
  float* rows;
  const Inst* inst;
  RowSumArgs rs;
  SmallRows sr;
  ExdmFEs lf;
  double* part;
  int64_t S;
  int64_t grid;
  size_t smem;
  cudaStream_t stream;
};

// Kernel configurations (FE_OPT_EXDM_PIPE values): 1 per-group small-FE
// tables (vector layout), 2 one table per warp (less shared memory), 3 one
// table per warp in CTAs of 4 warps, three per SM, the small FEs' rows read
// through L1.
struct ExdmCfg {
  int stages;
  bool per_group;
  int warps;
  bool vsm;  // the small FEs' coefficient rows held in shared memory
};
inline ExdmCfg exdm_cfg(int cfg) {
  if (cfg == 3) return ExdmCfg{2, false, 4, false};
  return cfg == 2 ? ExdmCfg{2, false, kWarps, true} : ExdmCfg{2, true, kWarps, true};
}

// Launches k_exdm_pipe<nl, ns, w, stages, per_group> of configuration
// `cfg` (atomic: the gathered FE's level sums by vector reductions, cfg 1
// and nl == 1 only); returns a CUDA status (0 = launched).
int launch_exdm_pipe(const ExdmLaunch& a, int nl, int ns, bool w, int cfg, bool atomic = false);

}  // namespace fe
