// fe_build.cu -- plan construction on the device: key grouping (the
// GroupedArray compaction behind FixedEffect(keys...), src/FixedEffect.jl:18-21),
// ref validation, and the integer plan (the sort of the observations by their
// primary level and each FE's level order; the bucketing of
// ext/MetalExt.jl:40-64 for every FE).
//
// Both rest on one primitive, a stable least-significant-digit radix sort of
// (key, index) pairs:
//   * a pass over one digit of up to 8 bits counts the digits of each tile of
//     4096 keys into a digit-major table hist[d][tile];
//   * an exclusive scan of that table gives every (digit, tile) its first
//     output slot;
//   * a second pass ranks each key among the equal digits of its tile in
//     input order (a warp matches equal digits with __match_any_sync, warps
//     keep running per-digit counts in shared memory) and stores the pair
//     there.
// Every placement follows input order within a digit, so the sort is stable
// and yields exactly the stable counting sort's permutation.  All counts are
// integers: the plan does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fe_b200.h"
#include "fe_plan.h"

namespace fe {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

constexpr int kRThreads = 256;
constexpr int kRWarps = kRThreads / 32;
constexpr int kRItems = 16;                     // keys per lane
constexpr int kRWarpSpan = 32 * kRItems;        // 512 consecutive keys per warp
constexpr int kRTile = kRThreads * kRItems;     // 4096 keys per tile
constexpr int kRBits = 8;                       // digit width at most

inline unsigned blocks_of(int64_t n, int64_t b) { return (unsigned)((n + b - 1) / b); }

// ---------------------------------------------------------------------------
// exclusive scan of int32 counts (totals below 2^31)
// ---------------------------------------------------------------------------
// One tile of kScanTile values per block, staged through shared memory so
// that global loads and stores are coalesced; the block total goes to part[].
__global__ void __launch_bounds__(kScanThreads)
k_scan_tile(const int32_t* in, int32_t* out, int64_t n, int32_t* part, int32_t* total) {
  __shared__ int32_t t[kScanTile + kScanTile / 32];
  __shared__ int32_t wsum[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // padded index: one skipped word per 32 keeps the per-thread runs of 8
  // consecutive values free of bank conflicts
#define PAD(i) ((i) + ((i) >> 5))
  for (int j = 0; j < kScanItems; ++j) {
    const int i = j * kScanThreads + tid;
    t[PAD(i)] = base + i < n ? in[base + i] : 0;
  }
  __syncthreads();
  int32_t v[kScanItems];
  int32_t s = 0;
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = t[PAD(tid * kScanItems + j)];
    s += v[j];
  }
  // block-wide exclusive scan of the per-thread sums
  int32_t incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int32_t w = lane < kScanThreads / 32 ? wsum[lane] : 0;
    int32_t wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kScanThreads / 32) wsum[lane] = wi - w;  // exclusive warp offsets
    if (lane == kScanThreads / 32 - 1) {
      if (part) part[blockIdx.x] = wi;
      if (total) *total = wi;
    }
  }
  __syncthreads();
  int32_t run = wsum[warp] + incl - s;
  for (int j = 0; j < kScanItems; ++j) {
    t[PAD(tid * kScanItems + j)] = run;
    run += v[j];
  }
  __syncthreads();
  for (int j = 0; j < kScanItems; ++j) {
    const int i = j * kScanThreads + tid;
    if (base + i < n) out[base + i] = t[PAD(i)];
  }
#undef PAD
}

__global__ void k_scan_add(int32_t* out, int64_t n, const int32_t* part) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += part[i / kScanTile];
}

// out[i] = sum of in[0..i); *total (device) = sum of all, when given.  in may
// equal out.
int scan_excl(const int32_t* in, int32_t* out, int64_t n, int32_t* total, cudaStream_t s) {
  if (n <= 0) {
    if (total) FE_CK(cudaMemsetAsync(total, 0, 4, s));
    return 0;
  }
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 1) {
    k_scan_tile<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
    FE_CK(cudaGetLastError());
    return 0;
  }
  DevBuf part;
  int st = part.ensure((size_t)nb * 4);
  if (st) return st;
  k_scan_tile<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, part.as<int32_t>(), nullptr);
  FE_CK(cudaGetLastError());
  st = scan_excl(part.as<int32_t>(), part.as<int32_t>(), nb, total, s);
  if (st) return st;
  k_scan_add<<<blocks_of(n, 256), 256, 0, s>>>(out, n, part.as<int32_t>());
  FE_CK(cudaGetLastError());
  FE_CK(cudaStreamSynchronize(s));  // part is freed on return
  return 0;
}

// ---------------------------------------------------------------------------
// stable LSD radix sort of (key, int32 value) pairs
// ---------------------------------------------------------------------------
// Keys of tile t: [t*kRTile, (t+1)*kRTile); warp w of the tile takes the
// kRWarpSpan keys from t*kRTile + w*kRWarpSpan on, 32 consecutive keys per
// round, so (warp, round, lane) runs in input order.
template <typename KT>
__global__ void __launch_bounds__(kRThreads)
k_radix_hist(const KT* __restrict__ keys, int64_t n, int shift, int bits, int32_t* __restrict__ hist,
             int64_t ntiles) {
  __shared__ int32_t cnt[1 << kRBits];
  const int nd = 1 << bits;
  for (int d = threadIdx.x; d < nd; d += kRThreads) cnt[d] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kRTile + (int64_t)warp * kRWarpSpan + lane;
  const KT mask = (KT)(nd - 1);
#pragma unroll 4
  for (int r = 0; r < kRItems; ++r) {
    const int64_t i = base + r * 32;
    if (i < n) atomicAdd(&cnt[(int)((keys[i] >> shift) & mask)], 1);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < nd; d += kRThreads) hist[(int64_t)d * ntiles + blockIdx.x] = cnt[d];
}

template <typename KT>
__global__ void __launch_bounds__(kRThreads)
k_radix_scatter(const KT* __restrict__ kin, const int32_t* __restrict__ vin, KT* __restrict__ kout,
                int32_t* __restrict__ vout, int64_t n, int shift, int bits,
                const int32_t* __restrict__ off, int64_t ntiles) {
  __shared__ int32_t wcnt[kRWarps][1 << kRBits];
  const int nd = 1 << bits;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = lane; d < nd; d += 32) wcnt[warp][d] = 0;
  __syncwarp();
  const int64_t base = (int64_t)blockIdx.x * kRTile + (int64_t)warp * kRWarpSpan + lane;
  const KT mask = (KT)(nd - 1);
  const unsigned lt = (1u << lane) - 1u;
  KT k[kRItems];
  int32_t v[kRItems];
  int32_t pos[kRItems];
#pragma unroll
  for (int r = 0; r < kRItems; ++r) {
    const int64_t i = base + r * 32;
    const bool ok = i < n;
    k[r] = ok ? kin[i] : (KT)0;
    v[r] = ok ? vin[i] : 0;
    // keys past the end form their own group (digit nd), after every real key
    const int d = ok ? (int)((k[r] >> shift) & mask) : nd;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int before = ok ? wcnt[warp][d] : 0;
    pos[r] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit: the tile's first slot plus the counts of the warps before
  for (int d = threadIdx.x; d < nd; d += kRThreads) {
    int32_t run = off[(int64_t)d * ntiles + blockIdx.x];
    for (int w = 0; w < kRWarps; ++w) {
      const int32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRItems; ++r) {
    const int64_t i = base + r * 32;
    if (i < n) {
      const int d = (int)((k[r] >> shift) & mask);
      const int32_t o = wcnt[warp][d] + pos[r];
      kout[o] = k[r];
      vout[o] = v[r];
    }
  }
}

int bits_for(uint64_t maxkey) {
  int b = 0;
  while (b < 64 && (maxkey >> b) != 0) ++b;
  return b;
}

// Sorts keys[0..n) with values (stable), keys below 2^total_bits.  The sorted
// pairs end in (keys, vals) or (kalt, valt); *in_alt says which.
template <typename KT>
int radix_sort(KT* keys, int32_t* vals, KT* kalt, int32_t* valt, int64_t n, int total_bits,
               bool* in_alt, cudaStream_t s) {
  *in_alt = false;
  if (n <= 1 || total_bits <= 0) return 0;
  const int passes = (total_bits + kRBits - 1) / kRBits;
  const int per = (total_bits + passes - 1) / passes;
  const int64_t ntiles = (n + kRTile - 1) / kRTile;
  DevBuf hist;
  int st = hist.ensure((size_t)(1 << per) * (size_t)ntiles * 4);
  if (st) return st;
  KT *ka = keys, *kb = kalt;
  int32_t *va = vals, *vb = valt;
  for (int shift = 0; shift < total_bits; shift += per) {
    const int b = std::min(per, total_bits - shift);
    k_radix_hist<KT><<<(unsigned)ntiles, kRThreads, 0, s>>>(ka, n, shift, b, hist.as<int32_t>(), ntiles);
    FE_CK(cudaGetLastError());
    st = scan_excl(hist.as<int32_t>(), hist.as<int32_t>(), (int64_t)(1 << b) * ntiles, nullptr, s);
    if (st) return st;
    k_radix_scatter<KT><<<(unsigned)ntiles, kRThreads, 0, s>>>(ka, va, kb, vb, n, shift, b,
                                                               hist.as<int32_t>(), ntiles);
    FE_CK(cudaGetLastError());
    std::swap(ka, kb);
    std::swap(va, vb);
    *in_alt = !*in_alt;
  }
  FE_CK(cudaStreamSynchronize(s));  // hist is freed on return
  return 0;
}

__global__ void k_iota(int32_t* v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int32_t)i;
}

// ---------------------------------------------------------------------------
// key grouping
// ---------------------------------------------------------------------------
__global__ void k_minmax(const int64_t* __restrict__ a, int64_t n, long long* mm) {
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const long long x = a[i];
    lo = min(lo, x);
    hi = max(hi, x);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
}
__global__ void k_mark(const int64_t* __restrict__ a, int64_t n, long long lo, int32_t* flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[(uint64_t)((unsigned long long)a[i] - (unsigned long long)lo)] = 1;
}
__global__ void k_lookup(const int64_t* __restrict__ a, int64_t n, long long lo,
                         const int32_t* __restrict__ rank, int32_t* __restrict__ id) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) id[i] = rank[(uint64_t)((unsigned long long)a[i] - (unsigned long long)lo)];
}
__global__ void k_offset_key(const int64_t* __restrict__ a, int64_t n, long long lo,
                             uint64_t* __restrict__ k) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) k[i] = (unsigned long long)a[i] - (unsigned long long)lo;
}
__global__ void k_first_flags(const uint64_t* __restrict__ sk, int64_t n, int32_t* __restrict__ f) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) f[q] = (q == 0 || sk[q] != sk[q - 1]) ? 1 : 0;
}
__global__ void k_rank_scatter(const int32_t* __restrict__ excl, const int32_t* __restrict__ f,
                               const int32_t* __restrict__ src, int64_t n, int32_t* __restrict__ id) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) id[src[q]] = excl[q] + f[q] - 1;
}
__global__ void k_fold(const int32_t* __restrict__ a, const int32_t* __restrict__ b, int64_t nb,
                       int64_t n, int64_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int64_t)a[i] * nb + b[i];
}
__global__ void k_to_refs(const int32_t* __restrict__ id, int64_t n, int64_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int64_t)id[i] + 1;
}

// id[i] = rank of a[i] among the distinct values of a[0..n) (0-based,
// ascending); *nlev = number of distinct values.  a is device memory.
int group_dev(const int64_t* a, int64_t n, int32_t* id, int64_t* nlev, cudaStream_t s) {
  *nlev = 0;
  if (n <= 0) return 0;
  DevBuf mm, tot;
  int st = mm.ensure(16);
  if (!st) st = tot.ensure(4);
  if (st) return st;
  const long long init[2] = {LLONG_MAX, LLONG_MIN};
  FE_CK(cudaMemcpyAsync(mm.p, init, 16, cudaMemcpyHostToDevice, s));
  k_minmax<<<std::min<unsigned>(blocks_of(n, 256), 4096), 256, 0, s>>>(a, n, mm.as<long long>());
  FE_CK(cudaGetLastError());
  long long h[2];
  FE_CK(cudaMemcpyAsync(h, mm.p, 16, cudaMemcpyDeviceToHost, s));
  FE_CK(cudaStreamSynchronize(s));
  const unsigned long long span = (unsigned long long)h[1] - (unsigned long long)h[0];
  const unsigned long long dense_max =
      std::max<unsigned long long>(2ull * (unsigned long long)n, 1ull << 20);
  int32_t total = 0;
  if (span < dense_max && span < (unsigned long long)INT32_MAX) {
    // dense keys: presence flags over [min, max] and their prefix sum
    const int64_t R = (int64_t)span + 1;
    DevBuf flag;
    st = flag.ensure((size_t)R * 4);
    if (st) return st;
    FE_CK(cudaMemsetAsync(flag.p, 0, (size_t)R * 4, s));
    k_mark<<<blocks_of(n, 256), 256, 0, s>>>(a, n, h[0], flag.as<int32_t>());
    FE_CK(cudaGetLastError());
    st = scan_excl(flag.as<int32_t>(), flag.as<int32_t>(), R, tot.as<int32_t>(), s);
    if (st) return st;
    k_lookup<<<blocks_of(n, 256), 256, 0, s>>>(a, n, h[0], flag.as<int32_t>(), id);
    FE_CK(cudaGetLastError());
  } else {
    // sparse keys: sort (key - min, position) pairs, number the runs
    DevBuf k0, k1, v0, v1;
    st = k0.ensure((size_t)n * 8);
    if (!st) st = k1.ensure((size_t)n * 8);
    if (!st) st = v0.ensure((size_t)n * 4);
    if (!st) st = v1.ensure((size_t)n * 4);
    if (st) return st;
    k_offset_key<<<blocks_of(n, 256), 256, 0, s>>>(a, n, h[0], k0.as<uint64_t>());
    k_iota<<<blocks_of(n, 256), 256, 0, s>>>(v0.as<int32_t>(), n);
    FE_CK(cudaGetLastError());
    bool alt = false;
    st = radix_sort<uint64_t>(k0.as<uint64_t>(), v0.as<int32_t>(), k1.as<uint64_t>(),
                              v1.as<int32_t>(), n, bits_for(span), &alt, s);
    if (st) return st;
    const uint64_t* sk = (alt ? k1 : k0).as<uint64_t>();
    const int32_t* src = (alt ? v1 : v0).as<int32_t>();
    int32_t* f = (alt ? v0 : v1).as<int32_t>();          // free value buffer
    int32_t* ex = reinterpret_cast<int32_t*>((alt ? k0 : k1).p);  // free key buffer
    k_first_flags<<<blocks_of(n, 256), 256, 0, s>>>(sk, n, f);
    FE_CK(cudaGetLastError());
    st = scan_excl(f, ex, n, tot.as<int32_t>(), s);
    if (st) return st;
    k_rank_scatter<<<blocks_of(n, 256), 256, 0, s>>>(ex, f, src, n, id);
    FE_CK(cudaGetLastError());
  }
  FE_CK(cudaMemcpyAsync(&total, tot.p, 4, cudaMemcpyDeviceToHost, s));
  FE_CK(cudaStreamSynchronize(s));
  *nlev = total;
  return 0;
}

// ---------------------------------------------------------------------------
// integer plan
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t problem_of(const int64_t* off, int32_t nprob, int64_t i) {
  // the last p with off[p] <= i (empty problems repeat an offset)
  int32_t lo = 0, hi = nprob;  // off[lo] <= i < off[hi]
  while (hi - lo > 1) {
    const int32_t mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Validates refs[k] (1-based; 0 where the problem lacks FE k) and converts it
// to global level ids: lev_off[p][k] + ref - 1, or nlev_k (the null level) for
// problems without FE k.  The first bad position goes to *bad.
__global__ void k_check_convert(const int64_t* __restrict__ r, int64_t N, int k, int K,
                                int32_t nprob, const int64_t* __restrict__ obs_off,
                                const int64_t* __restrict__ n_levels,
                                const int64_t* __restrict__ lev_off, int64_t nlev_k,
                                int32_t* __restrict__ g, unsigned long long* bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int32_t p = nprob == 1 ? 0 : problem_of(obs_off, nprob, i);
  const int64_t nl = n_levels[(int64_t)p * K + k];
  const int64_t v = r[i];
  const bool ok = nl == 0 ? v == 0 : (v >= 1 && v <= nl);
  if (!ok) {
    atomicMin(bad, (unsigned long long)i);
    g[i] = 0;
    return;
  }
  g[i] = nl == 0 ? (int32_t)nlev_k : (int32_t)(lev_off[(int64_t)p * K + k] + v - 1);
}

// Sort key of the observation order: problem p's levels of the primary FE
// shifted by p, so that each problem keeps a bucket of its own (its position
// when it lacks the primary FE) and problems stay in order.
__global__ void k_primary_key(const int32_t* __restrict__ g, int64_t N, int kp, int K,
                              int32_t nprob, const int64_t* __restrict__ obs_off,
                              const int64_t* __restrict__ n_levels,
                              const int64_t* __restrict__ lev_off, uint32_t* __restrict__ key) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int32_t p = nprob == 1 ? 0 : problem_of(obs_off, nprob, i);
  const bool absent = n_levels[(int64_t)p * K + kp] == 0;
  key[i] = (uint32_t)((absent ? lev_off[(int64_t)p * K + kp] : (int64_t)g[i]) + p);
}

__global__ void k_inverse(const int32_t* __restrict__ src, int64_t N, int32_t* __restrict__ dst) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < N) dst[src[q]] = (int32_t)q;
}
__global__ void k_gather_i(const int32_t* __restrict__ a, const int32_t* __restrict__ idx,
                           int64_t N, int32_t* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < N) out[q] = a[idx[q]];
}
__global__ void k_gather_f64(const double* __restrict__ a, const int32_t* __restrict__ idx,
                             int64_t N, double* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < N) out[q] = a[idx[q]];
}
// flag = 1 if the level ids are not nondecreasing or hold the null level
__global__ void k_not_identity(const int32_t* __restrict__ rs, int64_t N, int32_t null_lev,
                               int32_t* flag) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool bad = q < N && (rs[q] == null_lev || (q > 0 && rs[q] < rs[q - 1]));
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}
// Level offsets from sorted level ids: off[l] = first position with id >= l
// for l in [0, nb]; thread q writes the offsets of the ids skipped between
// position q-1 and q.
__global__ void k_level_offsets(const int32_t* __restrict__ sk, int64_t N, int64_t nb,
                                int32_t* __restrict__ off) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q > N) return;
  const int64_t a = q == 0 ? -1 : (int64_t)sk[q - 1];
  const int64_t b = q == N ? nb : (int64_t)sk[q];
  for (int64_t l = a + 1; l <= b; ++l) off[l] = (int32_t)q;
}

}  // namespace

// The integer plan of plan_build on the device (same outputs as stable
// counting sorts on the host): d_obs_src/d_obs_dst, per FE d_refs (sorted
// order), d_key and d_perm (level order), seg_off, seg_len, perm_identity, and
// the interactions in sorted order.  The host-side fields (nlev, prob_*_off,
// primary, lev_base, P) are set by the caller.
int plan_build_device(fe_plan* pl, const int64_t* const* refs, const int64_t* n_levels,
                      const double* const* interaction) {
  const int64_t N = pl->N;
  const int K = pl->K, nprob = pl->nprob;
  cudaStream_t s = pl->stream;
  DevBuf d_obs_off, d_nl, d_lev_off, d_bad, d_r64;
  int st = d_obs_off.ensure((size_t)(nprob + 1) * 8);
  if (!st) st = d_nl.ensure((size_t)nprob * K * 8);
  if (!st) st = d_lev_off.ensure((size_t)(nprob + 1) * K * 8);
  if (!st) st = d_bad.ensure((size_t)K * 8);
  if (!st) st = d_r64.ensure((size_t)std::max<int64_t>(N, 1) * 8);
  if (st) return st;
  FE_CK(cudaMemcpyAsync(d_obs_off.p, pl->prob_obs_off.data(), (size_t)(nprob + 1) * 8,
                        cudaMemcpyHostToDevice, s));
  FE_CK(cudaMemcpyAsync(d_nl.p, n_levels, (size_t)nprob * K * 8, cudaMemcpyHostToDevice, s));
  FE_CK(cudaMemcpyAsync(d_lev_off.p, pl->prob_lev_off.data(), (size_t)(nprob + 1) * K * 8,
                        cudaMemcpyHostToDevice, s));
  FE_CK(cudaMemsetAsync(d_bad.p, 0xff, (size_t)K * 8, s));

  // global level ids of every FE in the caller's observation order
  std::vector<DevBuf> g(K);
  for (int k = 0; k < K; ++k) {
    st = g[k].ensure((size_t)std::max<int64_t>(N, 1) * 4);
    if (st) return st;
    if (!N) continue;
    FE_CK(cudaMemcpyAsync(d_r64.p, refs[k], (size_t)N * 8, cudaMemcpyHostToDevice, s));
    k_check_convert<<<blocks_of(N, 256), 256, 0, s>>>(
        d_r64.as<int64_t>(), N, k, K, nprob, d_obs_off.as<int64_t>(), d_nl.as<int64_t>(),
        d_lev_off.as<int64_t>(), pl->nlev[k], g[k].as<int32_t>(), d_bad.as<unsigned long long>() + k);
    FE_CK(cudaGetLastError());
  }
  std::vector<unsigned long long> bad((size_t)K);
  FE_CK(cudaMemcpyAsync(bad.data(), d_bad.p, (size_t)K * 8, cudaMemcpyDeviceToHost, s));
  FE_CK(cudaStreamSynchronize(s));
  {
    // report the error a problem-by-problem, FE-by-FE scan meets first
    int bk = -1;
    int64_t bp = 0;
    for (int k = 0; k < K; ++k) {
      if (bad[(size_t)k] >= (unsigned long long)N) continue;
      const int64_t i = (int64_t)bad[(size_t)k];
      const int64_t p =
          (int64_t)(std::upper_bound(pl->prob_obs_off.begin(), pl->prob_obs_off.end(), i) -
                    pl->prob_obs_off.begin()) - 1;
      if (bk < 0 || p < bp) {
        bk = k;
        bp = p;
      }
    }
    if (bk >= 0) {
      const int64_t i = (int64_t)bad[(size_t)bk];
      const int64_t nl = n_levels[bp * K + bk];
      set_error("plan: refs[" + std::to_string(bk) + "][" + std::to_string(i) + "] = " +
                std::to_string(refs[bk][i]) + " is outside 1.." + std::to_string(nl));
      return 1;
    }
  }
  FE_CK(cudaFree(d_r64.p));  // the raw refs are no longer needed
  d_r64.p = nullptr;
  d_r64.bytes = 0;

  // observation order: stable sort by (problem, primary level)
  st = pl->d_obs_src.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  if (!st) st = pl->d_obs_dst.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  DevBuf ka, kb, va, vb;
  if (!st) st = ka.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  if (!st) st = kb.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  if (!st) st = va.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  if (!st) st = vb.ensure((size_t)std::max<int64_t>(N, 1) * 4);
  if (st) return st;
  const int kp = pl->primary;
  if (N) {
    k_primary_key<<<blocks_of(N, 256), 256, 0, s>>>(g[kp].as<int32_t>(), N, kp, K, nprob,
                                                    d_obs_off.as<int64_t>(), d_nl.as<int64_t>(),
                                                    d_lev_off.as<int64_t>(), ka.as<uint32_t>());
    k_iota<<<blocks_of(N, 256), 256, 0, s>>>(va.as<int32_t>(), N);
    FE_CK(cudaGetLastError());
    bool alt = false;
    st = radix_sort<uint32_t>(ka.as<uint32_t>(), va.as<int32_t>(), kb.as<uint32_t>(),
                              vb.as<int32_t>(), N,
                              bits_for((uint64_t)(pl->nlev[kp] + nprob - 1)), &alt, s);
    if (st) return st;
    FE_CK(cudaMemcpyAsync(pl->d_obs_src.p, (alt ? vb : va).p, (size_t)N * 4,
                          cudaMemcpyDeviceToDevice, s));
    k_inverse<<<blocks_of(N, 256), 256, 0, s>>>(pl->d_obs_src.as<int32_t>(), N,
                                                pl->d_obs_dst.as<int32_t>());
    FE_CK(cudaGetLastError());
  }

  // per FE: level ids in sorted order, then the level order of the positions
  pl->d_refs.resize(K);
  pl->d_perm.resize(K);
  pl->d_key.resize(K);
  pl->perm_identity.assign(K, false);
  pl->seg_off.assign(K, {});
  pl->seg_len.assign(K, 0);
  DevBuf flag, off;
  st = flag.ensure(4);
  if (st) return st;
  for (int k = 0; k < K; ++k) {
    const int64_t nb = pl->nlev[k] + 1;  // levels + the null level (last)
    st = pl->d_refs[k].ensure((size_t)std::max<int64_t>(N, 1) * 4);
    if (!st) st = off.ensure((size_t)(nb + 1) * 4);
    if (st) return st;
    int32_t* rs = pl->d_refs[k].as<int32_t>();
    bool ident = true;
    const int32_t* sk = rs;  // level ids in level order
    const int32_t* perm = nullptr;
    if (N) {
      k_gather_i<<<blocks_of(N, 256), 256, 0, s>>>(g[k].as<int32_t>(), pl->d_obs_src.as<int32_t>(),
                                                   N, rs);
      FE_CK(cudaMemsetAsync(flag.p, 0, 4, s));
      k_not_identity<<<blocks_of(N, 256), 256, 0, s>>>(rs, N, (int32_t)pl->nlev[k],
                                                       flag.as<int32_t>());
      FE_CK(cudaGetLastError());
      int32_t h = 0;
      FE_CK(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, s));
      FE_CK(cudaStreamSynchronize(s));
      ident = h == 0;
      if (!ident) {
        FE_CK(cudaMemcpyAsync(ka.p, rs, (size_t)N * 4, cudaMemcpyDeviceToDevice, s));
        k_iota<<<blocks_of(N, 256), 256, 0, s>>>(va.as<int32_t>(), N);
        FE_CK(cudaGetLastError());
        bool alt = false;
        st = radix_sort<uint32_t>(ka.as<uint32_t>(), va.as<int32_t>(), kb.as<uint32_t>(),
                                  vb.as<int32_t>(), N, bits_for((uint64_t)(nb - 1)), &alt, s);
        if (st) return st;
        sk = (alt ? kb : ka).as<int32_t>();
        perm = (alt ? vb : va).as<int32_t>();
      }
    }
    k_level_offsets<<<blocks_of(N + 1, 256), 256, 0, s>>>(sk, N, nb, off.as<int32_t>());
    FE_CK(cudaGetLastError());
    std::vector<int32_t> h((size_t)nb + 1);
    FE_CK(cudaMemcpyAsync(h.data(), off.p, (size_t)(nb + 1) * 4, cudaMemcpyDeviceToHost, s));
    FE_CK(cudaStreamSynchronize(s));
    std::vector<int64_t>& so = pl->seg_off[k];
    so.assign(h.begin(), h.end());
    const int64_t npos = so[(size_t)pl->nlev[k]];
    pl->seg_len[k] = npos;
    pl->perm_identity[k] = ident;
    st = pl->d_key[k].ensure((size_t)std::max<int64_t>(npos, 1) * 4);
    if (!st && !ident) st = pl->d_perm[k].ensure((size_t)std::max<int64_t>(npos, 1) * 4);
    if (st) return st;
    if (npos) {
      FE_CK(cudaMemcpyAsync(pl->d_key[k].p, sk, (size_t)npos * 4, cudaMemcpyDeviceToDevice, s));
      if (!ident)
        FE_CK(cudaMemcpyAsync(pl->d_perm[k].p, perm, (size_t)npos * 4, cudaMemcpyDeviceToDevice, s));
    }
    FE_CK(cudaStreamSynchronize(s));  // the sort buffers are reused
  }

  // interactions in sorted order
  pl->interacted.assign(K, false);
  pl->d_inter_sorted.resize(K);
  DevBuf tmp;
  for (int k = 0; k < K; ++k) {
    if (!interaction || !interaction[k]) continue;
    pl->interacted[k] = true;
    st = pl->d_inter_sorted[k].ensure((size_t)std::max<int64_t>(N, 1) * 8);
    if (!st) st = tmp.ensure((size_t)std::max<int64_t>(N, 1) * 8);
    if (st) return st;
    if (!N) continue;
    FE_CK(cudaMemcpyAsync(tmp.p, interaction[k], (size_t)N * 8, cudaMemcpyHostToDevice, s));
    k_gather_f64<<<blocks_of(N, 256), 256, 0, s>>>(tmp.as<double>(), pl->d_obs_src.as<int32_t>(), N,
                                                   pl->d_inter_sorted[k].as<double>());
    FE_CK(cudaGetLastError());
    FE_CK(cudaStreamSynchronize(s));
  }
  return 0;
}

}  // namespace fe

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int fe_group_keys(const int64_t* const* keys, int32_t n_keys, int64_t n, int32_t device,
                             int64_t* refs_out, int64_t* n_levels_out) {
  fe::DeviceRestore restore_device;
  using namespace fe;
  if (!keys || n_keys < 1 || n < 0 || !refs_out || !n_levels_out) {
    set_error("group_keys: need at least one key vector, n >= 0 and output pointers");
    return FE_ERR_INVALID;
  }
  if (n >= (int64_t)INT32_MAX) {
    set_error("group_keys: more than 2^31-1 observations is not supported");
    return FE_ERR_INVALID;
  }
  for (int j = 0; j < n_keys; ++j)
    if (n > 0 && !keys[j]) {
      set_error("group_keys: keys[" + std::to_string(j) + "] is null");
      return FE_ERR_INVALID;
    }
  *n_levels_out = 0;
  if (n == 0) return 0;
  FE_CK(cudaSetDevice(device));
  cudaStream_t s;
  FE_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  DevBuf a64, cur, nxt;
  int st = a64.ensure((size_t)n * 8);
  if (!st) st = cur.ensure((size_t)n * 4);
  if (!st) st = nxt.ensure((size_t)n * 4);
  if (st) return st;
  // the first key, then each further key folded in lexicographically:
  // (id so far, id of the key) -> id so far * levels of the key + id of the key
  FE_CK(cudaMemcpyAsync(a64.p, keys[0], (size_t)n * 8, cudaMemcpyHostToDevice, s));
  int64_t ncur = 0;
  st = group_dev(a64.as<int64_t>(), n, cur.as<int32_t>(), &ncur, s);
  if (st) return st;
  for (int j = 1; j < n_keys; ++j) {
    FE_CK(cudaMemcpyAsync(a64.p, keys[j], (size_t)n * 8, cudaMemcpyHostToDevice, s));
    int64_t nj = 0;
    st = group_dev(a64.as<int64_t>(), n, nxt.as<int32_t>(), &nj, s);
    if (st) return st;
    k_fold<<<blocks_of(n, 256), 256, 0, s>>>(cur.as<int32_t>(), nxt.as<int32_t>(), nj, n,
                                             a64.as<int64_t>());
    FE_CK(cudaGetLastError());
    st = group_dev(a64.as<int64_t>(), n, cur.as<int32_t>(), &ncur, s);
    if (st) return st;
  }
  k_to_refs<<<blocks_of(n, 256), 256, 0, s>>>(cur.as<int32_t>(), n, a64.as<int64_t>());
  FE_CK(cudaGetLastError());
  FE_CK(cudaMemcpyAsync(refs_out, a64.p, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  FE_CK(cudaStreamSynchronize(s));
  *n_levels_out = ncur;
  return 0;
}
