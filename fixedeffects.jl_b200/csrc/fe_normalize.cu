// fe_normalize.cu -- normalize! and full of FixedEffects.jl on the device
// (src/FixedEffect.jl:57-140), the post-processing of solve_coefficients!.
//
// normalize!: the coefficients of a fixed-effects fit are unique only up to
// one constant per FE per connected component of the observation/level graph.
// Within each component the reference demeans every non-interacted FE but the
// first and adds the means to the first (rescale!, :115-135).
//
// Components: the levels of the non-interacted FEs are the nodes; every
// observation links its levels.  Hooking with atomicMin on parent pointers and
// pointer jumping, repeated until a pass finds every observation's levels in
// one tree, leaves each node pointing at the smallest node id of its
// component: the labels do not depend on the order of the atomic updates.
// Parent pointers only decrease, so every walk to a root ends.
//
// Means: exact 64-bit fixed-point sums (integer atomics, order-independent)
// of the coefficients scaled by 2^e, e chosen per FE so that no sum can
// overflow; each mean is off by at most 2^-(e+1), under 1e-12 of the largest
// coefficient for a million levels.  The result is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/fe_b200.h"
#include "fe_internal.h"
#include "fe_plan.h"

namespace fe {
namespace {

struct NormFEs {
  const int32_t* refs[kMaxFE];  // sorted order, FE-local levels
  int64_t base[kMaxFE];         // node id of level 0
  int32_t nlev[kMaxFE];         // levels (a ref >= nlev is the null level)
  int32_t n;                    // FEs in the set
};

__device__ __forceinline__ int32_t cc_find(const int32_t* par, int32_t v) {
  // par[v] <= v everywhere, so the walk ends; the cap only bounds a bad input
  for (int s = 0; s < (1 << 24); ++s) {
    const int32_t p = par[v];
    if (p == v) break;
    v = p;
  }
  return v;
}

__global__ void k_cc_init(int32_t* par, int32_t* used, int64_t P) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < P) {
    par[v] = (int32_t)v;
    used[v] = 0;
  }
}

__global__ void k_cc_mark(NormFEs f, int64_t N, int32_t* used) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int j = 0; j < f.n; ++j) {
    const int32_t r = f.refs[j][i];
    if (r < f.nlev[j]) used[f.base[j] + r] = 1;
  }
}

// one hooking pass: every observation joins the trees of its levels
__global__ void k_cc_hook(NormFEs f, int64_t N, int32_t* par, int32_t* changed) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int32_t r0 = f.refs[0][i];
  if (r0 >= f.nlev[0]) return;
  int32_t a = cc_find(par, (int32_t)(f.base[0] + r0));
  for (int j = 1; j < f.n; ++j) {
    const int32_t r = f.refs[j][i];
    if (r >= f.nlev[j]) continue;
    const int32_t b = cc_find(par, (int32_t)(f.base[j] + r));
    if (a != b) {
      const int32_t hi = a > b ? a : b, lo = a > b ? b : a;
      atomicMin(par + hi, lo);
      *changed = 1;
      a = lo;
    }
  }
}

__global__ void k_cc_compress(int32_t* par, int64_t P) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < P) par[v] = cc_find(par, (int32_t)v);
}

// max |coef| over the observed levels of one FE (bit patterns of non-negative
// doubles order like the values)
__global__ void k_maxabs(const double* coef, int64_t n, const int32_t* used, int64_t base,
                         unsigned long long* out) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n && used[base + l]) {
    const double a = fabs(coef[l]);
    atomicMax(out, (unsigned long long)__double_as_longlong(a));
  }
}

__global__ void k_comp_sum(const double* coef, int64_t n, const int32_t* used, int64_t base,
                           const int32_t* par, double sc, long long* sum, int32_t* cnt) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n && used[base + l]) {
    const int32_t c = par[base + l];
    atomicAdd(reinterpret_cast<unsigned long long*>(sum + c),
              (unsigned long long)llrint(coef[l] * sc));
    atomicAdd(cnt + c, 1);
  }
}

// per component: mj = sum / count (0 without levels of this FE), m += mj;
// the sums are cleared for the next FE
__global__ void k_comp_mean(int64_t P, double inv_sc, long long* sum, int32_t* cnt, double* mj,
                            double* m) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= P) return;
  const int32_t c = cnt[v];
  double x = 0.0;
  if (c > 0) x = ((double)sum[v] * inv_sc) / (double)c;
  mj[v] = x;
  m[v] += x;
  sum[v] = 0;
  cnt[v] = 0;
}

__global__ void k_comp_apply(double* coef, int64_t n, const int32_t* used, int64_t base,
                             const int32_t* par, const double* add, double sign) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n && used[base + l]) coef[l] += sign * add[par[base + l]];
}

__global__ void k_full(const double* coef, const int32_t* refs_sorted, const int32_t* dst,
                       int32_t nlev, int64_t N, double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    const int32_t r = refs_sorted[dst[i]];
    out[i] = r < nlev ? coef[r] : 0.0;
  }
}

inline unsigned grid_of(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace
}  // namespace fe

using namespace fe;

extern "C" int fe_normalize_coefficients(fe_plan* plan, double* const* coefs,
                                         int32_t coefs_on_device) {
  fe::DeviceRestore restore_device;
  if (!plan || !coefs) {
    set_error_cstr("fe_normalize_coefficients: plan or coefs is NULL");
    return FE_ERR_INVALID;
  }
  if (plan->xchg) {
    // the connected components span every rank's observations
    set_error_cstr("fe_normalize_coefficients: not available for an observation-sharded plan "
                   "(the components need every rank's observations)");
    return FE_ERR_INVALID;
  }
  const int K = plan->K;
  for (int k = 0; k < K; ++k)
    if (!coefs[k] && plan->nlev[k] > 0) {
      set_error_cstr("fe_normalize_coefficients: coefs[k] is NULL");
      return FE_ERR_INVALID;
    }
  // the non-interacted FEs, in FE order (src/FixedEffect.jl:107-108)
  std::vector<int> idx;
  for (int k = 0; k < K; ++k)
    if (!plan->interacted[k]) idx.push_back(k);
  if (idx.size() < 2) return FE_OK;
  FE_CK(cudaSetDevice(plan->device));
  cudaStream_t s = plan->stream;
  const int64_t N = plan->N, P = plan->P;
  if (N == 0) return FE_OK;
  DevBuf par, used, sum, cnt, mj, m, flag, mx;
  std::vector<DevBuf> dcoef(K);
  int st = par.ensure((size_t)P * 4);
  if (!st) st = used.ensure((size_t)P * 4);
  if (!st) st = sum.ensure((size_t)P * 8);
  if (!st) st = cnt.ensure((size_t)P * 4);
  if (!st) st = mj.ensure((size_t)P * 8);
  if (!st) st = m.ensure((size_t)P * 8);
  if (!st) st = flag.ensure(4);
  if (!st) st = mx.ensure(8);
  if (st) return st;
  double* cf[kMaxFE] = {};
  for (int k : idx) {
    const int64_t n = plan->nlev[k];
    if (coefs_on_device) {
      cf[k] = coefs[k];
    } else if (n > 0) {
      if ((st = dcoef[k].ensure((size_t)n * 8))) return st;
      cf[k] = dcoef[k].as<double>();
      FE_CK(cudaMemcpyAsync(cf[k], coefs[k], (size_t)n * 8, cudaMemcpyHostToDevice, s));
    }
  }
  NormFEs f{};
  f.n = (int32_t)idx.size();
  for (int j = 0; j < f.n; ++j) {
    const int k = idx[(size_t)j];
    f.refs[j] = plan->d_refs[k].as<int32_t>();
    f.base[j] = plan->lev_base[k];
    f.nlev[j] = (int32_t)plan->nlev[k];
  }
  int32_t* dpar = par.as<int32_t>();
  int32_t* dused = used.as<int32_t>();
  k_cc_init<<<grid_of(P), 256, 0, s>>>(dpar, dused, P);
  k_cc_mark<<<grid_of(N), 256, 0, s>>>(f, N, dused);
  FE_CK(cudaGetLastError());
  // hook + compress until a pass changes nothing (bounded)
  int32_t changed = 1;
  int rounds = 0;
  for (; changed && rounds < 4096; ++rounds) {
    FE_CK(cudaMemsetAsync(flag.p, 0, 4, s));
    k_cc_hook<<<grid_of(N), 256, 0, s>>>(f, N, dpar, flag.as<int32_t>());
    k_cc_compress<<<grid_of(P), 256, 0, s>>>(dpar, P);
    FE_CK(cudaGetLastError());
    FE_CK(cudaMemcpyAsync(&changed, flag.p, 4, cudaMemcpyDeviceToHost, s));
    FE_CK(cudaStreamSynchronize(s));
  }
  if (changed) {
    set_error_cstr("fe_normalize_coefficients: connected components did not converge");
    return FE_ERR_CUDA;
  }
  FE_CK(cudaMemsetAsync(sum.p, 0, (size_t)P * 8, s));
  FE_CK(cudaMemsetAsync(cnt.p, 0, (size_t)P * 4, s));
  FE_CK(cudaMemsetAsync(m.p, 0, (size_t)P * 8, s));
  // demean every FE but the first, last to second (src/FixedEffect.jl:118-131)
  for (size_t jj = idx.size() - 1; jj >= 1; --jj) {
    const int k = idx[jj];
    const int64_t n = plan->nlev[k], base = plan->lev_base[k];
    if (n == 0) continue;
    FE_CK(cudaMemsetAsync(mx.p, 0, 8, s));
    k_maxabs<<<grid_of(n), 256, 0, s>>>(cf[k], n, dused, base, mx.as<unsigned long long>());
    unsigned long long bits = 0;
    FE_CK(cudaMemcpyAsync(&bits, mx.p, 8, cudaMemcpyDeviceToHost, s));
    FE_CK(cudaStreamSynchronize(s));
    double amax;
    memcpy(&amax, &bits, 8);
    if (!std::isfinite(amax)) {
      set_error_cstr("fe_normalize_coefficients: non-finite coefficient");
      return FE_ERR_INVALID;
    }
    // |sum| <= n * amax * 2^e <= 2^62
    int e = 0;
    if (amax > 0) e = (int)std::floor(62.0 - std::log2((double)n) - std::log2(amax)) - 1;
    e = std::min(e, 1000);  // 2^e stays finite for the tiniest coefficients
    const double sc = std::ldexp(1.0, e);
    k_comp_sum<<<grid_of(n), 256, 0, s>>>(cf[k], n, dused, base, dpar, sc, sum.as<long long>(),
                                          cnt.as<int32_t>());
    k_comp_mean<<<grid_of(P), 256, 0, s>>>(P, 1.0 / sc, sum.as<long long>(), cnt.as<int32_t>(),
                                           mj.as<double>(), m.as<double>());
    k_comp_apply<<<grid_of(n), 256, 0, s>>>(cf[k], n, dused, base, dpar, mj.as<double>(), -1.0);
    FE_CK(cudaGetLastError());
  }
  {
    const int k = idx[0];
    const int64_t n = plan->nlev[k];
    if (n > 0)
      k_comp_apply<<<grid_of(n), 256, 0, s>>>(cf[k], n, dused, plan->lev_base[k], dpar,
                                              m.as<double>(), 1.0);
    FE_CK(cudaGetLastError());
  }
  if (!coefs_on_device)
    for (int k : idx)
      if (plan->nlev[k] > 0)
        FE_CK(cudaMemcpyAsync(coefs[k], cf[k], (size_t)plan->nlev[k] * 8, cudaMemcpyDeviceToHost, s));
  FE_CK(cudaStreamSynchronize(s));
  return FE_OK;
}

extern "C" int fe_full_coefficients(fe_plan* plan, const double* const* coefs,
                                    int32_t coefs_on_device, double* const* out,
                                    int32_t out_on_device) {
  fe::DeviceRestore restore_device;
  if (!plan || !coefs || !out) {
    set_error_cstr("fe_full_coefficients: plan, coefs or out is NULL");
    return FE_ERR_INVALID;
  }
  const int K = plan->K;
  const int64_t N = plan->N;
  for (int k = 0; k < K; ++k)
    if (!out[k] || (!coefs[k] && plan->nlev[k] > 0)) {
      set_error_cstr("fe_full_coefficients: coefs[k] or out[k] is NULL");
      return FE_ERR_INVALID;
    }
  if (N == 0) return FE_OK;
  FE_CK(cudaSetDevice(plan->device));
  cudaStream_t s = plan->stream;
  DevBuf dc, dout;
  for (int k = 0; k < K; ++k) {
    const int64_t n = plan->nlev[k];
    const double* c = coefs[k];
    if (!coefs_on_device) {
      int st = dc.ensure((size_t)std::max<int64_t>(n, 1) * 8);
      if (st) return st;
      if (n > 0) FE_CK(cudaMemcpyAsync(dc.p, coefs[k], (size_t)n * 8, cudaMemcpyHostToDevice, s));
      c = dc.as<double>();
    }
    double* o = out[k];
    if (!out_on_device) {
      int st = dout.ensure((size_t)N * 8);
      if (st) return st;
      o = dout.as<double>();
    }
    k_full<<<grid_of(N), 256, 0, s>>>(c, plan->d_refs[k].as<int32_t>(), plan->d_obs_dst.as<int32_t>(),
                                      (int32_t)n, N, o);
    FE_CK(cudaGetLastError());
    if (!out_on_device)
      FE_CK(cudaMemcpyAsync(out[k], o, (size_t)N * 8, cudaMemcpyDeviceToHost, s));
    FE_CK(cudaStreamSynchronize(s));
  }
  return FE_OK;
}
