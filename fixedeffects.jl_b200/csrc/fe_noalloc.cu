// fe_noalloc.cu -- fe_plan_scales_noalloc: the Jacobi preconditioner of one
// fixed effect recomputed without any device allocation.
//
// Who needs it: a caller that must not call cudaMalloc at that moment.  The
// typical one owns the device heap itself: Julia's CUDA.jl hands out device
// memory from its own pool, and a cudaMalloc behind its back can fail once
// the pool holds the free memory, or breaks the memory budget the caller set.
// fe_plan_update_weights allocates its level-sum and piece-partial scratch on
// every call; this entry point keeps that scratch in one file-scope device
// array instead.
//
// The array is a fixed kNoAllocScratchBytes (8 MiB) per device, held from the
// moment the library is loaded until the process exits.  Every call shares
// it and it keeps the last call's contents, so each call clears what must
// start at zero; calls that overlap on the GPU (different streams, or
// different host threads) race on it and must be serialized by the caller.
#include <cuda_runtime.h>

#include "../../include/fe_b200.h"
#include "fe_kernels.cuh"
#include "fe_plan.h"

namespace fe {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)FE_NOALLOC_SCRATCH_BYTES;
static_assert(kNoAllocScratchBytes % 256 == 0, "scratch size");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol is only a host-side stand-in; the device address comes from
// cudaGetSymbolAddress with the plan's device current.  It is looked up on
// every call (no allocation, a few microseconds), so a device reset, after
// which the module and the array may be loaded at another address, leaves
// no stale pointer behind.
int scratch_address(void** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    (void)cudaGetLastError();
    set_error_cstr("fe_plan_scales_noalloc: cudaGetSymbolAddress of the scratch array failed");
    return FE_ERR_CUDA;
  }
  *out = p;
  return FE_OK;
}

// The level-sum kernel of the preconditioner (k_segsum with LoadScaleSq,
// C = 1) restricted to the items of one FE: sums of interaction^2 * w per
// level into sums[level] (FE-local), long levels through piece partials.
template <int U>
__global__ void __launch_bounds__(kThreads)
k_segsum_scale_one_fe(const FeDev d, const ReduceItem* __restrict__ items, int64_t n_items,
                      int fe, double* __restrict__ sums, SplitArgs sa) {
  using Sh = Shape<double, 1>;
  constexpr int VEC = Sh::VEC, CL = Sh::CL, G = Sh::G;
  constexpr int STEP = G * U;
  constexpr int NI = STEP >= 32 ? STEP / 32 : 1;
  static_assert(STEP <= 32 || STEP % 32 == 0, "a step's indices fill whole index registers");
  __shared__ double smt[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int g = lane / CL, jl = lane - g * CL;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (w >= n_items) return;
  const ReduceItem it = items[w];
  if (it.fe != fe || it.pe <= it.pb) return;
  const int32_t* __restrict__ perm = d.perm[fe];
  const int32_t* __restrict__ key = d.key[fe];
  const double* __restrict__ cwp = d.cwp_d[fe];
  SegRun<double, VEC, CL, G> run;
  run.init();
  for (int64_t base = it.pb; base < it.pe; base += STEP) {
    int kl[NI];
    double cl[NI];
#pragma unroll
    for (int r = 0; r < NI; ++r) {
      const int64_t p = base + r * 32 + lane;
      const bool ok = p < it.pe && (r * 32 + lane) < STEP;
      kl[r] = ok ? __ldg(key + p) : kSentinel;
      double c = 1.0;
      if (ok && cwp) c = __ldg(cwp + p);
      cl[r] = c * c;
    }
    (void)perm;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t b0 = base + (int64_t)u * G;
      if (b0 >= it.pe) break;  // warp-uniform
      const int q = u * G;
      const int src = (q & 31) + g;
      const int km = __shfl_sync(FE_FULL, kl[q >> 5], src);
      const double c = __shfl_sync(FE_FULL, cl[q >> 5], src);
      VA<double, VEC> x;
      x.v[0] = km != kSentinel ? c : 0.0;
      const int nvalid = (int)((it.pe - b0) < G ? (it.pe - b0) : G);
      run.push(km, x, nvalid, g, jl, 1, sums);
    }
  }
  run.finish(it.split, it.pad, sa, g, jl, 1, sums, smt[threadIdx.x >> 5]);
}

// scale = 1/sqrt(sum), or 0 for an empty sum (src/SolverCPU.jl:84-88)
__global__ void k_scale_from_sums(const double* __restrict__ sums, int64_t n,
                                  double* __restrict__ out) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n) {
    const double s = sums[l];
    out[l] = s > 0 ? 1.0 / sqrt(s) : 0.0;
  }
}

}  // namespace
}  // namespace fe

extern "C" int fe_plan_scales_noalloc(fe_plan* plan, int32_t fe_index, double* scale_out_dev,
                                      void* stream) {
  fe::DeviceRestore restore_device;
  using namespace fe;
  if (!plan) {
    set_error_cstr("fe_plan_scales_noalloc: plan is NULL");
    return FE_ERR_INVALID;
  }
  if (fe_index < 0 || fe_index >= plan->K) {
    set_error_cstr("fe_plan_scales_noalloc: fe_index out of range");
    return FE_ERR_INVALID;
  }
  const int64_t nlev = plan->nlev[fe_index];
  if (nlev == 0) return FE_OK;
  if (!scale_out_dev) {
    set_error_cstr("fe_plan_scales_noalloc: scale_out_dev is NULL");
    return FE_ERR_INVALID;
  }
  auto f = plan->items.find(1);  // built when the plan was created
  if (f == plan->items.end()) {
    set_error_cstr("fe_plan_scales_noalloc: the plan has no single-column work items");
    return FE_ERR_INVALID;
  }
  const ItemSet* its = f->second.get();
  // scratch layout: [level sums | piece partials | block partials |
  //                  level counters | block counters]
  const size_t sums_bytes = ((size_t)nlev * sizeof(double) + 255) & ~(size_t)255;
  const size_t piece_bytes = (((size_t)its->n_pieces) * sizeof(double) + 255) & ~(size_t)255;
  const size_t block_bytes = (((size_t)its->n_blocks) * sizeof(double) + 255) & ~(size_t)255;
  const size_t cnt_bytes = (its->splits.size() * sizeof(int32_t) + 255) & ~(size_t)255;
  const size_t bcnt_bytes = (((size_t)its->n_blocks) * sizeof(int32_t) + 255) & ~(size_t)255;
  if (sums_bytes + piece_bytes + block_bytes + cnt_bytes + bcnt_bytes > kNoAllocScratchBytes) {
    set_error_cstr(
        "fe_plan_scales_noalloc: the fixed effect needs more scratch than FE_NOALLOC_SCRATCH_BYTES "
        "(8 MiB: its level sums, about 1e6 levels at most, plus the piece partials of the long "
        "levels of every fixed effect of the plan); use fe_plan_update_weights/fe_plan_get_scales");
    return FE_ERR_INVALID;
  }
  if (cudaSetDevice(plan->device) != cudaSuccess) {
    (void)cudaGetLastError();
    set_error_cstr("fe_plan_scales_noalloc: cudaSetDevice failed");
    return FE_ERR_CUDA;
  }
  void* base = nullptr;
  int st = scratch_address(&base);
  if (st) return st;
  unsigned char* b = static_cast<unsigned char*>(base);
  double* sums = reinterpret_cast<double*>(b);
  double* pieces = reinterpret_cast<double*>(b + sums_bytes);
  double* blocks = reinterpret_cast<double*>(b + sums_bytes + piece_bytes);
  int32_t* cnt = reinterpret_cast<int32_t*>(b + sums_bytes + piece_bytes + block_bytes);
  int32_t* bcnt = reinterpret_cast<int32_t*>(b + sums_bytes + piece_bytes + block_bytes + cnt_bytes);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
  // a caller stream runs after the work already queued on the plan's stream
  // (fe_plan_update_weights rewrites the weight arrays read here): an event
  // recorded there and waited on here, created on the plan's first call
  if (s != plan->stream) {
    cudaError_t eo = cudaSuccess;
    if (!plan->noalloc_order)
      eo = cudaEventCreateWithFlags(&plan->noalloc_order, cudaEventDisableTiming);
    if (eo == cudaSuccess) eo = cudaEventRecord(plan->noalloc_order, plan->stream);
    if (eo == cudaSuccess) eo = cudaStreamWaitEvent(s, plan->noalloc_order, 0);
    if (eo != cudaSuccess) {
      (void)cudaGetLastError();
      set_error_cstr("fe_plan_scales_noalloc: ordering after the plan's stream failed");
      return FE_ERR_CUDA;
    }
  }
  // levels without positions are never written by the sum kernel and the
  // split counters must start at zero: clear both (the array keeps the
  // previous call's contents)
  cudaError_t e = cudaMemsetAsync(sums, 0, (size_t)nlev * sizeof(double), s);
  if (e == cudaSuccess && !its->splits.empty())
    e = cudaMemsetAsync(cnt, 0, its->splits.size() * sizeof(int32_t), s);
  if (e == cudaSuccess && its->n_blocks > 0)
    e = cudaMemsetAsync(bcnt, 0, (size_t)its->n_blocks * sizeof(int32_t), s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error_cstr("fe_plan_scales_noalloc: cudaMemsetAsync failed");
    return FE_ERR_CUDA;
  }
  FeDev d = plan->dev;
  d.C = 1;
  const int64_t n_items = (int64_t)its->rd.size();
  if (n_items > 0) {
    const unsigned grid = (unsigned)((n_items + kWarps - 1) / kWarps);
    SplitArgs sa{its->d_splits.as<SplitLevel>(), pieces, its->n_pieces, blocks, its->n_blocks, cnt,
                 bcnt};
    k_segsum_scale_one_fe<8><<<grid, kThreads, 0, s>>>(d, its->d_rd.as<ReduceItem>(), n_items,
                                                        fe_index, sums, sa);
  }
  k_scale_from_sums<<<(unsigned)((nlev + 255) / 256), 256, 0, s>>>(sums, nlev, scale_out_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_cstr("fe_plan_scales_noalloc: kernel launch failed");
    return FE_ERR_CUDA;
  }
  return FE_OK;
}
