// fe_exdm_pipe.cu -- instantiations and launch of the pipelined fused
// expand + demean kernel of the absorbed loop (fe_exdm_pipe.cuh).
#include <cuda_runtime.h>

#include "fe_exdm_pipe.cuh"
#include "fe_plan.h"

namespace fe {

namespace {

template <int NL, int NS, bool W, int STG, bool PG, bool ATOM = false, int WARPS = kWarps>
int launch_one(const ExdmLaunch& a) {
  auto kern = k_exdm_pipe<NL, NS, W, STG, PG, ATOM, WARPS>;
  // per instantiation and device: the opt-in size set so far (0: none).  The
  // size only grows; the mutex keeps two threads from setting it out of order.
  static std::atomic<size_t> attr_smem[kDeviceSlots];
  static std::mutex attr_mu;
  const int dev = current_device();
  const bool slot = dev >= 0 && dev < kDeviceSlots;
  if (!slot || a.smem > attr_smem[dev].load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lock(attr_mu);
    if (!slot || a.smem > attr_smem[dev].load(std::memory_order_acquire)) {
      FE_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem));
      // the largest shared-memory carve-out, so that the CTAs the grid counts
      // on (up to three of 4 warps) are resident together
      FE_CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
      if (slot) attr_smem[dev].store(a.smem, std::memory_order_release);
    }
  }
  kern<<<(unsigned)a.grid, WARPS * 32, a.smem, a.stream>>>(a.d, a.items, a.n_items, a.tab,
                                                          a.rows, a.inst, a.rs, a.sr, a.lf,
                                                          a.part, a.S);
  FE_CK(cudaGetLastError());
  return 0;
}

template <int NL, int NS, bool W>
int launch_cfg(const ExdmLaunch& a, int cfg, bool atomic) {
  if constexpr (NL == 1) {
    if (atomic) return launch_one<NL, NS, W, 2, true, true>(a);
  }
  if (cfg == 3) return launch_one<NL, NS, W, 2, false, false, 4>(a);
  return cfg == 2 ? launch_one<NL, NS, W, 2, false>(a) : launch_one<NL, NS, W, 2, true>(a);
}

}  // namespace

int launch_exdm_pipe(const ExdmLaunch& a, int nl, int ns, bool w, int cfg, bool atomic) {
  switch ((nl * 3 + ns) * 2 + (w ? 1 : 0)) {
    case 0: return launch_cfg<0, 0, false>(a, cfg, atomic);
    case 1: return launch_cfg<0, 0, true>(a, cfg, atomic);
    case 2: return launch_cfg<0, 1, false>(a, cfg, atomic);
    case 3: return launch_cfg<0, 1, true>(a, cfg, atomic);
    case 4: return launch_cfg<0, 2, false>(a, cfg, atomic);
    case 5: return launch_cfg<0, 2, true>(a, cfg, atomic);
    case 6: return launch_cfg<1, 0, false>(a, cfg, atomic);
    case 7: return launch_cfg<1, 0, true>(a, cfg, atomic);
    case 8: return launch_cfg<1, 1, false>(a, cfg, atomic);
    case 9: return launch_cfg<1, 1, true>(a, cfg, atomic);
    case 10: return launch_cfg<1, 2, false>(a, cfg, atomic);
    default: return launch_cfg<1, 2, true>(a, cfg, atomic);
  }
}

}  // namespace fe
