"""fe_plan_scales_noalloc: the allocation-free recomputation of one fixed
effect's Jacobi scales, for callers that cannot call cudaMalloc because the
device heap is not theirs to grow (a caller whose device memory belongs to its
own pool, such as Julia's CUDA.jl allocator).  Its output must equal what
fe_plan_get_scales returns for the same plan.

This file is collected last on purpose: it exercises a shared, fixed-size
device scratch array that keeps the previous call's contents."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan(fe, synth):
    pb = synth.make(1, scale=0.003)  # weighted; three FEs, the third interacted
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
    return fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64), fes


def test_scales_noalloc_matches_existing_entry_point(fe, synth):
    import torch
    feM, fes = _plan(fe, synth)
    ref = feM.scales()  # fe_plan_get_scales
    L = fe._lib.load()
    free_after_first = None
    for call in range(2):  # two calls in a row over every FE
        for k in range(len(fes)):
            out = torch.full((fes[k].n,), float("nan"), dtype=torch.float64, device="cuda")
            fe._lib.check(L.fe_plan_scales_noalloc(feM._h, k, ctypes.c_void_p(out.data_ptr()), None))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.allclose(got, ref[k], rtol=1e-13, atol=0), (call, k)
        free = torch.cuda.mem_get_info()[0]
        if free_after_first is None:
            free_after_first = free
        else:
            # the second round of calls took no device memory
            assert free >= free_after_first - (2 << 20)
    feM.close()


def test_scales_noalloc_rejects_oversized_fixed_effect(fe):
    L = fe._lib.load()
    n = 1_100_000  # level sums alone exceed the 8 MiB scratch
    rng = np.random.default_rng(0)
    r = np.concatenate([np.arange(1, n + 1), rng.integers(1, n + 1, 100_000)])
    g = rng.integers(1, 10, r.shape[0])
    feM = fe.AbstractFixedEffectSolver([fe.FixedEffect(r), fe.FixedEffect(g)], None, "CUDA", np.float64)
    import torch
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    st = L.fe_plan_scales_noalloc(feM._h, 0, ctypes.c_void_p(out.data_ptr()), None)
    assert st == fe._lib.FE_ERR_INVALID
    assert b"FE_NOALLOC_SCRATCH_BYTES" in L.fe_last_error()
    # the small fixed effect of the same plan still fits
    out2 = torch.empty(9, dtype=torch.float64, device="cuda")
    fe._lib.check(L.fe_plan_scales_noalloc(feM._h, 1, ctypes.c_void_p(out2.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.allclose(out2.cpu().numpy(), feM.scales()[1], rtol=1e-13, atol=0)
    feM.close()
