"""Host-side fault cases of the C ABI: NaN input, a failed device allocation
(injected on the host, no GPU fault), and the caller's current device left as
it was after successful and failing calls."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small(fe, synth, scale=0.003):
    pb = synth.make(2, scale=scale, ncols=32)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    return pb, fes


@pytest.mark.parametrize("prec,ncols", [("mixed", 32), ("fp64", 3)])
def test_nan_column_stops_unconverged_and_leaves_others_alone(fe, synth, prec, ncols):
    """A column holding NaN: the reference runs maxiter iterations on NaN
    norms and returns converged = false with NaN residuals.  Here the column
    stops at once with the same verdict, its residuals are not finite, and the
    other columns of the tile are solved exactly as without it."""
    pb, fes = _small(fe, synth)
    Y = np.asfortranarray(pb.Y[:, :ncols].astype(np.float64))
    Ybad = Y.copy()
    Ybad[5, 1] = np.nan
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64, precision=prec)
    try:
        R, its, cvs = feM.solve_residuals(Ybad.copy(), tol=1e-8, maxiter=10000)
        R0, its0, cvs0 = feM.solve_residuals(Y.copy(), tol=1e-8, maxiter=10000)
    finally:
        feM.close()
    assert not cvs[1]
    assert np.isnan(R[5, 1])
    assert its[1] <= 2, its[1]  # stopped at once, not after maxiter iterations
    others = [j for j in range(ncols) if j != 1]
    assert cvs[others].all()
    for j in others:
        assert np.allclose(R[:, j], R0[:, j], rtol=1e-12, atol=0), j
        assert its[j] == its0[j]


def test_injected_allocation_failure_is_reported(fe, synth, monkeypatch):
    """FE_B200_FAIL_ALLOC_BYTES makes every device allocation of at least that
    many bytes fail like an out-of-memory cudaMalloc: the call returns
    FE_ERR_ALLOC with a message, nothing crashes, and the plan stays usable."""
    pb, fes = _small(fe, synth, scale=0.05)  # N = 500k
    L = fe._lib.load()
    # plan construction: the refs alone are 2 MB per fixed effect
    monkeypatch.setenv("FE_B200_FAIL_ALLOC_BYTES", str(1 << 20))
    with pytest.raises(RuntimeError) as ei:
        fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    assert "injected" in str(ei.value)
    monkeypatch.delenv("FE_B200_FAIL_ALLOC_BYTES")
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    try:
        # the solve's 32-column workspace (N x 32 x 8 bytes = 128 MB per slab)
        monkeypatch.setenv("FE_B200_FAIL_ALLOC_BYTES", str(64 << 20))
        Y = np.asfortranarray(pb.Y.astype(np.float64))
        its = np.zeros(32, dtype=np.int64)
        cvs = np.zeros(32, dtype=np.uint8)
        st = L.fe_solve_residuals(feM._h, Y.ctypes.data, fe._lib.FE_DTYPE_F64, 32, pb.N,
                                  fe._lib.FE_PREC_MIXED, 1e-8, 10000,
                                  its.ctypes.data_as(fe._lib._i64p), cvs.ctypes.data_as(fe._lib._u8p))
        assert st == fe._lib.FE_ERR_ALLOC
        assert b"injected" in L.fe_last_error()
        monkeypatch.delenv("FE_B200_FAIL_ALLOC_BYTES")
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8, maxiter=10000)
        assert cvs.all()
    finally:
        feM.close()


def test_current_device_unchanged(fe, synth):
    """Calls leave the caller's current device as they found it, whether they
    succeed or fail (a bad device ordinal)."""
    import torch
    n = torch.cuda.device_count()
    torch.cuda.set_device(0)
    pb, fes = _small(fe, synth, scale=0.001)
    L = fe._lib.load()
    refs = [np.ascontiguousarray(r, dtype=np.int64) for r in pb.refs]
    nl = np.ascontiguousarray(pb.nlev, dtype=np.int64)
    pp = (ctypes.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    h = ctypes.c_void_p()
    st = L.fe_plan_create(ctypes.byref(h), pb.N, len(refs), pp, nl.ctypes.data_as(fe._lib._i64p),
                          None, None, n)
    assert st == fe._lib.FE_ERR_INVALID
    assert torch.cuda.current_device() == 0
    target = 1 if n > 1 else 0
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64, device=target)
    try:
        assert torch.cuda.current_device() == 0
        R, its, cvs = feM.solve_residuals(np.asfortranarray(pb.Y[:, :2].astype(np.float64)),
                                          tol=1e-8)
        assert cvs.all()
        assert torch.cuda.current_device() == 0
        st = L.fe_plan_set_option(feM._h, 9999, 0.0)
        assert st == fe._lib.FE_ERR_INVALID
        assert torch.cuda.current_device() == 0
    finally:
        feM.close()
    assert torch.cuda.current_device() == 0
