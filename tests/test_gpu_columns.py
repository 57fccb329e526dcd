"""The collection form of solve_residuals! (src/AbstractFixedEffectSolver.jl:74-97)
through fe_solve_residuals_columns: separate host vectors, batched like the
columns of a matrix.  Pinned columns take the tile-pipelined transfers
(uploads and downloads overlapped with the other tiles' solves), pageable
ones the tile-by-tile copies; every form must give the matrix path's
residuals bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,T", [(np.float32, np.float32), (np.float64, np.float64)])
def test_columns_match_matrix_bitwise(fe, synth, dtype, T):
    import torch
    pb = synth.make(2, scale=0.01, ncols=40)        # two tiles: 32 + 8 columns
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", T)
    Y = np.asfortranarray(pb.Y.astype(dtype))
    R, its, cvs = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    # pageable columns (copies: a column of the Fortran-ordered Y is itself a
    # contiguous view, and the solve works in place)
    cols = [Y[:, j].copy() for j in range(Y.shape[1])]
    out, its_c, cvs_c = feM.solve_residuals(cols, tol=1e-8)
    assert out is cols
    for j in range(Y.shape[1]):
        assert np.array_equal(cols[j], R[:, j])
    assert list(its) == its_c and list(cvs) == cvs_c
    # pinned columns (page-locked host memory from torch)
    pinned = []
    for j in range(Y.shape[1]):
        t = torch.empty(Y.shape[0], dtype=torch.float32 if dtype == np.float32 else torch.float64,
                        pin_memory=True)
        a = t.numpy()
        a[:] = Y[:, j]
        pinned.append(a)
    _, its_p, _ = feM.solve_residuals(pinned, tol=1e-8)
    bad = [(j, int(np.sum(pinned[j] != R[:, j])), float(np.max(np.abs(pinned[j] - R[:, j]))))
           for j in range(Y.shape[1]) if not np.array_equal(pinned[j], R[:, j])]
    assert not bad, (bad[:6], its_p, list(its))
    assert its_p == its_c
    # a pinned matrix through fe_solve_residuals takes the same pipelined path
    tm = torch.empty((Y.shape[1], Y.shape[0]), dtype=torch.float32 if dtype == np.float32
                     else torch.float64, pin_memory=True)
    M = tm.numpy().T            # column-major view of pinned memory
    M[...] = Y
    Rm, _, _ = feM.solve_residuals(M, tol=1e-8)
    assert np.array_equal(Rm, R)
    feM.close()


def test_columns_mixed_types_and_readonly(fe, synth):
    pb = synth.make(2, scale=0.004, ncols=3)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64)
    Y = np.asfortranarray(pb.Y.astype(np.float64))
    R, _, _ = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    ro = Y[:, 2].copy()
    ro.flags.writeable = False
    cols = [Y[:, 0].copy(), Y[:, 1].copy(), ro]
    out, its, cvs = feM.solve_residuals(cols, tol=1e-8)
    assert np.array_equal(out[0], R[:, 0]) and np.array_equal(out[1], R[:, 1])
    assert out[2] is not ro and np.array_equal(out[2], R[:, 2])
    assert all(cvs)
    with pytest.raises(ValueError):
        feM.solve_residuals([Y[:-1, 0]], tol=1e-8)
    feM.close()


def test_pageable_staging_ring_multi_chunk(fe):
    """Pageable columns longer than one pinned ring slot (16 MB), over two
    tiles (32 + 1 columns): the staged uploads and downloads give the
    device-resident solve's residuals bit for bit."""
    import torch
    rng = np.random.default_rng(12)
    N = 2_200_000  # 17.6 MB per FP64 column: two ring chunks
    r1 = rng.integers(1, 200_001, N)
    r2 = rng.integers(1, 31, N)
    fes = [fe.FixedEffect(r1), fe.FixedEffect(r2)]
    Y = np.asfortranarray(rng.standard_normal((N, 33)))
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    D = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t()
    Dr, its_d, _ = feM.solve_residuals(D, tol=1e-8)
    Rd = Dr.cpu().numpy()
    P = Y.copy(order="F")  # pageable
    R, its, cvs = feM.solve_residuals(P, tol=1e-8)
    feM.close()
    assert cvs.all()
    assert np.array_equal(R, Rd)
    assert np.array_equal(its, its_d)
