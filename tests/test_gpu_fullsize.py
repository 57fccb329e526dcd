"""The reference's workloads at full size, checked through properties that do
not depend on size (the oracle finishes only reduced sizes in seconds):

* orthogonality: the residual r of solve_residuals! satisfies the normal
  equations, sum over the rows of each level of w_i r_i = 0 for every FE
  (src/AbstractFixedEffectSolver.jl:49-68); checked here in numpy, FP64,
  independently of the library;
* idempotence: solving a residual again returns it;
* linearity: the residual of a sum of columns is the sum of the residuals.

Workloads: 10M observations with worker/firm/year FEs and 32 Float32
columns; 100M observations with 1e7 uniform and 1e4 Zipf(1.3) levels,
weighted, 8 columns; 256 independent problems of 1e3..1e6 observations.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# The FP64 test stops at ||D A'r|| <= tol ||A D|| ||r|| with tol = 1e-8, and
# LSMR's estimate of ||A D|| grows with the number of levels, so the level
# sums scaled like the Jacobi preconditioner are bounded by 1e-4 here (a
# random vector gives about 1).
ORTH = 1e-4


def _orth_ratio(r, refs, nlev, w):
    """max over FEs of ||A_k' W r|| / ||W^(1/2) r||: about 1 for a random r, 0
    for a residual of the normal equations."""
    rw = r.astype(np.float64) * (w if w is not None else 1.0)
    den = np.sqrt(np.dot(rw, r.astype(np.float64)))
    worst = 0.0
    for ref, n in zip(refs, nlev):
        s = np.bincount(ref - 1, weights=rw, minlength=n)
        if w is not None:
            s = s / np.sqrt(np.bincount(ref - 1, weights=w, minlength=n) + 1e-300)
        else:
            s = s / np.sqrt(np.maximum(np.bincount(ref - 1, minlength=n), 1))
        worst = max(worst, float(np.linalg.norm(s) / den))
    return worst


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b.astype(np.float64)))


def test_worker_firm_year_10m_32col(fe, synth):
    pb = synth.config2(scale=1.0, ncols=32)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32, precision="mixed")
    R, its, cvs = feM.solve_residuals(pb.Y.copy(order="F"), tol=1e-8, maxiter=10000)
    info = feM.last_solve_info(32)
    assert cvs.all() and info["test2"].max() <= 1e-8, (its, info["test2"].max())
    for j in (0, 13, 31):
        ratio = _orth_ratio(R[:, j], pb.refs, pb.nlev, None)
        assert ratio < ORTH, (j, ratio)
    # idempotence: the residuals are their own residuals
    R2, its2, cvs2 = feM.solve_residuals(R.copy(order="F"), tol=1e-8, maxiter=10000)
    assert cvs2.all(), its2
    assert max(_rel(R2[:, j], R[:, j]) for j in range(32)) < 1e-6
    # linearity (16 columns take the non-absorbed path, 32 the absorbed one)
    Ys = np.asfortranarray(pb.Y[:, :16] + pb.Y[:, 16:])
    Rs, _, cvs3 = feM.solve_residuals(Ys, tol=1e-8, maxiter=10000)
    assert cvs3.all()
    assert max(_rel(Rs[:, j], R[:, j] + R[:, 16 + j]) for j in range(16)) < 1e-6
    feM.close()


def test_large_zipf_100m_8col(fe, synth):
    pb = synth.config4(scale=1.0, ncols=8)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float32, precision="mixed")
    R, its, cvs = feM.solve_residuals(pb.Y.copy(order="F"), tol=1e-8, maxiter=10000)
    info = feM.last_solve_info(8)
    assert cvs.all() and info["test2"].max() <= 1e-8, (its, info["test2"].max())
    for j in (0, 7):
        ratio = _orth_ratio(R[:, j], pb.refs, pb.nlev, pb.weights)
        assert ratio < ORTH, (j, ratio)
    R2, its2, cvs2 = feM.solve_residuals(R[:, :2].copy(order="F"), tol=1e-8, maxiter=10000)
    assert cvs2.all(), its2
    assert max(_rel(R2[:, j], R[:, j]) for j in range(2)) < 1e-6
    feM.close()


def test_uneven_problems_256(fe, synth):
    probs = synth.config3(scale=1.0)
    bs = fe.BatchSolver([[fe.FixedEffect.from_refs(r, n, a) for r, n, a in
                          zip(p.refs, p.nlev, p.interaction)] for p in probs],
                        weights=[p.weights for p in probs], T=np.float32, precision="mixed")
    rs, its, cvs = bs.solve_residuals([p.Y[:, 0] for p in probs], tol=1e-8, maxiter=10000)
    assert cvs.all(), its
    for i in (0, 17, 101, 255):
        p = probs[i]
        # FEs with an interaction are left out (their normal equations weight
        # the rows by the interaction too)
        w = p.weights
        refs = [r for r, a in zip(p.refs, p.interaction) if a is None]
        nlev = [n for n, a in zip(p.nlev, p.interaction) if a is None]
        ratio = _orth_ratio(rs[i], refs, nlev, w)
        assert ratio < ORTH, (i, ratio)
    bs.close()
