"""normalize! and full on the device (fe_normalize_coefficients,
fe_full_coefficients) against the host restatement of src/FixedEffect.jl:57-140
and, through solve_coefficients!, against the oracle's normalized
coefficients."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _blocks_problem(fe, rng, N=20_000):
    # two disconnected blocks of levels for the three plain FEs, a fourth FE
    # with an interaction (left alone by normalize!), and unobserved levels
    blk = rng.random(N) < 0.5
    r1 = np.where(blk, rng.integers(1, 300, N), rng.integers(400, 700, N))
    r2 = np.where(blk, rng.integers(1, 50, N), rng.integers(60, 90, N))
    r3 = np.where(blk, rng.integers(1, 5, N), rng.integers(6, 9, N))
    r4 = rng.integers(1, 30, N)
    fes = [fe.FixedEffect.from_refs(r1, 720), fe.FixedEffect.from_refs(r2, 95),
           fe.FixedEffect.from_refs(r3, 10),
           fe.FixedEffect.from_refs(r4, 29, rng.uniform(0.5, 1.5, N))]
    return fes


def test_device_normalize_matches_host_restatement(fe):
    rng = np.random.default_rng(31)
    fes = _blocks_problem(fe, rng)
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64)
    coefs = [rng.standard_normal(f.n) * 3.0 for f in fes]
    dev = feM.normalize_coefficients([c.copy() for c in coefs])
    dev2 = feM.normalize_coefficients([c.copy() for c in coefs])
    host = fe.normalize([c.copy() for c in coefs], fes)
    for a, b, c in zip(dev, host, coefs):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(c))
    for a, b in zip(dev, dev2):  # deterministic
        assert np.array_equal(a, b)
    # the interacted FE is untouched
    assert np.array_equal(dev[3], coefs[3])
    full_d = feM.full_coefficients(dev)
    full_h = fe.full(dev, fes)
    for a, b in zip(full_d, full_h):
        assert np.array_equal(a, b)
    feM.close()


def test_normalized_coefficients_vs_oracle(fe, oracle):
    # the normalized coefficients are unique: compare them FE by FE
    rng = np.random.default_rng(32)
    N = 30_000
    r1 = rng.integers(1, 2000, N)
    r2 = rng.integers(1, 200, N)
    r3 = rng.integers(1, 12, N)
    refs = [r1, r2, r3]
    y = rng.standard_normal(N) + rng.standard_normal(2000)[r1 - 1] + rng.standard_normal(200)[r2 - 1]
    lv_o, full_o, _, cv_o = oracle.solve_coefficients(y, refs, None, None, None, tol=1e-10)
    assert cv_o
    fes = [fe.FixedEffect(r) for r in refs]
    full_g, _, cv = fe.solve_coefficients(y.copy(), fes, double_precision=True, tol=1e-10)
    assert cv
    for a, b in zip(full_g, full_o):
        assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b)
