"""The oracle (CPU FP64 restatement of the reference) pinned against the
reference's golden vectors (test/solve.jl) and against scipy's independent
LSMR implementation of the same algorithm (Fong & Saunders)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def isapprox(a, b, rtol=np.sqrt(np.finfo(np.float64).eps)):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


@pytest.fixture(scope="module")
def g(golden):
    return {k: np.asarray(v) for k, v in golden.items() if isinstance(v, list)}


def test_golden_residuals(oracle, g):
    r, it, cv = oracle.solve_residuals(g["x"], [g["p1"], g["p2"]])
    assert cv
    assert isapprox(r, g["r_ols"])
    assert np.max(np.abs(r - g["r_ols"])) < 1e-13


def test_golden_coefficients(oracle, g):
    lv, full, it, cv = oracle.solve_coefficients(g["x"], [g["p1"], g["p2"]])
    assert cv
    assert isapprox(g["x"] - full[0] - full[1], g["r_ols"])


def test_golden_relabelled_refs(oracle, g):
    # PooledArray / CategoricalArray (test/solve.jl:19-24): relabelled levels
    perm1 = np.array([3, 1, 5, 2, 4])
    r, _, _ = oracle.solve_residuals(g["x"], [perm1[g["p1"] - 1], g["p2"]])
    assert isapprox(r, g["r_ols"])


def test_interacted_convergence(oracle, g):
    inter = g["interaction"]
    _, _, cv = oracle.solve_residuals(g["x"], [g["p1"]], interaction=[inter])
    assert cv
    _, _, cv = oracle.solve_residuals(g["x"], [g["p1"], g["p1"]], interaction=[None, inter])
    assert cv


def test_weights_round_trip(oracle, g):
    # the unasserted update_weights! lines of test/solve.jl:45-55, asserted:
    # a weighted single-FE solve is the weighted within-group demeaning
    for w in (np.arange(1, 11, dtype=float), np.arange(10, 0, -1, dtype=float)):
        r, it, cv = oracle.solve_residuals(g["x"], [g["p1"]], weights=w)
        m = np.zeros(6)
        np.add.at(m, g["p1"], w * g["x"])
        den = np.zeros(6)
        np.add.at(den, g["p1"], w)
        expect = g["x"] - (m / np.maximum(den, 1e-300))[g["p1"]]
        assert np.allclose(r, expect, atol=1e-14)
        assert it == 1 and cv


def _sparse_A(refs, nlev, inter, w, O):
    N = len(refs[0])
    sw = np.sqrt(w) if w is not None else np.ones(N)
    rows, cols, vals = [], [], []
    off = 0
    for k, r in enumerate(refs):
        a = None if inter is None else inter[k]
        sc = O.scale(r, nlev[k], a, w)
        rows.append(np.arange(N))
        cols.append(off + r - 1)
        vals.append((np.ones(N) if a is None else a) * sw * sc[r - 1])
        off += nlev[k]
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(N, off)), sw


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_lsmr_matches_scipy(oracle, seed):
    rng = np.random.default_rng(seed)
    N = 20000
    nlev = [2000, 50, 300]
    refs = [rng.integers(1, n + 1, N) for n in nlev]
    nlev = [int(r.max()) for r in refs]
    w = rng.uniform(0.5, 1.5, N) if seed % 2 else None
    inter = [None, None, rng.random(N)] if seed >= 2 else None
    y = rng.standard_normal(N) + refs[0] * 1e-3
    A, sw = _sparse_A(refs, nlev, inter, w, oracle)
    x, istop, itn = spl.lsmr(A, y * sw, atol=1e-8, btol=1e-8, conlim=1e8, maxiter=10000)[:3]
    lv, full, it, cv = oracle.solve_coefficients(y, refs, nlev, inter, w, tol=1e-8)
    assert cv and istop in (1, 2)
    assert it == itn // 2  # the reference reports div(mvps, 2)
    fit_o = sum(f * (1 if inter is None or inter[k] is None else inter[k]) for k, f in enumerate(full))
    A_fit = (A @ x) / sw
    assert np.max(np.abs(fit_o - A_fit)) < 1e-9


@pytest.mark.parametrize("problem", ["hard_800k", "hard_800k_interacted"])
def test_reference_benchmark_problems_match_scipy(oracle, synth, problem):
    """The reference benchmark's worker-firm problems (benchmark/run.jl:17-27)
    at 1/200 of their size: workers linked to nearby firms, and the worker FE
    next to the same worker ids interacted with a variable (a slow-converging,
    ill-conditioned pair).  At a tight tolerance the oracle's residual is
    scipy's projection, and it is orthogonal to every column."""
    p = getattr(synth, problem)(scale=0.005)
    y = p.Y[:, 0].astype(np.float64)
    A, _ = _sparse_A(p.refs, p.nlev, p.interaction, None, oracle)
    x, istop = spl.lsmr(A, y, atol=1e-13, btol=1e-13, conlim=1e12, maxiter=100000)[:2]
    R, _, cv = oracle.solve_residuals_cols(np.asfortranarray(y[:, None]), p.refs, p.nlev,
                                           p.interaction, None, tol=1e-13, maxiter=100000,
                                           nthreads=4)
    assert istop in (1, 2) and bool(cv[0])
    r_s = y - A @ x
    assert np.linalg.norm(R[:, 0] - r_s) <= 1e-8 * np.linalg.norm(r_s)
    assert np.abs(A.T @ R[:, 0]).max() <= 1e-10 * np.linalg.norm(y)


def test_scale_zero_guard(oracle):
    # issue #97 of the reference: a level whose interaction is all zero gets scale 0
    refs = np.array([1, 1, 2, 2, 3])
    inter = np.array([0.0, 0.0, 1.0, 2.0, 3.0])
    s = oracle.scale(refs, 3, inter, None)
    assert s[0] == 0.0
    assert np.isclose(s[1], 1 / np.sqrt(5.0)) and np.isclose(s[2], 1 / 3.0)


def test_integer_plan_is_stable_counting_sort(oracle):
    rng = np.random.default_rng(4)
    N = 5000
    refs = [rng.integers(1, 300, N), rng.integers(1, 7, N)]
    nlev = [int(r.max()) for r in refs]
    perm0, offs, segs = oracle.integer_plan(refs, nlev, 0)
    assert np.array_equal(perm0, np.argsort(refs[0], kind="stable"))
    for k in range(2):
        key = refs[k][perm0]
        assert np.array_equal(segs[k], np.argsort(key, kind="stable"))
        assert np.array_equal(offs[k], np.concatenate([[0], np.cumsum(np.bincount(key, minlength=nlev[k] + 1)[1:])]))
    assert np.array_equal(segs[0], np.arange(N))


def test_components(oracle):
    # two disconnected worker-firm blocks plus one isolated pair
    r1 = np.array([1, 1, 2, 3, 3, 4, 5])
    r2 = np.array([1, 2, 2, 3, 4, 4, 5])
    nc, comp = oracle.components([r1, r2])
    assert nc == 3
    assert len(set(comp[:3])) == 1 and len(set(comp[3:6])) == 1 and comp[6] not in comp[:6]


def test_maxiter_one_quirk(oracle, g):
    # maxiter = 1 runs LSMR with maxiter 0: no iteration, converged (istop 0)
    r, it, cv = oracle.solve_residuals(g["x"], [g["p1"], g["p2"]], maxiter=1)
    assert it == 1 and cv


def test_invalid_refs_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.solve_residuals(np.ones(3), [np.array([1, 2, 5])], nlev=[3])
