"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's golden vectors (test/solve.jl)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-6  # residual / fitted-value bar (relative, 2-norm per column)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def julia_isapprox(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


@pytest.fixture(scope="module")
def g(golden):
    return {k: np.asarray(v) for k, v in golden.items() if isinstance(v, list)}


# --- test/solve.jl golden cases --------------------------------------------
def test_golden_residuals_fp64(fe, g, oracle):
    fes = [fe.FixedEffect(g["p1"]), fe.FixedEffect(g["p2"])]
    r, it, cv = fe.solve_residuals(g["x"].copy(), fes, double_precision=True)
    assert cv
    assert julia_isapprox(r, g["r_ols"], np.sqrt(np.finfo(np.float64).eps))
    _, it_o, _ = oracle.solve_residuals(g["x"], [g["p1"], g["p2"]])
    assert it == it_o


def test_golden_residuals_float32(fe, g):
    fes = [fe.FixedEffect(g["p1"]), fe.FixedEffect(g["p2"])]
    for prec in ("mixed", "fp32"):
        r, it, cv = fe.solve_residuals(g["x"].copy(), fes, double_precision=False, precision=prec)
        assert julia_isapprox(np.float32(r), np.float32(g["r_ols"]), np.sqrt(np.finfo(np.float32).eps))


def test_golden_coefficients(fe, g):
    fes = [fe.FixedEffect(g["p1"]), fe.FixedEffect(g["p2"])]
    for dp in (True, False):
        coefs, it, cv = fe.solve_coefficients(g["x"].copy(), fes, double_precision=dp)
        assert cv
        rtol = np.sqrt(np.finfo(np.float64 if dp else np.float32).eps)
        assert julia_isapprox(g["x"] - coefs[0] - coefs[1], g["r_ols"], rtol)


def test_golden_pooled_and_categorical_equivalents(fe, g):
    # PooledArray / CategoricalArray refs relabel levels; residuals must not move
    p1s = np.array([f"a{v}" for v in g["p1"]])
    p2s = (g["p2"] * 7 + 100)
    fes = [fe.FixedEffect(p1s), fe.FixedEffect(p2s)]
    r, _, _ = fe.solve_residuals(g["x"].copy(), fes, double_precision=True)
    assert julia_isapprox(r, g["r_ols"], np.sqrt(np.finfo(np.float64).eps))


def test_length_mismatch_message(fe):
    with pytest.raises(ValueError, match="FixedEffects must have the same length as y"):
        fe.solve_residuals(np.ones(100), [fe.FixedEffect([1, 2])])


def test_update_weights_round_trip(fe, g, oracle):
    fes = [fe.FixedEffect(g["p1"])]
    feM = fe.AbstractFixedEffectSolver(fes, np.ones(10), "CUDA", np.float64)
    for w in (np.arange(1, 11, dtype=float), np.arange(10, 0, -1, dtype=float)):
        fe.update_weights(feM, w)
        r1 = feM.solve_residuals(g["x"].copy())[0]
        r2 = fe.solve_residuals(g["x"].copy(), fes, w, double_precision=True)[0]
        ro = oracle.solve_residuals(g["x"], [g["p1"]], weights=w)[0]
        assert rel_err(r1, r2) < 1e-12
        assert rel_err(r1, ro) < 1e-12


def test_interacted_converges(fe, g):
    inter = g["interaction"]
    r, it, cv = fe.solve_residuals(g["x"].copy(), [fe.FixedEffect(g["p1"], interaction=inter)],
                                   double_precision=True)
    assert cv
    r, it, cv = fe.solve_residuals(
        g["x"].copy(), [fe.FixedEffect(g["p1"]), fe.FixedEffect(g["p1"], interaction=inter)],
        double_precision=True)
    assert cv


# --- seeded workloads at oracle-sized scales ---------------------------------
def _problem(synth, cfg, scale, ncols=None):
    kw = {}
    if ncols is not None:
        kw["ncols"] = ncols
    return synth.make(cfg, scale=scale, **kw)


@pytest.mark.parametrize("cfg,scale,ncols", [(0, 0.02, None), (1, 0.002, None), (2, 0.002, 5),
                                             (4, 0.0002, 3)])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_configs_vs_oracle(fe, oracle, synth, cfg, scale, ncols, prec):
    pb = _problem(synth, cfg, scale, ncols)
    Y = np.asfortranarray(pb.Y.astype(np.float64))
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
    R_o, it_o, cv_o = oracle.solve_residuals_cols(Y, pb.refs, pb.nlev, pb.interaction, pb.weights,
                                                 tol=1e-8, maxiter=10000)
    assert cv_o.all()
    for tile in (1, 0):
        feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64, precision=prec)
        feM.set_option(fe._lib.FE_OPT_TILE, tile)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8, maxiter=10000)
        feM.close()
        assert cvs.all()
        for j in range(Y.shape[1]):
            assert rel_err(R[:, j], R_o[:, j]) < REL
            assert rel_err(Y[:, j] - R[:, j], Y[:, j] - R_o[:, j]) < REL
        if prec == "fp64":
            assert np.all(np.abs(its - it_o) <= 1), (its, it_o)


def test_integer_plan_bit_exact(fe, oracle, synth):
    pb = synth.make(2, scale=0.002, ncols=1)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64)
    perm0, offs, segs = feM.integer_plan()
    p0, o_offs, o_segs = oracle.integer_plan(pb.refs, pb.nlev, feM.primary())
    assert np.array_equal(perm0, p0)
    for k in range(len(fes)):
        assert np.array_equal(offs[k], o_offs[k])
        assert np.array_equal(segs[k], o_segs[k])
    feM.close()


def test_scales_match_oracle(fe, oracle, synth):
    pb = synth.make(1, scale=0.002)
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
    feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64)
    sc = feM.scales()
    for k in range(len(fes)):
        so = oracle.scale(pb.refs[k], pb.nlev[k], pb.interaction[k], pb.weights)
        assert np.allclose(sc[k], so, rtol=1e-13, atol=0)
    feM.close()


def test_deterministic_bitwise(fe, synth):
    pb = synth.make(2, scale=0.003, ncols=4)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    outs = []
    for _ in range(2):
        feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
        R, its, cvs = feM.solve_residuals(np.asfortranarray(pb.Y.copy()), tol=1e-8)
        feM.close()
        outs.append((R, its))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_batch_problems_vs_oracle(fe, oracle, synth):
    probs = synth.make(3, scale=0.01, nproblems=12)
    fes_list = [[fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(p.refs, p.nlev, p.interaction)]
                for p in probs]
    for prec in ("fp64", "mixed"):
        bs = fe.BatchSolver(fes_list, [p.weights for p in probs], precision=prec)
        outs, its, cvs = bs.solve_residuals([p.Y[:, 0] for p in probs], tol=1e-8, maxiter=10000)
        bs.close()
        assert cvs.all()
        for p, r in zip(probs, outs):
            ro, it_o, cv_o = oracle.solve_residuals(p.Y[:, 0].astype(np.float64), p.refs, p.nlev,
                                                    p.interaction, p.weights, tol=1e-8)
            # inputs are Float32 columns.  Problems with about one observation
            # per level are nearly consistent: their residual is tiny and the
            # reference's test1 (src/utils/lsmr.jl:200-201) fixes it only to
            # about tol*||y||, so the bar is relative plus an absolute floor.
            y64 = p.Y[:, 0].astype(np.float64)
            err = np.linalg.norm(r - ro)
            assert err <= REL * np.linalg.norm(ro) + REL * np.linalg.norm(y64)


def test_device_tensor_path(fe, synth, oracle):
    import torch
    pb = synth.make(0, scale=0.01)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    y = pb.Y[:, 0].astype(np.float64)
    ro = oracle.solve_residuals(y, pb.refs, pb.nlev, tol=1e-8)[0]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    t = torch.tensor(y, device="cuda")
    t, it, cv = feM.solve_residuals(t, tol=1e-8)
    torch.cuda.synchronize()
    feM.close()
    assert cv
    assert rel_err(t.cpu().numpy(), ro) < REL


def test_coefficients_vs_oracle(fe, oracle, synth):
    pb = synth.make(1, scale=0.001)
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
    y = pb.Y[:, 0]
    lv_o, full_o, it_o, cv_o = oracle.solve_coefficients(y, pb.refs, pb.nlev, pb.interaction,
                                                          pb.weights, tol=1e-8)
    for dp in (True, False):
        full_g, it, cv = fe.solve_coefficients(y.copy(), fes, pb.weights, double_precision=dp,
                                               tol=1e-8)
        assert cv
        fit_g = sum(c * (1 if a is None else a) for c, a in zip(full_g, pb.interaction))
        fit_o = sum(c * (1 if a is None else a) for c, a in zip(full_o, pb.interaction))
        assert rel_err(fit_g, fit_o) < REL
        if dp:
            assert abs(it - it_o) <= 1


# --- edge cases --------------------------------------------------------------
def test_single_fe_is_projection(fe, oracle):
    rng = np.random.default_rng(5)
    r = rng.integers(1, 30, 500)
    y = rng.standard_normal(500)
    ro, it_o, cv_o = oracle.solve_residuals(y, [r])
    for dp in (True, False):
        out, it, cv = fe.solve_residuals(y.copy(), [fe.FixedEffect(r)], double_precision=dp)
        assert it == 1 and it_o == 1 and cv
        assert rel_err(out, ro) < 1e-12


def test_unobserved_levels_and_zero_weights(fe, oracle):
    rng = np.random.default_rng(6)
    N = 3000
    r1 = rng.integers(1, 200, N)
    r2 = rng.integers(1, 20, N)
    w = rng.uniform(0.5, 1.5, N)
    w[r2 == 3] = 0.0  # a level whose weights are all zero gets scale 0 (issue #97)
    y = rng.standard_normal(N)
    fes = [fe.FixedEffect.from_refs(r1, 250), fe.FixedEffect.from_refs(r2, 25)]
    w_pos = w.copy()
    w_pos[w_pos == 0] = 1.0  # residuals are divided by sqrt(w): compare where w > 0
    ro = oracle.solve_residuals(y, [r1, r2], [250, 25], weights=w)[0]
    out, it, cv = fe.solve_residuals(y.copy(), fes, w, double_precision=True)
    m = w > 0
    assert rel_err(out[m], ro[m]) < 1e-9


def test_maxiter_one_quirk(fe, oracle, g):
    fes = [fe.FixedEffect(g["p1"]), fe.FixedEffect(g["p2"])]
    r, it, cv = fe.solve_residuals(g["x"].copy(), fes, double_precision=True, maxiter=1)
    ro, it_o, cv_o = oracle.solve_residuals(g["x"], [g["p1"], g["p2"]], maxiter=1)
    assert (it, cv) == (it_o, cv_o)
    assert rel_err(r, ro) < 1e-12


def test_many_columns_tiles(fe, oracle, synth):
    pb = synth.make(0, scale=0.005)
    rng = np.random.default_rng(9)
    Y = np.asfortranarray(rng.standard_normal((pb.N, 43)))
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    R_o, _, _ = oracle.solve_residuals_cols(Y, pb.refs, pb.nlev, tol=1e-8)
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
    feM.close()
    assert cvs.all()
    assert max(rel_err(R[:, j], R_o[:, j]) for j in range(43)) < REL


def test_zipf_split_levels(fe, oracle):
    # one level holding most observations forces multi-piece (split) levels
    rng = np.random.default_rng(11)
    N = 200_000
    r1 = rng.integers(1, 20_000, N)
    r2 = np.where(rng.random(N) < 0.7, 1, rng.integers(2, 50, N))
    Y = np.asfortranarray(rng.standard_normal((N, 2)))
    R_o, it_o, _ = oracle.solve_residuals_cols(Y, [r1, r2], tol=1e-8)
    fes = [fe.FixedEffect(r1), fe.FixedEffect(r2)]
    for prec in ("fp64", "mixed"):
        feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64, precision=prec)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
        feM.close()
        assert cvs.all()
        assert max(rel_err(R[:, j], R_o[:, j]) for j in range(2)) < REL


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_rowsum_matches_segsum_path(fe, oracle, prec):
    # 32-column tile: the contiguous row-sum pass reduces the primary FE (one
    # level holds 30 % of the observations, so it is cut into pieces) and two
    # small FEs (20 levels with an interaction, 6 levels); weighted.  Compared
    # with the segsum-only path and the oracle, and bitwise across two calls.
    rng = np.random.default_rng(12)
    N = 40_000
    r1 = rng.integers(1, 3001, N)
    r1[rng.random(N) < 0.3] = 1
    r2 = rng.integers(1, 401, N)
    r3 = rng.integers(1, 21, N)
    r4 = rng.integers(1, 7, N)
    refs = [r1, r2, r3, r4]
    inter = [None, None, rng.uniform(0.5, 1.5, N), None]
    w = rng.uniform(0.5, 1.5, N)
    Y = np.asfortranarray(rng.standard_normal((N, 5)))
    R_o, _, _ = oracle.solve_residuals_cols(Y, refs, None, inter, w, tol=1e-8)
    fes = [fe.FixedEffect(r, interaction=a) for r, a in zip(refs, inter)]
    out = []
    # (row-sum pass, its variant): shared-memory ring, registers, segsum only
    for fuse, var in ((1, 0), (1, 1), (0, -1)):
        feM = fe.AbstractFixedEffectSolver(fes, w, "CUDA", np.float64, precision=prec)
        feM.set_option(fe._lib.FE_OPT_TILE, 32)
        feM.set_option(fe._lib.FE_OPT_FUSE, fuse)
        feM.set_option(fe._lib.FE_OPT_ROWSUM_VARIANT, var)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
        R2, its2, _ = feM.solve_residuals(Y.copy(), tol=1e-8)
        feM.close()
        assert cvs.all() and np.array_equal(R, R2) and np.array_equal(its, its2)
        err = max(rel_err(R[:, j], R_o[:, j]) for j in range(Y.shape[1]))
        assert err < REL, (fuse, var, err)
        out.append(R)
    # the two row-sum variants sum in the same order; the segsum in another
    assert np.array_equal(out[0], out[1])
    assert max(rel_err(out[0][:, j], out[2][:, j]) for j in range(Y.shape[1])) < REL


def test_autotuner_persists_choice(fe, synth, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FE_B200_TUNE_CACHE", str(cache))
    pb = synth.make(2, scale=0.002, ncols=8)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    Y = np.asfortranarray(pb.Y.astype(np.float64))
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    R1, _, _ = feM.solve_residuals(Y.copy(), tol=1e-8)
    feM.close()
    # mixed precision tunes its FP32 loop kernels (element size 4) and its
    # FP64 refinement kernels (recorded as 108): one line each
    lines = cache.read_text().strip().splitlines()
    assert len(lines) == 2
    shapes = set()
    for line in lines:
        sig, C, sT, ex, seg = line.split()
        shapes.add((int(C), int(sT)))
        assert 0 <= int(ex) < 6 and 0 <= int(seg) < 6
    assert shapes == {(8, 4), (8, 108)}
    # a second plan of the same shape reuses the cached choices (no new line)
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32)
    R2, _, _ = feM.solve_residuals(Y.copy(), tol=1e-8)
    feM.close()
    assert len(cache.read_text().strip().splitlines()) == 2
    assert np.array_equal(R1, R2)


@pytest.mark.parametrize("tile", [32, 8, 1])
def test_every_kernel_variant_matches_oracle(fe, synth, oracle, tile):
    # Zipf firms (split levels), a 20-level FE, weights: every code path of the
    # expand and segsum variants the autotuner can pick
    pb = synth.make(4, scale=0.0003, ncols=3)
    rng = np.random.default_rng(5)
    yr = rng.integers(1, 21, pb.N)
    refs = pb.refs + [yr]
    nlev = pb.nlev + [20]
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(refs, nlev)]
    Y = np.asfortranarray(pb.Y.astype(np.float64))
    R_o, _, _ = oracle.solve_residuals_cols(Y, refs, nlev, None, pb.weights, tol=1e-8)
    for prec in ("fp64", "mixed"):
        feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64, precision=prec)
        feM.set_option(fe._lib.FE_OPT_TILE, tile)
        for ev, sv in [(0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5)]:
            feM.set_option(fe._lib.FE_OPT_EXPAND_VARIANT, ev)
            feM.set_option(fe._lib.FE_OPT_SEGSUM_VARIANT, sv)
            R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
            assert cvs.all(), (prec, ev, sv)
            err = max(rel_err(R[:, j], R_o[:, j]) for j in range(Y.shape[1]))
            assert err < REL, (prec, ev, sv, err)
        feM.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_replay_matches_direct_launches(fe, synth, prec):
    pb = synth.make(0, scale=0.05)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    Y = np.asfortranarray(np.repeat(pb.Y.astype(np.float64), 3, axis=1))
    out = []
    for graph in (1, 0):
        feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64, precision=prec)
        feM.set_option(fe._lib.FE_OPT_GRAPH, graph)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
        R2, its2, _ = feM.solve_residuals(Y.copy(), tol=1e-8)  # a replay of the cached graph
        feM.close()
        assert cvs.all() and np.array_equal(R, R2) and np.array_equal(its, its2)
        out.append((R, its))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("case", ["weighted4", "two_fe_small", "unweighted3", "absorbed_levels"])
def test_absorbed_primary_matches_oracle(fe, oracle, case):
    # mixed residual solves of a 32-column tile with the primary FE projected
    # out (FE_OPT_ABSORB, the default) against the oracle's full LSMR and the
    # non-absorbed path; bitwise identical across two calls
    rng = np.random.default_rng(21)
    N = 60_000
    r1 = rng.integers(1, 5001, N)
    r1[rng.random(N) < 0.2] = 7  # one long primary level
    r2 = rng.integers(1, 801, N)  # large FE: gathered by the segsum
    r3 = rng.integers(1, 21, N)   # small FEs: shared-memory tables
    r4 = rng.integers(1, 5, N)
    if case == "weighted4":
        refs, inter, w = [r1, r2, r3, r4], [None, None, rng.uniform(0.5, 1.5, N), None], rng.uniform(0.5, 1.5, N)
    elif case == "two_fe_small":
        refs, inter, w = [r1, r3], [None, None], None
    elif case == "absorbed_levels":
        # firms 801.. are each staffed by a single worker (their columns lie in
        # the span of the worker columns, ||M a_l|| = 0), firm 2000 by two
        # workers of which one has a single other row (nearly absorbed)
        r2 = r2.copy()
        solo = r1 % 7 == 0
        r2[solo] = 800 + r1[solo]
        pair = np.flatnonzero(r1 == 5)
        r2[pair] = 2000 + 5000 + 1
        r2[np.flatnonzero(r1 == 11)[:1]] = 2000 + 5000 + 1
        refs, inter, w = [r1, r2, r3], [None, None, None], rng.uniform(0.5, 1.5, N)
    else:
        refs, inter, w = [r1, r2, r3], [None, None, None], None
    Y = np.asfortranarray(rng.standard_normal((N, 5)))
    R_o, _, _ = oracle.solve_residuals_cols(Y, refs, None, inter, w, tol=1e-8)
    fes = [fe.FixedEffect(r, interaction=a) for r, a in zip(refs, inter)]
    out = []
    # (absorb, fused expand + demean, columns scaled by 1/||M a_l||, pipelined
    # fused kernel): default, the unpipelined fused kernel, separate kernels,
    # Jacobi scales of A_r, full LSMR
    # and the gathered FE's level sums by vector reductions (atomic = 1; not
    # bitwise reproducible; its levels here hold at most ~100 positions) or by
    # the deterministic segmented sum (0); fres: the refinement's FP64
    # residual and its projection by the projection kernel (-1, the default,
    # and 2; the same sums as 0, so bitwise equal results), as two kernels
    # (0), or by the staged fused kernel (1)
    cases = ((1, 1, 1, -1, 0, -1), (1, 1, 1, -1, 1, -1), (1, 1, 1, 0, 0, -1), (1, 1, 1, 1, 0, -1),
             (1, 1, 1, 2, 0, -1), (1, 1, 1, 3, 0, -1), (1, 0, 1, -1, 0, -1), (1, 1, 0, -1, 0, -1),
             (0, 1, 1, -1, 0, -1),
             (1, 1, 1, -1, 0, 0), (1, 1, 1, -1, 0, 2), (1, 1, 1, -1, 0, 1), (1, 0, 1, -1, 0, 1))
    for absorb, fused, ascale, pipe, atomic, fres in cases:
        feM = fe.AbstractFixedEffectSolver(fes, w, "CUDA", np.float64, precision="mixed")
        feM.set_option(fe._lib.FE_OPT_TILE, 32)
        feM.set_option(fe._lib.FE_OPT_ABSORB, absorb)
        feM.set_option(fe._lib.FE_OPT_FUSED_DEMEAN, fused)
        feM.set_option(fe._lib.FE_OPT_ABSORB_SCALE, ascale)
        feM.set_option(fe._lib.FE_OPT_EXDM_PIPE, pipe)
        feM.set_option(fe._lib.FE_OPT_FIRM_ATOMIC, atomic)
        feM.set_option(fe._lib.FE_OPT_FUSED_RESID, fres)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
        R2, its2, _ = feM.solve_residuals(Y.copy(), tol=1e-8)
        feM.close()
        assert cvs.all(), (absorb, fused, ascale, its)
        if atomic == 0:
            assert np.array_equal(R, R2) and np.array_equal(its, its2)
        err = max(rel_err(R[:, j], R_o[:, j]) for j in range(Y.shape[1]))
        assert err < REL, (absorb, fused, ascale, err)
        out.append(R)
    for R in out[1:]:
        assert max(rel_err(out[0][:, j], R[:, j]) for j in range(Y.shape[1])) < REL
    # the projection kernel's residual form = the residual kernel + projection
    i_def, i_sep, i_two = (cases.index((1, 1, 1, -1, 0, f)) for f in (-1, 0, 2))
    assert np.array_equal(out[i_def], out[i_sep]) and np.array_equal(out[i_two], out[i_sep])


@pytest.mark.parametrize("ncols,weighted", [(1, False), (1, True), (3, True), (8, False), (8, True)])
def test_absorbed_narrow_tiles(fe, oracle, ncols, weighted):
    # mixed residual solves of tiles narrower than 32 columns with the primary
    # FE projected out (k_demean_narrow), with one primary level longer than a
    # demean item: against the oracle, the full-LSMR path (FE_OPT_ABSORB = 0)
    # and bitwise across two calls
    rng = np.random.default_rng(29)
    N = 50_000
    r1 = rng.integers(1, 5001, N)
    r1[rng.random(N) < 0.1] = 7  # one long primary level
    r2 = rng.integers(1, 601, N)
    r3 = rng.integers(1, 31, N)
    inter = [None, None, rng.uniform(0.5, 1.5, N) if weighted else None]
    w = rng.uniform(0.5, 1.5, N) if weighted else None
    refs = [r1, r2, r3]
    Y = np.asfortranarray(rng.standard_normal((N, ncols)) + (r1 % 11)[:, None] * 0.3)
    R_o, _, _ = oracle.solve_residuals_cols(Y, refs, None, inter, w, tol=1e-8)
    fes = [fe.FixedEffect(r, interaction=a) for r, a in zip(refs, inter)]
    out = []
    for absorb in (1, 0):
        feM = fe.AbstractFixedEffectSolver(fes, w, "CUDA", np.float64, precision="mixed")
        feM.set_option(fe._lib.FE_OPT_ABSORB, absorb)
        R, its, cvs = feM.solve_residuals(Y.copy(), tol=1e-8)
        R2, its2, _ = feM.solve_residuals(Y.copy(), tol=1e-8)
        feM.close()
        assert cvs.all(), (absorb, its)
        assert np.array_equal(R, R2) and np.array_equal(its, its2)
        err = max(rel_err(R[:, j], R_o[:, j]) for j in range(ncols))
        assert err < REL, (absorb, err)
        out.append((R, its))
    # the projected problem needs fewer LSMR iterations
    assert np.sum(out[0][1]) < np.sum(out[1][1]), (out[0][1], out[1][1])


@pytest.mark.parametrize("weighted", [False, True])
def test_batch_absorbed_vs_oracle(fe, oracle, weighted):
    # batch plans project each problem's primary FE out (demean items and norm
    # slots per problem, k_demean_narrow): against the oracle, against the
    # full-LSMR batch (FE_OPT_ABSORB = 0) and bitwise across two calls.  The
    # problems stop at different iterations, so the passes skip stopped
    # problems, whose rows must stay as they were.
    rng = np.random.default_rng(37 + int(weighted))
    probs = []
    for p in range(10):
        n = int(rng.integers(300, 20_000))
        r1 = rng.integers(1, max(3, n // 8) + 1, n)
        if p == 3:
            r1[rng.random(n) < 0.2] = 1  # a primary level longer than a demean item
        raw = [r1, rng.integers(1, 41, n)]
        inter = [None, None]
        if p % 2:
            raw.append(rng.integers(1, 301, n))
            inter.append(rng.uniform(0.5, 1.5, n) if weighted else None)
        refs = [np.unique(r, return_inverse=True)[1].astype(np.int64) + 1 for r in raw]
        w = rng.uniform(0.5, 1.5, n) if weighted else None
        y = rng.standard_normal(n) + (r1 % 7) * 0.4 + (raw[1] % 5) * 0.3
        probs.append((refs, inter, w, y))
    ref = [oracle.solve_residuals(y, refs, None, inter, w, tol=1e-8)[0] for refs, inter, w, y in probs]
    fes_list = [[fe.FixedEffect(r, interaction=a) for r, a in zip(refs, inter)]
                for refs, inter, _, _ in probs]
    ws = [w for _, _, w, _ in probs] if weighted else None
    iters = []
    for absorb in (1, 0):
        bs = fe.BatchSolver(fes_list, ws, precision="mixed")
        bs.set_option(fe._lib.FE_OPT_ABSORB, absorb)
        bs.set_option(fe._lib.FE_OPT_PROFILE, 1)
        outs, its, cvs = bs.solve_residuals([y for *_, y in probs], tol=1e-8, maxiter=10000)
        ran_demean = "demean" in bs.kernel_stats()
        bs.set_option(fe._lib.FE_OPT_PROFILE, 0)
        outs2, its2, _ = bs.solve_residuals([y for *_, y in probs], tol=1e-8, maxiter=10000)
        bs.close()
        assert ran_demean == (absorb == 1)
        assert cvs.all(), (absorb, its)
        assert np.array_equal(its, its2)
        for r, r2 in zip(outs, outs2):
            assert np.array_equal(r, r2)
        for (refs, inter, w, y), r, ro in zip(probs, outs, ref):
            err = np.linalg.norm(r - ro)
            assert err <= REL * np.linalg.norm(ro) + REL * np.linalg.norm(y), (absorb, err)
        iters.append(np.asarray(its))
    # the projected problems need fewer LSMR iterations in all
    assert iters[0].sum() < iters[1].sum(), iters


def test_batch_without_primary_everywhere_is_not_absorbed(fe, oracle):
    # slot 1 has the most levels (the primary FE); problem 2 holds only slot 0,
    # so its rows have no primary level to project out and the whole batch
    # keeps the full LSMR
    rng = np.random.default_rng(43)
    probs = []
    for p in range(4):
        n = int(rng.integers(2_000, 6_000))
        r0 = rng.integers(1, 31, n)
        refs = [r0] if p == 2 else [r0, rng.integers(1, n // 5 + 1, n)]
        refs = [np.unique(r, return_inverse=True)[1].astype(np.int64) + 1 for r in refs]
        probs.append((refs, rng.standard_normal(n) + (r0 % 3)))
    fes_list = [[fe.FixedEffect(r) for r in refs] for refs, _ in probs]
    bs = fe.BatchSolver(fes_list, precision="mixed")
    bs.set_option(fe._lib.FE_OPT_PROFILE, 1)
    outs, its, cvs = bs.solve_residuals([y for _, y in probs], tol=1e-8, maxiter=10000)
    assert "demean" not in bs.kernel_stats()
    bs.close()
    assert cvs.all()
    for (refs, y), r in zip(probs, outs):
        ro = oracle.solve_residuals(y, refs, None, None, None, tol=1e-8)[0]
        assert np.linalg.norm(r - ro) <= REL * np.linalg.norm(ro) + REL * np.linalg.norm(y)


def test_absorbed_column_stopping_at_round0(fe):
    # a zero column stops at refinement round 0 (||r0|| = 0): its residual is
    # r0 = M b = 0.  The plan first solves a nonzero column in the same slot,
    # so stale rows would show; the other columns are solved exactly as before.
    rng = np.random.default_rng(23)
    N = 40_000
    refs = [rng.integers(1, 4001, N), rng.integers(1, 401, N), rng.integers(1, 21, N)]
    fes = [fe.FixedEffect(r) for r in refs]
    Y = np.asfortranarray(rng.standard_normal((N, 4)))
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64, precision="mixed")
    feM.set_option(fe._lib.FE_OPT_TILE, 32)
    R1, its1, cv1 = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    Y2 = Y.copy(order="F")
    Y2[:, 2] = 0.0
    R2, its2, cv2 = feM.solve_residuals(Y2, tol=1e-8)
    feM.close()
    assert cv1.all() and cv2.all()
    assert np.array_equal(R2[:, 2], np.zeros(N))
    for j in (0, 1, 3):
        assert np.array_equal(R2[:, j], R1[:, j]) and its2[j] == its1[j]


def test_update_weights_drops_captured_loops(fe, synth):
    # a 32-column mixed solve captures its LSMR loop in a CUDA graph; switching
    # between unit and other weights must not replay the old capture
    pb = synth.make(2, scale=0.005, ncols=32)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    w = np.random.default_rng(5).uniform(0.5, 1.5, pb.N)
    Y = np.asfortranarray(pb.Y.astype(np.float64))
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32, precision="mixed")
    R0, _, c0 = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    fe.update_weights(feM, w)
    Rw, _, cw = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    fe.update_weights(feM, None)
    R1, _, c1 = feM.solve_residuals(Y.copy(order="F"), tol=1e-8)
    feM.close()
    feW = fe.AbstractFixedEffectSolver(fes, w, "CUDA", np.float32, precision="mixed")
    Rref, _, cref = feW.solve_residuals(Y.copy(order="F"), tol=1e-8)
    feW.close()
    assert c0.all() and cw.all() and c1.all() and cref.all()
    assert max(rel_err(Rw[:, j], Rref[:, j]) for j in range(32)) < 1e-6
    assert max(rel_err(R1[:, j], R0[:, j]) for j in range(32)) < 1e-6
    # the weights matter: the unit-weight residuals differ from the weighted ones
    assert max(rel_err(R0[:, j], Rref[:, j]) for j in range(32)) > 1e-3
