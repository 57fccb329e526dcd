"""Plan construction on the device: key grouping (fe_group_keys, the
GroupedArray compaction of src/FixedEffect.jl:18-21) against the host
grouping, and the integer plan built by radix sorts against the oracle's
stable counting sorts (ext/MetalExt.jl:40-64) and a numpy restatement for
batch plans.  Integer work: every comparison is exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

I64 = np.iinfo(np.int64)


CASES = ["dense", "negative", "sparse", "extremes", "repeats", "two_keys", "three_keys", "one",
         "empty", "dense_10m"]


@pytest.mark.parametrize("case", CASES)
def test_group_keys_matches_host(fe, case):
    rng = np.random.default_rng(100 + CASES.index(case))
    n = 50_000
    if case == "dense":
        keys = (rng.integers(0, 1000, n),)
    elif case == "negative":
        keys = (rng.integers(-5000, 5000, n),)
    elif case == "sparse":
        keys = (rng.integers(-2**62, 2**62, n),)
    elif case == "extremes":
        k = rng.integers(-2**40, 2**40, n)
        k[[3, 10, 99]] = [I64.min, I64.max, I64.min]
        keys = (k,)
    elif case == "repeats":
        keys = (rng.choice(rng.integers(0, 2**50, 300), n),)
    elif case == "two_keys":
        keys = (rng.integers(0, 40, n), rng.choice(rng.integers(-2**60, 2**60, 70), n))
    elif case == "three_keys":
        keys = (rng.integers(0, 7, n), rng.integers(100, 130, n), rng.integers(0, 2**33, n) // 2**28)
    elif case == "one":
        keys = (np.array([123456789012], dtype=np.int64),)
    elif case == "empty":
        keys = (np.zeros(0, dtype=np.int64),)
    else:  # dense range above 2^24: a three-level scan
        keys = (rng.integers(0, 20_000_000, 10_000_000),)
    refs, nl = fe.group_keys(*keys, device=0)
    host = fe.FixedEffect(*keys)  # numpy grouping on the host
    hr, hn = host.refs, host.n
    assert nl == hn
    assert np.array_equal(refs, hr)
    if case == "two_keys":
        f = fe.FixedEffect(*keys, device=0)
        assert f.n == hn and np.array_equal(f.refs, hr)


def test_group_keys_float_keys_and_rejects_strings(fe):
    rng = np.random.default_rng(9)
    x = np.concatenate([rng.standard_normal(20_000) * 1e3, [0.0, -0.0, np.inf, -np.inf, np.nan]])
    x = np.concatenate([x, rng.choice(x, 20_000)])
    k2 = rng.integers(0, 4, x.size)
    refs, nl = fe.group_keys(x, k2, device=0)
    host = fe.FixedEffect(x, k2)  # numpy grouping on the host
    assert nl == host.n and np.array_equal(refs, host.refs)
    with pytest.raises(TypeError):
        fe.group_keys(np.array(["a", "b"]), device=0)


@pytest.mark.parametrize("scale,extra", [(0.1, 0), (0.02, 37)])
def test_integer_plan_device_vs_oracle(fe, oracle, synth, scale, extra):
    # multi-pass radix sorts (2M/200K levels at full size), Zipf hot levels,
    # and (extra > 0) levels without observations
    pb = synth.make(2, scale=scale, ncols=1)
    nlev = [int(n) + extra for n in pb.nlev]
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float64)
    perm0, offs, segs = feM.integer_plan()
    p0, o_offs, o_segs = oracle.integer_plan(pb.refs, nlev, feM.primary())
    assert np.array_equal(perm0, p0)
    for k in range(len(fes)):
        assert np.array_equal(offs[k], o_offs[k])
        assert np.array_equal(segs[k], o_segs[k])
    feM.close()


def _batch_plan_numpy(refs, nlev, n_obs):
    """The integer plan of a batch plan restated with numpy stable sorts."""
    nprob, K = nlev.shape
    obs_off = np.concatenate([[0], np.cumsum(n_obs)])
    lev_off = np.vstack([np.zeros((1, K), dtype=np.int64), np.cumsum(nlev, axis=0)])
    tot = lev_off[-1]
    kp = int(np.argmax(tot))
    src = []
    for p in range(nprob):
        o0, o1 = obs_off[p], obs_off[p + 1]
        if nlev[p, kp] > 0:
            src.append(o0 + np.argsort(refs[kp][o0:o1], kind="stable"))
        else:
            src.append(np.arange(o0, o1))
    src = np.concatenate(src).astype(np.int32)
    prob = np.repeat(np.arange(nprob), n_obs)
    offs, segs = [], []
    for k in range(K):
        g = np.where(nlev[prob, k] == 0, tot[k], lev_off[prob, k] + refs[k] - 1)
        rs = g[src]
        order = np.argsort(rs, kind="stable")
        cnt = np.bincount(rs, minlength=tot[k] + 1)
        off = np.concatenate([[0], np.cumsum(cnt)])[:tot[k] + 1]
        offs.append(off)
        segs.append(order[:off[tot[k]]].astype(np.int32))
    return kp, src, offs, segs


def test_integer_plan_batch_vs_numpy(fe):
    # problems with 1, 2 or 3 FEs; slot 1 has the most levels in total, so
    # one-FE problems lack the primary FE and keep their order
    rng = np.random.default_rng(41)
    problems = []
    for p in range(40):
        n = int(rng.integers(1, 30_000))
        nfe = [1, 2, 3][p % 3]
        lv = [int(rng.integers(1, 60)), int(rng.integers(2, max(3, n // 3))), 9][:nfe]
        problems.append([fe.FixedEffect.from_refs(rng.integers(1, m + 1, n), m) for m in lv])
    bs = fe.BatchSolver(problems, T=np.float32, precision="mixed")
    perm0, offs, segs = bs.integer_plan()
    kp, src, o_offs, o_segs = _batch_plan_numpy(bs._refs, bs._nlev, bs.n_obs)
    assert kp == 1
    assert np.array_equal(perm0, src)
    for k in range(bs.K):
        assert np.array_equal(offs[k], o_offs[k])
        npos = int(o_offs[k][-1])
        assert np.array_equal(segs[k][:npos], o_segs[k])
    bs.close()


def test_invalid_refs_reported_like_a_host_scan(fe):
    # the first bad entry of a problem-by-problem, FE-by-FE scan is reported
    r0 = np.array([1, 2, 3, 9, 1], dtype=np.int64)     # bad at 3 (problem 1)
    r1 = np.array([1, 1, 2, 2, 1], dtype=np.int64)
    r1b = r1.copy()
    r1b[1] = 0                                          # bad at 1 (problem 0)
    with pytest.raises(fe.FEError, match=r"refs\[0\]\[3\] = 9 is outside 1\.\.3"):
        fe.AbstractFixedEffectSolver([fe.FixedEffect.from_refs(r0, 3),
                                      fe.FixedEffect.from_refs(r1, 2)], None, "CUDA")
    probs = [[fe.FixedEffect.from_refs(r0[:2], 3), fe.FixedEffect.from_refs(r1b[:2], 2)],
             [fe.FixedEffect.from_refs(r0[2:], 3), fe.FixedEffect.from_refs(r1b[2:], 2)]]
    with pytest.raises(fe.FEError, match=r"refs\[1\]\[1\] = 0 is outside 1\.\.2"):
        fe.BatchSolver(probs)
