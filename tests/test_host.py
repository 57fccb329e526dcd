"""Host-side logic of the binding that needs no GPU: FixedEffect (the
reference's test/types.jl), normalize!/full against the oracle, the C ABI's
presence, and the synthetic workloads."""
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


# --- FixedEffect (test/types.jl) ----------------------------------------------
def test_fixedeffect_basic(fe_host):
    fe1 = fe_host.FixedEffect(np.arange(1, 11))
    assert repr(fe1) == "Fixed Effects"
    assert fe1.refs.dtype == np.int64
    assert list(fe1.refs[:5]) == [1, 2, 3, 4, 5]
    assert fe1.interaction is None and fe1.n == 10
    assert len(fe1) == 10 and fe1.size == (10,)
    fe2 = fe_host.FixedEffect(np.arange(1, 11), interaction=np.full(10, 1.23456789))
    assert fe2.interaction.dtype == np.float64


def test_fixedeffect_dimension_mismatch(fe_host):
    with pytest.raises(fe_host.DimensionMismatch):
        fe_host.FixedEffect(np.arange(1, 11), interaction=np.ones(5))


def test_fixedeffect_getindex(fe_host):
    fe1 = fe_host.FixedEffect(np.arange(1, 11))
    assert fe1[:] is fe1
    sub = fe1[[0, 1]]
    assert np.array_equal(sub.refs, fe1.refs[:2]) and sub.n == fe1.n
    assert sub == fe1[np.arange(2)]
    assert sub == fe1[fe1.refs <= 2]
    with pytest.raises(TypeError):
        fe1[np.array([[0, 1]])]
    fe2 = fe_host.FixedEffect(np.arange(1, 11), interaction=np.full(10, 1.5))
    sub2 = fe2[[0, 1]]
    assert np.array_equal(sub2.interaction, fe2.interaction[:2])


def test_fixedeffect_compaction(fe_host):
    fe = fe_host.FixedEffect(np.array([10, 30, 10, 50]))
    assert list(fe.refs) == [1, 2, 1, 3] and fe.n == 3
    fs = fe_host.FixedEffect(np.array(["b", "a", "b"]))
    assert list(fs.refs) == [2, 1, 2] and fs.n == 2
    fm = fe_host.FixedEffect(np.array([1, 1, 2, 2]), np.array([1, 2, 1, 2]))
    assert fm.n == 4 and len(set(fm.refs)) == 4


# --- normalize! / full vs the oracle -------------------------------------------
def test_normalize_matches_oracle(fe_host, oracle):
    rng = np.random.default_rng(0)
    N = 3000
    # three blocks so that the graph has several connected components
    blocks = rng.integers(0, 3, N)
    r1 = blocks * 100 + rng.integers(1, 60, N)
    r2 = blocks * 40 + rng.integers(1, 30, N)
    y = rng.standard_normal(N)
    fes = [fe_host.FixedEffect(r1), fe_host.FixedEffect(r2)]
    refs = [f.refs for f in fes]
    nlev = [f.n for f in fes]
    lv, full_o, it, cv = oracle.solve_coefficients(y, refs, nlev, tol=1e-10)
    # undo the oracle's normalisation: recover raw coefficients by shifting
    # each component by an arbitrary constant, then normalise on the host
    lab, nc = fe_host.components(fes)
    assert nc == oracle.components(refs, nlev)[0]
    shift = rng.standard_normal(nc)
    raw = [lv[0] + shift[lab[0]], lv[1] - shift[lab[1]]]
    out = fe_host.normalize([c.copy() for c in raw], fes)
    assert np.allclose(out[0], lv[0], atol=1e-9) and np.allclose(out[1], lv[1], atol=1e-9)
    full = fe_host.full(out, fes)
    assert np.allclose(full[0], full_o[0], atol=1e-9)


def test_normalize_skips_interacted(fe_host):
    fes = [fe_host.FixedEffect(np.array([1, 2, 1])), fe_host.FixedEffect(np.array([1, 1, 2]),
                                                                         interaction=np.ones(3))]
    c = [np.array([1.0, 2.0]), np.array([3.0, 4.0])]
    out = fe_host.normalize([x.copy() for x in c], fes)
    assert np.array_equal(out[0], c[0]) and np.array_equal(out[1], c[1])


# --- the C ABI -------------------------------------------------------------------
def _declared_symbols():
    src = (ROOT / "include" / "fe_b200.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_match_binding(fe_host):
    assert _declared_symbols() == sorted(fe_host._lib.EXPORTS)


def test_library_exports_every_declared_symbol(fe_host):
    import ctypes
    lib = fe_host._lib.load()
    for name in _declared_symbols():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value
    assert lib.fe_version() == 1


def test_errors_are_reported_not_raised_by_the_library(fe_host):
    import ctypes
    from conftest import cuda_available
    lib = fe_host._lib.load()
    h = ctypes.c_void_p()
    # a null plan is an argument error on any machine
    assert lib.fe_plan_destroy(None) == 0
    assert lib.fe_plan_set_option(None, 1, 0.0) == fe_host._lib.FE_ERR_INVALID
    assert b"NULL" in lib.fe_last_error()
    if not cuda_available():
        refs = np.array([1, 2], dtype=np.int64)
        arr = (ctypes.c_void_p * 1)(refs.ctypes.data)
        nl = np.array([2], dtype=np.int64)
        st = lib.fe_plan_create(ctypes.byref(h), 2, 1, arr, nl.ctypes.data_as(fe_host._lib._i64p),
                                None, None, 0)
        assert st == fe_host._lib.FE_ERR_CUDA
        assert b"no CUDA device" in lib.fe_last_error()


def test_method_and_length_checks(fe_host):
    fe = fe_host.FixedEffect(np.array([1, 2]))
    with pytest.raises(ValueError, match="FixedEffects must have the same length as y"):
        fe_host.solve_residuals(np.ones(100), [fe])
    with pytest.raises(ValueError, match="not provided"):
        fe_host.FixedEffectSolverB200([fe], None, method="cpu")


# --- synthetic workloads ----------------------------------------------------------
def test_synth_shapes(synth):
    p0 = synth.config0(scale=0.01)
    assert p0.Y.shape == (10000, 1) and len(p0.refs) == 2
    assert all(r.min() == 1 and r.max() == n for r, n in zip(p0.refs, p0.nlev))
    p2 = synth.config2(scale=0.001, ncols=4)
    assert p2.Y.dtype == np.float32 and p2.Y.shape[1] == 4 and p2.Y.flags.f_contiguous
    counts = np.bincount(p2.refs[1])
    assert counts.max() > 10 * np.median(counts[1:])  # Zipf hot firms
    probs = synth.config3(scale=0.01, nproblems=8)
    assert len(probs) == 8 and all(len(p.refs) in (2, 3) for p in probs)
    p4 = synth.config4(scale=0.00005, ncols=2)
    assert p4.weights is not None and p4.Y.shape[1] == 2


def test_reference_benchmark_shapes(synth):
    """The problems of the reference's benchmark/run.jl:6-28: 100 levels per
    simple-FE level on average, firms within 10 of worker / 8, and the
    interacted case's two FEs on the same worker ids."""
    ps = synth.simple_10m(scale=0.01)
    assert ps.N == 100_000 and ps.nlev[1] == 100 and ps.Y.dtype == np.float64
    assert 0.0 <= ps.Y.min() and ps.Y.max() < 1.0
    rng = np.random.default_rng(0)
    N, pid, fid = synth._worker_firm_800k(rng, 1.0)
    assert N == 800_000 and pid.max() <= 400_000 and fid.min() >= 1 and fid.max() <= 50_000
    assert np.all(np.abs(fid - pid // 8) <= 10 + 1)  # +1: clipping at firm 1
    ph = synth.hard_800k(scale=0.01)
    assert len(ph.refs) == 2 and ph.meta["maxiter"] is None
    pi = synth.hard_800k_interacted(scale=0.01)
    assert np.array_equal(pi.refs[0], pi.refs[1]) and pi.interaction[0] is None
    assert pi.interaction[1] is not None and pi.meta["maxiter"] == 300


def test_synth_deterministic(synth):
    a = synth.config1(scale=0.0005)
    b = synth.config1(scale=0.0005)
    assert np.array_equal(a.Y, b.Y) and all(np.array_equal(x, y) for x, y in zip(a.refs, b.refs))


def test_zipf_sampler(synth):
    rng = np.random.default_rng(0)
    z = synth.zipf_refs(rng, 1.1, 1000, 200000)
    c = np.bincount(z, minlength=1001)[1:]
    p = np.arange(1, 1001, dtype=float) ** -1.1
    p /= p.sum()
    assert abs(c[0] / c.sum() - p[0]) < 0.01


# --- order keys of floating-point keys (device grouping, fe_group_keys) --------
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_float_order_keys_group_like_numpy(fe_host, dtype):
    # the device groups the int64 order keys; their ranks must be the host's
    # grouping of the float keys (np.unique: -0.0 == 0.0, NaN last and equal)
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.standard_normal(5000) * 10.0 ** rng.integers(-30, 30, 5000),
                        [0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 1e-310, -1e-310,
                         np.finfo(np.float64).max, -np.finfo(np.float64).max]])
    with np.errstate(over="ignore"):  # float32: values beyond its range become +-inf
        x = np.concatenate([x, rng.choice(x, 3000)]).astype(dtype)
    rng.shuffle(x)
    host = fe_host.FixedEffect(x)
    k = fe_host._order_key(x)
    uniq, inv = np.unique(k, return_inverse=True)
    assert uniq.size == host.n
    assert np.array_equal(inv.reshape(-1) + 1, host.refs)
    # multi-key tuples fold the same way
    y = rng.integers(0, 3, x.size)
    host2 = fe_host.FixedEffect(x, y)
    _, inv2 = np.unique(np.stack([k, y], axis=1), axis=0, return_inverse=True)
    assert np.array_equal(inv2.reshape(-1) + 1, host2.refs)


def test_bench_throughput_figures():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    stats = {"expand": {"bytes": 4e9, "ms": 10.0, "launches": 4},
             "scalar": {"bytes": 0.0, "ms": 1.0, "launches": 8}}
    t = b.throughput_figures(1000 * 8, [3, 5], stats, prof_steps=1, step_s=0.01, ranks=2)
    # 10 ms per step; 8 iterations of 1000 rows on each of 2 ranks
    assert t["observation_iterations_per_s"] == 1000 * 8 * 2 / 0.01
    assert t["lsmr_iterations_per_step"] == 16
    assert t["alg_bytes_per_step"] == 8e9
    assert abs(t["alg_GBps"] - 8e9 / 0.01 / 1e9) < 1e-9


@pytest.mark.parametrize("workload,maxiter", [("simple_10m", 10000), ("hard_800k_interacted", 300)])
def test_reference_arm_line_on_the_reference_benchmark_problems(workload, maxiter):
    """bench.py --impl reference prints one JSON line with the arm's fields on
    the reference's benchmark problems (shrunk 100x), with the problem's own
    iteration cap in its config."""
    import json
    import subprocess
    import sys
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--workload", workload, "--scale", "0.01", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    assert d["config"]["workload"] == workload and d["config"]["maxiter"] == maxiter
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def _entry_point_bodies():
    """(name, body) of every extern "C" entry point in the library sources."""
    csrc = Path(__file__).resolve().parent.parent / "fixedeffects.jl_b200" / "csrc"
    out = []
    for f in sorted(csrc.glob("*.cu")):
        src = f.read_text()
        # functions inside an extern "C" { ... } block, or declared extern "C" one by one
        for m in re.finditer(r'(?:^|\n)(?:extern "C" )?(?:int|const char\*) (fe_[a-z0-9_]+)\([^;{]*\)\s*\{',
                             src):
            start = m.end()
            depth, i = 1, start
            while depth and i < len(src):
                depth += {"{": 1, "}": -1}.get(src[i], 0)
                i += 1
            out.append((m.group(1), f.name, src[start:i]))
    return out


def test_every_entry_point_restores_the_callers_device():
    """Entry points that may switch devices save and restore the caller's
    current device (a Julia caller tracks its own device per task)."""
    bodies = _entry_point_bodies()
    names = {n for n, _, _ in bodies}
    assert set(_declared_symbols()) <= names | {"fe_version", "fe_last_error"}
    for name, fname, body in bodies:
        if name in ("fe_version", "fe_last_error"):
            continue
        assert "DeviceRestore" in body.split("\n", 2)[1], (name, fname)


def test_kernel_attributes_are_set_per_device():
    """cudaFuncSetAttribute applies to the current device only, so every
    setting of a kernel attribute sits behind a per-device record (a plan on a
    second GPU of the same process must set it again), never a process-wide
    flag."""
    csrc = Path(__file__).resolve().parent.parent / "fixedeffects.jl_b200" / "csrc"
    sites = 0
    for f in sorted(list(csrc.glob("*.cu")) + list(csrc.glob("*.cuh"))):
        lines = re.sub(r"//[^\n]*", "", f.read_text()).splitlines()
        assert not any(re.search(r"static bool attr_set", ln) for ln in lines), f.name
        for i, ln in enumerate(lines):
            if "cudaFuncSetAttribute(" in ln:
                sites += 1
                window = "\n".join(lines[max(0, i - 12):i])
                assert ("needed(" in window) or ("attr_smem[dev]" in window), (f.name, i + 1)
    assert sites >= 6


def test_noalloc_entry_point_calls_no_allocator():
    """fe_plan_scales_noalloc's translation unit never allocates device memory
    (no cudaMalloc / cudaFree / plan buffer growth)."""
    src = (Path(__file__).resolve().parent.parent / "fixedeffects.jl_b200" / "csrc"
           / "fe_noalloc.cu").read_text()
    code = re.sub(r"//[^\n]*", "", src)
    for word in ("cudaMalloc", "cudaFree", "cudaMallocAsync", ".ensure(", "new ", "malloc("):
        assert word not in code, word
