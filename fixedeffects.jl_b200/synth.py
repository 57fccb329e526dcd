"""Seeded synthetic workloads with the shapes of the five solver configurations
and of the reference's own benchmark problems (benchmark/run.jl).

The reference publishes no dataset for this path, so every workload here is
generated: numpy PCG64, seed 0 for the CPU-runnable two-FE case and the
configuration index otherwise.  Zipf(s) over 1..M is sampled by inverse CDF of
p(k) ~ k^-s; log-uniform N is exp(U(ln a, ln b)) rounded.  Level ids are
compacted to the observed levels (ascending original id), as FixedEffect's
GroupedArray compaction does (src/FixedEffect.jl:18-21).

``scale`` < 1 shrinks N and every level count by the same factor, which keeps
the observations-per-level ratios, for tests that must finish quickly.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

WORKLOADS = {
    0: "two_fe_1m: N=1e6, FEs 1e5 x 1e2 uniform, 1 column, unit weights",
    1: "three_fe_interacted_10m: N=1e7, FEs 1e6 x 1e2 x 1e3 (interacted), weighted, 1 column",
    2: "worker_firm_year_10m_32col: N=1e7, worker 2e6 uniform, firm Zipf(1.1) over 2e5, "
       "year 20, 32 Float32 columns",
    3: "uneven_256_problems: 256 problems, N log-uniform [1e3,1e6], 2-3 FEs, weighted",
    4: "large_zipf_100m_8col: N=1e8, FEs 1e7 uniform x Zipf(1.3) over 1e4, weighted, "
       "8 Float32 columns",
    5: "simple_10m: N=1e7, FEs 1e5 x 1e2 uniform, 1 column (the reference's benchmark)",
    6: "hard_800k: N=8e5, worker 4e5 x firm 5e4 linked locally, 1 column (the reference's "
       "benchmark)",
    7: "hard_800k_interacted: N=8e5, worker and worker x uniform, 1 column, maxiter 300 "
       "(the reference's benchmark)",
}


@dataclass
class Problem:
    refs: list            # list of int64 arrays, 1-based, compacted
    nlev: list            # level counts
    interaction: list     # per FE: None or float64 array
    weights: object       # None (unit) or float64 array
    Y: np.ndarray         # (N, ncols), Fortran order
    meta: dict = field(default_factory=dict)

    @property
    def N(self) -> int:
        return int(self.refs[0].shape[0])


def compact(refs: np.ndarray):
    """Maps arbitrary positive integer keys to 1..n (ascending original id)."""
    refs = np.asarray(refs, dtype=np.int64)
    if refs.size == 0:
        return refs.copy(), 0
    mx = int(refs.max())
    present = np.zeros(mx + 1, dtype=np.int64)
    present[refs] = 1
    newid = np.cumsum(present)
    out = newid[refs]
    return out.astype(np.int64, copy=False), int(newid[-1])


def zipf_refs(rng, s: float, M: int, N: int) -> np.ndarray:
    k = np.arange(1, M + 1, dtype=np.float64)
    p = k ** (-s)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    u = rng.random(N)
    return (np.searchsorted(cdf, u, side="left") + 1).astype(np.int64)


def _scaled(n: float, scale: float, lo: int = 2) -> int:
    return max(lo, int(round(n * scale)))


def config0(scale: float = 1.0, seed: int = 0) -> Problem:
    rng = np.random.default_rng(seed)
    N = _scaled(1_000_000, scale, 10)
    n1 = _scaled(100_000, scale)
    r1 = rng.integers(1, n1 + 1, N)
    r2 = rng.integers(1, 101, N)
    a = rng.standard_normal(n1 + 1)
    c = rng.standard_normal(101)
    y = a[r1] + c[r2] + rng.standard_normal(N)
    refs, nlev = zip(*(compact(r) for r in (r1, r2)))
    return Problem(list(refs), list(nlev), [None, None], None,
                   np.asfortranarray(y[:, None]), {"config": 0})


def config1(scale: float = 1.0, seed: int = 1) -> Problem:
    rng = np.random.default_rng(seed)
    N = _scaled(10_000_000, scale, 10)
    n1 = _scaled(1_000_000, scale)
    r1 = rng.integers(1, n1 + 1, N)
    r2 = rng.integers(1, 101, N)
    r3 = rng.integers(1, 1001, N)
    inter3 = rng.random(N)
    w = rng.uniform(0.5, 1.5, N)
    y = (rng.standard_normal(n1 + 1)[r1] + rng.standard_normal(101)[r2]
         + inter3 * rng.standard_normal(1001)[r3] + rng.standard_normal(N))
    refs, nlev = zip(*(compact(r) for r in (r1, r2, r3)))
    return Problem(list(refs), list(nlev), [None, None, inter3], w,
                   np.asfortranarray(y[:, None]), {"config": 1})


def _columns_like_config2(rng, refs_worker, refs_firm, nw, nf, N, ncols):
    Y = np.empty((N, ncols), dtype=np.float32, order="F")
    for j in range(ncols):
        s = rng.uniform(0.1, 2.0)
        col = rng.standard_normal(N, dtype=np.float32)
        col += np.float32(s) * rng.standard_normal(nf + 1, dtype=np.float32)[refs_firm]
        col += np.float32(s) * rng.standard_normal(nw + 1, dtype=np.float32)[refs_worker]
        Y[:, j] = col
    return Y


def config2(scale: float = 1.0, seed: int = 2, ncols: int = 32) -> Problem:
    rng = np.random.default_rng(seed)
    N = _scaled(10_000_000, scale, 10)
    nw = _scaled(2_000_000, scale)
    nf = _scaled(200_000, scale)
    worker = rng.integers(1, nw + 1, N)
    firm = zipf_refs(rng, 1.1, nf, N)
    year = rng.integers(1, 21, N)
    Y = _columns_like_config2(rng, worker, firm, nw, nf, N, ncols)
    refs, nlev = zip(*(compact(r) for r in (worker, firm, year)))
    return Problem(list(refs), list(nlev), [None, None, None], None, Y,
                   {"config": 2})


def config3(scale: float = 1.0, seed: int = 3, nproblems: int = 256) -> list:
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = np.log(1e3 * scale if scale < 1 else 1e3), np.log(1e6 * scale)
    lo = min(lo, hi)
    for _ in range(nproblems):
        N = max(10, int(round(np.exp(rng.uniform(lo, hi)))))
        three = bool(rng.random() < 0.5)
        n1 = max(2, N // 10)
        r1 = rng.integers(1, n1 + 1, N)
        r2 = rng.integers(1, 51, N)
        raw = [r1, r2]
        inter = [None, None]
        if three:
            raw.append(rng.integers(1, 501, N))
            inter.append(rng.random(N))
        w = rng.uniform(0.5, 1.5, N)
        y = (rng.standard_normal(n1 + 1)[r1] + rng.standard_normal(51)[r2]
             + rng.standard_normal(N)).astype(np.float32)
        refs, nlev = zip(*(compact(r) for r in raw))
        out.append(Problem(list(refs), list(nlev), inter, w,
                           np.asfortranarray(y[:, None]), {"config": 3}))
    return out


def config4(scale: float = 1.0, seed: int = 4, ncols: int = 8) -> Problem:
    rng = np.random.default_rng(seed)
    N = _scaled(100_000_000, scale, 10)
    n1 = _scaled(10_000_000, scale)
    n2 = _scaled(10_000, scale)
    r1 = rng.integers(1, n1 + 1, N)
    r2 = zipf_refs(rng, 1.3, n2, N)
    w = rng.uniform(0.5, 1.5, N)
    Y = _columns_like_config2(rng, r1, r2, n1, n2, N, ncols)
    refs, nlev = zip(*(compact(r) for r in (r1, r2)))
    return Problem(list(refs), list(nlev), [None, None], w, Y, {"config": 4})


# The reference's own benchmark problems (benchmark/run.jl:6-28), with its
# shapes and value distributions drawn from numpy instead of Julia's RNG:
# uniform level ids, columns uniform on [0, 1).  `maxiter` is the iteration
# cap that benchmark/run.jl gives the solve (None: the default 10000).
def simple_10m(scale: float = 1.0, seed: int = 5) -> Problem:
    """N = 1e7, FEs of N/100 and 100 uniform levels (benchmark/run.jl:9-15)."""
    rng = np.random.default_rng(seed)
    N = _scaled(10_000_000, scale, 10)
    K = 100
    r1 = rng.integers(1, max(2, N // K) + 1, N)
    r2 = rng.integers(1, K + 1, N)
    x = rng.random(N)
    refs, nlev = zip(*(compact(r) for r in (r1, r2)))
    return Problem(list(refs), list(nlev), [None, None], None,
                   np.asfortranarray(x[:, None]), {"config": 5, "maxiter": None})


def _worker_firm_800k(rng, scale):
    """pid uniform over M = 4e5 workers; each worker's firm is drawn from the
    21 firms around pid / 8, clipped to 1..5e4 (benchmark/run.jl:18-25)."""
    N = _scaled(800_000, scale, 10)
    M = _scaled(400_000, scale)
    O = _scaled(50_000, scale)
    pid = rng.integers(1, M + 1, N)
    lo = np.maximum(1, pid // 8 - 10)
    hi = np.minimum(O, pid // 8 + 10)
    hi = np.maximum(hi, lo)
    fid = lo + np.floor(rng.random(N) * (hi - lo + 1)).astype(np.int64)
    return N, pid, fid


def hard_800k(scale: float = 1.0, seed: int = 6) -> Problem:
    """Worker-firm FEs (4e5 x 5e4 levels, linked locally), one column
    (benchmark/run.jl:17-25, solved at the default maxiter as :39-42)."""
    rng = np.random.default_rng(seed)
    N, pid, fid = _worker_firm_800k(rng, scale)
    x = rng.random(N)
    refs, nlev = zip(*(compact(r) for r in (pid, fid)))
    return Problem(list(refs), list(nlev), [None, None], None,
                   np.asfortranarray(x[:, None]), {"config": 6, "maxiter": None})


def hard_800k_interacted(scale: float = 1.0, seed: int = 7) -> Problem:
    """The worker FE and the worker FE interacted with a uniform variable
    (benchmark/run.jl:26-27), maxiter = 300 as :49-52."""
    rng = np.random.default_rng(seed)
    N, pid, _ = _worker_firm_800k(rng, scale)
    x = rng.random(N)
    y = rng.random(N)
    ref, n = compact(pid)
    return Problem([ref, ref.copy()], [n, n], [None, y], None,
                   np.asfortranarray(x[:, None]), {"config": 7, "maxiter": 300})


def make(config: int, scale: float = 1.0, **kw):
    return {0: config0, 1: config1, 2: config2, 3: config3, 4: config4, 5: simple_10m,
            6: hard_800k, 7: hard_800k_interacted}[config](scale=scale, **kw)
