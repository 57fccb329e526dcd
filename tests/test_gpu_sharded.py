"""Observation-sharded solves (fe_plan_create_sharded) against the single-plan
solve and the oracle.

Two ranks (spawned processes, gloo) share the one GPU of the test host: each
builds the plan of its share of the observations (whole primary levels) and
the per-iteration sums are exchanged through host memory, so no kernel of one
process waits on the other.  The ranks' residuals, put back in the original
order, must match the single-plan solve and the oracle; the coefficients must
be identical on both ranks."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem(case):
    rng = np.random.default_rng(31)
    if case == "mixed_32col":
        # worker / firm (Zipf) / year, 32 columns: the absorbed 32-column path
        N = 120_000
        r1 = rng.integers(1, 24_001, N)
        k = np.arange(1, 2_401, dtype=np.float64)
        cdf = np.cumsum(k ** -1.1)
        r2 = np.searchsorted(cdf / cdf[-1], rng.random(N)) + 1
        r3 = rng.integers(1, 21, N)
        refs, inter, w = [r1, r2, r3], [None, None, None], None
        Y = np.asfortranarray(rng.standard_normal((N, 32)) + (r1 % 97)[:, None] * 0.1)
    else:
        # three FEs, the third interacted, weighted, one column
        N = 150_000
        r1 = rng.integers(1, 15_001, N)
        r2 = rng.integers(1, 101, N)
        r3 = rng.integers(1, 301, N)
        refs, inter, w = [r1, r2, r3], [None, None, rng.random(N)], rng.uniform(0.5, 1.5, N)
        Y = np.asfortranarray(rng.standard_normal((N, 1)) + (r1 % 13)[:, None])
    nlev = [int(r.max()) for r in refs]
    return refs, nlev, inter, w, Y


def _worker(rank, port, case, prec, out_dir):
    sys.path.insert(0, str(ROOT))
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                            timeout=datetime.timedelta(seconds=120))
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.dist as D
    refs, nlev, inter, w, Y = _problem(case)
    fes, ws, idx = D.shard_problem(refs, nlev, WORLD, rank, inter, w)
    sol = D.ShardedSolver(fes, nlev, ws, T=np.float64 if prec == "fp64" else np.float32,
                          precision=prec)
    R, its, cvs = sol.solve_residuals(np.asfortranarray(Y[idx]), tol=1e-8, maxiter=10000)
    np.save(os.path.join(out_dir, f"R{rank}.npy"), R)
    np.save(os.path.join(out_dir, f"idx{rank}.npy"), idx)
    np.save(os.path.join(out_dir, f"its{rank}.npy"), np.asarray(its))
    np.save(os.path.join(out_dir, f"cvs{rank}.npy"), np.asarray(cvs))
    if case == "fp64_1col":
        coefs, it, cv = sol.solve_coefficients(Y[idx, 0], tol=1e-8, maxiter=10000)
        for k, c in enumerate(coefs):
            np.save(os.path.join(out_dir, f"coef{rank}_{k}.npy"), c)
    sol.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("case,prec", [("fp64_1col", "fp64"), ("fp64_1col", "mixed"),
                                       ("mixed_32col", "mixed")])
def test_sharded_matches_single_plan(fe, oracle, tmp_path, case, prec):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, port, case, prec, str(tmp_path)))
             for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        if p.exitcode is None:
            p.kill()
        assert p.exitcode == 0, (case, prec)
    refs, nlev, inter, w, Y = _problem(case)
    R = np.empty_like(Y, dtype=np.float64)
    its_r = []
    for r in range(WORLD):
        idx = np.load(tmp_path / f"idx{r}.npy")
        R[idx] = np.load(tmp_path / f"R{r}.npy").reshape(len(idx), -1)
        its_r.append(np.load(tmp_path / f"its{r}.npy"))
        assert np.load(tmp_path / f"cvs{r}.npy").all()
    # every rank ran the same iterations (identical scalars)
    assert all(np.array_equal(its_r[0], x) for x in its_r[1:])
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(refs, nlev, inter)]
    feM = fe.AbstractFixedEffectSolver(fes, w, "CUDA", np.float64 if prec == "fp64" else np.float32,
                                       precision=prec)
    R1, its1, cvs1 = feM.solve_residuals(Y.copy(), tol=1e-8, maxiter=10000)
    feM.close()
    cols = range(0, Y.shape[1], 4)
    R_o, it_o, _ = oracle.solve_residuals_cols(Y[:, list(cols)], refs, nlev, inter, w, tol=1e-8)
    for jj, j in enumerate(cols):
        d1 = np.linalg.norm(R[:, j] - R1[:, j]) / np.linalg.norm(R1[:, j])
        do = np.linalg.norm(R[:, j] - R_o[:, jj]) / np.linalg.norm(R_o[:, jj])
        assert d1 < 1e-6 and do < 1e-6, (case, prec, j, d1, do)
    if prec == "fp64":
        assert np.all(np.abs(np.asarray(its_r[0]).reshape(-1) - np.asarray(it_o)) <= 1)
    if case == "fp64_1col":
        # global coefficients: the same on both ranks, and fitted values equal
        # to the oracle's (before normalisation the coefficients are unique
        # only up to one constant per component)
        for k in range(len(refs)):
            assert np.array_equal(np.load(tmp_path / f"coef0_{k}.npy"),
                                  np.load(tmp_path / f"coef1_{k}.npy"))
        coefs = [np.load(tmp_path / f"coef0_{k}.npy") for k in range(len(refs))]
        fit = sum(c[r - 1] * (1 if a is None else a) for c, r, a in zip(coefs, refs, inter))
        _, full_o, _, _ = oracle.solve_coefficients(Y[:, 0], refs, nlev, inter, w, tol=1e-8)
        fit_o = sum(c * (1 if a is None else a) for c, a in zip(full_o, inter))
        assert np.linalg.norm(fit - fit_o) / np.linalg.norm(fit_o) < 1e-6
