"""Multi-rank host logic on CPU: world_size 2 over gloo.  Column sharding:
each rank solves its columns (here with the oracle as the solver), keeps
them, and the optional tensor all-gather reassembles them in order; the
result equals a single-process solve.  Observation sharding: the split by
whole primary levels (the library's sharded solve itself needs a GPU and is
tested in test_gpu_sharded.py)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, Y, refs, nlev, out_dir):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.dist as D
    from oracle import oracle as O

    def solve(Ys):
        return O.solve_residuals_cols(Ys, refs, nlev, tol=1e-10, nthreads=1)

    lo, hi, Rs, its_s, _ = D.solve_columns_sharded(Y, solve)
    np.save(os.path.join(out_dir, f"Rs{rank}.npy"), Rs)
    np.save(os.path.join(out_dir, f"lohi{rank}.npy"), np.array([lo, hi]))
    R, its, cvs = D.solve_columns_sharded(Y, solve, gather=True)
    np.save(os.path.join(out_dir, f"R{rank}.npy"), R)
    np.save(os.path.join(out_dir, f"its{rank}.npy"), its)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range_partitions():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.dist as D
    for n in (0, 1, 7, 32, 33):
        for w in (1, 2, 3, 8):
            rs = [D.shard_range(n, w, r) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(h - l for l, h in rs) - min(h - l for l, h in rs) <= 1


def test_two_rank_gloo_matches_single(tmp_path, oracle):
    rng = np.random.default_rng(3)
    N, ncols = 4000, 5
    refs = [rng.integers(1, 200, N).astype(np.int64), rng.integers(1, 12, N).astype(np.int64)]
    nlev = [int(r.max()) for r in refs]
    Y = np.asfortranarray(rng.standard_normal((N, ncols)))
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, Y, refs, nlev, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    R_single, its_single, _ = oracle.solve_residuals_cols(Y, refs, nlev, tol=1e-10)
    for r in range(2):
        R = np.load(tmp_path / f"R{r}.npy")
        its = np.load(tmp_path / f"its{r}.npy")
        assert np.allclose(R, R_single, rtol=0, atol=1e-12)
        assert np.array_equal(its, its_single)
        lo, hi = np.load(tmp_path / f"lohi{r}.npy")
        assert np.array_equal(np.load(tmp_path / f"Rs{r}.npy"), R[:, lo:hi])


def test_shard_by_primary_levels():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.dist as D
    rng = np.random.default_rng(4)
    for n, N, world in ((50, 1000, 2), (7, 60, 3), (1000, 20000, 8), (4, 4, 3)):
        refs = rng.integers(1, n + 1, N) if N > n else np.arange(1, N + 1)
        refs = refs.copy()
        refs[refs == 2] = 3  # an unobserved level
        shards = D.shard_by_primary_levels(refs, n, world)
        assert len(shards) == world
        # consecutive whole-level ranges covering every level, every rank non-empty
        assert shards[0][0] == 1 and shards[-1][1] == n + 1
        assert all(a[1] == b[0] for a, b in zip(shards, shards[1:]))
        allidx = np.concatenate([s[2] for s in shards])
        assert np.array_equal(np.sort(allidx), np.arange(N))
        for lo, hi, idx in shards:
            assert idx.size > 0 and np.all(np.diff(idx) > 0)
            assert np.all((refs[idx] >= lo) & (refs[idx] < hi))
        sizes = [s[2].size for s in shards]
        if N >= 1000:  # balanced to within a few levels' rows
            assert max(sizes) - min(sizes) <= 4 * np.bincount(refs).max()
    with pytest.raises(ValueError):
        D.shard_by_primary_levels(np.array([1, 1, 1]), 1, 2)
    assert D.primary_index([10, 30, 30, 5]) == 1
    assert D.primary_index([3]) == 0
