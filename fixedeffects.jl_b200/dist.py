"""Column sharding over ranks (one process per GPU).

The columns of a solve_residuals! matrix are independent problems, so N GPUs
split them with no collective on the data path: rank r solves a contiguous
column range on its own device, and the results are gathered once at the end
(an all-gather over the process group; NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced [lo, hi) share of n items for `rank`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def solve_columns_sharded(Y, solve_fn, group=None):
    """Solves this rank's columns of Y with ``solve_fn(Y_shard) -> (R, iters,
    converged)`` and all-gathers the results.  Every rank returns the full
    (R, iterations, converged); columns keep their original order.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    Y = np.asarray(Y)
    ncols = Y.shape[1]
    lo, hi = shard_range(ncols, world, rank)
    R, its, cvs = solve_fn(np.asfortranarray(Y[:, lo:hi]))
    R = np.asarray(R, dtype=np.float64).reshape(Y.shape[0], hi - lo)
    payload = {"lo": lo, "hi": hi, "R": R, "its": np.asarray(its, dtype=np.int64),
               "cvs": np.asarray(cvs, dtype=bool)}
    parts = [None] * world
    dist.all_gather_object(parts, payload, group=group)
    R_all = np.empty((Y.shape[0], ncols), dtype=np.float64, order="F")
    its_all = np.zeros(ncols, dtype=np.int64)
    cvs_all = np.zeros(ncols, dtype=bool)
    for p in parts:
        R_all[:, p["lo"]:p["hi"]] = p["R"]
        its_all[p["lo"]:p["hi"]] = p["its"]
        cvs_all[p["lo"]:p["hi"]] = p["cvs"]
    return R_all, its_all, cvs_all
