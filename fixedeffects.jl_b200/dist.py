"""Multi-GPU forms of the solver (one process per GPU, torch.distributed).

Two ways to use N GPUs:

* Column sharding (independent units, no collective on the data path): the
  columns of a solve_residuals! matrix, or independent problems, are split
  into contiguous ranges; each rank solves its range on its own GPU and keeps
  its results where they are.  ``solve_columns_sharded`` does this and, on
  request, gathers the results with one tensor all-gather.

* Observation sharding of ONE problem (for a problem whose rows exceed one
  GPU, or to put N GPUs on a single column): the observations are split by
  whole levels of the primary FE (``shard_by_primary_levels``), each rank
  builds a sharded plan over its rows (``ShardedSolver``, the C entry point
  fe_plan_create_sharded) and LSMR runs over the global problem.  Every
  iteration sums, over the ranks, the per-column norms of the local rows and
  the per-level sums A'u of the local rows (the exchange between the two
  matrix-vector products of src/utils/lsmr.jl:104-109); the coefficient side
  is replicated and stays identical on every rank.  The exchange is an
  all-reduce: NCCL on the device for the "nccl" backend, or staged through
  host memory for "gloo".
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import FixedEffect, _ptrs, _weights_array, _precision_of


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced [lo, hi) share of n items for `rank`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def solve_columns_sharded(Y, solve_fn, group=None, gather: bool = False):
    """Solves this rank's contiguous column range of Y with
    ``solve_fn(Y_shard) -> (R, iterations, converged)``.

    Returns ``(lo, hi, R_shard, iterations, converged)``: the results stay on
    the rank that computed them.  With ``gather=True`` the residuals are
    all-gathered as one tensor in the shard's dtype (padded to equal widths)
    and every rank returns ``(R, iterations, converged)`` for all columns in
    their original order.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    Y = np.asarray(Y)
    N, ncols = Y.shape
    lo, hi = shard_range(ncols, world, rank)
    R, its, cvs = solve_fn(np.asfortranarray(Y[:, lo:hi]))
    R = np.asarray(R).reshape(N, hi - lo)
    its = np.asarray(its, dtype=np.int64).reshape(hi - lo)
    cvs = np.asarray(cvs, dtype=bool).reshape(hi - lo)
    if not gather:
        return lo, hi, R, its, cvs
    width = -(-ncols // world)
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    dt = torch.float32 if R.dtype == np.float32 else torch.float64
    mine = torch.zeros((width, N), dtype=dt, device=dev)
    meta = torch.zeros((width, 2), dtype=torch.int64, device=dev)
    if hi > lo:
        mine[: hi - lo] = torch.from_numpy(np.ascontiguousarray(R.T)).to(dev)
        meta[: hi - lo, 0] = torch.from_numpy(its).to(dev)
        meta[: hi - lo, 1] = torch.from_numpy(cvs.astype(np.int64)).to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    metas = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    dist.all_gather(metas, meta, group=group)
    R_all = np.empty((N, ncols), dtype=R.dtype, order="F")
    its_all = np.zeros(ncols, dtype=np.int64)
    cvs_all = np.zeros(ncols, dtype=bool)
    for r in range(world):
        a, b = shard_range(ncols, world, r)
        R_all[:, a:b] = parts[r][: b - a].cpu().numpy().T
        m = metas[r][: b - a].cpu().numpy()
        its_all[a:b] = m[:, 0]
        cvs_all[a:b] = m[:, 1] != 0
    return R_all, its_all, cvs_all


# ---------------------------------------------------------------------------
# observation sharding
# ---------------------------------------------------------------------------
def primary_index(n_levels) -> int:
    """The FE whose levels order the observations in a plan: the one with the
    most levels (the first of them on ties)."""
    n_levels = list(n_levels)
    return int(max(range(len(n_levels)), key=lambda k: (n_levels[k], -k)))


def shard_by_primary_levels(primary_refs, n_levels_primary: int, world: int):
    """Splits the observations of a problem over `world` ranks by whole
    levels of the primary FE: rank r gets the levels [lo_r, hi_r) (1-based,
    half-open, consecutive) chosen so that the ranks' row counts are as even
    as whole levels allow, and every rank gets at least one observation.

    Returns a list of (level_lo, level_hi, observation_index_array), the
    indices in ascending (original) order."""
    refs = np.asarray(primary_refs, dtype=np.int64)
    n = int(n_levels_primary)
    counts = np.bincount(refs, minlength=n + 1)[1:]
    nonempty = int(np.count_nonzero(counts))
    if world < 1 or nonempty < world:
        raise ValueError(f"cannot give {world} ranks whole primary levels: "
                         f"{nonempty} levels have observations")
    cum = np.cumsum(counts)
    total = int(cum[-1])
    ne = np.flatnonzero(counts)  # 0-based indices of the observed levels
    cuts = [0]
    for r in range(1, world):
        # the first level boundary at or past r/world of the rows, clamped so
        # that this rank gets an observed level and every later rank one too
        b = int(np.searchsorted(cum, total * r / world, side="left")) + 1
        first = int(ne[np.searchsorted(ne, cuts[-1])])  # this rank's first observed level
        b = max(b, first + 1)
        b = min(b, int(ne[len(ne) - (world - r)]))
        cuts.append(b)
    cuts.append(n)
    out = []
    for r in range(world):
        lo, hi = cuts[r] + 1, cuts[r + 1] + 1  # 1-based level ids [lo, hi)
        idx = np.flatnonzero((refs >= lo) & (refs < hi))
        if idx.size == 0:
            raise ValueError("a rank without observations (too few primary levels for the ranks)")
        out.append((lo, hi, idx))
    return out


class _DeviceArray:
    """A zero-copy view of library device memory for torch
    (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, count: int, dtype):
        self.__cuda_array_interface__ = {
            "shape": (int(count),), "typestr": np.dtype(dtype).str, "data": (int(ptr), False),
            "version": 3, "strides": None}


def make_exchange(group=None):
    """The fe_exchange_fn of a sharded plan over a torch.distributed group:
    an in-place sum all-reduce of the library's device buffer, on the
    library's stream.  NCCL reduces on the device; gloo goes through host
    memory (a synchronous device-to-host copy, the all-reduce, and the copy
    back)."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)

    def exchange(ctx, buf, count, dtype, stream):
        try:
            t = torch.as_tensor(_DeviceArray(buf, count, np.float64 if dtype == 0 else np.float32),
                                device="cuda")
            s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
            with torch.cuda.stream(s):
                if backend == "nccl":
                    dist.all_reduce(t, group=group)
                else:
                    h = t.cpu()
                    dist.all_reduce(h, group=group)
                    t.copy_(h)
            return 0
        except Exception:  # the library reports a failed exchange as FE_ERR_CUDA
            return 1

    return _lib.EXCHANGE_FN(exchange)


class ShardedSolver:
    """One rank's share of an observation-sharded problem.

    ``fes`` hold this rank's observations with GLOBAL level ids (1-based) and
    ``n_levels`` the global level counts; the share must consist of whole
    levels of the primary FE (``shard_by_primary_levels``).  Every rank of
    ``group`` constructs its solver and then makes the same calls with the
    same column counts, tolerances and options.
    """

    def __init__(self, fes, n_levels, weights=None, group=None, T=np.float32,
                 precision: str | None = None, device: int | None = None):
        import torch
        fes = list(fes)
        if not fes or any(len(f) != len(fes[0]) for f in fes):
            raise ValueError("the FixedEffects of a shard must have one common length")
        self.N = len(fes[0])
        self.K = len(fes)
        self.T = np.dtype(T)
        self.precision = _precision_of(precision, T)
        self.device = torch.cuda.current_device() if device is None else device
        self.n_levels = np.ascontiguousarray(n_levels, dtype=np.int64)
        self._refs = [np.ascontiguousarray(f.refs, dtype=np.int64) for f in fes]
        self._inter = [None if f.interaction is None else
                       np.ascontiguousarray(f.interaction, dtype=np.float64) for f in fes]
        w = _weights_array(weights, self.N)
        self._w = w
        self._xchg = make_exchange(group)  # kept alive as long as the plan
        h = ctypes.c_void_p()
        L = _lib.load()
        inter_pp = _ptrs(self._inter) if any(a is not None for a in self._inter) else None
        _lib.check(L.fe_plan_create_sharded(
            ctypes.byref(h), self.N, self.K, _ptrs(self._refs),
            self.n_levels.ctypes.data_as(_lib._i64p), inter_pp,
            None if w is None else w.ctypes.data_as(_lib._f64p), self.device, self._xchg, None))
        self._h = h

    def set_option(self, option: int, value: float) -> None:
        _lib.check(_lib.load().fe_plan_set_option(self._h, option, float(value)))

    def solve_residuals(self, Y, tol: float | None = None, maxiter: int = 100_000):
        """solve_residuals! of the global problem; returns the residuals of
        this rank's observations (Y: this rank's rows, a vector or an
        (N_local, ncols) matrix, solved in place when writable), the
        iterations and the convergence flags (the same on every rank)."""
        import math
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        a = np.asarray(Y)
        vec = a.ndim == 1
        if a.shape[0] != self.N:
            raise ValueError("Y must hold this rank's observations")
        if a.dtype not in (np.float64, np.float32):
            a = a.astype(np.float64)
        work = a if (a.flags.f_contiguous and a.flags.writeable) else np.array(a, order="F")
        if vec:
            work = work.reshape(-1, 1, order="F")
        ncols = work.shape[1]
        its = np.zeros(ncols, dtype=np.int64)
        cvs = np.zeros(ncols, dtype=np.uint8)
        dt = _lib.FE_DTYPE_F64 if work.dtype == np.float64 else _lib.FE_DTYPE_F32
        _lib.check(_lib.load().fe_solve_residuals(
            self._h, work.ctypes.data, dt, ncols, self.N, self.precision, float(tol),
            int(maxiter), its.ctypes.data_as(_lib._i64p), cvs.ctypes.data_as(_lib._u8p)))
        res = work.reshape(-1) if vec else work
        if isinstance(Y, np.ndarray) and res is not Y and Y.flags.writeable and Y.shape == res.shape:
            Y[...] = res
            res = Y
        if vec:
            return res, int(its[0]), bool(cvs[0])
        return res, its, cvs.astype(bool)

    def solve_coefficients(self, y, tol: float | None = None, maxiter: int = 100_000):
        """solve_coefficients! up to the normalisation: the global per-level
        coefficients x_k .* scale_k (the same on every rank), the iterations
        and the convergence flag."""
        import math
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        a = np.ascontiguousarray(y, dtype=np.float64 if np.asarray(y).dtype != np.float32
                                 else np.float32)
        if a.shape != (self.N,):
            raise ValueError("y must hold this rank's observations")
        coefs = [np.zeros(int(n), dtype=np.float64) for n in self.n_levels]
        it = ctypes.c_int64(0)
        cv = ctypes.c_uint8(0)
        dt = _lib.FE_DTYPE_F64 if a.dtype == np.float64 else _lib.FE_DTYPE_F32
        _lib.check(_lib.load().fe_solve_coefficients(
            self._h, a.ctypes.data, dt, self.precision, float(tol), int(maxiter), _ptrs(coefs),
            ctypes.byref(it), ctypes.byref(cv)))
        return coefs, int(it.value), bool(cv.value)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().fe_plan_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_problem(refs, n_levels, world: int, rank: int, interaction=None, weights=None):
    """This rank's FixedEffects (global level ids), weights and observation
    indices for an observation-sharded solve of the problem (refs: one
    1-based level-id array per FE)."""
    kp = primary_index(n_levels)
    lo, hi, idx = shard_by_primary_levels(refs[kp], n_levels[kp], world)[rank]
    inter = interaction if interaction is not None else [None] * len(refs)
    fes = [FixedEffect.from_refs(np.asarray(r)[idx], int(n), None if a is None else np.asarray(a)[idx])
           for r, n, a in zip(refs, n_levels, inter)]
    w = None if weights is None else np.asarray(weights)[idx]
    return fes, w, idx
