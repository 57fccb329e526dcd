"""B200-native solver path of FixedEffects.jl, with a Python host binding.

This package mirrors the reference's public API for its solver path
(src/FixedEffects.jl:42-45 exports, src/AbstractFixedEffectSolver.jl):

    FixedEffect(refs...; interaction)                 src/FixedEffect.jl:7-21
    AbstractFixedEffectSolver(fes, w, method, T)      src/AbstractFixedEffectSolver.jl:8,
                                                      ext/CUDAExt.jl:99-110
    update_weights(feM, w)                            src/SolverCPU.jl:67-76
    solve_residuals(y, fes, w; method, double_precision, tol, maxiter)
                                                      src/AbstractFixedEffectSolver.jl:37-97
    solve_coefficients(y, fes, w; ...)                src/AbstractFixedEffectSolver.jl:137-160

Julia's trailing ``!`` is dropped from the names.  All arithmetic runs in
libfe_b200.so (sm_100a CUDA) through the C ABI of include/fe_b200.h; there is
no CPU fallback.  The method symbols ``"CUDA"`` (the reference's
``Val{:CUDA}``) and ``"gpu"`` select it.

Precision: ``double_precision=True`` (or ``T=np.float64``) runs the plain FP64
LSMR.  ``double_precision=False`` runs FP32 bulk passes with FP64 scalars and
FP64 iterative refinement until the reference's tests hold in FP64 at ``tol``
(``precision="mixed"``); ``precision="fp32"`` skips the refinement.
"""
from __future__ import annotations

import ctypes
import math
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import (FE_DTYPE_F32, FE_DTYPE_F64, FE_PREC_FP32, FE_PREC_FP64,
                   FE_PREC_MIXED, FEError)

__all__ = [
    "FixedEffect", "AbstractFixedEffectSolver", "FixedEffectSolverB200", "BatchSolver",
    "solve_residuals", "solve_coefficients", "update_weights", "normalize", "full",
    "components", "group_keys", "DimensionMismatch", "FEError",
]

_METHODS = {"CUDA", "cuda", "gpu", "GPU"}
_PREC = {"fp64": FE_PREC_FP64, "mixed": FE_PREC_MIXED, "fp32": FE_PREC_FP32}


class DimensionMismatch(ValueError):
    """Raised where the reference throws DimensionMismatch."""


def _compact(keys) -> tuple[np.ndarray, int]:
    """GroupedArray-style compaction to 1..n (ascending key order)."""
    a = np.asarray(keys)
    if a.size == 0:
        return np.zeros(0, dtype=np.int64), 0
    if a.dtype.kind in "iu" and a.min() >= 0 and a.max() <= 4 * a.size + 1024:
        mx = int(a.max())
        present = np.zeros(mx + 1, dtype=np.int64)
        present[a] = 1
        newid = np.cumsum(present)
        return newid[a].astype(np.int64), int(newid[-1])
    uniq, inv = np.unique(a, return_inverse=True)
    return (inv.reshape(-1) + 1).astype(np.int64), int(uniq.size)


_SIGNLESS = np.int64(0x7FFFFFFFFFFFFFFF)


def _order_key(a: np.ndarray) -> np.ndarray:
    """int64 keys that sort and compare like the float values of ``a``, as
    ``np.unique`` does: -0.0 equals 0.0, every NaN is one value after +inf.
    Non-negative doubles keep their bit pattern; negative ones flip every bit
    but the sign, so a larger magnitude gives a smaller key."""
    x = np.array(a, dtype=np.float64)
    x[x == 0.0] = 0.0
    x[np.isnan(x)] = np.nan
    bits = x.view(np.int64)
    return np.where(bits < 0, bits ^ _SIGNLESS, bits)


def group_keys(*keys, device: int = 0) -> tuple[np.ndarray, int]:
    """Level ids of integer or floating-point key tuples, grouped on the GPU
    (fe_group_keys): 1-based ranks of the distinct tuples in lexicographic
    ascending order, and their count.  The same ids as the host grouping of
    ``FixedEffect``.  Floating-point keys are first mapped to int64 keys of
    the same order (``_order_key``)."""
    if not keys:
        raise ValueError("group_keys needs at least one key vector")
    cols = []
    for a in keys:
        a = np.asarray(a)
        if a.ndim != 1 or a.dtype.kind not in "iubf":
            raise TypeError("device grouping takes 1-d integer or floating-point key vectors")
        if a.dtype.kind == "f":
            cols.append(_order_key(a))
            continue
        if a.dtype.kind == "u" and a.size and int(a.max()) > np.iinfo(np.int64).max:
            raise TypeError("unsigned keys above 2^63-1 are not supported")
        cols.append(np.ascontiguousarray(a, dtype=np.int64))
    n = cols[0].shape[0]
    if any(c.shape[0] != n for c in cols):
        raise DimensionMismatch("all key vectors must have the same length")
    refs = np.empty(n, dtype=np.int64)
    nl = ctypes.c_int64(0)
    _lib.check(_lib.load().fe_group_keys(_ptrs(cols), len(cols), n, int(device),
                                         refs.ctypes.data_as(_lib._i64p), ctypes.byref(nl)))
    return refs, int(nl.value)


class FixedEffect:
    """A fixed effect: 1-based level ids, an optional interaction, level count.

    ``FixedEffect(a, b, ...)`` groups observations by the tuple of keys, like
    ``GroupedArray(args..., sort=nothing)`` (src/FixedEffect.jl:18-21); ids
    are assigned in ascending key order.  ``interaction=None`` is the
    reference's UnitWeights.  ``device=d`` groups integer or floating-point
    keys on GPU ``d`` (fe_group_keys: presence flags or a radix sort);
    otherwise the grouping runs in numpy on the host, where the reference runs
    it too.
    """

    __slots__ = ("refs", "interaction", "n")

    def __init__(self, *args, interaction=None, device: int | None = None):
        if not args:
            raise ValueError("FixedEffect needs at least one key vector")
        if device is not None:
            refs, n = group_keys(*args, device=device)
        elif len(args) == 1:
            refs, n = _compact(args[0])
        else:
            cols = [_compact(a)[0] for a in args]
            m = len(cols[0])
            if any(len(c) != m for c in cols):
                raise DimensionMismatch("all key vectors must have the same length")
            refs, n = _compact(np.unique(np.stack(cols, axis=1), axis=0, return_inverse=True)[1])
        if interaction is not None:
            interaction = np.asarray(interaction, dtype=np.float64)
            if interaction.shape[0] != refs.shape[0]:
                raise DimensionMismatch(
                    f"cannot match refs of length {refs.shape[0]} with interaction of length "
                    f"{interaction.shape[0]}")
        self.refs = refs
        self.interaction = interaction
        self.n = n

    @classmethod
    def from_refs(cls, refs, n: int, interaction=None) -> "FixedEffect":
        """The inner constructor FixedEffect{R,I}(refs, interaction, n): refs
        are taken as given (1-based, no compaction)."""
        fe = cls.__new__(cls)
        fe.refs = np.ascontiguousarray(refs, dtype=np.int64)
        if interaction is not None:
            interaction = np.asarray(interaction, dtype=np.float64)
            if interaction.shape[0] != fe.refs.shape[0]:
                raise DimensionMismatch(
                    f"cannot match refs of length {fe.refs.shape[0]} with interaction of "
                    f"length {interaction.shape[0]}")
        fe.interaction = interaction
        fe.n = int(n)
        return fe

    def __len__(self) -> int:
        return int(self.refs.shape[0])

    @property
    def size(self):
        return (len(self),)

    def __getitem__(self, esample):
        """Row subset keeping n (src/FixedEffect.jl:44-50)."""
        if isinstance(esample, slice) and esample == slice(None):
            return self
        idx = np.asarray(esample)
        if idx.ndim != 1:
            raise TypeError("FixedEffect rows are indexed by a vector")
        inter = None if self.interaction is None else self.interaction[idx]
        return FixedEffect.from_refs(self.refs[idx], self.n, inter)

    def __repr__(self) -> str:
        return "Fixed Effects"

    def __eq__(self, other) -> bool:
        if not isinstance(other, FixedEffect):
            return NotImplemented
        ia, ib = self.interaction, other.interaction
        same_i = (ia is None and ib is None) or (
            ia is not None and ib is not None and np.array_equal(ia, ib))
        return self.n == other.n and np.array_equal(self.refs, other.refs) and same_i


def _ptrs(arrays):
    return (ctypes.c_void_p * len(arrays))(*[0 if a is None else a.ctypes.data for a in arrays])


def _weights_array(w, n):
    if w is None:
        return None
    a = np.ascontiguousarray(w, dtype=np.float64)
    if a.shape != (n,):
        raise DimensionMismatch("weights must have one value per observation")
    return a


def _precision_of(precision, T):
    if precision is not None:
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        return _PREC[precision]
    return FE_PREC_FP64 if np.dtype(T) == np.float64 else FE_PREC_MIXED


class FixedEffectSolverB200:
    """The solver object: a device-resident plan plus solve options.

    Equivalent of FixedEffectSolverCUDA{T} (ext/CUDAExt.jl:86-97).  ``T`` is
    the reference's element type: float64 -> FP64 LSMR, float32 -> mixed
    precision refined in FP64 (unless ``precision`` says otherwise).
    """

    def __init__(self, fes: Sequence[FixedEffect], weights=None, method: str = "CUDA",
                 T=np.float64, precision: str | None = None, device: int = 0):
        if method not in _METHODS:
            raise ValueError(f"method {method!r} is not provided by this library (use 'CUDA')")
        fes = list(fes)
        if not fes:
            raise ValueError("at least one FixedEffect is required")
        N = len(fes[0])
        if any(len(fe) != N for fe in fes):
            raise DimensionMismatch("all FixedEffects must have the same length")
        self.fes = fes
        self.T = np.dtype(T)
        self.precision = _precision_of(precision, T)
        self.N = N
        self.device = device
        L = _lib.load()
        self._refs = [np.ascontiguousarray(fe.refs, dtype=np.int64) for fe in fes]
        self._nlev = np.ascontiguousarray([fe.n for fe in fes], dtype=np.int64)
        self._inter = [None if fe.interaction is None else
                       np.ascontiguousarray(fe.interaction, dtype=np.float64) for fe in fes]
        w = _weights_array(weights, N)
        self.weights = w
        h = ctypes.c_void_p()
        inter_pp = _ptrs(self._inter) if any(a is not None for a in self._inter) else None
        _lib.check(L.fe_plan_create(ctypes.byref(h), N, len(fes), _ptrs(self._refs),
                                    self._nlev.ctypes.data_as(_lib._i64p), inter_pp,
                                    None if w is None else w.ctypes.data_as(_lib._f64p), device))
        self._h = h

    # -- reference API ------------------------------------------------------
    def update_weights(self, weights) -> "FixedEffectSolverB200":
        w = _weights_array(weights, self.N)
        _lib.check(_lib.load().fe_plan_update_weights(
            self._h, None if w is None else w.ctypes.data_as(_lib._f64p)))
        self.weights = w
        return self

    def solve_residuals(self, y, tol: float | None = None, maxiter: int = 100_000):
        """solve_residuals!(r, feM; tol, maxiter) (src/AbstractFixedEffectSolver.jl:49-97).

        ``y``: a vector, an (N, ncols) matrix (columns solved as one batch), a
        list of vectors, or a CUDA torch tensor (solved in device memory).
        Returns (y, iterations, converged), y overwritten when writable.
        """
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        if _is_cuda_tensor(y):
            return self._solve_device(y, tol, maxiter)
        if isinstance(y, (list, tuple)):
            return self._solve_columns(y, tol, maxiter)
        a = np.asarray(y)
        vec = a.ndim == 1
        if a.shape[0] != self.N:
            raise ValueError("FixedEffects must have the same length as y")
        if a.dtype not in (np.float64, np.float32):
            a = a.astype(np.float64)
        work = a if (a.flags.f_contiguous and a.flags.writeable) else np.array(a, order="F")
        if vec:
            work = work.reshape(-1, 1, order="F")
        ncols = work.shape[1]
        its = np.zeros(ncols, dtype=np.int64)
        cvs = np.zeros(ncols, dtype=np.uint8)
        dt = FE_DTYPE_F64 if work.dtype == np.float64 else FE_DTYPE_F32
        _lib.check(_lib.load().fe_solve_residuals(
            self._h, work.ctypes.data, dt, ncols, self.N, self.precision, float(tol), int(maxiter),
            its.ctypes.data_as(_lib._i64p), cvs.ctypes.data_as(_lib._u8p)))
        res = work.reshape(-1) if vec else work
        if isinstance(y, np.ndarray) and res is not y and y.flags.writeable and y.shape == res.shape:
            y[...] = res
            res = y
        if vec:
            return res, int(its[0]), bool(cvs[0])
        return res, its, cvs.astype(bool)

    def _solve_columns(self, ys, tol, maxiter):
        """The collection method (src/AbstractFixedEffectSolver.jl:74-97): all
        columns in one batched call (fe_solve_residuals_columns), each solved
        in place when it is a writable float32/float64 vector."""
        cols = []
        for c in ys:
            a = np.asarray(c)
            if a.ndim != 1 or a.shape[0] != self.N:
                raise ValueError("FixedEffects must have the same length as y")
            cols.append(a)
        if not cols:
            return ys, [], []
        dt = np.float32 if all(a.dtype == np.float32 for a in cols) else np.float64
        # read-only or non-contiguous columns are solved in a copy
        work = [a if (a.dtype == dt and a.flags.c_contiguous and a.flags.writeable)
                else np.array(a, dtype=dt, order="C") for a in cols]
        its = np.zeros(len(work), dtype=np.int64)
        cvs = np.zeros(len(work), dtype=np.uint8)
        _lib.check(_lib.load().fe_solve_residuals_columns(
            self._h, _ptrs(work), FE_DTYPE_F64 if dt == np.float64 else FE_DTYPE_F32, len(work),
            self.precision, float(tol), int(maxiter), its.ctypes.data_as(_lib._i64p),
            cvs.ctypes.data_as(_lib._u8p)))
        out = list(ys) if isinstance(ys, tuple) else ys
        for j, (a, w) in enumerate(zip(cols, work)):
            if w is a:
                continue
            if (isinstance(ys[j], np.ndarray) and ys[j].flags.writeable
                    and ys[j].dtype.kind == "f"):
                ys[j][...] = w
            elif isinstance(out, list):
                out[j] = w
        return out, [int(i) for i in its], [bool(c) for c in cvs]

    def _solve_device(self, y, tol, maxiter):
        import torch
        if y.dtype not in (torch.float64, torch.float32):
            raise TypeError("device y must be float64 or float32")
        vec = y.dim() == 1
        if y.shape[0] != self.N:
            raise ValueError("FixedEffects must have the same length as y")
        ncols = 1 if vec else y.shape[1]
        if vec:
            if not y.is_contiguous():
                raise ValueError("device y must be contiguous")
            ld = self.N
        else:
            if y.stride(0) != 1 and ncols > 1:
                raise ValueError("device Y must be column-major (y.t() contiguous)")
            # a single column is contiguous whatever stride torch reports for
            # its size-1 dimension
            ld = y.stride(1) if ncols > 1 else self.N
        its = np.zeros(ncols, dtype=np.int64)
        cvs = np.zeros(ncols, dtype=np.uint8)
        dt = FE_DTYPE_F64 if y.dtype == torch.float64 else FE_DTYPE_F32
        L = _lib.load()
        _lib.check(L.fe_plan_set_stream(self._h, torch.cuda.current_stream(y.device).cuda_stream))
        _lib.check(L.fe_solve_residuals_device(
            self._h, y.data_ptr(), dt, ncols, ld, self.precision, float(tol), int(maxiter),
            its.ctypes.data_as(_lib._i64p), cvs.ctypes.data_as(_lib._u8p)))
        if vec:
            return y, int(its[0]), bool(cvs[0])
        return y, its, cvs.astype(bool)

    def solve_coefficients(self, y, tol: float | None = None, maxiter: int = 100_000):
        """solve_coefficients!(r, feM) (src/AbstractFixedEffectSolver.jl:147-160).

        Returns (full(normalize!(coefs)), iterations, converged)."""
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        a = np.asarray(y)
        if a.shape != (self.N,):
            raise ValueError("FixedEffects must have the same length as y")
        a = np.ascontiguousarray(a, dtype=np.float64 if a.dtype != np.float32 else np.float32)
        coefs = [np.zeros(fe.n, dtype=np.float64) for fe in self.fes]
        it = ctypes.c_int64(0)
        cv = ctypes.c_uint8(0)
        dt = FE_DTYPE_F64 if a.dtype == np.float64 else FE_DTYPE_F32
        _lib.check(_lib.load().fe_solve_coefficients(
            self._h, a.ctypes.data, dt, self.precision, float(tol), int(maxiter), _ptrs(coefs),
            ctypes.byref(it), ctypes.byref(cv)))
        # normalize! and full on the device (fe_normalize_coefficients,
        # fe_full_coefficients), in FP64
        L = _lib.load()
        _lib.check(L.fe_normalize_coefficients(self._h, _ptrs(coefs), 0))
        outs = [np.empty(self.N, dtype=np.float64) for _ in self.fes]
        _lib.check(L.fe_full_coefficients(self._h, _ptrs(coefs), 0, _ptrs(outs), 0))
        return [o.astype(a.dtype, copy=False) for o in outs], int(it.value), bool(cv.value)

    def normalize_coefficients(self, coefs):
        """normalize!(fecoefs, fes) on the device (src/FixedEffect.jl:106-135):
        per-level FP64 coefficient arrays, normalized in place and returned
        (arrays that cannot be written in place are normalized in a copy)."""
        coefs = [c if (isinstance(c, np.ndarray) and c.dtype == np.float64
                       and c.flags.c_contiguous and c.flags.writeable)
                 else np.array(c, dtype=np.float64) for c in coefs]
        _lib.check(_lib.load().fe_normalize_coefficients(self._h, _ptrs(coefs), 0))
        return coefs

    def full_coefficients(self, coefs):
        """full(fecoefs, fes) on the device (src/FixedEffect.jl:137-140)."""
        coefs = [np.ascontiguousarray(c, dtype=np.float64) for c in coefs]
        outs = [np.empty(self.N, dtype=np.float64) for _ in self.fes]
        _lib.check(_lib.load().fe_full_coefficients(self._h, _ptrs(coefs), 0, _ptrs(outs), 0))
        return outs

    # -- diagnostics ----------------------------------------------------------
    def set_option(self, option: int, value: float) -> None:
        _lib.check(_lib.load().fe_plan_set_option(self._h, option, float(value)))

    def last_solve_info(self, ncols: int):
        t2 = np.zeros(ncols)
        rounds = np.zeros(ncols, dtype=np.int32)
        raw = np.zeros(ncols, dtype=np.int64)
        _lib.check(_lib.load().fe_plan_last_solve_info(
            self._h, ncols, t2.ctypes.data_as(_lib._f64p), rounds.ctypes.data_as(_lib._i32p),
            raw.ctypes.data_as(_lib._i64p)))
        return {"test2": t2, "rounds": rounds, "lsmr_iters": raw}

    def integer_plan(self):
        N, K = self.N, len(self.fes)
        perm0 = np.zeros(N, dtype=np.int32)
        offs = [np.zeros(fe.n + 1, dtype=np.int64) for fe in self.fes]
        segs = [np.zeros(N, dtype=np.int32) for _ in range(K)]
        _lib.check(_lib.load().fe_plan_get_integer_plan(
            self._h, perm0.ctypes.data_as(_lib._i32p), _ptrs(offs), _ptrs(segs)))
        return perm0, offs, segs

    def scales(self):
        out = [np.zeros(fe.n) for fe in self.fes]
        _lib.check(_lib.load().fe_plan_get_scales(self._h, _ptrs(out)))
        return out

    def primary(self) -> int:
        v = ctypes.c_int32(0)
        _lib.check(_lib.load().fe_plan_primary(self._h, ctypes.byref(v)))
        return int(v.value)

    def kernel_stats(self):
        L = _lib.load()
        out = {}
        i = 0
        buf = ctypes.create_string_buffer(64)
        while True:
            n = ctypes.c_int64(0)
            ms = ctypes.c_double(0)
            by = ctypes.c_double(0)
            if L.fe_plan_kernel_stat(self._h, i, buf, 64, ctypes.byref(n), ctypes.byref(ms),
                                     ctypes.byref(by)) != 0:
                break
            t = np.zeros(max(n.value, 1), dtype=np.float32)
            m = ctypes.c_int64(0)
            _lib.check(L.fe_plan_kernel_times(self._h, i, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              t.size, ctypes.byref(m)))
            out[buf.value.decode()] = {"launches": n.value, "ms": ms.value, "bytes": by.value,
                                       "times_ms": t[:m.value].astype(np.float64)}
            i += 1
        return out

    def reset_stats(self):
        _lib.check(_lib.load().fe_plan_reset_stats(self._h))

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


def _is_cuda_tensor(y) -> bool:
    try:
        import torch
    except ImportError:
        return False
    return isinstance(y, torch.Tensor) and y.is_cuda


def AbstractFixedEffectSolver(fes, weights=None, method: str = "CUDA", T=np.float64, **kw):
    """AbstractFixedEffectSolver{T}(fes, w, Val{method}) (ext/CUDAExt.jl:99-110)."""
    return FixedEffectSolverB200(fes, weights, method=method, T=T, **kw)


def update_weights(feM: FixedEffectSolverB200, weights):
    """update_weights!(feM, w) (src/SolverCPU.jl:67-76, ext/CUDAExt.jl:112-121)."""
    return feM.update_weights(weights)


def solve_residuals(y, fes, weights=None, *, method: str = "CUDA",
                    double_precision: bool | None = None, tol: float | None = None,
                    maxiter: int | None = None, precision: str | None = None, device: int = 0):
    """solve_residuals!(y, fes, w; method, double_precision, tol, maxiter).

    With ``fes`` a list of FixedEffect this is the keyword front end of
    src/AbstractFixedEffectSolver.jl:37-45 (double_precision defaults to
    ``method == :cpu``, i.e. False here; tol to 1e-8 / 1e-6; maxiter 10000).
    With ``fes`` a solver object it is the solver-level method (:49-97).
    """
    if isinstance(fes, FixedEffectSolverB200):
        return fes.solve_residuals(y, tol=tol, maxiter=100_000 if maxiter is None else maxiter)
    fes = list(fes)
    n = (len(y) if not hasattr(y, "shape") else y.shape[0])
    if any(len(fe) != n for fe in fes):
        raise ValueError("FixedEffects must have the same length as y")
    if double_precision is None:
        double_precision = method == "cpu"
    if tol is None:
        tol = 1e-8 if double_precision else 1e-6
    feM = FixedEffectSolverB200(fes, weights, method=method,
                                T=np.float64 if double_precision else np.float32,
                                precision=precision, device=device)
    try:
        return feM.solve_residuals(y, tol=tol, maxiter=10000 if maxiter is None else maxiter)
    finally:
        feM.close()


def solve_coefficients(y, fes, weights=None, *, method: str = "CUDA",
                       double_precision: bool | None = None, tol: float | None = None,
                       maxiter: int | None = None, precision: str | None = None, device: int = 0):
    """solve_coefficients!(y, fes, w; ...) (src/AbstractFixedEffectSolver.jl:137-160)."""
    if isinstance(fes, FixedEffectSolverB200):
        return fes.solve_coefficients(y, tol=tol, maxiter=100_000 if maxiter is None else maxiter)
    fes = list(fes)
    if any(len(fe) != len(y) for fe in fes):
        raise ValueError("FixedEffects must have the same length as y")
    if double_precision is None:
        double_precision = method == "cpu"
    if tol is None:
        tol = 1e-8 if double_precision else 1e-6
    feM = FixedEffectSolverB200(fes, weights, method=method,
                                T=np.float64 if double_precision else np.float32,
                                precision=precision, device=device)
    try:
        return feM.solve_coefficients(y, tol=tol, maxiter=10000 if maxiter is None else maxiter)
    finally:
        feM.close()


# ---------------------------------------------------------------------------
# many independent problems in one batched solve
# ---------------------------------------------------------------------------
class BatchSolver:
    """Many independent fixed-effect problems solved as one batched LSMR.

    ``problems`` is a list of FE lists (problem p: its FixedEffects, 1 to 8 of
    them; a problem may have fewer FEs than others).  Slot k of every problem
    is its k-th FixedEffect.  Each problem keeps its own LSMR scalars and
    stopping test; all run in the same kernel launches.
    """

    def __init__(self, problems: Sequence[Sequence[FixedEffect]], weights=None,
                 T=np.float64, precision: str | None = None, device: int = 0):
        problems = [list(p) for p in problems]
        if not problems:
            raise ValueError("no problems")
        K = max(len(p) for p in problems)
        self.nprob = len(problems)
        self.n_obs = np.array([len(p[0]) for p in problems], dtype=np.int64)
        for p in problems:
            if any(len(fe) != len(p[0]) for fe in p):
                raise DimensionMismatch("all FixedEffects of a problem must have the same length")
        self.N = int(self.n_obs.sum())
        self.K = K
        self.precision = _precision_of(precision, T)
        self.T = np.dtype(T)
        self.offsets = np.concatenate([[0], np.cumsum(self.n_obs)])
        refs, nlev, inter = [], np.zeros((self.nprob, K), dtype=np.int64), []
        any_inter = [False] * K
        for k in range(K):
            parts, iparts = [], []
            for p, fes in enumerate(problems):
                n = int(self.n_obs[p])
                if k < len(fes):
                    parts.append(fes[k].refs)
                    nlev[p, k] = fes[k].n
                    if fes[k].interaction is not None:
                        any_inter[k] = True
                        iparts.append(fes[k].interaction)
                    else:
                        iparts.append(np.ones(n))
                else:
                    parts.append(np.zeros(n, dtype=np.int64))
                    iparts.append(np.ones(n))
            refs.append(np.ascontiguousarray(np.concatenate(parts), dtype=np.int64))
            inter.append(np.ascontiguousarray(np.concatenate(iparts)) if any_inter[k] else None)
        self._refs, self._nlev, self._inter = refs, np.ascontiguousarray(nlev), inter
        if weights is not None:
            w = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in weights]))
            if w.shape != (self.N,):
                raise DimensionMismatch("weights must match the problems' observations")
        else:
            w = None
        self._w = w
        h = ctypes.c_void_p()
        L = _lib.load()
        inter_pp = _ptrs(inter) if any(any_inter) else None
        _lib.check(L.fe_plan_create_batch(
            ctypes.byref(h), self.nprob, self.n_obs.ctypes.data_as(_lib._i64p), K, _ptrs(refs),
            self._nlev.ctypes.data_as(_lib._i64p), inter_pp,
            None if w is None else w.ctypes.data_as(_lib._f64p), device))
        self._h = h

    def solve_residuals(self, ys, tol: float | None = None, maxiter: int = 100_000):
        """Solves every problem's column; returns (list of r, iterations, converged)."""
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        if len(ys) != self.nprob:
            raise ValueError("one column per problem is required")
        dtype = np.float32 if all(np.asarray(y).dtype == np.float32 for y in ys) else np.float64
        Y = np.ascontiguousarray(np.concatenate([np.asarray(y, dtype=dtype).reshape(-1) for y in ys]))
        if Y.shape != (self.N,):
            raise ValueError("FixedEffects must have the same length as y")
        its = np.zeros(1, dtype=np.int64)
        cvs = np.zeros(1, dtype=np.uint8)
        L = _lib.load()
        dt = FE_DTYPE_F64 if dtype == np.float64 else FE_DTYPE_F32
        _lib.check(L.fe_solve_residuals(self._h, Y.ctypes.data, dt, 1, self.N, self.precision,
                                        float(tol), int(maxiter), its.ctypes.data_as(_lib._i64p),
                                        cvs.ctypes.data_as(_lib._u8p)))
        pit = np.zeros(self.nprob, dtype=np.int64)
        pcv = np.zeros(self.nprob, dtype=np.uint8)
        _lib.check(L.fe_plan_problem_results(self._h, pit.ctypes.data_as(_lib._i64p),
                                             pcv.ctypes.data_as(_lib._u8p)))
        out = [Y[self.offsets[p]:self.offsets[p + 1]].copy() for p in range(self.nprob)]
        return out, pit, pcv.astype(bool)

    def solve_residuals_device(self, y, tol: float | None = None, maxiter: int = 100_000):
        """Solves the problems' columns concatenated in one contiguous CUDA
        torch tensor (problem p at rows offsets[p]:offsets[p+1]), in place on
        the current torch stream; returns (y, iterations, converged) per
        problem."""
        import torch
        if tol is None:
            tol = math.sqrt(np.finfo(self.T).eps)
        if y.dtype not in (torch.float64, torch.float32) or y.dim() != 1 or not y.is_contiguous():
            raise ValueError("device y must be a contiguous float32/float64 vector")
        if y.shape[0] != self.N:
            raise ValueError("FixedEffects must have the same length as y")
        L = _lib.load()
        _lib.check(L.fe_plan_set_stream(self._h, torch.cuda.current_stream(y.device).cuda_stream))
        its = np.zeros(1, dtype=np.int64)
        cvs = np.zeros(1, dtype=np.uint8)
        dt = FE_DTYPE_F64 if y.dtype == torch.float64 else FE_DTYPE_F32
        _lib.check(L.fe_solve_residuals_device(self._h, y.data_ptr(), dt, 1, self.N,
                                               self.precision, float(tol), int(maxiter),
                                               its.ctypes.data_as(_lib._i64p),
                                               cvs.ctypes.data_as(_lib._u8p)))
        pit = np.zeros(self.nprob, dtype=np.int64)
        pcv = np.zeros(self.nprob, dtype=np.uint8)
        _lib.check(L.fe_plan_problem_results(self._h, pit.ctypes.data_as(_lib._i64p),
                                             pcv.ctypes.data_as(_lib._u8p)))
        return y, pit, pcv.astype(bool)

    def set_option(self, option: int, value: float) -> None:
        _lib.check(_lib.load().fe_plan_set_option(self._h, option, float(value)))

    def last_solve_info(self, ncols: int = 1):
        return FixedEffectSolverB200.last_solve_info(self, ncols)

    def kernel_stats(self):
        return FixedEffectSolverB200.kernel_stats(self)

    def reset_stats(self):
        _lib.check(_lib.load().fe_plan_reset_stats(self._h))

    def integer_plan(self):
        """(perm0, offsets[k], segperm[k]) over the concatenated problems;
        level k ids are numbered problem after problem."""
        nl = self._nlev.sum(axis=0)
        perm0 = np.zeros(self.N, dtype=np.int32)
        offs = [np.zeros(int(n) + 1, dtype=np.int64) for n in nl]
        segs = [np.zeros(self.N, dtype=np.int32) for _ in range(self.K)]
        _lib.check(_lib.load().fe_plan_get_integer_plan(
            self._h, perm0.ctypes.data_as(_lib._i32p), _ptrs(offs), _ptrs(segs)))
        return perm0, offs, segs

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


# ---------------------------------------------------------------------------
# normalize! / full (host side, as in the reference)
# ---------------------------------------------------------------------------
def components(fes: Sequence[FixedEffect]):
    """Connected components of the observation/level graph
    (src/FixedEffect.jl:68-98).  Returns, per FE, the component label of each
    level (-1 for levels without observations), and the component count."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    offs = np.concatenate([[0], np.cumsum([fe.n for fe in fes])])
    total = int(offs[-1])
    if len(fes) == 1:
        rows = cols = np.zeros(0, dtype=np.int64)
    else:
        base = fes[0].refs - 1 + offs[0]
        rows = np.concatenate([base for _ in fes[1:]])
        cols = np.concatenate([fe.refs - 1 + offs[k + 1] for k, fe in enumerate(fes[1:])])
    g = coo_matrix((np.ones(rows.shape[0], dtype=np.int8), (rows, cols)), shape=(total, total))
    ncomp, lab = connected_components(g, directed=False)
    used = np.zeros(total, dtype=bool)
    for k, fe in enumerate(fes):
        used[fe.refs - 1 + offs[k]] = True
    lab = np.where(used, lab, -1)
    return [lab[offs[k]:offs[k + 1]] for k in range(len(fes))], ncomp


def normalize(fecoefs: list, fes: Sequence[FixedEffect]) -> list:
    """normalize!: within each connected component, demean every
    non-interacted FE but the first and add the means to the first
    (src/FixedEffect.jl:106-135)."""
    idx = [k for k, fe in enumerate(fes) if fe.interaction is None]
    if len(idx) < 2:
        return fecoefs
    labels, ncomp = components([fes[k] for k in idx])
    m = np.zeros(ncomp)
    for jj in range(len(idx) - 1, 0, -1):
        k = idx[jj]
        lab = labels[jj]
        ok = lab >= 0
        s = np.bincount(lab[ok], weights=fecoefs[k][ok], minlength=ncomp)
        c = np.bincount(lab[ok], minlength=ncomp)
        mj = np.divide(s, c, out=np.zeros(ncomp), where=c > 0)
        fecoefs[k][ok] -= mj[lab[ok]].astype(fecoefs[k].dtype)
        m += mj
    k0 = idx[0]
    lab = labels[0]
    ok = lab >= 0
    fecoefs[k0][ok] += m[lab[ok]].astype(fecoefs[k0].dtype)
    return fecoefs


def full(fecoefs: list, fes: Sequence[FixedEffect]) -> list:
    """Per-observation coefficient vectors fecoef[refs] (src/FixedEffect.jl:137-140)."""
    return [c[fe.refs - 1] for c, fe in zip(fecoefs, fes)]
