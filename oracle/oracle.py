"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is a C, FP64 restatement of FixedEffects.jl v3.1.0's CPU solver
(src/SolverCPU.jl, src/utils/lsmr.jl, src/AbstractFixedEffectSolver.jl,
src/FixedEffect.jl).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use it, always as the checker; the product path never does.

Inputs follow the reference: ``refs`` are 1-based level ids (one int64 array
per fixed effect), ``interaction`` entries may be None (UnitWeights), and
``weights`` may be None (UnitWeights).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libfe_oracle.so"
_lib = None

TRACE_WIDTH = 10
TRACE_FIELDS = ("alpha", "beta", "normr", "normAr", "normA", "condA", "normx",
                "test1", "test2", "istop")

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)
_vpp = ctypes.POINTER(ctypes.c_void_p)


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc only)."""
    src = _HERE / "fe_oracle.c"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(_LIB_PATH))
        L.ora_solve_residuals.restype = ctypes.c_int
        L.ora_solve_residuals.argtypes = [
            ctypes.c_int64, ctypes.c_int32, _vpp, _i64p, _vpp, _f64p, _f64p,
            ctypes.c_double, ctypes.c_int64, ctypes.c_int32, _i64p, _i32p,
            _f64p, ctypes.c_int64]
        L.ora_solve_residuals_cols.restype = ctypes.c_int
        L.ora_solve_residuals_cols.argtypes = [
            ctypes.c_int64, ctypes.c_int32, _vpp, _i64p, _vpp, _f64p, _f64p,
            ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.c_int32,
            _i64p, _i32p]
        L.ora_solve_coefficients.restype = ctypes.c_int
        L.ora_solve_coefficients.argtypes = [
            ctypes.c_int64, ctypes.c_int32, _vpp, _i64p, _vpp, _f64p, _f64p,
            ctypes.c_double, ctypes.c_int64, ctypes.c_int32, _vpp, _vpp, _i64p,
            _i32p]
        L.ora_scale.restype = None
        L.ora_scale.argtypes = [_f64p, ctypes.c_int64, _i64p, _f64p, _f64p,
                                ctypes.c_int64]
        L.ora_integer_plan.restype = ctypes.c_int
        L.ora_integer_plan.argtypes = [ctypes.c_int64, ctypes.c_int32, _vpp,
                                       _i64p, ctypes.c_int32, _i32p, _vpp, _vpp]
        L.ora_components.restype = ctypes.c_int64
        L.ora_components.argtypes = [ctypes.c_int64, ctypes.c_int32, _vpp, _i64p,
                                     _i64p]
        _lib = L
    return _lib


def _ptr(a, t=_f64p):
    return None if a is None else a.ctypes.data_as(t)


class _Inputs:
    """Holds contiguous copies of the inputs so the pointers stay alive."""

    def __init__(self, refs, nlev, interaction=None, weights=None):
        self.refs = [np.ascontiguousarray(r, dtype=np.int64) for r in refs]
        self.K = len(self.refs)
        self.N = int(self.refs[0].shape[0]) if self.K else 0
        if nlev is None:
            nlev = [int(r.max()) if r.size else 0 for r in self.refs]
        self.nlev = np.ascontiguousarray(nlev, dtype=np.int64)
        inter = interaction if interaction is not None else [None] * self.K
        self.inter = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                      for a in inter]
        self.w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        self.refs_pp = (ctypes.c_void_p * self.K)(*[r.ctypes.data for r in self.refs])
        self.inter_pp = (ctypes.c_void_p * self.K)(
            *[0 if a is None else a.ctypes.data for a in self.inter])
        self.has_inter = any(a is not None for a in self.inter)

    def args(self):
        return (self.N, self.K, self.refs_pp, _ptr(self.nlev, _i64p),
                self.inter_pp if self.has_inter else None, _ptr(self.w))


def solve_residuals(y, refs, nlev=None, interaction=None, weights=None,
                    tol=1e-8, maxiter=10000, nthreads=0, trace_cap=0):
    """Oracle solve_residuals!: returns (r, iterations, converged[, trace])."""
    inp = _Inputs(refs, nlev, interaction, weights)
    r = np.array(y, dtype=np.float64, copy=True)
    it = ctypes.c_int64(0)
    cv = ctypes.c_int32(0)
    trace = np.zeros((max(trace_cap, 1), TRACE_WIDTH)) if trace_cap else None
    st = lib().ora_solve_residuals(*inp.args(), _ptr(r), tol, maxiter, nthreads,
                                   ctypes.byref(it), ctypes.byref(cv),
                                   _ptr(trace), trace_cap)
    if st != 0:
        raise ValueError(f"oracle solve_residuals failed with status {st}")
    if trace_cap:
        n = min(max(it.value - 1, 0), trace_cap)
        return r, it.value, bool(cv.value), trace[:n]
    return r, it.value, bool(cv.value)


def solve_residuals_cols(Y, refs, nlev=None, interaction=None, weights=None,
                         tol=1e-8, maxiter=10000, nthreads=0):
    """Oracle collection method: Y is (N, ncols); returns (R, iters, convs)."""
    inp = _Inputs(refs, nlev, interaction, weights)
    R = np.array(Y, dtype=np.float64, order="F", copy=True)
    if R.ndim == 1:
        R = R[:, None]
    nc = R.shape[1]
    its = np.zeros(nc, dtype=np.int64)
    cvs = np.zeros(nc, dtype=np.int32)
    st = lib().ora_solve_residuals_cols(*inp.args(), _ptr(R), nc, tol, maxiter,
                                        nthreads, _ptr(its, _i64p),
                                        _ptr(cvs, _i32p))
    if st != 0:
        raise ValueError(f"oracle solve_residuals_cols failed with status {st}")
    return R, its, cvs.astype(bool)


def solve_coefficients(y, refs, nlev=None, interaction=None, weights=None,
                       tol=1e-8, maxiter=10000, nthreads=0):
    """Oracle solve_coefficients!: returns (coef_levels, coef_full, iters, conv)."""
    inp = _Inputs(refs, nlev, interaction, weights)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    levels = [np.zeros(int(n)) for n in inp.nlev]
    full = [np.zeros(inp.N) for _ in range(inp.K)]
    lv = (ctypes.c_void_p * inp.K)(*[a.ctypes.data for a in levels])
    fv = (ctypes.c_void_p * inp.K)(*[a.ctypes.data for a in full])
    it = ctypes.c_int64(0)
    cv = ctypes.c_int32(0)
    st = lib().ora_solve_coefficients(*inp.args(), _ptr(yy), tol, maxiter,
                                      nthreads, lv, fv, ctypes.byref(it),
                                      ctypes.byref(cv))
    if st != 0:
        raise ValueError(f"oracle solve_coefficients failed with status {st}")
    return levels, full, it.value, bool(cv.value)


def scale(refs_k, nlev_k, interaction_k=None, weights=None):
    """Oracle scale! for one fixed effect (src/SolverCPU.jl:78-89)."""
    r = np.ascontiguousarray(refs_k, dtype=np.int64)
    a = None if interaction_k is None else np.ascontiguousarray(interaction_k, dtype=np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros(int(nlev_k))
    lib().ora_scale(_ptr(out), int(nlev_k), _ptr(r, _i64p), _ptr(a), _ptr(w), r.shape[0])
    return out


def integer_plan(refs, nlev, primary):
    """Oracle integer plan: (perm0, offsets[k], segperm[k]) as int arrays."""
    inp = _Inputs(refs, nlev)
    N, K = inp.N, inp.K
    perm0 = np.zeros(N, dtype=np.int32)
    offs = [np.zeros(int(n) + 1, dtype=np.int64) for n in inp.nlev]
    segs = [np.zeros(N, dtype=np.int32) for _ in range(K)]
    op = (ctypes.c_void_p * K)(*[a.ctypes.data for a in offs])
    sp = (ctypes.c_void_p * K)(*[a.ctypes.data for a in segs])
    st = lib().ora_integer_plan(N, K, inp.refs_pp, _ptr(inp.nlev, _i64p), primary,
                                _ptr(perm0, _i32p), op, sp)
    if st != 0:
        raise ValueError(f"oracle integer_plan failed with status {st}")
    return perm0, offs, segs


def components(refs, nlev=None):
    """Oracle connected components: (ncomp, comp_of_obs)."""
    inp = _Inputs(refs, nlev)
    comp = np.zeros(inp.N, dtype=np.int64)
    nc = lib().ora_components(inp.N, inp.K, inp.refs_pp, _ptr(inp.nlev, _i64p),
                              _ptr(comp, _i64p))
    if nc < 0:
        raise ValueError("oracle components failed")
    return int(nc), comp


def host_threads() -> int:
    return os.cpu_count() or 1
