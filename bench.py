"""Benchmark: batched FE solves/s of solve_residuals! at tol 1e-8 on B200s.

Workloads (seeded synthetic data with the shapes of the five solver
configurations; the reference publishes no dataset):

  worker_firm_year_10m_32col (default)  10M obs, worker uniform over 2M, firm
                                        Zipf(1.1) over 200k, year 20; 32 Float32
                                        columns per step
  two_fe_1m                             1M obs, 100k x 100 uniform; 1 Float64 column
  three_fe_interacted_10m               10M obs, 1M x 100 x 1000 (interacted),
                                        weights U(0.5, 1.5); 1 Float64 column
  uneven_256_problems                   256 problems, N log-uniform on [1e3, 1e6],
                                        2-3 FEs, weighted; one Float32 column each,
                                        all solved in one batched call
  large_zipf_100m_8col                  100M obs, 10M uniform x Zipf(1.3) over 10k,
                                        weighted; 8 Float32 columns per step

The reference's own benchmark problems (benchmark/run.jl:6-28), same shapes,
numpy draws:

  simple_10m                            10M obs, 100k x 100 uniform; 1 Float64 column
  hard_800k                             800k obs, worker 400k x firm 50k, each
                                        worker's firm near worker / 8; 1 Float64 column
  hard_800k_interacted                  800k obs, worker and worker x U(0, 1);
                                        1 Float64 column, maxiter 300 as there

One step = one batched solve of the step's columns (or problems) to the FP64
1e-8 stopping test in mixed precision (FP32 bulk, FP64 scalars, FP64
iterative refinement).

    python bench.py [--workload W] [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 and no torchrun environment, the script starts N ranks
itself through torch.distributed.run.  Each rank solves its own columns
(problems) over the same fixed effects: weak scaling, no collective on the
data path; the reported time is the max over ranks.

Reported: value = solves/s with inputs resident in HBM, timed with the
library's shipped defaults (CUDA-graph replay on), per-step CUDA events with
an L2 flush between steps; e2e = the same through the host-buffer C-ABI call,
from pinned and from pageable host memory (H2D and D2H inside the timed
call); the roofline of the dominant kernel from CUDA events of every launch
in a profiled pass of the same steps; the plain per-column FP64 form of this
library as a second baseline; the CPU oracle on a bounded sample.
`--impl reference` times the CPU restatement of the reference solver
(FixedEffects.jl's own CPU path cannot run here: Julia is not installed) on
the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "batched FE solves/s & HBM GB/s at 1e-8 vs FP64 oracle, mixed vs plain on B200"
WORKLOADS = {
    "worker_firm_year_10m_32col": 2,
    "two_fe_1m": 0,
    "three_fe_interacted_10m": 1,
    "uneven_256_problems": 3,
    "large_zipf_100m_8col": 4,
    # the reference's own benchmark problems (benchmark/run.jl:6-28)
    "simple_10m": 5,
    "hard_800k": 6,
    "hard_800k_interacted": 7,
}
DEFAULT_WORKLOAD = "worker_firm_year_10m_32col"
TOL = 1e-8
MAXITER = 10000
L2_FLUSH_BYTES = 256 << 20  # twice the 126 MB L2


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def spawn_ranks(args) -> int:
    """--gpus N > 1 without a torchrun environment: start the N ranks through
    torch.distributed.run (one process per GPU) and return its exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1",
           f"--master-port={_free_port()}", str(ROOT / "bench.py"), *sys.argv[1:]]
    log("starting ranks:", " ".join(cmd))
    return subprocess.call(cmd)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(workload: str, kernel: str):
    """Per-launch DRAM traffic of `kernel` on this workload from the committed
    ncu summary (profiles/traffic.json), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    e = d.get(workload, {}).get(kernel)
    return None if e is None else float(e["bytes_per_launch"])


def throughput_figures(obs_iters: float, lsmr_iters, stats: dict, prof_steps: int,
                       step_s: float, ranks: int) -> dict:
    """Whole-job observation-iterations/s (rows x LSMR iterations summed over
    the step's columns or problems, per second; rank 0's counts times the
    ranks) and the algorithmic bytes of every kernel of a step per second
    (kernel bytes from a profiled pass of `prof_steps` steps)."""
    iters = float(np.sum(np.asarray(lsmr_iters, dtype=np.float64)))
    alg = sum(float(v["bytes"]) for v in stats.values()) / max(prof_steps, 1)
    return {"observation_iterations_per_s": obs_iters * ranks / step_s,
            "lsmr_iterations_per_step": iters * ranks,
            "alg_bytes_per_step": alg * ranks,
            "alg_GBps": alg * ranks / step_s / 1e9}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 25 ms; entering
    waits (up to 3 s) for the first sample, so the samples cover the timed
    region that follows and not nvidia-smi's start-up."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "25"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        t0 = time.time()
        while time.time() - t0 < 3.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)
        self.skip = self._count()
        return self

    def _count(self):
        try:
            return len(Path(self.path).read_text().strip().splitlines())
        except Exception:
            return 0

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines()]
        except Exception:
            return out
        # the samples taken during the region (the one before it if none)
        skip = getattr(self, "skip", 0)
        rows = rows[skip:] if len(rows) > skip else rows[-1:]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(smax)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        return out


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def _synth():
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.synth as S
    return S


def _perturb(Y, rank):
    """Other ranks: the same fixed effects, their own columns."""
    if not rank:
        return Y
    rng = np.random.default_rng(1000 + rank)
    return np.asfortranarray(Y + rng.standard_normal(Y.shape).astype(Y.dtype))


class Columns:
    """One problem, `ncols` columns per step (configs 0, 1, 2, 4 and the
    reference's benchmark problems)."""

    batch = False

    def __init__(self, name, scale, rank, ncols):
        S = _synth()
        cfg = WORKLOADS[name]
        kw = {}
        if cfg in (2, 4):
            kw["ncols"] = ncols or (32 if cfg == 2 else 8)
        pb = S.make(cfg, scale=scale, **kw)
        Y = pb.Y if cfg in (2, 4) else pb.Y.astype(np.float64)  # Float32 or Float64 columns
        pb.Y = _perturb(np.asfortranarray(Y), rank)
        self.pb = pb
        self.name = name
        self.N = pb.N
        self.ncols = pb.Y.shape[1]
        self.solves = self.ncols
        self.nlev = [int(n) for n in pb.nlev]
        self.maxiter = int(pb.meta.get("maxiter") or MAXITER)

    def fes(self, fe):
        pb = self.pb
        return [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]

    def solver(self, fe, prec):
        T = np.float32 if self.pb.Y.dtype == np.float32 else np.float64
        return fe.AbstractFixedEffectSolver(self.fes(fe), self.pb.weights, "CUDA", T, precision=prec)

    def device_inputs(self, torch, dev):
        Y0 = torch.from_numpy(np.ascontiguousarray(self.pb.Y.T)).to(dev).t()
        Yw = torch.empty_like(Y0.t()).t()
        return Y0, Yw

    def solve_device(self, feM, Yw):
        _, its, cvs = feM.solve_residuals(Yw, tol=TOL, maxiter=self.maxiter)
        return its, cvs

    def host_buffers(self, torch, pinned):
        Y = self.pb.Y
        if pinned:
            buf = torch.empty((self.ncols, self.N), dtype=torch.float32 if Y.dtype == np.float32
                              else torch.float64, pin_memory=True)
            A = buf.numpy().T  # column-major view of pinned memory
        else:
            A = np.empty_like(Y, order="F")
            buf = None
        return buf, A

    def refresh_host(self, A):
        A[...] = self.pb.Y

    def solve_host(self, feM, A):
        feM.solve_residuals(A, tol=TOL, maxiter=self.maxiter)

    def io_bytes(self):
        return self.N * self.ncols * self.pb.Y.dtype.itemsize

    def obs_iters(self, its, info):
        """rows x LSMR iterations summed over the step's columns"""
        return float(self.N * np.sum(info["lsmr_iters"]))

    def result_col0(self, Yw):
        return Yw[:, 0].double().cpu().numpy()

    def oracle_sample(self, O, nthreads):
        """The CPU oracle on column 0 (bounded sample)."""
        pb = self.pb
        t = time.perf_counter()
        R, its, _ = O.solve_residuals_cols(pb.Y[:, :1].astype(np.float64), pb.refs, pb.nlev,
                                           pb.interaction, pb.weights, tol=TOL,
                                           maxiter=self.maxiter, nthreads=nthreads)
        dt = time.perf_counter() - t
        return {"solves": 1, "seconds": dt, "iterations": [int(x) for x in its],
                "sample": f"1 of {self.ncols} columns at full N={self.N} ({dt:.1f} s; serial "
                          f"reduce, expand on {nthreads} threads)"}, R[:, 0]

    def plain_inputs(self, torch, dev, ncols):
        Yp0 = torch.from_numpy(np.ascontiguousarray(self.pb.Y[:, :ncols].T.astype(np.float64)))
        return Yp0.to(dev).t()

    def config(self):
        return {"workload": self.name, "N": self.N, "fixed_effects": self.nlev,
                "weighted": self.pb.weights is not None,
                "interacted": [a is not None for a in self.pb.interaction],
                "columns_per_gpu": self.ncols, "input_dtype": str(self.pb.Y.dtype),
                "maxiter": self.maxiter}


class Problems:
    """256 independent problems, one column each, solved in one batched call
    (config 3)."""

    batch = True

    def __init__(self, name, scale, rank, ncols):
        S = _synth()
        self.probs = S.make(3, scale=scale)
        for p in self.probs:
            p.Y = _perturb(p.Y, rank)
        self.name = name
        self.N = int(sum(p.N for p in self.probs))
        self.ncols = 1
        self.solves = len(self.probs)
        self.offsets = np.concatenate([[0], np.cumsum([p.N for p in self.probs])])
        self.Ycat = np.concatenate([p.Y[:, 0] for p in self.probs]).astype(np.float32)

    def fes_list(self, fe):
        return [[fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(p.refs, p.nlev, p.interaction)]
                for p in self.probs]

    def solver(self, fe, prec):
        return fe.BatchSolver(self.fes_list(fe), [p.weights for p in self.probs], T=np.float32,
                              precision=prec)

    def device_inputs(self, torch, dev):
        Y0 = torch.from_numpy(self.Ycat).to(dev)
        return Y0, torch.empty_like(Y0)

    def solve_device(self, bs, Yw):
        _, its, cvs = bs.solve_residuals_device(Yw, tol=TOL, maxiter=MAXITER)
        return its, cvs

    def host_buffers(self, torch, pinned):
        if pinned:
            buf = torch.empty(self.N, dtype=torch.float32, pin_memory=True)
            return buf, buf.numpy()
        return None, np.empty(self.N, dtype=np.float32)

    def refresh_host(self, A):
        A[...] = self.Ycat

    def solve_host(self, bs, A):
        # the batched plan's host-buffer C-ABI call on the concatenated column
        fe = sys.modules["fe_b200"]
        L = fe._lib.load()
        its = np.zeros(1, dtype=np.int64)
        cvs = np.zeros(1, dtype=np.uint8)
        fe._lib.check(L.fe_solve_residuals(bs._h, A.ctypes.data, fe._lib.FE_DTYPE_F32, 1, self.N,
                                           bs.precision, TOL, MAXITER,
                                           its.ctypes.data_as(fe._lib._i64p),
                                           cvs.ctypes.data_as(fe._lib._u8p)))

    def io_bytes(self):
        return self.N * 4

    def obs_iters(self, its, info):
        """sum over problems of rows x LSMR iterations (its = iterations + 1)"""
        n = np.diff(self.offsets)
        return float(np.sum(n * (np.asarray(its, dtype=np.float64) - 1)))

    def result_col0(self, Yw):
        return Yw.double().cpu().numpy()

    def oracle_sample(self, O, nthreads):
        """The CPU oracle on every problem (the C oracle releases the GIL, so
        the problems run on all host threads)."""

        def one(p):
            r, it, _ = O.solve_residuals(p.Y[:, 0].astype(np.float64), p.refs, p.nlev,
                                         p.interaction, p.weights, tol=TOL, maxiter=MAXITER,
                                         nthreads=1)
            return r, int(it)

        t = time.perf_counter()
        with ThreadPoolExecutor(nthreads) as ex:
            outs = list(ex.map(one, self.probs))
        dt = time.perf_counter() - t
        return {"solves": len(self.probs), "seconds": dt, "iterations": [o[1] for o in outs],
                "sample": f"all {len(self.probs)} problems, N total {self.N} ({dt:.1f} s; one "
                          f"problem per thread on {nthreads} threads)"}, \
            np.concatenate([o[0] for o in outs])

    def plain_inputs(self, torch, dev, ncols):
        return torch.from_numpy(self.Ycat.astype(np.float64)).to(dev)

    def config(self):
        return {"workload": self.name, "problems": len(self.probs), "N_total": self.N,
                "columns_per_gpu": 1, "input_dtype": "float32", "weighted": True}


def plan_options(args):
    """--option FE_OPT_NAME=value pairs (plan options for experiments)."""
    out = []
    for o in args.option:
        name, _, val = o.partition("=")
        if not name.startswith("FE_OPT_"):
            raise SystemExit(f"--option wants FE_OPT_NAME=value, got {o!r}")
        out.append((name, float(val)))
    return out


def make_workload(name, scale, rank, ncols):
    cls = Problems if WORKLOADS[name] == 3 else Columns
    return cls(name, scale, rank, ncols)


def rel_err_vs(result, ref, wl):
    if wl.batch:
        # max over problems of the per-problem relative error
        errs = [np.linalg.norm(result[a:b] - ref[a:b]) / np.linalg.norm(ref[a:b])
                for a, b in zip(wl.offsets[:-1], wl.offsets[1:])]
        return float(max(errs))
    return float(np.linalg.norm(result - ref) / np.linalg.norm(ref))


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    wl = make_workload(args.workload, args.scale, 0, args.ncols)
    from oracle import oracle as O
    O.build()
    nthreads = O.host_threads()
    for _ in range(args.warmup):
        wl.oracle_sample(O, nthreads)
    t = time.perf_counter()
    solves = 0
    for _ in range(args.steps):
        info, _ = wl.oracle_sample(O, nthreads)
        solves += info["solves"]
    dt = time.perf_counter() - t
    value = solves / dt
    cfg = wl.config()
    cfg["solves_per_step"] = info["solves"]
    cfg["tol"] = TOL
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": max(ws, args.gpus), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "port",
                         "sample": info["sample"].split(" (")[0] + " per step"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "FixedEffects.jl (Julia) is not installed here; its CPU solver path is timed "
                "through the C restatement in oracle/ (serial reduce as src/SolverCPU.jl:20-27, "
                "threaded expand as :29-34)",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    import __graft_entry__ as g
    fe = g.load_package()

    t0 = time.perf_counter()
    wl = make_workload(args.workload, args.scale, rank, args.ncols)
    log(f"[rank {rank}] workload {wl.name} generated in {time.perf_counter() - t0:.1f} s; N={wl.N}")
    t0 = time.perf_counter()
    feM = wl.solver(fe, "mixed")
    torch.cuda.synchronize()
    plan_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    if args.no_absorb:  # the full-LSMR loop over all fixed effects
        feM.set_option(fe._lib.FE_OPT_ABSORB, 0)
    for name, val in plan_options(args):
        feM.set_option(getattr(fe._lib, name), val)

    # inputs resident in HBM: a pristine copy, refreshed into the work buffer
    # at the start of every step (the solve is in place)
    Y0, Yw = wl.device_inputs(torch, dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        Yw.copy_(Y0)
        return wl.solve_device(feM, Yw)

    for _ in range(args.warmup):
        its, cvs = step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # timed region: the shipped defaults (graph replay on); one event pair per
    # step, an L2 flush between steps outside the pairs
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        for a, b in evs:
            flush.fill_(1.0)
            a.record(stream)
            its, cvs = step()
            b.record(stream)
        torch.cuda.synchronize()
    ms = float(sum(a.elapsed_time(b) for a, b in evs))
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    conv_all = bool(np.all(cvs))
    its_list = [int(x) for x in np.atleast_1d(its)]
    info = feM.last_solve_info(wl.ncols)
    result_dev = wl.result_col0(Yw)

    # profiled pass of the same steps: a CUDA-event pair around every launch
    # (graph replay off), for the per-kernel times and the roofline
    prof_steps = max(1, min(args.steps, args.prof_steps))
    feM.reset_stats()
    feM.set_option(fe._lib.FE_OPT_PROFILE, 1)
    prof_ms = 0.0
    for _ in range(prof_steps):
        flush.fill_(1.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        torch.cuda.synchronize()
        prof_ms += a.elapsed_time(b)
    feM.set_option(fe._lib.FE_OPT_PROFILE, 0)
    stats = feM.kernel_stats()

    # e2e through the host-buffer C ABI (H2D + solve + D2H inside the call),
    # from pinned and from pageable host memory
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    feM_h = wl.solver(fe, "mixed")
    if args.no_absorb:
        feM_h.set_option(fe._lib.FE_OPT_ABSORB, 0)
    for name, val in plan_options(args):
        feM_h.set_option(getattr(fe._lib, name), val)
    e2e, e2e_calls = {}, {}
    for kind in ("pinned", "pageable"):
        buf, A = wl.host_buffers(torch, kind == "pinned")
        wl.refresh_host(A)
        wl.solve_host(feM_h, A)  # warm-up
        if dist:
            dist.barrier()
        calls = []
        for _ in range(e2e_steps):
            wl.refresh_host(A)  # fresh inputs (outside the timed call)
            torch.cuda.synchronize()
            t = time.perf_counter()
            wl.solve_host(feM_h, A)
            calls.append((time.perf_counter() - t) * 1e3)
        e2e_calls[kind] = [round(x, 3) for x in calls]
        tot = sum(calls) / e2e_steps
        if dist:
            t = torch.tensor([tot], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        e2e[kind] = tot
        del buf, A
    feM_h.close()

    # second baseline: the plain per-column FP64 form of this library
    plain = None
    if not args.no_plain and rank == 0:
        npl = min(args.plain_cols, wl.ncols)
        feP = wl.solver(fe, "fp64")
        if not wl.batch:
            feP.set_option(fe._lib.FE_OPT_TILE, 1)
        Yp0 = wl.plain_inputs(torch, dev, npl)
        Yp = Yp0.clone()
        wl.solve_device(feP, Yp)  # warm-up
        Yp.copy_(Yp0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pits, pcv = wl.solve_device(feP, Yp)
        b.record(stream)
        torch.cuda.synchronize()
        pms = a.elapsed_time(b)
        nsolves = wl.solves if wl.batch else npl
        plain = {"value": nsolves / (pms * 1e-3), "unit": "solves/s",
                 "solves_timed": nsolves, "form": "batched FP64 plan" if wl.batch
                 else "one FP64 column per LSMR tile",
                 "iterations_max": int(np.max(pits)), "converged": bool(np.all(pcv))}
        plain_result = wl.result_col0(Yp)
        feP.close()

    line = None
    if rank == 0:
        total = wl.solves * ws
        step_s = ms * 1e-3 / args.steps
        value = total / step_s
        kern = {k: v for k, v in stats.items() if v["bytes"] > 0}
        top = max(kern.items(), key=lambda kv: kv[1]["ms"])
        tname, tv = top

        def working(v):
            # launches that did the work: a launch that found every column
            # stopped (the tail of a replayed chunk) returns in microseconds
            t = np.asarray(v["times_ms"])
            return t[t >= 0.2 * t.max()] if t.size else t

        def gbps(v):
            w = working(v)
            return v["bytes"] / v["launches"] / (w.mean() * 1e-3) / 1e9 if v["bytes"] and w.size else None

        tw = working(tv)
        avg_s = float(tw.mean()) * 1e-3
        alg = tv["bytes"] / tv["launches"]
        achieved = alg / avg_s / 1e9
        peak, peak_kind = measured_peak()
        total_ms = sum(v["ms"] for v in stats.values())
        per_kernel = {k: {"launches": v["launches"], "working_launches": int(working(v).size),
                          "ms": round(v["ms"], 3), "share": round(v["ms"] / total_ms, 4),
                          "us_per_working_launch": round(float(working(v).mean()) * 1e3, 1)
                          if working(v).size else None,
                          "GBps": round(gbps(v), 1) if gbps(v) else None,
                          "frac_of_peak": round(gbps(v) / peak, 3) if gbps(v) else None}
                      for k, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])}
        launches_per_step = sum(v["launches"] for v in stats.values()) / prof_steps
        cfg = wl.config()
        cfg.update({"tol": TOL, "precision": "mixed", "solves_per_step_per_gpu": wl.solves,
                    "parallelism": f"columns (problems) sharded over {ws} GPU(s), no collective",
                    "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write outside "
                          "the per-step CUDA-event pairs)",
                    "timing": "shipped defaults (CUDA-graph replay of the LSMR loop)"})
        io = wl.io_bytes()
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic", "config": cfg,
            # the solver constructor: refs upload, validation and integer plan
            # (radix sorts) on the device, weights, preconditioner
            "plan_build": {"device_s": round(plan_s, 3)},
            "e2e": {"value": total / (e2e["pinned"] * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": io, "d2h_bytes_per_step": io,
                    "ms_per_step": e2e["pinned"], "host_memory": "pinned",
                    "pageable": {"value": total / (e2e["pageable"] * 1e-3),
                                 "ms_per_step": e2e["pageable"],
                                 "ratio_to_pinned_time": e2e["pageable"] / e2e["pinned"]},
                    "ms_per_call": e2e_calls},
            "roofline": {"bound": "hbm", "kernel": tname, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "frac_of_nominal_7700": achieved / 7700.0,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "traffic": committed_traffic(wl.name, tname),
                         "alg_bytes_per_launch": alg,
                         "launch_time": "mean CUDA-event time of the working launches "
                                        f"({tw.size} of {tv['launches']}) in a profiled pass of "
                                        f"{prof_steps} step(s) run right after the timed region"},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "profiled_pass": {"steps": prof_steps, "ms_per_step": prof_ms / prof_steps,
                              "kernel_ms_per_step": total_ms / prof_steps},
            "kernels": per_kernel,
            "throughput": throughput_figures(wl.obs_iters(its, info), info["lsmr_iters"] if not
                                             wl.batch else np.asarray(its) - 1, stats, prof_steps,
                                             step_s, ws),
            "iterations": its_list if len(its_list) <= 32 else
            {"max": int(max(its_list)), "mean": float(np.mean(its_list))},
            "converged": conv_all,
            "refinement_rounds": [int(x) for x in info["rounds"]],
            "fp64_test2": [float(x) for x in info["test2"]],
        }
        if wl.batch:
            line["iterations_note"] = "per problem"
        if plain is not None:
            line["plain_fp64_per_column"] = plain
            line["speedup_vs_plain_fp64"] = value / plain["value"]
        if not args.no_cpu_baseline:
            from oracle import oracle as O
            O.build()
            nthreads = O.host_threads()
            cb, ro = wl.oracle_sample(O, nthreads)
            line["cpu_baseline"] = {"value": cb["solves"] / cb["seconds"], "unit": "solves/s",
                                    "cores": nthreads, "kind": "port", "sample": cb["sample"]}
            line["max_rel_err_vs_oracle"] = {"mixed": rel_err_vs(result_dev, ro, wl),
                                             "compared": "all problems" if wl.batch else "column 0"}
            if plain is not None:
                line["max_rel_err_vs_oracle"]["plain_fp64"] = rel_err_vs(plain_result, ro, wl)
            it_o = cb["iterations"]
            line["oracle_iterations"] = it_o if len(it_o) <= 32 else \
                {"max": int(max(it_o)), "mean": float(np.mean(it_o))}
            line["oracle_iterations_note"] = (
                "FP64 LSMR of the reference (iterations = mvps + 1); the mixed solve's counts "
                "above are its refined inner LSMR iterations + 1 on the absorbed or full problem "
                "and have no oracle counterpart")
        line["clocks"] = clk.summary()
        print(json.dumps(line), flush=True)
    feM.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_sweep(args):
    """Times every expand x segsum kernel variant on the workload (mixed
    precision, 32-column tile) and for the per-column FP64 form; prints a
    markdown table.  The autotuner makes the same choice at run time."""
    import torch
    torch.cuda.set_device(0)
    import __graft_entry__ as g
    fe = g.load_package()
    wl = make_workload(DEFAULT_WORKLOAD, args.scale, 0, args.ncols)
    pb = wl.pb
    fes = wl.fes(fe)
    Y0 = torch.from_numpy(np.ascontiguousarray(pb.Y.T)).cuda().t()
    print("| mode | expand | segsum | ms per solve | solves/s |\n|---|---:|---:|---:|---:|")
    for prec, tile, ncols in (("mixed", 0, pb.Y.shape[1]), ("fp64", 1, min(4, pb.Y.shape[1]))):
        feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64, precision=prec)
        feM.set_option(fe._lib.FE_OPT_TILE, tile)
        combos = [(e, sv) for e in range(6) for sv in range(6)] + [(-1, -1)]  # last: tuned
        for e, sv in combos:
            feM.set_option(fe._lib.FE_OPT_EXPAND_VARIANT, e)
            feM.set_option(fe._lib.FE_OPT_SEGSUM_VARIANT, sv)
            best = 1e30
            for _ in range(3):
                Y = Y0[:, :ncols].clone().t().contiguous().t()
                if prec == "fp64":
                    Y = Y.double().t().contiguous().t()
                torch.cuda.synchronize()
                t = time.perf_counter()
                feM.solve_residuals(Y, tol=TOL, maxiter=MAXITER)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t)
            mode = f"{prec} C={'32' if tile == 0 else '1'}"
            es, ss = ("tuned", "tuned") if e < 0 else (e, sv)
            print(f"| {mode} | {es} | {ss} | {best * 1e3:.1f} | {ncols / best:.1f} |", flush=True)
        feM.close()
    return 0


def run_plan_build(args):
    """Times plan construction on the device against its host counterparts,
    on the 10M worker/firm/year workload and the 100M two-FE workload (10M
    uniform levels, 10K Zipf(1.3) levels):
      * the solver constructor (refs upload, validation, radix-sort integer
        plan, weights, preconditioner) vs the oracle's host integer plan
        (stable counting sorts, one core);
      * key grouping of raw int64 keys (level ids scattered over the int64
        range, so the radix-sort path runs) vs numpy's grouping on the host.
    Prints one JSON line; the device grouping must equal the host one."""
    import torch
    torch.cuda.set_device(0)
    import __graft_entry__ as g
    fe = g.load_package()
    import fe_b200.synth as S
    from oracle import oracle as O
    O.build()

    def scatter_keys(r):
        # an injective map of level ids onto sparse int64 keys
        return (r.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)).view(np.int64)

    # load the build kernels once (lazy module loading) on a small case
    pb = S.config2(scale=0.001, ncols=0)
    fe.AbstractFixedEffectSolver([fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)],
                                 None, "CUDA", np.float32).close()
    fe.group_keys(scatter_keys(pb.refs[0]), device=0)
    out = {"metric": "plan construction", "unit": "s", "higher_is_better": False,
           "data": "synthetic", "workloads": {}}
    scale = args.scale
    for name, mk in (("worker_firm_year_10m", lambda: S.config2(scale=scale, ncols=0)),
                     ("two_fe_100m", lambda: S.config4(scale=scale, ncols=0))):
        pb = mk()
        fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
        torch.cuda.synchronize()
        t = time.perf_counter()
        feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float32, precision="mixed")
        torch.cuda.synchronize()
        dev_plan = time.perf_counter() - t
        t = time.perf_counter()
        O.integer_plan(pb.refs, pb.nlev, feM.primary())
        host_plan = time.perf_counter() - t
        feM.close()
        # a second construction of the same plan (allocator and page state warm)
        torch.cuda.synchronize()
        t = time.perf_counter()
        fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float32, precision="mixed").close()
        torch.cuda.synchronize()
        dev_plan2 = time.perf_counter() - t
        dev_group = host_group = 0.0
        equal = True
        for r in pb.refs:
            raw = scatter_keys(r)
            t = time.perf_counter()
            dr, dn = fe.group_keys(raw, device=0)
            dev_group += time.perf_counter() - t
            t = time.perf_counter()
            h = fe.FixedEffect(raw)
            host_group += time.perf_counter() - t
            equal = equal and dn == h.n and bool(np.array_equal(dr, h.refs))
        out["workloads"][name] = {
            "N": pb.N, "fixed_effects": pb.nlev,
            "device_plan_s": round(dev_plan, 3), "device_plan_repeat_s": round(dev_plan2, 3),
            "oracle_integer_plan_s": round(host_plan, 3),
            "device_group_keys_s": round(dev_group, 3), "numpy_group_keys_s": round(host_group, 3),
            "group_keys_equal_host": equal}
        log(name, out["workloads"][name])
    print(json.dumps(out), flush=True)
    return 0


def run_host_columns(args):
    """Times one host-buffer solve of args.host_columns columns of the 10M
    workload (several 32-column tiles) from pageable and from pinned host
    memory (tile-pipelined transfers), next to the device-resident solve.
    Wall clock per call, best of two after a warm-up; prints one JSON line."""
    import torch
    torch.cuda.set_device(0)
    import __graft_entry__ as g
    fe = g.load_package()
    import fe_b200.synth as S
    ncols = args.host_columns
    pb = S.config2(scale=args.scale, ncols=ncols)
    fes = [fe.FixedEffect.from_refs(r, n) for r, n in zip(pb.refs, pb.nlev)]
    feM = fe.AbstractFixedEffectSolver(fes, None, "CUDA", np.float32, precision="mixed")
    Y = np.asfortranarray(pb.Y)
    N = Y.shape[0]
    P = torch.empty((ncols, N), dtype=torch.float32, pin_memory=True).numpy().T
    D = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t()

    def timed(kind):
        if kind == "device":
            A = D.clone().t().contiguous().t()
        elif kind == "pinned":
            P[...] = Y
            A = P
        else:
            A = Y.copy(order="F")
        torch.cuda.synchronize()
        t = time.perf_counter()
        feM.solve_residuals(A, tol=TOL, maxiter=MAXITER)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    timed("pageable")  # warm-up: tuning, graphs, staging
    out = {"metric": "host-buffer solve time", "unit": "s", "higher_is_better": False,
           "data": "synthetic", "config": {"workload": "worker_firm_year_10m", "N": N,
                                           "columns": ncols, "precision": "mixed", "tol": TOL}}
    for kind in ("device", "pinned", "pageable"):
        out[kind + "_s"] = round(min(timed(kind) for _ in range(2)), 4)
    feM.close()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--scale", type=float, default=1.0, help="shrink N and levels (debug only)")
    ap.add_argument("--ncols", type=int, default=0, help="columns per step (0: the workload's)")
    ap.add_argument("--plain-cols", type=int, default=4)
    ap.add_argument("--prof-steps", type=int, default=2,
                    help="steps of the profiled pass (per-launch CUDA events)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--option", action="append", default=[],
                    help="plan option FE_OPT_NAME=value for the timed solver (repeatable)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-variants", action="store_true",
                    help="time every expand/segsum kernel variant and print a table")
    ap.add_argument("--no-absorb", action="store_true",
                    help="mixed solves run the full LSMR over all fixed effects (FE_OPT_ABSORB 0)")
    ap.add_argument("--plan-build", action="store_true",
                    help="time plan construction and key grouping, device vs host")
    ap.add_argument("--host-columns", type=int, default=0,
                    help="time a host-buffer solve of this many columns: pageable, pinned, device")
    args = ap.parse_args()
    if args.host_columns:
        return run_host_columns(args)
    if args.plan_build:
        return run_plan_build(args)
    if args.sweep_variants:
        return run_sweep(args)
    ws = int(os.environ.get("WORLD_SIZE", "0") or 0)
    if args.impl == "reference":
        return run_reference(args)
    if args.gpus > 1 and ws == 0:
        return spawn_ranks(args)
    if ws and ws != args.gpus:
        log(f"--gpus {args.gpus} does not match WORLD_SIZE {ws}")
        return 2
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
