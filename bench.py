"""Benchmark: batched FE solves/s of solve_residuals! at tol 1e-8 on one B200.

Workload (default): 10M observations, three fixed effects (worker uniform over
2M, firm Zipf(1.1) over 200k, year 20), 32 Float32 columns, unit weights,
seeded synthetic data (the reference publishes no dataset).  One step = one
batched solve of all 32 columns to the FP64 1e-8 stopping test, mixed
precision (FP32 bulk, FP64 scalars, FP64 iterative refinement).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank solves its own 32 columns of the same fixed effects
(columns are independent: weak scaling, no collective on the data path); the
reported time is the max over ranks.

Reported: value = solves/s with inputs resident in HBM; e2e = the same through
the host-buffer C-ABI call (pinned host memory, H2D and D2H inside the timed
region); roofline of the dominant kernel from CUDA events inside the timed
region; the plain per-column FP64 form of this library as a second baseline;
the CPU oracle on a bounded sample.  `--impl reference` times the CPU
restatement of the reference solver (FixedEffects.jl's own CPU path cannot
run here: Julia is not installed) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD_NAME = "worker_firm_year_10m_32col"
METRIC = "batched FE solves/s & HBM GB/s at 1e-8 vs FP64 oracle, mixed vs plain on B200"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_workload(scale: float, rank: int, ncols: int):
    import __graft_entry__ as g
    g.load_package()
    import fe_b200.synth as S
    pb = S.config2(scale=scale, ncols=ncols, seed=2)
    if rank:
        # other ranks: the same fixed effects, their own columns
        rng = np.random.default_rng(1000 + rank)
        pb.Y = np.asfortranarray(
            pb.Y + rng.standard_normal(pb.Y.shape, dtype=np.float32))
    return pb


def throughput_figures(n_obs: int, lsmr_iters, stats: dict, ms_total: float, steps: int,
                       ranks: int) -> dict:
    """Whole-job observation-iterations/s (N x the LSMR iterations of every
    column, per second; rank 0's counts times the ranks) and the algorithmic
    bytes of every kernel of a step per second."""
    step_s = ms_total * 1e-3 / steps
    iters = float(np.sum(np.asarray(lsmr_iters, dtype=np.float64)))
    alg = sum(float(v["bytes"]) for v in stats.values()) / steps
    return {"observation_iterations_per_s": n_obs * iters * ranks / step_s,
            "lsmr_iterations_per_step": iters * ranks,
            "alg_bytes_per_step": alg * ranks,
            "alg_GBps": alg * ranks / step_s / 1e9}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str):
    """Per-launch DRAM traffic of `kernel` on this workload from the committed
    ncu summary (profiles/traffic.json), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    e = d.get(WORKLOAD_NAME, {}).get(kernel)
    return None if e is None else float(e["bytes_per_launch"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

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
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

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


def cpu_baseline(pb, max_cols: int = 1):
    """The CPU oracle (FP64 restatement of the reference's CPU solver) on a
    bounded sample: the first column(s) of the same workload."""
    from oracle import oracle as O
    O.build()
    nthreads = O.host_threads()
    ys = pb.Y[:, :max_cols].astype(np.float64)
    t = time.perf_counter()
    R, its, cvs = O.solve_residuals_cols(ys, pb.refs, pb.nlev, pb.interaction, pb.weights,
                                         tol=1e-8, maxiter=10000, nthreads=nthreads)
    dt = time.perf_counter() - t
    return {"value": max_cols / dt, "unit": "solves/s", "cores": nthreads, "kind": "port",
            "sample": f"{max_cols} of {pb.Y.shape[1]} columns at full N={pb.N} "
                      f"({dt:.1f} s; serial reduce, expand on {nthreads} threads)",
            "iterations": [int(x) for x in its]}, R


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    pb = make_workload(args.scale, 0, args.ncols)
    from oracle import oracle as O
    O.build()
    nthreads = O.host_threads()
    y = pb.Y[:, :1].astype(np.float64)
    for _ in range(args.warmup):
        O.solve_residuals_cols(y, pb.refs, pb.nlev, pb.interaction, pb.weights, tol=1e-8,
                               maxiter=10000, nthreads=nthreads)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.solve_residuals_cols(y, pb.refs, pb.nlev, pb.interaction, pb.weights, tol=1e-8,
                               maxiter=10000, nthreads=nthreads)
    dt = time.perf_counter() - t
    value = args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "N": pb.N, "fixed_effects": pb.nlev,
                   "columns_per_step": 1, "tol": 1e-8},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "port",
                         "sample": f"1 column of {pb.Y.shape[1]} per step at full N={pb.N}"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "FixedEffects.jl (Julia) is not installed here; its CPU solver path is timed "
                "through the C restatement in oracle/ (serial reduce as src/SolverCPU.jl:20-27, "
                "threaded expand as :29-34)",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    import __graft_entry__ as g
    fe = g.load_package()

    t0 = time.perf_counter()
    pb = make_workload(args.scale, rank, args.ncols)
    log(f"[rank {rank}] workload generated in {time.perf_counter() - t0:.1f} s; "
        f"N={pb.N} levels={pb.nlev}")
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
    t0 = time.perf_counter()
    feM = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float32, precision="mixed")
    torch.cuda.synchronize()
    plan_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    L = fe._lib.load()
    fe._lib.check(L.fe_plan_set_stream(feM._h, stream.cuda_stream))
    if args.no_absorb:  # the full-LSMR loop over all fixed effects
        feM.set_option(fe._lib.FE_OPT_ABSORB, 0)

    N, ncols = pb.N, pb.Y.shape[1]
    # inputs resident in HBM: a pristine column-major copy, refreshed into the
    # work buffer at the start of every step (the solve is in place)
    Y0 = torch.from_numpy(np.ascontiguousarray(pb.Y.T)).to(dev).t()
    Yw = torch.empty_like(Y0.t()).t()

    def step():
        Yw.copy_(Y0)
        return feM.solve_residuals(Yw, tol=1e-8, maxiter=10000)

    for _ in range(args.warmup):
        _, its, cvs = step()
    torch.cuda.synchronize()
    feM.reset_stats()
    feM.set_option(fe._lib.FE_OPT_PROFILE, 1)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            _, its, cvs = step()
        ev1.record(stream)
        torch.cuda.synchronize()
    feM.set_option(fe._lib.FE_OPT_PROFILE, 0)
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    stats = feM.kernel_stats()
    conv_all = bool(np.all(cvs))
    its_list = [int(x) for x in its]
    info = feM.last_solve_info(ncols)
    result_dev = Yw[:, 0].double().cpu().numpy()

    # e2e through the host-buffer C ABI (pinned host Y, H2D + D2H inside)
    e2e_steps = max(1, min(args.steps, 3))
    Yh_pin = torch.empty((ncols, N), dtype=torch.float32, pin_memory=True)
    Yh0 = np.ascontiguousarray(pb.Y.T)
    Yh = Yh_pin.numpy().T  # column-major view of pinned memory
    feM_h = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float32, precision="mixed")
    if args.no_absorb:
        feM_h.set_option(fe._lib.FE_OPT_ABSORB, 0)
    Yh_pin.numpy()[...] = Yh0
    feM_h.solve_residuals(Yh, tol=1e-8, maxiter=10000)  # warm-up
    if dist:
        dist.barrier()
    e2e_ms = 0.0
    for _ in range(e2e_steps):
        Yh_pin.numpy()[...] = Yh0  # refresh the inputs (outside the timed call)
        torch.cuda.synchronize()
        t = time.perf_counter()
        feM_h.solve_residuals(Yh, tol=1e-8, maxiter=10000)
        e2e_ms += (time.perf_counter() - t) * 1e3
    e2e_ms /= e2e_steps
    if dist:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    feM_h.close()

    # second baseline: the plain per-column FP64 form of this library
    plain = None
    if not args.no_plain and rank == 0:
        npl = min(args.plain_cols, ncols)
        feP = fe.AbstractFixedEffectSolver(fes, pb.weights, "CUDA", np.float64, precision="fp64")
        feP.set_option(fe._lib.FE_OPT_TILE, 1)
        Yp0 = torch.from_numpy(np.ascontiguousarray(pb.Y[:, :npl].T.astype(np.float64))).to(dev).t()
        Yp = Yp0.clone()
        feP.solve_residuals(Yp, tol=1e-8, maxiter=10000)
        Yp = torch.empty_like(Yp0.t()).t()
        Yp.copy_(Yp0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        fe._lib.check(L.fe_plan_set_stream(feP._h, stream.cuda_stream))
        a.record(stream)
        _, pits, pcv = feP.solve_residuals(Yp, tol=1e-8, maxiter=10000)
        b.record(stream)
        torch.cuda.synchronize()
        pms = a.elapsed_time(b)
        plain = {"value": npl / (pms * 1e-3), "unit": "solves/s", "columns_timed": npl,
                 "iterations": [int(x) for x in pits], "converged": bool(np.all(pcv))}
        plain_result = Yp[:, 0].double().cpu().numpy()
        feP.close()

    line = None
    if rank == 0:
        total_cols = ncols * ws
        value = total_cols / (ms * 1e-3 / args.steps)
        e2e_value = total_cols / (e2e_ms * 1e-3)
        # dominant kernel and its roofline (CUDA events inside the timed region)
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
                          "GBps": round(gbps(v), 1) if gbps(v) else None}
                      for k, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])}
        launches = int(sum(v["launches"] for v in stats.values() if v["launches"]))
        traffic = committed_traffic(tname)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "N": N, "fixed_effects": pb.nlev,
                       "columns_per_gpu": ncols, "tol": 1e-8, "precision": "mixed",
                       "parallelism": f"columns sharded over {ws} GPU(s)",
                       "l2": "inputs larger than L2 (1.28 GB per step)"},
            # the solver constructor: refs upload, validation and integer plan
            # (radix sorts) on the device, weights, preconditioner
            "plan_build": {"device_s": round(plan_s, 3)},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": N * ncols * 4,
                    "d2h_bytes_per_step": N * ncols * 4, "ms_per_step": e2e_ms},
            "roofline": {"bound": "hbm", "kernel": tname, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "frac_of_nominal_7700": achieved / 7700.0,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "traffic": traffic, "alg_bytes_per_launch": alg,
                         "launch_time": "mean CUDA-event time of the working launches "
                                        f"({tw.size} of {tv['launches']})"},
            "gpu_launches": launches,
            "kernels": per_kernel,
            "throughput": throughput_figures(N, info["lsmr_iters"], stats, ms, args.steps, ws),
            "iterations": its_list, "converged": conv_all,
            "refinement_rounds": [int(x) for x in info["rounds"]],
            "fp64_test2": [float(x) for x in info["test2"]],
        }
        if plain is not None:
            line["plain_fp64_per_column"] = plain
            line["speedup_vs_plain_fp64"] = value / plain["value"]
        if not args.no_cpu_baseline:
            cb, R = cpu_baseline(pb, 1)
            ro = R[:, 0]
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            rel = float(np.linalg.norm(result_dev - ro) / np.linalg.norm(ro))
            line["max_rel_err_vs_oracle"] = {"column0_mixed": rel}
            if plain is not None:
                line["max_rel_err_vs_oracle"]["column0_plain_fp64"] = float(
                    np.linalg.norm(plain_result - ro) / np.linalg.norm(ro))
            line["oracle_iterations"] = cb["iterations"]
            # the host integer plan (stable counting sorts, one core) for scale
            t0 = time.perf_counter()
            from oracle import oracle as O
            O.integer_plan(pb.refs, pb.nlev, feM.primary())
            line["plan_build"]["oracle_integer_plan_s"] = round(time.perf_counter() - t0, 3)
            line["plan_build"]["oracle_cores"] = 1
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
    pb = make_workload(args.scale, 0, args.ncols)
    fes = [fe.FixedEffect.from_refs(r, n, a) for r, n, a in zip(pb.refs, pb.nlev, pb.interaction)]
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
                feM.solve_residuals(Y, tol=1e-8, maxiter=10000)
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
        feM.solve_residuals(A, tol=1e-8, maxiter=10000)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    timed("pageable")  # warm-up: tuning, graphs, staging
    out = {"metric": "host-buffer solve time", "unit": "s", "higher_is_better": False,
           "data": "synthetic", "config": {"workload": "worker_firm_year_10m", "N": N,
                                           "columns": ncols, "precision": "mixed", "tol": 1e-8}}
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
    ap.add_argument("--scale", type=float, default=1.0, help="shrink N and levels (debug only)")
    ap.add_argument("--ncols", type=int, default=32)
    ap.add_argument("--plain-cols", type=int, default=4)
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
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
