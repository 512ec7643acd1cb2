#!/usr/bin/env python
"""Benchmark: CG probe-solves/s of the SEDI estimator on one B200 (or N, probe-sharded).

Workload (the drop-in configuration): 128x128x128 grid, the reference 7-point
operator (a=6, b=c=1), CG with the constant Jacobi preconditioner 1/a, tol
1e-9 run to convergence, 64 probes per GPU drawn exactly as the reference
does (std::mt19937(seed) -> uniform_real(0,1) -> +-1, seeds 1234+k on rank 0,
disjoint seed ranges on the other ranks).  One step = one full estimate of
the 64 probes (x = 0, solve to tol, t += x.*v, q += v.*v, D = t./q).  The
probes are synthetic in the reference's own sense; there is no dataset.

Arms:
  --impl sedi (default): the batched mixed-precision form (FP32 Krylov
      vectors, FP64 reductions and FP64 reliable update), device-resident
      inputs for `value`; `e2e` repeats the step through the C ABI from pinned
      host probes to the host D.  N > 1 (torchrun): each rank estimates its
      own 64 probes and t, q are summed with one NCCL all-reduce per step.
  --impl reference: the reference CPU build (stochastic-estimator.cg.exe,
      unmodified sources, single-rank MPI stand-in) on the host cores: one
      step = P concurrent single-rank processes, one 128^3 probe each.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

GRID = (128, 128, 128)
SAMPLES = 64
SEED = 1234
TOL = 1e-9
MAXITER = 5000
METRIC = "CG probe-solves/s at 1e-8 vs FP64 oracle"
UNIT = "probe-solves/s"
WORKLOAD = ("SEDI estimator, 128^3 7-point stencil (a=6,b=c=1), CG + Jacobi, tol 1e-9 to convergence, "
            "64 probes per GPU (std::mt19937(seed+k) +-1), D = sum x.*v / sum v.*v")
REF_EXE = os.path.join(REPO, "oracle", "_ref", "stochastic-estimator.cg.exe")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sedi", "reference"], default="sedi")
    ap.add_argument("--form", choices=["mixed", "fp64", "plain"], default="mixed",
                    help="mixed / fp64: batched forms; plain: the single-vector FP64 form (profiling cases)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # Small cases for profiler captures (not the benchmark configuration):
    ap.add_argument("--grid", default=None, help="override the grid, e.g. 128x128x64")
    ap.add_argument("--maxiter", type=int, default=None, help="override maxiter (with --tol 0: fixed iterations)")
    ap.add_argument("--tol", type=float, default=None)
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, kernel timing, accuracy and other forms")
    ap.add_argument("--solver", choices=["cg", "pcg", "bicgstab"], default="cg",
                    help="solver of the timed form (profiling cases; the benchmark configuration is CG)")
    ap.add_argument("--serve-jobs", type=int, default=12, help="jobs in the serving run (0: skip it)")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving measurement")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner (built-in launch choices)")
    ap.add_argument("--workload", choices=["dropin", "batched256", "large512"], default="dropin",
                    help="dropin: the benchmark line; batched256 / large512: the 256^3 x 128-probe and the "
                         "512^3 x 16-probe configurations, one line each")
    a = ap.parse_args()
    if (a.solver != "cg" or a.form == "plain") and not a.no_extras:
        ap.error("--solver pcg/bicgstab and --form plain are for profiling cases (with --no-extras)")
    global GRID, MAXITER, TOL
    if a.grid:
        GRID = tuple(int(v) for v in a.grid.split("x"))
    if a.maxiter is not None:
        MAXITER = a.maxiter
    if a.tol is not None:
        TOL = a.tol
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = str(index)
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                                      "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != self.index:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference (the reference's own binary), P concurrent single-rank processes.
# ---------------------------------------------------------------------------
def reference_sample(procs, seed0, grid=GRID):
    """One bounded sample: `procs` single-rank reference processes, one probe each.
    Returns (probe-solves/s, wall seconds, kind, iteration counts)."""
    g = "x".join(map(str, grid))
    jobs = []
    t0 = time.perf_counter()
    if os.path.exists(REF_EXE):
        kind = "reference"
        for j in range(procs):
            env = dict(os.environ, SEDI_SEED=str(seed0 + j), OMP_NUM_THREADS="1")
            jobs.append(subprocess.Popen([REF_EXE, "-g", g, "-p", "1x1x1", "-s", "1", "-e", repr(TOL), "-m",
                                          str(MAXITER)], env=env, stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True))
        iters = []
        for p in jobs:
            out, _ = p.communicate()
            if p.returncode != 0:
                raise RuntimeError("reference process failed")
            for line in out.splitlines():
                if line.startswith("Total solve time"):
                    iters.append(int(line.rsplit("max=", 1)[1]))
    else:
        kind = "port"
        code = ("import sys; sys.path.insert(0, %r); import _oracle as O; "
                "r = O.estimate(2, %r, 1, int(sys.argv[1]), %d, %r); print(int(r['iters'][0]))"
                % (os.path.join(REPO, "tests"), tuple(grid), MAXITER, TOL))
        for j in range(procs):
            jobs.append(subprocess.Popen([sys.executable, "-c", code, str(seed0 + j)], stdout=subprocess.PIPE,
                                         text=True))
        iters = [int(p.communicate()[0].strip()) for p in jobs]
    wall = time.perf_counter() - t0
    return procs / wall, wall, kind, iters


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    procs = host_cores()
    for w in range(args.warmup):
        reference_sample(procs, SEED, grid=(32, 32, 32))  # untimed warm-up on the small grid
    vals, walls, kind, iters = [], [], None, []
    for k in range(args.steps):
        v, wall, kind, it = reference_sample(procs, SEED + k * procs)
        vals.append(v)
        walls.append(wall)
        iters += it
    value = sum(procs for _ in vals) / sum(walls)
    sample = (f"{procs} concurrent single-rank processes x 1 probe each per step (128^3 CG tol 1e-9, "
              f"-p 1x1x1), {args.steps} steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": list(GRID), "probes_per_step": procs, "solver": "cg", "tol": TOL,
                   "parallelism": f"{procs} processes x -p 1x1x1"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": [min(iters), max(iters)] if iters else None,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Serving: Poisson-arriving estimation jobs on one GPU.
# ---------------------------------------------------------------------------
SERVE_EDGES = (32, 48, 64, 96, 128, 192)


def serve_jobs(njobs, seed=SEED):
    """Seeded job mix: cubic grid edge uniform over SERVE_EDGES, samples uniform
    8..64, tol log-uniform 1e-10..1e-6, solver uniform over CG / pipelined CG /
    BiCGStab, precision FP64 or FP32 + FP64 reliable update; probe seeds
    derived from the job id."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return {
        "edge": rng.choice(SERVE_EDGES, njobs),
        "samples": rng.integers(8, 65, njobs),
        "tol": 10.0 ** rng.uniform(-10.0, -6.0, njobs),
        "solver": rng.choice(["cg", "pcg", "bicgstab"], njobs),
        "precision": rng.integers(0, 2, njobs),
        "seed": SEED + 100003 * np.arange(njobs),
    }


def run_serving(S, njobs, maxiter=5000):
    """Capacity from a closed-loop run (every job queued at t = 0), then an
    open-loop run with Poisson arrivals (seeded) at 80% of that capacity.
    Latency = scheduled arrival to D on the host."""
    import numpy as np
    jobs = serve_jobs(njobs)
    args = (jobs["solver"], jobs["precision"], jobs["edge"], jobs["samples"], jobs["seed"], jobs["tol"], maxiter)
    with S.Server() as srv:
        lat0, rc0, mk0 = srv.replay(np.zeros(njobs), *args)
        cap = njobs / mk0
        rate = 0.8 * cap
        arrival = np.cumsum(np.random.default_rng(SEED + 1).exponential(1.0 / rate, njobs))
        arrival -= arrival[0]
        lat, rcs, mk = srv.replay(arrival, *args)
        st = srv.stats()
    probes = int(np.sum(jobs["samples"]))
    return {
        "jobs": njobs, "capacity_jobs_per_s": cap, "arrival_rate_jobs_per_s": rate,
        "jobs_per_s": njobs / mk, "probe_solves_per_s": probes / mk,
        "p50_latency_ms": 1e3 * float(np.percentile(lat, 50)), "p99_latency_ms": 1e3 * float(np.percentile(lat, 99)),
        "mean_latency_ms": 1e3 * float(lat.mean()), "closed_loop_p50_ms": 1e3 * float(np.percentile(lat0, 50)),
        "result_codes_nonzero": int(np.count_nonzero(rcs)) + int(np.count_nonzero(rc0)),
        "nonzero_jobs": [{"solver": str(jobs["solver"][k]), "edge": int(jobs["edge"][k]),
                          "precision": "fp64" if int(jobs["precision"][k]) == 0 else "mixed",
                          "tol": float(jobs["tol"][k]), "samples": int(jobs["samples"][k]),
                          "rc_open_loop": int(rcs[k]), "rc_closed_loop": int(rc0[k])}
                         for k in range(njobs) if rcs[k] != 0 or rc0[k] != 0],
        "peak_device_gb": st["peak_bytes"] / 1e9, "budget_gb": st["budget_bytes"] / 1e9,
        "contexts_created": st["ctx_created"], "contexts_reused": st["ctx_reused"], "max_running": st["max_running"],
        "mix": "edge U{32,48,64,96,128,192}^3, samples U{8..64}, tol logU[1e-10,1e-6], solver U{CG,PCG,BiCGStab}, "
               "precision U{FP64, FP32+RU}, seed 1234; Poisson arrivals at 0.8 x closed-loop capacity",
    }


# ---------------------------------------------------------------------------
# Large single-GPU configurations (one JSON line each, not the benchmark line).
# ---------------------------------------------------------------------------
def _peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    return (json.load(open(path))["hbm_gbs"], "measured") if os.path.exists(path) else (6650.0, "fallback")


def _kernel_table(ctx, peak):
    return [{"kernel": k, "ms": ms, "bytes": by, "GB/s": by / ms / 1e6, "frac": by / ms / 1e6 / peak}
            for k, ms, by in ctx.time_kernels(reps=10)]


def run_batched256(S, args):
    """256^3 grid, 128 probes interleaved (mixed precision, FP32 vectors with FP64
    reliable update at the autotuned period), CG and pipelined CG to 1e-9.  D
    error against the batched FP64 form on the same probes (which follows the
    single-vector FP64 method lane by lane), rate of the single-vector FP64 form
    on 4 of the probes."""
    import numpy as np
    import torch
    grid, samples, tol, maxiter = (256, 256, 256), 128, 1e-9, 20000
    peak, psrc = _peak()
    out = {"workload": "256^3 x 128 probes, FP32 + FP64 reliable update, tol 1e-9", "peak_gbs": peak,
           "peak_source": psrc, "solvers": {}}
    for solver in ("cg", "pcg"):
        tune = S.autotune(solver, grid, samples, precision=S.MIXED, maxiter=maxiter, tol=tol, seed=SEED)
        with S.Context(solver, grid, precision=S.MIXED, batch=samples) as c:
            cfg = c.config()
            for _ in range(max(args.warmup - 2, 1)):
                c.estimate(samples, SEED, maxiter, tol)
            torch.cuda.synchronize()
            clocks = Clocks(0)
            clocks.start()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                r = c.estimate(samples, SEED, maxiter, tol)
            dt = (time.perf_counter() - t0) / args.steps
            clk = clocks.stop()
            kern = _kernel_table(c, peak)
        Dm = r["D"]
        # FP64 form on the same probes, in two halves of 64 (pipelined CG in
        # FP64 for 128 probes would need 189 GB); t and q add up exactly.
        half = samples // 2
        with S.Context(solver, grid, precision=S.FP64, batch=half) as c64:
            t0 = time.perf_counter()
            ra = c64.estimate(half, SEED, maxiter, tol)
            rb = c64.estimate(half, SEED + half, maxiter, tol)
            dt64 = time.perf_counter() - t0
        r64 = {"D": (ra["t"] + rb["t"]) / (ra["q"] + rb["q"])}
        with S.Context(solver, grid) as cp:
            cp.estimate(1, SEED, maxiter, tol)
            t0 = time.perf_counter()
            cp.estimate(4, SEED, maxiter, tol)
            plain = 4 / (time.perf_counter() - t0)
        n = grid[0] * grid[1] * grid[2]
        out["solvers"][solver] = {
            "probe_solves_per_s": samples / dt, "ms_per_estimate": 1e3 * dt,
            "gpoint_iterations_per_s": float(np.sum(r["iters"])) * n / dt / 1e9,
            "iterations": [int(r["iters"].min()), int(r["iters"].max())],
            "results_nonzero": int(np.count_nonzero(r["results"])),
            "D_rel_err_vs_fp64": float(np.abs(Dm - r64["D"]).max() / np.abs(r64["D"]).max()),
            "batched_fp64_probe_solves_per_s": samples / dt64,
            "plain_fp64_probe_solves_per_s": plain, "speedup_vs_plain_fp64": samples / dt / plain,
            "autotuned": tune, "config": cfg, "kernels": kern, "clocks": clk,
        }
    print(json.dumps(out), flush=True)


def run_large512(S, args):
    """512^3 grid (134M points), pipelined CG, 16 probes in FP32 with FP64
    true-residual recompute and FP64 accumulators, tol 1e-8, maxiter 500 (the
    limit is reached: result 1 per probe); D error against the single-vector
    FP64 pipelined CG on the same probes."""
    import numpy as np
    import torch
    grid, samples, tol, maxiter = (512, 512, 512), 16, 1e-8, 500
    peak, psrc = _peak()
    with S.Context("pcg", grid, precision=S.MIXED, batch=samples) as c:
        c.estimate(samples, SEED, 20, tol, ignore_errors=True)  # warm-up (graph capture)
        torch.cuda.synchronize()
        clocks = Clocks(0)
        clocks.start()
        t0 = time.perf_counter()
        r = c.estimate(samples, SEED, maxiter, tol, ignore_errors=True)
        dt = time.perf_counter() - t0
        clk = clocks.stop()
        kern = _kernel_table(c, peak)
        cfg = c.config()
    with S.Context("pcg", grid) as cp:
        t0 = time.perf_counter()
        rp = cp.estimate(samples, SEED, maxiter, tol, ignore_errors=True)
        dtp = time.perf_counter() - t0
    n = grid[0] * grid[1] * grid[2]
    out = {"workload": "512^3 x 16 probes, pipelined CG, FP32 + FP64 reliable update, tol 1e-8, maxiter 500",
           "probe_solves_per_s": samples / dt, "ms_per_estimate": 1e3 * dt,
           "gpoint_iterations_per_s": float(np.sum(r["iters"])) * n / dt / 1e9,
           "iterations": [int(r["iters"].min()), int(r["iters"].max())], "results": sorted(set(map(int, r["results"]))),
           "D_rel_err_vs_plain_fp64": float(np.abs(r["D"] - rp["D"]).max() / np.abs(rp["D"]).max()),
           "final_err_mixed": [float(r["errs"].min()), float(r["errs"].max())],
           "final_err_fp64": [float(rp["errs"].min()), float(rp["errs"].max())],
           "plain_fp64_probe_solves_per_s": samples / dtp, "speedup_vs_plain_fp64": dtp / dt,
           "kernels": kern, "config": cfg, "clocks": clk, "peak_gbs": peak, "peak_source": psrc}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# The sedi_b200 arm.
# ---------------------------------------------------------------------------
def traffic_per_launch(kernel):
    """DRAM bytes per launch of `kernel` at the bench size, from the committed
    ncu summary (profiles/ncu_traffic.txt: '<kernel> <bytes per launch>')."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 2 and f[0] == kernel:
            try:
                return float(f[1])
            except ValueError:
                return None
    return None


def run_sedi(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import sedi_b200 as S

    rank, world, local = dist_env()
    if args.workload != "dropin":
        if rank == 0:
            (run_batched256 if args.workload == "batched256" else run_large512)(S, args)
        return
    if args.serve_only:
        if rank == 0:
            print(json.dumps({"serving": run_serving(S, args.serve_jobs)}), flush=True)
        return
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", torch.cuda.current_device())
    n = GRID[0] * GRID[1] * GRID[2]
    seed0 = SEED + rank * SAMPLES

    # Probes: generated once on the host with the reference's generator, pinned.
    host = torch.empty((SAMPLES, n), dtype=torch.float64).pin_memory()
    hv = host.numpy()
    for k in range(SAMPLES):
        hv[k] = S.fill_probe(seed0 + k, n)
    probes = host.to(dev)
    D = torch.empty(n, dtype=torch.float64, device=dev)
    t = torch.empty(n, dtype=torch.float64, device=dev)
    q = torch.empty(n, dtype=torch.float64, device=dev)
    prec = S.MIXED if args.form == "mixed" else S.FP64
    # Launch choices for this shape, measured before the timed region
    # (slice width, i3 split, graph chunk, reliable-update period).
    tuned = None
    if not args.no_autotune and not args.no_extras:
        tuned = S.autotune(args.solver, GRID, SAMPLES, precision=prec, maxiter=MAXITER, tol=TOL, seed=seed0)
    ctx = S.Context(args.solver, GRID, precision=prec, batch=1 if args.form == "plain" else SAMPLES)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream)

    def step():
        r = ctx.estimate_dev(SAMPLES, probes, D, t, q, maxiter=MAXITER, tol=TOL)
        if world > 1:
            dist.all_reduce(t)
            dist.all_reduce(q)
            torch.div(t, q, out=D)
        return r

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(args.warmup, 0)):
        res = step()
    barrier()
    clocks = Clocks(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else
                    os.environ["CUDA_VISIBLE_DEVICES"].split(",")[torch.cuda.current_device()])
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = ctx.launches
    e0.record(stream)
    iters = []
    for _ in range(args.steps):
        res = step()
        iters.append(res["iters"])
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    launches = ctx.launches - l0
    ms = e0.elapsed_time(e1)
    tmax = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    ms = float(tmax.item())
    value = world * SAMPLES * args.steps / (ms / 1e3)
    it_all = np.concatenate(iters)
    if TOL > 0:
        assert np.all(res["results"] == 0), "a probe did not converge"
    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "ms_per_step": ms / args.steps, "grid": list(GRID), "maxiter": MAXITER, "tol": TOL,
                              "solver": args.solver,
                              "gpu_launches": launches, "note": "profiling case, not the benchmark configuration"}),
                  flush=True)
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # End to end through the C ABI: pinned host probes in, host D out, per step.
    Dh = np.empty(n)
    barrier()
    w0 = time.perf_counter()
    for _ in range(args.steps):
        rr = ctx.estimate(SAMPLES, probes=hv, maxiter=MAXITER, tol=TOL)
        if world > 1:
            tt = torch.from_numpy(rr["t"]).to(dev)
            qq = torch.from_numpy(rr["q"]).to(dev)
            dist.all_reduce(tt)
            dist.all_reduce(qq)
            Dh[:] = (tt / qq).cpu().numpy()
        else:
            Dh[:] = rr["D"]
    barrier()
    e2e_s = torch.tensor([time.perf_counter() - w0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_val = world * SAMPLES * args.steps / float(e2e_s.item())

    out = None
    if rank == 0:
        # Roofline of the dominant per-iteration kernel (timed alone, CUDA events on this stream).
        kern = ctx.time_kernels(reps=20)
        dom = max(kern, key=lambda k: k[1])
        peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            peak = json.load(open(peaks_path))["hbm_gbs"]
            peak_src = "measured"
        else:
            peak, peak_src = 6650.0, "fallback"
        ach = dom[2] / (dom[1] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "peak_source": peak_src, "traffic": traffic_per_launch(dom[0]),
                    "bytes_per_launch": dom[2], "ms_per_launch": dom[1],
                    "kernels": [{"kernel": k[0], "ms": k[1], "bytes": k[2], "GB/s": k[2] / k[1] / 1e6,
                                 "frac": k[2] / k[1] / 1e6 / peak} for k in kern]}
        # Accuracy of this form's D against the reference's own 64-probe run
        # (strided sample of D) and against the FP64 GPU form on the same probes.
        acc = {}
        Dcur = D.cpu().numpy()
        fix = os.path.join(REPO, "tests", "golden", "full_cg_128.npz")
        if world == 1 and os.path.exists(fix):
            z = np.load(fix)
            samp = z["D_sample"]
            stride = int(eval(str(z["meta"]))["sample_stride"])
            acc["D_rel_err_vs_reference_sample"] = float(np.abs(Dcur[::stride] - samp).max() / np.abs(samp).max())
            acc["iters_equal_reference"] = bool(np.array_equal(iters[-1], z["iters"]))
        forms = {}
        with S.Context("cg", GRID, precision=S.FP64, batch=SAMPLES) as c64:
            c64.set_stream(stream)
            D64 = torch.empty_like(D)
            c64.estimate_dev(SAMPLES, probes, D64, maxiter=MAXITER, tol=TOL)
            torch.cuda.synchronize()
            a = time.perf_counter()
            c64.estimate_dev(SAMPLES, probes, D64, maxiter=MAXITER, tol=TOL)
            torch.cuda.synchronize()
            forms["batched_fp64"] = SAMPLES / (time.perf_counter() - a)
            d64 = D64.cpu().numpy()
            acc["D_rel_err_vs_gpu_fp64"] = float(np.abs(Dcur - d64).max() / np.abs(d64).max())
        with S.Context("cg", GRID) as cp:
            cp.set_stream(stream)
            Dp = torch.empty_like(D)
            k8 = 8
            cp.estimate_dev(1, probes, Dp, maxiter=MAXITER, tol=TOL)
            torch.cuda.synchronize()
            a = time.perf_counter()
            cp.estimate_dev(k8, probes, Dp, maxiter=MAXITER, tol=TOL)
            torch.cuda.synchronize()
            forms["plain_fp64_single_vector"] = k8 / (time.perf_counter() - a)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            procs = host_cores()
            v, wall, kind, it = reference_sample(procs, SEED)
            cpu = {"value": v, "unit": UNIT, "cores": procs, "kind": kind,
                   "sample": f"{procs} concurrent single-rank processes x 1 probe (128^3 CG tol 1e-9), {wall:.1f} s"}
        serving = run_serving(S, args.serve_jobs) if world == 1 and args.serve_jobs > 0 else None
        ctx_config = ctx.config()
        gpoint = float(np.sum(it_all)) * n / args.steps / (ms / 1e3 / args.steps) / 1e9 if world == 1 else None
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 vectors / f64 reductions+reliable update" if prec == S.MIXED else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(GRID), "probes_per_gpu": SAMPLES, "solver": "cg",
                       "tol": TOL, "form": args.form, "parallelism": f"probe-sharded x{world}",
                       "autotuned": tuned, "launch": ctx_config,
                       "l2": "inputs larger than L2 (1.07 GB probes + >=1.6 GB Krylov state per GPU)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": SAMPLES * n * 8,
                    "d2h_bytes_per_step": n * 8 * (3 if world > 1 else 1) + SAMPLES * 16},
            "clocks": clk,
            "gpu_launches": launches,
            "iterations": [int(it_all.min()), int(it_all.max())],
            "gpoint_iterations_per_s": gpoint,
            "accuracy": acc,
            "forms": forms,
            "serving": serving,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_sedi(args)


if __name__ == "__main__":
    main()
