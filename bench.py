#!/usr/bin/env python
"""Benchmark: CG probe-solves/s of the SEDI estimator, batched mixed precision, on one B200 (or N, probe-sharded).

Workload (the batched mixed-precision configuration): 256x256x256 grid, the
reference 7-point operator (a=6, b=c=1), 128 probe right-hand sides
interleaved in one streaming kernel per Krylov sweep, FP32 Krylov vectors with
an FP64 reliable update of x and r, FP64 reductions and estimator
accumulators, CG with the constant Jacobi preconditioner 1/a run to FP64
relative residual 1e-9, iterations replayed from captured CUDA graphs.
Probes are drawn exactly as the reference draws them (std::mt19937(seed) ->
uniform_real(0,1) -> +-1), seeds 1234+k on rank 0 and disjoint ranges on
the other ranks.  One step = one full estimate of the 128 probes (x = 0,
solve to tol, t += x.*v, q += v.*v, D = t./q).  The probes are synthetic in
the reference's own sense; there is no dataset.

Arms:
  --impl sedi (default): `value` = the estimate on probes resident in HBM;
      `e2e` = the same step through the C ABI from pinned host probes to the
      host D.  N > 1 (torchrun): each rank estimates its own 128 probes and t,
      q are summed by sedi_b200.dist.estimate_sharded (one NCCL all-reduce per
      step).  Extra keys: the 128^3 x 64-probe drop-in configuration for each
      solver (plain FP64 single-vector form against the reference's own
      output, batched FP64 and mixed forms), the serving mix, the roofline
      of every sweep.
  --impl reference: the reference CPU build (stochastic-estimator.cg.exe,
      unmodified sources, single-rank MPI stand-in) on the host cores: one
      step = P concurrent single-rank processes, one 256^3 probe each, run for
      a fixed number of iterations (-m M -i); the per-probe time to
      convergence is extrapolated with the reference's own converged
      iteration count on this grid (tests/golden/big_cg_256.npz).
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

SEED = 1234
METRIC = "CG probe-solves/s at 1e-8 vs FP64 oracle"
UNIT = "probe-solves/s"
REF_EXE = os.path.join(REPO, "oracle", "_ref", "stochastic-estimator.cg.exe")
BIG_FIXTURE = os.path.join(REPO, "tests", "golden", "big_cg_256.npz")

# Workloads: the benchmark line (batched256) and the other single-GPU configurations.
WORKLOADS = {
    "batched256": dict(grid=(256, 256, 256), samples=128, tol=1e-9, maxiter=20000, solver="cg", form="mixed",
                       text="SEDI estimator, 256^3 7-point stencil (a=6,b=c=1), CG + Jacobi to FP64 relative "
                            "residual 1e-9, 128 probe RHS per GPU interleaved (std::mt19937(seed+k) +-1), FP32 "
                            "Krylov vectors + FP64 reliable update, FP64 reductions and t/q, D = sum x.*v / sum v.*v"),
    "dropin": dict(grid=(128, 128, 128), samples=64, tol=1e-9, maxiter=5000, solver="cg", form="mixed",
                   text="SEDI estimator, 128^3 7-point stencil (a=6,b=c=1), CG + Jacobi, tol 1e-9 to convergence, "
                        "64 probes per GPU (std::mt19937(seed+k) +-1), D = sum x.*v / sum v.*v"),
}
# Compulsory bytes per point, lane and iteration (x, r, p read and written once)
# of CG: FP32 Krylov words for the mixed form, FP64 for the others.
CG_BYTES = {"mixed": 24, "fp64": 48, "plain": 48}
# Arithmetic of each form (the JSON line's dtype).
DTYPES = {"mixed": "f32 vectors / f64 reductions+reliable update", "fp64": "f64", "plain": "f64"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sedi", "reference"], default="sedi")
    ap.add_argument("--workload", choices=["batched256", "dropin", "large512", "accuracy", "sweeps", "slab", "periods"],
                    default="batched256",
                    help="batched256: the benchmark line (256^3 x 128 probes, mixed CG); dropin: 128^3 x 64 "
                         "probes; large512: the 512^3 x 16-probe pipelined-CG configuration (one JSON line); "
                         "accuracy: diagonal error of the mixed forms per in-loop target (JSON lines)")
    ap.add_argument("--form", choices=["mixed", "fp64", "plain"], default=None,
                    help="mixed / fp64: batched forms; plain: the single-vector FP64 form (profiling cases)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # Small cases for profiler captures (not the benchmark configuration):
    ap.add_argument("--grid", default=None, help="override the grid, e.g. 128x128x64")
    ap.add_argument("--samples", type=int, default=None, help="override the probes per GPU")
    ap.add_argument("--maxiter", type=int, default=None, help="override maxiter (with --tol 0: fixed iterations)")
    ap.add_argument("--tol", type=float, default=None)
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, kernel timing, accuracy and other forms")
    ap.add_argument("--solver", choices=["cg", "pcg", "bicgstab"], default=None,
                    help="solver of the timed form (profiling cases; the benchmark configuration is CG)")
    ap.add_argument("--serve-jobs", type=int, default=50, help="jobs in the serving run (0: skip it)")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving measurement")
    ap.add_argument("--e2e-steps", type=int, default=3, help="steps of the end-to-end measurement")
    ap.add_argument("--ref-iters", type=int, default=30,
                    help="iterations each reference process runs per sample (-m M -i), then extrapolated")
    a = ap.parse_args()
    wl = dict(WORKLOADS.get(a.workload, WORKLOADS["batched256"]))
    profiling = a.grid or a.samples or a.maxiter is not None or a.tol is not None or a.solver or a.form == "plain"
    if (a.solver not in (None, "cg") or a.form == "plain") and not a.no_extras:
        ap.error("--solver pcg/bicgstab and --form plain are for profiling cases (with --no-extras)")
    if a.grid:
        wl["grid"] = tuple(int(v) for v in a.grid.split("x"))
    for key in ("samples", "maxiter", "tol", "solver", "form"):
        if getattr(a, key) is not None:
            wl[key] = getattr(a, key)
    if profiling:
        wl["text"] = "profiling case (not the benchmark configuration)"
    a.wl = wl
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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
TIMER_KEYS = ("TIMER_GLOBAL", "TIMER_COMPUTE_STENCIL_INNER", "TIMER_COMPUTE_STENCIL_BORDER", "TIMER_COMPUTE_DOTPROD",
              "TIMER_COMPUTE_RNG", "TIMER_COMPUTE_MISC", "TIMER_HALO_PACK", "TIMER_HALO_ISEND_IRECV",
              "TIMER_HALO_UNPACK_WAIT", "TIMER_COMM_DOTPROD")


def parse_reference_output(text):
    """The reference's report (stochastic-estimator.cc:218-222, Timers.hpp:57-70):
    iteration min/max and its ten timer buckets in seconds."""
    out = {"timers": {}}
    for line in text.splitlines():
        if line.startswith("Total solve time"):
            out["seconds"] = float(line.split(":", 1)[1].split()[0])
            out["iter_min"] = int(line.split("min=", 1)[1].split()[0])
            out["iter_max"] = int(line.rsplit("max=", 1)[1])
        for k in TIMER_KEYS:
            if line.startswith(k + " "):
                out["timers"][k] = float(line.split("=", 1)[1].split()[0])
    return out


def reference_fixed_sample(procs, seed0, grid, iters, tol):
    """One bounded sample: `procs` concurrent single-rank reference processes,
    one probe each (seeds seed0 ..), `iters` iterations (-m iters -i).
    Returns (list of parsed reports, wall seconds, kind)."""
    g = "x".join(map(str, grid))
    t0 = time.perf_counter()
    if os.path.exists(REF_EXE):
        jobs = []
        for j in range(procs):
            env = dict(os.environ, SEDI_SEED=str(seed0 + j), OMP_NUM_THREADS="1")
            jobs.append(subprocess.Popen([REF_EXE, "-g", g, "-p", "1x1x1", "-s", "1", "-e", repr(tol), "-m",
                                          str(iters), "-i"], env=env, stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True))
        reps = []
        for p in jobs:
            out, _ = p.communicate()
            if p.returncode != 0:
                raise RuntimeError("reference process failed")
            reps.append(parse_reference_output(out))
        return reps, time.perf_counter() - t0, "reference"
    # Without the reference binary: the oracle's restatement (one process per core).
    code = ("import sys, time; sys.path.insert(0, %r); import _oracle as O; t = time.perf_counter(); "
            "r = O.estimate(2, %r, 1, int(sys.argv[1]), %d, %r); "
            "print('Total solve time: %%e seconds, iteration count min=%%d max=%%d' %% "
            "(time.perf_counter() - t, r['iters'][0], r['iters'][0]))"
            % (os.path.join(REPO, "tests"), tuple(grid), iters, tol))
    jobs = [subprocess.Popen([sys.executable, "-c", code, str(seed0 + j)], stdout=subprocess.PIPE, text=True)
            for j in range(procs)]
    reps = [parse_reference_output(p.communicate()[0]) for p in jobs]
    return reps, time.perf_counter() - t0, "port"


def converged_iterations(grid, tol):
    """The reference's own mean converged CG iteration count on `grid` at tol
    (committed fixture made by the reference binary), or None."""
    import numpy as np
    if tuple(grid) == (256, 256, 256) and tol == 1e-9 and os.path.exists(BIG_FIXTURE):
        return float(np.load(BIG_FIXTURE)["iters"].mean()), "reference run of 8 probes (tests/golden/big_cg_256.npz)"
    if tuple(grid) == (128, 128, 128) and tol == 1e-9:
        path = os.path.join(REPO, "tests", "golden", "full_cg_128.npz")
        if os.path.exists(path):
            return float(np.load(path)["iters"].mean()), "reference run of 64 probes (tests/golden/full_cg_128.npz)"
    return None, None


def extrapolate(reps, iters, n_conv):
    """Per-probe time to convergence from a fixed-iteration sample: the RNG fill
    once, the rest (setup residual + iterations + accumulation) scaled by
    n_conv / iters (the setup share is counted as iterations: conservative)."""
    per = []
    for r in reps:
        rng = r["timers"].get("TIMER_COMPUTE_RNG", 0.0)
        per.append(rng + (r["seconds"] - rng) * n_conv / iters)
    return per


def reference_baseline(procs, seed0, grid, iters, tol, points):
    """probe-solves/s of the reference on `procs` host cores (extrapolated to
    convergence), with its timer breakdown, GPoint-it/s and effective GB/s."""
    reps, wall, kind = reference_fixed_sample(procs, seed0, grid, iters, tol)
    n_conv, src = converged_iterations(grid, tol)
    if n_conv is None:
        n_conv, src = float(iters), "no converged count known: rate at the fixed iteration count"
    per = extrapolate(reps, iters, n_conv)
    value = procs / statistics.mean(per)
    timers = {k: statistics.mean(r["timers"].get(k, 0.0) for r in reps) for k in TIMER_KEYS} if reps[0]["timers"] \
        else None
    it_s = sum(r["iter_max"] for r in reps) / sum(r["seconds"] for r in reps)  # iterations per second per process
    return {
        "value": value, "kind": kind, "wall_s": wall, "per_probe_s": statistics.mean(per),
        "converged_iterations": n_conv, "converged_source": src, "sample_iterations": iters,
        "timers_s_per_process": timers,
        "gpoint_iterations_per_s": procs * it_s * points / 1e9,
        "effective_gbs": procs * it_s * points * CG_BYTES["fp64"] / 1e9,
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    wl = args.wl
    grid, tol = wl["grid"], wl["tol"]
    points = grid[0] * grid[1] * grid[2]
    procs = host_cores()
    for w in range(args.warmup):
        reference_fixed_sample(procs, SEED, grid, 2, tol)  # untimed: page-in, allocation, RNG
    vals, walls, last = [], [], None
    for k in range(args.steps):
        last = reference_baseline(procs, SEED + k * procs, grid, args.ref_iters, tol, points)
        vals.append(last["value"])
        walls.append(last["wall_s"])
    value = statistics.mean(vals)
    sample = (f"{procs} concurrent single-rank processes (-p 1x1x1) x 1 probe x {args.ref_iters} iterations "
              f"(-m {args.ref_iters} -i) per step on {'x'.join(map(str, grid))}, extrapolated per probe to "
              f"{last['converged_iterations']:.1f} iterations ({last['converged_source']}); {args.steps} steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["text"], "grid": list(grid), "probes_per_step": procs, "solver": "cg", "tol": tol,
                   "parallelism": f"{procs} processes x -p 1x1x1"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": last["kind"], "sample": sample,
                         "extrapolated": True},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timers_s_per_process": last["timers_s_per_process"],
        "gpoint_iterations_per_s": last["gpoint_iterations_per_s"],
        "effective_gbs": last["effective_gbs"],
        "effective_gbs_basis": "48 B per point per iteration (FP64 CG: x, r, p read and written)",
    }
    print(json.dumps(line), flush=True)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


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


def _latency_stats(lat):
    import numpy as np
    if len(lat) == 0:
        return None
    return {"jobs": int(len(lat)), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "max_ms": 1e3 * float(lat.max())}


def run_serving(S, njobs, maxiter=5000):
    """Capacity from a closed-loop run (every job queued at t = 0), then an
    open-loop run with Poisson arrivals (seeded) at 80% of that capacity.
    Latency = scheduled arrival to D on the host; p50/p99 overall, per
    precision, per solver and per grid edge, and the served GPoint-iterations/s."""
    import numpy as np
    jobs = serve_jobs(njobs)
    args = (jobs["solver"], jobs["precision"], jobs["edge"], jobs["samples"], jobs["seed"], jobs["tol"], maxiter)
    with S.Server() as srv:
        lat0, rc0, mk0 = srv.replay(np.zeros(njobs), *args)
        cap = njobs / mk0
        rate = 0.8 * cap
        arrival = np.cumsum(np.random.default_rng(SEED + 1).exponential(1.0 / rate, njobs))
        arrival -= arrival[0]
        lat, rcs, mk, its = srv.replay(arrival, *args, iterations=True)
        st = srv.stats()
    probes = int(np.sum(jobs["samples"]))
    pts = jobs["edge"].astype(np.float64) ** 3
    gpit = float(np.sum(pts * its)) / mk / 1e9
    prec_name = np.where(jobs["precision"] == 0, "fp64", "mixed")
    return {
        "jobs": njobs, "capacity_jobs_per_s": cap, "arrival_rate_jobs_per_s": rate,
        "jobs_per_s": njobs / mk, "probe_solves_per_s": probes / mk, "gpoint_iterations_per_s": gpit,
        "p50_latency_ms": 1e3 * float(np.percentile(lat, 50)), "p99_latency_ms": 1e3 * float(np.percentile(lat, 99)),
        "mean_latency_ms": 1e3 * float(lat.mean()), "closed_loop_p50_ms": 1e3 * float(np.percentile(lat0, 50)),
        "by_precision": {p: _latency_stats(lat[prec_name == p]) for p in ("fp64", "mixed")},
        "by_solver": {s: _latency_stats(lat[jobs["solver"] == s]) for s in ("cg", "pcg", "bicgstab")},
        "by_edge": {str(e): _latency_stats(lat[jobs["edge"] == e]) for e in SERVE_EDGES},
        "result_codes_nonzero": int(np.count_nonzero(rcs)) + int(np.count_nonzero(rc0)),
        "nonzero_jobs": [{"solver": str(jobs["solver"][k]), "edge": int(jobs["edge"][k]),
                          "precision": str(prec_name[k]), "tol": float(jobs["tol"][k]),
                          "samples": int(jobs["samples"][k]), "rc_open_loop": int(rcs[k]),
                          "rc_closed_loop": int(rc0[k])}
                         for k in range(njobs) if rcs[k] != 0 or rc0[k] != 0],
        "peak_device_gb": st["peak_bytes"] / 1e9, "budget_gb": st["budget_bytes"] / 1e9,
        "contexts_created": st["ctx_created"], "contexts_reused": st["ctx_reused"], "max_running": st["max_running"],
        "mix": "edge U{32,48,64,96,128,192}^3, samples U{8..64}, tol logU[1e-10,1e-6], solver U{CG,PCG,BiCGStab}, "
               "precision U{FP64, FP32+RU}, seed 1234; Poisson arrivals at 0.8 x closed-loop capacity",
    }


# ---------------------------------------------------------------------------
# Extra single-GPU measurements.
# ---------------------------------------------------------------------------
def _kernel_table(ctx, peak):
    return [{"kernel": k, "ms": ms, "bytes": by, "GB/s": by / ms / 1e6, "frac": by / ms / 1e6 / peak}
            for k, ms, by in ctx.time_kernels(reps=10)]


def _relmax(a, b):
    import numpy as np
    return float(np.abs(a - b).max() / np.abs(b).max())


def dropin_forms(S, stream):
    """The 128^3 x 64-probe drop-in configuration for each solver, tol 1e-9 to
    convergence: the plain FP64 single-vector form (the reference's method
    kernel by kernel) with its D against the reference's own 64-probe output
    (strided sample, tests/golden/full_<solver>_128.npz), the batched FP64
    form and the mixed form (its D against the batched FP64 form)."""
    import numpy as np
    import torch
    grid, samples, tol, maxiter = (128, 128, 128), 64, 1e-9, 5000
    n = grid[0] * grid[1] * grid[2]
    dev = torch.device("cuda", torch.cuda.current_device())
    probes = torch.empty((samples, n), dtype=torch.float64, device=dev)
    S.fill_probes_dev(SEED, probes, stream)
    D = torch.empty(n, dtype=torch.float64, device=dev)
    out = {}
    for solver in ("cg", "pcg", "bicgstab"):
        row = {}
        fix = os.path.join(REPO, "tests", "golden", f"full_{solver}_128.npz")
        z = np.load(fix) if os.path.exists(fix) else None
        stride = int(eval(str(z["meta"]))["sample_stride"]) if z is not None else None
        for form, prec, batch in (("plain_fp64", S.FP64, 1), ("batched_fp64", S.FP64, samples),
                                  ("mixed", S.MIXED, samples)):
            with S.Context(solver, grid, precision=prec, batch=batch) as c:
                c.set_stream(stream)
                c.estimate_dev(min(4, samples) if batch == 1 else samples, probes, D, maxiter=maxiter, tol=tol)
                torch.cuda.synchronize()
                a = time.perf_counter()
                r = c.estimate_dev(samples, probes, D, maxiter=maxiter, tol=tol)
                torch.cuda.synchronize()
                dt = time.perf_counter() - a
            Dh = D.cpu().numpy()
            ent = {"probe_solves_per_s": samples / dt, "iterations": [int(r["iters"].min()), int(r["iters"].max())],
                   "results_nonzero": int(np.count_nonzero(r["results"]))}
            if z is not None:
                ent["D_rel_err_vs_reference_sample"] = _relmax(Dh[::stride], z["D_sample"])
                ent["iters_equal_reference"] = bool(np.array_equal(r["iters"], z["iters"]))
            row[form] = ent
            row["_D_" + form] = Dh
        row["mixed"]["D_rel_err_vs_batched_fp64"] = _relmax(row.pop("_D_mixed"), row["_D_batched_fp64"])
        row.pop("_D_batched_fp64")
        row.pop("_D_plain_fp64")
        row["mixed_vs_plain_fp64"] = row["mixed"]["probe_solves_per_s"] / row["plain_fp64"]["probe_solves_per_s"]
        out[solver] = row
    del probes
    torch.cuda.empty_cache()
    return out


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
           "D_rel_err_vs_plain_fp64": _relmax(r["D"], rp["D"]),
           "final_err_mixed": [float(r["errs"].min()), float(r["errs"].max())],
           "final_err_fp64": [float(rp["errs"].min()), float(rp["errs"].max())],
           "plain_fp64_probe_solves_per_s": samples / dtp, "speedup_vs_plain_fp64": dtp / dt,
           "kernels": kern, "config": cfg, "clocks": clk, "peak_gbs": peak, "peak_source": psrc}
    print(json.dumps(out), flush=True)


def run_accuracy(S, args):
    """Diagonal error of the mixed forms against the FP64 form on the same
    probes and against the converged diagonal (FP64 CG to 1e-13), per in-loop
    target theta, tol 1e-9: 48^3 and 128^3 x 64 probes (every solver),
    256^3 x 32 probes (CG, pipelined CG).  One JSON line per grid and solver."""
    import numpy as np

    def est(solver, g, k, tol, prec, theta=None):
        with S.Context(solver, g, precision=prec, batch=k) as c:
            if theta is not None:
                c.mixed_target = theta
            t0 = time.perf_counter()
            r = c.estimate(k, SEED, 20000, tol)
            return r, time.perf_counter() - t0

    for g, k, solvers in (((48, 48, 48), 64, ("cg", "pcg", "bicgstab")),
                          ((128, 128, 128), 64, ("cg", "pcg", "bicgstab")), ((256, 256, 256), 32, ("cg", "pcg"))):
        ex, _ = est("cg", g, k, 1e-13, S.FP64)
        for solver in solvers:
            r64, dt64 = est(solver, g, k, 1e-9, S.FP64)
            row = {"grid": list(g), "probes": k, "solver": solver, "fp64_vs_converged": _relmax(r64["D"], ex["D"]),
                   "fp64_iterations": float(r64["iters"].mean()), "fp64_s": dt64, "mixed": []}
            for name, prec in (("mixed", S.MIXED),):
                for th in (1.0, 0.3, 0.1, 0.03):
                    rm, dtm = est(solver, g, k, 1e-9, prec, th)
                    row["mixed"].append({"form": name, "theta": th, "vs_fp64": _relmax(rm["D"], r64["D"]),
                                         "vs_converged": _relmax(rm["D"], ex["D"]),
                                         "iterations": float(rm["iters"].mean()), "s": dtm,
                                         "results_nonzero": int(np.count_nonzero(rm["results"]))})
            print(json.dumps(row), flush=True)


def run_sweeps(S, args):
    """Each streaming sweep alone (CUDA events, 10-20 launches after one)
    across the narrow-sweep forms (1 ring, 2 in place on 32x16 tiles with two
    blocks per SM, 3 in place on 32x32 tiles with six stages) and L2 prefetch
    distances: mixed CG and BiCGStab at 128^3 x 64 and 256^3 x 128 lanes,
    batched FP64 (CG, BiCGStab, pipelined CG) at 256^3 x 64 lanes (slice
    width 8 and 2), and the
    single-vector FP64 sweeps of the three solvers at 256^3.  One JSON line
    per configuration with each sweep's ms, GB/s and fraction of the
    measured HBM bandwidth."""
    peak, psrc = _peak()

    def row(tag, ks):
        tag["kernels"] = [{"kernel": k, "ms": ms, "GB/s": by / ms / 1e6, "frac": by / ms / 1e6 / peak}
                          for k, ms, by in ks]
        tag["peak_gbs"], tag["peak_source"] = peak, psrc
        print(json.dumps(tag), flush=True)

    for g, k in (((128, 128, 128), 64), ((256, 256, 256), 128)):
        for solver, pfs in (("cg", (0, 2)), ("bicgstab", (0,))):
            for form in (1, 2, 3):
                for pf in pfs:
                    S.set_tuning(solver, g, k, precision=S.MIXED, sweep_a_form=form, prefetch_planes=pf)
                    with S.Context(solver, g, precision=S.MIXED, batch=k) as c:
                        row({"grid": list(g), "lanes": k, "solver": solver, "form": "mixed", "sweep_form": form,
                             "prefetch_planes": pf, "config": c.config()}, c.time_kernels(reps=10))
    g = (256, 256, 256)
    for solver in ("cg", "bicgstab", "pcg"):
        for W in (8, 2):
            for form in ((1, 3) if solver != "pcg" else (1,)):
                S.set_tuning(solver, g, 64, precision=S.FP64, slice_width=W, sweep_a_form=form, prefetch_planes=0)
                with S.Context(solver, g, precision=S.FP64, batch=64) as c:
                    row({"grid": list(g), "lanes": 64, "solver": solver, "form": "fp64", "sweep_form": form,
                         "slice_width": W, "config": c.config()}, c.time_kernels(reps=5))
    for solver in ("cg", "bicgstab", "pcg"):
        for form in (1, 2, 3):
            S.set_tuning(solver, g, 1, precision=S.FP64, sweep_a_form=form, prefetch_planes=2)
            with S.Context(solver, g) as c:
                row({"grid": list(g), "lanes": 1, "solver": solver, "form": "plain", "sweep_form": form,
                     "prefetch_planes": 2}, c.time_kernels(reps=20))


def run_slab(S, args):
    """The slab (i3) decomposition on one GPU, P slabs in one process (halos
    by device copies), FP64, against the single-vector form on the same
    probe: (1) each solver at 512^3 (--grid), one probe, 200 fixed iterations
    (--maxiter), P = 1, 2, 4: GPoint-iterations/s of the solve alone (probe
    generation outside the timed region) and the host time spent reading dot
    products; (2) unless --no-extras, CG at 256^3 to tol 1e-9, P = 1 and 2:
    iteration counts and whether D matches across P bit for bit."""
    import numpy as np
    import torch
    from sedi_b200.domain import slab_solver

    def solve_slabs(solver, g, parts, maxiter, tol):
        sv = slab_solver(solver, g, parts, loopback=True)
        x, b = sv.zeros(), sv.zeros()
        work = sv.work()
        plane = g[0] * g[1]
        for j, s_ in enumerate(sv.local):
            sv.backend.fill_probe(b[j], SEED, sv.ranges[s_][0] * plane)
        sv.solve(x, b, 3, tol, work)  # warm-up
        for j in range(len(sv.local)):
            x[j].zero_()
        torch.cuda.synchronize()
        sv.timers = {"halo_wait": 0.0, "dot_comm": 0.0}
        t0 = time.perf_counter()
        res, err, it = sv.solve(x, b, maxiter, tol, work)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out = (it, dt, sv.timers["dot_comm"], err)
        del sv, x, b, work
        torch.cuda.empty_cache()
        return out

    g = tuple(int(v) for v in args.grid.split("x")) if args.grid else (512, 512, 512)
    iters = args.maxiter if args.maxiter else 200
    n = g[0] * g[1] * g[2]
    probe = torch.empty((1, n), dtype=torch.float64, device="cuda")
    S.fill_probes_dev(SEED, probe)
    D = torch.empty(n, dtype=torch.float64, device="cuda")
    for solver in ("cg", "pcg", "bicgstab"):
        with S.Context(solver, g) as c:
            c.estimate_dev(1, probe, D, maxiter=5, tol=0.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rp = c.estimate_dev(1, probe, D, maxiter=iters, tol=0.0)
            torch.cuda.synchronize()
            dtp = time.perf_counter() - t0
        row = {"workload": f"slab decomposition on one GPU, {solver}, {g[0]}x{g[1]}x{g[2]}, 1 probe, {iters} fixed "
                           f"iterations, FP64",
               "single_vector_gpoint_iterations_per_s": float(rp["iters"][0]) * n / dtp / 1e9, "slabs": []}
        for parts in (1, 2, 4):
            it, dt, dots, err = solve_slabs(solver, g, parts, iters, 0.0)
            row["slabs"].append({"parts": parts, "gpoint_iterations_per_s": it * n / dt / 1e9, "s": dt,
                                 "dot_read_s": dots, "final_err": err})
        print(json.dumps(row), flush=True)
    del probe, D
    torch.cuda.empty_cache()
    if args.no_extras:
        return
    g = (256, 256, 256)
    with S.Context("cg", g) as c:
        rp = c.estimate(2, SEED, 5000, 1e-9)
    row = {"workload": "slab decomposition on one GPU, cg, 256^3, 2 probes, tol 1e-9, FP64",
           "single_vector_iterations": rp["iters"].tolist(), "slabs": []}
    D1 = None
    for parts in (1, 2):
        sv = slab_solver("cg", g, parts, loopback=True)
        r = sv.estimate(2, SEED, 5000, 1e-9)
        Dg = sv.gather(r["D"])
        D1 = Dg if D1 is None else D1
        row["slabs"].append({"parts": parts, "iterations": r["iters"].tolist(),
                             "D_equal_to_one_slab": bool(np.array_equal(Dg, D1)),
                             "D_rel_err_vs_single_vector": _relmax(Dg, rp["D"])})
        del sv
        torch.cuda.empty_cache()
    print(json.dumps(row), flush=True)


def run_periods(S, args):
    """Reliable-update period of the mixed forms: BiCGStab and CG at 128^3 x
    64 probes, tol 1e-9, periods 8 to 50.  Per period: mean iterations,
    seconds per estimate, D error against the FP64 form on the same probes
    and against the converged diagonal (FP64 CG to 1e-13).  One JSON line
    per solver."""
    g, k, tol = (128, 128, 128), 64, 1e-9

    def est(solver, prec, period=0, t=tol):
        S.set_tuning(solver, g, k, precision=prec, period=period)
        with S.Context(solver, g, precision=prec, batch=k) as c:
            c.estimate(k, SEED, 20, t, ignore_errors=True)  # graph capture
            t0 = time.perf_counter()
            r = c.estimate(k, SEED, 20000, t)
            return r, time.perf_counter() - t0

    ex, _ = est("cg", S.FP64, t=1e-13)
    for solver in ("bicgstab", "cg"):
        r64, dt64 = est(solver, S.FP64)
        row = {"workload": f"reliable-update period, mixed {solver}, 128^3 x 64 probes, tol 1e-9",
               "fp64": {"iterations": float(r64["iters"].mean()), "s": dt64,
                        "vs_converged": _relmax(r64["D"], ex["D"])}, "mixed": []}
        for period in (8, 12, 16, 24, 32, 50):
            rm, dtm = est(solver, S.MIXED, period)
            row["mixed"].append({"period": period, "iterations": float(rm["iters"].mean()), "s": dtm,
                                 "vs_fp64": _relmax(rm["D"], r64["D"]), "vs_converged": _relmax(rm["D"], ex["D"])})
        S.set_tuning(solver, g, k, precision=S.MIXED)
        print(json.dumps(row), flush=True)


def per_iteration(name, kern):
    """Launches of a timed kernel per iteration: the mixed CG's second sweep
    alternates between cg_b (odd iterations) and cg_bx (even ones)."""
    deferred = any(k[0].startswith("cg_bx") for k in kern)
    return 0.5 if deferred and name.startswith("cg_b") else 1.0


def traffic_per_launch(kernel, grid, lanes):
    """DRAM bytes per launch of `kernel` at this size, from the committed ncu
    summary (profiles/ncu_traffic.txt lines '<kernel> <n1>x<n2>x<n3> <lanes>
    <bytes per launch>'), scaled by point-lanes (traffic is proportional to
    the grid and the lanes)."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 4 and f[0] == kernel and not line.startswith("#"):
            try:
                g = [int(v) for v in f[1].split("x")]
                return float(f[3]) * (grid[0] * grid[1] * grid[2] * lanes) / (g[0] * g[1] * g[2] * int(f[2]))
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# The sedi_b200 arm.
# ---------------------------------------------------------------------------
def run_sedi(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import sedi_b200 as S
    from sedi_b200 import dist as sdist

    rank, world, local = dist_env()
    wl = args.wl
    aux = {"large512": run_large512, "accuracy": run_accuracy, "sweeps": run_sweeps, "slab": run_slab,
           "periods": run_periods}
    if args.workload in aux:
        if rank == 0:
            aux[args.workload](S, args)
        return
    if args.serve_only:
        if rank == 0:
            print(json.dumps({"serving": run_serving(S, args.serve_jobs)}), flush=True)
        return
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    GRID, SAMPLES, TOL, MAXITER = wl["grid"], wl["samples"], wl["tol"], wl["maxiter"]
    solver, form = wl["solver"], wl["form"]
    dev = torch.device("cuda", torch.cuda.current_device())
    n = GRID[0] * GRID[1] * GRID[2]
    stream = torch.cuda.current_stream()
    prec = S.MIXED if form == "mixed" else S.FP64
    batch = 1 if form == "plain" else SAMPLES
    peak, peak_src = _peak()

    # This rank's probes (seeds SEED + rank*SAMPLES + k), generated on the
    # device with the reference's generator: resident for `value`, copied
    # once to pinned host memory for `e2e`.
    probes = torch.empty((SAMPLES, n), dtype=torch.float64, device=dev)
    S.fill_probes_dev(SEED + rank * SAMPLES, probes, stream)
    D = torch.empty(n, dtype=torch.float64, device=dev)
    t = torch.empty(n, dtype=torch.float64, device=dev)
    q = torch.empty(n, dtype=torch.float64, device=dev)
    # Launch choices for this shape, measured before the timed region (lane
    # slice width and i3 split from the sweeps' own timing).
    tuned = None
    if form != "plain" and not args.no_extras:
        tuned = S.autotune(solver, GRID, SAMPLES, precision=prec, maxiter=MAXITER, tol=TOL, solve=False)
    ctx = S.Context(solver, GRID, precision=prec, batch=batch)
    ctx.set_stream(stream)

    def local_dev(solver_, dims, count, first_seed, maxiter, tol, precision, batch_, stencil):
        r = ctx.estimate_dev(count, probes, D, t, q, maxiter=maxiter, tol=tol)
        return dict(r, t=t, q=q)

    def step():
        return sdist.estimate_sharded(solver, GRID, SAMPLES * world, seed=SEED, maxiter=MAXITER, tol=TOL,
                                      precision=prec, batch=batch, device=dev, local_estimate=local_dev)

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
    Dcur = res["D"].cpu().numpy() if rank == 0 else None
    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "ms_per_step": ms / args.steps, "grid": list(GRID), "samples": SAMPLES,
                              "maxiter": MAXITER, "tol": TOL, "solver": solver, "form": form,
                              "gpu_launches": launches, "note": "profiling case, not the benchmark configuration"}),
                  flush=True)
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # End to end through the C ABI: pinned host probes in, host D out, per step.
    host = torch.empty((SAMPLES, n), dtype=torch.float64).pin_memory()
    host.copy_(probes)
    hv = host.numpy()

    def local_host(solver_, dims, count, first_seed, maxiter, tol, precision, batch_, stencil):
        return ctx.estimate(count, probes=hv, maxiter=maxiter, tol=tol)

    e2e_steps = max(1, min(args.e2e_steps, args.steps))
    barrier()
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        rr = sdist.estimate_sharded(solver, GRID, SAMPLES * world, seed=SEED, maxiter=MAXITER, tol=TOL,
                                    precision=prec, batch=batch, device=dev, local_estimate=local_host)
        Dh = rr["D"].cpu().numpy()
    barrier()
    e2e_s = torch.tensor([time.perf_counter() - w0], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_val = world * SAMPLES * e2e_steps / float(e2e_s.item())
    del host, hv

    out = None
    if rank == 0:
        # Roofline of the dominant per-iteration sweep (each sweep timed alone,
        # CUDA events on the launching stream), and of the whole iteration
        # against the compulsory bytes of CG (x, r, p read and written).
        kern = ctx.time_kernels(reps=10) if form != "plain" else []
        ctx_config = ctx.config() if form != "plain" else None
        theta = ctx.mixed_target if form == "mixed" else None
        roofline = None
        if kern:
            dom = max(kern, key=lambda k: k[1])
            ach = dom[2] / (dom[1] * 1e-3) / 1e9
            it_ms = sum(k[1] * per_iteration(k[0], kern) for k in kern)
            it_bytes = CG_BYTES[form] * n * SAMPLES
            roofline = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": peak, "unit": "GB/s",
                        "frac": ach / peak, "peak_source": peak_src,
                        "traffic": traffic_per_launch(dom[0], GRID, SAMPLES),
                        "bytes_per_launch": dom[2], "ms_per_launch": dom[1],
                        "kernels": [{"kernel": k[0], "ms": k[1], "bytes": k[2], "GB/s": k[2] / k[1] / 1e6,
                                     "frac": k[2] / k[1] / 1e6 / peak} for k in kern],
                        "iteration": {"ms": it_ms, "compulsory_bytes": it_bytes,
                                      "basis": f"{CG_BYTES[form]} B per point-lane (x, r, p read and written)",
                                      "GB/s": it_bytes / it_ms / 1e6, "frac": it_bytes / it_ms / 1e6 / peak}}
        ctx.close()
        acc = {}
        forms = {}
        if world == 1 and form == "mixed":
            # The FP64 batched form on the same probes (two halves of the lanes:
            # t and q add up exactly), and the plain single-vector FP64 form.
            half = SAMPLES // 2
            with S.Context(solver, GRID, precision=S.FP64, batch=half) as c64:
                c64.set_stream(stream)
                t64 = torch.zeros(n, dtype=torch.float64, device=dev)
                q64 = torch.zeros(n, dtype=torch.float64, device=dev)
                D64 = torch.empty(n, dtype=torch.float64, device=dev)
                torch.cuda.synchronize()
                a = time.perf_counter()
                for h in range(2):
                    c64.estimate_dev(half, probes[h * half:(h + 1) * half], D64, t, q, maxiter=MAXITER, tol=TOL)
                    t64 += t
                    q64 += q
                torch.cuda.synchronize()
                forms["batched_fp64"] = SAMPLES / (time.perf_counter() - a)
            d64 = (t64 / q64).cpu().numpy()
            acc["D_rel_err_vs_batched_fp64"] = _relmax(Dcur, d64)
            acc["tolerance"] = 1e-8
            acc["mixed_target_theta"] = theta
            del t64, q64, D64
            with S.Context(solver, GRID) as cp:
                cp.set_stream(stream)
                kp = 2
                cp.estimate_dev(1, probes, D, maxiter=MAXITER, tol=TOL)
                torch.cuda.synchronize()
                a = time.perf_counter()
                rp = cp.estimate_dev(kp, probes, D, maxiter=MAXITER, tol=TOL)
                torch.cuda.synchronize()
                forms["plain_fp64_single_vector"] = kp / (time.perf_counter() - a)
                forms["plain_fp64_iterations"] = [int(v) for v in rp["iters"]]
                try:  # the single-vector form's streaming sweeps (n1 even), timed alone
                    forms["plain_fp64_kernels"] = [{"kernel": k, "ms": ms_, "GB/s": by / ms_ / 1e6,
                                                    "frac": by / ms_ / 1e6 / peak}
                                                   for k, ms_, by in cp.time_kernels(reps=5)]
                except S.SediError:
                    pass
            forms["mixed_vs_plain_fp64"] = value / forms["plain_fp64_single_vector"]
            forms["mixed_vs_batched_fp64"] = value / forms["batched_fp64"]
            # The reference's own converged run of probes 0..7 on this grid.
            if tuple(GRID) == (256, 256, 256) and os.path.exists(BIG_FIXTURE):
                z = np.load(BIG_FIXTURE)
                kz = len(z["iters"])
                acc["iters_probes_0_7_mixed"] = [int(v) for v in iters[-1][:kz]]
                acc["iters_probes_0_7_reference"] = [int(v) for v in z["iters"]]
                acc["iters_probes_0_7_plain_fp64_first2_equal_reference"] = bool(
                    np.array_equal(rp["iters"], z["iters"][:kp]))
        del probes
        torch.cuda.empty_cache()
        dropin = dropin_forms(S, stream) if world == 1 and tuple(GRID) == (256, 256, 256) else None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            procs = host_cores()
            rb = reference_baseline(procs, SEED, GRID, args.ref_iters, TOL, n)
            cpu = {"value": rb["value"], "unit": UNIT, "cores": procs, "kind": rb["kind"], "extrapolated": True,
                   "sample": f"{procs} concurrent single-rank processes x 1 probe x {args.ref_iters} iterations "
                             f"({'x'.join(map(str, GRID))} CG, -p 1x1x1, {rb['wall_s']:.1f} s), extrapolated per "
                             f"probe to {rb['converged_iterations']:.1f} iterations ({rb['converged_source']})",
                   "gpoint_iterations_per_s": rb["gpoint_iterations_per_s"], "effective_gbs": rb["effective_gbs"],
                   "timers_s_per_process": rb["timers_s_per_process"]}
        serving = run_serving(S, args.serve_jobs) if world == 1 and args.serve_jobs > 0 else None
        gpoint = float(np.sum(it_all)) * n / (ms / 1e3) / 1e9 * world
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": DTYPES[form],
            "data": "synthetic",
            "config": {"workload": wl["text"], "grid": list(GRID), "probes_per_gpu": SAMPLES, "solver": solver,
                       "tol": TOL, "form": form, "parallelism": f"probe-sharded x{world}",
                       "autotuned": tuned, "launch": ctx_config,
                       "l2": f"inputs larger than L2 ({SAMPLES * n * 8 / 1e9:.1f} GB probes + Krylov state per GPU)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "steps": e2e_steps, "h2d_bytes_per_step": SAMPLES * n * 8,
                    "d2h_bytes_per_step": n * 8 * 3 + SAMPLES * 16},
            "clocks": clk,
            "gpu_launches": launches,
            "iterations": [int(it_all.min()), int(it_all.max())],
            "gpoint_iterations_per_s": gpoint,
            "accuracy": acc,
            "forms": forms,
            "dropin_128": dropin,
            "serving": serving,
        }
    else:
        ctx.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
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
