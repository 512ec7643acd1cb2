"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference SEDI sources compiled as ``oracle/_ref/ref_driver`` (the
unmodified reference headers plus single-rank MPI / raw-HDF5 / seeded
random_device stand-ins; build with ``make -C oracle ref``).  Needs the
reference checkout, so it only runs where that exists; the fixtures it writes
are committed and travel with the tests.

Probe k of a run with seed S is std::mt19937(S + k) -> uniform_real(0,1) ->
(x > 0.5 ? +1 : -1), the reference's own DistrRngStd code (DistrRngStd.hpp).

Usage:  python tests/golden/make_golden.py [--full | --big]
  --big  runs only the 256^3 CG configuration for 8 probes (one single-rank
         process per probe) and stores its iteration counts, solve seconds
         and a strided sample + checksums of D.
  --full also runs the 128^3 x 64-probe drop-in configuration for each solver
         (several CPU minutes, run as 8 parallel single-rank processes over
         disjoint probe ranges, t and q summed) and stores iteration counts,
         errors and a strided sample + checksums of D.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(REPO, "oracle", "_ref", "ref_driver")
SOLVERS = {1: "bicgstab", 2: "cg", 3: "pcg"}


def run_ref(solver, grid, samples, tol, maxiter, seed=1234, coeffs=(6.0, 1.0, 1.0), dump_vx=False, mode=0):
    with tempfile.TemporaryDirectory() as d:
        cmd = [DRIVER, "-g", "x".join(map(str, grid)), "-S", str(solver), "-s", str(samples),
               "-e", repr(tol), "-m", str(maxiter), "-a", ",".join(repr(c) for c in coeffs), "-f", str(mode),
               "-q", "-o", d]
        if dump_vx:
            cmd.append("-x")
        env = dict(os.environ, SEDI_SEED=str(seed))
        subprocess.check_call(cmd, env=env)
        out = {
            "D": np.fromfile(os.path.join(d, "D.f64")),
            "t": np.fromfile(os.path.join(d, "t.f64")),
            "q": np.fromfile(os.path.join(d, "q.f64")),
            "iters": np.fromfile(os.path.join(d, "iters.i32"), np.int32),
            "errs": np.fromfile(os.path.join(d, "errs.f64")),
            "results": np.fromfile(os.path.join(d, "results.i32"), np.int32),
            "seconds": float(open(os.path.join(d, "time.txt")).read()),
        }
        if dump_vx:
            out["v"] = np.fromfile(os.path.join(d, "v.f64"))
            out["x"] = np.fromfile(os.path.join(d, "x.f64"))
        return out


def save(name, meta, arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, meta=np.array(repr(meta)), **arrays)
    print("wrote", path, os.path.getsize(path), "bytes", meta)


def case(name, solver, grid, samples, tol, maxiter, coeffs=(6.0, 1.0, 1.0), keep_x=False, seed=1234, mode=0):
    r = run_ref(solver, grid, samples, tol, maxiter, seed=seed, coeffs=coeffs, dump_vx=keep_x, mode=mode)
    meta = dict(solver=solver, grid=tuple(grid), samples=samples, tol=tol, maxiter=maxiter,
                coeffs=tuple(coeffs), seed=seed, mode=mode)
    arrays = {k: r[k] for k in ("D", "t", "q", "iters", "errs", "results")}
    if keep_x:
        arrays["x"] = r["x"]
        arrays["v_bits"] = np.packbits(r["v"] > 0)
    save(name, meta, arrays)


def full_config(solver, procs=8, samples=64, grid=(128, 128, 128), tol=1e-9, maxiter=5000):
    """Drop-in configuration: P single-rank processes over disjoint probe ranges."""
    per = samples // procs
    tmp = tempfile.mkdtemp()
    jobs = []
    for j in range(procs):
        d = os.path.join(tmp, str(j))
        cmd = [DRIVER, "-g", "x".join(map(str, grid)), "-S", str(solver), "-s", str(per),
               "-e", repr(tol), "-m", str(maxiter), "-q", "-o", d]
        jobs.append((d, subprocess.Popen(cmd, env=dict(os.environ, SEDI_SEED=str(1234 + j * per)))))
    t = q = None
    iters, errs, results = [], [], []
    for d, p in jobs:
        if p.wait() != 0:
            raise SystemExit("ref_driver failed")
        tj = np.fromfile(os.path.join(d, "t.f64"))
        qj = np.fromfile(os.path.join(d, "q.f64"))
        t = tj if t is None else t + tj
        q = qj if q is None else q + qj
        iters.append(np.fromfile(os.path.join(d, "iters.i32"), np.int32))
        errs.append(np.fromfile(os.path.join(d, "errs.f64")))
        results.append(np.fromfile(os.path.join(d, "results.i32"), np.int32))
    D = t / q
    stride = 1009
    meta = dict(solver=solver, grid=grid, samples=samples, tol=tol, maxiter=maxiter, coeffs=(6.0, 1.0, 1.0),
                seed=1234, procs=procs, sample_stride=stride)
    save(f"full_{SOLVERS[solver]}_128", meta, dict(
        iters=np.concatenate(iters), errs=np.concatenate(errs), results=np.concatenate(results),
        D_sample=D[::stride], D_sum=np.array(D.sum()), D_sumsq=np.array((D * D).sum()),
        D_min=np.array(D.min()), D_max=np.array(D.max())))


def big_config(solver=2, procs=8, grid=(256, 256, 256), tol=1e-9, maxiter=20000):
    """The 256^3 batched configuration's grid: `procs` single-rank processes,
    one probe each (seeds 1234..1234+procs-1), solved to tol.  Stores the
    reference's per-probe iteration counts, errors and per-process solve
    seconds, a strided sample and checksums of D over those probes."""
    tmp = tempfile.mkdtemp()
    jobs = []
    for j in range(procs):
        d = os.path.join(tmp, str(j))
        cmd = [DRIVER, "-g", "x".join(map(str, grid)), "-S", str(solver), "-s", "1",
               "-e", repr(tol), "-m", str(maxiter), "-q", "-o", d]
        jobs.append((d, subprocess.Popen(cmd, env=dict(os.environ, SEDI_SEED=str(1234 + j)))))
    t = q = None
    iters, errs, results, secs = [], [], [], []
    for d, p in jobs:
        if p.wait() != 0:
            raise SystemExit("ref_driver failed")
        tj = np.fromfile(os.path.join(d, "t.f64"))
        qj = np.fromfile(os.path.join(d, "q.f64"))
        t = tj if t is None else t + tj
        q = qj if q is None else q + qj
        iters.append(np.fromfile(os.path.join(d, "iters.i32"), np.int32))
        errs.append(np.fromfile(os.path.join(d, "errs.f64")))
        results.append(np.fromfile(os.path.join(d, "results.i32"), np.int32))
        secs.append(float(open(os.path.join(d, "time.txt")).read()))
    D = t / q
    stride = 4099
    meta = dict(solver=solver, grid=grid, samples=procs, tol=tol, maxiter=maxiter, coeffs=(6.0, 1.0, 1.0),
                seed=1234, procs=procs, sample_stride=stride)
    save(f"big_{SOLVERS[solver]}_256", meta, dict(
        iters=np.concatenate(iters), errs=np.concatenate(errs), results=np.concatenate(results),
        seconds=np.array(secs), D_sample=D[::stride], D_sum=np.array(D.sum()), D_sumsq=np.array((D * D).sum()),
        D_min=np.array(D.min()), D_max=np.array(D.max())))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--big", action="store_true",
                    help="only the 256^3 CG run of 8 probes (about 5 CPU minutes on 8 cores)")
    args = ap.parse_args()
    if not os.path.exists(DRIVER):
        raise SystemExit("build the reference oracle first: make -C oracle ref")
    if args.big:
        big_config()
        return

    # Probe generator pin: 5 probes of the 32^3 configuration, packed sign bits.
    r = run_ref(2, (32, 32, 32), 5, 1e-9, 1, dump_vx=True)
    save("probes_32", dict(grid=(32, 32, 32), samples=5, seed=1234), dict(v_bits=np.packbits(r["v"] > 0)))

    # The CPU-runnable configuration: CG, 32^3, 5 probes, tol 1e-9, maxiter 50, -i.
    case("cfg1_cg_32", 2, (32, 32, 32), 5, 1e-9, 50)
    # Same grid, fixed iteration counts, the other two solvers.  BiCGStab is
    # kept at 20 iterations: its rounding sensitivity grows ~2.4x per
    # iteration in the reference itself, so longer fixed horizons do not
    # define a 1e-10 answer.
    case("pcg_32_m50", 3, (32, 32, 32), 5, 1e-9, 50)
    case("bicgstab_32_m20", 1, (32, 32, 32), 5, 0.0, 20)
    # Converged solves on a non-cubic grid.
    for s in (1, 2, 3):
        case(f"conv_{SOLVERS[s]}_24x20x16", s, (24, 20, 16), 3, 1e-9, 1000)
    # Ragged / degenerate shapes, solutions kept.
    for s in (1, 2, 3):
        case(f"odd_{SOLVERS[s]}_5x7x9", s, (5, 7, 9), 3, 1e-12, 1000, keep_x=True)
        # Unit dimensions: the reference's asynchronous stencil path (mode 0)
        # splits the grid into inner cells and border slabs (Grid3d.hpp:54,
        # :79-91) that do not cover every cell when n1 or n2 is 1 (cells are
        # left at uninitialised values, or BlockSliceIterator.hpp:114
        # asserts).  Its synchronous stencil mode (-f 1) applies the whole
        # grid (DistrAsyncStencil.hpp:87-97) and is the reference answer here.
        for g in ((1, 1, 8), (1, 13, 1), (11, 1, 1), (1, 1, 1), (1, 5, 5), (5, 1, 5), (5, 5, 1)):
            case(f"line_{SOLVERS[s]}_" + "x".join(map(str, g)), s, g, 2, 1e-12, 100, keep_x=True, mode=1)
        for g in ((2, 2, 2), (2, 3, 4), (3, 3, 3), (2, 5, 7)):
            case(f"tiny_{SOLVERS[s]}_" + "x".join(map(str, g)), s, g, 2, 1e-12, 100, keep_x=True)
    # Non-symmetric operator (b != c) through BiCGStab; the reference Stencil
    # class is general (Stencil.hpp:12-19, :43-50).
    case("nonsym_bicgstab_12x10x8", 1, (12, 10, 8), 3, 1e-10, 1000, coeffs=(6.0, 1.3, 0.7), keep_x=True)
    # maxiter reached, result 1.
    case("maxiter_cg_16", 2, (16, 16, 16), 2, 1e-14, 7)
    if args.full:
        for s in (2, 3, 1):
            full_config(s)


if __name__ == "__main__":
    sys.exit(main())
