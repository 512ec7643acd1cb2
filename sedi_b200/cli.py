"""Decomposed-grid command-line driver: ``-p 1x1xP`` over P GPUs.

    torchrun --nproc-per-node P -m sedi_b200.cli -g N1xN2xN3 -p 1x1xP [-s S] [-e TOL] [-m MAXITER] [-i] [-f MODE]
                                                 [--solver cg|pcg|bicgstab]
    python -m sedi_b200.cli -g ... -p 1x1xP --loopback      # P slabs in one process on one GPU

The counterpart of ``mpirun -n P stochastic-estimator.cg.exe -g ... -p ...``
(README.md:74-82) for slab decompositions along i3: the options and printed
lines are the reference's (CmdLineParser.hpp:43-136, stochastic-estimator.cc,
DomainDecomposition.hpp:43-48, Cg.hpp:192, PipelinedCg.hpp:228,
BiCgStab.hpp:228, Timers.hpp:57-70) and the solver is the reference's CG,
pipelined CG or BiCGStab in FP64 (sedi_b200.domain; the reference picks it at
compile time, here --solver, default cg).  Probe k is the global
std::mt19937(seed + k) probe (--seed, default 1234).  The one-GPU driver with
every solver and precision is the ``sedi`` binary (-p 1x1x1).
"""
import argparse
import os
import sys
import time

import numpy as np


def parse(argv=None):
    ap = argparse.ArgumentParser(prog="sedi_b200.cli", add_help=True)
    ap.add_argument("-g", required=True, help="size of the global 3D grid, NxNxN")
    ap.add_argument("-p", required=True, help="decomposition into ranks, 1x1xP (slabs along i3)")
    ap.add_argument("-s", type=int, default=400, help="number of samples for stochastic estimation")
    ap.add_argument("-e", type=float, default=1e-4, help="solver tolerance")
    ap.add_argument("-m", type=int, default=1000, help="solver maximum iterations")
    ap.add_argument("-i", action="store_true", help="ignore solver convergence errors and keep going")
    ap.add_argument("-f", type=int, default=0, help="solver operation mode bits (Cg::mode_t)")
    ap.add_argument("-F", action="store_true", help="accepted; the GPU does not trap floating-point exceptions")
    ap.add_argument("--solver", default="cg", choices=["cg", "pcg", "pipelined_cg", "bicgstab"])
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--quiet", action="store_true", help="no per-iteration lines")
    ap.add_argument("--loopback", action="store_true", help="all slabs in this process, on one GPU")
    ap.add_argument("--write-d", default=None, help="write D (raw doubles, i1 fastest) from rank 0")
    a = ap.parse_args(argv)
    try:
        a.dims = tuple(int(v) for v in a.g.lower().split("x"))
        if len(a.dims) != 3 or min(a.dims) < 1:
            raise ValueError
    except ValueError:
        ap.error(f"-g {a.g}: expected N1xN2xN3")
    from sedi_b200.domain import parse_decomposition
    try:
        a.parts = parse_decomposition(a.p, a.dims[2])
    except ValueError as e:
        ap.error(str(e))
    if a.f & ~3:
        ap.error("-f: mode bits 0..3")
    return a


def main(argv=None):
    a = parse(argv)
    import torch
    import torch.distributed as dist
    from sedi_b200.domain import slab_solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    distributed = world > 1 and not a.loopback
    if distributed:
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    elif a.parts > 1 and not a.loopback:
        print(f"sedi_b200.cli: -p {a.p} needs {a.parts} ranks (torchrun --nproc-per-node {a.parts}) or --loopback",
              file=sys.stderr)
        return 1
    cg = slab_solver(a.solver, a.dims, a.parts, loopback=not distributed, mode=a.f)
    rank0 = cg.rank == 0
    out = (lambda *x: print(*x, flush=True)) if rank0 else (lambda *x: None)
    n1, n2, n3 = a.dims
    out(f"Global grid shape is ({n1}, {n2}, {n3})")
    out(f"Domain decomposition across {a.parts} MPI ranks")
    out(f"Processor decomposition is (1, 1, {a.parts})")
    out(f"Process block shape is ({n1}, {n2}, {cg.ranges[0][1]})")
    out(f"Initialized {cg.NAME} solver, sync_dotprod={int(bool(a.f & 2))}, sync_stencil={int(bool(a.f & 1))}")

    x, b, t, q = cg.zeros(), cg.zeros(), cg.zeros(), cg.zeros()
    work = cg.work()
    plane = n1 * n2
    iters = []
    t_rng = 0.0
    t0 = time.perf_counter()
    for k in range(a.s):
        out(f"Solving for sample {k + 1}/{a.s}...")
        r0 = time.perf_counter()
        for j, s in enumerate(cg.local):
            cg.backend.fill_probe(b[j], a.seed + k, cg.ranges[s][0] * plane)
            x[j].zero_()
        t_rng += time.perf_counter() - r0
        res, err, it = cg.solve(x, b, a.m, a.e, work)
        if not a.quiet:
            for i, e in enumerate(cg.last_history[1:], 1):
                out(f"{cg.NAME}: after iter={i}, err={e:.10e}")
        for j in range(len(cg.local)):
            cg.backend.accumulate(x[j], b[j], t[j], q[j], k == 0)
        iters.append(it)
        if res != 0 and not a.i:  # stochastic-estimator.cc:181-184
            print(f"Incomplete convergence in solver, errcode={res}", file=sys.stderr, flush=True)
            if distributed:
                dist.destroy_process_group()
            return 100 + res
    D = cg.zeros()
    if a.s > 0:
        for j in range(len(cg.local)):
            cg.backend.divide(t[j], q[j], D[j])
    torch.cuda.synchronize()
    total = time.perf_counter() - t0
    Dg = cg.gather(D)
    out(f"Total solve time: {total:.4e} seconds, iteration count min={min(iters, default=0)} "
        f"max={max(iters, default=0)}")
    out("===========================================")
    tm = cg.timers
    rows = [("TIMER_GLOBAL", total), ("TIMER_COMPUTE_STENCIL_INNER", total - t_rng - tm["halo_wait"] - tm["dot_comm"]),
            ("TIMER_COMPUTE_STENCIL_BORDER", 0.0), ("TIMER_COMPUTE_DOTPROD", 0.0), ("TIMER_COMPUTE_RNG", t_rng),
            ("TIMER_COMPUTE_MISC", 0.0), ("TIMER_HALO_PACK", 0.0), ("TIMER_HALO_ISEND_IRECV", 0.0),
            ("TIMER_HALO_UNPACK_WAIT", tm["halo_wait"]), ("TIMER_COMM_DOTPROD", tm["dot_comm"])]
    for name, v in rows:
        out(f"{name:<28} = {v:.4e} s")
    out("===========================================")
    free, total_mem = torch.cuda.mem_get_info()
    out(f"Device memory [MB]: used={(total_mem - free) / 2 ** 20:.3e}, total={total_mem / 2 ** 20:.3e}")
    if rank0 and a.write_d:
        np.asarray(Dg, np.float64).tofile(a.write_d)
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
