"""Slab (i3) domain decomposition of the three solvers on CPU ranks (gloo), -p 1x1xP.

The host logic of sedi_b200.domain -- halo exchange between ranks, the
plane-ordered dot reduction, the CG, pipelined CG and BiCGStab loops and the
estimator -- runs with the NumPy stand-in for the slab kernels.  A run split
over 2 or 3 ranks (or several slabs in one process) must give the
single-slab result bit for bit, and that result matches the oracle's solver
(the reference method): same iteration counts and results, D to 1e-12
(BiCGStab 1e-9).
"""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import _oracle as O
import sedi_b200 as S
from sedi_b200.domain import SlabCg, parse_decomposition, slab_range, slab_solver
from _slab_numpy import NumpySlabBackend

DIMS = (9, 8, 7)
SOLVERS = {"cg": 2, "pcg": 3, "bicgstab": 1}  # the oracle's solver ids


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run(parts, dims, samples, loopback=False, stencil=None, mode=0, solver="cg", maxiter=300, tol=1e-10):
    sv = slab_solver(solver, dims, parts, stencil=stencil, backend=NumpySlabBackend(dims, stencil), loopback=loopback,
                     mode=mode)
    r = sv.estimate(samples, 1234, maxiter, tol)
    return dict(D=sv.gather(r["D"]), iters=r["iters"], errs=r["errs"], results=r["results"])


def _worker(rank, world, port, out_dir, dims, samples, mode, solver):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r = _run(world, dims, samples, mode=mode, solver=solver)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), **r)
    dist.barrier()
    dist.destroy_process_group()


def test_slab_ranges_and_decomposition_argument():
    for n3 in (1, 7, 64):
        for parts in range(1, min(n3, 5) + 1):
            spans = [slab_range(n3, parts, s) for s in range(parts)]
            assert [k for f, c in spans for k in range(f, f + c)] == list(range(n3))
            assert min(c for _, c in spans) >= 1
    assert parse_decomposition("1x1x4", 8) == 4
    for bad in ("2x1x1", "1x2x2", "1x1x9", "1x1", "axbxc", "1x1x0"):
        with pytest.raises(ValueError):
            parse_decomposition(bad, 8)


def test_probe_range_is_a_slice_of_the_global_probe():
    n = 5000
    full = S.fill_probe(77, n)
    for off, cnt in ((0, 10), (1, 1), (1234, 999), (4000, 1000)):
        part = np.empty(cnt)
        S.load().sedi_fill_probe_range(77, off, cnt, part.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(part, full[off:off + cnt])


@pytest.mark.parametrize("solver", list(SOLVERS))
def test_one_slab_matches_the_oracle(solver):
    one = _run(1, DIMS, 3, solver=solver)
    ref = O.estimate(SOLVERS[solver], DIMS, 3, 1234, 300, 1e-10)
    assert np.array_equal(one["results"], ref["results"])
    assert np.array_equal(one["iters"], ref["iters"])
    # BiCGStab amplifies the different order of the dot sums (per plane here,
    # sequential in the oracle) more than the CG forms.
    assert O.relmax(one["D"], ref["D"]) <= (1e-9 if solver == "bicgstab" else 1e-12)
    if solver == "bicgstab":  # its last residual is a cancellation: compare with the tolerance only
        assert np.all(one["errs"] <= 1e-10) and np.all(ref["errs"] <= 1e-10)
    else:
        assert np.allclose(one["errs"], ref["errs"], rtol=1e-6, atol=1e-14)  # errs near 1e-10: rounding-level


@pytest.mark.parametrize("solver", list(SOLVERS))
@pytest.mark.parametrize("parts", [2, 3, 7])
def test_slabs_in_one_process_are_bit_exact(parts, solver):
    one = _run(1, DIMS, 3, solver=solver)
    many = _run(parts, DIMS, 3, loopback=True, solver=solver)
    assert np.array_equal(many["D"], one["D"])
    assert np.array_equal(many["iters"], one["iters"]) and np.array_equal(many["errs"], one["errs"])


@pytest.mark.parametrize("solver", ["pcg", "bicgstab"])
def test_solver_edge_cases_follow_the_oracle(solver):
    """maxiter reached, maxiter 0, a zero right-hand side."""
    sid = SOLVERS[solver]
    for maxiter, tol in ((4, 1e-14), (0, 1e-14)):
        one = _run(2, DIMS, 2, loopback=True, solver=solver, maxiter=maxiter, tol=tol)
        ref = O.estimate(sid, DIMS, 2, 1234, maxiter, tol)
        assert np.array_equal(one["results"], ref["results"]), (maxiter, one["results"], ref["results"])
        assert np.array_equal(one["iters"], ref["iters"])
        assert np.allclose(one["errs"], ref["errs"], rtol=1e-9, atol=0)
        assert O.relmax(one["D"], ref["D"]) <= 1e-11
    sv = slab_solver(solver, DIMS, 3, backend=NumpySlabBackend(DIMS), loopback=True)
    x, b = sv.zeros(), sv.zeros()
    assert sv.solve(x, b, 50, 1e-10) == (0, 0.0, 0)


@pytest.mark.parametrize("world,mode,solver", [(2, 0, "cg"), (3, 0, "cg"), (2, 1, "cg"), (3, 0, "pcg"),
                                               (2, 1, "bicgstab"), (3, 0, "bicgstab")])
def test_ranks_are_bit_exact(tmp_path, world, mode, solver):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path), DIMS, 3, mode, solver), nprocs=world,
                       start_method="spawn")
    one = _run(1, DIMS, 3, solver=solver)
    for rank in range(world):
        r = np.load(tmp_path / f"r{rank}.npz")
        assert np.array_equal(r["D"], one["D"])
        assert np.array_equal(r["iters"], one["iters"]) and np.array_equal(r["errs"], one["errs"])


def test_nonsymmetric_stencil_and_apply():
    st = S.Stencil(6.0, 1.3, 0.7)
    dims = (6, 5, 8)
    x_full = np.random.default_rng(3).standard_normal(int(np.prod(dims)))
    outs = []
    for parts in (1, 3):
        cg = SlabCg(dims, parts, stencil=st, backend=NumpySlabBackend(dims, st), loopback=True)
        xs, ys = cg.zeros(), cg.zeros()
        plane = dims[0] * dims[1]
        for j, s in enumerate(cg.local):
            f, c = cg.ranges[s]
            cg.backend.set_interior(xs[j], x_full[f * plane:(f + c) * plane])
        cg.apply(xs, ys)
        outs.append(cg.gather(ys))
    assert np.array_equal(outs[0], outs[1])
    ref = O.stencil(dims, x_full, (6.0, 1.3, 0.7))
    assert np.array_equal(outs[0], ref)


def test_decomposed_cli_rejects_bad_arguments_before_device_use():
    import subprocess
    import sys
    for args in (["-g", "8x8x8", "-p", "2x1x1"], ["-g", "8x8x8", "-p", "1x1x9"], ["-g", "8x8", "-p", "1x1x1"],
                 ["-g", "8x8x8", "-p", "1x1x2", "-f", "8"], ["-p", "1x1x1"],
                 ["-g", "8x8x8", "-p", "1x1x1", "--solver", "gmres"]):
        r = subprocess.run([sys.executable, "-m", "sedi_b200.cli"] + args, capture_output=True, text=True, timeout=120,
                           cwd=O.REPO)
        assert r.returncode == 2, (args, r.stderr)
    # -p 1x1x2 without torchrun ranks or --loopback is refused.
    r = subprocess.run([sys.executable, "-m", "sedi_b200.cli", "-g", "8x8x8", "-p", "1x1x2"], capture_output=True,
                       text=True, timeout=120, cwd=O.REPO)
    assert r.returncode == 1 and "--loopback" in r.stderr
