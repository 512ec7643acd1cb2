"""Probe sharding across ranks (world size 2, gloo on CPU).

The per-rank solve is replaced by the CPU oracle (the GPU path is covered by
the GPU tests); what is checked here is the sharding itself: the probe ranges,
the seed of each probe, the all-reduce of t and q and the gathered per-probe
arrays, against one process estimating every probe.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import _oracle as O
from sedi_b200.dist import estimate_sharded, probe_range


def _oracle_local(solver, dims, count, seed, maxiter, tol, precision, batch, stencil):
    return O.estimate(solver, dims, count, seed, maxiter, tol)


def _oracle_local_tensors(solver, dims, count, seed, maxiter, tol, precision, batch, stencil):
    """As the benchmark's per-rank estimate: t and q come back as torch tensors
    (its device buffers), reduced in place."""
    import torch
    r = O.estimate(solver, dims, count, seed, maxiter, tol)
    return dict(r, t=torch.from_numpy(r["t"].copy()), q=torch.from_numpy(r["q"].copy()))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir, samples, tensors):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = _oracle_local_tensors if tensors else _oracle_local
    r = estimate_sharded(2, (9, 8, 7), samples, seed=1234, maxiter=300, tol=1e-10, local_estimate=local)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), **{k: (v.numpy() if hasattr(v, "numpy") and not
                                                            isinstance(v, np.ndarray) else v) for k, v in r.items()})
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("samples,tensors", [(6, False), (5, False), (1, False), (6, True)])
def test_two_ranks_match_one_process(tmp_path, samples, tensors):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path), samples, tensors), nprocs=2, start_method="spawn")
    full = O.estimate(2, (9, 8, 7), samples, 1234, 300, 1e-10)
    for rank in range(2):
        r = np.load(tmp_path / f"r{rank}.npz")
        assert O.relmax(r["D"], full["D"]) <= 1e-14
        assert np.array_equal(r["q"], full["q"])
        assert np.array_equal(r["iters"], full["iters"]) and np.array_equal(r["results"], full["results"])


def test_probe_ranges_partition():
    for samples in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            spans = [probe_range(samples, world, r) for r in range(world)]
            covered = [k for f, c in spans for k in range(f, f + c)]
            assert covered == list(range(samples))
