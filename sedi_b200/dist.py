"""Probe-sharded estimation across GPUs (one process per GPU).

The reference parallelises over space (MPI domain decomposition + halo
exchange, CommHalo.hpp) and runs its probes one after another
(stochastic-estimator.cc:158).  Probes are independent, so here each rank
estimates its own contiguous range of probes -- probe k still uses
std::mt19937(seed + k) -- and the per-point accumulators t = sum x.*v and
q = sum v.*v (stochastic-estimator.cc:195, :198) are summed across ranks with
one all-reduce per estimate; D = t ./ q (:216).  No collective runs inside
the solves.

``estimate_sharded`` is the one implementation: the benchmark's multi-GPU
step calls it with the NCCL group and a per-rank estimate on a resident
context, the CPU tests call it with gloo ranks.
"""
import numpy as np

__all__ = ["probe_range", "estimate_sharded", "reduce_accumulators"]


def probe_range(samples, world, rank):
    """Contiguous probe range [first, first+count) of `rank` among `world` ranks."""
    base, extra = divmod(int(samples), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _gpu_local_estimate(solver, dims, count, seed, maxiter, tol, precision, batch, stencil):
    import sedi_b200 as S
    with S.Context(solver, dims, stencil, 0, precision, max(1, min(batch, max(count, 1)))) as ctx:
        return ctx.estimate(count, seed, maxiter, tol, ignore_errors=True)


def _world_rank(group):
    import torch.distributed as dist
    if not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def reduce_accumulators(t, q, group=None):
    """Sum the ranks' t and q (torch tensors, in place) and return D = t ./ q
    (stochastic-estimator.cc:195-216): the only collective of an estimate."""
    import torch
    import torch.distributed as dist
    world, _ = _world_rank(group)
    if world > 1:
        dist.all_reduce(t, group=group)
        dist.all_reduce(q, group=group)
    return torch.div(t, q)


def estimate_sharded(solver, dims, samples, seed=1234, maxiter=1000, tol=1e-4, precision=0, batch=1, stencil=None,
                     group=None, device=None, local_estimate=None):
    """Estimate D over `samples` probes split across the ranks of `group`.

    Every rank calls this with the same arguments.  Rank r estimates probes
    [first, first+count) of probe_range(samples, world, r), i.e. seeds
    seed+first ...  `local_estimate` replaces the per-rank GPU estimate on a
    fresh context (the benchmark passes one on its resident context, the CPU
    tests the oracle); it receives (solver, dims, count, first_seed, maxiter,
    tol, precision, batch, stencil) and returns a dict with t, q (numpy
    arrays or torch tensors), iters, errs, results.

    Returns dict(D, t, q, iters, errs, results): D, t, q are torch tensors on
    `device` (default: the device of the local t, else the CPU), summed over
    the ranks; the per-probe arrays (numpy) are gathered in probe order on
    every rank.
    """
    import torch
    import torch.distributed as dist

    world, rank = _world_rank(group)
    first, count = probe_range(samples, world, rank)
    fn = local_estimate or _gpu_local_estimate
    n = int(np.prod(dims))
    if count > 0:
        r = fn(solver, dims, count, seed + first, maxiter, tol, precision, batch, stencil)
        t, q = r["t"], r["q"]
        meta = np.stack([np.asarray(r["iters"], np.float64), np.asarray(r["errs"], np.float64),
                         np.asarray(r["results"], np.float64)], 1)
    else:
        t = q = None
        meta = np.zeros((0, 3))
    if device is None:
        device = t.device if isinstance(t, torch.Tensor) else torch.device("cpu")

    def as_tensor(a):
        if a is None:
            return torch.zeros(n, dtype=torch.float64, device=device)
        if isinstance(a, torch.Tensor):
            return a.to(device=device, dtype=torch.float64)
        return torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(device)

    t, q = as_tensor(t), as_tensor(q)
    D = reduce_accumulators(t, q, group)
    per = np.zeros((samples, 3))
    per[first:first + count] = meta
    pt = torch.from_numpy(per).to(device)
    if world > 1:
        dist.all_reduce(pt, group=group)
    per = pt.cpu().numpy()
    return dict(D=D, t=t, q=q, iters=per[:, 0].astype(np.int32), errs=per[:, 1], results=per[:, 2].astype(np.int32))
