"""Probe-sharded estimation across GPUs (one process per GPU).

The reference parallelises over space (MPI domain decomposition + halo
exchange, CommHalo.hpp) and runs its probes one after another
(stochastic-estimator.cc:158).  Probes are independent, so here each rank
estimates its own contiguous range of probes -- probe k still uses
std::mt19937(seed + k) -- and the per-point accumulators t = sum x.*v and
q = sum v.*v (stochastic-estimator.cc:195, :198) are summed across ranks with
one all-reduce per estimate; D = t ./ q (:216).  No collective runs inside
the solves.
"""
import numpy as np

__all__ = ["probe_range", "estimate_sharded"]


def probe_range(samples, world, rank):
    """Contiguous probe range [first, first+count) of `rank` among `world` ranks."""
    base, extra = divmod(int(samples), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _gpu_local_estimate(solver, dims, count, seed, maxiter, tol, precision, batch, stencil):
    import sedi_b200 as S
    with S.Context(solver, dims, stencil, 0, precision, max(1, min(batch, max(count, 1)))) as ctx:
        return ctx.estimate(count, seed, maxiter, tol, ignore_errors=True)


def estimate_sharded(solver, dims, samples, seed=1234, maxiter=1000, tol=1e-4, precision=0, batch=1, stencil=None,
                     group=None, device=None, local_estimate=None):
    """Estimate D over `samples` probes split across the ranks of `group`.

    Every rank calls this with the same arguments.  `local_estimate` (for
    tests) replaces the per-rank GPU estimate; it receives (solver, dims,
    count, first_seed, maxiter, tol, precision, batch, stencil) and returns a
    dict with t, q, iters, errs, results.  Returns dict(D, t, q, iters, errs,
    results) with the per-probe arrays gathered in probe order on every rank.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    first, count = probe_range(samples, world, rank)
    fn = local_estimate or _gpu_local_estimate
    n = int(np.prod(dims))
    if count > 0:
        r = fn(solver, dims, count, seed + first, maxiter, tol, precision, batch, stencil)
        t_loc, q_loc = np.asarray(r["t"], np.float64), np.asarray(r["q"], np.float64)
        meta = np.stack([np.asarray(r["iters"], np.float64), np.asarray(r["errs"], np.float64),
                         np.asarray(r["results"], np.float64)], 1)
    else:
        t_loc, q_loc = np.zeros(n), np.zeros(n)
        meta = np.zeros((0, 3))
    dev = device if device is not None else torch.device("cpu")
    tq = torch.from_numpy(np.concatenate([t_loc, q_loc])).to(dev)
    per = np.zeros((samples, 3))
    per[first:first + count] = meta
    pt = torch.from_numpy(per).to(dev)
    if world > 1:
        dist.all_reduce(tq, group=group)
        dist.all_reduce(pt, group=group)
    tq = tq.cpu().numpy()
    per = pt.cpu().numpy()
    t, q = tq[:n], tq[n:]
    return dict(D=t / q, t=t, q=q, iters=per[:, 0].astype(np.int32), errs=per[:, 1],
                results=per[:, 2].astype(np.int32))
