"""Estimation-job server (sedi_server_* through the C ABI).

Continuous admission: jobs of different grids, sample counts, tolerances,
solvers and precisions run concurrently on one GPU, each on its own stream
and context; the device-byte budget bounds what is admitted.  A job's result
does not depend on the mix: D, per-probe iterations, errors and codes are
bit-identical alone, in a mix, and through the direct estimator entry point
on a context of the same lane count (tolerance 0: every reduction runs in a
fixed order independent of other streams).
"""
import numpy as np
import pytest

import sedi_b200 as S

pytestmark = pytest.mark.gpu

JOB = ("cg", (40, 36, 32), 12, 77, 2000, 1e-9, S.MIXED)
MIX = [
    ("pcg", (48, 48, 48), 8, 1000, 3000, 1e-8, S.FP64),
    ("bicgstab", (32, 32, 32), 20, 2000, 3000, 1e-7, S.MIXED),
    ("cg", (64, 64, 64), 16, 3000, 3000, 1e-10, S.FP64),
    ("pcg", (24, 20, 16), 40, 4000, 3000, 1e-6, S.MIXED),
    ("bicgstab", (48, 32, 40), 9, 5000, 3000, 1e-9, S.FP64),
]


def _submit(srv, job):
    solver, dims, samples, seed, maxiter, tol, prec = job
    return srv.submit(solver, dims, samples, seed, maxiter, tol, precision=prec)


def _direct(job, lanes):
    solver, dims, samples, seed, maxiter, tol, prec = job
    with S.Context(solver, dims, precision=prec, batch=lanes) as c:
        return c.estimate(samples, seed, maxiter, tol, ignore_errors=True)


def _same(a, b):
    assert np.array_equal(a["D"], b["D"], equal_nan=True)
    assert np.array_equal(a["iters"], b["iters"]) and np.array_equal(a["results"], b["results"])
    assert np.array_equal(a["errs"], b["errs"])


def test_job_same_alone_in_mix_and_direct():
    with S.Server() as srv:
        j = _submit(srv, JOB)
        srv.wait(j)
        lanes = srv.info(j)["lanes"]
        alone = srv.take(j)
        ids = [_submit(srv, m) for m in MIX[:3]]
        j2 = _submit(srv, JOB)
        ids += [_submit(srv, m) for m in MIX[3:]]
        srv.wait()
        infos = {i: srv.info(i) for i in ids + [j2]}
        mixed = srv.take(j2)
        others = {i: srv.take(i) for i in ids}
        st = srv.stats()
    _same(alone, mixed)
    _same(alone, _direct(JOB, lanes))
    for i, m in zip(ids, MIX):
        assert infos[i]["state"] == "done"
        _same(others[i], _direct(m, infos[i]["lanes"]))
    assert st["max_running"] >= 2
    # Work of different jobs overlapped in time.
    spans = sorted((infos[i]["t_start"], infos[i]["t_done"]) for i in infos)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))


def test_budget_bounds_admission():
    dims, lanes = (64, 64, 64), 16
    one = S.job_bytes("cg", dims, lanes, S.FP64)
    with S.Server(budget_bytes=2.5 * one) as srv:
        ids = [srv.submit("cg", dims, lanes, 10 + k, 2000, 1e-8) for k in range(6)]
        srv.wait()
        st = srv.stats()
        res = [srv.take(i) for i in ids]
    assert st["peak_bytes"] <= st["budget_bytes"]
    assert st["max_running"] <= 2
    assert st["ctx_created"] <= 2 and st["ctx_reused"] >= 4
    assert all(r["rc"] == 0 for r in res)


def test_large_job_not_starved():
    big, small = (96, 96, 96), (32, 32, 32)
    bb = S.job_bytes("cg", big, 32, S.FP64)
    sb = S.job_bytes("cg", small, 8, S.FP64)
    assert bb > 3 * sb
    with S.Server(budget_bytes=bb + 0.5 * sb, max_active=8) as srv:
        first = [srv.submit("cg", small, 8, k, 2000, 1e-8) for k in range(2)]
        b = srv.submit("cg", big, 32, 99, 2000, 1e-8)
        later = [srv.submit("cg", small, 8, 100 + k, 2000, 1e-8) for k in range(10)]
        srv.wait()
        tb = srv.info(b)["t_start"]
        started_before = sum(srv.info(i)["t_start"] < tb for i in later)
        for i in first + [b] + later:
            assert srv.take(i)["rc"] == 0
    assert started_before <= 4


def test_replay_open_loop():
    rng = np.random.default_rng(5)
    k = 10
    arrival = np.cumsum(rng.exponential(0.01, k))
    solver = rng.choice(["cg", "pcg", "bicgstab"], k)
    prec = rng.integers(0, 2, k)
    edge = rng.choice([16, 24, 32], k)
    samples = rng.integers(2, 12, k)
    seed = np.arange(k) * 1000 + 1234
    tol = 10.0 ** rng.uniform(-10, -6, k)
    with S.Server() as srv:
        lat, rcs, mk = srv.replay(arrival, solver, prec, edge, samples, seed, tol, 3000)
        st = srv.stats()
    assert np.all(rcs == 0)
    assert np.all(lat > 0) and mk >= arrival[-1]
    assert st["launches"] > 0


def test_submit_rejects_what_cannot_fit():
    with S.Server(budget_bytes=64 << 20) as srv:
        with pytest.raises(S.SediError):
            srv.submit("cg", (256, 256, 256), 64, 1, 10, 1e-8)


def test_burst_of_fresh_contexts_matches_direct():
    """Many jobs submitted at once: every context is created while others
    already run on the GPU.  Each result must still equal the direct
    estimator's bit for bit (the contexts' zero-fills are ordered before
    their first kernels on their own streams)."""
    rng = np.random.default_rng(11)
    jobs = []
    for k in range(10):
        solver = ["cg", "pcg", "bicgstab"][k % 3]
        edge = int(rng.choice([24, 32, 40, 48]))
        jobs.append((solver, (edge, edge, edge), int(rng.integers(6, 40)), 500 + 37 * k, 3000,
                     float(10.0 ** rng.uniform(-10, -7)), S.MIXED if k % 2 else S.FP64))
    with S.Server(max_active=8) as srv:
        ids = [_submit(srv, j) for j in jobs]
        srv.wait()
        lanes = [srv.info(i)["lanes"] for i in ids]
        got = [srv.take(i) for i in ids]
    for j, l, g in zip(jobs, lanes, got):
        _same(g, _direct(j, l))


def test_contexts_reused_across_sample_counts_of_one_padded_lane_count():
    """Mixed jobs of 17, 20 and 30 probes on one grid all pad to 32 lanes: one
    context serves them one after another, and each result is bit-identical
    to the direct estimate on a context created for its own sample count."""
    jobs = [("cg", (40, 36, 32), k, 50 + k, 2000, 1e-9, S.MIXED) for k in (17, 20, 30)]
    with S.Server() as srv:
        got = []
        for job in jobs:
            j = _submit(srv, job)
            srv.wait(j)
            got.append(srv.take(j))
        st = srv.stats()
    assert st["ctx_created"] == 1 and st["ctx_reused"] == 2
    for job, g in zip(jobs, got):
        _same(g, _direct(job, job[2]))
