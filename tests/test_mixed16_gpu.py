"""CG with r and p stored in FP16 (SEDI_PREC_MIXED16).

Per lane the stored FP16 value times a power-of-two scale is the field; the
arithmetic is FP32 and every reduction, the reliable update and the stop test
are FP64, so each lane must meet tol on its FP64 true residual, and the
estimate must stay within 1e-8 (relative max-norm) of the FP64 form on the
same probes -- the bar of the mixed forms.
"""
import numpy as np
import pytest

import _oracle as O
import sedi_b200 as S

pytestmark = pytest.mark.gpu


def true_err(dims, x, b):
    r = b - O.stencil(dims, x)
    return np.sqrt((r @ r) / (b @ b))


@pytest.mark.parametrize("dims,nrhs,tol", [((24, 22, 20), 8, 1e-9), ((33, 17, 9), 16, 1e-10), ((64, 48, 40), 24, 1e-9)])
def test_mixed16_true_residual(dims, nrhs, tol):
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(51 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, precision=S.MIXED16, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=5000, tol=tol)
    assert np.all(res == 0)
    fi64 = O.solve(2, dims, B[0], maxiter=5000, tol=tol)[2]
    for k in range(nrhs):
        e = true_err(dims, X[k], B[k])
        assert e <= tol * 1.0000001, (k, e)
        assert abs(fe[k] - e) <= 1e-3 * e + 1e-16
    assert fi[0] <= fi64 * 1.5 + 20


@pytest.mark.parametrize("dims,samples", [((48, 48, 48), 32), ((128, 128, 128), 64)])
def test_mixed16_estimator_no_farther_from_converged_than_fp64(dims, samples):
    """FP16 rounding of r and p moves the iterates off the FP64 path (at
    theta = 1 the diagonal is 1e-8 .. 9e-8 from the FP64 form's); with its
    default in-loop target 0.1 the FP16 form's diagonal is nearer the
    converged one (FP64 CG to 1e-13 on the same probes) than the FP64
    form's at the same tol."""
    with S.Context("cg", dims, batch=samples) as cx:
        ex = cx.estimate(samples, 1234, 8000, 1e-13)
    with S.Context("cg", dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 1234, 5000, 1e-9)
    with S.Context("cg", dims, precision=S.MIXED16, batch=samples) as c:
        assert c.mixed_target == 0.1
        r = c.estimate(samples, 1234, 5000, 1e-9)
    assert np.all(r["results"] == 0)
    assert np.array_equal(r["q"], r64["q"])
    e16, e64 = O.relmax(r["D"], ex["D"]), O.relmax(r64["D"], ex["D"])
    assert e16 <= e64, (e16, e64)


def test_mixed16_edge_lanes_and_refusals():
    dims = (12, 10, 8)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(5, n), np.zeros(n), 1e-20 * O.fill_probe(6, n), 1e20 * O.fill_probe(7, n)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, precision=S.MIXED16, batch=4) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=2000, tol=1e-10)
    assert np.all(res == 0)
    assert (fi[1], fe[1]) == (0, 0.0) and np.all(X[1] == 0.0)
    for k in (0, 2, 3):  # scales follow the lane's own magnitude
        assert true_err(dims, X[k], B[k]) <= 1e-10 * 1.0000001, k
    with S.Context("cg", dims, precision=S.MIXED16, batch=4) as c:
        res, fe, fi = c.solve_batch(np.zeros_like(B[:1]), B[:1], maxiter=5, tol=1e-14)
    assert res[0] == 1 and fi[0] == 5
    for solver in ("pcg", "bicgstab"):
        with pytest.raises(S.SediError) as e:
            S.Context(solver, dims, precision=S.MIXED16, batch=8)
        assert e.value.code == -5


def test_mixed16_server_job_same_alone_and_direct():
    dims, samples = (32, 32, 32), 16
    with S.Context("cg", dims, precision=S.MIXED16, batch=samples) as c:
        direct = c.estimate(samples, 77, 3000, 1e-9)
    with S.Server() as srv:
        a = srv.submit("cg", dims, samples, 77, 3000, 1e-9, precision=S.MIXED16)
        b = srv.submit("pcg", (40, 40, 40), 8, 5, 3000, 1e-9, precision=S.MIXED)
        srv.wait()
        ra, rb = srv.take(a), srv.take(b)
    assert ra["rc"] == 0 and rb["rc"] == 0
    assert np.array_equal(ra["D"], direct["D"]) and np.array_equal(ra["iters"], direct["iters"])


def test_mixed16_kernel_timing_lists_both_sweeps():
    with S.Context("cg", (64, 64, 64), precision=S.MIXED16, batch=16) as c:
        ks = c.time_kernels(reps=2)
    assert [k[0] for k in ks] == ["cg_a_fp16", "cg_b_fp16"] and all(ms > 0 for _, ms, _ in ks)
