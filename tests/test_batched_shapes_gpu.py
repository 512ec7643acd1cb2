"""Batched forms on odd, thin and unit-dimension grids and on a nonsymmetric
operator, against the oracle lane by lane.  TMA boxes here are larger than
the grid in some dimension (the copy's zero fill is the ghost layer) and
the i3 split leaves chunks of one or two planes.

Bars: FP64 CG and pipelined CG converged to 1e-10 with the reference's
iteration counts and x within 1e-9 relative max-norm; FP64 BiCGStab within
1e-10 up to 8 iterations (its iterates are rounding-chaotic beyond ~20);
mixed CG and BiCGStab meet tol on their FP64 true residual.
"""
import numpy as np
import pytest

import _oracle as O
import sedi_b200 as S

pytestmark = pytest.mark.gpu

SHAPES = [(5, 7, 9), (1, 13, 1), (11, 1, 1), (16, 3, 2), (33, 17, 9), (2, 2, 40), (1, 1, 1)]
SID = {"cg": 2, "pcg": 3, "bicgstab": 1}


def _probes(dims, k, seed):
    n = int(np.prod(dims))
    return np.stack([O.fill_probe(seed + j, n) for j in range(k)])


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("solver", ["cg", "pcg"])
def test_fp64_batched_converged_odd_shapes(dims, solver):
    B = _probes(dims, 5, 900)
    X = np.zeros_like(B)
    with S.Context(solver, dims, batch=5) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=500, tol=1e-10)
    for k in range(5):
        rc0, fe0, fi0, x0, _ = O.solve(SID[solver], dims, B[k], maxiter=500, tol=1e-10)
        assert (res[k], fi[k]) == (rc0, fi0), (k, res[k], fi[k], rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-9


@pytest.mark.parametrize("dims", [d for d in SHAPES if np.prod(d) > 8])
def test_fp64_batched_bicgstab_odd_shapes(dims):
    B = _probes(dims, 4, 950)
    X = np.zeros_like(B)
    with S.Context("bicgstab", dims, batch=4) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=8, tol=0.0)
    for k in range(4):
        rc0, fe0, fi0, x0, _ = O.solve(1, dims, B[k], maxiter=8, tol=0.0)
        assert (res[k], fi[k]) == (rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-10


def test_fp64_batched_bicgstab_nonsymmetric():
    dims, coeffs = (12, 10, 8), (6.0, 1.3, 0.7)
    B = _probes(dims, 6, 31)
    X = np.zeros_like(B)
    with S.Context("bicgstab", dims, S.Stencil(*coeffs), batch=6) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=10, tol=0.0)
    for k in range(6):
        rc0, fe0, fi0, x0, _ = O.solve(1, dims, B[k], maxiter=10, tol=0.0, coeffs=coeffs)
        assert (res[k], fi[k]) == (rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-10


@pytest.mark.parametrize("dims", [(5, 7, 9), (1, 13, 1), (33, 17, 9), (2, 2, 40), (1, 1, 1)])
@pytest.mark.parametrize("solver", ["cg", "pcg", "bicgstab"])
def test_mixed_batched_odd_shapes_true_residual(dims, solver):
    """Tiny systems converge exactly within a few FP32 steps; the recurrence
    then divides 0 by 0 or drifts far below the true residual.  Such lanes
    hold, take a reliable update and restart, and still stop on their FP64
    true residual.  (The mixed pipelined CG runs the CG recurrence.)"""
    B = _probes(dims, 6, 970)
    X = np.zeros_like(B)
    with S.Context(solver, dims, precision=S.MIXED, batch=6) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=2000, tol=1e-10)
    assert np.all(res == 0)
    for k in range(6):
        r = B[k] - O.stencil(dims, X[k])
        assert np.sqrt((r @ r) / (B[k] @ B[k])) <= 1e-10 * 1.0000001

