"""The deferred x step of the CG sweeps, restated on the CPU.

The GPU CG updates r every iteration but applies x's steps in pairs: an odd
iteration keeps alpha, the next even one computes
x = (x + alpha_odd p_odd) + alpha p, and a solve that ends on an odd
iteration applies its last step afterwards.  In FP64 with the updates in
that order (no FMA) every rounding is the reference's x = x + alpha p
(Cg.hpp:169) taken twice, so x is bit-identical.  This test runs the
reference CG iteration (Cg.hpp:150-193) in NumPy with both schedules: the
scalars do not depend on x, so the two x arrays must be equal bit for bit,
and the per-iteration schedule must be the oracle's solve.
"""
import numpy as np
import pytest

import _oracle as O


def _cg(dims, b, maxiter, tol, deferred):
    a_c = 6.0
    iM = 1.0 / a_c
    x = np.zeros_like(b)
    r = b - O.stencil(dims, x)                     # :119-123
    bb = float(np.dot(b, b)) or 1.0                 # :112-115
    if np.sqrt(np.dot(r, r) / bb) < tol:
        return x, 0
    p = None
    ru = 0.0
    beta = 0.0
    pending = None  # (alpha, p) of an odd iteration whose x step waits
    it = 0
    for it in range(1, maxiter + 1):
        u = r * iM
        if it == 1:
            p = u.copy()
            ru = float(np.dot(r, u))
        else:
            p = u + beta * p                        # :150-158
        s = O.stencil(dims, p)
        alpha = ru / float(np.dot(s, p))           # :160-166
        if not deferred:
            x = x + alpha * p                       # :169
        elif it % 2 == 1:
            pending = (alpha, p)
        else:
            x = (x + pending[0] * pending[1]) + alpha * p
            pending = None
        r = r + (-alpha) * s                        # :172
        u = r * iM
        ru_new = float(np.dot(r, u))
        beta = ru_new / ru                          # :185
        ru = ru_new
        if np.sqrt(np.dot(r, r) / bb) <= tol:      # :191-193
            break
    if pending is not None:                         # the solve ended on an odd iteration
        x = x + pending[0] * pending[1]
    return x, it


@pytest.mark.parametrize("maxiter,tol", [(30, 0.0), (31, 0.0), (1, 0.0), (500, 1e-9)])
def test_deferred_x_step_is_bit_identical(maxiter, tol):
    dims = (18, 14, 12)
    n = dims[0] * dims[1] * dims[2]
    b = O.fill_probe(1234, n)
    x1, it1 = _cg(dims, b, maxiter, tol, deferred=False)
    x2, it2 = _cg(dims, b, maxiter, tol, deferred=True)
    assert it1 == it2
    assert np.array_equal(x1, x2)
    # The per-iteration schedule is the reference method (the oracle sums its
    # dot products in another order, so the match is to rounding level).
    rc0, fe0, fi0, x0, _ = O.solve(2, dims, b, maxiter=maxiter, tol=tol)
    assert fi0 == it1
    assert O.relmax(x1, x0) <= 1e-12


def test_converged_run_ends_on_both_parities():
    """Probes whose converged iteration counts are odd and even (the flush
    after an odd last iteration and the even form's paired step)."""
    dims = (18, 14, 12)
    n = dims[0] * dims[1] * dims[2]
    parities = set()
    for seed in range(1234, 1240):
        b = O.fill_probe(seed, n)
        x1, it1 = _cg(dims, b, 500, 1e-9, deferred=False)
        x2, it2 = _cg(dims, b, 500, 1e-9, deferred=True)
        assert it1 == it2 and np.array_equal(x1, x2)
        parities.add(it1 % 2)
    assert parities == {0, 1}
