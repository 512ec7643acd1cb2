"""Batched (RHS-interleaved) forms through the C ABI.

FP64 batched: the reference method lane by lane -- every right-hand side must
reproduce the single-vector FP64 path and the reference (same iteration
counts, x within 1e-10 relative max-norm: elementwise rounding is the
reference's, only dot-product summation order differs).

MIXED (FP32 vectors + FP64 reliable update): every right-hand side must meet
the reference's stopping test on its FP64 TRUE residual,
sqrt(<b-Ax, b-Ax>/<b,b>) <= tol (checked here on the CPU with the oracle's
stencil), and the estimated diagonal must stay within 1e-8 relative
max-norm of the FP64 answer on the same probes.
"""
import numpy as np
import pytest

import _oracle as O
import sedi_b200 as S

pytestmark = pytest.mark.gpu


def true_err(dims, x, b):
    r = b - O.stencil(dims, x)
    bb = float(b @ b) or 1.0
    return np.sqrt(float(r @ r) / bb)


@pytest.mark.parametrize("nrhs", [1, 3, 16, 64])
def test_fp64_batch_matches_single_vector(nrhs):
    dims = (20, 18, 16)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(1234 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=1000, tol=1e-9)
    for k in range(nrhs):
        rc0, fe0, fi0, x0, _ = O.solve(2, dims, B[k], maxiter=1000, tol=1e-9)
        assert (res[k], fi[k]) == (rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-10
        assert abs(fe[k] - fe0) <= 1e-10 * fe0 + 1e-15


@pytest.mark.parametrize("K", [200, 31])
def test_fp64_batch_fixed_iterations(K):
    """K odd: the batch ends on an odd iteration, whose deferred x step is
    applied after the last sweep (kb_x_flush)."""
    dims = (24, 20, 16)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(99 + k, n) for k in range(5)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, batch=8) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=K, tol=0.0)
    for k in range(5):
        rc0, fe0, fi0, x0, _ = O.solve(2, dims, B[k], maxiter=K, tol=0.0)
        assert (res[k], fi[k]) == (rc0, fi0) == (1, K)
        assert O.relmax(X[k], x0) <= 1e-10


def test_fp64_batch_estimator_vs_reference():
    g = O.golden("cfg1_cg_32")
    m = g["meta"]
    with S.Context("cg", m["grid"], batch=8) as c:
        r = c.estimate(m["samples"], m["seed"], m["maxiter"], m["tol"])
    assert np.array_equal(r["iters"], g["iters"]) and np.array_equal(r["results"], g["results"])
    assert O.relmax(r["D"], g["D"]) <= 1e-10
    assert np.array_equal(r["q"], g["q"])


@pytest.mark.parametrize("nrhs,tol", [(4, 1e-9), (16, 1e-9), (64, 1e-10), (128, 1e-9)])
def test_mixed_batch_true_residual(nrhs, tol):
    dims = (24, 22, 20)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(7 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, precision=S.MIXED, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=2000, tol=tol)
    assert np.all(res == 0)
    fi64 = []
    for k in range(nrhs):
        e = true_err(dims, X[k], B[k])
        assert e <= tol * 1.0000001, (k, e)
        assert abs(fe[k] - e) <= 1e-3 * e + 1e-16  # reported err is the FP64 true residual
        if k < 4:
            fi64.append(O.solve(2, dims, B[k], maxiter=2000, tol=tol)[2])
    # Mixed precision may need a few more iterations than FP64, not many.
    assert np.all(fi[: len(fi64)] <= np.array(fi64) * 1.25 + 10)


def test_mixed_estimator_diagonal_error():
    dims = (32, 32, 32)
    samples = 16
    with S.Context("cg", dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 1234, 2000, 1e-9)
    with S.Context("cg", dims, precision=S.MIXED, batch=samples) as cm:
        rm = cm.estimate(samples, 1234, 2000, 1e-9)
    assert np.all(rm["results"] == 0)
    assert O.relmax(rm["D"], r64["D"]) <= 1e-8, O.relmax(rm["D"], r64["D"])


def test_mixed_maxiter_reports_result_1():
    dims = (16, 16, 16)
    n = 16 ** 3
    B = np.stack([O.fill_probe(3 + k, n) for k in range(4)])
    X = np.zeros_like(B)
    with S.Context("cg", dims, precision=S.MIXED, batch=4) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=7, tol=1e-14)
    assert np.all(res == 1) and np.all(fi == 7)
    for k in range(4):
        assert abs(fe[k] - true_err(dims, X[k], B[k])) <= 1e-3 * fe[k]


def test_batch_padding_lanes_and_zero_rhs():
    dims = (12, 10, 8)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(11, n), np.zeros(n), O.fill_probe(12, n)])
    for prec in (S.FP64, S.MIXED):
        X = np.zeros_like(B)
        with S.Context("cg", dims, precision=prec, batch=7) as c:
            res, fe, fi = c.solve_batch(X, B, maxiter=500, tol=1e-10)
        assert np.all(res == 0)
        assert fi[1] == 0 and fe[1] == 0.0 and np.all(X[1] == 0.0)


@pytest.mark.parametrize("nrhs", [1, 5, 16])
def test_fp64_batch_pcg_matches_single_vector(nrhs):
    dims = (20, 18, 16)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(555 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("pcg", dims, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=1000, tol=1e-9)
    for k in range(nrhs):
        rc0, fe0, fi0, x0, _ = O.solve(3, dims, B[k], maxiter=1000, tol=1e-9)
        assert (res[k], fi[k]) == (rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-10
        assert abs(fe[k] - fe0) <= 1e-8 * fe0 + 1e-15


def test_fp64_batch_pcg_estimator_vs_reference():
    g = O.golden("pcg_32_m50")
    m = g["meta"]
    with S.Context("pcg", m["grid"], batch=8) as c:
        r = c.estimate(m["samples"], m["seed"], m["maxiter"], m["tol"])
    assert np.array_equal(r["iters"], g["iters"]) and np.array_equal(r["results"], g["results"])
    assert O.relmax(r["D"], g["D"]) <= 1e-10


@pytest.mark.parametrize("nrhs,tol", [(4, 1e-9), (32, 1e-10)])
def test_mixed_batch_pcg_true_residual(nrhs, tol):
    dims = (24, 22, 20)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(31 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("pcg", dims, precision=S.MIXED, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=3000, tol=tol)
    assert np.all(res == 0)
    for k in range(nrhs):
        assert true_err(dims, X[k], B[k]) <= tol * 1.0000001, k
    fi64 = O.solve(3, dims, B[0], maxiter=3000, tol=tol)[2]
    assert fi[0] <= fi64 * 1.25 + 10


def test_mixed_pcg_estimator_diagonal_error():
    dims = (32, 32, 32)
    samples = 16
    with S.Context("pcg", dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 1234, 3000, 1e-9)
    with S.Context("pcg", dims, precision=S.MIXED, batch=samples) as cm:
        rm = cm.estimate(samples, 1234, 3000, 1e-9)
    assert np.all(rm["results"] == 0)
    assert O.relmax(rm["D"], r64["D"]) <= 1e-8, O.relmax(rm["D"], r64["D"])


# BiCGStab: FP64 lanes follow the single-vector parity bars (1e-10 in x up to
# 20 iterations with identical result codes and counts; converged runs 1e-6
# with counts within 15%: the reference's own BiCGStab iterates move by 1.5e-3
# between two floating-point contractions of the same source).
@pytest.mark.parametrize("nrhs", [1, 5, 16])
def test_fp64_batch_bicgstab_fixed_iterations(nrhs):
    dims = (24, 20, 16)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(700 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("bicgstab", dims, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=15, tol=0.0)
    for k in range(nrhs):
        rc0, fe0, fi0, x0, _ = O.solve(1, dims, B[k], maxiter=15, tol=0.0)
        assert (res[k], fi[k]) == (rc0, fi0)
        assert O.relmax(X[k], x0) <= 1e-10
        assert abs(fe[k] - fe0) <= 1e-8 * fe0 + 1e-15


def test_fp64_batch_bicgstab_estimator_vs_reference():
    g = O.golden("bicgstab_32_m20")
    m = g["meta"]
    with S.Context("bicgstab", m["grid"], batch=8) as c:
        r = c.estimate(m["samples"], m["seed"], m["maxiter"], m["tol"], ignore_errors=True)
    assert np.array_equal(r["iters"], g["iters"]) and np.array_equal(r["results"], g["results"])
    assert O.relmax(r["D"], g["D"]) <= 1e-10
    assert np.all(np.abs(r["errs"] - g["errs"]) <= 1e-8 * np.abs(g["errs"]) + 1e-15)


def test_fp64_batch_bicgstab_converged_vs_reference():
    g = O.golden("conv_bicgstab_24x20x16")
    m = g["meta"]
    with S.Context("bicgstab", m["grid"], batch=16) as c:
        r = c.estimate(m["samples"], m["seed"], m["maxiter"], m["tol"], ignore_errors=True)
    assert np.array_equal(r["results"], g["results"])
    assert np.all(np.abs(r["iters"] - g["iters"]) <= np.ceil(0.15 * g["iters"]) + 1)
    assert O.relmax(r["D"], g["D"]) <= 1e-6


def test_fp64_batch_bicgstab_edge_lanes():
    """Zero right-hand side with tol 0 (rho = 0 at iteration 1: the reference
    reports success at iteration 1), a maxiter stop, and padding lanes."""
    dims = (12, 10, 8)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(5, n), np.zeros(n), O.fill_probe(6, n)])
    X = np.zeros_like(B)
    with S.Context("bicgstab", dims, batch=7) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=6, tol=0.0)
    for k in range(3):
        rc0, fe0, fi0, x0, _ = O.solve(1, dims, B[k], maxiter=6, tol=0.0)
        assert (res[k], fi[k]) == (rc0, fi0), k
        assert O.relmax(X[k], x0) <= 1e-10 if k != 1 else np.all(X[k] == 0.0)
    assert (res[1], fi[1], fe[1]) == (0, 1, 0.0)


@pytest.mark.parametrize("nrhs,tol", [(4, 1e-9), (32, 1e-10)])
def test_mixed_batch_bicgstab_true_residual(nrhs, tol):
    dims = (24, 22, 20)
    n = int(np.prod(dims))
    B = np.stack([O.fill_probe(41 + k, n) for k in range(nrhs)])
    X = np.zeros_like(B)
    with S.Context("bicgstab", dims, precision=S.MIXED, batch=nrhs) as c:
        res, fe, fi = c.solve_batch(X, B, maxiter=3000, tol=tol)
    assert np.all(res == 0)
    for k in range(nrhs):
        e = true_err(dims, X[k], B[k])
        assert e <= tol * 1.0000001, (k, e)
        assert abs(fe[k] - e) <= 1e-3 * e + 1e-16
    fi64 = O.solve(1, dims, B[0], maxiter=3000, tol=tol)[2]
    assert fi[0] <= fi64 * 1.5 + 10


@pytest.mark.parametrize("dims", [(32, 32, 32), (48, 48, 48)])
def test_mixed_bicgstab_closer_to_converged_diagonal_than_fp64(dims):
    """BiCGStab's diagonal at tol 1e-9 is not reproducible to 1e-8 in any
    precision: the FP64 form lies 1e-7 .. 4e-7 from the converged diagonal
    (and two compilations of the reference differ by 2e-7).  The mixed lanes
    stop on their FP64 true residual at 0.1 tol, which puts their diagonal
    within 2e-8 of the converged one (FP64 CG to 1e-13 on the same probes),
    several times closer than the FP64 form's."""
    samples = 16
    with S.Context("cg", dims, batch=samples) as cx:
        ex = cx.estimate(samples, 1234, 5000, 1e-13)
    with S.Context("bicgstab", dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 1234, 3000, 1e-9)
    with S.Context("bicgstab", dims, precision=S.MIXED, batch=samples) as cm:
        assert cm.mixed_target == 0.1
        rm = cm.estimate(samples, 1234, 3000, 1e-9)
    assert np.all(rm["results"] == 0)
    e_mixed, e_fp64 = O.relmax(rm["D"], ex["D"]), O.relmax(r64["D"], ex["D"])
    assert e_mixed <= 2e-8 and e_mixed <= 0.5 * e_fp64, (e_mixed, e_fp64)


@pytest.mark.parametrize("solver", ["cg", "pcg"])
def test_mixed_estimator_within_1e8_of_fp64_48cube(solver):
    """Diagonal error of the mixed form against the FP64 form on the same 32
    probes, 48^3, tol 1e-9: <= 1e-8 relative max-norm (the mixed pipelined CG
    runs the CG recurrence, whose FP32 iterates follow the FP64 ones)."""
    dims, samples = (48, 48, 48), 32
    with S.Context(solver, dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 4321, 5000, 1e-9)
    with S.Context(solver, dims, precision=S.MIXED, batch=samples) as cm:
        assert cm.mixed_target == 1.0
        rm = cm.estimate(samples, 4321, 5000, 1e-9)
    assert np.all(rm["results"] == 0) and np.all(r64["results"] == 0)
    assert np.array_equal(rm["q"], r64["q"])
    assert O.relmax(rm["D"], r64["D"]) <= 1e-8, O.relmax(rm["D"], r64["D"])


@pytest.mark.parametrize("solver", ["cg", "pcg"])
def test_mixed_estimator_within_1e8_of_fp64_256cube(solver):
    """The batched mixed configuration's grid (256^3, tol 1e-9) with 32 of its
    128 probes: D of the mixed form within 1e-8 of the FP64 form's."""
    dims, samples = (256, 256, 256), 32
    with S.Context(solver, dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 1234, 20000, 1e-9)
    with S.Context(solver, dims, precision=S.MIXED, batch=samples) as cm:
        rm = cm.estimate(samples, 1234, 20000, 1e-9)
    assert np.all(rm["results"] == 0) and np.all(r64["results"] == 0)
    assert O.relmax(rm["D"], r64["D"]) <= 1e-8, O.relmax(rm["D"], r64["D"])


def test_large_512cube_mixed_pcg_vs_single_vector_fp64():
    """The large single-domain configuration: 512^3 (134M points), pipelined
    CG, 16 probes batched in FP32 with the FP64 reliable update, tol 1e-8,
    maxiter 500 (no probe reaches tol: result 1, as in the reference's
    -m 500 run).  Neither form has converged at 500 iterations (residuals
    2e-4 to 7e-4), so the diagonal differs by the FP32 rounding of the
    unconverged iterates (1.1e-7 measured), not by a truncation bar; the
    mixed form's final FP64 true residuals are the FP64 form's within 2%."""
    dims, samples = (512, 512, 512), 16
    with S.Context("pcg", dims, precision=S.MIXED, batch=samples) as cm:
        rm = cm.estimate(samples, 1234, 500, 1e-8, ignore_errors=True)
    with S.Context("pcg", dims) as cp:
        rp = cp.estimate(samples, 1234, 500, 1e-8, ignore_errors=True)
    assert np.all(rm["results"] == 1) and np.all(rp["results"] == 1)
    assert np.array_equal(rm["iters"], rp["iters"])
    assert np.array_equal(rm["q"], rp["q"])
    assert O.relmax(rm["D"], rp["D"]) <= 3e-7, O.relmax(rm["D"], rp["D"])
    assert np.all(np.abs(rm["errs"] - rp["errs"]) <= 0.02 * rp["errs"]), (rm["errs"], rp["errs"])


@pytest.mark.parametrize("period", [7, 32])
def test_mixed_cg_deferred_x_steps_with_odd_updates(period):
    """The mixed CG applies the x step of an odd iteration together with the
    next even one's; a reliable update after an odd iteration (period 7:
    every other update; lane-triggered ones at any iteration) folds the
    pending step into x_hi.  A lost or doubled step would show as a true
    residual off the recurrence and extra iterations: the iteration counts
    stay within one of the FP64 form's and D within 1e-8 of it."""
    dims, samples = (48, 48, 48), 16
    with S.Context("cg", dims, batch=samples) as c64:
        r64 = c64.estimate(samples, 99, 5000, 1e-9)
    S.set_tuning("cg", dims, samples, precision=S.MIXED, period=period)
    try:
        with S.Context("cg", dims, precision=S.MIXED, batch=samples) as cm:
            assert cm.config()["period"] == period
            rm = cm.estimate(samples, 99, 5000, 1e-9)
    finally:
        S.set_tuning("cg", dims, samples, precision=S.MIXED)
    assert np.all(rm["results"] == 0) and np.all(r64["results"] == 0)
    assert np.abs(rm["iters"] - r64["iters"]).max() <= 1, (rm["iters"], r64["iters"])
    assert O.relmax(rm["D"], r64["D"]) <= 1e-8, O.relmax(rm["D"], r64["D"])


@pytest.mark.parametrize("solver,prec,nk", [("cg", S.MIXED, 3), ("pcg", S.MIXED, 3), ("bicgstab", S.MIXED, 3),
                                            ("pcg", S.FP64, 1), ("cg", S.FP64, 3)])
def test_time_kernels_lists_solver_sweeps(solver, prec, nk):
    """Per-iteration sweeps: BiCGStab 3, pipelined CG 1 in FP64.  CG (and the
    mixed pipelined CG, which runs the CG recurrence) lists sweep A and the
    two parity forms of sweep B: cg_b on odd iterations (r only, 3 words)
    and cg_bx on even ones (both x steps, 6)."""
    with S.Context(solver, (64, 64, 64), precision=prec, batch=16) as c:
        ks = c.time_kernels(reps=2)
    assert len(ks) == nk and all(ms > 0 and by > 0 for _, ms, by in ks)
    if solver == "cg" or (prec == S.MIXED and solver == "pcg"):
        t = "fp32" if prec == S.MIXED else "fp64"
        names = [k[0] for k in ks]
        assert names == [f"cg_a_{t}", f"cg_b_{t}", f"cg_bx_{t}"], names
        assert ks[2][2] == 2 * ks[1][2] == 2 * ks[0][2]


@pytest.mark.parametrize("solver,prec", [("cg", S.FP64), ("cg", S.MIXED), ("pcg", S.MIXED), ("bicgstab", S.FP64)])
def test_autotuned_context_keeps_results(solver, prec):
    """The autotuner's choices (slice width, i3 split, graph chunk, reliable-update
    period) change only launch shapes and summation order: FP64 CG/PCG stay
    within 1e-10 of the untuned run with the same iteration counts, BiCGStab
    FP64 within its 20-iteration bar, mixed CG and pipelined CG within 1e-8
    of FP64."""
    dims, samples = (40, 36, 48), 16
    maxiter, tol = (20, 0.0) if solver == "bicgstab" else (3000, 1e-9)
    with S.Context(solver, dims, precision=prec, batch=samples) as c:
        ref = c.estimate(samples, 321, maxiter, tol, ignore_errors=True)
        before = c.config()
    choice = S.autotune(solver, dims, samples, precision=prec, maxiter=maxiter, tol=tol, seed=321)
    with S.Context(solver, dims, precision=prec, batch=samples) as c:
        after = c.config()
        got = c.estimate(samples, 321, maxiter, tol, ignore_errors=True)
    assert after["slice_width"] == choice["slice_width"] and after["lanes"] == before["lanes"]
    if choice["chunk"]:
        assert after["chunk"] == choice["chunk"]
    if prec == S.MIXED:
        # Two mixed runs that both meet tol land at different x; each must be
        # within the mixed bar of the FP64 answer on the same probes.
        assert 20 <= after["period"] <= 50
        with S.Context(solver, dims, precision=S.FP64, batch=samples) as c64:
            r64 = c64.estimate(samples, 321, maxiter, tol, ignore_errors=True)
        assert O.relmax(got["D"], r64["D"]) <= 1e-8
        assert O.relmax(ref["D"], r64["D"]) <= 1e-8
    else:
        assert np.array_equal(got["iters"], ref["iters"]) and np.array_equal(got["results"], ref["results"])
        assert O.relmax(got["D"], ref["D"]) <= 1e-10


@pytest.mark.parametrize("prec", [S.FP64, S.MIXED])
def test_cg_sweep_a_forms_agree(prec):
    """CG's sweep A as a ring of computed planes (form 1) or with the stencil
    input written over p_old in the stage (forms 2 and 3, no ring): the same
    values, summed on other tiles.  FP64: same iteration counts and D within
    1e-12; mixed: within 1e-9 of each other."""
    dims, samples = (40, 36, 30), 16
    out = {}
    for form in (1, 2, 3):
        S.set_tuning("cg", dims, samples, precision=prec, sweep_a_form=form)
        with S.Context("cg", dims, precision=prec, batch=samples) as c:
            assert c.config()["sweep_a_form"] == form
            out[form] = c.estimate(samples, 99, 3000, 1e-10)
    S.set_tuning("cg", dims, samples, precision=prec)
    for form in (2, 3):
        assert np.array_equal(out[form]["results"], out[1]["results"])
        if prec == S.FP64:
            assert np.array_equal(out[form]["iters"], out[1]["iters"])
            assert O.relmax(out[form]["D"], out[1]["D"]) <= 1e-12
        else:
            assert O.relmax(out[form]["D"], out[1]["D"]) <= 1e-9


@pytest.mark.parametrize("prec", [S.FP64, S.MIXED])
def test_bicgstab_sweep_forms_agree(prec):
    """BiCGStab's sweeps 2 and 3 as a ring of s (form 1) or with s written
    over v in the stage (forms 2 and 3): the same values summed on other
    tiles.  At 20 fixed iterations FP64 agrees to 1e-9 (BiCGStab amplifies
    the other summation order: 2.8e-11 measured), mixed to 1e-6 (the FP32
    iterates, no reliable-update target at tol 0)."""
    dims, samples = (40, 36, 30), 16
    out = {}
    for form in (1, 2, 3):
        S.set_tuning("bicgstab", dims, samples, precision=prec, sweep_a_form=form)
        with S.Context("bicgstab", dims, precision=prec, batch=samples) as c:
            assert c.config()["sweep_a_form"] == form
            out[form] = c.estimate(samples, 99, 20, 0.0, ignore_errors=True)
    S.set_tuning("bicgstab", dims, samples, precision=prec)
    for form in (2, 3):
        assert np.array_equal(out[form]["results"], out[1]["results"])
        assert O.relmax(out[form]["D"], out[1]["D"]) <= (1e-9 if prec == S.FP64 else 1e-6)


def test_single_vector_autotune_keeps_results():
    """The autotuner on one FP64 right-hand side tunes the single-vector
    streaming sweeps (i3 split, prefetch, sweep form): at 30 fixed CG
    iterations D stays within 1e-12 of the untuned run.  Odd n1 has no
    streaming form: SEDI_ERR_UNSUPPORTED."""
    dims = (256, 128, 128)
    with S.Context("cg", dims) as c:
        ref = c.estimate(2, 7, 30, 0.0, ignore_errors=True)
    choice = S.autotune("cg", dims, 1, precision=S.FP64, maxiter=30, tol=0.0, solve=False)
    assert choice["slice_width"] == 2 and choice["sweep_a_form"] in (1, 2, 3)
    with S.Context("cg", dims) as c:
        got = c.estimate(2, 7, 30, 0.0, ignore_errors=True)
    S.set_tuning("cg", dims, 1, precision=S.FP64)
    assert np.array_equal(got["iters"], ref["iters"])
    assert O.relmax(got["D"], ref["D"]) <= 1e-12
    with pytest.raises(S.SediError):
        S.autotune("cg", (255, 128, 130), 1, precision=S.FP64, solve=False)
