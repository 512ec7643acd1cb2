"""Pin the CPU oracle (oracle/sedi_oracle.c) against the reference's own outputs.

The golden fixtures under tests/golden/ were produced by the reference sources
themselves (tests/golden/make_golden.py, oracle/ref_driver.cc).  These tests
need no GPU.

Tolerances: relative max-norm |a-b|max/|b|max.  CG and pipelined CG are
compared at 1e-10 at fixed iteration counts and to convergence.  BiCGStab is
compared at 1e-10 up to 20 iterations; past that its iterates depend on the
last bit of every rounding (the reference itself moves by 1.5e-3 at 32^3 /
50 iterations between a contracted and an uncontracted build), so converged
BiCGStab runs are compared at 1e-6 with iteration counts within 15%.
"""
import numpy as np
import pytest

import _oracle as O

SOLVER_OF = {"cg": 2, "pcg": 3, "bicgstab": 1}


def test_probes_bit_exact():
    g = O.golden("probes_32")
    n = 32 ** 3
    bits = np.unpackbits(g["v_bits"])[: 5 * n].reshape(5, n)
    for k in range(5):
        v = O.fill_probe(1234 + k, n)
        assert np.array_equal(v > 0, bits[k].astype(bool)), f"probe {k}"
        assert set(np.unique(v)) <= {-1.0, 1.0}


@pytest.mark.parametrize("dims", [(5, 7, 9), (1, 1, 1), (1, 13, 1), (16, 3, 2), (8, 8, 8)])
@pytest.mark.parametrize("coeffs", [(6.0, 1.0, 1.0), (6.0, 1.3, 0.7), (-2.5, 0.25, -3.0)])
def test_stencil_matches_numpy_restatement(dims, coeffs):
    rng = np.random.default_rng(7)
    n = dims[0] * dims[1] * dims[2]
    x = rng.standard_normal(n)
    assert np.array_equal(O.stencil(dims, x, coeffs), O.numpy_stencil(dims, x, coeffs))


def _check_case(name, tol_D, tol_x=None, iter_slack=0.0, tol_err=None):
    g = O.golden(name)
    m = g["meta"]
    r = O.estimate(m["solver"], m["grid"], m["samples"], m["seed"], m["maxiter"], m["tol"], m["coeffs"],
                   keep="x" in g)
    assert O.relmax(r["D"], g["D"]) <= tol_D, (name, O.relmax(r["D"], g["D"]))
    if iter_slack == 0.0:
        assert np.array_equal(r["iters"], g["iters"]), (r["iters"], g["iters"])
        assert np.array_equal(r["results"], g["results"])
        # final_err differences below 1e-15 are below what an FP64 relative
        # residual resolves (converged tiny grids end at err ~1e-17).
        rtol = tol_err or tol_D
        assert np.all(np.abs(r["errs"] - g["errs"]) <= rtol * np.abs(g["errs"]) + 1e-15), (r["errs"], g["errs"])
    else:
        assert np.all(np.abs(r["iters"] - g["iters"]) <= np.ceil(iter_slack * g["iters"]) + 1)
        assert np.array_equal(r["results"], g["results"])
    if tol_x is not None:
        n = int(np.prod(m["grid"]))
        for k in range(m["samples"]):
            xs = slice(k * n, (k + 1) * n)
            assert O.relmax(r["x"][xs], g["x"][xs]) <= tol_x, (name, k)
        bits = np.unpackbits(g["v_bits"])[: m["samples"] * n].astype(bool)
        assert np.array_equal(r["v"] > 0, bits)
    # q accumulates v.*v = 1 exactly (stochastic-estimator.cc:198).
    assert np.all(g["q"] == m["samples"])


def test_config1_cg_32():
    _check_case("cfg1_cg_32", 1e-10)


def test_pcg_32_fixed_50():
    _check_case("pcg_32_m50", 1e-10)


def test_bicgstab_32_fixed_20():
    # The residual norm after 20 BiCGStab steps carries ~2e-10 relative rounding
    # noise (it is a small difference of large terms); D itself holds 1e-10.
    _check_case("bicgstab_32_m20", 1e-10, tol_err=1e-8)


@pytest.mark.parametrize("solver", ["cg", "pcg"])
def test_converged_krylov_24x20x16(solver):
    _check_case(f"conv_{solver}_24x20x16", 1e-10)


def test_converged_bicgstab_24x20x16():
    _check_case("conv_bicgstab_24x20x16", 1e-6, iter_slack=0.15)


@pytest.mark.parametrize("name", O.golden_names("odd_") + O.golden_names("tiny_") + O.golden_names("line_"))
def test_small_shapes(name):
    _check_case(name, 1e-9, tol_x=1e-9, iter_slack=0.0 if "bicgstab" not in name else 0.15)


def test_nonsymmetric_bicgstab():
    _check_case("nonsym_bicgstab_12x10x8", 1e-6, tol_x=1e-6, iter_slack=0.15)


def test_maxiter_result():
    g = O.golden("maxiter_cg_16")
    assert np.all(g["results"] == 1) and np.all(g["iters"] == 7)
    _check_case("maxiter_cg_16", 1e-10)


def test_exact_diag_inverse_formula():
    for dims in [(3, 4, 5), (6, 6, 6), (2, 7, 3)]:
        n = int(np.prod(dims))
        A = np.zeros((n, n))
        for j in range(n):
            e = np.zeros(n)
            e[j] = 1.0
            A[:, j] = O.numpy_stencil(dims, e)
        np.testing.assert_allclose(O.exact_diag_inv(dims), np.diag(np.linalg.inv(A)), rtol=1e-12)


def test_oracle_cg_recovers_exact_diagonal_entries():
    dims = (9, 8, 7)
    n = int(np.prod(dims))
    exact = O.exact_diag_inv(dims)
    for j in (0, 17, n // 2, n - 1):
        e = np.zeros(n)
        e[j] = 1.0
        rc, fe, fi, x, _ = O.solve(2, dims, e, maxiter=500, tol=1e-14)
        assert rc == 0
        assert abs(x[j] - exact[j]) <= 1e-12 * exact[j]


def test_estimator_unbiased_on_exact_diagonal():
    # With many probes D -> diag(A^-1); the estimator error shrinks like 1/sqrt(samples).
    dims = (6, 5, 4)
    r = O.estimate(2, dims, 400, 1234, 500, 1e-13)
    exact = O.exact_diag_inv(dims)
    assert np.abs(r["D"] - exact).max() < 0.05
