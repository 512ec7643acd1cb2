"""ctypes binding to the CPU oracle (oracle/sedi_oracle.c) -- test-side checker only."""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(REPO, "oracle", "_build", "libsedi_oracle.so")
GOLDEN = os.path.join(REPO, "tests", "golden")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(PATH):
            subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle"), "port"])
        L = ctypes.CDLL(PATH)
        c_long, c_double, vp, c_int = ctypes.c_long, ctypes.c_double, ctypes.c_void_p, ctypes.c_int
        L.so_fill_probe.argtypes = [ctypes.c_uint32, c_long, vp]
        L.so_fill_probe.restype = None
        L.so_stencil.argtypes = [c_long, c_long, c_long, c_double, c_double, c_double, vp, vp]
        L.so_stencil.restype = None
        L.so_dot.argtypes = [c_long, vp, vp]
        L.so_dot.restype = c_double
        for f in (L.so_cg, L.so_pcg, L.so_bicgstab):
            f.argtypes = [c_long, c_long, c_long, c_double, c_double, c_double, vp, vp, vp, c_int, c_double,
                          vp, vp, vp]
            f.restype = c_int
        L.so_estimate.argtypes = [c_int, c_long, c_long, c_long, c_double, c_double, c_double, c_int,
                                  ctypes.c_uint32, c_int, c_double] + [vp] * 8
        L.so_estimate.restype = c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def fill_probe(seed, n):
    out = np.empty(n)
    lib().so_fill_probe(seed & 0xFFFFFFFF, n, _p(out))
    return out


def stencil(dims, x, coeffs=(6.0, 1.0, 1.0)):
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    lib().so_stencil(*dims, *coeffs, _p(x), _p(y))
    return y


def solve(solver, dims, b, x0=None, iM=None, maxiter=1000, tol=1e-9, coeffs=(6.0, 1.0, 1.0)):
    """Returns (result, final_err, final_iter, x, err_hist)."""
    n = dims[0] * dims[1] * dims[2]
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    fe, fi = ctypes.c_double(0), ctypes.c_int(0)
    hist = np.full(maxiter + 1, np.nan)
    f = {1: lib().so_bicgstab, 2: lib().so_cg, 3: lib().so_pcg}[solver]
    rc = f(*dims, *coeffs, _p(x), _p(b), _p(None if iM is None else np.ascontiguousarray(iM, np.float64)),
           maxiter, tol, ctypes.byref(fe), ctypes.byref(fi), _p(hist))
    return rc, fe.value, fi.value, x, hist


def estimate(solver, dims, samples, seed=1234, maxiter=1000, tol=1e-9, coeffs=(6.0, 1.0, 1.0), keep=False):
    n = dims[0] * dims[1] * dims[2]
    D, t, q = np.empty(n), np.empty(n), np.empty(n)
    iters = np.zeros(samples, np.int32)
    errs = np.zeros(samples)
    results = np.zeros(samples, np.int32)
    X = np.empty(n * samples) if keep else None
    V = np.empty(n * samples) if keep else None
    lib().so_estimate(solver, *dims, *coeffs, samples, seed, maxiter, tol, _p(D), _p(t), _p(q), _p(iters),
                      _p(errs), _p(results), _p(X), _p(V))
    return dict(D=D, t=t, q=q, iters=iters, errs=errs, results=results, x=X, v=V)


def golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {k: z[k] for k in z.files}
    out["meta"] = eval(str(out["meta"]))  # repr of a dict of literals, written by make_golden.py
    return out


def golden_names(prefix=""):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith(prefix))


def relmax(a, b):
    """|a-b|max / |b|max; NaN at the same place in both counts as equal (the
    reference itself produces NaN in a few degenerate cases, e.g. pipelined CG
    on a 1x1x1 grid), NaN in only one of them is an infinite error."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    na, nb = np.isnan(a), np.isnan(b)
    if np.any(na != nb):
        return float("inf")
    a, b = a[~na], b[~nb]
    if a.size == 0:
        return 0.0
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def numpy_stencil(dims, x, coeffs=(6.0, 1.0, 1.0)):
    """Independent numpy restatement of Stencil::apply_direct (term order kept)."""
    n1, n2, n3 = dims
    a, b, c = coeffs
    X = np.zeros((n3 + 2, n2 + 2, n1 + 2))
    X[1:-1, 1:-1, 1:-1] = np.asarray(x).reshape(n3, n2, n1)
    C = X[1:-1, 1:-1, 1:-1]
    y = (a * C - c * X[1:-1, 1:-1, :-2] - c * X[1:-1, :-2, 1:-1] - c * X[:-2, 1:-1, 1:-1]
         - b * X[1:-1, 1:-1, 2:] - b * X[1:-1, 2:, 1:-1] - b * X[2:, 1:-1, 1:-1])
    return y.reshape(-1)


def exact_diag_inv(dims, a=6.0, b=1.0):
    """diag(A^-1) for the symmetric stencil (b == c) by separable sine expansion:
    A = a I - b (T1 + T2 + T3) with Dirichlet path matrices; eigenpairs
    lambda = a - 2b sum_d cos(pi k_d/(n_d+1)), phi = prod_d sqrt(2/(n_d+1)) sin(pi k_d i_d/(n_d+1))."""
    n1, n2, n3 = dims
    def modes(n):
        k = np.arange(1, n + 1)
        i = np.arange(1, n + 1)
        return np.cos(np.pi * k / (n + 1)), np.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(i, k) / (n + 1))
    c1, P1 = modes(n1)
    c2, P2 = modes(n2)
    c3, P3 = modes(n3)
    lam = a - 2 * b * (c1[None, None, :] + c2[None, :, None] + c3[:, None, None])  # [k3,k2,k1]
    inv = 1.0 / lam
    # diag[i3,i2,i1] = sum_k P3[i3,k3]^2 P2[i2,k2]^2 P1[i1,k1]^2 / lam[k3,k2,k1]
    D = np.einsum("ac,bd,ef,cdf->abe", P3 ** 2, P2 ** 2, P1 ** 2, inv)
    return D.reshape(-1)
