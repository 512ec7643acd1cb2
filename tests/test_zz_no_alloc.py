"""sedi_residual_noalloc: the residual entry point that allocates nothing.

It serves callers that cannot allocate device memory where they need a
residual check (pools or arenas that own all device memory, allocation-free
serving loops, frameworks with their own allocator); its scratch is a fixed
array inside the library.  Checked here through the C ABI against the
existing entry points on the same inputs: r against sedi_stencil_apply
(b - A x, bit for bit: same operations in the same order) and err against
the initial residual sedi_solve reports with maxiter 0 (1e-12 relative, the
tests' tolerance for a reduction), on two calls in a row.  This file is
collected last so a run that stops at its first failure has run every other
test already.
"""
import ctypes

import numpy as np
import pytest

import sedi_b200 as S

pytestmark = pytest.mark.gpu


def _noalloc(dims, x, b, coeffs=(6.0, 1.0, 1.0)):
    import torch
    xd = torch.from_numpy(x).cuda()
    bd = torch.from_numpy(b).cuda()
    rd = torch.full_like(bd, float("nan"))
    err = ctypes.c_double(-1.0)
    torch.cuda.synchronize()
    rc = S.load().sedi_residual_noalloc(*dims, *coeffs, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(bd.data_ptr()),
                                        ctypes.c_void_p(rd.data_ptr()), ctypes.byref(err), None)
    return rc, rd.cpu().numpy(), err.value


def _existing(dims, x, b, coeffs=(6.0, 1.0, 1.0)):
    with S.Context("cg", dims, S.Stencil(*coeffs)) as c:
        r = b - c.stencil_apply(x)
        xx = x.copy()
        res, fe, fi = c.solve(xx, b, None, 0, 0.0)
    return r, fe


def test_noalloc_residual_matches_existing_entry_points_twice():
    dims = (40, 33, 17)
    n = int(np.prod(dims))
    rng = np.random.default_rng(5)
    for call in range(2):
        x = rng.standard_normal(n)
        b = S.fill_probe(1234 + call, n)
        rc, r, err = _noalloc(dims, x, b)
        assert rc == 0
        r0, e0 = _existing(dims, x, b)
        assert np.array_equal(r, r0), call
        assert abs(err - e0) <= 1e-12 * e0, (call, err, e0)


def test_noalloc_zero_rhs_and_limit():
    dims = (16, 8, 4)
    n = int(np.prod(dims))
    z = np.zeros(n)
    rc, r, err = _noalloc(dims, z, z)
    assert rc == 0 and err == 0.0 and np.all(r == 0.0)
    # ceil(n1/32) * ceil(n2/8) > 4096 blocks is rejected before any launch
    # (three disjoint address ranges, never dereferenced).
    err = ctypes.c_double(0.0)
    size = 32 * 4097 * 8 * 8
    rc = S.load().sedi_residual_noalloc(32 * 4097, 8, 1, 6.0, 1.0, 1.0, ctypes.c_void_p(256),
                                        ctypes.c_void_p(256 + size), ctypes.c_void_p(256 + 2 * size),
                                        ctypes.byref(err), None)
    assert rc == -1


def test_noalloc_rejects_output_overlapping_an_input():
    import torch
    dims = (16, 8, 4)
    n = int(np.prod(dims))
    x = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    b = torch.zeros(n, dtype=torch.float64, device="cuda")
    err = ctypes.c_double(0.0)
    lib = S.load()
    vp = ctypes.c_void_p
    for r_ptr in (x.data_ptr(), x.data_ptr() + 8 * (n // 2), b.data_ptr()):
        rc = lib.sedi_residual_noalloc(*dims, 6.0, 1.0, 1.0, vp(x.data_ptr()), vp(b.data_ptr()), vp(r_ptr),
                                       ctypes.byref(err), None)
        assert rc == -1
    # The second half of x is disjoint from its first n elements: accepted.
    rc = lib.sedi_residual_noalloc(*dims, 6.0, 1.0, 1.0, vp(x.data_ptr()), vp(b.data_ptr()),
                                   vp(x.data_ptr() + 8 * n), ctypes.byref(err), None)
    assert rc == 0 and err.value == 0.0
