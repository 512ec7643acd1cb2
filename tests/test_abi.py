"""The C-ABI library loads, exports what include/sedi_b200.h declares, validates
its arguments and reports a missing device -- all without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import _oracle as O
import sedi_b200

HEADER = os.path.join(O.REPO, "include", "sedi_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sedi_\w+)\s*\(", text)))


def test_library_built_and_loads():
    assert os.path.exists(sedi_b200.library_path())
    lib = sedi_b200.load()
    assert b"sm_100a" in lib.sedi_version()


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(sedi_b200.library_path())
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name


def test_invalid_arguments_rejected_before_device_use():
    lib = sedi_b200.load()
    err = ctypes.c_int(0)
    bad = [
        (0, 8, 8, 8, 0, 1),    # solver id
        (4, 8, 8, 8, 0, 1),
        (2, 0, 8, 8, 0, 1),    # empty grid
        (2, 8, -1, 8, 0, 1),
        (2, 8, 8, 8, 7, 1),    # precision
        (2, 8, 8, 8, 0, 0),    # batch
    ]
    for solver, n1, n2, n3, prec, batch in bad:
        h = lib.sedi_create(solver, n1, n2, n3, 6.0, 1.0, 1.0, 0, prec, batch, ctypes.byref(err))
        assert not h and err.value == -1
    h = lib.sedi_create(2, 8, 8, 8, 6.0, 1.0, 1.0, 8, 0, 1, ctypes.byref(err))  # unknown mode bit
    assert not h and err.value == -1
    assert lib.sedi_solve(None, None, None, None, 10, 1e-9, None, None) == -1
    assert lib.sedi_estimate(None, 1, 1234, 10, 1e-9, 1, None, None, None, None, None, None) == -1


def test_missing_device_reported(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(sedi_b200.SediError) as e:
        sedi_b200.Context("cg", (8, 8, 8))
    assert e.value.code == -4


def test_host_probe_generator_bit_exact():
    g = O.golden("probes_32")
    n = 32 ** 3
    bits = np.unpackbits(g["v_bits"])[: 5 * n].reshape(5, n).astype(bool)
    for k in range(5):
        v = sedi_b200.fill_probe(1234 + k, n)
        assert np.array_equal(v > 0, bits[k])
        assert np.all(np.abs(v) == 1.0)


def test_solver_classes_mirror_reference_enums():
    assert sedi_b200.Cg.CG_REACHED_MAXITER == 1
    assert sedi_b200.PipelinedCg.PLCG_SOLUTION_FOUND == 0
    assert sedi_b200.BiCgStab.BICGSTAB_BREAKDOWN_RHO == 2
    assert sedi_b200.BiCgStab.BICGSTAB_BREAKDOWN_OMEGA == 3
    with pytest.raises(ValueError):
        sedi_b200.Cg((4, 4, 4), nghost=2)


def test_job_bytes_is_host_arithmetic():
    """The server's admission size needs no device: the lane-sliced fields of
    a batched context plus its small per-lane and reduction buffers."""
    n = 64 ** 3
    # CG mixed, 16 lanes: x_lo, r, p0, p1 in FP32 and b, x_hi in FP64 per point and lane.
    cg = sedi_b200.job_bytes("cg", (64, 64, 64), 16, sedi_b200.MIXED)
    assert cg >= n * 16 * (4 * 4 + 2 * 8)
    assert cg <= n * 16 * (4 * 4 + 2 * 8) * 1.05 + 64 * 2 ** 20
    # BiCGStab adds four FP32 fields; the mixed pipelined CG runs the CG
    # recurrence (same fields as CG), its FP64 form six more FP64 fields.
    pcg = sedi_b200.job_bytes("pcg", (64, 64, 64), 16, sedi_b200.MIXED)
    bicg = sedi_b200.job_bytes("bicgstab", (64, 64, 64), 16, sedi_b200.MIXED)
    assert pcg == cg and bicg - cg >= 4 * n * 16 * 4
    cg64 = sedi_b200.job_bytes("cg", (64, 64, 64), 16, sedi_b200.FP64)
    assert cg64 > cg and sedi_b200.job_bytes("pcg", (64, 64, 64), 16, sedi_b200.FP64) - cg64 >= 6 * n * 16 * 8
    # Monotone in lanes and grid; lanes are padded to whole lane vectors.
    assert sedi_b200.job_bytes("cg", (64, 64, 64), 32, sedi_b200.MIXED) > cg
    assert sedi_b200.job_bytes("cg", (96, 96, 96), 16, sedi_b200.MIXED) > cg
    assert sedi_b200.job_bytes("cg", (64, 64, 64), 13, sedi_b200.MIXED) == cg
    assert load_bad_job_bytes() == 0.0


def load_bad_job_bytes():
    lib = sedi_b200.load()
    return lib.sedi_job_bytes(9, 0, 4, 8, 8, 8)


def test_server_and_autotune_argument_checks_without_device():
    lib = sedi_b200.load()
    choice = np.zeros(4, np.int32)
    assert lib.sedi_autotune(7, 1, 16, 8, 8, 8, 10, 1e-9, 1, 0, choice.ctypes.data_as(ctypes.c_void_p), None) == -1
    assert lib.sedi_autotune(2, 1, 16, 0, 8, 8, 10, 1e-9, 1, 0, choice.ctypes.data_as(ctypes.c_void_p), None) == -1
    assert lib.sedi_server_submit(None, 2, 1, 8, 8, 8, 4, 1, 10, 1e-9) == -1
    assert lib.sedi_server_step(None, None) == -1
    assert lib.sedi_server_take(None, 0, None, None, None, None) == -1
    timed_out = ctypes.c_int(0)
    assert lib.sedi_selftest_bounded_wait(0.0, ctypes.byref(timed_out), None) == -1
    assert lib.sedi_selftest_bounded_wait(10000.0, ctypes.byref(timed_out), None) == -1


def test_slab_sweep_argument_checks_without_device():
    """sedi_slab_sweep refuses bad modes, plane ranges, grids and missing
    vectors before any device call; a dot mode needs its scratch buffers."""
    from sedi_b200.domain import _SlabArgs, APPLY, CG_SP, SETUP
    lib = sedi_b200.load()
    vp, c_long, c_double, c_int = ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_int
    lib.sedi_slab_sweep.argtypes = [c_int, c_long, c_long, c_long, c_double, c_double, c_double, c_long, c_long,
                                    ctypes.POINTER(_SlabArgs), vp, vp, vp]
    fake = 0x1000  # never dereferenced: every call below fails its checks first
    a = _SlabArgs()
    a.src = a.y = fake

    def call(mode, n1=8, n2=8, nloc=4, z_lo=1, z_hi=5, args=a, chunk=None, plane=None):
        return lib.sedi_slab_sweep(mode, n1, n2, nloc, 6.0, 1.0, 1.0, z_lo, z_hi, ctypes.byref(args) if args else None,
                                   chunk, plane, None)

    assert call(13) == -1 and call(-1) == -1              # mode
    assert call(APPLY, z_lo=0) == -1                      # ghost plane 0 is not swept
    assert call(APPLY, z_hi=6) == -1                      # past plane nloc
    assert call(APPLY, z_lo=3, z_hi=2) == -1
    assert call(APPLY, n1=0) == -1 and call(APPLY, nloc=0) == -1
    assert call(APPLY, args=None) == -1
    assert call(SETUP) == -1                              # r and b missing
    assert call(CG_SP) == -1                              # a dot mode without scratch
    b = _SlabArgs()
    b.src = fake
    assert call(APPLY, args=b) == -1                      # y missing
    assert call(APPLY, z_lo=3, z_hi=3) == 0               # empty range: nothing to launch
    assert lib.sedi_slab_chunks() == 8
