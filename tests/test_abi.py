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
