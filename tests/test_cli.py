"""The `sedi` command-line driver (drop-in for stochastic-estimator.*.exe).

CPU tests: option handling that does not need a GPU.  GPU tests (marked):
the printed lines and the estimate against the reference's own binary and
golden fixtures, the -V / -E validators, abort codes.
"""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import _oracle as O

CLI = os.path.join(O.REPO, "sedi_b200", "_lib", "sedi")
REF_EXE = os.path.join(O.REPO, "oracle", "_ref", "stochastic-estimator.cg.exe")


def run(args, **kw):
    return subprocess.run([CLI] + args, capture_output=True, text=True, timeout=600, **kw)


def write_raw(archive, name, dims, dense):
    """Raw archive dataset in Slice3d::pack_into order (i1 outer, i3 fastest)."""
    os.makedirs(archive, exist_ok=True)
    n1, n2, n3 = dims
    packed = np.asarray(dense, np.float64).reshape(n3, n2, n1).transpose(2, 1, 0).copy()
    with open(os.path.join(archive, name + ".raw"), "wb") as f:
        f.write(b"SEDIRAW1" + struct.pack("<II", 3, 8) + struct.pack("<3Q", n1, n2, n3))
        f.write(packed.tobytes())


def test_cli_built():
    assert os.access(CLI, os.X_OK)


def test_decomposition_must_be_one_gpu():
    r = run(["-g", "8x8x8", "-p", "2x1x1", "-s", "1"])
    assert r.returncode == 1 and "-p 1x1x1" in r.stderr


@pytest.mark.parametrize("args", [["-p", "1x1x1"], ["-g", "8x8x8"], ["-g", "8x8", "-p", "1x1x1"],
                                  ["-g", "8x8x8", "-p", "1x1x1", "-s", "x"], ["-Z"]])
def test_usage_errors(args):
    r = run(args)
    assert r.returncode == 1 and "Usage:" in r.stderr


@pytest.mark.gpu
def test_config1_against_reference_binary(tmp_path):
    """CG, 32^3, 5 probes, tol 1e-9, maxiter 50, -i: D vs the reference's golden D,
    and every per-iteration err line vs the reference binary's own output."""
    dfile = tmp_path / "D.bin"
    r = run(["-g", "32x32x32", "-p", "1x1x1", "-s", "5", "-e", "1e-9", "-m", "50", "-i", "--write-d", str(dfile)])
    assert r.returncode == 0, r.stderr
    g = O.golden("cfg1_cg_32")
    D = np.fromfile(dfile)
    assert O.relmax(D, g["D"]) <= 1e-10
    assert "Total solve time" in r.stdout and "iteration count min=50 max=50" in r.stdout
    ours = [float(v) for v in re.findall(r"Cg: after iter=\d+, err=(\S+)", r.stdout)]
    assert len(ours) == 250
    if os.path.exists(REF_EXE):
        ref = subprocess.run([REF_EXE, "-g", "32x32x32", "-p", "1x1x1", "-s", "5", "-e", "1e-9", "-m", "50", "-i"],
                             capture_output=True, text=True, env=dict(os.environ, SEDI_SEED="1234"), timeout=600)
        theirs = [float(v) for v in re.findall(r"Cg: after iter=\d+, err=(\S+)", ref.stdout)]
        assert len(theirs) == 250
        assert np.allclose(ours, theirs, rtol=1e-9, atol=0)
        for key in ("Global grid shape is (32, 32, 32)", "Process block shape is (32, 32, 32)",
                    "Initialized Cg solver, sync_dotprod=0, sync_stencil=0", "Solving for sample 5/5..."):
            assert key in r.stdout and key in ref.stdout


@pytest.mark.gpu
def test_validate_solver_archive(tmp_path):
    dims = (20, 18, 16)
    n = int(np.prod(dims))
    v = O.fill_probe(77, n)
    _, _, _, x, _ = O.solve(2, dims, v, maxiter=2000, tol=1e-14)
    arch = str(tmp_path / "vs.h5")
    write_raw(arch, "x_k", dims, x)
    write_raw(arch, "v_k", dims, v)
    r = run(["-g", "20x18x16", "-p", "1x1x1", "-s", "2", "-e", "1e-9", "-m", "1000", "-V", arch, "--quiet"])
    assert r.returncode == 0, r.stderr
    errs = [tuple(map(float, m)) for m in re.findall(r"VALIDATION: rel L2 error=(\S+), rel Linf error=(\S+)", r.stdout)]
    assert len(errs) == 2 and all(e[0] < 1e-7 and e[1] < 1e-7 for e in errs)
    if os.path.exists(REF_EXE):
        ref = subprocess.run([REF_EXE, "-g", "20x18x16", "-p", "1x1x1", "-s", "2", "-e", "1e-9", "-m", "1000", "-V",
                              arch], capture_output=True, text=True, timeout=600)
        theirs = [tuple(map(float, m)) for m in
                  re.findall(r"VALIDATION: rel L2 error=(\S+), rel Linf error=(\S+)", ref.stdout)]
        assert len(theirs) == 2
        np.testing.assert_allclose(np.array(errs), np.array(theirs), rtol=1e-3)


@pytest.mark.gpu
def test_validate_estimator_archive(tmp_path):
    dims = (12, 10, 8)
    arch = str(tmp_path / "ve.h5")
    write_raw(arch, "diag_inv", dims, O.exact_diag_inv(dims))
    r = run(["-g", "12x10x8", "-p", "1x1x1", "-s", "3", "-e", "1e-12", "-m", "1000", "-E", arch, "--quiet"])
    assert r.returncode == 0, r.stderr
    ours = [tuple(map(float, m)) for m in re.findall(r"VALIDATION_ESTIMATOR: L2 error=(\S+), Linf error=(\S+)", r.stdout)]
    assert len(ours) == 3
    if os.path.exists(REF_EXE):
        ref = subprocess.run([REF_EXE, "-g", "12x10x8", "-p", "1x1x1", "-s", "3", "-e", "1e-12", "-m", "1000", "-E",
                              arch], capture_output=True, text=True, env=dict(os.environ, SEDI_SEED="1234"),
                             timeout=600)
        theirs = [tuple(map(float, m)) for m in
                  re.findall(r"VALIDATION_ESTIMATOR: L2 error=(\S+), Linf error=(\S+)", ref.stdout)]
        np.testing.assert_allclose(np.array(ours), np.array(theirs), rtol=2e-4)  # %.4e print resolution


@pytest.mark.gpu
def test_abort_code_without_ignore():
    r = run(["-g", "16x16x16", "-p", "1x1x1", "-s", "2", "-e", "1e-12", "-m", "5", "--quiet"])
    assert r.returncode == 101 and "Incomplete convergence in solver, errcode=1" in r.stderr


@pytest.mark.gpu
def test_batched_mixed_path(tmp_path):
    d64, dmx = tmp_path / "a.bin", tmp_path / "b.bin"
    base = ["-g", "32x32x32", "-p", "1x1x1", "-s", "16", "-e", "1e-9", "-m", "2000"]
    assert run(base + ["--quiet", "--write-d", str(d64)]).returncode == 0
    r = run(base + ["--precision", "mixed", "--batch", "16", "--write-d", str(dmx)])
    assert r.returncode == 0, r.stderr
    assert O.relmax(np.fromfile(dmx), np.fromfile(d64)) <= 1e-8
