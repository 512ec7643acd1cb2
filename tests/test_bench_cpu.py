"""bench.py helpers that need no GPU: the seeded serving mix and argument checks."""
import os
import subprocess
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_serving_mix_is_seeded_and_in_range():
    a, b = bench.serve_jobs(40), bench.serve_jobs(40)
    for k in a:
        assert np.array_equal(a[k], b[k])
    assert set(a["edge"]) <= set(bench.SERVE_EDGES)
    assert a["samples"].min() >= 8 and a["samples"].max() <= 64
    assert a["tol"].min() >= 1e-10 and a["tol"].max() <= 1e-6
    assert set(a["solver"]) <= {"cg", "pcg", "bicgstab"}
    assert set(a["precision"]) <= {0, 1}
    assert len(set(a["seed"])) == 40


def test_profiling_solver_requires_no_extras():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--solver", "pcg"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0 and "--no-extras" in r.stderr
