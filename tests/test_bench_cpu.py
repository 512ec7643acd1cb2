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


def test_iteration_weights_of_the_deferred_cg_sweeps():
    """The mixed CG runs sweep A every iteration and the two parity forms of
    sweep B every other one: the iteration time is A + (cg_b + cg_bx) / 2."""
    mixed = [("cg_a_fp32", 4.0, 1.0), ("cg_b_fp32", 4.0, 1.0), ("cg_bx_fp32", 8.0, 2.0)]
    assert [bench.per_iteration(k[0], mixed) for k in mixed] == [1.0, 0.5, 0.5]
    fp64 = [("cg_a_fp64", 4.0, 1.0), ("cg_b_fp64", 6.0, 1.0)]
    assert [bench.per_iteration(k[0], fp64) for k in fp64] == [1.0, 1.0]


def test_traffic_lines_cover_the_bench_sweeps():
    """profiles/ncu_traffic.txt holds DRAM bytes for the mixed CG sweeps the
    bench line reports, scaled by point-lanes to the bench size."""
    small = bench.traffic_per_launch("cg_bx_fp32", (128, 128, 64), 64)
    big = bench.traffic_per_launch("cg_bx_fp32", (256, 256, 256), 128)
    assert small and big == small * 32
    for k in ("cg_a_fp32", "cg_b_fp32"):
        assert bench.traffic_per_launch(k, (256, 256, 256), 128)
