"""Failure detection without a GPU fault.

The batched sweeps wait on copy barriers with a time limit; here a kernel
waits on a barrier that nothing completes (a flag nothing sets) and must give
up after the limit with an error status the host reads, leaving the context
usable.  Host-side failures (bad arguments, jobs that cannot fit) return the
library's error codes.
"""
import numpy as np
import pytest

import _oracle as O
import sedi_b200 as S

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable():
    timed_out, ms = S.selftest_bounded_wait(50.0)
    assert timed_out
    assert 45.0 <= ms <= 2000.0
    dims = (12, 10, 8)
    b = O.fill_probe(3, int(np.prod(dims)))
    x = np.zeros_like(b)
    with S.Context("cg", dims) as c:
        rc, fe, fi = c.solve(x, b, None, 100, 1e-10)
    assert rc == 0 and fe <= 1e-10


def test_bad_arguments_are_errors():
    with pytest.raises(S.SediError):
        S.Context("cg", (0, 4, 4))
    with S.Server() as srv:
        with pytest.raises(S.SediError):
            srv.submit("cg", (8, 8, 8), -1, 1, 10, 1e-8)
        with pytest.raises(S.SediError):
            srv.submit("cg", (8, 8, 8), 4, 1, 10, float("nan"))
