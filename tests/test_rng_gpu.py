"""Device probe generator (MT19937 on the GPU) against the reference's own
generator: bit-identical probes, and the seeded batched estimate equal to the
same estimate fed with host-generated probes."""
import numpy as np
import pytest

import _oracle as O
import sedi_b200 as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 311, 312, 313, 624, 1000, 32 ** 3])
def test_device_probes_bit_exact(n):
    import torch
    out = torch.empty((5, n), dtype=torch.float64, device="cuda")
    S.fill_probes_dev(1234, out)
    dev = out.cpu().numpy()
    for k in range(5):
        assert np.array_equal(dev[k], S.fill_probe(1234 + k, n)), (n, k)


def test_device_probes_match_reference_golden():
    import torch
    n = 32 ** 3
    out = torch.empty((5, n), dtype=torch.float64, device="cuda")
    S.fill_probes_dev(1234, out)
    bits = np.unpackbits(O.golden("probes_32")["v_bits"])[: 5 * n].reshape(5, n).astype(bool)
    assert np.array_equal(out.cpu().numpy() > 0, bits)


@pytest.mark.parametrize("prec", [S.FP64, S.MIXED])
def test_seeded_batched_estimate_equals_uploaded_probes(prec):
    dims = (24, 20, 16)
    n = int(np.prod(dims))
    samples = 20
    probes = np.stack([S.fill_probe(99 + k, n) for k in range(samples)])
    with S.Context("cg", dims, precision=prec, batch=8) as c:
        a = c.estimate(samples, 99, 1000, 1e-9)
        b = c.estimate(samples, probes=probes, maxiter=1000, tol=1e-9)
    assert np.array_equal(a["D"], b["D"]) and np.array_equal(a["iters"], b["iters"])
