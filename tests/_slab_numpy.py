"""A NumPy stand-in for the slab kernels (test infrastructure).

It implements the interface of sedi_b200.domain.GpuSlabBackend on CPU torch
tensors so that the slab decomposition's host logic -- halo exchange, the
plane-ordered dot reduction, the CG loop -- runs on gloo ranks without a GPU.
Elementwise values round as the reference's (numpy evaluates one operator at
a time, no FMA: Stencil.hpp:43-50, SliceOps.hpp:17-108); a plane's dot
product is np.sum over the plane, the same whichever slab holds it.
"""
import ctypes

import numpy as np
import torch

import sedi_b200 as S
from sedi_b200.domain import APPLY, SETUP, SP, UPDATE


class NumpySlabBackend:
    def __init__(self, dims, stencil=None):
        self.n1, self.n2, self.n3 = (int(d) for d in dims)
        st = stencil or S.Stencil()
        self.a, self.b, self.c = st.a, st.b, st.c

    def zeros(self, nloc):
        return torch.zeros((nloc + 2, self.n2, self.n1), dtype=torch.float64)

    def interior(self, buf):
        return buf[1:-1]

    def set_interior(self, buf, host):
        buf[1:-1].copy_(torch.from_numpy(np.ascontiguousarray(host).reshape(buf.shape[0] - 2, self.n2, self.n1)))

    def to_numpy(self, t):
        return t.numpy()

    def new_plane_part(self, nloc):
        return torch.zeros((nloc, 2), dtype=torch.float64)

    def _apply_plane(self, X, z):
        a, b, c = self.a, self.b, self.c
        xc = X[z]
        xm1 = np.zeros_like(xc)
        xm1[:, 1:] = xc[:, :-1]
        xp1 = np.zeros_like(xc)
        xp1[:, :-1] = xc[:, 1:]
        xm2 = np.zeros_like(xc)
        xm2[1:, :] = xc[:-1, :]
        xp2 = np.zeros_like(xc)
        xp2[:-1, :] = xc[1:, :]
        y = a * xc
        y = y - c * xm1
        y = y - c * xm2
        y = y - c * X[z - 1]
        y = y - b * xp1
        y = y - b * xp2
        y = y - b * X[z + 1]
        return y

    def sweep(self, mode, src, z_lo, z_hi, plane_part=None, x=None, r=None, b=None, y=None, iM=1.0 / 6.0,
              alpha=0.0, first=False):
        X = src.numpy()
        for z in range(z_lo, z_hi):
            s = self._apply_plane(X, z)
            if mode == APPLY:
                y.numpy()[z] = s
                continue
            if mode == SETUP:
                bi = b.numpy()[z]
                ri = bi + (-1.0) * s
                r.numpy()[z] = ri
                d0, d1 = np.sum(bi * bi), np.sum(ri * ri)
            elif mode == SP:
                d0 = np.sum(s * X[z])
                d1 = np.sum(r.numpy()[z] * (r.numpy()[z] * iM)) if first else 0.0
            else:
                xv, rv = x.numpy(), r.numpy()
                xv[z] = xv[z] + alpha * X[z]
                rv[z] = rv[z] + (-alpha) * s
                d0, d1 = np.sum(rv[z] * (rv[z] * iM)), np.sum(rv[z] * rv[z])
            plane_part.numpy()[z - 1] = (d0, d1)

    def p_update(self, r, p, iM, beta, first):
        u = r.numpy()[1:-1] * iM
        pv = p.numpy()
        pv[1:-1] = u if first else u + beta * pv[1:-1]

    def accumulate(self, x, v, t, q, reset):
        xv, vv, tv, qv = x.numpy()[1:-1], v.numpy()[1:-1], t.numpy()[1:-1], q.numpy()[1:-1]
        if reset:
            tv[:] = 0.0 + xv * vv
            qv[:] = 0.0 + vv * vv
        else:
            tv[:] = tv + xv * vv
            qv[:] = qv + vv * vv

    def divide(self, t, q, D):
        D.numpy()[1:-1] = t.numpy()[1:-1] / q.numpy()[1:-1]

    def fill_probe(self, buf, seed, offset):
        count = (buf.shape[0] - 2) * self.n1 * self.n2
        host = np.empty(count)
        S.load().sedi_fill_probe_range(int(seed) & 0xFFFFFFFF, int(offset), int(count),
                                       host.ctypes.data_as(ctypes.c_void_p))
        self.set_interior(buf, host)
