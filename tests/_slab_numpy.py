"""A NumPy stand-in for the slab kernels (test infrastructure).

It implements the interface of sedi_b200.domain.GpuSlabBackend on CPU torch
tensors so that the slab decomposition's host logic -- halo exchange, the
per-plane dot reduction, the three solver loops -- runs on gloo ranks
without a GPU.  Elementwise values round as the reference's (numpy evaluates
one operator at a time, no FMA: Stencil.hpp:43-50, SliceOps.hpp:17-108); a
plane's dot product is np.sum over the plane, the same whichever slab holds
it.  Each mode follows the sedi_slab_sweep description in
include/sedi_b200.h.
"""
import ctypes

import numpy as np
import torch

import sedi_b200 as S
from sedi_b200.domain import (APPLY, BICG_P, BICG_S, BICG_T, BICG_V, BICG_X, BICG_XR, CG_P, CG_SP, CG_UPDATE, DOTS,
                              MODE_DOTS, PCG_ITER, PCG_SETUP, SETUP)

SCALED = (PCG_SETUP, PCG_ITER, BICG_V, BICG_T)  # modes whose stencil input is src .* iM


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

    def copy(self, dst, src):
        dst.copy_(src)

    def to_numpy(self, t):
        return t.numpy()

    def plane_sums(self, n3):
        return torch.zeros((n3, DOTS), dtype=torch.float64)

    def totals(self, G):
        return tuple(G.sum(0).tolist())

    def _apply_plane(self, X, z, scale=None):
        f = (lambda k: X[k] * scale) if scale is not None else (lambda k: X[k])
        a, b, c = self.a, self.b, self.c
        xc = f(z)
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
        y = y - c * f(z - 1)
        y = y - b * xp1
        y = y - b * xp2
        y = y - b * f(z + 1)
        return y

    def sweep(self, mode, nloc, z_lo, z_hi, plane_part=None, first=False, src=None, iM=1.0 / 6.0, alpha=0.0,
              beta=0.0, bo=0.0, omega=0.0, **vec):
        V = {k: v.numpy() for k, v in vec.items() if v is not None}
        X = src.numpy() if src is not None else None
        for z in range(z_lo, z_hi):
            st = self._apply_plane(X, z, iM if mode in SCALED else None) if X is not None and mode not in (
                BICG_P, BICG_S, BICG_X, CG_P) else None
            d = [0.0] * DOTS
            if mode == APPLY:
                V["y"][z] = st
            elif mode == SETUP:
                bi = V["b"][z]
                ri = bi + (-1.0) * st
                V["r"][z] = ri
                d[0], d[1] = np.sum(bi * bi), np.sum(ri * ri)
            elif mode == CG_SP:
                d[0] = np.sum(st * X[z])
                if first:
                    rz = V["r"][z]
                    d[1] = np.sum(rz * (rz * iM))
            elif mode == CG_UPDATE:
                V["x"][z] = V["x"][z] + alpha * X[z]
                V["r"][z] = V["r"][z] + (-alpha) * st
                rz = V["r"][z]
                d[0], d[1] = np.sum(rz * (rz * iM)), np.sum(rz * rz)
            elif mode == CG_P:
                u = V["r"][z] * iM
                V["p"][z] = u if first else u + beta * V["p"][z]
            elif mode == PCG_SETUP:
                ri = X[z]
                ui = ri * iM
                V["u"][z] = ui
                V["w"][z] = st
                for k in ("q", "s", "p", "z"):
                    V[k][z] = 0.0
                d[0], d[1], d[2] = np.sum(ri * ui), np.sum(st * ui), np.sum(ri * ri)
            elif mode == PCG_ITER:
                wi = X[z]
                mi = wi * iM
                qi = mi + beta * V["q"][z]
                si = wi + beta * V["s"][z]
                u0 = V["u"][z].copy()
                pi = u0 + beta * V["p"][z]
                zi = st + beta * V["z"][z]
                ri = V["r"][z] + (-alpha) * si
                xi = V["x"][z] + alpha * pi
                ui = u0 + (-alpha) * qi
                wni = wi + (-alpha) * zi
                V["q"][z], V["s"][z], V["p"][z], V["z"][z] = qi, si, pi, zi
                V["r"][z], V["x"][z], V["u"][z], V["wn"][z] = ri, xi, ui, wni
                d[0], d[1], d[2] = np.sum(ri * ui), np.sum(wni * ui), np.sum(ri * ri)
            elif mode == BICG_P:
                ri = V["r"][z]
                V["p"][z] = ri.copy() if first else (ri + beta * V["p"][z]) + bo * V["v"][z]
            elif mode == BICG_V:
                V["v"][z] = st
                d[0] = np.sum(st * V["rhat"][z])
            elif mode == BICG_S:
                V["s"][z] = V["r"][z] + (-alpha) * V["v"][z]
            elif mode == BICG_T:
                si = X[z]
                V["t"][z] = st
                d[0], d[1], d[2] = np.sum(si * si), np.sum(st * si), np.sum(st * st)
            elif mode == BICG_XR:
                si = V["s"][z]
                phi, shi = V["p"][z] * iM, si * iM
                V["x"][z] = (V["x"][z] + alpha * phi) + omega * shi
                ri = si + (-omega) * V["t"][z]
                V["r"][z] = ri
                d[0], d[1] = np.sum(ri * ri), np.sum(ri * V["rhat"][z])
            elif mode == BICG_X:
                V["x"][z] = V["x"][z] + alpha * (V["p"][z] * iM)
            else:
                raise ValueError(mode)
            if mode in MODE_DOTS:
                plane_part.numpy()[z - 1] = d

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
