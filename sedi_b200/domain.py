"""Slab (i3) domain decomposition of the FP64 CG method across GPUs (``-p 1x1xP``).

The reference scales one grid over many processes with a block domain
decomposition (DomainDecomposition.hpp:51-80), a ghost layer refreshed by a
halo exchange before every stencil (CommHalo.hpp:84-181, overlapped with the
inner cells: DistrAsyncStencil.hpp:52-100) and dot products summed with an
allreduce (DistrAsyncDotProds.hpp:85-136).  Here the grid is cut along i3
into P slabs, one per GPU process (torchrun; NCCL moves the halos over
NVLink), or several slabs in one process on one GPU (``loopback``, halos are
device copies).

* A slab of nloc planes is stored with one ghost plane on each side,
  ``[nloc + 2][n2][n1]``; a halo is one contiguous plane, sent as is.
* Each stencil sweep starts the exchange, computes the planes that need no
  ghost (2 .. nloc-1) while it is in flight, waits, then computes planes 1 and
  nloc -- the reference's inner/border split.
* Dot products come back per plane, each summed in an order that depends only
  on (n1, n2); the planes are gathered from all slabs and added in global
  plane order with ``math.fsum``.  x, r and p are therefore identical bit for
  bit for every P, including P = 1.
* The probe of a decomposed run is the global probe (std::mt19937(seed + k)
  over the whole grid, i1 fastest); each slab fills its own range of it.  The
  reference instead fills each rank's cells from the rank's own generator
  (DistrRngStd.hpp:22-42), so its probes depend on -p.

The per-slab work runs in the CUDA library (``sedi_slab_*`` in the C ABI);
``GpuSlabBackend`` binds it.  The loop itself (``SlabCg``) only sequences
kernels and collectives, so any object with the backend's methods can run
it (the CPU tests use a NumPy one on gloo ranks).
"""
import ctypes
import math
import time

import numpy as np

__all__ = ["slab_range", "parse_decomposition", "GpuSlabBackend", "SlabCg"]

SETUP, SP, UPDATE, APPLY = 0, 1, 2, 3  # sedi_slab_sweep modes


def slab_range(n3, parts, index):
    """Planes [first, first + count) of slab `index` of `parts` along i3."""
    base, extra = divmod(int(n3), int(parts))
    first = index * base + min(index, extra)
    return first, base + (1 if index < extra else 0)


def parse_decomposition(text, n3):
    """The reference's -p P1xP2xP3 (CmdLineParser.hpp:43, :81-93) for a slab
    decomposition: P1 = P2 = 1, 1 <= P3 <= n3.  Returns P3."""
    try:
        p = [int(v) for v in str(text).lower().split("x")]
    except ValueError:
        raise ValueError(f"bad decomposition {text!r}")
    if len(p) != 3 or p[0] != 1 or p[1] != 1 or p[2] < 1:
        raise ValueError(f"decomposition {text!r}: only 1x1xP (slabs along i3) is supported")
    if p[2] > n3:
        raise ValueError(f"decomposition {text!r}: more slabs than planes ({n3})")
    return p[2]


class GpuSlabBackend:
    """Slab vectors as CUDA float64 tensors; the sweeps are the library's
    sedi_slab_* kernels on the current torch stream."""

    def __init__(self, dims, stencil=None, device=None):
        import torch
        import sedi_b200 as S
        self.torch = torch
        self.lib = S.load()
        vp, c_long, c_double, c_int = ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_int
        L = self.lib
        L.sedi_slab_sweep.argtypes = [c_int, c_long, c_long, c_long, c_double, c_double, c_double, c_long, c_long,
                                      c_double, c_double, c_int, vp, vp, vp, vp, vp, vp, vp, vp]
        L.sedi_slab_p.argtypes = [c_long, vp, vp, c_double, c_double, c_int, vp]
        L.sedi_slab_accumulate.argtypes = [c_long, vp, vp, vp, vp, c_int, vp]
        L.sedi_slab_divide.argtypes = [c_long, vp, vp, vp, vp]
        self.chunks = int(L.sedi_slab_chunks())
        self.n1, self.n2, self.n3 = (int(d) for d in dims)
        st = stencil or S.Stencil()
        self.coef = (st.a, st.b, st.c)
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._scratch = {}

    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def zeros(self, nloc):
        return self.torch.zeros((nloc + 2, self.n2, self.n1), dtype=self.torch.float64, device=self.device)

    def interior(self, buf):
        return buf[1:-1]

    def set_interior(self, buf, host):
        buf[1:-1].copy_(self.torch.from_numpy(np.ascontiguousarray(host).reshape(buf.shape[0] - 2, self.n2, self.n1)))

    def to_numpy(self, t):
        return t.detach().cpu().numpy()

    def _parts(self, nloc):
        if nloc not in self._scratch:
            self._scratch[nloc] = (self.torch.zeros(nloc * self.chunks * 2, dtype=self.torch.float64,
                                                    device=self.device),
                                   self.torch.zeros((nloc, 2), dtype=self.torch.float64, device=self.device))
        return self._scratch[nloc]

    def new_plane_part(self, nloc):
        return self.torch.zeros((nloc, 2), dtype=self.torch.float64, device=self.device)

    def sweep(self, mode, src, z_lo, z_hi, plane_part=None, x=None, r=None, b=None, y=None, iM=1.0 / 6.0,
              alpha=0.0, first=False):
        nloc = src.shape[0] - 2
        chunk, _ = self._parts(nloc)
        a, bb, c = self.coef
        rc = self.lib.sedi_slab_sweep(mode, self.n1, self.n2, nloc, a, bb, c, z_lo, z_hi, iM, alpha, int(first),
                                      self._ptr(src), self._ptr(x), self._ptr(r), self._ptr(b), self._ptr(y),
                                      self._ptr(chunk) if mode != APPLY else None,
                                      self._ptr(plane_part) if mode != APPLY else None, self._stream())
        if rc != 0:
            raise RuntimeError(f"sedi_slab_sweep failed ({rc})")

    def p_update(self, r, p, iM, beta, first):
        n = (r.shape[0] - 2) * self.n1 * self.n2
        rc = self.lib.sedi_slab_p(n, self._ptr(r[1:-1]), self._ptr(p[1:-1]), iM, beta, int(first), self._stream())
        if rc != 0:
            raise RuntimeError(f"sedi_slab_p failed ({rc})")

    def accumulate(self, x, v, t, q, reset):
        n = (x.shape[0] - 2) * self.n1 * self.n2
        rc = self.lib.sedi_slab_accumulate(n, self._ptr(x[1:-1]), self._ptr(v[1:-1]), self._ptr(t[1:-1]),
                                           self._ptr(q[1:-1]), int(reset), self._stream())
        if rc != 0:
            raise RuntimeError(f"sedi_slab_accumulate failed ({rc})")

    def divide(self, t, q, D):
        n = (t.shape[0] - 2) * self.n1 * self.n2
        rc = self.lib.sedi_slab_divide(n, self._ptr(t[1:-1]), self._ptr(q[1:-1]), self._ptr(D[1:-1]), self._stream())
        if rc != 0:
            raise RuntimeError(f"sedi_slab_divide failed ({rc})")

    def fill_probe(self, buf, seed, offset):
        import sedi_b200 as S
        count = (buf.shape[0] - 2) * self.n1 * self.n2
        host = np.empty(count)
        S.load().sedi_fill_probe_range(int(seed) & 0xFFFFFFFF, int(offset), int(count),
                                       host.ctypes.data_as(ctypes.c_void_p))
        self.set_interior(buf, host)


class SlabCg:
    """The reference CG (Cg.hpp:70-207) over i3 slabs.

    ``parts`` slabs along i3.  Under torch.distributed (``group``, every
    rank calling with the same arguments) rank r holds slab r and the world
    size must equal ``parts``; with ``loopback=True`` this process holds all
    slabs (one GPU, halos by device copies).  ``mode`` is the reference's
    sync bit set (Cg.hpp:36-40): bit 0 computes the whole slab after the
    exchange instead of overlapping the inner planes with it.
    """

    def __init__(self, dims, parts, stencil=None, group=None, backend=None, loopback=False, mode=0):
        import torch.distributed as dist
        self.dims = tuple(int(d) for d in dims)
        self.n1, self.n2, self.n3 = self.dims
        self.parts = int(parts)
        if not 1 <= self.parts <= self.n3:
            raise ValueError("1 <= parts <= n3 required")
        self.group = group
        self.dist = dist
        self.mode = int(mode)
        dist_on = dist.is_available() and dist.is_initialized() and not loopback
        self.world = dist.get_world_size(group) if dist_on else 1
        self.rank = dist.get_rank(group) if dist_on else 0
        if dist_on and self.world != self.parts:
            raise ValueError(f"-p 1x1x{self.parts} needs {self.parts} ranks, have {self.world}")
        self.local = list(range(self.parts)) if not dist_on else [self.rank]
        self.ranges = [slab_range(self.n3, self.parts, s) for s in range(self.parts)]
        self.backend = backend or GpuSlabBackend(self.dims, stencil)
        from sedi_b200 import Stencil
        self.stencil = stencil or Stencil()
        self.iM = 1.0 / self.stencil.a  # constant Jacobi preconditioner (stochastic-estimator.cc:101-103)
        self.timers = {"halo_wait": 0.0, "dot_comm": 0.0}
        self.last_history = []

    # ---- vectors -----------------------------------------------------------
    def zeros(self):
        """One zero slab vector per local slab."""
        return [self.backend.zeros(self.ranges[s][1]) for s in self.local]

    def _nloc(self, j):
        return self.ranges[self.local[j]][1]

    # ---- communication -----------------------------------------------------
    def _exchange(self, bufs):
        """Fill the ghost planes of every local slab from its neighbours
        (CommHalo.hpp:84-124: post receives, send the boundary planes).
        Returns the outstanding requests."""
        ops = []
        owner = {s: j for j, s in enumerate(self.local)}
        for j, s in enumerate(self.local):
            buf, nloc = bufs[j], self._nloc(j)
            for nb, ghost, mine in ((s - 1, 0, 1), (s + 1, nloc + 1, nloc)):
                if nb < 0 or nb >= self.parts:
                    continue
                if nb in owner:
                    jn = owner[nb]
                    src = 1 if nb > s else self._nloc(jn)  # the neighbour's plane next to this slab
                    buf[ghost].copy_(bufs[jn][src])
                else:
                    ops.append(self.dist.P2POp(self.dist.irecv, buf[ghost], nb, self.group))
                    ops.append(self.dist.P2POp(self.dist.isend, buf[mine], nb, self.group))
        return self.dist.batch_isend_irecv(ops) if ops else []

    def _wait(self, reqs):
        t0 = time.perf_counter()
        for q in reqs:
            q.wait()
        self.timers["halo_wait"] += time.perf_counter() - t0

    def _dots(self, plane_parts):
        """Global dot products from the local slabs' per-plane partials:
        gathered from every rank, added in global plane order."""
        import torch
        t0 = time.perf_counter()
        loc = torch.cat(plane_parts, 0) if len(plane_parts) > 1 else plane_parts[0]
        if self.world > 1:
            most = max(c for _, c in self.ranges)
            pad = torch.zeros((most, 2), dtype=loc.dtype, device=loc.device)
            pad[:loc.shape[0]] = loc
            got = [torch.empty_like(pad) for _ in range(self.world)]
            self.dist.all_gather(got, pad, group=self.group)
            allp = np.concatenate([self.backend.to_numpy(got[s])[:self.ranges[s][1]] for s in range(self.parts)])
        else:
            allp = self.backend.to_numpy(loc)
        self.timers["dot_comm"] += time.perf_counter() - t0
        return math.fsum(allp[:, 0].tolist()), math.fsum(allp[:, 1].tolist())

    # ---- fused stencil sweeps ----------------------------------------------
    def _stencil_sweep(self, mode, srcs, outs, **kw):
        """Exchange srcs' halos and run `mode` on every local slab: the inner
        planes while the halos move, then the border planes
        (DistrAsyncStencil.hpp:52-100); mode bit 0 = one sweep after the
        exchange (:87-97)."""
        reqs = self._exchange(srcs)
        parts = []
        overlap = not (self.mode & 1)
        for j in range(len(self.local)):
            nloc = self._nloc(j)
            pp = self.backend.new_plane_part(nloc) if mode != APPLY else None
            parts.append(pp)
            if overlap and nloc > 2:
                self.backend.sweep(mode, srcs[j], 2, nloc, pp, **{k: (v[j] if isinstance(v, list) else v)
                                                                  for k, v in kw.items()})
        self._wait(reqs)
        for j in range(len(self.local)):
            nloc = self._nloc(j)
            args = {k: (v[j] if isinstance(v, list) else v) for k, v in kw.items()}
            if overlap and nloc > 2:
                self.backend.sweep(mode, srcs[j], 1, 2, parts[j], **args)
                self.backend.sweep(mode, srcs[j], nloc, nloc + 1, parts[j], **args)
            else:
                self.backend.sweep(mode, srcs[j], 1, nloc + 1, parts[j], **args)
        return parts

    def apply(self, x, y):
        """y = A x (Stencil.hpp:38-54 through DistrAsyncStencil)."""
        self._stencil_sweep(APPLY, x, None, y=y)

    # ---- the solver --------------------------------------------------------
    def solve(self, x, b, maxiter, tol, work=None):
        """Cg::solve (Cg.hpp:70-207) with iM = 1/a: x (in: first guess, out:
        solution) and b are lists of local slab vectors.  Returns (result_t,
        final_err, final_iter)."""
        r, p = work if work is not None else (self.zeros(), self.zeros())
        hist = []
        # r = b - A x; <b,b>, <r,r> (:112-129)
        bb, rr = self._dots(self._stencil_sweep(SETUP, x, None, r=r, b=b))
        if bb == 0.0:
            bb = 1.0
        err = math.sqrt(rr / bb)
        hist.append(err)
        self.last_history = hist
        if err < tol:  # :130-134
            return 0, err, 0
        if maxiter < 1:
            return 1, err, maxiter
        ru = 0.0
        beta = 0.0
        for it in range(1, maxiter + 1):
            first = it == 1
            for j in range(len(self.local)):  # p = u + beta p, u = r .* iM (:144-147, :175, :188)
                self.backend.p_update(r[j], p[j], self.iM, beta, first)
            sp, ru1 = self._dots(self._stencil_sweep(SP, p, None, r=r, iM=self.iM, first=first))  # :152-165
            if first:
                ru = ru1
            alpha = ru / sp  # :166
            # x += alpha p, r -= alpha s, u = r .* iM; <r,u>, <r,r> (:169-182); the ghosts of p are current
            parts = []
            for j in range(len(self.local)):
                pp = self.backend.new_plane_part(self._nloc(j))
                self.backend.sweep(UPDATE, p[j], 1, self._nloc(j) + 1, pp, x=x[j], r=r[j], iM=self.iM,
                                   alpha=alpha)
                parts.append(pp)
            ru_new, rr = self._dots(parts)
            beta = ru_new / ru  # :185
            ru = ru_new
            err = math.sqrt(rr / bb)  # :191
            hist.append(err)
            if err <= tol:  # :193
                return 0, err, it
        return 1, err, maxiter  # :197-206

    def estimate(self, samples, seed=1234, maxiter=1000, tol=1e-4, ignore_errors=True):
        """The estimator loop (stochastic-estimator.cc:155-216) over the slabs:
        probe k is the global std::mt19937(seed + k) probe; x = 0 (:175);
        t += x .* v, q += v .* v (:195, :198); D = t ./ q (:216).  Returns
        dict(D, t, q: lists of local slab vectors, iters, errs, results, rc)."""
        x, b, t, q = self.zeros(), self.zeros(), self.zeros(), self.zeros()
        work = (self.zeros(), self.zeros())
        iters, errs, results = [], [], []
        rc = 0
        plane = self.n1 * self.n2
        for k in range(samples):
            for j, s in enumerate(self.local):
                self.backend.fill_probe(b[j], seed + k, self.ranges[s][0] * plane)
                x[j].zero_()
            res, fe, fi = self.solve(x, b, maxiter, tol, work)
            iters.append(fi)
            errs.append(fe)
            results.append(res)
            for j in range(len(self.local)):
                self.backend.accumulate(x[j], b[j], t[j], q[j], k == 0)
            if res != 0 and not ignore_errors:  # :181-184
                rc = res
                break
            rc = max(rc, res)
        D = self.zeros()
        if samples > 0:
            for j in range(len(self.local)):
                self.backend.divide(t[j], q[j], D[j])
        return dict(D=D, t=t, q=q, iters=np.array(iters, np.int32), errs=np.array(errs),
                    results=np.array(results, np.int32), rc=rc)

    def gather(self, vecs):
        """The global n1*n2*n3 array (numpy, i1 fastest) of slab vectors, on every rank."""
        import torch
        if self.world == 1:
            return np.concatenate([self.backend.to_numpy(self.backend.interior(v)).reshape(-1) for v in vecs])
        most = max(c for _, c in self.ranges)
        loc = self.backend.interior(vecs[0])
        pad = torch.zeros((most, self.n2, self.n1), dtype=loc.dtype, device=loc.device)
        pad[:loc.shape[0]] = loc
        got = [torch.empty_like(pad) for _ in range(self.world)]
        self.dist.all_gather(got, pad, group=self.group)
        return np.concatenate([self.backend.to_numpy(got[s])[:self.ranges[s][1]].reshape(-1)
                               for s in range(self.parts)])
