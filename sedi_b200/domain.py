"""Slab (i3) domain decomposition of the FP64 solvers across GPUs (``-p 1x1xP``).

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
  on (n1, n2), into one [n3, 3] array of all planes (a slab writes its own
  rows; across ranks the rows are summed with zeros in an all-reduce, which
  is exact); that array is then reduced over planes on the device, an order
  fixed by its shape.  Every vector of the solve is therefore identical bit
  for bit for every P, including P = 1.
* The three solvers are the reference's CG (Cg.hpp), pipelined CG
  (PipelinedCg.hpp) and BiCGStab (BiCgStab.hpp) with the constant Jacobi
  preconditioner 1/a; each sweep fuses a stencil with the elementwise updates
  and dot products around it.
* The probe of a decomposed run is the global probe (std::mt19937(seed + k)
  over the whole grid, i1 fastest); each slab fills its own range of it.  The
  reference instead fills each rank's cells from the rank's own generator
  (DistrRngStd.hpp:22-42), so its probes depend on -p.

The per-slab work runs in the CUDA library (``sedi_slab_*`` in the C ABI);
``GpuSlabBackend`` binds it.  The solver loops (``SlabCg``,
``SlabPipelinedCg``, ``SlabBiCgStab``) only sequence kernels and
collectives, so any object with the backend's methods can run them (the CPU
tests use a NumPy one on gloo ranks).
"""
import ctypes
import math
import time

import numpy as np

__all__ = ["slab_range", "parse_decomposition", "GpuSlabBackend", "SlabCg", "SlabPipelinedCg", "SlabBiCgStab",
           "slab_solver", "MODE_DOTS"]

# sedi_slab_sweep modes (include/sedi_b200.h)
(SETUP, CG_SP, CG_UPDATE, APPLY, PCG_SETUP, PCG_ITER, BICG_P, BICG_V, BICG_S, BICG_T, BICG_XR, BICG_X,
 CG_P) = range(13)
MODE_DOTS = {SETUP: 2, CG_SP: 2, CG_UPDATE: 2, PCG_SETUP: 3, PCG_ITER: 3, BICG_V: 1, BICG_T: 3, BICG_XR: 2}
DOTS = 3  # dot products per plane in a plane_part row
VECTORS = ("src", "b", "rhat", "x", "r", "y", "u", "w", "wn", "q", "s", "p", "z", "v", "t")
SCALARS = ("iM", "alpha", "beta", "bo", "omega")


def _fdiv(a, b):
    """a / b with IEEE semantics (inf or nan on a zero divisor), as the reference's C++ divides."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float64(a) / np.float64(b))


def _sqrt(a):
    return math.sqrt(a) if a >= 0.0 else float("nan")


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


class _SlabArgs(ctypes.Structure):
    """sedi_slab_args (include/sedi_b200.h)."""
    _fields_ = ([(n, ctypes.c_void_p) for n in VECTORS] + [(n, ctypes.c_double) for n in SCALARS]
                + [("first", ctypes.c_int)])


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
                                      ctypes.POINTER(_SlabArgs), vp, vp, vp]
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

    def copy(self, dst, src):
        dst.copy_(src)

    def to_numpy(self, t):
        return t.detach().cpu().numpy()

    def _chunk(self, nloc):
        if nloc not in self._scratch:
            self._scratch[nloc] = self.torch.zeros(nloc * self.chunks * DOTS, dtype=self.torch.float64,
                                                   device=self.device)
        return self._scratch[nloc]

    def plane_sums(self, n3):
        """The [n3, 3] per-plane dot products of every slab."""
        return self.torch.zeros((n3, DOTS), dtype=self.torch.float64, device=self.device)

    def totals(self, G):
        """The three dot products: G summed over planes (device reduction of a
        fixed shape, so of a fixed order), read back once."""
        return tuple(G.sum(0).tolist())

    def sweep(self, mode, nloc, z_lo, z_hi, plane_part=None, first=False, **kw):
        """sedi_slab_sweep over ghosted planes [z_lo, z_hi): vectors (slab
        tensors) and scalars by their sedi_slab_args names."""
        args = _SlabArgs()
        for k, v in kw.items():
            if k in SCALARS:
                setattr(args, k, float(v))
            elif v is not None:
                setattr(args, k, v.data_ptr())
        args.first = int(bool(first))
        dots = mode in MODE_DOTS
        a, bb, c = self.coef
        rc = self.lib.sedi_slab_sweep(mode, self.n1, self.n2, nloc, a, bb, c, z_lo, z_hi, ctypes.byref(args),
                                      self._ptr(self._chunk(nloc)) if dots else None,
                                      self._ptr(plane_part) if dots else None, self._stream())
        if rc != 0:
            raise RuntimeError(f"sedi_slab_sweep mode {mode} failed ({rc})")

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


class _SlabSolver:
    """Slab storage, halo exchange, plane-ordered dot products and the
    estimator loop shared by the three solvers.

    ``parts`` slabs along i3.  Under torch.distributed (``group``, every
    rank calling with the same arguments) rank r holds slab r and the world
    size must equal ``parts``; with ``loopback=True`` this process holds all
    slabs (one GPU, halos by device copies).  ``mode`` is the reference's
    sync bit set (Cg.hpp:36-40, PipelinedCg.hpp:33-37, BiCgStab.hpp:36-40):
    bit 0 computes the whole slab after the exchange instead of overlapping
    the inner planes with it.
    """

    NAME = ""
    WORK = ()  # names of the work vectors of one solve

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
        self._G = self.backend.plane_sums(self.n3)

    # ---- vectors -----------------------------------------------------------
    def zeros(self):
        """One zero slab vector per local slab."""
        return [self.backend.zeros(self.ranges[s][1]) for s in self.local]

    def work(self):
        """The work vectors of one solve, by name."""
        return {k: self.zeros() for k in self.WORK}

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
                    self.backend.copy(buf[ghost], bufs[jn][src])
                else:
                    ops.append(self.dist.P2POp(self.dist.irecv, buf[ghost], nb, self.group))
                    ops.append(self.dist.P2POp(self.dist.isend, buf[mine], nb, self.group))
        return self.dist.batch_isend_irecv(ops) if ops else []

    def _wait(self, reqs):
        t0 = time.perf_counter()
        for q in reqs:
            q.wait()
        self.timers["halo_wait"] += time.perf_counter() - t0

    def _plane_part(self, j):
        """Rows of the global per-plane array that local slab j writes."""
        first, count = self.ranges[self.local[j]]
        return self._G[first:first + count]

    def _dots(self):
        """The three global dot products of a sweep from the per-plane array:
        across ranks the rows of the other slabs are zero here, so an
        all-reduce assembles it exactly (DistrAsyncDotProds.hpp:85-136 sums
        rank partials with an allreduce); then one reduction over all n3
        planes on the device, whose order depends only on n3."""
        t0 = time.perf_counter()
        if self.world > 1:
            self.dist.all_reduce(self._G, group=self.group)
        tot = self.backend.totals(self._G)
        self.timers["dot_comm"] += time.perf_counter() - t0
        return tot

    # ---- sweeps --------------------------------------------------------------
    def _args(self, kw, j):
        return {k: (v[j] if isinstance(v, list) else v) for k, v in kw.items()}

    def _sweep(self, mode, **kw):
        """`mode` over every plane of every local slab, no exchange (an
        elementwise mode, or a stencil whose source's ghosts are current).
        Returns the mode's three global dot products (None without dots)."""
        dots = mode in MODE_DOTS
        if dots and self.world > 1:
            self._G.zero_()
        for j in range(len(self.local)):
            nloc = self._nloc(j)
            self.backend.sweep(mode, nloc, 1, nloc + 1, self._plane_part(j) if dots else None, **self._args(kw, j))
        return self._dots() if dots else None

    def _stencil_sweep(self, mode, src, **kw):
        """Exchange src's halos and run `mode` on every local slab: the inner
        planes while the halos move, then the border planes
        (DistrAsyncStencil.hpp:52-100); mode bit 0 = one sweep after the
        exchange (:87-97).  Returns the mode's three global dot products
        (None without dots)."""
        reqs = self._exchange(src)
        kw["src"] = src
        dots = mode in MODE_DOTS
        if dots and self.world > 1:
            self._G.zero_()
        parts = [self._plane_part(j) if dots else None for j in range(len(self.local))]
        # Only halos from other ranks are in flight; a process's own slabs get
        # theirs by copies already queued before the sweep.
        overlap = not (self.mode & 1) and self.world > 1
        for j in range(len(self.local)):
            nloc = self._nloc(j)
            if overlap and nloc > 2:
                self.backend.sweep(mode, nloc, 2, nloc, parts[j], **self._args(kw, j))
        self._wait(reqs)
        for j in range(len(self.local)):
            nloc = self._nloc(j)
            args = self._args(kw, j)
            if overlap and nloc > 2:
                self.backend.sweep(mode, nloc, 1, 2, parts[j], **args)
                self.backend.sweep(mode, nloc, nloc, nloc + 1, parts[j], **args)
            else:
                self.backend.sweep(mode, nloc, 1, nloc + 1, parts[j], **args)
        return self._dots() if dots else None

    def apply(self, x, y):
        """y = A x (Stencil.hpp:38-54 through DistrAsyncStencil)."""
        self._stencil_sweep(APPLY, x, y=y)

    def _residual(self, x, b, r):
        """r = b - A x; returns (<b,b> with 0 taken as 1, <r,r>) -- the common
        start of the three solvers (Cg.hpp:112-129, PipelinedCg.hpp:104-123,
        BiCgStab.hpp:122-139)."""
        bb, rr, _ = self._stencil_sweep(SETUP, x, r=r, b=b)
        return (1.0 if bb == 0.0 else bb), rr

    def solve(self, x, b, maxiter, tol, work=None):
        raise NotImplementedError

    # ---- the estimator -------------------------------------------------------
    def estimate(self, samples, seed=1234, maxiter=1000, tol=1e-4, ignore_errors=True):
        """The estimator loop (stochastic-estimator.cc:155-216) over the slabs:
        probe k is the global std::mt19937(seed + k) probe; x = 0 (:175);
        t += x .* v, q += v .* v (:195, :198); D = t ./ q (:216).  Returns
        dict(D, t, q: lists of local slab vectors, iters, errs, results, rc)."""
        x, b, t, q = self.zeros(), self.zeros(), self.zeros(), self.zeros()
        work = self.work()
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


class SlabCg(_SlabSolver):
    """The reference CG (Cg.hpp:70-207) over i3 slabs."""

    NAME = "Cg"
    WORK = ("r", "p")

    def solve(self, x, b, maxiter, tol, work=None):
        """Cg::solve with iM = 1/a: x (in: first guess, out: solution) and b
        are lists of local slab vectors.  Returns (result_t, final_err,
        final_iter)."""
        w = work if work is not None else self.work()
        r, p = w["r"], w["p"]
        bb, rr = self._residual(x, b, r)
        err = _sqrt(_fdiv(rr, bb))
        hist = [err]
        self.last_history = hist
        if err < tol:  # :130-134
            return 0, err, 0
        if maxiter < 1:
            return 1, err, maxiter
        ru = 0.0
        beta = 0.0
        for it in range(1, maxiter + 1):
            first = it == 1
            self._sweep(CG_P, r=r, p=p, iM=self.iM, beta=beta, first=first)  # p = u + beta p (:144-147, :188)
            sp, ru1, _ = self._stencil_sweep(CG_SP, p, r=r, iM=self.iM, first=first)  # :152-165
            if first:
                ru = ru1
            alpha = _fdiv(ru, sp)  # :166
            # x += alpha p, r -= alpha s, u = r .* iM; <r,u>, <r,r> (:169-182); the ghosts of p are current
            ru_new, rr, _ = self._sweep(CG_UPDATE, src=p, x=x, r=r, iM=self.iM, alpha=alpha)
            beta = _fdiv(ru_new, ru)  # :185
            ru = ru_new
            err = _sqrt(_fdiv(rr, bb))  # :191
            hist.append(err)
            if err <= tol:  # :193
                return 0, err, it
        return 1, err, maxiter  # :197-206


class SlabPipelinedCg(_SlabSolver):
    """The reference pipelined CG (PipelinedCg.hpp:75-243) over i3 slabs.

    One fused sweep per iteration: m = w .* iM and n = A m on the fly, the
    eight vector updates, and the next iteration's <r,u>, <w,u>, <r,r> -- the
    reference computes those dots at the top of the next iteration from the
    same vectors (:152-180).  w is double-buffered because the stencil reads
    the neighbours' w while the update writes it.
    """

    NAME = "PipelinedCg"
    WORK = ("r", "u", "w", "wn", "q", "s", "p", "z")

    def solve(self, x, b, maxiter, tol, work=None):
        W = work if work is not None else self.work()
        r, u, q, s, p, z = (W[k] for k in ("r", "u", "q", "s", "p", "z"))
        w, wn = W["w"], W["wn"]
        bb, rr = self._residual(x, b, r)
        err = _sqrt(_fdiv(rr, bb))
        hist = [err]
        self.last_history = hist
        if err < tol:  # :124-128
            return 0, err, 0
        # u = r .* iM, w = A u, z = q = s = p = 0 (:138-149); dots of iteration 1 (:155, :169-172)
        gamma, delta, rr = self._stencil_sweep(PCG_SETUP, r, u=u, w=w, q=q, s=s, p=p, z=z, iM=self.iM)
        alpha = beta = 0.0
        for it in range(1, maxiter + 1):
            if it > 1:  # :175-181
                beta = _fdiv(gamma, gamma_old)
                alpha = _fdiv(1.0, _fdiv(delta, gamma) - _fdiv(beta, alpha))
            else:
                beta = 0.0
                alpha = _fdiv(gamma, delta)
            gamma_old = gamma
            rr_it = rr
            gamma, delta, rr = self._stencil_sweep(PCG_ITER, w, x=x, r=r, u=u, wn=wn, q=q, s=s, p=p, z=z,
                                                   iM=self.iM, alpha=alpha, beta=beta)
            w, wn = wn, w
            err = _sqrt(_fdiv(rr_it, bb))  # :227 (the <r,r> of the iteration's start)
            hist.append(err)
            if err <= tol:  # :229
                return 0, err, it
        return 1, err, maxiter  # :233-242


class SlabBiCgStab(_SlabSolver):
    """The reference BiCGStab (BiCgStab.hpp:75-263) over i3 slabs."""

    NAME = "BiCgStab"
    WORK = ("r", "rhat", "p", "v", "s", "t")

    def solve(self, x, b, maxiter, tol, work=None):
        W = work if work is not None else self.work()
        r, rhat, p, v, s, t = (W[k] for k in self.WORK)
        iM = self.iM
        bb, rr = self._residual(x, b, r)
        err = _sqrt(_fdiv(rr, bb))
        hist = [err]
        self.last_history = hist
        if err < tol:  # :142-146
            return 0, err, 0
        omega, alpha, rho_prev = 1.0, 0.0, 0.0  # :148-151
        for j in range(len(self.local)):
            self.backend.copy(rhat[j], r[j])  # :154
        rho_next = rr  # <r, r_hat> with r_hat = r: the same sums as <r,r>
        s_norm2 = 0.0
        it = maxiter + 1
        for k in range(1, maxiter + 1):
            rho = rho_next  # :160-161
            if rho == 0.0:  # :163
                it = k
                break
            if k > 1:
                beta = _fdiv(rho, rho_prev) * _fdiv(alpha, omega)  # :167
                self._sweep(BICG_P, r=r, p=p, v=v, beta=beta, bo=-beta * omega)  # :169
            else:
                self._sweep(BICG_P, r=r, p=p, first=True)  # :172
            vr, _, _ = self._stencil_sweep(BICG_V, p, v=v, rhat=rhat, iM=iM)  # :176-186
            alpha = _fdiv(rho, vr)  # :187
            self._sweep(BICG_S, r=r, v=v, s=s, alpha=alpha)  # :190
            # t = A (s .* iM) with <s,s>, <t,s>, <t,t>: t is computed before the
            # early-exit test on <s,s> (:193-199) and unused when it exits.
            ss, ts, tt = self._stencil_sweep(BICG_T, s, t=t, iM=iM)
            s_norm2 = ss
            if ss < tol * tol:  # :195
                self._sweep(BICG_X, x=x, p=p, alpha=alpha, iM=iM)  # :197
                it = k
                break
            omega = _fdiv(ts, tt)  # :213
            rr, rho_next, _ = self._sweep(BICG_XR, x=x, p=p, s=s, t=t, r=r, rhat=rhat, alpha=alpha,
                                            omega=omega, iM=iM)  # :217-224
            err = _sqrt(_fdiv(rr, bb))  # :227
            hist.append(err)
            if err <= tol:  # :229
                it = k
                break
            if omega == 0.0:  # :230
                it = k
                break
            rho_prev = rho  # :232
        if err <= tol:  # :236-240
            return 0, err, it
        if s_norm2 <= tol * tol:  # :242-246
            return 0, _sqrt(_fdiv(s_norm2, bb)), it
        if omega == 0.0:  # :248-252
            return 3, err, it
        if rho == 0.0:  # :254-258
            return 2, err, it
        return 1, err, maxiter  # :260-263


SOLVERS = {"cg": SlabCg, "pcg": SlabPipelinedCg, "pipelined_cg": SlabPipelinedCg, "bicgstab": SlabBiCgStab,
           2: SlabCg, 3: SlabPipelinedCg, 1: SlabBiCgStab}


def slab_solver(solver, dims, parts, **kw):
    """A slab solver by name ("cg", "pcg", "bicgstab") or the library's
    solver id (SEDI_CG, SEDI_PIPELINED_CG, SEDI_BICGSTAB)."""
    try:
        cls = SOLVERS[solver.lower() if isinstance(solver, str) else int(solver)]
    except KeyError:
        raise ValueError(f"unknown solver {solver!r}")
    return cls(dims, parts, **kw)
