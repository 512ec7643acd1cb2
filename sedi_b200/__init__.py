"""sedi_b200 -- B200-native SEDI estimator hot path (host-side Python mirror).

The compute path is the CUDA library ``sedi_b200/_lib/libsedi_b200.so``
(C ABI in ``include/sedi_b200.h``); this module binds it with ctypes and
mirrors the reference solver interface so a caller written against the
reference reads the same:

    reference (C++)                                   here
    Stencil<real_t> stencil(6.0, 1.0, 1.0)            Stencil(6.0, 1.0, 1.0)
    Cg<real_t> solver(dd, nghost, mode, &timers)      Cg((n1, n2, n3), nghost=1, mode=0)
    solver.solve(stencil, comm_halo, x, b, iM,        res, err, it = solver.solve(stencil, None, x, b, iM,
                 maxiter, tol, &final_err, &iter)                               maxiter, tol)

(Cg.hpp:48-82, PipelinedCg.hpp:48-84, BiCgStab.hpp:55-89).  ``x``, ``b``,
``iM`` are dense n1*n2*n3 float64 arrays, i1 fastest (numpy arrays, or torch
CUDA tensors for the device-pointer path); ``iM`` may be None for the
constant 1/a of stochastic-estimator.cc:103.  ``x`` is updated in place.
Result codes are the reference's result_t values.

There is no CPU fallback: if the native library is missing or no CUDA device
is present, calls raise ``SediError``.
"""
import ctypes
import os

import numpy as np

__all__ = [
    "SediError", "Stencil", "Cg", "PipelinedCg", "BiCgStab", "Context", "Server", "autotune", "set_tuning", "estimate",
    "fill_probe",
    "job_bytes", "library_path", "load", "SOLVER_IDS", "FP64", "MIXED",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_lib", "libsedi_b200.so")

BICGSTAB, CG, PIPELINED_CG = 1, 2, 3
SOLVER_IDS = {"bicgstab": BICGSTAB, "cg": CG, "pcg": PIPELINED_CG, "pipelined_cg": PIPELINED_CG}
FP64, MIXED = 0, 1

ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "device out of memory", -4: "no CUDA device",
          -5: "unsupported"}

_lib = None


class SediError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"sedi_b200 error {code} ({ERRORS.get(code, '?')}){': ' + msg if msg else ''}")


def library_path():
    return _LIB_PATH


def load():
    """Load the native library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise SediError(-4, f"native library missing: {_LIB_PATH} (run python -m sedi_b200.build)")
    lib = ctypes.CDLL(_LIB_PATH)
    c_int, c_long, c_double, vp = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_void_p
    pi, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    lib.sedi_create.restype = vp
    lib.sedi_create.argtypes = [c_int, c_long, c_long, c_long, c_double, c_double, c_double, c_int, c_int, c_int, pi]
    lib.sedi_destroy.argtypes = [vp]
    lib.sedi_destroy.restype = None
    lib.sedi_ctx_error.argtypes = [vp]
    lib.sedi_ctx_error.restype = ctypes.c_char_p
    lib.sedi_solve.argtypes = [vp, vp, vp, vp, c_int, c_double, pd, pi]
    lib.sedi_solve_dev.argtypes = [vp, vp, vp, vp, c_int, c_double, pd, pi]
    lib.sedi_solve_batch.argtypes = [vp, c_int, vp, vp, c_int, c_double, vp, vp, vp]
    lib.sedi_estimate.argtypes = [vp, c_int, ctypes.c_uint32, c_int, c_double, c_int, vp, vp, vp, vp, vp, vp]
    lib.sedi_estimate_probes.argtypes = [vp, c_int, vp, c_int, c_double, c_int, vp, vp, vp, vp, vp, vp]
    lib.sedi_fill_probe.argtypes = [ctypes.c_uint32, c_long, vp]
    lib.sedi_fill_probe.restype = None
    lib.sedi_stencil_apply.argtypes = [vp, vp, vp]
    lib.sedi_last_history.argtypes = [vp, vp, c_int]
    lib.sedi_launch_count.argtypes = [vp]
    lib.sedi_launch_count.restype = ctypes.c_longlong
    lib.sedi_version.restype = ctypes.c_char_p
    lib.sedi_estimate_dev.argtypes = [vp, c_int, vp, c_int, c_double, c_int, vp, vp, vp, vp, vp, vp]
    lib.sedi_set_stream.argtypes = [vp, vp]
    lib.sedi_time_kernels.argtypes = [vp, c_int, vp, vp, vp, vp]
    lib.sedi_fill_probes_dev.argtypes = [ctypes.c_uint32, c_int, c_long, vp, vp]
    lib.sedi_residual_noalloc.argtypes = [c_long, c_long, c_long, c_double, c_double, c_double, vp, vp, vp, pd, vp]
    lib.sedi_server_create.restype = vp
    lib.sedi_server_create.argtypes = [c_double, c_int, c_double, pi]
    lib.sedi_server_destroy.argtypes = [vp]
    lib.sedi_server_destroy.restype = None
    lib.sedi_server_submit.restype = c_long
    lib.sedi_server_submit.argtypes = [vp, c_int, c_int, c_long, c_long, c_long, c_int, ctypes.c_uint32, c_int,
                                       c_double]
    lib.sedi_server_step.argtypes = [vp, pi]
    lib.sedi_server_wait.argtypes = [vp, c_long]
    lib.sedi_server_job_info.argtypes = [vp, c_long, pi, pi, pd, pd, pd, pi, pd]
    lib.sedi_server_take.argtypes = [vp, c_long, vp, vp, vp, vp]
    lib.sedi_server_replay.argtypes = [vp, c_int, vp, vp, vp, vp, vp, vp, vp, c_int, vp, vp, pd, vp]
    lib.sedi_server_stats.argtypes = [vp, pd, pd, pi, pi, pi, ctypes.POINTER(ctypes.c_longlong)]
    lib.sedi_autotune.argtypes = [c_int, c_int, c_int, c_long, c_long, c_long, c_int, c_double, ctypes.c_uint32,
                                  c_int, vp, pd]
    lib.sedi_ctx_config.argtypes = [vp, vp]
    lib.sedi_set_tuning.argtypes = [c_int, c_int, c_int, c_long, c_long, c_long, vp]
    lib.sedi_set_mixed_target.argtypes = [vp, c_double]
    lib.sedi_mixed_target.argtypes = [vp]
    lib.sedi_mixed_target.restype = c_double
    lib.sedi_selftest_bounded_wait.argtypes = [c_double, pi, pd]
    lib.sedi_job_bytes.restype = c_double
    lib.sedi_job_bytes.argtypes = [c_int, c_int, c_int, c_long, c_long, c_long]
    _lib = lib
    return lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p)
    return ctypes.c_void_p(int(a.data_ptr()))  # torch tensor


def _host_f64(a, n, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous or a.size != n:
        raise ValueError(f"{name} must be a C-contiguous float64 array of {n} elements")
    return a


def _is_device(a):
    return a is not None and not isinstance(a, np.ndarray) and hasattr(a, "data_ptr") and a.is_cuda


def fill_probe(seed, n):
    """DistrRngStd::fill_plusminusone with std::mt19937(seed) (DistrRngStd.hpp:22-42)."""
    out = np.empty(int(n), np.float64)
    load().sedi_fill_probe(int(seed) & 0xFFFFFFFF, int(n), _ptr(out))
    return out


def fill_probes_dev(seed, out, stream=None):
    """Device generator: fills the CUDA float64 tensor out (nprobes, n) with
    probes seed, seed+1, ... (bit-identical to fill_probe)."""
    nprobes, n = out.shape
    handle = None if stream is None else int(getattr(stream, "cuda_stream", stream))
    rc = load().sedi_fill_probes_dev(int(seed) & 0xFFFFFFFF, int(nprobes), int(n), _ptr(out),
                                     ctypes.c_void_p(handle) if handle else None)
    if rc < 0:
        raise SediError(rc, "fill_probes_dev")
    return out


class Stencil:
    """Stencil<Dtype>(a, b, c) (Stencil.hpp:12-19): y = a x_c - c (x_{i-1}...) - b (x_{i+1}...)."""

    def __init__(self, a=6.0, b=1.0, c=1.0):
        self.a, self.b, self.c = float(a), float(b), float(c)


class Context:
    """One solver context on the current CUDA device (sedi_create / sedi_destroy)."""

    def __init__(self, solver, dims, stencil=None, mode=0, precision=FP64, batch=1):
        lib = load()
        if isinstance(solver, str):
            solver = SOLVER_IDS[solver.lower()]
        self.solver = int(solver)
        self.dims = tuple(int(d) for d in dims)
        if len(self.dims) != 3:
            raise ValueError("dims must be (n1, n2, n3)")
        self.n = self.dims[0] * self.dims[1] * self.dims[2]
        self.stencil = stencil or Stencil()
        self.precision = precision
        self.batch = int(batch)
        err = ctypes.c_int(0)
        s = self.stencil
        self._h = lib.sedi_create(self.solver, *self.dims, s.a, s.b, s.c, int(mode), int(precision), self.batch,
                                  ctypes.byref(err))
        if not self._h:
            raise SediError(err.value, "sedi_create")

    def close(self):
        if getattr(self, "_h", None):
            load().sedi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc < 0:
            raise SediError(rc, f"{what}: {load().sedi_ctx_error(self._h).decode()}")
        return rc

    @property
    def launches(self):
        return int(load().sedi_launch_count(self._h))

    def config(self):
        """Launch choices of a batched context (see autotune)."""
        cf = np.zeros(7, np.int32)
        self._check(load().sedi_ctx_config(self._h, _ptr(cf)), "config")
        return {"slice_width": int(cf[0]), "z_chunks": int(cf[1]), "period": int(cf[2]), "chunk": int(cf[3]),
                "lanes": int(cf[4]), "prefetch_planes": int(cf[5]), "sweep_a_form": int(cf[6])}

    @property
    def mixed_target(self):
        """theta of the mixed form: lanes stop on FP64 true residual <= theta * tol."""
        return float(load().sedi_mixed_target(self._h))

    @mixed_target.setter
    def mixed_target(self, theta):
        self._check(load().sedi_set_mixed_target(self._h, float(theta)), "mixed_target")

    def solve(self, x, b, iM=None, maxiter=1000, tol=1e-4):
        """Returns (result_t, final_err, final_iter); x is overwritten with the solution."""
        lib = load()
        fe, fi = ctypes.c_double(0.0), ctypes.c_int(0)
        if _is_device(x) or _is_device(b):
            for t, nm in ((x, "x"), (b, "b"), (iM, "iM")):
                if t is not None and (not _is_device(t) or t.numel() != self.n or not t.is_contiguous()
                                      or str(t.dtype) != "torch.float64"):
                    raise ValueError(f"{nm} must be a contiguous float64 CUDA tensor of {self.n} elements")
            rc = lib.sedi_solve_dev(self._h, _ptr(b), _ptr(x), _ptr(iM), int(maxiter), float(tol),
                                    ctypes.byref(fe), ctypes.byref(fi))
        else:
            _host_f64(x, self.n, "x")
            _host_f64(b, self.n, "b")
            if iM is not None:
                _host_f64(iM, self.n, "iM")
            rc = lib.sedi_solve(self._h, _ptr(b), _ptr(x), _ptr(iM), int(maxiter), float(tol),
                                ctypes.byref(fe), ctypes.byref(fi))
        self._check(rc, "solve")
        return rc, fe.value, fi.value

    def solve_batch(self, x, b, maxiter=1000, tol=1e-4):
        """x, b: (nrhs, n) float64.  Returns (results, final_errs, final_iters) arrays."""
        b = np.ascontiguousarray(b, np.float64).reshape(-1, self.n)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous
                and x.size == b.size):
            raise ValueError("x must be a C-contiguous float64 array shaped like b")
        nrhs = b.shape[0]
        res = np.zeros(nrhs, np.int32)
        fe = np.zeros(nrhs, np.float64)
        fi = np.zeros(nrhs, np.int32)
        rc = load().sedi_solve_batch(self._h, nrhs, _ptr(b), _ptr(x), int(maxiter), float(tol), _ptr(fe),
                                     _ptr(fi), _ptr(res))
        self._check(rc, "solve_batch")
        return res, fe, fi

    def estimate(self, samples, seed=1234, maxiter=1000, tol=1e-4, ignore_errors=True, probes=None):
        """Estimator loop; returns dict(D, t, q, iters, errs, results, rc)."""
        n = self.n
        D, t, q = np.empty(n), np.empty(n), np.empty(n)
        iters = np.zeros(samples, np.int32)
        errs = np.zeros(samples, np.float64)
        results = np.zeros(samples, np.int32)
        lib = load()
        if probes is None:
            rc = lib.sedi_estimate(self._h, int(samples), int(seed) & 0xFFFFFFFF, int(maxiter), float(tol),
                                   int(bool(ignore_errors)), _ptr(D), _ptr(t), _ptr(q), _ptr(iters), _ptr(errs),
                                   _ptr(results))
        else:
            probes = np.ascontiguousarray(probes, np.float64).reshape(samples, n)
            rc = lib.sedi_estimate_probes(self._h, int(samples), _ptr(probes), int(maxiter), float(tol),
                                          int(bool(ignore_errors)), _ptr(D), _ptr(t), _ptr(q), _ptr(iters),
                                          _ptr(errs), _ptr(results))
        self._check(rc, "estimate")
        return dict(D=D, t=t, q=q, iters=iters, errs=errs, results=results, rc=rc)

    def set_stream(self, stream):
        """Run on a caller stream (torch.cuda.Stream, cudaStream_t int, or None)."""
        handle = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        self._check(load().sedi_set_stream(self._h, ctypes.c_void_p(handle) if handle else None), "set_stream")

    def estimate_dev(self, samples, probes, D, t=None, q=None, maxiter=1000, tol=1e-4, ignore_errors=True):
        """Estimator on device buffers (torch CUDA float64 tensors): probes (samples, n), D (n,)."""
        iters = np.zeros(samples, np.int32)
        errs = np.zeros(samples, np.float64)
        results = np.zeros(samples, np.int32)
        rc = load().sedi_estimate_dev(self._h, int(samples), _ptr(probes), int(maxiter), float(tol),
                                      int(bool(ignore_errors)), _ptr(D), _ptr(t), _ptr(q), _ptr(iters), _ptr(errs),
                                      _ptr(results))
        self._check(rc, "estimate_dev")
        return dict(iters=iters, errs=errs, results=results, rc=rc)

    def time_kernels(self, reps=10):
        """Per-iteration kernels timed in isolation: list of (name, ms per launch, algorithmic bytes)."""
        ms = np.zeros(8)
        by = np.zeros(8)
        names = ctypes.create_string_buffer(8 * 32)
        cnt = ctypes.c_int(0)
        self._check(load().sedi_time_kernels(self._h, int(reps), _ptr(ms), _ptr(by), names, ctypes.byref(cnt)),
                    "time_kernels")
        raw = names.raw
        return [(raw[32 * k: 32 * k + 32].split(b"\0")[0].decode(), float(ms[k]), float(by[k]))
                for k in range(cnt.value)]

    def stencil_apply(self, x):
        x = _host_f64(np.ascontiguousarray(x, np.float64).reshape(-1), self.n, "x")
        y = np.empty_like(x)
        self._check(load().sedi_stencil_apply(self._h, _ptr(x), _ptr(y)), "stencil_apply")
        return y

    def history(self, length=None):
        length = length or 100000
        h = np.empty(length, np.float64)
        k = self._check(load().sedi_last_history(self._h, _ptr(h), length), "history")
        return h[:k].copy()


class _SolverBase:
    """Shared shape of Cg / PipelinedCg / BiCgStab (reference ctor + solve)."""
    SOLVER = CG

    def __init__(self, dims, nghost=1, mode=0, timers=None, precision=FP64, batch=1):
        if nghost != 1:
            raise ValueError("the reference stencil needs exactly one ghost layer")
        self.dims = tuple(dims)
        self.mode = mode
        self.precision = precision
        self.batch = batch
        self._ctx = {}

    def _context(self, A):
        key = (A.a, A.b, A.c)
        if key not in self._ctx:
            self._ctx[key] = Context(self.SOLVER, self.dims, A, self.mode, self.precision, self.batch)
        return self._ctx[key]

    def solve(self, A, comm_halo, x, b, iM, maxiter, tol):
        """solve(Stencil&, CommHalo&, x, b, iM, maxiter, tol) -> (result_t, final_err, final_iter).

        comm_halo is accepted for signature parity and ignored: on one GPU the
        zero ghost layer is applied inside the kernels."""
        return self._context(A).solve(x, b, iM, maxiter, tol)


class Cg(_SolverBase):
    SOLVER = CG
    CG_SOLUTION_FOUND, CG_REACHED_MAXITER = 0, 1
    CG_ASYNCHRONOUS, CG_SYNCHRONOUS_STENCIL, CG_SYNCHRONOUS_DOTPROD = 0, 1, 2


class PipelinedCg(_SolverBase):
    SOLVER = PIPELINED_CG
    PLCG_SOLUTION_FOUND, PLCG_REACHED_MAXITER = 0, 1
    PLCG_ASYNCHRONOUS, PLCG_SYNCHRONOUS_STENCIL, PLCG_SYNCHRONOUS_DOTPROD = 0, 1, 2


class BiCgStab(_SolverBase):
    SOLVER = BICGSTAB
    BICGSTAB_SOLUTION_FOUND, BICGSTAB_REACHED_MAXITER, BICGSTAB_BREAKDOWN_RHO, BICGSTAB_BREAKDOWN_OMEGA = 0, 1, 2, 3
    BICGSTAB_ASYNCHRONOUS, BICGSTAB_SYNCHRONOUS_STENCIL, BICGSTAB_SYNCHRONOUS_DOTPROD = 0, 1, 2


def estimate(solver, dims, samples, seed=1234, maxiter=1000, tol=1e-4, ignore_errors=True, stencil=None,
             precision=FP64, batch=1, probes=None):
    """The estimator loop of stochastic-estimator.cc:155-216 (one call)."""
    with Context(solver, dims, stencil, 0, precision, batch) as ctx:
        return ctx.estimate(samples, seed, maxiter, tol, ignore_errors, probes)


def autotune(solver, dims, batch, precision=MIXED, maxiter=5000, tol=1e-9, seed=1234, solve=True):
    """Pick the launch choices for this shape by measurement (sedi_autotune);
    contexts created afterwards use them.  With precision FP64 and batch 1 it
    tunes the single-vector streaming sweeps.  Returns {"slice_width",
    "z_chunks", "period", "chunk", "prefetch_planes" (-1: the built-in
    distance), "sweep_a_form" (narrow-sweep form 1, 2 or 3), "score_ms"}."""
    sid = SOLVER_IDS[solver] if isinstance(solver, str) else int(solver)
    ch = np.zeros(6, np.int32)
    ms = ctypes.c_double(0.0)
    rc = load().sedi_autotune(sid, int(precision), int(batch), *[int(d) for d in dims], int(maxiter), float(tol),
                              int(seed) & 0xFFFFFFFF, 1 if solve else 0, _ptr(ch), ctypes.byref(ms))
    if rc < 0:
        raise SediError(rc, "sedi_autotune")
    return {"slice_width": int(ch[0]), "z_chunks": int(ch[1]), "period": int(ch[2]), "chunk": int(ch[3]),
            "prefetch_planes": int(ch[4]), "sweep_a_form": int(ch[5]), "score_ms": ms.value}


def set_tuning(solver, dims, batch, precision=MIXED, slice_width=0, z_chunks=0, period=0, chunk=0,
               prefetch_planes=-1, sweep_a_form=0):
    """Record launch choices for contexts of this shape without measuring
    (sedi_set_tuning), e.g. an earlier autotune result.  0 (-1 for
    prefetch_planes) keeps the built-in choice."""
    sid = SOLVER_IDS[solver] if isinstance(solver, str) else int(solver)
    ch = np.array([slice_width, z_chunks, period, chunk, prefetch_planes, sweep_a_form], np.int32)
    rc = load().sedi_set_tuning(sid, int(precision), int(batch), *[int(d) for d in dims], _ptr(ch))
    if rc < 0:
        raise SediError(rc, "sedi_set_tuning")


def job_bytes(solver, dims, lanes, precision=FP64):
    """Device bytes of a batched context: the server's admission size."""
    sid = SOLVER_IDS[solver] if isinstance(solver, str) else int(solver)
    return float(load().sedi_job_bytes(sid, int(precision), int(lanes), *[int(d) for d in dims]))


class Server:
    """Estimation-job server over one GPU (sedi_server_* in the C ABI).

    ``submit`` queues an estimator job (seeded device probes, x = 0, -i
    semantics) and returns its id; ``step`` advances all running jobs without
    waiting on the GPU and admits queued jobs while their device bytes fit
    ``budget_bytes``; ``wait`` steps until a job (or all) is done; ``take``
    returns a finished job's results.  ``replay`` runs an open-loop arrival
    schedule natively and returns per-job latencies."""

    STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}

    def __init__(self, budget_bytes=0, max_active=0, job_cap_bytes=0):
        err = ctypes.c_int(0)
        self._h = load().sedi_server_create(float(budget_bytes), int(max_active), float(job_cap_bytes),
                                            ctypes.byref(err))
        if not self._h:
            raise SediError(err.value, "sedi_server_create")

    def close(self):
        if getattr(self, "_h", None):
            load().sedi_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()

    def submit(self, solver, dims, samples, seed, maxiter, tol, precision=FP64):
        sid = SOLVER_IDS[solver] if isinstance(solver, str) else int(solver)
        jid = load().sedi_server_submit(self._h, sid, int(precision), *[int(d) for d in dims], int(samples),
                                        int(seed) & 0xFFFFFFFF, int(maxiter), float(tol))
        if jid < 0:
            raise SediError(int(jid), "sedi_server_submit")
        self._dims = getattr(self, "_dims", {})
        self._dims[jid] = (tuple(int(d) for d in dims), int(samples))
        return jid

    def step(self):
        done = ctypes.c_int(0)
        rc = load().sedi_server_step(self._h, ctypes.byref(done))
        if rc < 0:
            raise SediError(rc, "sedi_server_step")
        return rc, done.value

    def wait(self, jid=-1):
        rc = load().sedi_server_wait(self._h, int(jid))
        if rc < 0:
            raise SediError(rc, "sedi_server_wait")

    def info(self, jid):
        st, rc, lanes = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ts, t0, t1, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        r = load().sedi_server_job_info(self._h, int(jid), ctypes.byref(st), ctypes.byref(rc), ctypes.byref(ts),
                                        ctypes.byref(t0), ctypes.byref(t1), ctypes.byref(lanes), ctypes.byref(by))
        if r < 0:
            raise SediError(r, "sedi_server_job_info")
        return {"state": self.STATES[st.value], "rc": rc.value, "t_submit": ts.value, "t_start": t0.value,
                "t_done": t1.value, "lanes": lanes.value, "bytes": by.value}

    def take(self, jid):
        dims, samples = self._dims.pop(jid)
        n = int(np.prod(dims))
        D = np.zeros(n)
        iters = np.zeros(samples, np.int32)
        errs = np.zeros(samples)
        res = np.zeros(samples, np.int32)
        rc = load().sedi_server_take(self._h, int(jid), _ptr(D), _ptr(iters), _ptr(errs), _ptr(res))
        if rc < 0:
            raise SediError(rc, "job failed")
        return {"rc": rc, "D": D, "iters": iters, "errs": errs, "results": res}

    def replay(self, arrival_s, solver, precision, edge, samples, seed, tol, maxiter, iterations=False):
        """Open-loop schedule (arrays of one entry per job); returns
        (latency_s, result codes, makespan_s), and with iterations=True also
        each job's summed per-probe iteration counts."""
        k = len(arrival_s)
        a = np.ascontiguousarray(arrival_s, np.float64)
        so = np.ascontiguousarray([SOLVER_IDS[x] if isinstance(x, str) else int(x) for x in solver], np.int32)
        pr = np.ascontiguousarray(precision, np.int32)
        ed = np.ascontiguousarray(edge, np.int64)
        sa = np.ascontiguousarray(samples, np.int32)
        se = np.ascontiguousarray(np.asarray(seed, np.int64) & 0xFFFFFFFF, np.uint32)
        to = np.ascontiguousarray(tol, np.float64)
        lat = np.zeros(k)
        rcs = np.zeros(k, np.int32)
        mk = ctypes.c_double(0.0)
        its = np.zeros(k, np.int64)
        r = load().sedi_server_replay(self._h, k, _ptr(a), _ptr(so), _ptr(pr), _ptr(ed), _ptr(sa), _ptr(se), _ptr(to),
                                      int(maxiter), _ptr(lat), _ptr(rcs), ctypes.byref(mk), _ptr(its))
        if r < 0:
            raise SediError(r, "sedi_server_replay")
        return (lat, rcs, mk.value, its) if iterations else (lat, rcs, mk.value)

    def stats(self):
        pk, bu = ctypes.c_double(), ctypes.c_double()
        cr, ru, mr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        la = ctypes.c_longlong()
        load().sedi_server_stats(self._h, ctypes.byref(pk), ctypes.byref(bu), ctypes.byref(cr), ctypes.byref(ru),
                                 ctypes.byref(mr), ctypes.byref(la))
        return {"peak_bytes": pk.value, "budget_bytes": bu.value, "ctx_created": cr.value, "ctx_reused": ru.value,
                "max_running": mr.value, "launches": la.value}


def selftest_bounded_wait(limit_ms=50.0):
    """Run the device wait on a barrier nothing completes; returns
    (timed_out, waited_ms).  See sedi_selftest_bounded_wait."""
    to, ms = ctypes.c_int(0), ctypes.c_double(0.0)
    rc = load().sedi_selftest_bounded_wait(float(limit_ms), ctypes.byref(to), ctypes.byref(ms))
    if rc < 0:
        raise SediError(rc, "sedi_selftest_bounded_wait")
    return bool(to.value), ms.value
