/*
 * sedi_b200 -- B200 (sm_100a) implementation of the SEDI estimator hot path.
 *
 * C ABI: plain pointers and sizes, no C++ or torch types.  Every grid is a
 * dense n1*n2*n3 array of doubles, i1 fastest, then i2, then i3 -- the element
 * order of the reference's Grid3d::rank_cells (Slice3d.hpp:30-32) without its
 * ghost layer; the zero ghost layer of the reference (Cg.hpp:57-62) is applied
 * inside the kernels.
 *
 * Reference interfaces replaced (paths relative to the reference checkout):
 *   sedi_create          <- {Cg,PipelinedCg,BiCgStab}(DomainDecomposition&, long nghost, int mode, Timers*)
 *                           Cg.hpp:48-68, PipelinedCg.hpp:48-70, BiCgStab.hpp:55-75, plus
 *                           Stencil(a,b,c) Stencil.hpp:18-19 and the solver typedef chosen by
 *                           -DSOLVER in stochastic-estimator.cc:134-142
 *   sedi_solve[_dev]     <- solver_t::solve(Stencil&, CommHalo&, Grid3d& x, Grid3d& b, Grid3d& iM,
 *                           int maxiter, Dtype tol, Dtype* final_err, int* final_iter)
 *                           Cg.hpp:70-82, PipelinedCg.hpp:72-84, BiCgStab.hpp:77-89
 *   sedi_solve_batch     <- the same solve() applied to many right-hand sides at once
 *   sedi_estimate[_probes] <- the probe loop of main(), stochastic-estimator.cc:155-216
 *                           (RNG fill :165, x=0 :175, solve :176-179, abort unless -i :181-184,
 *                            t += x.*v :195, q += v.*v :198, D = t./q :216)
 *   sedi_fill_probe      <- DistrRngStd::fill_plusminusone, DistrRngStd.hpp:22-42
 *   sedi_stencil_apply   <- Stencil::apply / DistrAsyncStencil at -p 1x1x1, Stencil.hpp:21-54,
 *                           DistrAsyncStencil.hpp:52-100
 *
 * Return values of the solve/estimate entry points are the reference's
 * result_t values (0 solution found, 1 reached maxiter, 2 BiCGStab rho
 * breakdown, 3 BiCGStab omega breakdown; Cg.hpp:31-34, BiCgStab.hpp:32-37)
 * or a negative SEDI_ERR_* code.  A context is not thread-safe (one host
 * thread per context), like the reference solver objects that share one
 * CommHalo (Cg.hpp:95-98).
 */
#ifndef SEDI_B200_H
#define SEDI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solver ids: the reference's -DSOLVER values (stochastic-estimator.cc:134-142). */
#define SEDI_BICGSTAB 1
#define SEDI_CG 2
#define SEDI_PIPELINED_CG 3

/* Arithmetic forms. */
#define SEDI_PREC_FP64 0  /* the reference method in FP64, kernel by kernel */
#define SEDI_PREC_MIXED 1 /* FP32 Krylov vectors, FP64 reductions, FP64 reliable update of x and r */

/* Reference result_t values. */
#define SEDI_SOLUTION_FOUND 0
#define SEDI_REACHED_MAXITER 1
#define SEDI_BREAKDOWN_RHO 2
#define SEDI_BREAKDOWN_OMEGA 3

/* Errors (negative). */
#define SEDI_ERR_ARG (-1)     /* invalid argument (sizes, solver id, NULL pointer) */
#define SEDI_ERR_CUDA (-2)    /* a CUDA call failed; see sedi_ctx_error() */
#define SEDI_ERR_NOMEM (-3)   /* device allocation failed */
#define SEDI_ERR_NODEV (-4)   /* no CUDA device / kernels not loadable */
#define SEDI_ERR_UNSUPPORTED (-5)

/* Mode bits (Cg.hpp:36-40).  At one GPU there is no halo exchange or
 * allreduce to overlap, so both bits are accepted and have no numerical
 * effect, exactly as at -p 1x1x1 in the reference. */
#define SEDI_MODE_SYNC_STENCIL 1
#define SEDI_MODE_SYNC_DOTPROD 2

typedef struct sedi_ctx sedi_ctx;

/*
 * Create a solver context on the current CUDA device.
 *   solver     SEDI_CG / SEDI_PIPELINED_CG / SEDI_BICGSTAB
 *   n1,n2,n3   grid (every dimension >= 1)
 *   a,b,c      stencil coefficients: y = a*x_c - c*(x_{i-1}+...) - b*(x_{i+1}+...)
 *   mode       SEDI_MODE_* bits (accepted, no effect on one GPU)
 *   precision  SEDI_PREC_FP64 or SEDI_PREC_MIXED.  The mixed forms of CG
 *              and pipelined CG run the CG recurrence (one GPU has no
 *              reduction latency for pipelining to hide; see
 *              sedi_set_mixed_target for their accuracy).
 *   batch      right-hand sides in flight per launch (1 = single-vector form)
 *   err        out: 0 or a negative SEDI_ERR_* (may be NULL)
 * Returns NULL on error.
 */
sedi_ctx *sedi_create(int solver, long n1, long n2, long n3, double a, double b, double c, int mode,
                      int precision, int batch, int *err);
void sedi_destroy(sedi_ctx *ctx);
/* Message for the last failure on this context ("" if none). */
const char *sedi_ctx_error(const sedi_ctx *ctx);

/*
 * Solve A x = b for one right-hand side (host buffers, n1*n2*n3 doubles).
 * x: in first guess, out solution.  iM: inverse-diagonal preconditioner as a
 * vector, or NULL for the constant 1/a the reference uses
 * (stochastic-estimator.cc:101-103).  final_err, final_iter: as the reference.
 */
int sedi_solve(sedi_ctx *ctx, const double *b, double *x, const double *iM, int maxiter, double tol,
               double *final_err, int *final_iter);
/* Same with device pointers (already resident in HBM); runs on the context's stream. */
int sedi_solve_dev(sedi_ctx *ctx, const double *b_dev, double *x_dev, const double *iM_dev, int maxiter,
                   double tol, double *final_err, int *final_iter);

/*
 * nrhs right-hand sides (host buffers; right-hand side k at offset k*n).
 * Per right-hand side: results[k] (result_t), final_err[k], final_iter[k].
 * Returns the largest result_t seen, or a negative error.
 */
int sedi_solve_batch(sedi_ctx *ctx, int nrhs, const double *b, double *x, int maxiter, double tol,
                     double *final_err, int *final_iter, int *results);

/*
 * The estimator loop of stochastic-estimator.cc:155-216 on the GPU.
 * Probe k is DistrRngStd's ±1 vector from std::mt19937(seed + k).
 *   D           out: t ./ q (n doubles)
 *   t, q        out, may be NULL: the accumulators
 *   iters, errs, results   out, may be NULL: per-probe final_iter, final_err, result_t
 *   ignore_errors  0: stop at the first probe whose result is not 0 and return
 *                  that result (the reference aborts with 100+code unless -i)
 * Returns 0, a positive result_t (first failure, when !ignore_errors), or an error.
 */
int sedi_estimate(sedi_ctx *ctx, int samples, uint32_t seed, int maxiter, double tol, int ignore_errors,
                  double *D, double *t, double *q, int *iters, double *errs, int *results);
/* Same with caller-provided probes: samples*n doubles in host memory. */
int sedi_estimate_probes(sedi_ctx *ctx, int samples, const double *probes, int maxiter, double tol,
                         int ignore_errors, double *D, double *t, double *q, int *iters, double *errs,
                         int *results);

/* Same with device pointers: probes (samples*n doubles) already resident in
 * HBM, D/t/q device outputs (t, q may be NULL); per-probe arrays on the host.
 * Runs on the context's stream (see sedi_set_stream). */
int sedi_estimate_dev(sedi_ctx *ctx, int samples, const double *probes_dev, int maxiter, double tol,
                      int ignore_errors, double *D_dev, double *t_dev, double *q_dev, int *iters, double *errs,
                      int *results);

/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*); NULL restores the context's own stream. */
int sedi_set_stream(sedi_ctx *ctx, void *stream);

/*
 * Time the context's per-iteration stencil kernels in isolation: each of the
 * solver's per-iteration kernels is launched `reps` times back to back on the
 * context's stream between CUDA events (after one warm-up launch), on the
 * context's current buffers and a state with every right-hand side active.
 * Outputs per kernel k < *count: ms[k] average duration of one launch,
 * bytes[k] its algorithmic DRAM bytes per launch (compulsory reads + writes
 * of the Krylov vectors it streams), names (count*32 chars, NUL-terminated
 * slots).  The buffers' contents are scratch afterwards.  Returns 0 or error.
 * A single-vector FP64 context (batch 1) times its streaming sweeps (names
 * ending in _sv), which serve grids with n1 even and at least 2^22 points;
 * SEDI_ERR_UNSUPPORTED for other grids, which use column-march kernels.
 * CG lists three kernels: cg_a every iteration, and its second sweep in two
 * forms that alternate, cg_b on odd iterations (r only) and cg_bx on even
 * ones (the x steps of both iterations).
 */
int sedi_time_kernels(sedi_ctx *ctx, int reps, double *ms, double *bytes, char *names, int *count);

/*
 * Residual without device allocation.  No counterpart in the reference: it
 * is for callers that cannot allocate device memory where they need a
 * residual check (memory pools or arenas that own all device memory,
 * allocation-free serving loops, host frameworks with their own allocator).
 * Computes r = b - A x with zero ghosts (x_dev, b_dev inputs, r_dev output;
 * device pointers, n1*n2*n3 doubles, i1 fastest) and *err_out (host) =
 * sqrt(<r,r>/<b,b>) with <b,b> taken as 1 when it is 0, the solvers' initial
 * residual test.  r_dev must not overlap x_dev or b_dev (SEDI_ERR_ARG).
 * Runs on `stream` (a cudaStream_t as void*, NULL = default stream); the
 * call synchronizes that stream and copies err into host memory before it
 * returns.
 * Scratch: a fixed device array in the library (about 64 KiB per GPU, held
 * until the process exits) -- nothing is allocated per call.  Limit: the
 * grid's sweep may use at most 4096 thread blocks, which holds whenever
 * ceil(n1/32)*ceil(n2/8) <= 4096 (any n3); larger grids return SEDI_ERR_ARG.
 * The first call on a device looks up the array's device address, so make
 * that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (different streams or threads) race.
 */
int sedi_residual_noalloc(long n1, long n2, long n3, double a, double b, double c, const double *x_dev,
                          const double *b_dev, double *r_dev, double *err_out, void *stream);

/*
 * Slab (i3) domain decomposition of the FP64 solvers (CG, pipelined CG,
 * BiCGStab): the kernels one rank runs on its slab (the host loop, halo
 * exchange and collectives are in sedi_b200/domain.py).  Replaces, for a
 * decomposition -p 1x1xP, the reference's DomainDecomposition
 * (DomainDecomposition.hpp:51-80), the halo exchange (CommHalo.hpp:84-181) --
 * a halo is one contiguous ghost plane --, the inner/border stencil split
 * (DistrAsyncStencil.hpp:52-100) and the local part of DistrAsyncDotProds
 * (DistrAsyncDotProds.hpp:85-136).  Every slab vector is [nloc + 2][n2][n1]
 * doubles (device), i1 fastest, with ghost planes 0 and nloc+1; ghost planes
 * on the global boundary are zero.
 */
typedef struct sedi_slab_args {
	const double *src;  /* stencil input (ghost planes current), or the mode's first vector */
	const double *b;
	const double *rhat;
	double *x, *r, *y, *u, *w, *wn, *q, *s, *p, *z, *v, *t;
	double iM;     /* constant Jacobi preconditioner 1/a */
	double alpha, beta;
	double bo;     /* BiCGStab: -beta*omega */
	double omega;
	int first;     /* first iteration */
} sedi_slab_args;

/*
 * sedi_slab_sweep: for ghosted planes z in [z_lo, z_hi) (1 <= z_lo <= z_hi
 * <= nloc+1), with A the stencil applied to src (or to src .* iM where noted):
 *   mode  0  r = b - A src; dots <b,b>, <r,r>                       (Cg.hpp:112-129)
 *   mode  1  dots <A src, src> and, when first, <r, r*iM>          (Cg.hpp:152-166)
 *   mode  2  x += alpha src; r -= alpha A src; dots <r, r*iM>, <r,r> (Cg.hpp:169-182)
 *   mode  3  y = A src                                              (Stencil.hpp:38-54)
 *   mode  4  u = src*iM, w = A(src*iM), q = s = p = z = 0;
 *            dots <src,u>, <w,u>, <src,src>                         (PipelinedCg.hpp:138-155)
 *   mode  5  m = src*iM, n = A m; q = m + beta q, s = src + beta s,
 *            p = u + beta p, z = n + beta z, r -= alpha s, x += alpha p,
 *            u -= alpha q, wn = src - alpha z; dots <r,u>, <wn,u>, <r,r>
 *            (src is w; wn must not be src)                         (PipelinedCg.hpp:155-223)
 *   mode  6  p = r (first) or r + beta p + bo v                     (BiCgStab.hpp:165-173)
 *   mode  7  v = A(src*iM); dot <v, rhat>                           (BiCgStab.hpp:175-187)
 *   mode  8  s = r - alpha v                                        (BiCgStab.hpp:189)
 *   mode  9  t = A(src*iM); dots <src,src>, <t,src>, <t,t>          (BiCgStab.hpp:192-212)
 *   mode 10  x += alpha p*iM + omega s*iM; r = s - omega t;
 *            dots <r,r>, <r,rhat>                                   (BiCgStab.hpp:216-224)
 *   mode 11  x += alpha p*iM                                        (BiCgStab.hpp:193-199)
 *   mode 12  p = r*iM (first) or r*iM + beta p                      (Cg.hpp:144-147, :188)
 * Modes 6, 8, 11 and 12 are elementwise; 3 returns no dots.  The others
 * write plane_part[(z-1)*3 + d], plane z's dot d (0 for unused d), summed in
 * an order fixed by n1 and n2 only (sedi_slab_chunks() row chunks per plane,
 * scratch chunk_part of nloc*chunks*3 doubles), so plane sums, and the
 * solves, do not depend on how the planes are split into slabs.  Elementwise
 * values round as the reference's.  Pointers a mode does not use may be
 * NULL; a missing one it uses returns SEDI_ERR_ARG.  Runs on `stream`
 * (cudaStream_t as void*).
 */
int sedi_slab_sweep(int mode, long n1, long n2, long nloc, double a, double b, double c, long z_lo, long z_hi,
                    const sedi_slab_args *args, double *chunk_part, double *plane_part, void *stream);
/* t += x .* v, q += v .* v (t = x .* v, q = v .* v when reset) over n elements
 * (stochastic-estimator.cc:195, :198). */
int sedi_slab_accumulate(long n, const double *x, const double *v, double *t, double *q, int reset, void *stream);
/* D = t ./ q over n elements (stochastic-estimator.cc:216). */
int sedi_slab_divide(long n, const double *t, const double *q, double *D, void *stream);
/* Row chunks per plane of sedi_slab_sweep's dot products. */
int sedi_slab_chunks(void);

/* Device probe generator: probes seed, seed+1, ..., seed+nprobes-1 (each
 * DistrRngStd's +-1 vector from std::mt19937(seed + k), bit-identical to
 * sedi_fill_probe) into out_dev[k*n + i], on `stream` (cudaStream_t as void*). */
int sedi_fill_probes_dev(uint32_t seed, int nprobes, long n, double *out_dev, void *stream);

/* Host probe generator, bit-identical to DistrRngStd with std::mt19937(seed). */
void sedi_fill_probe(uint32_t seed, long n, double *out);
/* Points [offset, offset + count) of the probe sedi_fill_probe(seed, ...)
 * writes (the part of the global probe one slab of a decomposed grid holds;
 * the reference fills each rank's cells from its own generator,
 * DistrRngStd.hpp:22-42, so its probes depend on -p -- these do not). */
void sedi_fill_probe_range(uint32_t seed, long offset, long count, double *out);

/* y = A x with zero ghosts (host buffers), the kernel the solvers use. */
int sedi_stencil_apply(sedi_ctx *ctx, const double *x, double *y);

/*
 * Per-iteration relative residual of the last single-vector solve:
 * hist[0] is the initial err, hist[i] the err printed by the reference after
 * iteration i (Cg.hpp:192, PipelinedCg.hpp:228, BiCgStab.hpp:228).
 * Returns the number of entries written.
 */
int sedi_last_history(sedi_ctx *ctx, double *hist, int len);

/* Device memory of the current GPU in MB (used = total - free), the device
 * counterpart of the reference's resident-set report (stochastic-estimator.cc:31-55). */
int sedi_device_memory(double *used_mb, double *total_mb);

/* Kernel launches issued by this context since creation (for benchmarks). */
long long sedi_launch_count(const sedi_ctx *ctx);

/* Library version string. */
const char *sedi_version(void);

/*
 * Estimation-job server (no counterpart in the reference, which runs one
 * estimate per process: stochastic-estimator.cc:57-232).  Jobs of any grid,
 * sample count, tolerance, solver and precision are admitted as they arrive
 * while their device bytes fit the budget, each on its own batched context
 * and CUDA stream with all Krylov state resident on the GPU; running jobs
 * overlap on the device and advance without blocking one another.  Every job
 * is an estimator run with seeded device probes (probe k of a job is
 * std::mt19937(seed + k), as DistrRngStd draws them), x = 0, the 7-point
 * operator a = 6, b = c = 1, iM = 1/6 and -i semantics (all samples run;
 * per-probe result codes are reported).  A job's result does not depend on
 * what else runs: the same job gives the same D alone and in any mix.
 * Not thread-safe: one thread drives a server.
 */
typedef struct sedi_server sedi_server;

/* budget_bytes: device memory for job contexts (0: 85% of the free memory);
 * max_active: jobs running at once (0: 8); job_cap_bytes: largest context of
 * one job (0: 32 GiB) -- a job whose samples do not fit runs in batches. */
sedi_server *sedi_server_create(double budget_bytes, int max_active, double job_cap_bytes, int *err);
void sedi_server_destroy(sedi_server *srv);

/* Queue a job; returns its id (>= 0) or a negative error (SEDI_ERR_NOMEM
 * when even one batch of it exceeds the budget). */
long sedi_server_submit(sedi_server *srv, int solver, int precision, long n1, long n2, long n3, int samples,
                        uint32_t seed, int maxiter, double tol);

/* Advance every running job and admit queued ones, without waiting on the
 * GPU.  Returns the number of jobs queued or running; *completed (optional)
 * = jobs finished since creation. */
int sedi_server_step(sedi_server *srv, int *completed);

/* Step until job `id` is finished (id < 0: until no job is left). */
int sedi_server_wait(sedi_server *srv, long id);

/* state: 0 queued, 1 running, 2 done, 3 failed; rc: the estimator's code
 * (worst per-probe result, or a negative error); times in seconds on the
 * server's clock; lanes: right-hand sides per batch; bytes: device bytes of
 * its context.  Any output may be NULL. */
int sedi_server_job_info(sedi_server *srv, long id, int *state, int *rc, double *t_submit, double *t_start,
                         double *t_done, int *lanes, double *bytes);

/* Copy out a finished job's D (n1*n2*n3), per-probe iterations, final errors
 * and result codes (any may be NULL) and forget the job.  Returns its rc. */
int sedi_server_take(sedi_server *srv, long id, double *D, int *iters, double *errs, int *results);

/* Open-loop replay: job k (cubic grid edge[k]) is submitted when arrival_s[k]
 * seconds (non-decreasing) have passed since the call; the server runs until
 * all are done.  latency_s[k] = done - scheduled arrival; rcs[k] (optional)
 * its code; *makespan_s (optional) = first arrival to last completion;
 * iterations[k] (optional) = the sum of job k's per-probe iteration counts.
 * Results are discarded. */
int sedi_server_replay(sedi_server *srv, int njobs, const double *arrival_s, const int *solver, const int *precision,
                       const long *edge, const int *samples, const uint32_t *seed, const double *tol, int maxiter,
                       double *latency_s, int *rcs, double *makespan_s, long long *iterations);

/* Peak device bytes held, the budget, contexts created and reused, most jobs
 * running at once, kernel launches of finished jobs. */
int sedi_server_stats(const sedi_server *srv, double *peak_bytes, double *budget_bytes, int *ctx_created,
                      int *ctx_reused, int *max_running, long long *launches);

/*
 * Autotuner of the batched form (no counterpart in the reference).  For
 * contexts of this solver, precision, batch size and grid it picks, by
 * measurement on scratch contexts: the lane-slice width of the interleaved
 * Krylov fields (FP32 8 or 4 lanes, FP64 8, 4 or 2), the i3 split of the
 * sweeps, how many planes ahead of its TMA loads a sweep prefetches into L2
 * (0, 2, 4 or 8), for CG and BiCGStab the form of the narrow sweeps (CG's
 * sweep A, BiCGStab's sweeps 2 and 3; 1: a ring of computed planes on 32x32
 * tiles; 2: in place, 32x16 tiles, two blocks per SM; 3: in place, 32x32
 * tiles, six stages), and with flags & 1 the iterations per
 * captured graph and (mixed
 * precision) the reliable-update period in 20..50, the last two by timing a
 * real estimate of `batch` probes seeded `seed` to `tol`.  The choice is kept
 * for the process and used by every context created afterwards with the
 * same parameters (and by the server's admission sizes).
 * choice[0..5] = slice width, i3 chunks (0: the built-in model), period,
 * iterations per graph, L2 prefetch distance in planes (-1: the built-in
 * distance), narrow-sweep form; *score_ms (optional)
 * = the winning estimate time (flags & 1) or the sweep time of one
 * iteration (CG's two parity forms of sweep B count half each).  Needs
 * device memory for one such context at a time.
 */
int sedi_autotune(int solver, int precision, int batch, long n1, long n2, long n3, int maxiter, double tol,
                  uint32_t seed, int flags, int *choice, double *score_ms);

/* Record launch choices for contexts of this solver, precision, batch size
 * and grid without measuring (no counterpart in the reference): a caller
 * that saved an earlier sedi_autotune result (choice[0..5] as there; 0
 * selects the built-in choice of the first four and of the narrow-sweep form, -1
 * that of the prefetch distance) sets it again at start-up.  With
 * SEDI_PREC_FP64 and batch 1 it sets the single-vector streaming sweeps
 * (even n1, 2^22 points or more): i3 chunks, prefetch distance and
 * narrow-sweep form (the slice width is fixed).  Host-only; SEDI_ERR_ARG on
 * bad values. */
int sedi_set_tuning(int solver, int precision, int batch, long n1, long n2, long n3, const int *choice);

/*
 * In-loop stop target of the mixed-precision batched form (no counterpart in
 * the reference, whose FP64 method needs none).  A mixed lane leaves its loop
 * when its FP64 true residual sqrt(<b - A x, b - A x>/<b,b>) <= theta * tol,
 * 0 < theta <= 1; result codes and final_err are still checked against tol
 * as the reference does (Cg.hpp:191-206), and the initial test stays
 * err < tol (Cg.hpp:130-134).  Two solutions that both meet tol differ by
 * the error each leaves behind the residual bound.  The FP32 CG iterates
 * follow the FP64 ones, so theta = 1 keeps the CG and pipelined-CG
 * diagonals within 1e-8 of the FP64 form's (measured 1.5e-9 at 128^3,
 * 3.9e-9 at 256^3, tol 1e-9); BiCGStab's FP64 diagonal itself lies 1e-7
 * to 4e-7 from the converged answer at tol 1e-9, and theta = 0.1 puts the
 * mixed one ten times closer to it than that.  Defaults: CG and pipelined
 * CG 1, BiCGStab 0.1 (sedi_mixed_target reads them).
 * SEDI_ERR_UNSUPPORTED for FP64 contexts, SEDI_ERR_ARG for theta outside (0, 1].
 */
int sedi_set_mixed_target(sedi_ctx *ctx, double theta);
double sedi_mixed_target(const sedi_ctx *ctx);

/* Launch choices of a batched context: config[0..6] = lane-slice width, i3
 * chunks of a sweep, reliable-update period, iterations per captured graph,
 * lanes (padded right-hand sides), L2 prefetch distance in planes, form of
 * the narrow sweeps (see sedi_autotune).  SEDI_ERR_UNSUPPORTED for the
 * single-vector form. */
int sedi_ctx_config(const sedi_ctx *ctx, int *config);

/*
 * Self-test of the bounded device wait that every batched sweep uses on its
 * copy barriers (no counterpart in the reference): one kernel waits on a
 * barrier that nothing completes, with a limit of limit_ms (0 < limit_ms <=
 * 5000).  *timed_out = 1 when the wait gave up as it must; *waited_ms
 * (optional) = how long it waited.  The GPU and any context stay usable.
 */
int sedi_selftest_bounded_wait(double limit_ms, int *timed_out, double *waited_ms);

/* Device bytes of a batched context (the server's admission size). */
double sedi_job_bytes(int solver, int precision, int lanes, long n1, long n2, long n3);

#ifdef __cplusplus
}
#endif

#endif
