// Internal declarations shared by the sedi_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "sedi_common.cuh"
#include "../../include/sedi_b200.h"

namespace sedi {

// Stop reasons recorded by the device when a solve leaves its loop.
enum StopReason : int {
	STOP_NONE = 0,
	STOP_EARLY = 1,      // initial residual below tol (iteration 0)
	STOP_CONVERGED = 2,  // err <= tol inside the loop
	STOP_MAXITER = 3,    // loop ran to maxiter
	STOP_RHO = 4,        // BiCGStab rho == 0 at the top of an iteration
	STOP_OMEGA = 5,      // BiCGStab omega == 0
	STOP_SNORM = 6,      // BiCGStab ||s||^2 < tol^2 early exit
};

// Scalar state of one single-vector solve, resident in device memory.  All
// Krylov scalars are computed on the device (last block of each reduction),
// so an iteration needs no host round trip.
struct SolveState {
	// inputs
	double tol;
	int maxiter;
	// common
	double bb;       // <b,b> (1 if 0)
	double rr;       // <r,r>
	double err;      // sqrt(rr/bb)
	int iter;        // iteration the next launch executes (1-based)
	int done;        // loop left
	int exit_iter;   // value of the reference's loop variable when the loop was left
	int reason;      // StopReason
	int wsel;        // ping-pong selector for stencil inputs
	int pad0;
	// CG
	double ru, ru_new, sp, alpha, beta;
	// pipelined CG
	double gamma, gamma_old, delta, rr_top;
	// BiCGStab
	double rho, rho_prev, omega, vr, s_norm2, ts, tt;
	int s_exit;
	int pad1;
};

struct Ctx {
	int solver, precision, batch, mode;
	Geo g;
	Coef k;
	int device;
	cudaStream_t stream;      // stream the context's work runs on
	cudaStream_t own_stream;  // the context's own stream
	int nblocks;

	// single-vector FP64 buffers (n doubles each)
	double *x, *b, *iM, *r, *rhat, *p[2], *v[2], *w[2], *u, *q, *s, *z;
	double *partials;
	unsigned int *ticket;
	SolveState *st;        // device
	SolveState *st_host;   // pinned mirror
	double *hist;          // device, maxiter_cap+1
	int hist_cap;
	int hist_len;
	cudaGraphExec_t chunk_graph[2];  // [iM is a vector]
	int chunk_iters;

	// estimator accumulators (n doubles)
	double *t_acc, *q_acc;
	// host-facing estimator staging (batched form): probes, D, t, q on the device
	double *stage_probes, *stage_out;
	size_t stage_probe_bytes;

	void *batched;  // batched-form state (batched.cu)
	void *pairs;    // single-vector form on the streaming sweeps (n1 even; batched.cu)

	long long launches;
	std::string error;
};

int set_cuda_error(Ctx *c, cudaError_t e, const char *where);

// plain.cu
int plain_alloc(Ctx *c);
void plain_free(Ctx *c);
int plain_solve_dev(Ctx *c, const double *b, double *x, const double *iM, int maxiter, double tol,
                    double *final_err, int *final_iter);
int plain_solve_resident(Ctx *c, bool vim, int maxiter, double tol, double *final_err, int *final_iter);
int plain_history(Ctx *c, double *out, int len);
int plain_stencil(Ctx *c, const double *x_dev, double *y_dev);
int plain_accumulate(Ctx *c, const double *x_dev, const double *v_dev, int reset);
int plain_divide(Ctx *c, double *D_dev);

// batched.cu
int batched_alloc(Ctx *c);
// Single-vector form on the streaming sweeps (n1 even): state aliasing the
// plain form's vectors; solve with b, x already in c->b, c->x (constant iM).
int pairs_alloc(Ctx *c);
void pairs_free(Ctx *c);
int pairs_solve_resident(Ctx *c, int maxiter, double tol, double *final_err, int *final_iter);
int pairs_time_kernels(Ctx *c, int reps, double *ms, double *bytes, char *names, int *count);
void batched_free(Ctx *c);
int batched_solve_dev(Ctx *c, int nrhs, const double *b, double *x, int maxiter, double tol, double *final_err,
                      int *final_iter, int *results);
int batched_estimate_dev(Ctx *c, int samples, const double *probes_dev, int maxiter, double tol,
                         int ignore_errors, double *D_dev, double *t_dev, double *q_dev, int *iters,
                         double *errs, int *results);
int batched_time_kernels(Ctx *c, int reps, double *ms, double *bytes, char *names, int *count);
int batched_estimate_src(Ctx *c, int samples, const double *probes_dev, uint32_t seed, int maxiter, double tol,
                         int ignore_errors, double *D_dev, double *t_dev, double *q_dev, int *iters, double *errs,
                         int *results);

// Non-blocking estimator on a batched context: begin enqueues the first
// batch; advance checks the context's event and enqueues the next step
// (never waits), *done = 1 when D (and the D_host copy) are complete;
// est_result gives the estimator's return code (worst result, the first
// failing probe's code without -i, or a negative error).
int batched_est_begin(Ctx *c, int samples, const double *probes_dev, uint32_t seed, int maxiter, double tol,
                      int ignore_errors, double *D_dev, double *t_dev, double *q_dev, double *D_host, int *iters,
                      double *errs, int *results);
int batched_est_advance(Ctx *c, int *done);
int batched_est_result(const Ctx *c);
// Autotuner and the launch choices of a batched context (see batched.cu).
int batched_autotune(int solver, int precision, int batch, long long n1, long long n2, long long n3, int maxiter,
                     double tol, uint32_t seed, int flags, int *out, double *score_ms);
int batched_config(const Ctx *c, int *out);
int batched_set_tuning(int solver, int precision, int batch, long long n1, long long n2, long long n3,
                       const int *choice);
// In-loop target factor of the mixed form (lanes stop on true err <= theta * tol).
int batched_set_theta(Ctx *c, double theta);
double batched_theta(const Ctx *c);
// Device bytes a batched context allocates (0 for the single-vector form).
size_t batched_bytes(int solver, int precision, int batch, long long n1, long long n2, long long n3);
// Lanes (padded right-hand sides) of a batched context created for `batch`.
int batched_lanes(int precision, int batch);

// rng.cu
void host_fill_probe(uint32_t seed, long n, double *out);
void host_fill_probe_range(uint32_t seed, long long offset, long long count, double *out);
// Probes seed..seed+nprobes-1 on the device: lane-sliced (W > 0) or dense (W == 0).
int device_fill_probes(uint32_t seed, int nprobes, long long npts, int W, double *out, cudaStream_t s);

}  // namespace sedi

struct sedi_ctx {
	sedi::Ctx c;
};
