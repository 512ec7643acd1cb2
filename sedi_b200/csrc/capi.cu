// C ABI of sedi_b200 (declarations and reference mapping in include/sedi_b200.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "sedi_internal.h"

namespace sedi {

int set_cuda_error(Ctx *c, cudaError_t e, const char *where) {
	c->error = std::string(where) + ": " + cudaGetErrorString(e);
	if (e == cudaErrorMemoryAllocation) return SEDI_ERR_NOMEM;
	return SEDI_ERR_CUDA;
}

static bool plain_form(const Ctx *c) { return c->batch == 1 && c->precision == SEDI_PREC_FP64; }

}  // namespace sedi

using namespace sedi;

#define CAPI_TRY(expr)                                                        \
	do {                                                                      \
		cudaError_t e_ = (expr);                                              \
		if (e_ != cudaSuccess) return set_cuda_error(c, e_, #expr);           \
	} while (0)

extern "C" {

const char *sedi_version(void) { return "sedi_b200 1.0 (sm_100a)"; }

sedi_ctx *sedi_create(int solver, long n1, long n2, long n3, double a, double b, double cc, int mode,
                      int precision, int batch, int *err) {
	int dummy;
	if (!err) err = &dummy;
	*err = 0;
	if (solver < 1 || solver > 3 || n1 < 1 || n2 < 1 || n3 < 1 || batch < 1 ||
	    (precision != SEDI_PREC_FP64 && precision != SEDI_PREC_MIXED) || (mode & ~3) != 0 ||
	    n1 > (1L << 30) || n2 > (1L << 30) || n3 > (1L << 30) || (double)n1 * n2 * n3 > 4.0e9) {
		*err = SEDI_ERR_ARG;
		return nullptr;
	}
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
		cudaGetLastError();
		*err = SEDI_ERR_NODEV;
		return nullptr;
	}
	sedi_ctx *h = new (std::nothrow) sedi_ctx();
	if (!h) {
		*err = SEDI_ERR_NOMEM;
		return nullptr;
	}
	Ctx *c = &h->c;
	c->solver = solver;
	c->precision = precision;
	c->batch = batch;
	c->mode = mode;
	c->g.n1 = (int)n1;
	c->g.n2 = (int)n2;
	c->g.n3 = (int)n3;
	c->g.n = (long long)n1 * n2 * n3;
	c->k.a = a;
	c->k.b = b;
	c->k.c = cc;
	cudaGetDevice(&c->device);
	if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
		cudaGetLastError();
		delete h;
		*err = SEDI_ERR_CUDA;
		return nullptr;
	}
	c->stream = c->own_stream;
	int rc = plain_form(c) ? plain_alloc(c) : batched_alloc(c);
	if (rc) {
		*err = rc;
		sedi_destroy(h);
		return nullptr;
	}
	return h;
}

void sedi_destroy(sedi_ctx *h) {
	if (!h) return;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	if (c->stream) cudaStreamSynchronize(c->stream);
	if (c->own_stream) cudaStreamSynchronize(c->own_stream);
	plain_free(c);
	batched_free(c);
	if (c->stage_probes) cudaFree(c->stage_probes);
	if (c->stage_out) cudaFree(c->stage_out);
	if (c->own_stream) cudaStreamDestroy(c->own_stream);
	delete h;
}

const char *sedi_ctx_error(const sedi_ctx *h) { return h ? h->c.error.c_str() : "null context"; }

long long sedi_launch_count(const sedi_ctx *h) { return h ? h->c.launches : 0; }

int sedi_autotune(int solver, int precision, int batch, long n1, long n2, long n3, int maxiter, double tol,
                  uint32_t seed, int flags, int *choice, double *score_ms) {
	if (solver < 1 || solver > 3 ||
	    (precision != SEDI_PREC_FP64 && precision != SEDI_PREC_MIXED) || batch < 1 ||
	    n1 < 1 || n2 < 1 || n3 < 1 || maxiter < 0 || !choice)
		return SEDI_ERR_ARG;
	return batched_autotune(solver, precision, batch, n1, n2, n3, maxiter, tol, seed, flags, choice, score_ms);
}

int sedi_set_mixed_target(sedi_ctx *h, double theta) {
	if (!h) return SEDI_ERR_ARG;
	return batched_set_theta(&h->c, theta);
}

double sedi_mixed_target(const sedi_ctx *h) { return h ? batched_theta(&h->c) : 1.0; }

int sedi_set_tuning(int solver, int precision, int batch, long n1, long n2, long n3, const int *choice) {
	if (solver < 1 || solver > 3 ||
	    (precision != SEDI_PREC_FP64 && precision != SEDI_PREC_MIXED) || batch < 1 ||
	    n1 < 1 || n2 < 1 || n3 < 1 || !choice)
		return SEDI_ERR_ARG;
	return batched_set_tuning(solver, precision, batch, n1, n2, n3, choice);
}

int sedi_ctx_config(const sedi_ctx *h, int *config) {
	if (!h || !config) return SEDI_ERR_ARG;
	return batched_config(&h->c, config);
}

int sedi_device_memory(double *used_mb, double *total_mb) {
	if (!used_mb || !total_mb) return SEDI_ERR_ARG;
	size_t fr = 0, tot = 0;
	if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
		cudaGetLastError();
		return SEDI_ERR_NODEV;
	}
	*used_mb = (double)(tot - fr) / (1024.0 * 1024.0);
	*total_mb = (double)tot / (1024.0 * 1024.0);
	return 0;
}

void sedi_fill_probe(uint32_t seed, long n, double *out) {
	if (out && n > 0) host_fill_probe(seed, n, out);
}

int sedi_solve_dev(sedi_ctx *h, const double *b, double *x, const double *iM, int maxiter, double tol,
                   double *final_err, int *final_iter) {
	if (!h || !b || !x || !final_err || !final_iter || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	if (!plain_form(c)) {
		if (iM) return SEDI_ERR_UNSUPPORTED;
		int res = 0;
		int rc = batched_solve_dev(c, 1, b, x, maxiter, tol, final_err, final_iter, &res);
		return rc < 0 ? rc : res;
	}
	return plain_solve_dev(c, b, x, iM, maxiter, tol, final_err, final_iter);
}

int sedi_solve(sedi_ctx *h, const double *b, double *x, const double *iM, int maxiter, double tol,
               double *final_err, int *final_iter) {
	if (!h || !b || !x || !final_err || !final_iter || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	const size_t bytes = sizeof(double) * (size_t)c->g.n;
	if (!plain_form(c)) {
		if (iM) return SEDI_ERR_UNSUPPORTED;
		double *db = nullptr, *dx = nullptr;
		CAPI_TRY(cudaMalloc(&db, bytes));
		if (cudaMalloc(&dx, bytes) != cudaSuccess) {
			cudaFree(db);
			return set_cuda_error(c, cudaErrorMemoryAllocation, "cudaMalloc");
		}
		int res = 0, rc = 0;
		if (cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
		    cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
			rc = set_cuda_error(c, cudaGetLastError(), "cudaMemcpy");
		if (!rc) rc = batched_solve_dev(c, 1, db, dx, maxiter, tol, final_err, final_iter, &res);
		if (!rc && (cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
		            cudaStreamSynchronize(c->stream) != cudaSuccess))
			rc = set_cuda_error(c, cudaGetLastError(), "cudaMemcpy");
		cudaFree(db);
		cudaFree(dx);
		return rc < 0 ? rc : res;
	}
	CAPI_TRY(cudaMemcpyAsync(c->b, b, bytes, cudaMemcpyHostToDevice, c->stream));
	CAPI_TRY(cudaMemcpyAsync(c->x, x, bytes, cudaMemcpyHostToDevice, c->stream));
	if (iM) CAPI_TRY(cudaMemcpyAsync(c->iM, iM, bytes, cudaMemcpyHostToDevice, c->stream));
	const int rc = plain_solve_resident(c, iM != nullptr, maxiter, tol, final_err, final_iter);
	if (rc < 0) return rc;
	CAPI_TRY(cudaMemcpyAsync(x, c->x, bytes, cudaMemcpyDeviceToHost, c->stream));
	CAPI_TRY(cudaStreamSynchronize(c->stream));
	return rc;
}

int sedi_last_history(sedi_ctx *h, double *hist, int len) {
	if (!h || !hist || len < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	if (!plain_form(c)) return 0;
	cudaSetDevice(c->device);
	return plain_history(c, hist, len);
}

int sedi_stencil_apply(sedi_ctx *h, const double *x, double *y) {
	if (!h || !x || !y) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	const size_t bytes = sizeof(double) * (size_t)c->g.n;
	double *dx = nullptr, *dy = nullptr;
	CAPI_TRY(cudaMalloc(&dx, bytes));
	if (cudaMalloc(&dy, bytes) != cudaSuccess) {
		cudaFree(dx);
		return set_cuda_error(c, cudaErrorMemoryAllocation, "cudaMalloc");
	}
	int rc = 0;
	if (cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) rc = set_cuda_error(c, cudaGetLastError(), "H2D");
	if (!rc) rc = plain_stencil(c, dx, dy);
	if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = set_cuda_error(c, cudaGetLastError(), "stencil");
	if (!rc && (cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
	            cudaStreamSynchronize(c->stream) != cudaSuccess))
		rc = set_cuda_error(c, cudaGetLastError(), "D2H");
	cudaFree(dx);
	cudaFree(dy);
	return rc;
}

// Estimator loop shared by the seeded and the caller-probe entry points
// (stochastic-estimator.cc:158-216).
static int estimate_common(Ctx *c, int samples, uint32_t seed, const double *probes, int maxiter, double tol,
                           int ignore_errors, double *D, double *t, double *q, int *iters, double *errs,
                           int *results) {
	const long long n = c->g.n;
	const size_t bytes = sizeof(double) * (size_t)n;
	if (!plain_form(c)) {
		// Batched form: stage the probes in a context-owned device buffer
		// (reused across calls), run them as right-hand sides, copy D (t, q) back.
		const size_t need = bytes * (size_t)(samples > 0 ? samples : 1);
		if (probes && c->stage_probe_bytes < need) {
			if (c->stage_probes) cudaFree(c->stage_probes);
			c->stage_probes = nullptr;
			c->stage_probe_bytes = 0;
			if (cudaMalloc(&c->stage_probes, need) != cudaSuccess) {
				cudaGetLastError();
				c->error = "device allocation failed (probe staging)";
				return SEDI_ERR_NOMEM;
			}
			c->stage_probe_bytes = need;
		}
		if (!c->stage_out && cudaMalloc(&c->stage_out, 3 * bytes) != cudaSuccess) {
			cudaGetLastError();
			c->stage_out = nullptr;
			c->error = "device allocation failed (result staging)";
			return SEDI_ERR_NOMEM;
		}
		// Seeded probes are generated on the device (bit-identical to the host
		// generator); caller probes are uploaded.
		if (probes) CAPI_TRY(cudaMemcpyAsync(c->stage_probes, probes, need, cudaMemcpyHostToDevice, c->stream));
		double *dD = c->stage_out, *dt = c->stage_out + n, *dq = c->stage_out + 2 * n;
		int rc = batched_estimate_src(c, samples, probes ? c->stage_probes : nullptr, seed, maxiter, tol,
		                              ignore_errors, dD, dt, dq, iters, errs, results);
		if (rc < 0) return rc;
		CAPI_TRY(cudaMemcpyAsync(D, dD, bytes, cudaMemcpyDeviceToHost, c->stream));
		if (t) CAPI_TRY(cudaMemcpyAsync(t, dt, bytes, cudaMemcpyDeviceToHost, c->stream));
		if (q) CAPI_TRY(cudaMemcpyAsync(q, dq, bytes, cudaMemcpyDeviceToHost, c->stream));
		CAPI_TRY(cudaStreamSynchronize(c->stream));
		return rc;
	}
	double *host_probe = nullptr;
	CAPI_TRY(cudaMallocHost(&host_probe, bytes));
	int worst = 0;
	for (int k = 0; k < samples; k++) {
		if (probes) std::memcpy(host_probe, probes + (size_t)k * n, bytes);
		else host_fill_probe(seed + (uint32_t)k, (long)n, host_probe);  // :163-166
		cudaError_t e = cudaMemcpyAsync(c->b, host_probe, bytes, cudaMemcpyHostToDevice, c->stream);
		if (e == cudaSuccess) e = cudaMemsetAsync(c->x, 0, bytes, c->stream);  // :175
		if (e != cudaSuccess) {
			cudaFreeHost(host_probe);
			return set_cuda_error(c, e, "probe upload");
		}
		double fe = 0.0;
		int fi = 0;
		const int res = plain_solve_resident(c, false, maxiter, tol, &fe, &fi);  // :176-179
		if (res < 0) {
			cudaFreeHost(host_probe);
			return res;
		}
		if (iters) iters[k] = fi;
		if (errs) errs[k] = fe;
		if (results) results[k] = res;
		int rc = plain_accumulate(c, c->x, c->b, k == 0);  // :195, :198
		if (rc) {
			cudaFreeHost(host_probe);
			return rc;
		}
		if (res != 0 && !ignore_errors) {  // :181-184
			cudaFreeHost(host_probe);
			return res;
		}
		if (res > worst) worst = res;
	}
	cudaFreeHost(host_probe);
	if (samples == 0) {
		CAPI_TRY(cudaMemsetAsync(c->t_acc, 0, bytes, c->stream));
		CAPI_TRY(cudaMemsetAsync(c->q_acc, 0, bytes, c->stream));
	}
	int rc = plain_divide(c, c->r);  // :216 (r is free scratch after the solves)
	if (rc) return rc;
	CAPI_TRY(cudaMemcpyAsync(D, c->r, bytes, cudaMemcpyDeviceToHost, c->stream));
	if (t) CAPI_TRY(cudaMemcpyAsync(t, c->t_acc, bytes, cudaMemcpyDeviceToHost, c->stream));
	if (q) CAPI_TRY(cudaMemcpyAsync(q, c->q_acc, bytes, cudaMemcpyDeviceToHost, c->stream));
	CAPI_TRY(cudaStreamSynchronize(c->stream));
	return worst;
}

int sedi_estimate(sedi_ctx *h, int samples, uint32_t seed, int maxiter, double tol, int ignore_errors, double *D,
                  double *t, double *q, int *iters, double *errs, int *results) {
	if (!h || !D || samples < 0 || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	return estimate_common(c, samples, seed, nullptr, maxiter, tol, ignore_errors, D, t, q, iters, errs, results);
}

int sedi_estimate_probes(sedi_ctx *h, int samples, const double *probes, int maxiter, double tol,
                         int ignore_errors, double *D, double *t, double *q, int *iters, double *errs,
                         int *results) {
	if (!h || !D || !probes || samples < 0 || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	return estimate_common(c, samples, 0, probes, maxiter, tol, ignore_errors, D, t, q, iters, errs, results);
}

int sedi_set_stream(sedi_ctx *h, void *stream) {
	if (!h) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	c->stream = stream ? (cudaStream_t)stream : c->own_stream;
	return 0;
}

int sedi_estimate_dev(sedi_ctx *h, int samples, const double *probes_dev, int maxiter, double tol, int ignore_errors,
                      double *D_dev, double *t_dev, double *q_dev, int *iters, double *errs, int *results) {
	if (!h || !D_dev || !probes_dev || samples < 0 || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	if (!plain_form(c))
		return batched_estimate_dev(c, samples, probes_dev, maxiter, tol, ignore_errors, D_dev, t_dev, q_dev, iters,
		                            errs, results);
	const long long n = c->g.n;
	const size_t bytes = sizeof(double) * (size_t)n;
	int worst = 0;
	for (int k = 0; k < samples; k++) {
		CAPI_TRY(cudaMemcpyAsync(c->b, probes_dev + (size_t)k * n, bytes, cudaMemcpyDeviceToDevice, c->stream));
		CAPI_TRY(cudaMemsetAsync(c->x, 0, bytes, c->stream));
		double fe = 0.0;
		int fi = 0;
		const int res = plain_solve_resident(c, false, maxiter, tol, &fe, &fi);
		if (res < 0) return res;
		if (iters) iters[k] = fi;
		if (errs) errs[k] = fe;
		if (results) results[k] = res;
		int rc = plain_accumulate(c, c->x, c->b, k == 0);
		if (rc) return rc;
		if (res != 0 && !ignore_errors) return res;
		if (res > worst) worst = res;
	}
	if (samples == 0) {
		CAPI_TRY(cudaMemsetAsync(c->t_acc, 0, bytes, c->stream));
		CAPI_TRY(cudaMemsetAsync(c->q_acc, 0, bytes, c->stream));
	}
	int rc = plain_divide(c, D_dev);
	if (rc) return rc;
	if (t_dev) CAPI_TRY(cudaMemcpyAsync(t_dev, c->t_acc, bytes, cudaMemcpyDeviceToDevice, c->stream));
	if (q_dev) CAPI_TRY(cudaMemcpyAsync(q_dev, c->q_acc, bytes, cudaMemcpyDeviceToDevice, c->stream));
	CAPI_TRY(cudaStreamSynchronize(c->stream));
	return worst;
}

int sedi_time_kernels(sedi_ctx *h, int reps, double *ms, double *bytes, char *names, int *count) {
	if (!h || reps < 1 || !ms || !bytes || !names || !count) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	if (plain_form(c)) {
		*count = 0;
		return pairs_time_kernels(c, reps, ms, bytes, names, count);  // unsupported for odd n1
	}
	return batched_time_kernels(c, reps, ms, bytes, names, count);
}

int sedi_solve_batch(sedi_ctx *h, int nrhs, const double *b, double *x, int maxiter, double tol, double *final_err,
                     int *final_iter, int *results) {
	if (!h || !b || !x || !final_err || !final_iter || !results || nrhs < 0 || maxiter < 0) return SEDI_ERR_ARG;
	Ctx *c = &h->c;
	cudaSetDevice(c->device);
	const long long n = c->g.n;
	const size_t bytes = sizeof(double) * (size_t)n;
	if (plain_form(c)) {
		int worst = 0;
		for (int k = 0; k < nrhs; k++) {
			const int rc = sedi_solve(h, b + (size_t)k * n, x + (size_t)k * n, nullptr, maxiter, tol, &final_err[k],
			                          &final_iter[k]);
			if (rc < 0) return rc;
			results[k] = rc;
			if (rc > worst) worst = rc;
		}
		return worst;
	}
	double *db = nullptr, *dx = nullptr;
	const size_t all = bytes * (size_t)(nrhs > 0 ? nrhs : 1);
	CAPI_TRY(cudaMalloc(&db, all));
	if (cudaMalloc(&dx, all) != cudaSuccess) {
		cudaFree(db);
		return set_cuda_error(c, cudaErrorMemoryAllocation, "cudaMalloc");
	}
	int rc = 0;
	if (cudaMemcpyAsync(db, b, bytes * nrhs, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
	    cudaMemcpyAsync(dx, x, bytes * nrhs, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
		rc = set_cuda_error(c, cudaGetLastError(), "upload");
	if (!rc) rc = batched_solve_dev(c, nrhs, db, dx, maxiter, tol, final_err, final_iter, results);
	if (rc >= 0 && (cudaMemcpyAsync(x, dx, bytes * nrhs, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
	                cudaStreamSynchronize(c->stream) != cudaSuccess))
		rc = set_cuda_error(c, cudaGetLastError(), "download");
	cudaFree(db);
	cudaFree(dx);
	return rc;
}

}  // extern "C"
