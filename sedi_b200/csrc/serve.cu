// Estimation-job server: continuous admission of estimator jobs of any grid
// size, sample count, tolerance, solver and precision onto one GPU.
//
// Every job runs on a batched context (its own CUDA stream, its Krylov state
// resident in device memory, one captured graph per context).  The server
// advances all running jobs without blocking: each step polls every job's
// event and enqueues that job's next piece of work (the next graph chunk of
// 16 iterations, the lane results and accumulation of a finished batch, the
// next batch, the final D = t / q and its copy to pinned host memory).  Jobs
// on different streams overlap on the device.
//
// Admission: a job needs the device bytes of its context
// (batched_bytes(solver, precision, lanes, grid)).  Queued jobs are admitted
// in arrival order while the bytes in use stay within the budget and fewer
// than max_active jobs run; when the oldest queued job does not fit, later
// jobs that do fit may start ahead of it, at most kMaxBypass of them, so a
// large job is never starved.  Finished contexts stay allocated as idle slots
// and are reused by later jobs of the same solver, precision, grid and padded
// lane count (no allocation, no graph instantiation); idle slots are freed
// oldest first when a new context needs their memory.
//
// A job's lane count depends only on the job and the server's per-job byte
// cap, never on the load, and every reduction runs in a fixed order, so a
// job's result is the same alone and in any mix.  A context's launch shapes
// depend only on its padded lane count, so a job whose probes fit one batch
// may run on any context of its padded lane count with room for them (new
// contexts are created with every padded lane usable); a job of several
// batches runs only on contexts of its own batch size.
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <thread>
#include <vector>

#include "sedi_internal.h"

namespace sedi {
namespace {

constexpr int kMaxBypass = 4;

struct Key {
	int solver, precision, lanes;  // lanes: padded right-hand sides of the context
	long long n1, n2, n3;
	bool operator==(const Key &o) const {
		return solver == o.solver && precision == o.precision && lanes == o.lanes && n1 == o.n1 && n2 == o.n2 &&
		       n3 == o.n3;
	}
};

struct Slot {
	sedi_ctx *h = nullptr;
	Key key;
	int batch = 0;  // right-hand sides per batch of the context
	size_t bytes = 0;
	double *D_host = nullptr;  // pinned, n doubles
	bool busy = false;
	double last_used = 0.0;
};

enum JobState { JOB_QUEUED = 0, JOB_RUNNING = 1, JOB_DONE = 2, JOB_FAILED = 3 };

struct Job {
	long id = 0;
	Key key;
	int lanes = 0;  // right-hand sides per batch (the job's own context batch)
	int samples = 0, maxiter = 0;
	uint32_t seed = 0;
	double tol = 0.0;
	size_t bytes = 0;
	int state = JOB_QUEUED, rc = 0, bypassed = 0;
	double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
	Slot *slot = nullptr;
	std::vector<double> D, errs;
	std::vector<int> iters, results;
};

}  // namespace
}  // namespace sedi

using namespace sedi;

struct sedi_server {
	size_t budget = 0, used = 0, peak = 0, job_cap = 0;
	int max_active = 8;
	int device = 0;
	std::vector<Slot *> slots;
	std::deque<long> queue;
	std::vector<long> running;
	std::map<long, Job> jobs;
	long next_id = 0;
	int completed = 0, created = 0, reused = 0, max_running = 0;
	long long launches_done = 0;
	std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
	double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// Lane count of a job: all samples in one batch when that context fits the
// per-job cap, else the largest lane count that does (at least 2: the
// batched form).
int job_lanes(const sedi_server *S, int solver, int precision, int samples, long long n1, long long n2,
              long long n3) {
	int b = samples < 1 ? 1 : samples;
	const int cap = precision == SEDI_PREC_FP64 ? 128 : 256;
	if (b > cap) b = cap;
	while (b > 2 && batched_bytes(solver, precision, b, n1, n2, n3) > S->job_cap) b = b > 16 ? b - 16 : b / 2;
	return b < 2 ? 2 : b;  // one lane would select the single-vector form
}

void free_slot(sedi_server *S, Slot *sl) {
	sedi_destroy(sl->h);
	if (sl->D_host) cudaFreeHost(sl->D_host);
	S->used -= sl->bytes;
	delete sl;
}

// An idle slot of this shape, or a new one if the budget allows (freeing idle
// slots oldest first).  nullptr when the job cannot start now.
Slot *acquire(sedi_server *S, const Job &J, int *err) {
	*err = 0;
	const bool one_batch = J.lanes >= J.samples;
	for (Slot *sl : S->slots)
		if (!sl->busy && sl->key == J.key && (one_batch ? sl->batch >= J.samples : sl->batch == J.lanes)) {
			S->reused++;
			return sl;
		}
	size_t idle = 0;
	for (Slot *sl : S->slots)
		if (!sl->busy) idle += sl->bytes;
	if (S->used - idle + J.bytes > S->budget) return nullptr;  // does not fit even with every idle slot freed
	while (S->used + J.bytes > S->budget) {
		Slot *old = nullptr;
		size_t oi = 0;
		for (size_t i = 0; i < S->slots.size(); i++)
			if (!S->slots[i]->busy && (!old || S->slots[i]->last_used < old->last_used)) {
				old = S->slots[i];
				oi = i;
			}
		if (!old) return nullptr;
		S->slots.erase(S->slots.begin() + (long)oi);
		free_slot(S, old);
	}
	Slot *sl = new (std::nothrow) Slot();
	if (!sl) {
		*err = SEDI_ERR_NOMEM;
		return nullptr;
	}
	sl->key = J.key;
	sl->batch = one_batch ? J.key.lanes : J.lanes;
	sl->bytes = J.bytes;
	sl->h = sedi_create(J.key.solver, (long)J.key.n1, (long)J.key.n2, (long)J.key.n3, 6.0, 1.0, 1.0, 0,
	                    J.key.precision, sl->batch, err);
	if (!sl->h || cudaMallocHost(&sl->D_host, sizeof(double) * (size_t)(J.key.n1 * J.key.n2 * J.key.n3)) != cudaSuccess) {
		cudaGetLastError();
		if (!*err) *err = SEDI_ERR_NOMEM;
		if (sl->h) sedi_destroy(sl->h);
		delete sl;
		return nullptr;
	}
	S->used += sl->bytes;
	if (S->used > S->peak) S->peak = S->used;
	S->slots.push_back(sl);
	S->created++;
	return sl;
}

void finish(sedi_server *S, Job &J, int rc) {
	J.rc = rc;
	J.state = rc < 0 ? JOB_FAILED : JOB_DONE;
	J.t_done = S->now();
	S->completed++;
}

int start(sedi_server *S, Job &J, Slot *sl) {
	sl->busy = true;
	J.slot = sl;
	J.state = JOB_RUNNING;
	J.t_start = S->now();
	J.iters.assign(J.samples, 0);
	J.errs.assign(J.samples, 0.0);
	J.results.assign(J.samples, 0);
	Ctx *c = &sl->h->c;
	const int rc = batched_est_begin(c, J.samples, nullptr, J.seed, J.maxiter, J.tol, 1, nullptr, nullptr, nullptr,
	                                 sl->D_host, J.iters.data(), J.errs.data(), J.results.data());
	if (rc) {
		sl->busy = false;
		finish(S, J, rc);
		return rc;
	}
	S->running.push_back(J.id);
	if ((int)S->running.size() > S->max_running) S->max_running = (int)S->running.size();
	return 0;
}

void admit(sedi_server *S) {
	size_t qi = 0;
	while (qi < S->queue.size() && (int)S->running.size() < S->max_active) {
		Job &head = S->jobs[S->queue.front()];
		if (qi > 0 && head.bypassed >= kMaxBypass) break;
		Job &J = S->jobs[S->queue[qi]];
		int err = 0;
		Slot *sl = acquire(S, J, &err);
		if (!sl) {
			// Out of device memory with other jobs running: wait for them.
			if (err && !(err == SEDI_ERR_NOMEM && !S->running.empty())) {
				finish(S, J, err);
				S->queue.erase(S->queue.begin() + (long)qi);
			} else {
				qi++;
			}
			continue;
		}
		if (qi > 0) head.bypassed++;
		S->queue.erase(S->queue.begin() + (long)qi);
		start(S, J, sl);
	}
}

void poll(sedi_server *S) {
	for (size_t i = 0; i < S->running.size();) {
		Job &J = S->jobs[S->running[i]];
		Ctx *c = &J.slot->h->c;
		int done = 0;
		const int rc = batched_est_advance(c, &done);
		if (!done && rc == 0) {
			i++;
			continue;
		}
		const int res = rc < 0 ? rc : batched_est_result(c);
		if (res >= 0) {
			const long long n = J.key.n1 * J.key.n2 * J.key.n3;
			J.D.assign(J.slot->D_host, J.slot->D_host + n);
		}
		S->launches_done += c->launches;
		c->launches = 0;
		J.slot->busy = false;
		J.slot->last_used = S->now();
		J.slot = nullptr;
		finish(S, J, res);
		S->running.erase(S->running.begin() + (long)i);
	}
}

}  // namespace

extern "C" {

sedi_server *sedi_server_create(double budget_bytes, int max_active, double job_cap_bytes, int *err) {
	int dummy;
	if (!err) err = &dummy;
	*err = 0;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
		cudaGetLastError();
		*err = SEDI_ERR_NODEV;
		return nullptr;
	}
	if (budget_bytes < 0 || max_active < 0 || job_cap_bytes < 0) {
		*err = SEDI_ERR_ARG;
		return nullptr;
	}
	sedi_server *S = new (std::nothrow) sedi_server();
	if (!S) {
		*err = SEDI_ERR_NOMEM;
		return nullptr;
	}
	cudaGetDevice(&S->device);
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	S->budget = budget_bytes > 0 ? (size_t)budget_bytes : (size_t)(0.85 * (double)fr);
	S->job_cap = job_cap_bytes > 0 ? (size_t)job_cap_bytes : (size_t)32 << 30;
	if (S->job_cap > S->budget) S->job_cap = S->budget;
	S->max_active = max_active > 0 ? max_active : 8;
	return S;
}

void sedi_server_destroy(sedi_server *S) {
	if (!S) return;
	cudaSetDevice(S->device);
	for (Slot *sl : S->slots) free_slot(S, sl);
	delete S;
}

long sedi_server_submit(sedi_server *S, int solver, int precision, long n1, long n2, long n3, int samples,
                        uint32_t seed, int maxiter, double tol) {
	if (!S || solver < 1 || solver > 3 || (precision != SEDI_PREC_FP64 && precision != SEDI_PREC_MIXED) || n1 < 1 ||
	    n2 < 1 || n3 < 1 || samples < 0 || maxiter < 0 || !(tol >= 0.0))
		return SEDI_ERR_ARG;
	Job J;
	J.id = S->next_id++;
	J.key.solver = solver;
	J.key.precision = precision;
	J.key.n1 = n1;
	J.key.n2 = n2;
	J.key.n3 = n3;
	J.lanes = job_lanes(S, solver, precision, samples, n1, n2, n3);
	J.key.lanes = batched_lanes(precision, J.lanes);
	J.bytes = batched_bytes(solver, precision, J.lanes, n1, n2, n3);
	if (J.bytes > S->budget) return SEDI_ERR_NOMEM;
	J.samples = samples;
	J.seed = seed;
	J.maxiter = maxiter;
	J.tol = tol;
	J.t_submit = S->now();
	const long id = J.id;
	S->jobs[id] = std::move(J);
	S->queue.push_back(id);
	return id;
}

int sedi_server_step(sedi_server *S, int *completed) {
	if (!S) return SEDI_ERR_ARG;
	cudaSetDevice(S->device);
	poll(S);
	admit(S);
	if (completed) *completed = S->completed;
	return (int)(S->queue.size() + S->running.size());
}

int sedi_server_wait(sedi_server *S, long id) {
	if (!S) return SEDI_ERR_ARG;
	if (id >= 0 && !S->jobs.count(id)) return SEDI_ERR_ARG;
	for (;;) {
		const int pending = sedi_server_step(S, nullptr);
		if (pending < 0) return pending;
		if (id >= 0 ? S->jobs[id].state >= JOB_DONE : pending == 0) return 0;
		std::this_thread::yield();
	}
}

int sedi_server_job_info(sedi_server *S, long id, int *state, int *rc, double *t_submit, double *t_start,
                         double *t_done, int *lanes, double *bytes) {
	if (!S || !S->jobs.count(id)) return SEDI_ERR_ARG;
	const Job &J = S->jobs[id];
	if (state) *state = J.state;
	if (rc) *rc = J.rc;
	if (t_submit) *t_submit = J.t_submit;
	if (t_start) *t_start = J.t_start;
	if (t_done) *t_done = J.t_done;
	if (lanes) *lanes = J.lanes;
	if (bytes) *bytes = (double)J.bytes;
	return 0;
}

int sedi_server_take(sedi_server *S, long id, double *D, int *iters, double *errs, int *results) {
	if (!S || !S->jobs.count(id)) return SEDI_ERR_ARG;
	Job &J = S->jobs[id];
	if (J.state < JOB_DONE) return SEDI_ERR_ARG;
	const int rc = J.rc;
	if (J.state == JOB_DONE) {
		if (D) std::memcpy(D, J.D.data(), sizeof(double) * J.D.size());
		if (iters) std::memcpy(iters, J.iters.data(), sizeof(int) * J.iters.size());
		if (errs) std::memcpy(errs, J.errs.data(), sizeof(double) * J.errs.size());
		if (results) std::memcpy(results, J.results.data(), sizeof(int) * J.results.size());
	}
	S->jobs.erase(id);
	return rc;
}

int sedi_server_replay(sedi_server *S, int njobs, const double *arrival_s, const int *solver, const int *precision,
                       const long *edge, const int *samples, const uint32_t *seed, const double *tol, int maxiter,
                       double *latency_s, int *rcs, double *makespan_s, long long *iterations) {
	if (!S || njobs < 0 || (njobs && (!arrival_s || !solver || !precision || !edge || !samples || !seed || !tol ||
	                                  !latency_s)))
		return SEDI_ERR_ARG;
	for (int k = 1; k < njobs; k++)
		if (arrival_s[k] < arrival_s[k - 1]) return SEDI_ERR_ARG;
	std::vector<long> ids(njobs, -1);
	const double base = S->now();
	int next = 0, done = 0;
	std::vector<char> finished(njobs, 0);
	while (done < njobs) {
		const double t = S->now() - base;
		while (next < njobs && arrival_s[next] <= t) {
			const long id = sedi_server_submit(S, solver[next], precision[next], edge[next], edge[next], edge[next],
			                                   samples[next], seed[next], maxiter, tol[next]);
			if (id < 0) return (int)id;
			S->jobs[id].t_submit = base + arrival_s[next];  // latency counts from the scheduled arrival
			ids[next++] = id;
		}
		const int pending = sedi_server_step(S, nullptr);
		if (pending < 0) return pending;
		for (int k = 0; k < next; k++) {
			if (finished[k]) continue;
			const Job &J = S->jobs[ids[k]];
			if (J.state >= JOB_DONE) {
				finished[k] = 1;
				done++;
				latency_s[k] = J.t_done - J.t_submit;
				if (rcs) rcs[k] = J.rc;
				if (iterations) {
					long long it = 0;
					for (int v : J.iters) it += v;
					iterations[k] = it;
				}
			}
		}
		if (pending == 0 && next < njobs) {
			const double wait = arrival_s[next] - (S->now() - base);
			if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait < 1e-3 ? wait : 1e-3));
		} else {
			std::this_thread::yield();
		}
	}
	if (makespan_s) *makespan_s = S->now() - base;
	for (int k = 0; k < njobs; k++) S->jobs.erase(ids[k]);
	return 0;
}

int sedi_server_stats(const sedi_server *S, double *peak_bytes, double *budget_bytes, int *ctx_created,
                      int *ctx_reused, int *max_running, long long *launches) {
	if (!S) return SEDI_ERR_ARG;
	if (peak_bytes) *peak_bytes = (double)S->peak;
	if (budget_bytes) *budget_bytes = (double)S->budget;
	if (ctx_created) *ctx_created = S->created;
	if (ctx_reused) *ctx_reused = S->reused;
	if (max_running) *max_running = S->max_running;
	if (launches) *launches = S->launches_done;
	return 0;
}

double sedi_job_bytes(int solver, int precision, int lanes, long n1, long n2, long n3) {
	if (solver < 1 || solver > 3 || lanes < 1 || n1 < 1 || n2 < 1 || n3 < 1) return 0.0;
	return (double)batched_bytes(solver, precision, lanes, n1, n2, n3);
}

}  // extern "C"
