// Single-vector FP64 form of the three reference solvers on sm_100a.
//
// Each solver iteration is a short, fixed sequence of fused kernels.  Every
// elementwise value the reference stores (Stencil.hpp:43-50,
// SliceOps.hpp:17-108) is computed with the same operations in the same
// order, without FMA contraction, so it rounds identically; intermediates the
// reference stores only to read them back (u = r.*iM, s = A p, m = w.*iM,
// p_hat = p.*iM, s_hat = s.*iM, n = A m, and the stencil inputs at
// neighbouring points) are recomputed in registers instead of round-tripping
// through HBM.  Dot products are two-stage deterministic reductions whose
// last block also computes the Krylov scalars, so an iteration needs no host
// synchronisation; a CUDA graph replays a chunk of iterations and kernels
// after the stopping iteration return at once.
#include <cmath>
#include <cstdio>

#include "sedi_internal.h"

namespace sedi {

namespace {

template <bool VIM>
struct IMv {
	const double *v;
	double c;
	__device__ __forceinline__ double operator()(long long i) const { return VIM ? __ldg(v + i) : c; }
};

__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }
__device__ __forceinline__ long long gstart() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

// Sweep launch shape: 32x8 column tiles, i3 split into chunks so that the
// grid has about 6 blocks per SM.
struct Launch {
	dim3 grid;
	int zc;
};

static Launch launch_shape(const Geo &g) {
	const int gx = (g.n1 + kTile1 - 1) / kTile1, gy = (g.n2 + kTile2 - 1) / kTile2;
	long long want = 148LL * 6;
	long long nz = (want + (long long)gx * gy - 1) / ((long long)gx * gy);
	if (nz < 1) nz = 1;
	if (nz > g.n3) nz = g.n3;
	const int zc = (int)((g.n3 + nz - 1) / nz);
	nz = (g.n3 + zc - 1) / zc;
	Launch l;
	l.grid = dim3(gx, gy, (unsigned)nz);
	l.zc = zc;
	return l;
}

// ---------------------------------------------------------------------------
// Setup: r = b - A x (Cg.hpp:119-123), <b,b> (:112-115), <r,r> (:126-129),
// r_hat = r for BiCGStab (BiCgStab.hpp:153).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_setup(Geo g, Coef k, int zc, const double *__restrict__ x,
                                                    const double *__restrict__ b, double *__restrict__ r,
                                                    double *__restrict__ rhat, double *partials, unsigned *ticket,
                                                    SolveState *st, double *hist, double tol, int maxiter,
                                                    int solver) {
	double v[2] = {0.0, 0.0};
	march(g, k, sweep(g, zc), [&](long long j) { return __ldg(x + j); }, [&](long long i, double, double ax) {
		const double bi = __ldg(b + i);
		const double ri = add(bi, mul(-1.0, ax));  // combine2(1.0, b, -1.0, r, r)
		r[i] = ri;
		if (rhat) rhat[i] = ri;
		v[0] = fma(bi, bi, v[0]);
		v[1] = fma(ri, ri, v[1]);
	});
	double out[2];
	if (grid_sum<2>(v, partials, ticket, out) && threadIdx.x == 0) {
		SolveState s = {};
		s.tol = tol;
		s.maxiter = maxiter;
		s.bb = out[0] == 0.0 ? 1.0 : out[0];
		s.rr = out[1];
		s.err = sqrt(__ddiv_rn(s.rr, s.bb));
		hist[0] = s.err;
		s.iter = 1;
		s.omega = 1.0;  // BiCgStab.hpp:147-150
		if (s.err < tol) {
			s.done = 1;
			s.exit_iter = 0;
			s.reason = STOP_EARLY;
		} else if (maxiter < 1) {
			s.done = 1;
			s.exit_iter = 1;  // the reference loop variable after zero passes
			s.reason = STOP_MAXITER;
		} else if (solver == 1) {
			s.rho = s.rr;  // <r, r_hat> with r_hat == r (BiCgStab.hpp:159-160)
			if (s.rho == 0.0) {
				s.done = 1;
				s.exit_iter = 1;
				s.reason = STOP_RHO;
			}
		}
		*st = s;
	}
}

// ---------------------------------------------------------------------------
// CG (Cg.hpp:150-194), two kernels per iteration.
//   A: p = u + beta p (u = r.*iM; p = u on iteration 1), s = A p, <s,p>
//      (and <r,u> on iteration 1); alpha = <r,u>/<s,p>.
//   B: s = A p again, x += alpha p, r -= alpha s, u = r.*iM, <r,u>, <r,r>;
//      beta, err, stop test.
// p ping-pongs between two buffers because neighbours are read while the
// kernel writes the new p.
// ---------------------------------------------------------------------------
template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_cg_a(Geo g, Coef k, int zc, IMv<VIM> im, const double *__restrict__ r,
                                                   double *p0, double *p1, double *partials, unsigned *ticket,
                                                   SolveState *st) {
	if (st->done) return;
	const int it = st->iter;
	const bool first = (it == 1);
	const double beta = st->beta;
	const double *__restrict__ pold = (it & 1) ? p0 : p1;
	double *__restrict__ pnew = (it & 1) ? p1 : p0;
	auto pn = [&](long long j) {
		const double uj = mul(__ldg(r + j), im(j));       // u = r .* iM (:175)
		return first ? uj : add(uj, mul(beta, __ldg(pold + j)));  // p = 1*u + beta*p (:188)
	};
	double v[2] = {0.0, 0.0};
	march(g, k, sweep(g, zc), pn, [&](long long i, double pi, double si) {
		pnew[i] = pi;
		v[0] = fma(si, pi, v[0]);
		if (first) {
			const double ri = __ldg(r + i);
			v[1] = fma(ri, mul(ri, im(i)), v[1]);
		}
	});
	double out[2];
	if (grid_sum<2>(v, partials, ticket, out) && threadIdx.x == 0) {
		st->sp = out[0];
		const double ru = first ? out[1] : st->ru_new;  // :157-163
		st->ru = ru;
		st->alpha = __ddiv_rn(ru, out[0]);               // :166
	}
}

template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_cg_b(Geo g, Coef k, int zc, IMv<VIM> im, double *__restrict__ x,
                                                   double *__restrict__ r, const double *p0, const double *p1,
                                                   double *partials, unsigned *ticket, SolveState *st,
                                                   double *hist) {
	if (st->done) return;
	const int it = st->iter;
	const double alpha = st->alpha;
	const double *__restrict__ p = (it & 1) ? p1 : p0;
	double v[2] = {0.0, 0.0};
	march(g, k, sweep(g, zc), [&](long long j) { return __ldg(p + j); }, [&](long long i, double pi, double si) {
		x[i] = add(x[i], mul(alpha, pi));              // :169
		const double ri = add(r[i], mul(-alpha, si));  // :172
		r[i] = ri;
		const double ui = mul(ri, im(i));                        // :175
		v[0] = fma(ri, ui, v[0]);
		v[1] = fma(ri, ri, v[1]);
	});
	double out[2];
	if (grid_sum<2>(v, partials, ticket, out) && threadIdx.x == 0) {
		st->ru_new = out[0];                               // :179-181
		st->rr = out[1];
		st->beta = __ddiv_rn(out[0], st->ru);              // :185
		const double err = sqrt(__ddiv_rn(out[1], st->bb));  // :191
		st->err = err;
		hist[it] = err;
		if (err <= st->tol) {                               // :193
			st->done = 1;
			st->exit_iter = it;
			st->reason = STOP_CONVERGED;
		} else if (it >= st->maxiter) {
			st->done = 1;
			st->exit_iter = st->maxiter + 1;
			st->reason = STOP_MAXITER;
		}
		st->iter = it + 1;
	}
}

// ---------------------------------------------------------------------------
// Pipelined CG (PipelinedCg.hpp:136-230).
// Setup2: u = r.*iM (:138), w = A u (:141-143), z=q=s=p=0 (:146-149) and the
// first iteration's <r,u>, <w,u>, <r,r> (:155).
// Iteration: one kernel.  m = w.*iM (:158), n = A m (:161-184), the eight
// fused updates (:199-221) and the next iteration's three dots.  w
// ping-pongs (neighbours of w are read while the new w is written).
// ---------------------------------------------------------------------------
template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_pcg_setup(Geo g, Coef k, int zc, IMv<VIM> im,
                                                        const double *__restrict__ r, double *__restrict__ u,
                                                        double *__restrict__ w, double *__restrict__ zq,
                                                        double *__restrict__ qq, double *__restrict__ ss,
                                                        double *__restrict__ pp, double *partials, unsigned *ticket,
                                                        SolveState *st) {
	if (st->done) return;
	auto uf = [&](long long j) { return mul(__ldg(r + j), im(j)); };
	double v[3] = {0.0, 0.0, 0.0};
	march(g, k, sweep(g, zc), uf, [&](long long i, double ui, double wi) {
		const double ri = __ldg(r + i);
		u[i] = ui;
		w[i] = wi;
		zq[i] = 0.0;
		qq[i] = 0.0;
		ss[i] = 0.0;
		pp[i] = 0.0;
		v[0] = fma(ri, ui, v[0]);
		v[1] = fma(wi, ui, v[1]);
		v[2] = fma(ri, ri, v[2]);
	});
	double out[3];
	if (grid_sum<3>(v, partials, ticket, out) && threadIdx.x == 0) {
		st->gamma = out[0];
		st->delta = out[1];
		st->rr_top = out[2];
		st->gamma_old = 0.0;
		st->alpha = 0.0;
		st->wsel = 0;
	}
}

template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_pcg_iter(Geo g, Coef k, int zc, IMv<VIM> im, double *__restrict__ x,
                                                       double *__restrict__ r, double *__restrict__ u, double *w0,
                                                       double *w1, double *__restrict__ qv, double *__restrict__ sv,
                                                       double *__restrict__ pv, double *__restrict__ zv,
                                                       double *partials, unsigned *ticket, SolveState *st,
                                                       double *hist) {
	if (st->done) return;
	const int it = st->iter;
	const double gamma = st->gamma, delta = st->delta;
	double alpha, beta;
	if (it > 1) {  // :175-178
		beta = __ddiv_rn(gamma, st->gamma_old);
		alpha = __ddiv_rn(1.0, __dsub_rn(__ddiv_rn(delta, gamma), __ddiv_rn(beta, st->alpha)));
	} else {       // :179-181
		beta = 0.0;
		alpha = __ddiv_rn(gamma, delta);
	}
	const double *__restrict__ wc = st->wsel ? w1 : w0;
	double *__restrict__ wn = st->wsel ? w0 : w1;
	auto mf = [&](long long j) { return mul(__ldg(wc + j), im(j)); };
	double v[3] = {0.0, 0.0, 0.0};
	march(g, k, sweep(g, zc), mf, [&](long long i, double mi, double ni) {
		const double wi = __ldg(wc + i);
		const double qi = add(mi, mul(beta, qv[i]));   // :200
		const double si = add(wi, mul(beta, sv[i]));   // :203
		const double ui0 = u[i];
		const double pi = add(ui0, mul(beta, pv[i]));  // :206
		const double zi = add(ni, mul(beta, zv[i]));   // :209
		const double ri = add(r[i], mul(-alpha, si));  // :212
		const double xi = add(x[i], mul(alpha, pi));   // :215
		const double ui = add(ui0, mul(-alpha, qi));   // :218
		const double wni = add(wi, mul(-alpha, zi));   // :221
		qv[i] = qi;
		sv[i] = si;
		pv[i] = pi;
		zv[i] = zi;
		r[i] = ri;
		x[i] = xi;
		u[i] = ui;
		wn[i] = wni;
		v[0] = fma(ri, ui, v[0]);   // next gamma  = <r,u>
		v[1] = fma(wni, ui, v[1]);  // next delta  = <w,u>
		v[2] = fma(ri, ri, v[2]);   // next <r,r>
	});
	double out[3];
	if (grid_sum<3>(v, partials, ticket, out) && threadIdx.x == 0) {
		// The stop test uses <r,r> from the top of this iteration (:173, :227).
		const double err = sqrt(__ddiv_rn(st->rr_top, st->bb));
		st->err = err;
		st->rr = st->rr_top;
		hist[it] = err;
		st->gamma_old = gamma;
		st->alpha = alpha;
		st->beta = beta;
		st->gamma = out[0];
		st->delta = out[1];
		st->rr_top = out[2];
		st->wsel ^= 1;
		if (err <= st->tol) {
			st->done = 1;
			st->exit_iter = it;
			st->reason = STOP_CONVERGED;
		} else if (it >= st->maxiter) {
			st->done = 1;
			st->exit_iter = st->maxiter + 1;
			st->reason = STOP_MAXITER;
		}
		st->iter = it + 1;
	}
}

// ---------------------------------------------------------------------------
// BiCGStab (BiCgStab.hpp:157-232), three kernels per iteration.
//   1: p = r + beta p - beta omega v (p = r on iteration 1), p_hat = p.*iM,
//      v = A p_hat, <v,r_hat>; alpha = rho/<v,r_hat>.
//   2: s = r - alpha v, s_hat = s.*iM, t = A s_hat; <s,s>, <t,s>, <t,t>;
//      early exit flag on <s,s> < tol^2, omega = <t,s>/<t,t>.
//   3: x += alpha p_hat (+ omega s_hat), r = s - omega t, <r,r>, next
//      rho = <r,r_hat>; stop tests.
// p, v and r ping-pong (their neighbours are read while new values are
// written).  s, s_hat, t are never stored.
// ---------------------------------------------------------------------------
template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_bicg_1(Geo g, Coef k, int zc, IMv<VIM> im, const double *r0,
                                                     const double *r1, const double *__restrict__ rhat, double *p0,
                                                     double *p1, double *v0, double *v1, double *partials,
                                                     unsigned *ticket, SolveState *st) {
	if (st->done) return;
	const int it = st->iter;
	const bool first = (it == 1);
	const double rho = st->rho;
	double beta = 0.0, bo = 0.0;
	if (!first) {
		beta = __dmul_rn(__ddiv_rn(rho, st->rho_prev), __ddiv_rn(st->alpha, st->omega));  // :166
		bo = __dmul_rn(-beta, st->omega);                                                     // -beta*omega
	}
	const int sel = st->wsel;  // r buffer in use
	const double *__restrict__ r = sel ? r1 : r0;
	const double *__restrict__ pold = (it & 1) ? p0 : p1;
	double *__restrict__ pnew = (it & 1) ? p1 : p0;
	const double *__restrict__ vold = (it & 1) ? v0 : v1;
	double *__restrict__ vnew = (it & 1) ? v1 : v0;
	auto pf = [&](long long j) {
		const double rj = __ldg(r + j);
		return first ? rj : add(add(rj, mul(beta, __ldg(pold + j))), mul(bo, __ldg(vold + j)));  // :168
	};
	auto phf = [&](long long j) { return mul(pf(j), im(j)); };  // :175
	double v[1] = {0.0};
	march(g, k, sweep(g, zc), phf, [&](long long i, double, double vi) {  // v = A p_hat (:178-180)
		pnew[i] = pf(i);
		vnew[i] = vi;
		v[0] = fma(vi, __ldg(rhat + i), v[0]);
	});
	double out[1];
	if (grid_sum<1>(v, partials, ticket, out) && threadIdx.x == 0) {
		st->vr = out[0];
		st->alpha = __ddiv_rn(rho, out[0]);  // :186
	}
}

template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_bicg_2(Geo g, Coef k, int zc, IMv<VIM> im, const double *r0,
                                                     const double *r1, const double *v0, const double *v1,
                                                     double *partials, unsigned *ticket, SolveState *st) {
	if (st->done) return;
	const int it = st->iter;
	const double alpha = st->alpha;
	const double *__restrict__ r = st->wsel ? r1 : r0;
	const double *__restrict__ vv = (it & 1) ? v1 : v0;
	auto sf = [&](long long j) { return add(__ldg(r + j), mul(-alpha, __ldg(vv + j))); };  // :189
	auto shf = [&](long long j) { return mul(sf(j), im(j)); };                                        // :201
	double v[3] = {0.0, 0.0, 0.0};
	march(g, k, sweep(g, zc), shf, [&](long long i, double, double ti) {  // t = A s_hat (:204-206)
		const double si = sf(i);
		v[0] = fma(si, si, v[0]);
		v[1] = fma(ti, si, v[1]);
		v[2] = fma(ti, ti, v[2]);
	});
	double out[3];
	if (grid_sum<3>(v, partials, ticket, out) && threadIdx.x == 0) {
		st->s_norm2 = out[0];  // :192-193
		st->ts = out[1];
		st->tt = out[2];
		if (out[0] < __dmul_rn(st->tol, st->tol)) {
			st->s_exit = 1;    // :194
		} else {
			st->s_exit = 0;
			st->omega = __ddiv_rn(out[1], out[2]);  // :212
		}
	}
}

template <bool VIM>
__global__ void __launch_bounds__(kThreads) k_bicg_3(Geo g, Coef k, int zc, IMv<VIM> im, double *__restrict__ x,
                                                     double *r0, double *r1, const double *__restrict__ rhat,
                                                     const double *p0, const double *p1, const double *v0,
                                                     const double *v1, double *partials, unsigned *ticket,
                                                     SolveState *st, double *hist) {
	if (st->done) return;
	const int it = st->iter;
	const double alpha = st->alpha, omega = st->omega;
	const bool s_exit = st->s_exit != 0;
	const int sel = st->wsel;
	const double *__restrict__ r = sel ? r1 : r0;
	double *__restrict__ rn = sel ? r0 : r1;
	const double *__restrict__ p = (it & 1) ? p1 : p0;
	const double *__restrict__ vv = (it & 1) ? v1 : v0;
	auto sf = [&](long long j) { return add(__ldg(r + j), mul(-alpha, __ldg(vv + j))); };
	auto shf = [&](long long j) { return mul(sf(j), im(j)); };
	double v[2] = {0.0, 0.0};
	const Sweep w = sweep(g, zc);
	if (s_exit) {
		visit(g, w, [&](long long i) { x[i] = add(x[i], mul(alpha, mul(__ldg(p + i), im(i)))); });  // :196
	} else {
		march(g, k, w, shf, [&](long long i, double shi, double ti) {
			const double phi = mul(__ldg(p + i), im(i));                          // p_hat
			x[i] = add(add(x[i], mul(alpha, phi)), mul(omega, shi));  // :216
			const double ri = add(sf(i), mul(-omega, ti));            // :219
			rn[i] = ri;
			v[0] = fma(ri, ri, v[0]);
			v[1] = fma(ri, __ldg(rhat + i), v[1]);
		});
	}
	double out[2];
	if (grid_sum<2>(v, partials, ticket, out) && threadIdx.x == 0) {
		if (s_exit) {
			st->done = 1;
			st->exit_iter = it;
			st->reason = STOP_SNORM;
		} else {
			st->wsel = sel ^ 1;
			st->rr = out[0];
			const double err = sqrt(__ddiv_rn(out[0], st->bb));  // :226
			st->err = err;
			hist[it] = err;
			if (err <= st->tol) {                                  // :228
				st->done = 1;
				st->exit_iter = it;
				st->reason = STOP_CONVERGED;
			} else if (omega == 0.0) {                             // :229
				st->done = 1;
				st->exit_iter = it;
				st->reason = STOP_OMEGA;
			} else {
				st->rho_prev = st->rho;                             // :231
				if (it >= st->maxiter) {
					st->done = 1;
					st->exit_iter = st->maxiter + 1;
					st->reason = STOP_MAXITER;
				} else {
					st->rho = out[1];                                // next iteration :159-160
					if (out[1] == 0.0) {                             // :162
						st->done = 1;
						st->exit_iter = it + 1;
						st->reason = STOP_RHO;
					}
				}
			}
		}
		st->iter = it + 1;
	}
}

// ---------------------------------------------------------------------------
// Utility kernels: y = A x, accumulators (SliceOps::accumulate_product,
// SliceOps.hpp:96-108), D = t ./ q (SliceOps::divide, :68-79).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_stencil(Geo g, Coef k, int zc, const double *__restrict__ x,
                                                      double *__restrict__ y) {
	march(g, k, sweep(g, zc), [&](long long j) { return __ldg(x + j); },
	      [&](long long i, double, double yi) { y[i] = yi; });
}

__global__ void __launch_bounds__(kThreads) k_accumulate(long long n, const double *__restrict__ x,
                                                         const double *__restrict__ v, double *__restrict__ t,
                                                         double *__restrict__ q, int reset) {
	for (long long i = gstart(); i < n; i += gstride()) {
		const double vi = __ldg(v + i);
		const double t0 = reset ? 0.0 : t[i];
		const double q0 = reset ? 0.0 : q[i];
		t[i] = add(t0, mul(__ldg(x + i), vi));
		q[i] = add(q0, mul(vi, vi));
	}
}

__global__ void __launch_bounds__(kThreads) k_divide(long long n, const double *__restrict__ t,
                                                     const double *__restrict__ q, double *__restrict__ D) {
	for (long long i = gstart(); i < n; i += gstride()) D[i] = __ddiv_rn(__ldg(t + i), __ldg(q + i));
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
#define SEDI_TRY(expr)                                                        \
	do {                                                                      \
		cudaError_t e_ = (expr);                                              \
		if (e_ != cudaSuccess) return set_cuda_error(c, e_, #expr);           \
	} while (0)

static int blocks_for(long long n) {
	long long b = (n + kThreads - 1) / kThreads;
	if (b > 148LL * 8) b = 148LL * 8;
	if (b < 1) b = 1;
	return (int)b;
}

int plain_alloc(Ctx *c) {
	const size_t bytes = sizeof(double) * (size_t)c->g.n;
	c->nblocks = blocks_for(c->g.n);
	double **vecs[] = {&c->x, &c->b, &c->iM, &c->r, &c->rhat, &c->p[0], &c->p[1], &c->v[0], &c->v[1],
	                   &c->w[0], &c->w[1], &c->u, &c->q, &c->s, &c->z, &c->t_acc, &c->q_acc};
	for (double **pp : vecs) {
		if (cudaMalloc(pp, bytes) != cudaSuccess) {
			cudaGetLastError();
			c->error = "device allocation failed";
			return SEDI_ERR_NOMEM;
		}
	}
	const Launch l = launch_shape(c->g);
	const size_t sweep_blocks = (size_t)l.grid.x * l.grid.y * l.grid.z;
	SEDI_TRY(cudaMalloc(&c->partials, sizeof(double) * kMaxDots * (sweep_blocks > (size_t)c->nblocks ? sweep_blocks : (size_t)c->nblocks)));
	SEDI_TRY(cudaMalloc(&c->ticket, sizeof(unsigned)));
	SEDI_TRY(cudaMemsetAsync(c->ticket, 0, sizeof(unsigned), c->stream));  // ordered before the context's kernels
	SEDI_TRY(cudaStreamSynchronize(c->stream));
	SEDI_TRY(cudaMalloc(&c->st, sizeof(SolveState)));
	SEDI_TRY(cudaMallocHost(&c->st_host, sizeof(SolveState)));
	c->hist_cap = 0;
	c->hist = nullptr;
	c->chunk_iters = 16;
	return pairs_alloc(c);
}

void plain_free(Ctx *c) {
	pairs_free(c);
	double *vecs[] = {c->x, c->b, c->iM, c->r, c->rhat, c->p[0], c->p[1], c->v[0], c->v[1],
	                  c->w[0], c->w[1], c->u, c->q, c->s, c->z, c->t_acc, c->q_acc, c->partials, c->hist};
	for (double *p : vecs)
		if (p) cudaFree(p);
	if (c->ticket) cudaFree(c->ticket);
	if (c->st) cudaFree(c->st);
	if (c->st_host) cudaFreeHost(c->st_host);
	for (int i = 0; i < 2; i++)
		if (c->chunk_graph[i]) cudaGraphExecDestroy(c->chunk_graph[i]);
}

// Enqueue one iteration of the context's solver (kernels early-exit once done).
template <bool VIM>
static void enqueue_iteration(Ctx *c, IMv<VIM> im) {
	const Launch l = launch_shape(c->g);
	const dim3 nb = l.grid;
	const int zc = l.zc;
	cudaStream_t s = c->stream;
	if (c->solver == 2) {
		k_cg_a<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->r, c->p[0], c->p[1], c->partials, c->ticket, c->st);
		k_cg_b<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->x, c->r, c->p[0], c->p[1], c->partials, c->ticket,
		                                     c->st, c->hist);
		c->launches += 2;
	} else if (c->solver == 3) {
		k_pcg_iter<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->x, c->r, c->u, c->w[0], c->w[1], c->q, c->s,
		                                         c->p[0], c->z, c->partials, c->ticket, c->st, c->hist);
		c->launches += 1;
	} else {
		// BiCGStab keeps r in r (sel 0) / p[1]-free buffer pair: r0 = c->r, r1 = c->u.
		k_bicg_1<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->r, c->u, c->rhat, c->p[0], c->p[1], c->v[0],
		                                       c->v[1], c->partials, c->ticket, c->st);
		k_bicg_2<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->r, c->u, c->v[0], c->v[1], c->partials,
		                                       c->ticket, c->st);
		k_bicg_3<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->x, c->r, c->u, c->rhat, c->p[0], c->p[1],
		                                       c->v[0], c->v[1], c->partials, c->ticket, c->st, c->hist);
		c->launches += 3;
	}
}

static int kernels_per_iteration(const Ctx *c) { return c->solver == 2 ? 2 : (c->solver == 3 ? 1 : 3); }

template <bool VIM>
static int run_chunk(Ctx *c, IMv<VIM> im) {
	cudaGraphExec_t &ge = c->chunk_graph[VIM ? 1 : 0];
	if (!ge) {
		cudaGraph_t graph;
		const long long before = c->launches;
		SEDI_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
		for (int i = 0; i < c->chunk_iters; i++) enqueue_iteration<VIM>(c, im);
		SEDI_TRY(cudaStreamEndCapture(c->stream, &graph));
		c->launches = before;
		cudaError_t e = cudaGraphInstantiate(&ge, graph, 0);
		cudaGraphDestroy(graph);
		if (e != cudaSuccess) {
			ge = nullptr;
			return set_cuda_error(c, e, "cudaGraphInstantiate");
		}
	}
	SEDI_TRY(cudaGraphLaunch(ge, c->stream));
	c->launches += (long long)c->chunk_iters * kernels_per_iteration(c);
	return 0;
}

static int ensure_hist(Ctx *c, int maxiter) {
	if (c->hist && c->hist_cap >= maxiter + 1) return 0;
	int cap = maxiter + 1 < 1024 ? 1024 : maxiter + 1;
	if (c->hist) cudaFree(c->hist);
	c->hist = nullptr;
	SEDI_TRY(cudaMalloc(&c->hist, sizeof(double) * (size_t)cap));
	c->hist_cap = cap;
	// Graphs captured the old history pointer.
	for (int i = 0; i < 2; i++)
		if (c->chunk_graph[i]) {
			cudaGraphExecDestroy(c->chunk_graph[i]);
			c->chunk_graph[i] = nullptr;
		}
	return 0;
}

// Reference post-loop logic: Cg.hpp:197-206, PipelinedCg.hpp:233-242,
// BiCgStab.hpp:235-262.
static int finish_result(const Ctx *c, const SolveState &s, double *final_err, int *final_iter) {
	if (s.reason == STOP_EARLY) {
		*final_iter = 0;
		*final_err = s.err;
		return 0;
	}
	const int iter = s.exit_iter;
	if (s.err <= s.tol) {
		*final_iter = iter;
		*final_err = s.err;
		return 0;
	}
	if (c->solver == 1) {
		if (s.s_norm2 <= s.tol * s.tol) {
			*final_iter = iter;
			*final_err = std::sqrt(s.s_norm2 / s.bb);
			return 0;
		}
		if (s.omega == 0.0) {
			*final_iter = iter;
			*final_err = s.err;
			return 3;
		}
		if (s.rho == 0.0) {
			*final_iter = iter;
			*final_err = s.err;
			return 2;
		}
	}
	*final_iter = s.maxiter;
	*final_err = s.err;
	return 1;
}

template <bool VIM>
static int solve_impl(Ctx *c, IMv<VIM> im, int maxiter, double tol, double *final_err, int *final_iter) {
	const Launch l = launch_shape(c->g);
	const dim3 nb = l.grid;
	const int zc = l.zc;
	cudaStream_t s = c->stream;
	int rc = ensure_hist(c, maxiter);
	if (rc) return rc;
	k_setup<<<nb, kThreads, 0, s>>>(c->g, c->k, zc, c->x, c->b, c->r, c->solver == 1 ? c->rhat : nullptr,
	                                c->partials, c->ticket, c->st, c->hist, tol, maxiter, c->solver);
	c->launches++;
	if (c->solver == 3) {
		k_pcg_setup<VIM><<<nb, kThreads, 0, s>>>(c->g, c->k, zc, im, c->r, c->u, c->w[0], c->z, c->q, c->s, c->p[0],
		                                          c->partials, c->ticket, c->st);
		c->launches++;
	}
	SEDI_TRY(cudaGetLastError());
	// Replay chunks of iterations until the device reports the loop left.
	int launched = 0;
	for (;;) {
		rc = run_chunk<VIM>(c, im);
		if (rc) return rc;
		launched += c->chunk_iters;
		SEDI_TRY(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
		SEDI_TRY(cudaStreamSynchronize(s));
		if (c->st_host->done) break;
		if (launched > maxiter + c->chunk_iters) {
			c->error = "solver state machine did not stop";
			return SEDI_ERR_CUDA;
		}
	}
	const SolveState st = *c->st_host;
	// Entries written: hist[0] plus one per iteration that printed its err
	// (the s-norm exit and the rho breakdown leave before printing).
	if (st.reason == STOP_EARLY) c->hist_len = 1;
	else if (st.reason == STOP_SNORM || st.reason == STOP_RHO) c->hist_len = st.exit_iter;
	else c->hist_len = (st.exit_iter > maxiter ? maxiter : st.exit_iter) + 1;
	return finish_result(c, st, final_err, final_iter);
}

// Solve with b, x (and iM when vim) already in the context's buffers.
int plain_solve_resident(Ctx *c, bool vim, int maxiter, double tol, double *final_err, int *final_iter) {
	if (!vim && c->pairs) {  // n1 even, constant iM: the streaming sweeps
		const int rc = ensure_hist(c, maxiter);
		if (rc) return rc;
		return pairs_solve_resident(c, maxiter, tol, final_err, final_iter);
	}
	if (vim) {
		IMv<true> im{c->iM, 0.0};
		return solve_impl<true>(c, im, maxiter, tol, final_err, final_iter);
	}
	IMv<false> im{nullptr, 1.0 / c->k.a};  // stochastic-estimator.cc:103
	return solve_impl<false>(c, im, maxiter, tol, final_err, final_iter);
}

int plain_solve_dev(Ctx *c, const double *b, double *x, const double *iM, int maxiter, double tol,
                    double *final_err, int *final_iter) {
	const size_t bytes = sizeof(double) * (size_t)c->g.n;
	cudaStream_t s = c->stream;
	SEDI_TRY(cudaMemcpyAsync(c->b, b, bytes, cudaMemcpyDeviceToDevice, s));
	SEDI_TRY(cudaMemcpyAsync(c->x, x, bytes, cudaMemcpyDeviceToDevice, s));
	if (iM) SEDI_TRY(cudaMemcpyAsync(c->iM, iM, bytes, cudaMemcpyDeviceToDevice, s));
	const int rc = plain_solve_resident(c, iM != nullptr, maxiter, tol, final_err, final_iter);
	if (rc < 0) return rc;
	SEDI_TRY(cudaMemcpyAsync(x, c->x, bytes, cudaMemcpyDeviceToDevice, s));
	SEDI_TRY(cudaStreamSynchronize(s));
	return rc;
}

int plain_stencil(Ctx *c, const double *x_dev, double *y_dev) {
	const Launch l = launch_shape(c->g);
	k_stencil<<<l.grid, kThreads, 0, c->stream>>>(c->g, c->k, l.zc, x_dev, y_dev);
	c->launches++;
	SEDI_TRY(cudaGetLastError());
	return 0;
}

int plain_accumulate(Ctx *c, const double *x_dev, const double *v_dev, int reset) {
	k_accumulate<<<c->nblocks, kThreads, 0, c->stream>>>(c->g.n, x_dev, v_dev, c->t_acc, c->q_acc, reset);
	c->launches++;
	SEDI_TRY(cudaGetLastError());
	return 0;
}

int plain_divide(Ctx *c, double *D_dev) {
	k_divide<<<c->nblocks, kThreads, 0, c->stream>>>(c->g.n, c->t_acc, c->q_acc, D_dev);
	c->launches++;
	SEDI_TRY(cudaGetLastError());
	return 0;
}

int plain_history(Ctx *c, double *out, int len) {
	int n = c->hist_len < len ? c->hist_len : len;
	if (n <= 0 || !c->hist) return 0;
	SEDI_TRY(cudaMemcpyAsync(out, c->hist, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
	SEDI_TRY(cudaStreamSynchronize(c->stream));
	return n;
}

}  // namespace sedi
