/*
 * SEDI CPU oracle -- plain-C restatement of the reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): loaded by
 * tests/, the smoke check and the benchmark's CPU-baseline leg.
 *
 * Each function cites the reference lines it restates.  Arithmetic follows
 * the reference operator by operator, compiled with -ffp-contract=off so
 * every `*` and `+` rounds once, as in the oracle build of the reference.
 * The only intended difference from the reference is the summation order of
 * dot products: the reference sums with `omp simd` lanes and L3 cache
 * blocks (SliceOps.hpp:117, DistrAsyncDotProds.hpp:73-98), this file sums
 * sequentially.  Pinned against the reference's own outputs in
 * tests/test_oracle.py.
 */
#include "sedi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------- */
/* Probe generator.                                                        */
/* ---------------------------------------------------------------------- */

/*
 * MT19937 (Matsumoto & Nishimura 1998, ACM TOMACS 8(1)), the engine the
 * reference uses through std::mt19937 (DistrRngStd.hpp:28).  Parameters are
 * the published ones: n=624, m=397, matrix a=0x9908b0df, tempering
 * (u,d)=(11,0xffffffff) (s,b)=(7,0x9d2c5680) (t,c)=(15,0xefc60000) l=18,
 * initialisation multiplier f=1812433253.
 */
typedef struct { uint32_t mt[624]; int idx; } mt19937_t;

static void mt_seed(mt19937_t *g, uint32_t seed) {
	g->mt[0] = seed;
	for (int i = 1; i < 624; i++) g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
	g->idx = 624;
}

static uint32_t mt_next(mt19937_t *g) {
	if (g->idx >= 624) {
		for (int i = 0; i < 624; i++) {
			uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
			g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		}
		g->idx = 0;
	}
	uint32_t y = g->mt[g->idx++];
	y ^= y >> 11;
	y ^= (y << 7) & 0x9d2c5680u;
	y ^= (y << 15) & 0xefc60000u;
	y ^= y >> 18;
	return y;
}

/*
 * std::uniform_real_distribution<double>(0,1) over a 32-bit engine is
 * generate_canonical<double,53>: two draws g1, g2 combined as
 * (g1 + g2 * 2^32) / 2^64 in double arithmetic (the first product and the
 * final scaling are exact, the sum rounds once), clamped below 1.
 * DistrRngStd.hpp:32-40 then maps x > 0.5 to +1 and everything else to -1,
 * visiting i1 fastest, then i2, then i3.
 */
void so_fill_probe(uint32_t seed, long n, double *out) {
	mt19937_t g;
	mt_seed(&g, seed);
	for (long i = 0; i < n; i++) {
		double sum = (double)mt_next(&g);
		sum += (double)mt_next(&g) * 4294967296.0;
		double x = sum / 18446744073709551616.0;
		if (x >= 1.0) x = nextafter(1.0, 0.0);
		x = x * (1.0 - 0.0) + 0.0;
		out[i] = (x > 0.5) ? 1.0 : -1.0;
	}
}

/* ---------------------------------------------------------------------- */
/* Local kernels.                                                          */
/* ---------------------------------------------------------------------- */

/*
 * Stencil::apply_direct (Stencil.hpp:38-54): the seven terms in the same
 * order, left to right; ghost reads (outside the grid) are the value 0.0.
 */
void so_stencil(long n1, long n2, long n3, double a, double b, double c, const double *x, double *y) {
	const long s2 = n1, s3 = n1 * n2;
	for (long i3 = 0; i3 < n3; i3++)
		for (long i2 = 0; i2 < n2; i2++)
			for (long i1 = 0; i1 < n1; i1++) {
				const long i = i1 + i2 * s2 + i3 * s3;
				const double xc = x[i];
				const double xm1 = i1 > 0 ? x[i - 1] : 0.0;
				const double xm2 = i2 > 0 ? x[i - s2] : 0.0;
				const double xm3 = i3 > 0 ? x[i - s3] : 0.0;
				const double xp1 = i1 < n1 - 1 ? x[i + 1] : 0.0;
				const double xp2 = i2 < n2 - 1 ? x[i + s2] : 0.0;
				const double xp3 = i3 < n3 - 1 ? x[i + s3] : 0.0;
				y[i] = a * xc - c * xm1 - c * xm2 - c * xm3 - b * xp1 - b * xp2 - b * xp3;
			}
}

/* SliceOps::dotprod (SliceOps.hpp:111-125), sequential order. */
double so_dot(long n, const double *u, const double *v) {
	double r = 0.0;
	for (long i = 0; i < n; i++) r += u[i] * v[i];
	return r;
}

/* SliceOps::combine2 z = a*u + b*v (SliceOps.hpp:17-32). */
static void combine2(long n, double a, const double *u, double b, const double *v, double *z) {
	for (long i = 0; i < n; i++) z[i] = a * u[i] + b * v[i];
}

/* SliceOps::combine3 z = a*u + b*v + c*w (SliceOps.hpp:35-52). */
static void combine3(long n, double a, const double *u, double b, const double *v, double c, const double *w, double *z) {
	for (long i = 0; i < n; i++) z[i] = a * u[i] + b * v[i] + c * w[i];
}

/* SliceOps::multiply z = u .* v (SliceOps.hpp:82-93); v NULL means the constant iMc. */
static void multiply(long n, const double *u, const double *v, double vc, double *z) {
	for (long i = 0; i < n; i++) z[i] = u[i] * (v ? v[i] : vc);
}

typedef struct {
	long n1, n2, n3, n;
	double a, b, c;
} grid_t;

static double *zalloc(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* ---------------------------------------------------------------------- */
/* Cg::solve (Cg.hpp:70-207).                                             */
/* ---------------------------------------------------------------------- */
int so_cg(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
          const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist) {
	const long n = n1 * n2 * n3;
	const double iMc = 1.0 / a;
	double *r = zalloc(n), *s = zalloc(n), *u = zalloc(n), *p = zalloc(n);

	double b_norm2 = so_dot(n, rhs, rhs);                   /* :112-114 */
	if (b_norm2 == 0.0) b_norm2 = 1.0;                      /* :115 */
	so_stencil(n1, n2, n3, a, b, c, x, r);                   /* :119-121 */
	combine2(n, 1.0, rhs, -1.0, r, r);                       /* :123 */
	double r_norm2 = so_dot(n, r, r);                        /* :126-129 */
	double err = sqrt(r_norm2 / b_norm2);
	if (err_hist) err_hist[0] = err;
	int ret;
	if (err < tol) {                                         /* :130-134 */
		*final_iter = 0;
		*final_err = err;
		ret = 0;
		goto done;
	}
	double alpha = 0.0, beta = 0.0, s_dot_p = 0.0, r_dot_u = 0.0, r_dot_u_new = 0.0;
	multiply(n, r, iM, iMc, u);                              /* :144 */
	memcpy(p, u, sizeof(double) * (size_t)n);                /* :147 */
	int iter;
	for (iter = 1; iter < maxiter + 1; iter++) {
		so_stencil(n1, n2, n3, a, b, c, p, s);               /* :152-154 */
		if (iter == 1) r_dot_u = so_dot(n, r, u);            /* :157-160 */
		else r_dot_u = r_dot_u_new;                          /* :161-163 */
		s_dot_p = so_dot(n, s, p);                           /* :164-165 */
		alpha = r_dot_u / s_dot_p;                           /* :166 */
		combine2(n, 1.0, x, alpha, p, x);                    /* :169 */
		combine2(n, 1.0, r, -alpha, s, r);                   /* :172 */
		multiply(n, r, iM, iMc, u);                          /* :175 */
		r_dot_u_new = so_dot(n, r, u);                       /* :179-181 */
		r_norm2 = so_dot(n, r, r);                           /* :182 */
		beta = r_dot_u_new / r_dot_u;                        /* :185 */
		combine2(n, 1.0, u, beta, p, p);                     /* :188 */
		err = sqrt(r_norm2 / b_norm2);                       /* :191 */
		if (err_hist) err_hist[iter] = err;
		if (err <= tol) break;                               /* :193 */
	}
	if (err <= tol) {                                        /* :197-201 */
		*final_iter = iter;
		*final_err = err;
		ret = 0;
	} else {                                                 /* :203-206 */
		*final_iter = maxiter;
		*final_err = err;
		ret = 1;
	}
done:
	free(r); free(s); free(u); free(p);
	return ret;
}

/* ---------------------------------------------------------------------- */
/* PipelinedCg::solve (PipelinedCg.hpp:72-244).                           */
/* ---------------------------------------------------------------------- */
int so_pcg(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
           const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist) {
	const long n = n1 * n2 * n3;
	const double iMc = 1.0 / a;
	double *r = zalloc(n), *w = zalloc(n), *nn = zalloc(n), *z = zalloc(n), *q = zalloc(n);
	double *s = zalloc(n), *p = zalloc(n), *u = zalloc(n), *m = zalloc(n);

	double b_norm2 = so_dot(n, rhs, rhs);                   /* :106-108 */
	if (b_norm2 == 0.0) b_norm2 = 1.0;                      /* :109 */
	so_stencil(n1, n2, n3, a, b, c, x, r);                   /* :113-115 */
	combine2(n, 1.0, rhs, -1.0, r, r);                       /* :117 */
	double r_norm2 = so_dot(n, r, r);                        /* :120-122 */
	double err = sqrt(r_norm2 / b_norm2);
	if (err_hist) err_hist[0] = err;
	int ret;
	if (err < tol) {                                         /* :124-128 */
		*final_iter = 0;
		*final_err = err;
		ret = 0;
		goto done;
	}
	double alpha = 0.0, beta = 0.0, gamma = 0.0, gamma_old = 0.0, delta = 0.0;
	multiply(n, r, iM, iMc, u);                              /* :138 */
	so_stencil(n1, n2, n3, a, b, c, u, w);                   /* :141-143 */
	/* z, q, s, p start at 0 (:146-149): zalloc. */
	int iter;
	for (iter = 1; iter < maxiter + 1; iter++) {
		double g = so_dot(n, r, u), d = so_dot(n, w, u), rr = so_dot(n, r, r); /* :155 */
		multiply(n, w, iM, iMc, m);                          /* :158 */
		so_stencil(n1, n2, n3, a, b, c, m, nn);              /* :161-164, :184 */
		gamma_old = gamma;                                   /* :167 */
		gamma = g;                                           /* :170-173 */
		delta = d;
		r_norm2 = rr;
		if (iter > 1) {                                      /* :175-181 */
			beta = gamma / gamma_old;
			alpha = 1.0 / (delta / gamma - beta / alpha);
		} else {
			beta = 0.0;
			alpha = gamma / delta;
		}
		combine2(n, 1.0, m, beta, q, q);                     /* :200 */
		combine2(n, 1.0, w, beta, s, s);                     /* :203 */
		combine2(n, 1.0, u, beta, p, p);                     /* :206 */
		combine2(n, 1.0, nn, beta, z, z);                    /* :209 */
		combine2(n, 1.0, r, -alpha, s, r);                   /* :212 */
		combine2(n, 1.0, x, alpha, p, x);                    /* :215 */
		combine2(n, 1.0, u, -alpha, q, u);                   /* :218 */
		combine2(n, 1.0, w, -alpha, z, w);                   /* :221 */
		err = sqrt(r_norm2 / b_norm2);                       /* :227: r_norm2 from before the r update */
		if (err_hist) err_hist[iter] = err;
		if (err <= tol) break;                               /* :229 */
	}
	if (err <= tol) {                                        /* :233-237 */
		*final_iter = iter;
		*final_err = err;
		ret = 0;
	} else {                                                 /* :239-242 */
		*final_iter = maxiter;
		*final_err = err;
		ret = 1;
	}
done:
	free(r); free(w); free(nn); free(z); free(q); free(s); free(p); free(u); free(m);
	return ret;
}

/* ---------------------------------------------------------------------- */
/* BiCgStab::solve (BiCgStab.hpp:77-264).                                 */
/* ---------------------------------------------------------------------- */
int so_bicgstab(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
                const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist) {
	const long n = n1 * n2 * n3;
	const double iMc = 1.0 / a;
	double *r = zalloc(n), *r_hat = zalloc(n), *p = zalloc(n), *s = zalloc(n), *v = zalloc(n);
	double *t = zalloc(n), *p_hat = zalloc(n), *s_hat = zalloc(n);

	double b_norm2 = so_dot(n, rhs, rhs);                   /* :123-125 */
	if (b_norm2 == 0.0) b_norm2 = 1.0;                      /* :126 */
	so_stencil(n1, n2, n3, a, b, c, x, r);                   /* :130-132 */
	combine2(n, 1.0, rhs, -1.0, r, r);                       /* :134 */
	double r_norm2 = so_dot(n, r, r);                        /* :137-139 */
	double err = sqrt(r_norm2 / b_norm2);
	if (err_hist) err_hist[0] = err;
	int ret;
	if (err < tol) {                                         /* :141-145 */
		*final_iter = 0;
		*final_err = err;
		ret = 0;
		goto done;
	}
	double omega = 1.0, alpha = 0.0, rho_prev = 0.0, rho = 0.0; /* :147-150 */
	memcpy(r_hat, r, sizeof(double) * (size_t)n);           /* :153 */
	int iter;
	double s_norm2 = 0.0;
	for (iter = 1; iter < maxiter + 1; iter++) {
		rho = so_dot(n, r, r_hat);                           /* :159-160 */
		if (rho == 0.0) break;                               /* :162 */
		double beta;
		if (iter > 1) {                                      /* :165-172 */
			beta = (rho / rho_prev) * (alpha / omega);
			combine3(n, 1.0, r, beta, p, -beta * omega, v, p);
		} else {
			memcpy(p, r, sizeof(double) * (size_t)n);
		}
		multiply(n, p, iM, iMc, p_hat);                      /* :175 */
		so_stencil(n1, n2, n3, a, b, c, p_hat, v);           /* :178-180 */
		double v_dot_rhat = so_dot(n, v, r_hat);             /* :183-185 */
		alpha = rho / v_dot_rhat;                            /* :186 */
		combine2(n, 1.0, r, -alpha, v, s);                   /* :189 */
		s_norm2 = so_dot(n, s, s);                           /* :192-193 */
		if (s_norm2 < tol * tol) {                           /* :194-198 */
			combine2(n, 1.0, x, alpha, p_hat, x);
			break;
		}
		multiply(n, s, iM, iMc, s_hat);                      /* :201 */
		so_stencil(n1, n2, n3, a, b, c, s_hat, t);           /* :204-206 */
		double ts = so_dot(n, t, s), tt = so_dot(n, t, t);   /* :209-211 */
		omega = ts / tt;                                     /* :212 */
		combine3(n, 1.0, x, alpha, p_hat, omega, s_hat, x);  /* :216 */
		combine2(n, 1.0, s, -omega, t, r);                   /* :219 */
		r_norm2 = so_dot(n, r, r);                           /* :222-223 */
		err = sqrt(r_norm2 / b_norm2);                       /* :226 */
		if (err_hist) err_hist[iter] = err;
		if (err <= tol) break;                               /* :228 */
		if (omega == 0.0) break;                             /* :229 */
		rho_prev = rho;                                      /* :231 */
	}
	if (err <= tol) {                                        /* :235-239 */
		*final_iter = iter;
		*final_err = err;
		ret = 0;
	} else if (s_norm2 <= tol * tol) {                       /* :241-245 */
		*final_iter = iter;
		*final_err = sqrt(s_norm2 / b_norm2);
		ret = 0;
	} else if (omega == 0.0) {                               /* :247-251 */
		*final_iter = iter;
		*final_err = err;
		ret = 3;
	} else if (rho == 0.0) {                                 /* :253-257 */
		*final_iter = iter;
		*final_err = err;
		ret = 2;
	} else {                                                 /* :259-262 */
		*final_iter = maxiter;
		*final_err = err;
		ret = 1;
	}
done:
	free(r); free(r_hat); free(p); free(s); free(v); free(t); free(p_hat); free(s_hat);
	return ret;
}

/* ---------------------------------------------------------------------- */
/* Estimator loop (stochastic-estimator.cc:158-216).                       */
/* ---------------------------------------------------------------------- */
int so_estimate(int solver, long n1, long n2, long n3, double a, double b, double c, int samples,
                uint32_t seed, int maxiter, double tol, double *D, double *t, double *q, int *iters,
                double *errs, int *results, double *x_out, double *v_out) {
	const long n = n1 * n2 * n3;
	double *x = zalloc(n), *v = zalloc(n), *tk = zalloc(n), *qk = zalloc(n);
	int worst = 0;
	for (int k = 0; k < samples; k++) {
		so_fill_probe(seed + (uint32_t)k, n, v);             /* :165 */
		memset(x, 0, sizeof(double) * (size_t)n);            /* :175 */
		double fe = 0.0;
		int fi = 0, res;
		if (solver == 1) res = so_bicgstab(n1, n2, n3, a, b, c, x, v, NULL, maxiter, tol, &fe, &fi, NULL);
		else if (solver == 2) res = so_cg(n1, n2, n3, a, b, c, x, v, NULL, maxiter, tol, &fe, &fi, NULL);
		else res = so_pcg(n1, n2, n3, a, b, c, x, v, NULL, maxiter, tol, &fe, &fi, NULL);
		if (iters) iters[k] = fi;
		if (errs) errs[k] = fe;
		if (results) results[k] = res;
		if (res > worst) worst = res;
		if (x_out) memcpy(x_out + (size_t)n * k, x, sizeof(double) * (size_t)n);
		if (v_out) memcpy(v_out + (size_t)n * k, v, sizeof(double) * (size_t)n);
		for (long i = 0; i < n; i++) tk[i] = tk[i] + x[i] * v[i]; /* :195 (SliceOps.hpp:96-108) */
		for (long i = 0; i < n; i++) qk[i] = qk[i] + v[i] * v[i]; /* :198 */
	}
	for (long i = 0; i < n; i++) D[i] = tk[i] / qk[i];        /* :216 (SliceOps.hpp:68-79) */
	if (t) memcpy(t, tk, sizeof(double) * (size_t)n);
	if (q) memcpy(q, qk, sizeof(double) * (size_t)n);
	free(x); free(v); free(tk); free(qk);
	return worst;
}
