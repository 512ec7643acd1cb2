/*
 * SEDI CPU oracle: a plain-C restatement of the reference estimator hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against; only tests/, the smoke check and the benchmark's CPU
 * baseline load it.  The product library never links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * golden vectors produced by the reference sources themselves (compiled with
 * single-rank MPI / raw-HDF5 / seeded-random_device stand-ins, see
 * oracle/ref_driver.cc), committed under tests/golden/.
 *
 * Layout: every grid is dense n1*n2*n3 doubles, i1 fastest, then i2, then i3
 * (the element order of Grid3d::rank_cells, Slice3d.hpp:30-32).  Points
 * outside the grid read as 0.0 (zero ghost layer, Cg.hpp:57-62).
 */
#ifndef SEDI_ORACLE_H
#define SEDI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* DistrRngStd::fill_plusminusone with std::mt19937(seed) (DistrRngStd.hpp:22-42). */
void so_fill_probe(uint32_t seed, long n, double *out);

/* Stencil::apply_direct (Stencil.hpp:38-54) with zero ghosts. */
void so_stencil(long n1, long n2, long n3, double a, double b, double c, const double *x, double *y);

/* Sequential-order dot product (SliceOps.hpp:111-125). */
double so_dot(long n, const double *u, const double *v);

/*
 * Solvers.  x: in initial guess, out solution.  iM: inverse-diagonal vector
 * (NULL means the constant 1/a of stochastic-estimator.cc:103).  err_hist,
 * when not NULL, receives err after each iteration (maxiter+1 slots; slot 0
 * holds the initial relative residual).  Return value = reference result_t.
 */
int so_cg(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
          const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist);
int so_pcg(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
           const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist);
int so_bicgstab(long n1, long n2, long n3, double a, double b, double c, double *x, const double *rhs,
                const double *iM, int maxiter, double tol, double *final_err, int *final_iter, double *err_hist);

/*
 * Estimator loop (stochastic-estimator.cc:158-216): probe k uses
 * std::mt19937(seed + k).  solver: 1 BiCgStab, 2 Cg, 3 PipelinedCg.
 * t, q, D: n doubles each (may be NULL except D).  iters/errs/results:
 * per probe (may be NULL).  x_out, v_out: samples*n doubles (may be NULL).
 */
int so_estimate(int solver, long n1, long n2, long n3, double a, double b, double c, int samples,
                uint32_t seed, int maxiter, double tol, double *D, double *t, double *q, int *iters,
                double *errs, int *results, double *x_out, double *v_out);

#ifdef __cplusplus
}
#endif

#endif
