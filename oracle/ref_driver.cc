/*
 * Reference-oracle driver (test infrastructure, not product code).
 *
 * Compiled against the UNMODIFIED reference headers (include path points at
 * the reference checkout) with the single-rank MPI stand-in (shim/mpi.h),
 * the raw-file HDF5 stand-in (shim/hdf5.h) and the seeded random_device
 * pre-include (shim/seeded_rd.h).  It restates the estimator loop of
 * stochastic-estimator.cc:144-216 and, instead of printing only, writes every
 * quantity the GPU build is checked against:
 *
 *   <out>/D.f64        final D = t / q                (stochastic-estimator.cc:216)
 *   <out>/t.f64        t = sum_k x_k .* v_k           (:195)
 *   <out>/q.f64        q = sum_k v_k .* v_k           (:198)
 *   <out>/iters.i32    final_iter per probe           (:176-179)
 *   <out>/errs.f64     final_err per probe
 *   <out>/results.i32  solver result_t per probe
 *   <out>/v.f64, x.f64 per-probe RHS and solution     (with -x)
 *   <out>/time.txt     wall seconds of the probe loop (:152-212)
 *
 * All grids are written dense, i1 fastest, then i2, then i3 (the element
 * order of Grid3d::rank_cells, Slice3d.hpp:30-32).
 *
 * usage: ref_driver -g N1xN2xN3 -S {1,2,3} [-s samples] [-e tol] [-m maxiter]
 *                   [-a A,B,C] [-f mode] [-x] [-q] [-o outdir]
 *   -S  1 BiCgStab, 2 Cg, 3 PipelinedCg (the reference's -DSOLVER values)
 *   -a  stencil coefficients (reference default 6,1,1; stochastic-estimator.cc:74)
 *   -f  solver mode bits (Cg.hpp:36-40); 1 = synchronous stencil, which applies
 *       the stencil to the whole grid in one call (DistrAsyncStencil.hpp:87-97)
 *   -q  send the solvers' per-iteration printf lines to /dev/null
 */
#include <mpi.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <sys/stat.h>

#include "Types.hpp"
#include "DomainDecomposition.hpp"
#include "Grid3d.hpp"
#include "SliceOps.hpp"
#include "CommHalo.hpp"
#include "Stencil.hpp"
#include "DistrAsyncStencil.hpp"
#include "PipelinedCg.hpp"
#include "Cg.hpp"
#include "BiCgStab.hpp"
#include "DistrRngStd.hpp"
#include "Timers.hpp"

static void dump(const std::string &path, const void *p, size_t bytes) {
	FILE *f = fopen(path.c_str(), "wb");
	if (!f || fwrite(p, 1, bytes, f) != bytes) {
		fprintf(stderr, "ref_driver: cannot write %s\n", path.c_str());
		exit(3);
	}
	fclose(f);
}

static void to_dense(const Slice3d<real_t> &s, real_t *out) {
	long i = 0;
	for (long i3 = 0; i3 < s.n3; i3++)
		for (long i2 = 0; i2 < s.n2; i2++)
			for (long i1 = 0; i1 < s.n1; i1++) out[i++] = s.element_ref(i1, i2, i3);
}

struct Opts {
	long n1, n2, n3;
	int solver, samples, maxiter, mode;
	double tol, a, b, c;
	bool dump_vx, quiet;
	std::string out;
};

template <class solver_t>
static int run(const Opts &o) {
	Timers timers;
	Stencil<real_t> stencil(o.a, o.b, o.c);
	const long nghost = 1, ninner = nghost;
	DomainDecomposition dd(o.n1, o.n2, o.n3, 1, 1, 1);
	CommHalo<real_t> comm_halo(dd, nghost, &timers);
	Grid3d<real_t> x_k(dd, nghost, ninner); x_k.all_cells.fill(0.0);
	Grid3d<real_t> v_k(dd, 0, ninner); v_k.all_cells.fill(0.0);
	Grid3d<real_t> t_k(dd, 0, ninner); t_k.all_cells.fill(0.0);
	Grid3d<real_t> q_k(dd, 0, ninner); q_k.all_cells.fill(0.0);
	Grid3d<real_t> D(dd, 0, ninner); D.all_cells.fill(0.0);
	Grid3d<real_t> precond(dd, 0, ninner);
	precond.all_cells.fill(1.0 / stencil.a);
	DistrRngStd<real_t> rng(dd);
	solver_t solver(dd, nghost, o.mode, &timers);
	SliceOps<real_t> slice_ops(&timers);

	const long n = dd.ngp;
	std::vector<int> iters(o.samples), results(o.samples);
	std::vector<double> errs(o.samples);
	std::vector<real_t> vbuf, xbuf;
	if (o.dump_vx) { vbuf.resize((size_t)n * o.samples); xbuf.resize((size_t)n * o.samples); }

	double t0 = MPI_Wtime();
	for (int k = 0; k < o.samples; k++) {
		rng.fill_plusminusone(v_k.rank_cells);
		x_k.all_cells.fill(0.0);
		int final_iter = -1;
		real_t final_err = 0;
		int res = (int)solver.solve(stencil, comm_halo, x_k, v_k, precond, o.maxiter, o.tol, &final_err, &final_iter);
		iters[k] = final_iter;
		errs[k] = final_err;
		results[k] = res;
		if (o.dump_vx) {
			to_dense(v_k.rank_cells, &vbuf[(size_t)n * k]);
			to_dense(x_k.rank_cells, &xbuf[(size_t)n * k]);
		}
		slice_ops.accumulate_product(x_k.rank_cells, v_k.rank_cells, t_k.rank_cells);
		slice_ops.accumulate_product(v_k.rank_cells, v_k.rank_cells, q_k.rank_cells);
	}
	double t1 = MPI_Wtime();
	slice_ops.divide(t_k.rank_cells, q_k.rank_cells, D.rank_cells);

	std::vector<real_t> dense(n);
	to_dense(D.rank_cells, dense.data()); dump(o.out + "/D.f64", dense.data(), n * sizeof(real_t));
	to_dense(t_k.rank_cells, dense.data()); dump(o.out + "/t.f64", dense.data(), n * sizeof(real_t));
	to_dense(q_k.rank_cells, dense.data()); dump(o.out + "/q.f64", dense.data(), n * sizeof(real_t));
	dump(o.out + "/iters.i32", iters.data(), iters.size() * sizeof(int));
	dump(o.out + "/errs.f64", errs.data(), errs.size() * sizeof(double));
	dump(o.out + "/results.i32", results.data(), results.size() * sizeof(int));
	if (o.dump_vx) {
		dump(o.out + "/v.f64", vbuf.data(), vbuf.size() * sizeof(real_t));
		dump(o.out + "/x.f64", xbuf.data(), xbuf.size() * sizeof(real_t));
	}
	FILE *f = fopen((o.out + "/time.txt").c_str(), "w");
	if (f) { fprintf(f, "%.9e\n", t1 - t0); fclose(f); }
	return 0;
}

int main(int argc, char **argv) {
	MPI_Init(&argc, &argv);
	Opts o;
	o.n1 = o.n2 = o.n3 = 0;
	o.solver = 2; o.samples = 1; o.maxiter = 1000; o.mode = 0;
	o.tol = 1e-4; o.a = 6.0; o.b = 1.0; o.c = 1.0;
	o.dump_vx = false; o.quiet = false; o.out = ".";
	int ch;
	while ((ch = getopt(argc, argv, "g:S:s:e:m:a:f:xqo:")) != -1) {
		switch (ch) {
		case 'g': if (sscanf(optarg, "%ldx%ldx%ld", &o.n1, &o.n2, &o.n3) != 3) return 1; break;
		case 'S': o.solver = atoi(optarg); break;
		case 's': o.samples = atoi(optarg); break;
		case 'e': o.tol = atof(optarg); break;
		case 'm': o.maxiter = atoi(optarg); break;
		case 'a': if (sscanf(optarg, "%lf,%lf,%lf", &o.a, &o.b, &o.c) != 3) return 1; break;
		case 'f': o.mode = atoi(optarg); break;
		case 'x': o.dump_vx = true; break;
		case 'q': o.quiet = true; break;
		case 'o': o.out = optarg; break;
		default: fprintf(stderr, "bad option\n"); return 1;
		}
	}
	if (o.n1 <= 0 || o.n2 <= 0 || o.n3 <= 0) { fprintf(stderr, "need -g N1xN2xN3\n"); return 1; }
	mkdir(o.out.c_str(), 0755);
	if (o.quiet && !freopen("/dev/null", "w", stdout)) return 1;
	int rc;
	if (o.solver == 1) rc = run<BiCgStab<real_t> >(o);
	else if (o.solver == 2) rc = run<Cg<real_t> >(o);
	else if (o.solver == 3) rc = run<PipelinedCg<real_t> >(o);
	else { fprintf(stderr, "-S must be 1, 2 or 3\n"); rc = 1; }
	MPI_Finalize();
	return rc;
}
