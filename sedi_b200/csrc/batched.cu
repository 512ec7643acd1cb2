// Batched (RHS-interleaved) forms of the solvers on sm_100a.
//
// Layout: element (point i, right-hand side j) of every Krylov vector is at
// i*R + j -- the R right-hand sides of one grid point are contiguous.  Grid
// points are i1 fastest, then i2, i3, as in the reference's
// Grid3d::rank_cells (Slice3d.hpp:30-32).
//
// Each stencil sweep is one streaming kernel (stream.cuh): a block owns a
// point tile, a slice of lanes and a chunk of planes; planes arrive through a
// TMA/mbarrier ring in shared memory, the stencil input is computed once per
// halo point, and the epilogue fuses the pointwise updates and the dot
// products.  Every right-hand side keeps its own Krylov scalars, reduction
// results and stop state in device arrays; the last block of each reduction
// computes them for all lanes, so an iteration needs no host round trip.
// Reductions are per lane over a block -> point assignment that depends only
// on the grid and the batch width, so a batch's results do not depend on what
// else runs on the GPU.
//
// Forms:
//   FP64  (T = double): the reference method lane by lane; elementwise values
//         round exactly as the reference's (no FMA contraction), dot
//         products differ from the reference only in summation order.
//   MIXED (T = float): Krylov vectors in FP32, all reductions and scalars in
//         FP64, x kept as x_hi (FP64) + x_lo (FP32 correction since the last
//         reliable update).  A reliable update (Sleijpen & van der Vorst
//         1996; van der Vorst & Ye 2000; as used for mixed-precision GPU
//         Krylov solvers by Clark et al. 2010) folds x_lo into x_hi and
//         replaces r by the FP64 true residual b - A x_hi every `period`
//         iterations and whenever a lane's FP32 residual reaches tol; a lane
//         stops only when its FP64 true residual satisfies the reference's
//         test err = sqrt(<r,r>/<b,b>) <= tol (Cg.hpp:191-193).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "sedi_internal.h"
#include "stream.cuh"

namespace sedi {

namespace {

// ---------------------------------------------------------------------------
// Per-lane solver state (device).
// ---------------------------------------------------------------------------
struct LaneState {
	double *bb, *rr, *err, *ru, *ru_new, *sp, *alpha, *beta;  // CG
	double *gamma, *gamma_old, *delta, *rr_top;                 // pipelined CG
	double *rho, *rho_prev, *omega, *s_norm2, *ts, *tt;         // BiCGStab
	double *xa;  // CG: alpha of the x step an odd iteration leaves to the next even one
	int *done, *exit_iter, *reason, *pending, *s_exit;
	double *hist;  // single-vector form: err after each iteration (lane 0), else null
};

// Single-vector (pairs) form: lane 1 is the odd i1 points of lane 0's vector
// and carries the same scalars.
__device__ __forceinline__ void mirror_lane0(const LaneState &ls) {
	double *const d[] = {ls.bb, ls.rr, ls.err, ls.ru, ls.ru_new, ls.sp, ls.alpha, ls.beta, ls.gamma, ls.gamma_old,
	                     ls.delta, ls.rr_top, ls.rho, ls.rho_prev, ls.omega, ls.s_norm2, ls.ts, ls.tt, ls.xa};
	for (double *a : d) a[1] = a[0];
	int *const n[] = {ls.done, ls.exit_iter, ls.reason, ls.pending, ls.s_exit};
	for (int *a : n) a[1] = a[0];
}

struct Global {
	int iter;       // iteration the next launch executes
	int active;     // lanes still iterating
	int maxiter;
	int ru_due;     // a reliable update runs after this iteration
	double tol;
	int period;     // reliable-update period (mixed)
	int nrhs;
	int err;        // a bounded wait timed out
	int ru_all;     // the pending reliable update covers every lane (periodic)
	double tol_in;  // in-loop stop target: tol (FP64 form), theta * tol (mixed lanes)
	int b_iter;     // iteration of the last CG sweep A (gates the parity forms of sweep B)
	int x_pending;  // the last CG sweep B was the odd form: its x step is still pending
};

// Arithmetic: FP64 keeps the reference's operator-by-operator rounding (no
// contraction); FP32 lets the compiler fuse.
__device__ __forceinline__ double amul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double aadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double asub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float amul(float a, float b) { return a * b; }
__device__ __forceinline__ float aadd(float a, float b) { return a + b; }
__device__ __forceinline__ float asub(float a, float b) { return a - b; }

template <class T>
__device__ __forceinline__ T st7(T a, T b, T c, T xc, T xm1, T xm2, T xm3, T xp1, T xp2, T xp3) {
	T y = amul(a, xc);  // Stencil.hpp:43-50 term order
	y = asub(y, amul(c, xm1));
	y = asub(y, amul(c, xm2));
	y = asub(y, amul(c, xm3));
	y = asub(y, amul(b, xp1));
	y = asub(y, amul(b, xp2));
	y = asub(y, amul(b, xp3));
	return y;
}

// FP64 with b = c = 1 (the estimator's stencil, stochastic-estimator.cc:74):
// 1.0 * x == x exactly, so dropping those products leaves every rounding of
// st7 unchanged and halves the FP64 instructions of the stencil.
template <class T>
__device__ __forceinline__ T st7x(bool unit, T a, T b, T c, T xc, T xm1, T xm2, T xm3, T xp1, T xp2, T xp3) {
	if (sizeof(T) == 8 && unit) {
		T y = amul(a, xc);
		y = asub(y, xm1);
		y = asub(y, xm2);
		y = asub(y, xm3);
		y = asub(y, xp1);
		y = asub(y, xp2);
		y = asub(y, xp3);
		return y;
	}
	return st7<T>(a, b, c, xc, xm1, xm2, xm3, xp1, xp2, xp3);
}

template <class T>
__device__ __forceinline__ void dacc(double &acc, T a, T b) {
	acc = fma((double)a, (double)b, acc);
}

// Map slots (Maps::m) for the per-type descriptor sets.
enum {
	MT_R_HALO = 0, MT_P0_HALO, MT_P1_HALO, MT_X_INT, MT_R_INT, MT_W0_HALO, MT_W1_HALO, MT_Q_HALO,
	MT_R1_HALO, MT_V0_HALO, MT_V1_HALO, MT_P1_INT
};  // fields of type T
enum { MD_X_HALO = 0, MD_B_INT };                                     // FP64 fields

// ---------------------------------------------------------------------------
// The streaming kernel.
// Op provides: NS, NQ, ND, ka/kb/kc; enabled(gl); begin(gl, ls, lane);
// src_map(s); q_map(q); src(raw[NS]) -> stencil input; out(o, c, y, q[NQ],
// raw_c[NS], part); fin(lane, tot[ND], gl, ls).
// ---------------------------------------------------------------------------
template <class C, class Op>
__global__ void __launch_bounds__(C::THREADS, C::MINB) k_stream(SGeo g, const __grid_constant__ Maps maps, Op op,
                                                       double *partials, unsigned *ticket, Global *gl, LaneState ls) {
	typedef typename C::type E;   // storage element of the streamed fields
	typedef typename C::ctype T;  // arithmetic type
	constexpr int V = C::V, LG = C::LG, RB = C::RB, P1 = C::P1, H1 = C::H1, HALO = C::HALO, INT = C::INT,
	              NPS = C::NPS, KC = C::KC, KO = C::KO, ME = C::ME;
	constexpr int NS = Op::NS, NQ = Op::NQ, ND = Op::ND, NGX = Op::NG > 0 ? Op::NG : 1;
	constexpr bool IDENT = Op::IDENT, INPLACE = Op::INPLACE, STAGED = IDENT || INPLACE;
	typedef Layout<C, NS, NQ, ND, IDENT, INPLACE> Lay;
	constexpr int NST = Lay::NST, KEEP = Lay::KEEP;
	extern __shared__ __align__(128) unsigned char smem[];
	if (gl->active == 0 || !op.enabled(gl)) return;

	E *const stage0 = reinterpret_cast<E *>(smem);
	E *const ring = reinterpret_cast<E *>(smem + Lay::OFF_RING);
	uint64_t *const bar = reinterpret_cast<uint64_t *>(smem + Lay::OFF_BAR);
	constexpr int SE = (int)(Lay::STAGE_PAD / sizeof(E));
	constexpr int HE = (int)Lay::HALO_ELEMS, IE = (int)Lay::INT_ELEMS;

	const int t = threadIdx.x, lg = t % LG, ps = t / LG;
	const int tile = blockIdx.x;
	const int i1_0 = (tile % g.tiles1) * P1, i2_0 = (tile / g.tiles1) * C::P2;
	const int slice = blockIdx.y, lane0 = slice * RB;
	const int zoff = slice * g.n3;  // plane offset of this slice in the 4-D map
	const int z0 = blockIdx.z * g.zc, z1 = min(z0 + g.zc, g.n3);
	// Planes z0-1 .. z1 (relative index j = p - z0 + 1); none when the op has
	// no work for this lane slice (the block still joins the reduction).
	const int np = op.slice_live(gl, ls, lane0, RB) ? z1 - z0 + 2 : 0;
	const int lo = lg * V;
	op.begin(gl, ls, lane0 + lo);

	// Per-thread work, identical in every plane: halo vectors (stencil input)
	// and output points, with their shared-memory offsets and grid validity.
	int hoff[KC];
	unsigned hval = 0;
#pragma unroll
	for (int k = 0; k < KC; k++) {
		const int e = t + k * C::THREADS;
		const int h = e / LG;
		const int gi1 = i1_0 - 1 + h % H1, gi2 = i2_0 - 1 + h / H1;
		hoff[k] = e < HALO * LG ? h * RB + lo : -1;
		if (e < HALO * LG && gi1 >= 0 && gi1 < g.n1 && gi2 >= 0 && gi2 < g.n2) hval |= 1u << k;
	}
	// A thread's KO output points are KO consecutive rows of one column when
	// the tile allows it (ROWS), so inside the group a point's i2 neighbour
	// is another point's centre, already in registers.
	constexpr bool ROWS = (NPS % P1 == 0) && (KO * NPS == INT);
	int ooff[KO], qoff[KO];
	long long obase[KO];
	unsigned oval = 0, oin = 0;
#pragma unroll
	for (int k = 0; k < KO; k++) {
		const int q = ROWS ? (KO * (ps / P1) + k) * P1 + ps % P1 : ps + k * NPS;
		const int q1 = q % P1, q2 = q / P1;
		const int gi1 = i1_0 + q1, gi2 = i2_0 + q2;
		ooff[k] = ((q2 + 1) * H1 + (q1 + 1)) * RB + lo;
		qoff[k] = q * RB + lo;
		obase[k] = (long long)gi2 * g.n1 + gi1;
		if (q < INT) oin |= 1u << k;
		if (q < INT && gi1 < g.n1 && gi2 < g.n2) oval |= 1u << k;
	}
	// Column centres of the stencil input at planes m-1, m, m+1 of the current
	// output plane m: two of them were read one step earlier (the planes stay
	// in the ring or the stages until then), so each step reads one new centre.
	Vec<T> zprev[KO], zcur[KO], znext[KO];
	const long long plane = (long long)g.n1 * g.n2;
	const bool unit = op.kb == T(1) && op.kc == T(1);

	if (t == 0) {
		for (int s = 0; s < NST; s++) mbar_init(&bar[s], 1);
		mbar_init_fence();
	}
	__syncthreads();

	auto issue = [&](int j) {  // thread 0
		const int p = z0 - 1 + j;
		uint64_t *b = &bar[j % NST];
		E *st = stage0 + (j % NST) * SE;
		if (p < 0 || p >= g.n3) {
			mbar_arrive(b);  // ghost plane: completes the phase without data
			return;
		}
		// Stages are only read by the generic proxy during the sweep (the
		// reduction scratch that aliases them is written after the last wait),
		// so no proxy fence is needed before the copy.
		mbar_arrive_tx(b, Lay::TX);
#pragma unroll
		for (int s = 0; s < NS; s++)
			tma_load3(st + s * HE, &maps.m[op.src_map(s)], b, (i1_0 - 1) * ME, i2_0 - 1, zoff + p);
#pragma unroll
		for (int q = 0; q < NQ; q++) tma_load3(st + NS * HE + q * IE, &maps.m[op.q_map(q)], b, i1_0 * ME, i2_0, zoff + p);
		// The same tiles pfd planes further on, into L2 (within this block's planes).
		const int pf = p + g.pfd;
		if (g.pfd > 0 && pf <= z1 && pf < g.n3) {
#pragma unroll
			for (int s = 0; s < NS; s++) tma_prefetch3(&maps.m[op.src_map(s)], (i1_0 - 1) * ME, i2_0 - 1, zoff + pf);
#pragma unroll
			for (int q = 0; q < NQ; q++) tma_prefetch3(&maps.m[op.q_map(q)], i1_0 * ME, i2_0, zoff + pf);
		}
	};
	int issued = 0;
	if (t == 0)
		for (; issued < NST && issued < np; issued++) issue(issued);

	constexpr int NDX = ND > 0 ? ND : 1;
	double part[NDX][V];
#pragma unroll
	for (int d = 0; d < NDX; d++)
#pragma unroll
		for (int e = 0; e < V; e++) part[d][e] = 0.0;

	bool failed = false;
	int waited = 0;  // planes whose stage has arrived
	int sj = 0;      // stage slot of plane j (j mod NST)
	unsigned par = 0;  // barrier parity of plane j ((j / NST) & 1)
	for (int j = 0; j <= np; j++, sj = (sj + 1 == NST) ? 0 : sj + 1, par ^= (sj == 0)) {
		// Each thread waits for plane j's stage itself (the mbarrier's acquire
		// makes the TMA data visible); a timeout is combined into the one
		// block barrier at the end of the step.
		bool ok = true;
		if (j < np) ok = mbar_wait(&bar[sj], par);
		// Pointwise fields an op reads with plain loads (Op::NG of them): issue
		// the loads for this step's outputs (plane j-2) before the halo
		// transform, so they are in flight during it.
		Vec<T> gv[KO][NGX];
		if (Op::NG > 0 && j >= 3) {
			const long long zb = (long long)(z0 - 1 + j - 2) * plane;
#pragma unroll
			for (int k = 0; k < KO; k++)
				if (oval >> k & 1u) op.gload(((long long)slice * g.npts + zb + obase[k]) * RB + lo, gv[k]);
		}
		// Phase 1: stencil input of plane j (transforming ops only).
		if (!IDENT && j < np) {
			const int p = z0 - 1 + j;
			E *const st = stage0 + sj * SE;
			// In place: over the source field INPLACE_SLOT of this plane's stage
			// (each thread rewrites only the points it read).
			E *cr = INPLACE ? st + Op::INPLACE_SLOT * HE : ring + (j & 3) * HE;
			const bool pin = p >= 0 && p < g.n3;
#pragma unroll
			for (int k = 0; k < KC; k++) {
				if (hoff[k] < 0) continue;
				Vec<T> cv;
				if (pin && (hval >> k & 1u)) {
					Vec<T> raw[NS];
#pragma unroll
					for (int s = 0; s < NS; s++) raw[s] = lds(st + s * HE + hoff[k]);
					cv = op.src(raw);
				} else {
					cv = vzero<T>();  // zero ghost layer
				}
				sts(cr + hoff[k], cv);
			}
			// The stage is refilled by TMA later: order these generic writes
			// before those async-proxy writes.
			if (INPLACE) fence_async_smem();
		}
		// Phase 2: outputs of plane m = j-2 from planes m-1, m, m+1.
		if (j >= 3) {
			const int m = j - 2;
			const int z = z0 - 1 + m;
			// Stage slots of planes m-1, m, m+1 (sj is the slot of plane j = m+2).
			const int sm1 = sj >= 3 ? sj - 3 : sj - 3 + NST;
			const int s0 = sj >= 2 ? sj - 2 : sj - 2 + NST;
			const int sp1 = sj >= 1 ? sj - 1 : sj - 1 + NST;
			const E *stz = stage0 + s0 * SE;
			const E *cm, *c0, *cp;
			bool zm = true, zp = true;  // planes m-1, m+1 inside the grid
			if (STAGED) {
				const int off = INPLACE ? Op::INPLACE_SLOT * HE : 0;
				cm = stage0 + sm1 * SE + off;
				c0 = stz + off;
				cp = stage0 + sp1 * SE + off;
				zm = z - 1 >= 0;
				zp = z + 1 < g.n3;
			} else {
				cm = ring + ((m - 1) & 3) * HE;
				c0 = ring + (m & 3) * HE;
				cp = ring + ((m + 1) & 3) * HE;
			}
#pragma unroll
			for (int k = 0; k < KO; k++) {
				if (!(oin >> k & 1u)) continue;
				if (j > 3) {  // planes m-1 and m were planes m and m+1 of the previous step
					zprev[k] = zcur[k];
					zcur[k] = znext[k];
				} else {
					zprev[k] = zm ? lds(cm + ooff[k]) : vzero<T>();
					zcur[k] = lds(c0 + ooff[k]);
				}
				znext[k] = zp ? lds(cp + ooff[k]) : vzero<T>();
			}
#pragma unroll
			for (int k = 0; k < KO; k++) {
				if (!(oval >> k & 1u)) continue;
				const int hc = ooff[k];
				const Vec<T> &xc = zcur[k];
				const Vec<T> xm1 = lds(c0 + hc - RB);
				const Vec<T> xp1 = lds(c0 + hc + RB);
				const Vec<T> xm2 = (ROWS && k > 0) ? zcur[k > 0 ? k - 1 : 0] : lds(c0 + hc - H1 * RB);
				const Vec<T> xp2 = (ROWS && k + 1 < KO) ? zcur[k + 1 < KO ? k + 1 : k] : lds(c0 + hc + H1 * RB);
				const Vec<T> &xm3 = zprev[k];
				const Vec<T> &xp3 = znext[k];
				Vec<T> y;
				if constexpr (Op::SCALED) {
					// The ring holds f and the stencil input is f .* iM: FP64
					// scales each neighbour as the reference rounds p_hat and
					// s_hat; FP32 folds iM into the coefficients.
					if constexpr (sizeof(T) == 8) {
						const T im = op.iMc;
						if (C::PAIRS) {
							const T c0 = amul(xc.v[0], im), c1 = amul(xc.v[1], im);
							y.v[0] = st7x<T>(unit, op.ka, op.kb, op.kc, c0, amul(xm1.v[1], im), amul(xm2.v[0], im),
							                amul(xm3.v[0], im), c1, amul(xp2.v[0], im), amul(xp3.v[0], im));
							y.v[1] = st7x<T>(unit, op.ka, op.kb, op.kc, c1, c0, amul(xm2.v[1], im), amul(xm3.v[1], im),
							                amul(xp1.v[0], im), amul(xp2.v[1], im), amul(xp3.v[1], im));
						} else {
#pragma unroll
							for (int e = 0; e < V; e++)
								y.v[e] = st7x<T>(unit, op.ka, op.kb, op.kc, amul(xc.v[e], im), amul(xm1.v[e], im),
								                amul(xm2.v[e], im), amul(xm3.v[e], im), amul(xp1.v[e], im),
								                amul(xp2.v[e], im), amul(xp3.v[e], im));
						}
					} else {
#pragma unroll
						for (int e = 0; e < V; e++)
							y.v[e] = st7<T>(op.kas, op.kbs, op.kcs, xc.v[e], xm1.v[e], xm2.v[e], xm3.v[e], xp1.v[e],
							                xp2.v[e], xp3.v[e]);
					}
				} else if (C::PAIRS) {
					// Points 2m, 2m+1 of one vector: i1 neighbours across the pair.
					y.v[0] = st7x<T>(unit, op.ka, op.kb, op.kc, xc.v[0], xm1.v[1], xm2.v[0], xm3.v[0], xc.v[1], xp2.v[0],
					                xp3.v[0]);
					y.v[1] = st7x<T>(unit, op.ka, op.kb, op.kc, xc.v[1], xc.v[0], xm2.v[1], xm3.v[1], xp1.v[0], xp2.v[1],
					                xp3.v[1]);
				} else {
#pragma unroll
					for (int e = 0; e < V; e++)
						y.v[e] = st7x<T>(unit, op.ka, op.kb, op.kc, xc.v[e], xm1.v[e], xm2.v[e], xm3.v[e], xp1.v[e], xp2.v[e],
						                xp3.v[e]);
				}
				Vec<T> qv[NQ > 0 ? NQ : 1];
#pragma unroll
				for (int qq = 0; qq < NQ; qq++) qv[qq] = lds(stz + NS * HE + qq * IE + qoff[k]);
				Vec<T> rc[NS];
				if (Op::USES_RAW_CENTER && op.raw_center()) {
#pragma unroll
					for (int s = 0; s < NS; s++) rc[s] = lds(stz + s * HE + hc);
				}
				const long long pidx = (long long)z * plane + obase[k];
				const long long o = ((long long)slice * g.npts + pidx) * RB + lo;
				op.out(o, pidx, lane0 + lo, xc, y, qv, rc, gv[k], part);
			}
		}
		if (__syncthreads_or(!ok)) {
			failed = true;  // outputs of this step may be wrong; the host sees gl->err
			break;
		}
		if (j < np) waited = j + 1;
		// The stage of plane j-KEEP has been read for the last time.
		if (t == 0 && j >= KEEP && issued < np) {
			issue(issued);
			issued++;
		}
	}
	if (failed) {
		// Timed out: flag the error and wait (bounded) for the copies still in
		// flight.  The block still takes part in the reduction ticket below so
		// the next kernel's last-block detection stays consistent; the host
		// sees the flag and reports the solve as failed.
		if (t == 0) {
			atomicExch(&gl->err, 1);
			for (int jj = waited; jj < issued; jj++) mbar_wait(&bar[jj % NST], (unsigned)((jj / NST) & 1));
		}
		__syncthreads();
	}
	if (ND == 0) return;

	// Per-lane block reduction over point slots (scratch in the dead stages),
	// then across blocks.
	double *const red = reinterpret_cast<double *>(smem);
	const int R = g.R;
#pragma unroll
	for (int d = 0; d < NDX; d++)
#pragma unroll
		for (int e = 0; e < V; e++) red[((size_t)d * NPS + ps) * RB + lo + e] = part[d][e];
	__syncthreads();
	const unsigned pb = blockIdx.x + gridDim.x * blockIdx.z;
	const unsigned npb = gridDim.x * gridDim.z;
	for (int u = t; u < ND * RB; u += C::THREADS) {
		const int d = u / RB, l = u % RB;
		double s = 0.0;
		for (int q = 0; q < NPS; q++) s += red[((size_t)d * NPS + q) * RB + l];
		partials[((size_t)pb * ND + d) * R + lane0 + l] = s;
	}
	__shared__ bool last;
	__threadfence();
	__syncthreads();
	if (t == 0) last = (atomicAdd(ticket, 1u) == gridDim.x * gridDim.y * gridDim.z - 1);
	__syncthreads();
	if (!last) return;
	__threadfence();
	const int parts = C::THREADS / R > 0 ? C::THREADS / R : 1;
	double *acc = red;  // [parts][ND][R]
	for (int u = t; u < parts * R; u += C::THREADS) {
		const int pid = u / R, lane = u % R;
		for (int d = 0; d < ND; d++) {
			double s = 0.0;
			for (unsigned b = pid; b < npb; b += parts) s += __ldcg(&partials[((size_t)b * ND + d) * R + lane]);
			acc[((size_t)pid * ND + d) * R + lane] = s;
		}
	}
	__syncthreads();
	if (C::PAIRS) {
		// One vector: the even and odd points' sums are one dot product.
		if (t == 0) {
			double tot[NDX];
			for (int d = 0; d < ND; d++) {
				double s0 = 0.0, s1 = 0.0;
				for (int q = 0; q < parts; q++) {
					s0 += acc[((size_t)q * ND + d) * R + 0];
					s1 += acc[((size_t)q * ND + d) * R + 1];
				}
				tot[d] = s0 + s1;
			}
			op.fin(0, tot, gl, ls);
			mirror_lane0(ls);
		}
	} else {
		for (int lane = t; lane < R; lane += C::THREADS) {
			double tot[NDX];
			for (int d = 0; d < ND; d++) {
				double s = 0.0;
				for (int q = 0; q < parts; q++) s += acc[((size_t)q * ND + d) * R + lane];
				tot[d] = s;
			}
			op.fin(lane, tot, gl, ls);
		}
	}
	__syncthreads();
	if (t == 0) {
		op.after(gl);
		// The sweep that ends an iteration advances the counter unless a
		// reliable update is due (it advances it after the update).
		if (Op::ADVANCE && gl->active != 0 && gl->ru_due == 0) gl->iter += 1;
		*ticket = 0u;
	}
}

template <class T>
struct OpBase {
	static constexpr int KIND = 0;  // tile configuration (see CfgFor)
	static constexpr int NG = 0;    // pointwise fields read with plain loads, prefetched by gload
	static constexpr bool INPLACE = false;  // stencil input written over source INPLACE_SLOT (no ring)
	static constexpr int INPLACE_SLOT = 1;
	// SCALED: src() gives f and the stencil is applied to f .* iMc (the op
	// provides iMc and, for FP32, the scaled coefficients kas, kbs, kcs).
	static constexpr bool SCALED = false;
	// ADVANCE: the last block ends the iteration (gl->iter += 1 unless a
	// reliable update is due), so no kernel follows the sweep for that.
	static constexpr bool ADVANCE = false;
	T ka, kb, kc;
	__device__ void gload(long long, Vec<T> *) const {}
	__device__ bool enabled(const Global *) const { return true; }
	__device__ void after(Global *) const {}  // last block, after every lane's fin
	__device__ bool slice_live(const Global *, const LaneState &, int, int) const { return true; }
};

// ---------------------------------------------------------------------------
// Residual sweep (FP64 stream over x and b): r = b - A x (Cg.hpp:119-123).
// Setup (ru == 0): <b,b>, <r,r> per lane, initial stop test; r stored as TR,
// optional r_hat copy, MIXED: x_lo = 0.
// Reliable update (ru == 1, x = x_hi): true <r,u>, <r,r>; lanes whose true
// err <= tol stop, the others continue from the replaced residual.
// ---------------------------------------------------------------------------
template <class TR>
struct OpResid : OpBase<double> {
	static constexpr int NS = 1, NQ = 1, ND = 2;
	static constexpr bool IDENT = true, USES_RAW_CENTER = false;
	TR *r, *rhat, *xlo;  // stored in the TR layout (slice width WT)
	TR *r_alt;           // BiCGStab reliable update: r buffers by iteration parity
	double iMd;
	int solver, ru, WT;
	int pcg;  // reliable update of pipelined CG: the following sweeps rebuild its scalars
	TR *rdst;
	long long npts;
	int it;
	int keep[2], restart[2];
	__device__ bool enabled(const Global *gl) const { return !ru || gl->ru_due; }
	// A reliable update triggered by single lanes sweeps only their slices.
	__device__ bool slice_live(const Global *gl, const LaneState &ls, int lane0, int nl) const {
		if (!ru || pcg || gl->ru_all) return true;
		for (int l = lane0; l < lane0 + nl; l++)
			if (ls.pending[l]) return true;
		return false;
	}
	__device__ bool raw_center() const { return false; }
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
		for (int e = 0; e < 2; e++) {
			// Lanes outside a lane-triggered update keep their recurrence r
			// (their x_lo was not folded, so b - A x_hi is not their residual).
			keep[e] = ru ? (ls.done[lane + e] || (!pcg && !gl->ru_all && !ls.pending[lane + e])) : 0;
			restart[e] = ru && solver == 1 && !keep[e] && ls.s_exit[lane + e] == 2;
		}
		// BiCGStab: iteration it+1 reads r from R[(it+1)&1 ? 0 : 1].
		rdst = (ru && solver == 1) ? (((it + 1) & 1) ? r : r_alt) : r;
	}
	__device__ int src_map(int) const { return MD_X_HALO; }
	__device__ int q_map(int) const { return MD_B_INT; }
	__device__ Vec<double> src(const Vec<double> *raw) const { return raw[0]; }
	__device__ void out(long long, long long pidx, int lane, const Vec<double> &, const Vec<double> &ax,
	                    const Vec<double> *q, const Vec<double> *, const Vec<double> *gv, double (&part)[ND][2]) const {
		const long long ot = sliced(pidx, lane, WT, npts);  // lanes lane, lane+1 share a TR slice
#pragma unroll
		for (int e = 0; e < 2; e++) {
			const double bi = q[0].v[e];
			const double ri = aadd(bi, -ax.v[e]);  // combine2(1.0, b, -1.0, r, r)
			const TR rt = (TR)ri;
			if (!keep[e]) rdst[ot + e] = rt;
			if (xlo) xlo[ot + e] = TR(0);
			if (ru && solver == 1) {
				if (restart[e]) rhat[ot + e] = rt;
				part[0][e] = fma((double)rt, (double)(restart[e] ? rt : rhat[ot + e]), part[0][e]);  // rho = <r, r_hat>
			} else {
				if (rhat) rhat[ot + e] = rt;
				if (ru) part[0][e] = fma(ri, ri * iMd, part[0][e]);
				else part[0][e] = fma(bi, bi, part[0][e]);
			}
			part[1][e] = fma(ri, ri, part[1][e]);
		}
	}
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		// The setup keeps the reference's initial test against tol (:130-134);
		// a reliable update stops a lane on the in-loop target.
		const double tol = ru ? gl->tol_in : gl->tol;
		const int maxiter = gl->maxiter;
		if (ru) {
			if (ls.done[lane]) return;
			if (!pcg && !gl->ru_all && !ls.pending[lane]) return;  // not part of this update
			ls.xa[lane] = 0.0;  // a deferred x step was folded into x_hi
			// The FP32 recurrence's <r,r> before the replacement: when it sits
			// far below the true one (squared norms 1e-6 apart: the recurrence
			// converged in FP32 arithmetic, as small systems do exactly), its
			// search directions no longer describe the residual and the lane
			// restarts from the replaced residual.
			const double rr_rec = pcg ? ls.rr_top[lane] : ls.rr[lane];
			const bool lost = !(rr_rec >= 1e-6 * tot[1]);
			const double err = sqrt(tot[1] / ls.bb[lane]);
			ls.err[lane] = err;
			ls.rr[lane] = tot[1];
			ls.pending[lane] = 0;
			if (err <= tol) {
				ls.done[lane] = 1;
				ls.exit_iter[lane] = it;
				ls.reason[lane] = STOP_CONVERGED;
				atomicSub(&gl->active, 1);
			} else if (it >= maxiter) {
				ls.done[lane] = 1;
				ls.exit_iter[lane] = maxiter + 1;
				ls.reason[lane] = STOP_MAXITER;
				atomicSub(&gl->active, 1);
			} else if (solver == 1) {
				ls.rho[lane] = tot[0];  // continue from the replaced residual (restart keeps s_exit = 2)
				if (ls.s_exit[lane] != 2) ls.s_exit[lane] = 0;
			} else if (!pcg) {
				ls.ru_new[lane] = tot[0];  // continue from the replaced residual
				double be = tot[0] / ls.ru[lane];
				if (lost || ls.s_exit[lane] == 2 || !(be >= 0.0 && isfinite(be))) be = 0.0;  // restart: p = u
				ls.beta[lane] = be;
				ls.s_exit[lane] = 0;
			} else {
				ls.s_exit[lane] = (lost || ls.s_exit[lane] == 2) ? 2 : 0;  // pipelined CG restarts in its next sweep
			}
			return;
		}
		const double bb = tot[0] == 0.0 ? 1.0 : tot[0];  // Cg.hpp:112-115
		ls.bb[lane] = bb;
		ls.rr[lane] = tot[1];
		const double err = sqrt(__ddiv_rn(tot[1], bb));
		ls.err[lane] = err;
		if (ls.hist && lane == 0) ls.hist[0] = err;
		ls.alpha[lane] = 0.0;
		ls.beta[lane] = 0.0;
		ls.omega[lane] = 1.0;
		ls.rho[lane] = 0.0;
		ls.rho_prev[lane] = 0.0;
		ls.s_norm2[lane] = 0.0;
		ls.s_exit[lane] = 0;
		ls.pending[lane] = 0;
		ls.gamma[lane] = 0.0;
		ls.gamma_old[lane] = 0.0;
		ls.xa[lane] = 0.0;
		int done = 0, reason = STOP_NONE, ex = 0;
		if (lane >= gl->nrhs) {
			done = 1;
		} else if (err < tol) {  // :130-134
			done = 1;
			reason = STOP_EARLY;
		} else if (maxiter < 1) {
			done = 1;
			reason = STOP_MAXITER;
			ex = 1;
		} else if (solver == 1) {
			ls.rho[lane] = tot[1];
			if (tot[1] == 0.0) {
				done = 1;
				reason = STOP_RHO;
				ex = 1;
			}
		}
		ls.done[lane] = done;
		ls.reason[lane] = reason;
		ls.exit_iter[lane] = ex;
		if (!done) atomicAdd(&gl->active, 1);
	}
};

// ---------------------------------------------------------------------------
// CG kernel A: p = u + beta p (u = r .* iM; p = u on iteration 1), s = A p,
// <s,p> (and <r,u> on iteration 1); alpha = <r,u>/<s,p>  (Cg.hpp:150-166, :188).
// ---------------------------------------------------------------------------
template <class T>
struct OpCgA : OpBase<T> {
	static constexpr int KIND = 1;
	static constexpr int NS = 2, NQ = 0, ND = 2;
	static constexpr bool IDENT = false, USES_RAW_CENTER = true;
	static constexpr int V = Vec<T>::V;
	T iMc;
	T *p0, *p1;
	T *pout;  // p buffer written this iteration
	int it, mixed;
	bool first;
	T beta[V];
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
		first = (it == 1);
		pout = (it & 1) ? p1 : p0;
#pragma unroll
		for (int e = 0; e < V; e++) beta[e] = (T)ls.beta[lane + e];
	}
	__device__ bool raw_center() const { return first; }  // <r,u> is only needed on iteration 1
	__device__ int src_map(int s) const { return s == 0 ? MT_R_HALO : ((it & 1) ? MT_P0_HALO : MT_P1_HALO); }
	__device__ int q_map(int) const { return 0; }
	__device__ Vec<T> src(const Vec<T> *raw) const {
		// 1.0*u == u and (-1.0)*v == -v exactly, so the reference's
		// combine2(1.0, u, beta, p) rounds as u + round(beta*p).
		Vec<T> o;
		if (first) {
#pragma unroll
			for (int e = 0; e < V; e++) o.v[e] = amul(raw[0].v[e], iMc);
		} else {
#pragma unroll
			for (int e = 0; e < V; e++) o.v[e] = aadd(amul(raw[0].v[e], iMc), amul(beta[e], raw[1].v[e]));
		}
		return o;
	}
	__device__ void out(long long o, long long, int, const Vec<T> &pc, const Vec<T> &s, const Vec<T> *,
	                    const Vec<T> *rc, const Vec<T> *gv, double (&part)[ND][V]) const {
		stg(pout + o, pc);
#pragma unroll
		for (int e = 0; e < V; e++) dacc(part[0][e], s.v[e], pc.v[e]);
		if (first) {
#pragma unroll
			for (int e = 0; e < V; e++) dacc(part[1][e], rc[0].v[e], amul(rc[0].v[e], iMc));
		}
	}
	__device__ void after(Global *gl) const { gl->b_iter = gl->iter; }
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		if (ls.done[lane]) {
			ls.alpha[lane] = 0.0;
			return;
		}
		ls.sp[lane] = tot[0];
		const double ru = first ? tot[1] : ls.ru_new[lane];
		ls.ru[lane] = ru;
		const double al = __ddiv_rn(ru, tot[0]);
		if (mixed && !(tot[0] > 0.0 && isfinite(al))) {
			// FP32 breakdown (p = 0 once the recurrence residual is exactly
			// zero, or overflow): no step now; a reliable update replaces r
			// and the lane restarts from p = u (s_exit = 2 marks the restart).
			ls.alpha[lane] = 0.0;
			ls.pending[lane] = 1;
			ls.s_exit[lane] = 2;
			gl->ru_due = 1;
			return;
		}
		ls.alpha[lane] = al;
	}
};

// A transforming sweep with its stencil input written over source field
// SLOT in the stage instead of a ring (KIND 2: two blocks per SM on 32x16
// tiles; KIND 3: 32x32 tiles, 6 stages).  The op must not read source SLOT
// at the centre after phase 1; the values computed are those of Op.
template <class Op, int K, int SLOT = 1>
struct InPlace : Op {
	static constexpr int KIND = K;
	static constexpr bool INPLACE = true;
	static constexpr int INPLACE_SLOT = SLOT;
	InPlace() = default;
	explicit InPlace(const Op &o) : Op(o) {}
};

// CG sweep A in place: p_old (slot 1) is dead once p is formed at a point,
// and r (slot 0) stays for iteration 1's <r,u>.
template <class T, int K>
using OpCgAv = InPlace<OpCgA<T>, K>;

// ---------------------------------------------------------------------------
// CG kernel B: s = A p, x += alpha p, r -= alpha s, u = r .* iM, <r,u>, <r,r>;
// beta, err, stop test (Cg.hpp:169-193).
// XS defers x (no sweep reads x during the solve): XS_R runs on odd
// iterations and updates r alone, leaving its x step (alpha in xa) to XS_X
// on the next even iteration, which applies both in order,
// x = (x + xa p_old) + alpha p, with p_old the previous iteration's
// direction (still in the other p buffer).  In FP64 that rounds exactly as
// two reference updates (Cg.hpp:169).  Two iterations move 3 + 6 instead of
// 5 + 5 words per point and lane; r, the scalars and every iteration count
// are those of the undeferred sweep.  A pending step after an odd iteration
// is folded by the mixed form's reliable update (kb_ru_fold) and applied by
// kb_x_flush when an FP64 batch ends there.
// ---------------------------------------------------------------------------
enum { XS_EVERY = 0, XS_R = 1, XS_X = 2 };
template <class T, int XS = XS_EVERY>
struct OpCgB : OpBase<T> {
	// XS_R streams two words like sweep A and takes its 32x32 tiles (KIND 1).
	static constexpr int KIND = XS == XS_R ? 1 : 0;
	static constexpr int NS = 1, NQ = XS == XS_EVERY ? 2 : (XS == XS_R ? 1 : 3), ND = 2;
	static constexpr bool IDENT = true, USES_RAW_CENTER = false, ADVANCE = true;
	static constexpr int V = Vec<T>::V;
	T iMc;
	T *x, *r;
	int mixed;
	int it;
	T alpha[V];
	T xap[V];  // XS_X: the odd iteration's deferred alpha
	// The parity forms run once per sweep A: the one that ran advances the
	// iteration, so the other sees b_iter != iter and leaves.
	__device__ bool enabled(const Global *gl) const {
		return XS == XS_EVERY || (gl->b_iter == gl->iter && (gl->iter & 1) == (XS == XS_R ? 1 : 0));
	}
	__device__ void after(Global *gl) const {
		if (XS != XS_EVERY) gl->x_pending = XS == XS_R ? 1 : 0;
	}
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
#pragma unroll
		for (int e = 0; e < V; e++) {
			alpha[e] = (T)ls.alpha[lane + e];
			xap[e] = XS == XS_X ? (T)ls.xa[lane + e] : T(0);
		}
	}
	__device__ int src_map(int) const { return (it & 1) ? MT_P1_HALO : MT_P0_HALO; }
	__device__ int q_map(int q) const {
		if (XS == XS_R) return MT_R_INT;
		return q == 0 ? MT_X_INT : (q == 1 ? MT_R_INT : MT_P1_INT);  // XS_X: p_old of an odd iteration is P1
	}
	__device__ bool raw_center() const { return false; }
	__device__ Vec<T> src(const Vec<T> *raw) const { return raw[0]; }
	__device__ void out(long long o, long long, int, const Vec<T> &pc, const Vec<T> &s, const Vec<T> *q,
	                    const Vec<T> *, const Vec<T> *gv, double (&part)[ND][V]) const {
		Vec<T> xv, rv = q[XS == XS_R ? 0 : 1];
		if (XS != XS_R) xv = q[0];
#pragma unroll
		for (int e = 0; e < V; e++) {
			if (XS == XS_X) xv.v[e] = aadd(xv.v[e], amul(xap[e], q[2].v[e]));
			if (XS != XS_R) xv.v[e] = aadd(xv.v[e], amul(alpha[e], pc.v[e]));  // :169
			rv.v[e] = aadd(rv.v[e], amul(-alpha[e], s.v[e]));  // :172
			const T u = amul(rv.v[e], iMc);                                // :175
			dacc(part[0][e], rv.v[e], u);
			dacc(part[1][e], rv.v[e], rv.v[e]);
		}
		if (XS != XS_R) stg(x + o, xv);
		stg(r + o, rv);
	}
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		if (XS == XS_R) ls.xa[lane] = ls.alpha[lane];  // this iteration's x step, applied by the next
		if (ls.done[lane]) return;
		ls.ru_new[lane] = tot[0];
		ls.rr[lane] = tot[1];
		ls.beta[lane] = __ddiv_rn(tot[0], ls.ru[lane]);           // :185
		const double err = sqrt(__ddiv_rn(tot[1], ls.bb[lane]));  // :191
		ls.err[lane] = err;
		if (ls.hist && lane == 0) ls.hist[it] = err;              // :192
		const double tol = gl->tol_in;
		const int maxiter = gl->maxiter;
		if (mixed) {
			// The FP32 recurrence only proposes; the FP64 true residual decides.
			if (!(err == err)) ls.s_exit[lane] = 2;  // NaN recurrence: restart after the update
			if (err <= tol || it >= maxiter || !(err == err)) {
				ls.pending[lane] = 1;
				gl->ru_due = 1;
			}
			if (gl->period > 0 && it % gl->period == 0) gl->ru_due = gl->ru_all = 1;
		} else if (err <= tol) {  // :193
			ls.done[lane] = 1;
			ls.exit_iter[lane] = it;
			ls.reason[lane] = STOP_CONVERGED;
			atomicSub(&gl->active, 1);
		} else if (it >= maxiter) {
			ls.done[lane] = 1;
			ls.exit_iter[lane] = maxiter + 1;
			ls.reason[lane] = STOP_MAXITER;
			atomicSub(&gl->active, 1);
		}
	}
};

// ---------------------------------------------------------------------------
// Pipelined CG (PipelinedCg.hpp:136-230), one sweep per iteration.  The
// stencil input is m = w .* iM (:158) from the w halo; the seven pointwise
// fields q, s, p, z, r, x, u are read directly in the epilogue (a TMA ring
// of eight fields would not fit in shared memory); the eight fused updates
// (:199-221) and the next iteration's <r,u>, <w,u>, <r,r> (:155) follow.
// w ping-pongs: iteration it reads W[(it+1)&1] and writes W[it&1].
// ---------------------------------------------------------------------------
template <class T>
struct OpPcg : OpBase<T> {
	static constexpr int NS = 1, NQ = 0, ND = 3;
	static constexpr bool IDENT = false, USES_RAW_CENTER = true, ADVANCE = true;
	static constexpr int V = Vec<T>::V;
	T iMc;
	T *x, *r, *u, *q, *s, *p, *z, *w0, *w1;
	T *wn;
	int it, mixed;
	T alpha[V], beta[V];
	bool fresh[V];  // iteration 1, or a lane restarted after an FP32 breakdown (mixed)
	bool hold[V];   // non-finite step (FP32 breakdown): the lane's fields stay as they are
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
		wn = (it & 1) ? w1 : w0;
#pragma unroll
		for (int e = 0; e < V; e++) {
			const int l = lane + e;
			const double g = ls.gamma[l], d = ls.delta[l];
			double al, be;
			fresh[e] = it == 1 || ls.s_exit[l] == 2;
			if (!fresh[e]) {  // :175-178
				be = __ddiv_rn(g, ls.gamma_old[l]);
				al = __ddiv_rn(1.0, __dsub_rn(__ddiv_rn(d, g), __ddiv_rn(be, ls.alpha[l])));
			} else {       // :179-181
				be = 0.0;
				al = __ddiv_rn(g, d);
			}
			if (ls.done[l]) al = be = 0.0;  // finished lanes stay frozen
			hold[e] = mixed && !(isfinite(al) && isfinite(be));
			if (hold[e]) al = be = 0.0;
			alpha[e] = (T)al;
			beta[e] = (T)be;
		}
	}
	__device__ bool raw_center() const { return true; }
	__device__ int src_map(int) const { return (it & 1) ? MT_W0_HALO : MT_W1_HALO; }
	__device__ int q_map(int) const { return 0; }
	__device__ Vec<T> src(const Vec<T> *raw) const {
		Vec<T> o;
#pragma unroll
		for (int e = 0; e < V; e++) o.v[e] = amul(raw[0].v[e], iMc);  // m = w .* iM
		return o;
	}
	__device__ void out(long long o, long long, int, const Vec<T> &mc, const Vec<T> &nc, const Vec<T> *,
	                    const Vec<T> *rc, const Vec<T> *gv, double (&part)[ND][V]) const {
		const Vec<T> wv = rc[0];
		Vec<T> qv = ldg_rw(q + o), sv = ldg_rw(s + o), pv = ldg_rw(p + o), zv = ldg_rw(z + o);
		Vec<T> rv = ldg_rw(r + o), xv = ldg_rw(x + o), uv = ldg_rw(u + o), wnv;
#pragma unroll
		for (int e = 0; e < V; e++) {
			if (hold[e]) {
				wnv.v[e] = wv.v[e];
				continue;
			}
			if (fresh[e]) {  // beta = 0, without multiplying stale values
				qv.v[e] = mc.v[e];
				sv.v[e] = wv.v[e];
				pv.v[e] = uv.v[e];
				zv.v[e] = nc.v[e];
			} else {
				qv.v[e] = aadd(mc.v[e], amul(beta[e], qv.v[e]));       // :200
				sv.v[e] = aadd(wv.v[e], amul(beta[e], sv.v[e]));       // :203
				pv.v[e] = aadd(uv.v[e], amul(beta[e], pv.v[e]));       // :206
				zv.v[e] = aadd(nc.v[e], amul(beta[e], zv.v[e]));       // :209
			}
			rv.v[e] = aadd(rv.v[e], amul(-alpha[e], sv.v[e]));     // :212
			xv.v[e] = aadd(xv.v[e], amul(alpha[e], pv.v[e]));      // :215
			uv.v[e] = aadd(uv.v[e], amul(-alpha[e], qv.v[e]));     // :218
			wnv.v[e] = aadd(wv.v[e], amul(-alpha[e], zv.v[e]));    // :221
			dacc(part[0][e], rv.v[e], uv.v[e]);
			dacc(part[1][e], wnv.v[e], uv.v[e]);
			dacc(part[2][e], rv.v[e], rv.v[e]);
		}
		stg(q + o, qv);
		stg(s + o, sv);
		stg(p + o, pv);
		stg(z + o, zv);
		stg(r + o, rv);
		stg(x + o, xv);
		stg(u + o, uv);
		stg(wn + o, wnv);
	}
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		if (ls.done[lane]) return;
		// The stop test uses <r,r> from the top of this iteration (:173, :227).
		const double err = sqrt(__ddiv_rn(ls.rr_top[lane], ls.bb[lane]));
		ls.err[lane] = err;
		if (ls.hist && lane == 0) ls.hist[it] = err;  // :228
		const double g = ls.gamma[lane], d = ls.delta[lane];
		double al;
		const bool restarted = ls.s_exit[lane] == 2;
		ls.s_exit[lane] = 0;
		if (it > 1 && !restarted) {
			const double be = __ddiv_rn(g, ls.gamma_old[lane]);
			al = __ddiv_rn(1.0, __dsub_rn(__ddiv_rn(d, g), __ddiv_rn(be, ls.alpha[lane])));
		} else {
			al = __ddiv_rn(g, d);
		}
		ls.gamma_old[lane] = g;
		ls.alpha[lane] = al;
		ls.gamma[lane] = tot[0];
		ls.delta[lane] = tot[1];
		ls.rr_top[lane] = tot[2];
		const double tol = gl->tol_in;
		const int maxiter = gl->maxiter;
		if (mixed) {
			if (!isfinite(al) || !(err == err)) ls.s_exit[lane] = 2;  // FP32 breakdown: restart after the update
			if (err <= tol || it >= maxiter || ls.s_exit[lane] == 2) {
				ls.pending[lane] = 1;
				gl->ru_due = 1;
			}
			if (gl->period > 0 && it % gl->period == 0) gl->ru_due = gl->ru_all = 1;
		} else if (err <= tol) {
			ls.done[lane] = 1;
			ls.exit_iter[lane] = it;
			ls.reason[lane] = STOP_CONVERGED;
			atomicSub(&gl->active, 1);
		} else if (it >= maxiter) {
			ls.done[lane] = 1;
			ls.exit_iter[lane] = maxiter + 1;
			ls.reason[lane] = STOP_MAXITER;
			atomicSub(&gl->active, 1);
		}
	}
};

// Pipelined CG setup and residual replacement: from r, u = r .* iM (:138)
// and w = A u (:141-143) into the w buffer the next iteration reads, plus the
// next iteration's <r,u>, <w,u>, <r,r>.  With `zero`, also q = s = p = z = 0
// (:146-149).  In a reliable update it runs only when one is due.
template <class T>
struct OpPcgUW : OpBase<T> {
	static constexpr int NS = 1, NQ = 0, ND = 3;
	static constexpr bool IDENT = false, USES_RAW_CENTER = true;
	static constexpr int V = Vec<T>::V;
	T iMc;
	T *u, *w0, *w1, *q, *s, *p, *z;
	T *wdst;
	int zero, ru;
	__device__ bool enabled(const Global *gl) const { return !ru || gl->ru_due; }
	__device__ void begin(const Global *gl, const LaneState &, int) {
		// The next iteration (gl->iter + 1 after a reliable update, 1 at setup) reads W[(it+1)&1].
		const int next = ru ? gl->iter + 1 : 1;
		wdst = (next & 1) ? w0 : w1;
	}
	__device__ bool raw_center() const { return true; }
	__device__ int src_map(int) const { return MT_R_HALO; }
	__device__ int q_map(int) const { return 0; }
	__device__ Vec<T> src(const Vec<T> *raw) const {
		Vec<T> o;
#pragma unroll
		for (int e = 0; e < V; e++) o.v[e] = amul(raw[0].v[e], iMc);
		return o;
	}
	__device__ void out(long long o, long long, int, const Vec<T> &uc, const Vec<T> &wv, const Vec<T> *,
	                    const Vec<T> *rc, const Vec<T> *gv, double (&part)[ND][V]) const {
		stg(u + o, uc);
		stg(wdst + o, wv);
		if (zero) {
			stg(q + o, vzero<T>());
			stg(s + o, vzero<T>());
			stg(p + o, vzero<T>());
			stg(z + o, vzero<T>());
		}
#pragma unroll
		for (int e = 0; e < V; e++) {
			dacc(part[0][e], rc[0].v[e], uc.v[e]);
			dacc(part[1][e], wv.v[e], uc.v[e]);
			dacc(part[2][e], rc[0].v[e], rc[0].v[e]);
		}
	}
	__device__ void fin(int lane, const double *tot, Global *, const LaneState &ls) const {
		if (ru && ls.done[lane]) return;
		ls.gamma[lane] = tot[0];
		ls.delta[lane] = tot[1];
		ls.rr_top[lane] = tot[2];
		if (!ru) {
			ls.gamma_old[lane] = 0.0;
			ls.alpha[lane] = 0.0;
		}
	}
};

// y = A f (+ y2 = y .* iM): the reliable update's s = A p, q = s .* iM and
// z = A q for pipelined CG.  No reductions.
template <class T>
struct OpApply : OpBase<T> {
	static constexpr int NS = 1, NQ = 0, ND = 0;
	static constexpr bool IDENT = true, USES_RAW_CENTER = false;
	static constexpr int V = Vec<T>::V;
	T iMc;
	T *y, *y2;
	int map;
	__device__ bool enabled(const Global *gl) const { return gl->ru_due != 0; }
	__device__ void begin(const Global *, const LaneState &, int) {}
	__device__ bool raw_center() const { return false; }
	__device__ int src_map(int) const { return map; }
	__device__ int q_map(int) const { return 0; }
	__device__ Vec<T> src(const Vec<T> *raw) const { return raw[0]; }
	__device__ void out(long long o, long long, int, const Vec<T> &, const Vec<T> &yv, const Vec<T> *, const Vec<T> *,
	                    const Vec<T> *, double (&)[1][V]) const {
		stg(y + o, yv);
		if (y2) {
			Vec<T> t;
#pragma unroll
			for (int e = 0; e < V; e++) t.v[e] = amul(yv.v[e], iMc);
			stg(y2 + o, t);
		}
	}
	__device__ void fin(int, const double *, Global *, const LaneState &) const {}
};

// ---------------------------------------------------------------------------
// BiCGStab (BiCgStab.hpp:157-232), three sweeps per iteration as in the
// single-vector form.  r, p and v ping-pong by iteration parity (iteration
// `it` reads R/P/V[(it&1) ? 0 : 1]-indexed as below and writes the other).
//   1: p = r + beta (p - omega v) (p = r on iteration 1), p_hat = p .* iM,
//      v = A p_hat, <v, r_hat>; alpha = rho / <v, r_hat>.
//   2: s = r - alpha v, s_hat = s .* iM, t = A s_hat; <s,s>, <t,s>, <t,t>;
//      early-exit flag on <s,s> < tol^2 or omega = <t,s>/<t,t>.
//   3: x += alpha p_hat (+ omega s_hat), r = s - omega t, <r,r>, next rho.
// Finished lanes are frozen with alpha = omega = 0.
// ---------------------------------------------------------------------------
template <class T>
struct OpBicg1 : OpBase<T> {
	static constexpr int NS = 3, NQ = 0, ND = 1, NG = 1;
	static constexpr bool IDENT = false, USES_RAW_CENTER = false, SCALED = true;
	static constexpr int V = Vec<T>::V;
	T iMc, kas, kbs, kcs;
	T *p0, *p1, *v0, *v1, *rhat;
	T *pn, *vn;
	int it;
	bool fresh[V];  // p = r: iteration 1, finished lanes, restarted lanes
	T beta[V], bo[V];
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
		pn = (it & 1) ? p1 : p0;
		vn = (it & 1) ? v1 : v0;
#pragma unroll
		for (int e = 0; e < V; e++) {
			const int l = lane + e;
			fresh[e] = it == 1 || ls.done[l] || ls.s_exit[l] == 2;
			double be = 0.0, bw = 0.0;
			if (!fresh[e]) {
				be = __dmul_rn(__ddiv_rn(ls.rho[l], ls.rho_prev[l]), __ddiv_rn(ls.alpha[l], ls.omega[l]));  // :166
				bw = __dmul_rn(-be, ls.omega[l]);
			}
			beta[e] = (T)be;
			bo[e] = (T)bw;
		}
	}
	__device__ bool raw_center() const { return true; }
	__device__ void gload(long long o, Vec<T> *gv) const { gv[0] = ldg_rw(rhat + o); }
	__device__ int src_map(int s) const {
		if (s == 0) return (it & 1) ? MT_R_HALO : MT_R1_HALO;
		if (s == 1) return (it & 1) ? MT_P0_HALO : MT_P1_HALO;
		return (it & 1) ? MT_V0_HALO : MT_V1_HALO;
	}
	__device__ int q_map(int) const { return 0; }
	__device__ Vec<T> pval(const Vec<T> *raw) const {
		Vec<T> o;
#pragma unroll
		for (int e = 0; e < V; e++)
			o.v[e] = fresh[e] ? raw[0].v[e]  // :171
			                  : aadd(aadd(raw[0].v[e], amul(beta[e], raw[1].v[e])), amul(bo[e], raw[2].v[e]));  // :168
		return o;
	}
	// The stencil input is p_hat = p .* iM (:175), formed at each read.
	__device__ Vec<T> src(const Vec<T> *raw) const { return pval(raw); }
	__device__ void out(long long o, long long, int, const Vec<T> &pv, const Vec<T> &vv, const Vec<T> *, const Vec<T> *,
	                    const Vec<T> *gv, double (&part)[ND][V]) const {
		stg(pn + o, pv);
		stg(vn + o, vv);
		const Vec<T> &rh = gv[0];  // r_hat
#pragma unroll
		for (int e = 0; e < V; e++) dacc(part[0][e], vv.v[e], rh.v[e]);
	}
	__device__ void fin(int lane, const double *tot, Global *, const LaneState &ls) const {
		if (ls.done[lane]) {
			ls.alpha[lane] = 0.0;
			return;
		}
		ls.alpha[lane] = __ddiv_rn(ls.rho[lane], tot[0]);  // :186
	}
};

template <class T>
struct OpBicgS : OpBase<T> {  // sweeps 2 and 3 share s, s_hat, t
	static constexpr int V = Vec<T>::V;
	static constexpr bool SCALED = true;  // the stencil input is s_hat = s .* iM (:201), formed at each read
	T iMc, kas, kbs, kcs;
	int it;
	T alpha[V];
	__device__ void load_alpha(const Global *gl, const LaneState &ls, int lane) {
		it = gl->iter;
#pragma unroll
		for (int e = 0; e < V; e++) alpha[e] = (T)(ls.done[lane + e] ? 0.0 : ls.alpha[lane + e]);
	}
	__device__ int src_map(int s) const {
		if (s == 0) return (it & 1) ? MT_R_HALO : MT_R1_HALO;
		return (it & 1) ? MT_V1_HALO : MT_V0_HALO;  // v written by sweep 1 of this iteration
	}
	__device__ Vec<T> sval(const Vec<T> *raw) const {
		Vec<T> o;
#pragma unroll
		for (int e = 0; e < V; e++) o.v[e] = aadd(raw[0].v[e], amul(-alpha[e], raw[1].v[e]));  // :189
		return o;
	}
	__device__ Vec<T> src(const Vec<T> *raw) const { return sval(raw); }
};

template <class T>
struct OpBicg2 : OpBicgS<T> {
	static constexpr int KIND = 1;
	static constexpr int NS = 2, NQ = 0, ND = 3;
	static constexpr bool IDENT = false, USES_RAW_CENTER = false;
	static constexpr int V = Vec<T>::V;
	__device__ bool enabled(const Global *) const { return true; }
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) { this->load_alpha(gl, ls, lane); }
	__device__ bool raw_center() const { return false; }
	__device__ int q_map(int) const { return 0; }
	__device__ void out(long long, long long, int, const Vec<T> &sv, const Vec<T> &tv, const Vec<T> *, const Vec<T> *,
	                    const Vec<T> *gv, double (&part)[ND][V]) const {
#pragma unroll
		for (int e = 0; e < V; e++) {
			dacc(part[0][e], sv.v[e], sv.v[e]);
			dacc(part[1][e], tv.v[e], sv.v[e]);
			dacc(part[2][e], tv.v[e], tv.v[e]);
		}
	}
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		if (ls.done[lane]) return;
		ls.s_norm2[lane] = tot[0];  // :192-193
		ls.ts[lane] = tot[1];
		ls.tt[lane] = tot[2];
		if (tot[0] < __dmul_rn(gl->tol_in, gl->tol_in)) {
			ls.s_exit[lane] = 1;  // :194
		} else {
			ls.s_exit[lane] = 0;
			ls.omega[lane] = __ddiv_rn(tot[1], tot[2]);  // :212
		}
	}
};

template <class T>
struct OpBicg3 : OpBicgS<T> {
	static constexpr int KIND = 1;
	static constexpr int NS = 2, NQ = 0, ND = 2, NG = 3;
	static constexpr bool IDENT = false, USES_RAW_CENTER = true, ADVANCE = true;
	static constexpr int V = Vec<T>::V;
	T *x, *r0, *r1, *p0, *p1, *rhat;
	T *rn, *pc;
	int mixed;
	T omega[V];
	int mode[V];  // 0: full update, 1: early exit on s (x only), 2: finished lane (x, r kept)
	bool keep_r;  // some lane of this thread keeps r: read the raw r at the centre
	__device__ bool enabled(const Global *) const { return true; }
	__device__ void begin(const Global *gl, const LaneState &ls, int lane) {
		this->load_alpha(gl, ls, lane);
		const int it = this->it;
		rn = (it & 1) ? r1 : r0;
		pc = (it & 1) ? p1 : p0;
#pragma unroll
		for (int e = 0; e < V; e++) {
			const int l = lane + e;
			mode[e] = ls.done[l] ? 2 : (ls.s_exit[l] ? 1 : 0);
			omega[e] = (T)(mode[e] ? 0.0 : ls.omega[l]);
		}
		keep_r = false;
#pragma unroll
		for (int e = 0; e < V; e++) keep_r |= mode[e] != 0;
	}
	__device__ bool raw_center() const { return keep_r; }
	__device__ void gload(long long o, Vec<T> *gv) const {
		gv[0] = ldg_rw(x + o);
		gv[1] = ldg_rw(pc + o);
		gv[2] = ldg_rw(rhat + o);
	}
	__device__ int q_map(int) const { return 0; }
	__device__ void out(long long o, long long, int, const Vec<T> &sv, const Vec<T> &tv, const Vec<T> *, const Vec<T> *rc,
	                    const Vec<T> *gv, double (&part)[ND][V]) const {
		Vec<T> shv;
#pragma unroll
		for (int e = 0; e < V; e++) shv.v[e] = amul(sv.v[e], this->iMc);  // s_hat (:201)
		Vec<T> xv = gv[0];
		const Vec<T> &pv = gv[1], &rh = gv[2];
		Vec<T> rv;
#pragma unroll
		for (int e = 0; e < V; e++) {
			const T ph = amul(pv.v[e], this->iMc);
			if (mode[e] == 2) {
				rv.v[e] = rc[0].v[e];
			} else if (mode[e] == 1) {
				xv.v[e] = aadd(xv.v[e], amul(this->alpha[e], ph));  // :196
				rv.v[e] = rc[0].v[e];
			} else {
				xv.v[e] = aadd(aadd(xv.v[e], amul(this->alpha[e], ph)), amul(omega[e], shv.v[e]));  // :216
				rv.v[e] = aadd(sv.v[e], amul(-omega[e], tv.v[e]));                                  // :219
			}
			dacc(part[0][e], rv.v[e], rv.v[e]);
			dacc(part[1][e], rv.v[e], rh.v[e]);
		}
		stg(x + o, xv);
		stg(rn + o, rv);
	}
	__device__ void fin(int lane, const double *tot, Global *gl, const LaneState &ls) const {
		if (ls.done[lane]) return;
		const int it = this->it;
		const double tol = gl->tol_in;
		const int maxiter = gl->maxiter;
		if (ls.s_exit[lane]) {
			if (mixed) {
				// The FP64 true residual decides; if it is still above tol the
				// lane restarts from it (s_exit = 2: r_hat = r, p = r).
				ls.s_exit[lane] = 2;
				ls.pending[lane] = 1;
				gl->ru_due = 1;
				return;
			}
			ls.done[lane] = 1;
			ls.exit_iter[lane] = it;
			ls.reason[lane] = STOP_SNORM;
			atomicSub(&gl->active, 1);
			return;
		}
		ls.rr[lane] = tot[0];
		const double err = sqrt(__ddiv_rn(tot[0], ls.bb[lane]));  // :226
		ls.err[lane] = err;
		if (ls.hist && lane == 0) ls.hist[it] = err;              // :228
		const double om = ls.omega[lane];
		if (mixed) {
			ls.rho_prev[lane] = ls.rho[lane];
			ls.rho[lane] = tot[1];
			if (om == 0.0 || tot[1] == 0.0) ls.s_exit[lane] = 2;  // breakdown: restart unless converged
			if (err <= tol || it >= maxiter || om == 0.0 || tot[1] == 0.0) {
				ls.pending[lane] = 1;
				gl->ru_due = 1;
			}
			if (gl->period > 0 && it % gl->period == 0) gl->ru_due = gl->ru_all = 1;
			return;
		}
		int stop = STOP_NONE, ex = 0;
		if (err <= tol) {                      // :228
			stop = STOP_CONVERGED;
			ex = it;
		} else if (om == 0.0) {                // :229
			stop = STOP_OMEGA;
			ex = it;
		} else {
			ls.rho_prev[lane] = ls.rho[lane];  // :231
			if (it >= maxiter) {
				stop = STOP_MAXITER;
				ex = maxiter + 1;
			} else {
				ls.rho[lane] = tot[1];           // next iteration :159-160
				if (tot[1] == 0.0) {             // :162
					stop = STOP_RHO;
					ex = it + 1;
				}
			}
		}
		if (stop != STOP_NONE) {
			ls.done[lane] = 1;
			ls.exit_iter[lane] = ex;
			ls.reason[lane] = stop;
			atomicSub(&gl->active, 1);
		}
	}
};

// Iteration bookkeeping between launches.
__global__ void kb_setup_done(Global *gl) { gl->active -= 1; }  // drops the setup sweep's guard

__global__ void kb_ru_done(Global *gl) {
	if (gl->ru_due) {
		gl->ru_due = 0;
		gl->ru_all = 0;
		gl->iter += 1;
	}
}

// Reliable update (MIXED): x_hi += x_lo, x_lo = 0.  x_hi uses FP64 slices
// of width WD, x_lo FP32 slices of width WT.  An update triggered by single
// lanes (convergence claims, maxiter, breakdowns) folds only those lanes;
// a periodic one (or any pipelined-CG one) folds every lane.  With CG's
// deferred x step (p_odd non-null) an update after an odd iteration also
// adds that iteration's step xa * p (its direction is in p_odd); the
// residual sweep that follows clears xa of the folded lanes.
__global__ void __launch_bounds__(256) kb_ru_fold(long long npts, int R, int WD, int WT, double *__restrict__ xh,
                                                  float *__restrict__ xl, const float *__restrict__ p_odd,
                                                  const double *__restrict__ xa, const int *__restrict__ pending,
                                                  int all, Global *gl) {
	if (gl->active == 0 || gl->ru_due == 0) return;
	all = all || gl->ru_all;
	const bool step = p_odd != nullptr && (gl->iter & 1);
	const long long pairs = npts * R / 2;
	for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < pairs;
	     u += (long long)gridDim.x * blockDim.x) {
		const long long od = 2 * u;  // FP64 offset
		const long long sd = od / ((long long)WD * npts);
		const long long rem = od - sd * WD * npts;
		const long long i = rem / WD;
		const int j = (int)(sd * WD + rem % WD);
		const bool f0 = all || pending[j], f1 = all || pending[j + 1];  // lanes j, j+1 share the pair
		if (!f0 && !f1) continue;
		// Both lanes of the pair fold x_lo (x_hi + x_lo is unchanged for a
		// lane outside the update); only the lanes in the update take their
		// pending x step.
		const long long ot = sliced(i, j, WT, npts);
		const float2 lo = *reinterpret_cast<const float2 *>(xl + ot);
		double2 hi = *reinterpret_cast<double2 *>(xh + od);
		hi.x += (double)lo.x;
		hi.y += (double)lo.y;
		if (step) {
			const float2 pv = *reinterpret_cast<const float2 *>(p_odd + ot);
			if (f0) hi.x += xa[j] * (double)pv.x;
			if (f1) hi.y += xa[j + 1] * (double)pv.y;
		}
		*reinterpret_cast<double2 *>(xh + od) = hi;
		*reinterpret_cast<float2 *>(xl + ot) = make_float2(0.f, 0.f);
	}
}

// FP64 CG with the deferred x step: a batch whose last iteration was odd
// (every lane stopped in the odd form of sweep B) still owes that
// iteration's step, x += alpha p (lanes stopped earlier have alpha 0).  The
// step rounds as the reference's x update (Cg.hpp:169).  Runs at the end of
// every graph chunk; kb_x_flush_done clears the flag so it applies once.
template <class T>
__global__ void __launch_bounds__(256) kb_x_flush(long long npts, int R, int W, T *__restrict__ x,
                                                  const T *__restrict__ p_odd, const double *__restrict__ xa,
                                                  const Global *gl) {
	if (gl->active != 0 || !gl->x_pending) return;
	const long long total = npts * R;
	for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < total;
	     u += (long long)gridDim.x * blockDim.x) {
		const int j = (int)(u / ((long long)W * npts)) * W + (int)(u % W);  // lane of element u
		x[u] = aadd(x[u], amul((T)xa[j], p_odd[u]));
	}
}

__global__ void kb_x_flush_done(Global *gl) {
	if (gl->active == 0) gl->x_pending = 0;
}

// ---------------------------------------------------------------------------
// Estimator accumulation over a batch: t += x .* v, q += v .* v per point,
// lanes in probe order (stochastic-estimator.cc:195, :198).  x and v are FP64
// fields in the sliced layout of width W.
// ---------------------------------------------------------------------------
__global__ void kb_accumulate(long long npts, int W, int nrhs, const double *__restrict__ x,
                              const double *__restrict__ v, double *__restrict__ t, double *__restrict__ q, int reset) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (long long)gridDim.x * blockDim.x) {
		double tt = reset ? 0.0 : t[i];
		double qq = reset ? 0.0 : q[i];
		for (int j = 0; j < nrhs; j++) {
			const long long o = sliced(i, j, W, npts);
			const double vj = v[o];
			tt = __dadd_rn(tt, __dmul_rn(x[o], vj));
			qq = __dadd_rn(qq, __dmul_rn(vj, vj));
		}
		t[i] = tt;
		q[i] = qq;
	}
}

__global__ void kb_divide(long long n, const double *__restrict__ t, const double *__restrict__ q,
                          double *__restrict__ D) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		D[i] = __ddiv_rn(t[i], q[i]);
}

// Dense right-hand sides (k*npts + i) -> sliced FP64 layout of width W over R
// lanes, zero padding lanes >= nrhs.
__global__ void kb_interleave(long long npts, int R, int W, int nrhs, const double *__restrict__ src,
                              double *__restrict__ dst) {
	const long long total = npts * R;
	for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (long long)gridDim.x * blockDim.x) {
		const long long s = u / ((long long)W * npts);
		const long long rem = u - s * W * npts;
		const long long i = rem / W;
		const int j = (int)(s * W + rem % W);
		dst[u] = j < nrhs ? src[(long long)j * npts + i] : 0.0;
	}
}

__global__ void kb_deinterleave(long long npts, int W, int nrhs, const double *__restrict__ src,
                                double *__restrict__ dst) {
	const long long total = npts * nrhs;
	for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (long long)gridDim.x * blockDim.x) {
		const long long j = u / npts;
		const long long i = u - j * npts;
		dst[u] = src[sliced(i, (int)j, W, npts)];
	}
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
	static EncodeTiledFn fn = nullptr;
	if (!fn) {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = (EncodeTiledFn)p;
		else
			cudaGetLastError();
	}
	return fn;
}

// 3-D map over a sliced field ([R/W slices][n3][n2][n1][W] of `eb`-byte
// elements) seen as [n3*slices][n2][n1*W]: one slice row of n1 points is a
// single contiguous TMA row.  Box W*b1 x b2 x 1; elements outside a row
// (points i1 < 0 or >= n1) and rows outside the grid read as zero.  Planes
// are never addressed outside a slice (planes -1 and n3 are handled without
// loads).
static bool make_map(CUtensorMap *m, void *base, int eb, const Geo &g, int R, int W, int b1, int b2) {
	EncodeTiledFn fn = encode_fn();
	if (!fn) return false;
	const cuuint64_t dims[3] = {(cuuint64_t)W * g.n1, (cuuint64_t)g.n2, (cuuint64_t)g.n3 * (R / W)};
	const cuuint64_t strides[2] = {(cuuint64_t)g.n1 * W * eb, (cuuint64_t)g.n1 * g.n2 * W * eb};
	const cuuint32_t box[3] = {(cuuint32_t)(W * b1), (cuuint32_t)b2, 1};
	const cuuint32_t es[3] = {1, 1, 1};
	return fn(m, eb == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides,
	          box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
	          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launch choices of the batched form for one (solver, precision, lanes,
// grid): lane-slice width of the Krylov fields, i3 split of the sweeps,
// reliable-update period and iterations per captured graph.  Zero fields
// mean "default".  Filled by sedi_autotune, read when a context is created.
// Default L2 prefetch distance of the sweeps, in planes (-1: 2 when a block
// streams at most 64 planes, else 0).  Measured on B200: at 128^3 x 64 lanes
// (32-plane chunks) 2 planes took mixed CG B from 462 to 442 us and the ring
// form of sweep A from 350 to 318 us, and the single-vector sweeps at 256^3
// (29-plane chunks) from 102 / 137 to 96 / 131 us; at 256^3 x 128 (whole
// columns) CG B went from 6.88 to 6.97 ms and in-place sweep A from 4.21 to
// 4.26 ms.
#ifndef SEDI_STREAM_PFD
#define SEDI_STREAM_PFD -1
#endif
// Form of the narrow sweeps (CG sweep A, BiCGStab sweeps 2 and 3): 1 ring
// (32x32), 2 in place (32x16, 2 blocks/SM), 3 in place (32x32, 6 stages).
// Defaults by measurement on B200 (kernels alone, fraction of measured HBM
// bandwidth, 256^3): batched CG sweep A form 3 (mixed x 128 lanes 4.21 ms,
// 95%, against 4.78 ms ring; FP64 2-lane slices 97% against 83%); BiCGStab
// sweep 2 ring (mixed 73% against 71%, FP64 74% against 67%); the
// single-vector sweeps ring (CG A 68% against 65%, BiCGStab 2 51% against
// 44%).
#ifndef SEDI_CGA_FORM
#define SEDI_CGA_FORM 3
#endif
#ifndef SEDI_NARROW_FORM
#define SEDI_NARROW_FORM 1
#endif
static int default_form(int ks, bool single) { return !single && ks == SEDI_CG ? SEDI_CGA_FORM : SEDI_NARROW_FORM; }
struct Tuning {
	int W = 0, nz = 0, period = 0, chunk = 0;
	int pfd = -1;   // L2 prefetch distance in planes (-1: the default, see SEDI_STREAM_PFD)
	int acfg = 0;   // form of the narrow sweeps (0: default_form)
};
struct TuneKey {
	int solver, precision, R;
	long long n1, n2, n3;
	bool operator<(const TuneKey &o) const {
		if (solver != o.solver) return solver < o.solver;
		if (precision != o.precision) return precision < o.precision;
		if (R != o.R) return R < o.R;
		if (n1 != o.n1) return n1 < o.n1;
		if (n2 != o.n2) return n2 < o.n2;
		return n3 < o.n3;
	}
};
static std::mutex g_tune_mu;
static std::map<TuneKey, Tuning> g_tune;

static Tuning tuning_for(const TuneKey &k) {
	std::lock_guard<std::mutex> lk(g_tune_mu);
	auto it = g_tune.find(k);
	return it == g_tune.end() ? Tuning() : it->second;
}

static void set_tuning(const TuneKey &k, const Tuning &t) {
	std::lock_guard<std::mutex> lk(g_tune_mu);
	g_tune[k] = t;
}

constexpr int kLaneDoubles = 19, kLaneInts = 5;  // LaneState arrays

#ifndef SEDI_MIXED_THETA_CG
#define SEDI_MIXED_THETA_CG 1.0
#endif
#ifndef SEDI_MIXED_THETA_PCG
#define SEDI_MIXED_THETA_PCG 1.0
#endif
// CG defers the x step of odd iterations to the next even one (OpCgB).
#ifndef SEDI_DEFER_X
#define SEDI_DEFER_X 1
#endif
#ifndef SEDI_MIXED_THETA_BICGSTAB
#define SEDI_MIXED_THETA_BICGSTAB 0.1
#endif


struct Batched;
typedef int (*SetupFn)(Ctx *, Batched *, int nrhs, int maxiter, double tol);
typedef int (*ChunkFn)(Ctx *, Batched *);

// Non-blocking estimator over the context's batches (stochastic-estimator.cc:158-216).
enum EstStage { EST_IDLE = 0, EST_SOLVE, EST_LANES, EST_FINAL, EST_DONE };
struct EstState {
	int stage = EST_IDLE;
	int samples = 0, k0 = 0, nb = 0, maxiter = 0, ignore_errors = 0, worst = 0, rc = 0;
	double tol = 0.0;
	uint32_t seed = 0;
	const double *probes_dev = nullptr;
	double *D_dev = nullptr, *t_dev = nullptr, *q_dev = nullptr, *D_host = nullptr;
	int *iters = nullptr, *results = nullptr;
	double *errs = nullptr;
	bool first = true;
	long long rounds = 0;
};

struct Batched {
	int R = 0;
	bool mixed = false;  // FP32 Krylov fields, FP64 x_hi, reductions and reliable update
	bool pairs = false;  // single-vector FP64 form: lanes 0/1 = even/odd i1 points of one vector
	bool defer_x = false;  // CG: x steps of odd iterations deferred to the next even one (OpCgB XS)
	int acfg = SEDI_NARROW_FORM;  // form of the narrow sweeps (see CfgFor, InPlace, default_form)
	int ks = 0;          // solver whose sweeps run (the mixed pipelined CG runs the CG recurrence)
	bool aliased = false;  // the Krylov fields belong to the context (single-vector form)
	const double *graph_hist = nullptr;  // history pointer the captured graph holds
	size_t elems = 0;  // npts * R
	// vectors ([point][R])
	void *x = nullptr;     // FP64 form: x; MIXED: x_lo (FP32)
	double *xh = nullptr;  // MIXED x_hi
	double *b = nullptr;   // right-hand sides (FP64)
	void *r = nullptr, *p0 = nullptr, *p1 = nullptr;
	void *w[2] = {nullptr, nullptr}, *u = nullptr, *q = nullptr, *sv = nullptr, *z = nullptr;  // pipelined CG
	void *r1 = nullptr, *v[2] = {nullptr, nullptr}, *rhat = nullptr;                        // BiCGStab
	double *partials = nullptr;
	unsigned *ticket = nullptr;
	Global *gl = nullptr, *gl_host = nullptr, *g0_host = nullptr;  // gl_host[0]: read back, g0_host: setup
	LaneState ls;
	double *lane_mem = nullptr, *lane_host = nullptr;
	int *lane_int = nullptr, *lane_host_int = nullptr;
	SetupFn setup_fn = nullptr;
	ChunkFn chunk_fn = nullptr;
	cudaEvent_t ev = nullptr;
	Tuning tuned;
	EstState est;
	std::vector<int> lane_res;  // result codes of the batch being processed
	double *t_acc = nullptr, *q_acc = nullptr;
	int period = 32;
	int chunk = 16;
	double theta = 1.0;  // mixed lanes stop on the FP64 true residual <= theta * tol
	cudaGraphExec_t graph = nullptr;
	long long graph_kernels = 0;
	// launch shapes
	int rbT = 0, rbD = 0;  // lanes per block slice for T and FP64 streams
	SGeo gT, gD, gT1;
	dim3 gridT, gridD, gridT1;
	Maps mapsT, mapsD, mapsT1;  // mapsT1, gT1: the wide-tile (KIND 1) sweeps
};

#define BTRY(expr)                                                            \
	do {                                                                      \
		cudaError_t e_ = (expr);                                              \
		if (e_ != cudaSuccess) return set_cuda_error(c, e_, #expr);           \
	} while (0)

// Stream configurations per (type, lane slice width).  The full slice is
// kSliceBytes per point; the point tile gives every block at least THREADS
// (point, lane group) slots.
#ifndef SEDI_STREAM_THREADS
#define SEDI_STREAM_THREADS 512
#endif
#ifndef SEDI_SLICE_LANES
#define SEDI_SLICE_LANES 8
#endif
constexpr int kThr = SEDI_STREAM_THREADS, kSliceLanes = SEDI_SLICE_LANES;

// Point tiles: at least THREADS (point, lane group) slots per block, and a
// merged TMA row W*(P1+2) within the 256-element box limit.
#ifndef SEDI_TILE_P1_LG1
#define SEDI_TILE_P1_LG1 32
#endif
#ifndef SEDI_TILE_P2_LG1
#define SEDI_TILE_P2_LG1 16
#endif
#ifndef SEDI_TILE_P1_LG2
#define SEDI_TILE_P1_LG2 16
#endif
#ifndef SEDI_TILE_P2_LG2
#define SEDI_TILE_P2_LG2 16
#endif
#ifndef SEDI_TILE_P1_LG4
#define SEDI_TILE_P1_LG4 16
#endif
#ifndef SEDI_TILE_P2_LG4
#define SEDI_TILE_P2_LG4 8
#endif
#ifndef SEDI_BLOCKS_PER_SM
#define SEDI_BLOCKS_PER_SM 1  // resident sweep blocks per SM (shared memory bound)
#endif
__host__ __device__ constexpr int tile_p1(int lg) {
	return lg == 1 ? SEDI_TILE_P1_LG1 : (lg == 2 ? SEDI_TILE_P1_LG2 : SEDI_TILE_P1_LG4);
}
__host__ __device__ constexpr int tile_p2(int lg) {
	return lg == 1 ? SEDI_TILE_P2_LG1 : (lg == 2 ? SEDI_TILE_P2_LG2 : SEDI_TILE_P2_LG4);
}

// KIND 1 ("wide") for sweeps with at most two stencil sources and no TMA
// pointwise fields: with one lane group per point (FP32 4-lane slices) a
// 32x32 tile, two output points per thread and a 4-stage ring (the per-plane
// barrier and latency are paid once per two points; 222 KB of shared
// memory).  Measured on B200 at 128^3 x 64 lanes: CG A 449 -> 372 us,
// BiCGStab 2 463 -> 353 us, BiCGStab 3 877 -> 787 us.
// KIND 2 and 3 are the in-place forms of CG's sweep A (no ring): KIND 2 the
// 32x16 tile with a 5-stage ring, small enough for two blocks per SM
// (98 KB each, 64 registers per thread); KIND 3 the 32x32 tile with a
// 6-stage ring (three planes of TMA lookahead instead of two).
template <class T, int RB, int KIND = 0, bool PAIRS = false>
struct CfgFor {
	static constexpr int LG = RB * (int)sizeof(T) / 16;
	static constexpr bool WIDE = (KIND == 1 || KIND == 3) && LG == 1;
	static constexpr int NSTR = LG != 1 ? 0 : (KIND == 1 ? 4 : (KIND == 2 ? 5 : (KIND == 3 ? 6 : 0)));
	static constexpr int MINB = (KIND == 2 && LG == 1) ? 2 : 1;
	typedef Cfg<T, RB, tile_p1(LG), WIDE ? 32 : tile_p2(LG), kThr, NSTR, PAIRS, MINB> type;
};

static int pick_R(int nrhs, bool mixed) {
	const int V = mixed ? 4 : 2, full = 8 * V;
	if (nrhs <= V) return V;
	if (nrhs <= 2 * V) return 2 * V;
	if (nrhs <= 4 * V) return 4 * V;
	return (nrhs + full - 1) / full * full;
}

// Lanes per slice: FP32 Krylov fields 4 (16 B per point); FP64 Krylov fields
// of CG and BiCGStab 2 (16 B per point), of pipelined CG 8 (64 B per point);
// the FP64 x and b of the mixed form 8 (mixed_slice_fp64).  16 B per point gets the 32x32 tiles
// and deep stage rings of the narrow sweeps.  Measured on B200 (kernels
// alone, 64 lanes): FP64 CG sweep A at 256^3 4.11 ms with 2 lanes against
// 5.83 ms with 8, BiCGStab sweep 2 3.98 against 5.20 ms, sweep 3 10.79
// against 12.78 ms; pipelined CG 21.6 ms with 8 against 22.7 ms with 2; the
// FP32 sweeps 2-19% faster with 4 lanes than with 8 at 128^3.  The
// autotuner may override it per shape.
#ifndef SEDI_SLICE_LANES_FP32
#define SEDI_SLICE_LANES_FP32 4
#endif
#ifndef SEDI_SLICE_LANES_FP64_NARROW
#define SEDI_SLICE_LANES_FP64_NARROW 2
#endif
static int slice_for(int R, bool fp64, int ks = 0) {
	const int w = !fp64 ? SEDI_SLICE_LANES_FP32
	                    : ((ks == SEDI_CG || ks == SEDI_BICGSTAB) ? SEDI_SLICE_LANES_FP64_NARROW : kSliceLanes);
	return R >= w ? w : R;
}

// FP64 fields of the mixed form (x_hi, b), streamed by the setup and
// reliable-update residual sweep and the fold: 8-lane slices, so a block's
// FP32 r (and the fold's x_lo) covers whole 4-lane vectors.  With 2-lane
// slices (32x16 tiles instead of 16x8) the residual sweep kept its 12.8 ms
// at 256^3 x 128 (each block wrote half of every FP32 r vector), setup took
// 16.7 against 12.6 ms and the fold 11.1 against 9.6 ms (ncu launch lists).
static int mixed_slice_fp64(int R) { return slice_for(R, true); }

static void tile_for(int rb, int eb, int *P1, int *P2, int kind = 0) {
	const int lg = rb * eb / 16;
	*P1 = tile_p1(lg);
	*P2 = (kind == 1 && lg == 1) ? 32 : tile_p2(lg);
}

static void shape(const Geo &g, int R, int rb, int eb, SGeo *sg, dim3 *grid, int nz_force = 0, int kind = 0,
                  int pfd = -1) {
	int P1, P2;
	tile_for(rb, eb, &P1, &P2, kind);
	const int t1 = (g.n1 + P1 - 1) / P1, t2 = (g.n2 + P2 - 1) / P2;
	const int slices = R / rb;
	// Split i3 into nz chunks of zc planes.  Blocks run in waves of
	// 148 x SEDI_BLOCKS_PER_SM; a block streams zc + 2 planes and costs about
	// four more in pipeline fill, launch and its share of the reduction
	// (single-vector CG sweep A at 256^3 on B200: one wave of 128 blocks of
	// 64 planes, 92 us, beats two waves of 29-plane blocks, 95 us).  Pick the
	// split with the fewest wave-planes (the last wave counts in full), the
	// smaller split on ties.
	const long long per = (long long)t1 * t2 * slices;
	const long long wave = 148LL * SEDI_BLOCKS_PER_SM;
	long long best = -1;
	int zc = g.n3, nz = 1;
	const int maxz = g.n3 < 64 ? g.n3 : 64;
	for (int k = 1; k <= maxz; k++) {
		const int z = (g.n3 + k - 1) / k;
		if (z < 2 && g.n3 >= 2) break;
		const int kk = (g.n3 + z - 1) / z;
		const long long waves = (per * kk + wave - 1) / wave;
		const long long cost = waves * (z + 6);
		if (best < 0 || cost < best) {
			best = cost;
			zc = z;
			nz = kk;
		}
	}
	if (nz_force > 0) {  // autotuned split
		const int k = nz_force < g.n3 ? nz_force : g.n3;
		zc = (g.n3 + k - 1) / k;
		nz = (g.n3 + zc - 1) / zc;
	}
	sg->n1 = g.n1;
	sg->n2 = g.n2;
	sg->n3 = g.n3;
	sg->R = R;
	sg->W = rb;
	sg->npts = g.n;
	sg->zc = zc;
	sg->tiles1 = t1;
	sg->pfd = pfd >= 0 ? pfd : (SEDI_STREAM_PFD >= 0 ? SEDI_STREAM_PFD : (zc <= 64 ? 2 : 0));
	*grid = dim3((unsigned)(t1 * t2), (unsigned)slices, (unsigned)nz);
}

template <class C, class Op>
static int launch(Ctx *c, Batched *B, const SGeo &sg, dim3 grid, const Maps &maps, const Op &op, cudaStream_t s) {
	const size_t sm = Layout<C, Op::NS, Op::NQ, Op::ND, Op::IDENT, Op::INPLACE>::BYTES;
	static bool attr_set = false;
	if (!attr_set) {
		cudaFuncSetAttribute(k_stream<C, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
		attr_set = true;
	}
	k_stream<C, Op><<<grid, C::THREADS, sm, s>>>(sg, maps, op, B->partials, B->ticket, B->gl, B->ls);
	c->launches++;
	return 0;
}

// Launch of a sweep over the T (Krylov) fields with the op's tile kind.
template <class T, int RBT, bool PAIRS = false, class Op>
static int launchT(Ctx *c, Batched *B, const Op &op, cudaStream_t s) {
	typedef typename CfgFor<T, RBT, Op::KIND, PAIRS>::type C;
	if (Op::KIND == 1 || Op::KIND == 3) return launch<C>(c, B, B->gT1, B->gridT1, B->mapsT1, op, s);
	return launch<C>(c, B, B->gT, B->gridT, B->mapsT, op, s);
}

static void bind_impl(Batched *B);

// Sweeps a context runs.  The mixed form of pipelined CG runs the CG
// recurrence: pipelining hides the latency of a distributed reduction
// (PipelinedCg.hpp:155-184), which one GPU, whose reductions end on the
// device, does not have; in FP32 its extra recurrences (w, z, s, q) drift
// from the FP64 iterates (27% more iterations and a diagonal 9e-8 from the
// FP64 form's at 256^3 x 32 probes, tol 1e-9), while CG's FP32 iterates
// follow the FP64 ones and FP64 CG and FP64 pipelined CG give the same
// diagonal to about 1e-9.  It also moves 8 instead of 16 words per point
// and iteration.
static int kernel_solver(int solver, bool mixed) { return mixed && solver == SEDI_PIPELINED_CG ? SEDI_CG : solver; }

// Default in-loop target of the mixed form, theta * tol on the FP64 true
// residual (measured at 48^3, 128^3 and 256^3, tol 1e-9, against the FP64
// form and against a solve to 1e-13).  CG's FP32 iterates follow the FP64
// ones, so theta = 1 gives the FP64 diagonal to 1.1e-9 .. 3.9e-9; a tighter
// target moves the mixed solution towards the exact one and so away from
// the FP64 form's, whose own truncation error is 4e-9 .. 4e-8.  BiCGStab's
// FP64 diagonal lies 1e-7 .. 4e-7 from the exact one, and theta = 0.1 puts
// the mixed diagonal ten times closer to it (10% more iterations).
static double default_theta(int solver) {
	switch (solver) {
	case 2: return SEDI_MIXED_THETA_CG;
	case 3: return SEDI_MIXED_THETA_PCG;
	default: return SEDI_MIXED_THETA_BICGSTAB;
	}
}

int batched_set_theta(Ctx *c, double theta) {
	Batched *B = (Batched *)c->batched;
	if (!B || !B->mixed) {
		c->error = "the in-loop target applies to the mixed-precision batched form";
		return SEDI_ERR_UNSUPPORTED;
	}
	if (!(theta > 0.0 && theta <= 1.0)) {
		c->error = "theta must be in (0, 1]";
		return SEDI_ERR_ARG;
	}
	B->theta = theta;
	return 0;
}

double batched_theta(const Ctx *c) {
	const Batched *B = (const Batched *)c->batched;
	return B && B->mixed ? B->theta : 1.0;
}

int batched_alloc(Ctx *c) {
	Batched *B = new (std::nothrow) Batched();
	if (!B) return SEDI_ERR_NOMEM;
	c->batched = B;
	B->mixed = c->precision == SEDI_PREC_MIXED;
	B->ks = kernel_solver(c->solver, B->mixed);
	B->defer_x = SEDI_DEFER_X && B->ks == SEDI_CG;
	if (c->batch > (B->mixed ? 256 : 128)) {
		c->error = "batch too large for one context (max 256 FP32 / 128 FP64 right-hand sides)";
		return SEDI_ERR_ARG;
	}
	if (!encode_fn()) {
		c->error = "cuTensorMapEncodeTiled unavailable";
		return SEDI_ERR_NODEV;
	}
	B->R = pick_R(c->batch, B->mixed);
	B->elems = (size_t)c->g.n * B->R;
	const int ebT = B->mixed ? 4 : 8;
	const Tuning tu = tuning_for(TuneKey{c->solver, c->precision, B->R, c->g.n1, c->g.n2, c->g.n3});
	B->rbT = slice_for(B->R, !B->mixed, B->ks);
	if (tu.W > 0 && tu.W <= B->R && B->R % tu.W == 0) B->rbT = tu.W;
	B->rbD = B->mixed ? mixed_slice_fp64(B->R) : B->rbT;  // FP64 x is read through the FP64 maps
	B->tuned = tu;
	if (tu.period > 0) B->period = tu.period;
	B->acfg = tu.acfg >= 1 && tu.acfg <= 3 ? tu.acfg : default_form(B->ks, false);
	B->theta = default_theta(B->ks);
	if (tu.chunk > 0) B->chunk = tu.chunk;
	shape(c->g, B->R, B->rbT, ebT, &B->gT, &B->gridT, tu.nz, 0, tu.pfd);
	shape(c->g, B->R, B->rbT, ebT, &B->gT1, &B->gridT1, tu.nz, 1, tu.pfd);
	shape(c->g, B->R, B->rbD, 8, &B->gD, &B->gridD, tu.nz, 0, tu.pfd);
	const size_t ts = (size_t)ebT;                                  // Krylov field element
	const size_t xs = B->mixed ? sizeof(float) : sizeof(double);   // x (FP64 form) or x_lo (mixed)
	const size_t nblkT = (size_t)B->gridT.x * B->gridT.z, nblkD = (size_t)B->gridD.x * B->gridD.z;
	const size_t nblkT1 = (size_t)B->gridT1.x * B->gridT1.z;
	size_t nblk = nblkT > nblkD ? nblkT : nblkD;
	if (nblkT1 > nblk) nblk = nblkT1;
	if (cudaMalloc(&B->x, B->elems * xs) != cudaSuccess || cudaMalloc(&B->r, B->elems * ts) != cudaSuccess ||
	    cudaMalloc(&B->p0, B->elems * ts) != cudaSuccess || cudaMalloc(&B->p1, B->elems * ts) != cudaSuccess ||
	    cudaMalloc(&B->b, B->elems * sizeof(double)) != cudaSuccess ||
	    (B->mixed && cudaMalloc(&B->xh, B->elems * sizeof(double)) != cudaSuccess) ||
	    cudaMalloc(&B->partials, sizeof(double) * nblk * kMaxDots * B->R) != cudaSuccess ||
	    cudaMalloc(&B->ticket, sizeof(unsigned)) != cudaSuccess || cudaMalloc(&B->gl, sizeof(Global)) != cudaSuccess ||
	    cudaMallocHost(&B->gl_host, 2 * sizeof(Global)) != cudaSuccess ||
	    cudaMallocHost(&B->lane_host, sizeof(double) * kLaneDoubles * B->R) != cudaSuccess ||
	    cudaMallocHost(&B->lane_host_int, sizeof(int) * kLaneInts * B->R) != cudaSuccess ||
	    cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming) != cudaSuccess ||
	    cudaMalloc(&B->lane_mem, sizeof(double) * kLaneDoubles * B->R) != cudaSuccess ||
	    cudaMalloc(&B->lane_int, sizeof(int) * 5 * B->R) != cudaSuccess ||
	    cudaMalloc(&B->t_acc, sizeof(double) * c->g.n) != cudaSuccess ||
	    cudaMalloc(&B->q_acc, sizeof(double) * c->g.n) != cudaSuccess) {
		cudaGetLastError();
		c->error = "device allocation failed (batched form)";
		return SEDI_ERR_NOMEM;
	}
	if (B->ks == 3 || B->ks == 1) {
		void **pcg[] = {&B->w[0], &B->w[1], &B->u, &B->q, &B->sv, &B->z};
		void **bicg[] = {&B->r1, &B->v[0], &B->v[1], &B->rhat};
		void ***pv = B->ks == 3 ? pcg : bicg;
		const int np = B->ks == 3 ? 6 : 4;
		for (int i = 0; i < np; i++) {
			if (cudaMalloc(pv[i], B->elems * ts) != cudaSuccess) {
				cudaGetLastError();
				c->error = "device allocation failed (batched solver vectors)";
				return SEDI_ERR_NOMEM;
			}
			cudaMemsetAsync(*pv[i], 0, B->elems * ts, c->stream);
		}
	}
	// Zero-fills on the context's stream (its own, non-blocking one at this
	// point): legacy-stream memsets would not be ordered before its kernels.
	cudaMemsetAsync(B->ticket, 0, sizeof(unsigned), c->stream);
	cudaMemsetAsync(B->x, 0, B->elems * xs, c->stream);
	cudaMemsetAsync(B->r, 0, B->elems * ts, c->stream);
	cudaMemsetAsync(B->p0, 0, B->elems * ts, c->stream);
	cudaMemsetAsync(B->p1, 0, B->elems * ts, c->stream);
	cudaMemsetAsync(B->lane_mem, 0, sizeof(double) * kLaneDoubles * B->R, c->stream);
	cudaMemsetAsync(B->lane_int, 0, sizeof(int) * kLaneInts * B->R, c->stream);
	const int R = B->R;
	LaneState &ls = B->ls;
	double **dp[] = {&ls.bb, &ls.rr, &ls.err, &ls.ru, &ls.ru_new, &ls.sp, &ls.alpha, &ls.beta, &ls.gamma,
	                 &ls.gamma_old, &ls.delta, &ls.rr_top, &ls.rho, &ls.rho_prev, &ls.omega, &ls.s_norm2, &ls.ts,
	                 &ls.tt, &ls.xa};
	static_assert(sizeof(dp) / sizeof(dp[0]) == kLaneDoubles, "lane arrays");
	for (size_t i = 0; i < sizeof(dp) / sizeof(dp[0]); i++) *dp[i] = B->lane_mem + i * R;
	int **ip[] = {&ls.done, &ls.exit_iter, &ls.reason, &ls.pending, &ls.s_exit};
	for (size_t i = 0; i < 5; i++) *ip[i] = B->lane_int + i * R;
	// Tensor maps.
	int P1, P2;
	auto t_maps = [&](Maps &M, int kind) {
		int Q1, Q2;
		tile_for(B->rbT, ebT, &Q1, &Q2, kind);
		bool k = make_map(&M.m[MT_R_HALO], B->r, ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_P0_HALO], B->p0, ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_P1_HALO], B->p1, ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_X_INT], B->x, ebT, c->g, R, B->rbT, Q1, Q2) &&
		         make_map(&M.m[MT_R_INT], B->r, ebT, c->g, R, B->rbT, Q1, Q2) &&
		         make_map(&M.m[MT_P1_INT], B->p1, ebT, c->g, R, B->rbT, Q1, Q2);
		if (B->ks == 3)
			k = k && make_map(&M.m[MT_W0_HALO], B->w[0], ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_W1_HALO], B->w[1], ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_Q_HALO], B->q, ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2);
		if (B->ks == 1)
			k = k && make_map(&M.m[MT_R1_HALO], B->r1, ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_V0_HALO], B->v[0], ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_V1_HALO], B->v[1], ebT, c->g, R, B->rbT, Q1 + 2, Q2 + 2);
		return k;
	};
	bool ok = t_maps(B->mapsT, 0) && t_maps(B->mapsT1, 1);
	tile_for(B->rbD, 8, &P1, &P2);
	ok = ok && make_map(&B->mapsD.m[MD_X_HALO], B->mixed ? (void *)B->xh : B->x, 8, c->g, R, B->rbD, P1 + 2, P2 + 2) &&
	     make_map(&B->mapsD.m[MD_B_INT], B->b, 8, c->g, R, B->rbD, P1, P2);
	if (!ok) {
		c->error = "tensor map encoding failed";
		return SEDI_ERR_CUDA;
	}
	B->g0_host = B->gl_host + 1;
	B->lane_res.assign(B->R, 0);
	bind_impl(B);
	// The zero-fills must be complete before a caller stream (sedi_set_stream) uses the buffers.
	if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_cuda_error(c, cudaGetLastError(), "batched_alloc");
	return 0;
}

// Device bytes batched_alloc takes for a context (each allocation rounded
// up to the 2 MiB granularity of large device allocations).
int batched_lanes(int precision, int batch) { return pick_R(batch, precision == SEDI_PREC_MIXED); }

size_t batched_bytes(int solver, int precision, int batch, long long n1, long long n2, long long n3) {
	const bool mixed = precision == SEDI_PREC_MIXED;
	Geo g;
	g.n1 = (int)n1;
	g.n2 = (int)n2;
	g.n3 = (int)n3;
	g.n = n1 * n2 * n3;
	const int R = pick_R(batch, mixed);
	const size_t elems = (size_t)g.n * R, ts = mixed ? 4 : 8, xs = mixed ? 4 : 8;
	const Tuning tu = tuning_for(TuneKey{solver, precision, R, n1, n2, n3});
	int wT = slice_for(R, !mixed, kernel_solver(solver, mixed));
	if (tu.W > 0 && tu.W <= R && R % tu.W == 0) wT = tu.W;
	SGeo sT, sD;
	dim3 gT, gD;
	shape(g, R, wT, (int)ts, &sT, &gT, tu.nz);
	shape(g, R, mixed ? mixed_slice_fp64(R) : wT, 8, &sD, &gD, tu.nz);
	SGeo sT1;
	dim3 gT1;
	shape(g, R, wT, (int)ts, &sT1, &gT1, tu.nz, 1);
	const size_t nblkT = (size_t)gT.x * gT.z, nblkD = (size_t)gD.x * gD.z, nblkT1 = (size_t)gT1.x * gT1.z;
	size_t nblk = nblkT > nblkD ? nblkT : nblkD;
	if (nblkT1 > nblk) nblk = nblkT1;
	auto up = [](size_t b) { return (b + (2u << 20) - 1) / (2u << 20) * (2u << 20); };
	const int ks = kernel_solver(solver, mixed);
	const int nT = 3 + (ks == 3 ? 6 : 0) + (ks == 1 ? 4 : 0);  // r, p0, p1 and the solver's own
	size_t total = nT * up(elems * ts) + up(elems * xs) + up(elems * 8) * (mixed ? 2 : 1);
	total += up(sizeof(double) * nblk * kMaxDots * R) + 3 * up(1) + up(sizeof(double) * kLaneDoubles * R) +
	         up(sizeof(int) * 5 * R) + 2 * up(sizeof(double) * g.n);
	return total;
}

static void free_batched(Batched *B) {
	if (!B) return;
	void *fields[] = {B->x, B->xh, B->b, B->r, B->p0, B->p1, B->t_acc, B->q_acc, B->w[0], B->w[1], B->u, B->q,
	                  B->sv, B->z, B->r1, B->v[0], B->v[1], B->rhat};
	if (!B->aliased)
		for (void *p : fields)
			if (p) cudaFree(p);
	void *own[] = {B->partials, B->ticket, B->gl, B->lane_mem, B->lane_int};
	for (void *p : own)
		if (p) cudaFree(p);
	if (B->gl_host) cudaFreeHost(B->gl_host);
	if (B->lane_host) cudaFreeHost(B->lane_host);
	if (B->lane_host_int) cudaFreeHost(B->lane_host_int);
	if (B->ev) cudaEventDestroy(B->ev);
	if (B->graph) cudaGraphExecDestroy(B->graph);
	delete B;
}

void batched_free(Ctx *c) {
	Batched *B = (Batched *)c->batched;
	if (!B) return;
	void *ptrs[] = {B->x, B->xh, B->b, B->r, B->p0, B->p1, B->partials, B->ticket, B->gl, B->lane_mem, B->lane_int,
	                B->t_acc, B->q_acc, B->w[0], B->w[1], B->u, B->q, B->sv, B->z, B->r1, B->v[0], B->v[1],
	                B->rhat};
	for (void *p : ptrs)
		if (p) cudaFree(p);
	if (B->gl_host) cudaFreeHost(B->gl_host);
	if (B->lane_host) cudaFreeHost(B->lane_host);
	if (B->lane_host_int) cudaFreeHost(B->lane_host_int);
	if (B->ev) cudaEventDestroy(B->ev);
	if (B->graph) cudaGraphExecDestroy(B->graph);
	delete B;
	c->batched = nullptr;
}

template <int RBD, bool PAIRS = false>
static void enqueue_resid(Ctx *c, Batched *B, bool ru) {
	const int pcg = B->ks == 3 ? 1 : 0;
	typedef typename CfgFor<double, RBD, 0, PAIRS>::type CD;
	cudaStream_t s = c->stream;
	if (B->mixed) {
		OpResid<float> op;
		op.ka = c->k.a;
		op.kb = c->k.b;
		op.kc = c->k.c;
		op.r = (float *)B->r;
		op.r_alt = (float *)B->r1;
		op.rhat = (float *)B->rhat;  // BiCGStab only (null otherwise)
		op.xlo = ru ? nullptr : (float *)B->x;
		op.WT = B->rbT;
		op.npts = c->g.n;
		op.iMd = 1.0 / c->k.a;
		op.solver = B->ks;
		op.ru = ru ? 1 : 0;
		op.pcg = pcg;
		launch<CD>(c, B, B->gD, B->gridD, B->mapsD, op, s);
	} else {
		OpResid<double> op;
		op.ka = c->k.a;
		op.kb = c->k.b;
		op.kc = c->k.c;
		op.r = (double *)B->r;
		op.r_alt = (double *)B->r1;
		op.rhat = (double *)B->rhat;
		op.xlo = nullptr;
		op.WT = B->rbT;
		op.npts = c->g.n;
		op.iMd = 1.0 / c->k.a;
		op.solver = B->ks;
		op.ru = 0;
		op.pcg = pcg;
		launch<CD>(c, B, B->gD, B->gridD, B->mapsD, op, s);
	}
}

template <class T, int RBT, bool PAIRS = false>
static void launch_cg_a(Ctx *c, Batched *B, const OpCgA<T> &a, cudaStream_t s) {
	switch (B->acfg) {
	case 2: launchT<T, RBT, PAIRS>(c, B, OpCgAv<T, 2>(a), s); break;
	case 3: launchT<T, RBT, PAIRS>(c, B, OpCgAv<T, 3>(a), s); break;
	default: launchT<T, RBT, PAIRS>(c, B, a, s);
	}
}

template <int XS, class T>
static OpCgB<T, XS> cg_b_as(const OpCgB<T> &o) {
	OpCgB<T, XS> d;
	d.ka = o.ka;
	d.kb = o.kb;
	d.kc = o.kc;
	d.iMc = o.iMc;
	d.x = o.x;
	d.r = o.r;
	d.mixed = o.mixed;
	return d;
}

template <class T, int RBT, int RBD, bool PAIRS = false>
static void enqueue_cg_iteration(Ctx *c, Batched *B) {
	cudaStream_t s = c->stream;
	OpCgA<T> a;
	a.ka = (T)c->k.a;
	a.kb = (T)c->k.b;
	a.kc = (T)c->k.c;
	a.iMc = (T)(1.0 / c->k.a);
	a.p0 = (T *)B->p0;
	a.p1 = (T *)B->p1;
	a.mixed = B->mixed ? 1 : 0;
	launch_cg_a<T, RBT, PAIRS>(c, B, a, s);
	OpCgB<T> bo;
	bo.ka = (T)c->k.a;
	bo.kb = (T)c->k.b;
	bo.kc = (T)c->k.c;
	bo.iMc = (T)(1.0 / c->k.a);
	bo.x = (T *)B->x;
	bo.r = (T *)B->r;
	bo.mixed = B->mixed ? 1 : 0;
	if (B->defer_x) {
		// Both are captured; each runs only on its iteration parity.
		launchT<T, RBT, PAIRS>(c, B, cg_b_as<XS_R>(bo), s);
		launchT<T, RBT, PAIRS>(c, B, cg_b_as<XS_X>(bo), s);
	} else {
		launchT<T, RBT, PAIRS>(c, B, bo, s);
	}
	if (B->mixed) {
		const long long nb = ((long long)B->elems / 2 + 255) / 256;
		kb_ru_fold<<<(int)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(c->g.n, B->R, B->rbD, B->rbT, B->xh,
		                                                                 (float *)B->x, B->defer_x ? (const float *)B->p1 : nullptr,
		                                                                 B->ls.xa, B->ls.pending, B->ks == 3 ? 1 : 0, B->gl);
		c->launches++;
		enqueue_resid<RBD, PAIRS>(c, B, true);
		kb_ru_done<<<1, 1, 0, s>>>(B->gl);
		c->launches++;
	}
}

template <class T, int RBT, bool PAIRS = false>
static void enqueue_pcg_uw(Ctx *c, Batched *B, int zero, int ru) {
	OpPcgUW<T> o;
	o.ka = (T)c->k.a;
	o.kb = (T)c->k.b;
	o.kc = (T)c->k.c;
	o.iMc = (T)(1.0 / c->k.a);
	o.u = (T *)B->u;
	o.w0 = (T *)B->w[0];
	o.w1 = (T *)B->w[1];
	o.q = (T *)B->q;
	o.s = (T *)B->sv;
	o.p = (T *)B->p0;
	o.z = (T *)B->z;
	o.zero = zero;
	o.ru = ru;
	launchT<T, RBT, PAIRS>(c, B, o, c->stream);
}

template <class T, int RBT, int RBD, bool PAIRS = false>
static void enqueue_pcg_iteration(Ctx *c, Batched *B) {
	cudaStream_t s = c->stream;
	OpPcg<T> o;
	o.ka = (T)c->k.a;
	o.kb = (T)c->k.b;
	o.kc = (T)c->k.c;
	o.iMc = (T)(1.0 / c->k.a);
	o.x = (T *)B->x;
	o.r = (T *)B->r;
	o.u = (T *)B->u;
	o.q = (T *)B->q;
	o.s = (T *)B->sv;
	o.p = (T *)B->p0;
	o.z = (T *)B->z;
	o.w0 = (T *)B->w[0];
	o.w1 = (T *)B->w[1];
	o.mixed = B->mixed ? 1 : 0;
	launchT<T, RBT, PAIRS>(c, B, o, s);
	if (B->mixed) {
		// Residual replacement (reliable update) of pipelined CG: x_hi += x_lo;
		// r = b - A x_hi (FP64); s = A p, q = s .* iM; z = A q; u = r .* iM,
		// w = A u and the next iteration's dots.
		const long long nb = ((long long)B->elems / 2 + 255) / 256;
		kb_ru_fold<<<(int)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(c->g.n, B->R, B->rbD, B->rbT, B->xh,
		                                                                 (float *)B->x, nullptr, B->ls.xa, B->ls.pending,
		                                                                 B->ks == 3 ? 1 : 0, B->gl);
		c->launches++;
		enqueue_resid<RBD, PAIRS>(c, B, true);
		OpApply<T> a1;
		a1.ka = (T)c->k.a;
		a1.kb = (T)c->k.b;
		a1.kc = (T)c->k.c;
		a1.iMc = (T)(1.0 / c->k.a);
		a1.y = (T *)B->sv;
		a1.y2 = (T *)B->q;
		a1.map = MT_P0_HALO;
		launchT<T, RBT, PAIRS>(c, B, a1, s);
		OpApply<T> a2 = a1;
		a2.y = (T *)B->z;
		a2.y2 = nullptr;
		a2.map = MT_Q_HALO;
		launchT<T, RBT, PAIRS>(c, B, a2, s);
		enqueue_pcg_uw<T, RBT, PAIRS>(c, B, 0, 1);
		kb_ru_done<<<1, 1, 0, s>>>(B->gl);
		c->launches++;
	}
}

// Coefficients of an op whose stencil input is f .* iM (Op::SCALED): FP64
// scales each value read, FP32 uses the coefficients times iM.
template <class Op>
static void set_scaled_coef(const Ctx *c, Op &o) {
	typedef decltype(o.ka) T;
	const double iM = 1.0 / c->k.a;
	o.ka = (T)c->k.a;
	o.kb = (T)c->k.b;
	o.kc = (T)c->k.c;
	o.iMc = (T)iM;
	o.kas = (T)(c->k.a * iM);
	o.kbs = (T)(c->k.b * iM);
	o.kcs = (T)(c->k.c * iM);
}

// BiCGStab sweeps 2 and 3 in the form of B->acfg: ring, or s written over v
// (slot 1) in the stage; r (slot 0) stays for the lanes that keep it.
template <class T, int RBT, bool PAIRS, class Op>
static void launch_bicg_s(Ctx *c, Batched *B, const Op &o, cudaStream_t s) {
	switch (B->acfg) {
	case 2: launchT<T, RBT, PAIRS>(c, B, InPlace<Op, 2>(o), s); break;
	case 3: launchT<T, RBT, PAIRS>(c, B, InPlace<Op, 3>(o), s); break;
	default: launchT<T, RBT, PAIRS>(c, B, o, s);
	}
}

// BiCGStab sweep 1 (three stencil sources) in form 3: p written over p_old
// (slot 1) in the stage, on its own 32x16 tiles with six stages instead of
// five and a ring.
template <class T, int RBT, bool PAIRS>
static void launch_bicg_1(Ctx *c, Batched *B, const OpBicg1<T> &o, cudaStream_t s) {
	if (B->acfg == 3) launchT<T, RBT, PAIRS>(c, B, InPlace<OpBicg1<T>, 0>(o), s);
	else launchT<T, RBT, PAIRS>(c, B, o, s);
}

template <class T, int RBT, int RBD, bool PAIRS = false>
static void enqueue_bicg_iteration(Ctx *c, Batched *B) {
	cudaStream_t s = c->stream;
	OpBicg1<T> o1;
	set_scaled_coef(c, o1);
	o1.p0 = (T *)B->p0;
	o1.p1 = (T *)B->p1;
	o1.v0 = (T *)B->v[0];
	o1.v1 = (T *)B->v[1];
	o1.rhat = (T *)B->rhat;
	launch_bicg_1<T, RBT, PAIRS>(c, B, o1, s);
	OpBicg2<T> o2;
	set_scaled_coef(c, o2);
	launch_bicg_s<T, RBT, PAIRS>(c, B, o2, s);
	OpBicg3<T> o3;
	set_scaled_coef(c, o3);
	o3.x = (T *)B->x;
	o3.r0 = (T *)B->r;
	o3.r1 = (T *)B->r1;
	o3.p0 = (T *)B->p0;
	o3.p1 = (T *)B->p1;
	o3.rhat = (T *)B->rhat;
	o3.mixed = B->mixed ? 1 : 0;
	launch_bicg_s<T, RBT, PAIRS>(c, B, o3, s);
	if (B->mixed) {
		// Reliable update: x_hi += x_lo; r = b - A x_hi (FP64) into the r buffer
		// the next iteration reads; rho = <r, r_hat> (restarted lanes: r_hat = r).
		const long long nb = ((long long)B->elems / 2 + 255) / 256;
		kb_ru_fold<<<(int)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(c->g.n, B->R, B->rbD, B->rbT, B->xh,
		                                                                 (float *)B->x, nullptr, B->ls.xa, B->ls.pending,
		                                                                 B->ks == 3 ? 1 : 0, B->gl);
		c->launches++;
		enqueue_resid<RBD, PAIRS>(c, B, true);
		kb_ru_done<<<1, 1, 0, s>>>(B->gl);
		c->launches++;
	}
}

// Per-configuration driver pieces, bound to the context at allocation.
// setup: r = b - A x for a batch already in b (and x / x_hi), per-lane <b,b>,
// <r,r> and the initial stop test, all on the stream (no host round trip:
// the setup sweep runs under a +1 guard on `active` that kb_setup_done drops).
// chunk: one launch of the captured graph of `chunk` iterations; lanes and
// launches past the stop are no-ops.
template <class T, int RBT, int RBD, bool PAIRS = false>
struct Impl {
	static int setup(Ctx *c, Batched *B, int nrhs, int maxiter, double tol) {
		cudaStream_t s = c->stream;
		Global g0 = {};
		g0.iter = 1;
		g0.maxiter = maxiter;
		g0.tol = tol;
		g0.tol_in = B->mixed ? B->theta * tol : tol;
		g0.period = B->period;
		g0.nrhs = nrhs;
		g0.active = 1;
		*B->g0_host = g0;  // read by the copy below; rewritten only after this batch is over
		BTRY(cudaMemcpyAsync(B->gl, B->g0_host, sizeof(Global), cudaMemcpyHostToDevice, s));
		enqueue_resid<RBD, PAIRS>(c, B, false);
		kb_setup_done<<<1, 1, 0, s>>>(B->gl);
		c->launches++;
		if (B->ks == 3) enqueue_pcg_uw<T, RBT, PAIRS>(c, B, 1, 0);  // :138-149 (skipped when no lane is live)
		BTRY(cudaGetLastError());
		return 0;
	}
	static int chunk(Ctx *c, Batched *B) {
		cudaStream_t s = c->stream;
		if (!B->graph) {
			// The graph reads tol/maxiter/iteration only from Global (device): reusable.
			cudaGraph_t graph;
			const long long before = c->launches;
			BTRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
			for (int i = 0; i < B->chunk; i++) {
				if (B->ks == 3) enqueue_pcg_iteration<T, RBT, RBD, PAIRS>(c, B);
				else if (B->ks == 1) enqueue_bicg_iteration<T, RBT, RBD, PAIRS>(c, B);
				else enqueue_cg_iteration<T, RBT, RBD, PAIRS>(c, B);
			}
			if (B->defer_x && !B->mixed) {  // the mixed form folds pending steps in its reliable update
				const long long npts = PAIRS ? c->g.n / 2 : c->g.n;
				const long long nb = ((long long)B->elems + 255) / 256;
				kb_x_flush<T><<<(int)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, s>>>(npts, B->R, RBT, (T *)B->x,
				                                                                    (const T *)B->p1, B->ls.xa, B->gl);
				kb_x_flush_done<<<1, 1, 0, s>>>(B->gl);
				c->launches += 2;
			}
			BTRY(cudaStreamEndCapture(s, &graph));
			B->graph_kernels = c->launches - before;
			c->launches = before;
			cudaError_t e = cudaGraphInstantiate(&B->graph, graph, 0);
			cudaGraphDestroy(graph);
			if (e != cudaSuccess) {
				B->graph = nullptr;
				return set_cuda_error(c, e, "cudaGraphInstantiate");
			}
		}
		BTRY(cudaGraphLaunch(B->graph, s));
		c->launches += B->graph_kernels;
		return 0;
	}
};

static void bind_impl(Batched *B) {
	if (B->mixed) {  // FP64 fields in slices of mixed_slice_fp64 lanes
		if (B->rbT == 4 && B->rbD == 4) {
			B->setup_fn = Impl<float, 4, 4>::setup;
			B->chunk_fn = Impl<float, 4, 4>::chunk;
		} else if (B->rbT == 4) {
			B->setup_fn = Impl<float, 4, 8>::setup;
			B->chunk_fn = Impl<float, 4, 8>::chunk;
		} else {
			B->setup_fn = Impl<float, 8, 8>::setup;
			B->chunk_fn = Impl<float, 8, 8>::chunk;
		}
		return;
	}
	switch (B->rbT) {
	case 2:
		B->setup_fn = Impl<double, 2, 2>::setup;
		B->chunk_fn = Impl<double, 2, 2>::chunk;
		break;
	case 4:
		B->setup_fn = Impl<double, 4, 4>::setup;
		B->chunk_fn = Impl<double, 4, 4>::chunk;
		break;
	default:
		B->setup_fn = Impl<double, 8, 8>::setup;
		B->chunk_fn = Impl<double, 8, 8>::chunk;
	}
}

constexpr long long kPairsMinPoints = 1LL << 22;  // smallest grid of the streaming single-vector form

// Single-vector FP64 form on the streaming sweeps.  A dense vector with n1
// even is the 2-lane sliced layout of the (n1/2, n2, n3) grid: lane 0 holds
// the even i1 points, lane 1 the odd ones, so the sweeps of the batched FP64
// form run on the context's own vectors (aliased, nothing copied), with the
// stencil's i1 neighbours taken across each pair and the two lanes' sums
// added into one dot product (Cfg::PAIRS).  Elementwise values round as the
// reference's, as in the batched FP64 form.  Odd n1, and solves with a
// vector iM, use the context's march kernels (plain.cu).
int pairs_alloc(Ctx *c) {
	c->pairs = nullptr;
	// Small grids stay on the march kernels: below about 4M points the
	// single-vector working set sits in the 126 MB L2 and a plane-streaming
	// block gets too few planes (128^3 CG: 34 probe-solves/s streaming, 43
	// marching; 256^3: 4.1 against 2.2).
	if (c->g.n1 % 2 != 0 || c->g.n < kPairsMinPoints || !encode_fn()) return 0;
	Batched *B = new (std::nothrow) Batched();
	if (!B) return SEDI_ERR_NOMEM;
	B->pairs = B->aliased = true;
	B->ks = c->solver;
	B->defer_x = SEDI_DEFER_X && B->ks == SEDI_CG;
	B->R = 2;
	B->rbT = B->rbD = 2;
	B->elems = (size_t)c->g.n;
	Geo g = c->g;
	g.n1 = c->g.n1 / 2;
	g.n = c->g.n / 2;
	B->x = c->x;
	B->b = c->b;
	B->r = c->r;
	B->p0 = c->p[0];
	B->p1 = c->p[1];
	B->w[0] = c->w[0];
	B->w[1] = c->w[1];
	B->u = c->u;
	B->q = c->q;
	B->sv = c->s;
	B->z = c->z;
	B->r1 = c->u;  // BiCGStab's second r buffer (it has no u)
	B->v[0] = c->v[0];
	B->v[1] = c->v[1];
	B->rhat = c->rhat;
	// A tuning recorded for this solver, FP64 and one right-hand side (no
	// batched context has that key) sets the i3 split, the prefetch distance
	// and the narrow-sweep form.
	const Tuning tu = tuning_for(TuneKey{c->solver, SEDI_PREC_FP64, pick_R(1, false), c->g.n1, c->g.n2, c->g.n3});
	B->acfg = tu.acfg >= 1 && tu.acfg <= 3 ? tu.acfg : default_form(B->ks, true);
	B->tuned = tu;
	shape(g, 2, 2, 8, &B->gT, &B->gridT, tu.nz, 0, tu.pfd);
	shape(g, 2, 2, 8, &B->gT1, &B->gridT1, tu.nz, 1, tu.pfd);
	shape(g, 2, 2, 8, &B->gD, &B->gridD, tu.nz, 0, tu.pfd);
	size_t nblk = (size_t)B->gridT.x * B->gridT.z;
	if ((size_t)B->gridT1.x * B->gridT1.z > nblk) nblk = (size_t)B->gridT1.x * B->gridT1.z;
	if (cudaMalloc(&B->partials, sizeof(double) * nblk * kMaxDots * B->R) != cudaSuccess ||
	    cudaMalloc(&B->ticket, sizeof(unsigned)) != cudaSuccess || cudaMalloc(&B->gl, sizeof(Global)) != cudaSuccess ||
	    cudaMallocHost(&B->gl_host, 2 * sizeof(Global)) != cudaSuccess ||
	    cudaMallocHost(&B->lane_host, sizeof(double) * kLaneDoubles * B->R) != cudaSuccess ||
	    cudaMallocHost(&B->lane_host_int, sizeof(int) * kLaneInts * B->R) != cudaSuccess ||
	    cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming) != cudaSuccess ||
	    cudaMalloc(&B->lane_mem, sizeof(double) * kLaneDoubles * B->R) != cudaSuccess ||
	    cudaMalloc(&B->lane_int, sizeof(int) * kLaneInts * B->R) != cudaSuccess) {
		cudaGetLastError();
		free_batched(B);
		c->error = "device allocation failed (single-vector sweeps)";
		return SEDI_ERR_NOMEM;
	}
	cudaMemsetAsync(B->ticket, 0, sizeof(unsigned), c->stream);
	cudaMemsetAsync(B->lane_mem, 0, sizeof(double) * kLaneDoubles * B->R, c->stream);
	cudaMemsetAsync(B->lane_int, 0, sizeof(int) * kLaneInts * B->R, c->stream);
	LaneState &ls = B->ls;
	double **dp[] = {&ls.bb, &ls.rr, &ls.err, &ls.ru, &ls.ru_new, &ls.sp, &ls.alpha, &ls.beta, &ls.gamma,
	                 &ls.gamma_old, &ls.delta, &ls.rr_top, &ls.rho, &ls.rho_prev, &ls.omega, &ls.s_norm2, &ls.ts,
	                 &ls.tt, &ls.xa};
	for (size_t i = 0; i < sizeof(dp) / sizeof(dp[0]); i++) *dp[i] = B->lane_mem + i * B->R;
	int **ip[] = {&ls.done, &ls.exit_iter, &ls.reason, &ls.pending, &ls.s_exit};
	for (size_t i = 0; i < 5; i++) *ip[i] = B->lane_int + i * B->R;
	ls.hist = nullptr;
	auto t_maps = [&](Maps &M, int kind) {
		int Q1, Q2;
		tile_for(2, 8, &Q1, &Q2, kind);
		bool k = make_map(&M.m[MT_R_HALO], B->r, 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_P0_HALO], B->p0, 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_P1_HALO], B->p1, 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
		         make_map(&M.m[MT_X_INT], B->x, 8, g, 2, 2, Q1, Q2) &&
		         make_map(&M.m[MT_R_INT], B->r, 8, g, 2, 2, Q1, Q2) &&
		         make_map(&M.m[MT_P1_INT], B->p1, 8, g, 2, 2, Q1, Q2);
		if (B->ks == 3)
			k = k && make_map(&M.m[MT_W0_HALO], B->w[0], 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_W1_HALO], B->w[1], 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_Q_HALO], B->q, 8, g, 2, 2, Q1 + 2, Q2 + 2);
		if (B->ks == 1)
			k = k && make_map(&M.m[MT_R1_HALO], B->r1, 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_V0_HALO], B->v[0], 8, g, 2, 2, Q1 + 2, Q2 + 2) &&
			    make_map(&M.m[MT_V1_HALO], B->v[1], 8, g, 2, 2, Q1 + 2, Q2 + 2);
		return k;
	};
	int P1, P2;
	tile_for(2, 8, &P1, &P2);
	const bool ok = t_maps(B->mapsT, 0) && t_maps(B->mapsT1, 1) &&
	                make_map(&B->mapsD.m[MD_X_HALO], B->x, 8, g, 2, 2, P1 + 2, P2 + 2) &&
	                make_map(&B->mapsD.m[MD_B_INT], B->b, 8, g, 2, 2, P1, P2);
	if (!ok) {
		free_batched(B);
		c->error = "tensor map encoding failed (single-vector sweeps)";
		return SEDI_ERR_CUDA;
	}
	B->g0_host = B->gl_host + 1;
	B->lane_res.assign(B->R, 0);
	B->setup_fn = Impl<double, 2, 2, true>::setup;
	B->chunk_fn = Impl<double, 2, 2, true>::chunk;
	c->pairs = B;
	if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_cuda_error(c, cudaGetLastError(), "pairs_alloc");
	return 0;
}

void pairs_free(Ctx *c) {
	free_batched((Batched *)c->pairs);
	c->pairs = nullptr;
}

static int check_flags(Ctx *c, Batched *B) {
	if (B->gl_host->err) {
		c->error = "batched sweep timed out waiting for its data";
		return SEDI_ERR_CUDA;
	}
	return 0;
}

static long long max_rounds(const Batched *B, int maxiter) { return (long long)maxiter * 2 / B->chunk + 4; }

// Blocking solve of the batch in the context's buffers.
static int run_batched(Ctx *c, Batched *B, int nrhs, int maxiter, double tol) {
	cudaStream_t s = c->stream;
	int rc = B->setup_fn(c, B, nrhs, maxiter, tol);
	if (rc) return rc;
	for (long long rounds = 0;; rounds++) {
		if (rounds > max_rounds(B, maxiter)) {
			c->error = "batched solver did not stop";
			return SEDI_ERR_CUDA;
		}
		if ((rc = B->chunk_fn(c, B))) return rc;
		BTRY(cudaMemcpyAsync(B->gl_host, B->gl, sizeof(Global), cudaMemcpyDeviceToHost, s));
		BTRY(cudaStreamSynchronize(s));
		if ((rc = check_flags(c, B))) return rc;
		if (B->gl_host->active == 0) return 0;
	}
}

// Per-lane scalars the post-loop logic reads.
struct LaneOut {
	int reason, exit_iter;
	double err, bb, s_norm2, omega, rho;
};

// Result per lane with the reference post-loop logic (Cg.hpp:197-206,
// BiCgStab.hpp:234-262; the BiCGStab breakdown branches only in the FP64
// form: MIXED lanes stop on their FP64 true residual or at maxiter).
static int lane_result(const LaneOut &l, bool bicg, double tol, int maxiter, double *fe, int *fi) {
	if (l.reason == STOP_EARLY) {
		*fi = 0;
		*fe = l.err;
		return 0;
	}
	if (l.err <= tol) {
		// A mixed lane that met tol but not its tighter in-loop target by
		// maxiter still has a solution in the reference's sense.
		*fi = l.reason == STOP_MAXITER ? maxiter : l.exit_iter;
		*fe = l.err;
		return 0;
	}
	if (bicg) {
		if (l.s_norm2 <= tol * tol) {
			*fi = l.exit_iter;
			*fe = std::sqrt(l.s_norm2 / l.bb);
			return 0;
		}
		if (l.omega == 0.0) {
			*fi = l.exit_iter;
			*fe = l.err;
			return 3;
		}
		if (l.rho == 0.0) {
			*fi = l.exit_iter;
			*fe = l.err;
			return 2;
		}
	}
	*fi = maxiter;
	*fe = l.err;
	return 1;
}


// Copies the per-lane state to the pinned mirror (stream-ordered).
static int enqueue_lane_copy(Ctx *c, Batched *B) {
	const int R = B->R;
	BTRY(cudaMemcpyAsync(B->lane_host, B->lane_mem, sizeof(double) * kLaneDoubles * R, cudaMemcpyDeviceToHost,
	                     c->stream));
	BTRY(cudaMemcpyAsync(B->lane_host_int, B->lane_int, sizeof(int) * kLaneInts * R, cudaMemcpyDeviceToHost,
	                     c->stream));
	return 0;
}

// Per-lane results from the pinned mirror (after enqueue_lane_copy completed).
static int process_lanes(Ctx *c, Batched *B, int nrhs, int maxiter, double tol, double *final_err, int *final_iter,
                         int *results) {
	const int R = B->R;
	const double *lm = B->lane_host;
	const int *lint = B->lane_host_int;
	auto at = [&](const double *dev, int j) { return lm[(size_t)(dev - B->lane_mem) + j]; };
	const bool bicg = B->ks == 1 && !B->mixed;
	int worst = 0;
	for (int j = 0; j < nrhs; j++) {
		LaneOut l;
		l.reason = lint[2 * R + j];
		l.exit_iter = lint[1 * R + j];
		l.err = at(B->ls.err, j);
		l.bb = at(B->ls.bb, j);
		l.s_norm2 = at(B->ls.s_norm2, j);
		l.omega = at(B->ls.omega, j);
		l.rho = at(B->ls.rho, j);
		double fe;
		int fi;
		const int res = lane_result(l, bicg, tol, maxiter, &fe, &fi);
		if (final_err) final_err[j] = fe;
		if (final_iter) final_iter[j] = fi;
		if (results) results[j] = res;
		if (res > worst) worst = res;
	}
	return worst;
}

static int batched_run_resident(Ctx *c, int nrhs, int maxiter, double tol, double *final_err, int *final_iter,
                                int *results) {
	Batched *B = (Batched *)c->batched;
	int rc = run_batched(c, B, nrhs, maxiter, tol);
	if (rc) return rc;
	if ((rc = enqueue_lane_copy(c, B))) return rc;
	BTRY(cudaStreamSynchronize(c->stream));
	return process_lanes(c, B, nrhs, maxiter, tol, final_err, final_iter, results);
}

// Single-vector solve on the streaming sweeps: b and x (the initial guess)
// already in the context's vectors; the history of errors is written into
// c->hist as the single-vector kernels do.
int pairs_solve_resident(Ctx *c, int maxiter, double tol, double *final_err, int *final_iter) {
	Batched *B = (Batched *)c->pairs;
	B->ls.hist = c->hist;
	if (B->graph && B->graph_hist != c->hist) {  // the graph holds the old history pointer
		cudaGraphExecDestroy(B->graph);
		B->graph = nullptr;
	}
	int rc = run_batched(c, B, 1, maxiter, tol);
	B->graph_hist = c->hist;
	if (rc) return rc;
	if ((rc = enqueue_lane_copy(c, B))) return rc;
	BTRY(cudaStreamSynchronize(c->stream));
	int res = 0;
	process_lanes(c, B, 1, maxiter, tol, final_err, final_iter, &res);
	// Entries of the history: the initial err plus one per iteration that
	// printed its err (the s-norm exit and the rho breakdown leave before).
	const int reason = B->lane_host_int[2 * B->R], ex = B->lane_host_int[1 * B->R];
	if (reason == STOP_EARLY) c->hist_len = 1;
	else if (reason == STOP_SNORM || reason == STOP_RHO) c->hist_len = ex;
	else c->hist_len = (ex > maxiter ? maxiter : ex) + 1;
	return res;
}

static int blocks1d(long long n) {
	long long b = (n + 255) / 256;
	return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

int batched_solve_dev(Ctx *c, int nrhs, const double *b, double *x, int maxiter, double tol, double *final_err,
                      int *final_iter, int *results) {
	Batched *B = (Batched *)c->batched;
	if (!B || nrhs < 1 || nrhs > c->batch) {
		c->error = "nrhs outside 1..batch";
		return SEDI_ERR_ARG;
	}
	cudaStream_t s = c->stream;
	const long long n = c->g.n;
	kb_interleave<<<blocks1d(n * B->R), 256, 0, s>>>(n, B->R, B->rbD, nrhs, b, B->b);
	kb_interleave<<<blocks1d(n * B->R), 256, 0, s>>>(n, B->R, B->rbD, nrhs, x, B->mixed ? B->xh : (double *)B->x);
	c->launches += 2;
	int rc = batched_run_resident(c, nrhs, maxiter, tol, final_err, final_iter, results);
	if (rc < 0) return rc;
	kb_deinterleave<<<blocks1d(n * nrhs), 256, 0, s>>>(n, B->rbD, nrhs, B->mixed ? B->xh : (const double *)B->x, x);
	c->launches++;
	BTRY(cudaStreamSynchronize(s));
	return rc;
}

// Per-iteration kernels of the batched CG timed in isolation (see
// sedi_time_kernels): every lane active, no lane stops, no reliable update.
template <class T, int RBT, bool PAIRS = false>
static int time_cg_kernels(Ctx *c, Batched *B, int reps, double *ms, double *bytes, char *names, int *count) {
	cudaStream_t s = c->stream;
	Global g = {};
	g.iter = 2;
	g.active = B->R;
	g.maxiter = 1 << 30;
	g.tol = 0.0;
	g.tol_in = 0.0;
	g.period = 0;
	g.nrhs = B->R;
	*B->gl_host = g;
	BTRY(cudaMemcpyAsync(B->gl, B->gl_host, sizeof(Global), cudaMemcpyHostToDevice, s));
	BTRY(cudaMemsetAsync(B->ls.done, 0, sizeof(int) * B->R, s));
	BTRY(cudaMemsetAsync(B->lane_mem, 0, sizeof(double) * kLaneDoubles * B->R, s));
	OpCgA<T> a;
	a.ka = (T)c->k.a;
	a.kb = (T)c->k.b;
	a.kc = (T)c->k.c;
	a.iMc = (T)(1.0 / c->k.a);
	a.p0 = (T *)B->p0;
	a.p1 = (T *)B->p1;
	a.mixed = 0;
	OpCgB<T> bo;
	bo.ka = (T)c->k.a;
	bo.kb = (T)c->k.b;
	bo.kc = (T)c->k.c;
	bo.iMc = (T)(1.0 / c->k.a);
	bo.x = (T *)B->x;
	bo.r = (T *)B->r;
	bo.mixed = 0;
	cudaEvent_t e0, e1;
	BTRY(cudaEventCreate(&e0));
	BTRY(cudaEventCreate(&e1));
	const double ts = (double)sizeof(T) * (double)B->elems;
	if (B->ks == 3) {
		OpPcg<T> o;
		o.ka = (T)c->k.a;
		o.kb = (T)c->k.b;
		o.kc = (T)c->k.c;
		o.iMc = (T)(1.0 / c->k.a);
		o.x = (T *)B->x;
		o.r = (T *)B->r;
		o.u = (T *)B->u;
		o.q = (T *)B->q;
		o.s = (T *)B->sv;
		o.p = (T *)B->p0;
		o.z = (T *)B->z;
		o.w0 = (T *)B->w[0];
		o.w1 = (T *)B->w[1];
		o.mixed = 0;
		launchT<T, RBT, PAIRS>(c, B, o, s);
		BTRY(cudaEventRecord(e0, s));
		for (int i = 0; i < reps; i++) launchT<T, RBT, PAIRS>(c, B, o, s);
		BTRY(cudaEventRecord(e1, s));
		BTRY(cudaEventSynchronize(e1));
		float t = 0.f;
		BTRY(cudaEventElapsedTime(&t, e0, e1));
		ms[0] = (double)t / reps;
		bytes[0] = 16.0 * ts;  // w, q, s, p, z, r, x, u in and out
		snprintf(names, 32, "%s%s", B->mixed ? "pcg_fp32" : "pcg_fp64", PAIRS ? "_sv" : "");
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		*count = 1;
		BTRY(cudaGetLastError());
		return 0;
	}
	if (B->ks == 1) {
		OpBicg1<T> o1;
		set_scaled_coef(c, o1);
		o1.p0 = (T *)B->p0;
		o1.p1 = (T *)B->p1;
		o1.v0 = (T *)B->v[0];
		o1.v1 = (T *)B->v[1];
		o1.rhat = (T *)B->rhat;
		OpBicg2<T> o2;
		set_scaled_coef(c, o2);
		OpBicg3<T> o3;
		set_scaled_coef(c, o3);
		o3.x = (T *)B->x;
		o3.r0 = (T *)B->r;
		o3.r1 = (T *)B->r1;
		o3.p0 = (T *)B->p0;
		o3.p1 = (T *)B->p1;
		o3.rhat = (T *)B->rhat;
		o3.mixed = 0;
		// Lanes run the full update (no early exit) with zero scalars.
		BTRY(cudaMemsetAsync(B->ls.s_exit, 0, sizeof(int) * B->R, s));
		const char *nm[3] = {"bicg_1", "bicg_2", "bicg_3"};
		const double words[3] = {6.0, 2.0, 7.0};  // 1: r, p, v, r_hat in, p, v out; 2: r, v in;
		                                          // 3: r, v, x, p, r_hat in, x, r out
		for (int k = 0; k < 3; k++) {
			auto one = [&]() {
				if (k == 0) launch_bicg_1<T, RBT, PAIRS>(c, B, o1, s);
				else if (k == 1) launch_bicg_s<T, RBT, PAIRS>(c, B, o2, s);
				else launch_bicg_s<T, RBT, PAIRS>(c, B, o3, s);
			};
			one();
			BTRY(cudaEventRecord(e0, s));
			for (int i = 0; i < reps; i++) one();
			BTRY(cudaEventRecord(e1, s));
			BTRY(cudaEventSynchronize(e1));
			float t = 0.f;
			BTRY(cudaEventElapsedTime(&t, e0, e1));
			ms[k] = (double)t / reps;
			bytes[k] = words[k] * ts;
			snprintf(names + 32 * k, 32, "%s_%s%s", nm[k], B->mixed ? "fp32" : "fp64", PAIRS ? "_sv" : "");
		}
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		*count = 3;
		BTRY(cudaGetLastError());
		return 0;
	}
	// With the deferred x step, sweep B runs as cg_b (odd iterations: r only)
	// and cg_bx (even: both x steps); each is timed on its own parity.
	const int nk = B->defer_x ? 3 : 2;
	for (int k = 0; k < nk; k++) {
		if (B->defer_x) {
			// Each form on its own parity; ru_due holds the counter (no advance).
			g.iter = g.b_iter = k == 1 ? 3 : 2;
			g.ru_due = 1;
			*B->gl_host = g;
			BTRY(cudaMemcpyAsync(B->gl, B->gl_host, sizeof(Global), cudaMemcpyHostToDevice, s));
		}
		auto one = [&]() {
			if (k == 0) launch_cg_a<T, RBT, PAIRS>(c, B, a, s);
			else if (!B->defer_x) launchT<T, RBT, PAIRS>(c, B, bo, s);
			else if (k == 1) launchT<T, RBT, PAIRS>(c, B, cg_b_as<XS_R>(bo), s);
			else launchT<T, RBT, PAIRS>(c, B, cg_b_as<XS_X>(bo), s);
		};
		one();
		BTRY(cudaEventRecord(e0, s));
		for (int i = 0; i < reps; i++) one();
		BTRY(cudaEventRecord(e1, s));
		BTRY(cudaEventSynchronize(e1));
		float t = 0.f;
		BTRY(cudaEventElapsedTime(&t, e0, e1));
		ms[k] = (double)t / reps;
		// A: r, p_old in, p out; B: p, x, r in, x, r out; deferred: cg_b p, r in, r out,
		// cg_bx p, p_old, x, r in, x, r out.
		const double words = k == 0 ? 3.0 : (!B->defer_x ? 5.0 : (k == 1 ? 3.0 : 6.0));
		bytes[k] = words * ts;
		const char *nm = k == 0 ? "cg_a" : (k == 1 ? "cg_b" : "cg_bx");
		snprintf(names + 32 * k, 32, "%s_%s%s", nm, B->mixed ? "fp32" : "fp64", PAIRS ? "_sv" : "");
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	BTRY(cudaGetLastError());
	if (B->gl_host && cudaMemcpyAsync(B->gl_host, B->gl, sizeof(Global), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
	    cudaStreamSynchronize(s) == cudaSuccess && B->gl_host->err) {
		c->error = "batched sweep timed out waiting for its data";
		return SEDI_ERR_CUDA;
	}
	*count = nk;
	return 0;
}

// Single-vector form: its streaming sweeps timed alone (names end in _sv).
int pairs_time_kernels(Ctx *c, int reps, double *ms, double *bytes, char *names, int *count) {
	Batched *B = (Batched *)c->pairs;
	if (!B) return SEDI_ERR_UNSUPPORTED;
	return time_cg_kernels<double, 2, true>(c, B, reps, ms, bytes, names, count);
}

int batched_time_kernels(Ctx *c, int reps, double *ms, double *bytes, char *names, int *count) {
	Batched *B = (Batched *)c->batched;
	if (B->mixed) {
		switch (B->rbT) {
		case 4: return time_cg_kernels<float, 4>(c, B, reps, ms, bytes, names, count);
		default: return time_cg_kernels<float, 8>(c, B, reps, ms, bytes, names, count);
		}
	}
	switch (B->rbT) {
	case 2: return time_cg_kernels<double, 2>(c, B, reps, ms, bytes, names, count);
	case 4: return time_cg_kernels<double, 4>(c, B, reps, ms, bytes, names, count);
	default: return time_cg_kernels<double, 8>(c, B, reps, ms, bytes, names, count);
	}
}

int batched_estimate_dev(Ctx *c, int samples, const double *probes_dev, int maxiter, double tol, int ignore_errors,
                         double *D_dev, double *t_dev, double *q_dev, int *iters, double *errs, int *results) {
	return batched_estimate_src(c, samples, probes_dev, 0u, maxiter, tol, ignore_errors, D_dev, t_dev, q_dev, iters,
	                            errs, results);
}

// Starts the next batch of probes: fill (device generator or caller probes),
// x = 0 (:175), setup, first chunk, status copy, event.
static int est_start_batch(Ctx *c, Batched *B) {
	EstState &E = B->est;
	cudaStream_t s = c->stream;
	const long long n = c->g.n;
	E.nb = E.samples - E.k0 < c->batch ? E.samples - E.k0 : c->batch;
	if (E.probes_dev) {
		kb_interleave<<<blocks1d(n * B->R), 256, 0, s>>>(n, B->R, B->rbD, E.nb, E.probes_dev + (size_t)E.k0 * n, B->b);
	} else {
		if (E.nb < B->R) BTRY(cudaMemsetAsync(B->b, 0, B->elems * sizeof(double), s));  // padding lanes
		if (device_fill_probes(E.seed + (uint32_t)E.k0, E.nb, n, B->rbD, B->b, s))
			return set_cuda_error(c, cudaGetLastError(), "device probes");
	}
	c->launches++;
	BTRY(cudaMemsetAsync(B->mixed ? (void *)B->xh : B->x, 0, B->elems * sizeof(double), s));  // x = 0 (:175)
	int rc = B->setup_fn(c, B, E.nb, E.maxiter, E.tol);
	if (!rc) rc = B->chunk_fn(c, B);
	if (rc) return rc;
	BTRY(cudaMemcpyAsync(B->gl_host, B->gl, sizeof(Global), cudaMemcpyDeviceToHost, s));
	BTRY(cudaEventRecord(B->ev, s));
	E.rounds = 0;
	E.stage = EST_SOLVE;
	return 0;
}

// D = t / q and the result copies.
static int est_final(Ctx *c, Batched *B) {
	EstState &E = B->est;
	cudaStream_t s = c->stream;
	const long long n = c->g.n;
	if (E.samples == 0) {
		BTRY(cudaMemsetAsync(B->t_acc, 0, sizeof(double) * n, s));
		BTRY(cudaMemsetAsync(B->q_acc, 0, sizeof(double) * n, s));
	}
	if (E.t_dev) BTRY(cudaMemcpyAsync(E.t_dev, B->t_acc, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
	if (E.q_dev) BTRY(cudaMemcpyAsync(E.q_dev, B->q_acc, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
	kb_divide<<<blocks1d(n), 256, 0, s>>>(n, B->t_acc, B->q_acc, E.D_dev);  // :216 (D_dev may alias t_acc)
	c->launches++;
	if (E.D_host) BTRY(cudaMemcpyAsync(E.D_host, E.D_dev, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
	BTRY(cudaEventRecord(B->ev, s));
	E.stage = EST_FINAL;
	return 0;
}

int batched_est_begin(Ctx *c, int samples, const double *probes_dev, uint32_t seed, int maxiter, double tol,
                      int ignore_errors, double *D_dev, double *t_dev, double *q_dev, double *D_host, int *iters,
                      double *errs, int *results) {
	Batched *B = (Batched *)c->batched;
	if (B->est.stage != EST_IDLE && B->est.stage != EST_DONE) {
		c->error = "an estimate is already running on this context";
		return SEDI_ERR_ARG;
	}
	EstState &E = B->est;
	E = EstState();
	E.samples = samples;
	E.probes_dev = probes_dev;
	E.seed = seed;
	E.maxiter = maxiter;
	E.tol = tol;
	E.ignore_errors = ignore_errors;
	E.D_dev = D_dev ? D_dev : B->t_acc;
	E.t_dev = t_dev;
	E.q_dev = q_dev;
	E.D_host = D_host;
	E.iters = iters;
	E.errs = errs;
	E.results = results;
	int rc = samples > 0 ? est_start_batch(c, B) : est_final(c, B);
	if (rc) E.stage = EST_DONE, E.rc = rc;
	return rc;
}

// Advances the estimate without blocking: *done = 1 once D (and D_host) are
// ready, with the result code in the return value's place of the blocking
// call available through batched_est_result.
int batched_est_advance(Ctx *c, int *done) {
	Batched *B = (Batched *)c->batched;
	EstState &E = B->est;
	*done = 0;
	if (E.stage == EST_DONE || E.stage == EST_IDLE) {
		*done = 1;
		return E.rc < 0 ? E.rc : 0;
	}
	const cudaError_t q = cudaEventQuery(B->ev);
	if (q == cudaErrorNotReady) return 0;
	int rc = 0;
	if (q != cudaSuccess) rc = set_cuda_error(c, q, "estimate");
	cudaStream_t s = c->stream;
	const long long n = c->g.n;
	if (!rc) switch (E.stage) {
	case EST_SOLVE:
		if ((rc = check_flags(c, B))) break;
		if (B->gl_host->active > 0) {
			if (++E.rounds > max_rounds(B, E.maxiter)) {
				c->error = "batched solver did not stop";
				rc = SEDI_ERR_CUDA;
				break;
			}
			if ((rc = B->chunk_fn(c, B))) break;
			if (cudaMemcpyAsync(B->gl_host, B->gl, sizeof(Global), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
			    cudaEventRecord(B->ev, s) != cudaSuccess)
				rc = set_cuda_error(c, cudaGetLastError(), "estimate");
			break;
		}
		// Batch solved: lane results and t += x.*v, q += v.*v (:195, :198).
		if ((rc = enqueue_lane_copy(c, B))) break;
		kb_accumulate<<<blocks1d(n), 256, 0, s>>>(n, B->rbD, E.nb, B->mixed ? B->xh : (const double *)B->x, B->b,
		                                          B->t_acc, B->q_acc, E.first);
		c->launches++;
		E.first = false;
		if (cudaEventRecord(B->ev, s) != cudaSuccess) rc = set_cuda_error(c, cudaGetLastError(), "estimate");
		E.stage = EST_LANES;
		break;
	case EST_LANES: {
		const int k0 = E.k0;
		const int w = process_lanes(c, B, E.nb, E.maxiter, E.tol, E.errs ? E.errs + k0 : nullptr,
		                            E.iters ? E.iters + k0 : nullptr, B->lane_res.data());
		if (E.results) std::memcpy(E.results + k0, B->lane_res.data(), sizeof(int) * E.nb);
		if (w > E.worst) E.worst = w;
		if (w != 0 && !E.ignore_errors) {  // :181-184: the first failing probe's code, no D
			for (int j = 0; j < E.nb; j++)
				if (B->lane_res[j] != 0) {
					E.rc = B->lane_res[j];
					break;
				}
			E.stage = EST_DONE;
			*done = 1;
			return 0;
		}
		E.k0 += E.nb;
		rc = E.k0 < E.samples ? est_start_batch(c, B) : est_final(c, B);
		break;
	}
	case EST_FINAL:
		E.rc = E.worst;
		E.stage = EST_DONE;
		*done = 1;
		return 0;
	default:
		break;
	}
	if (rc) {
		E.rc = rc;
		E.stage = EST_DONE;
		*done = 1;
	}
	return rc;
}

int batched_est_result(const Ctx *c) {
	const Batched *B = (const Batched *)c->batched;
	return B ? B->est.rc : SEDI_ERR_ARG;
}

// Blocking estimator: probes from device memory (probes_dev) or, when
// probes_dev is NULL, from the device generator (probe k = std::mt19937(seed
// + k)), written straight into the lane-sliced right-hand-side buffer.
int batched_estimate_src(Ctx *c, int samples, const double *probes_dev, uint32_t seed, int maxiter, double tol,
                         int ignore_errors, double *D_dev, double *t_dev, double *q_dev, int *iters, double *errs,
                         int *results) {
	Batched *B = (Batched *)c->batched;
	int rc = batched_est_begin(c, samples, probes_dev, seed, maxiter, tol, ignore_errors, D_dev, t_dev, q_dev,
	                           nullptr, iters, errs, results);
	if (rc) return rc;
	for (;;) {
		BTRY(cudaEventSynchronize(B->ev));
		int done = 0;
		if ((rc = batched_est_advance(c, &done))) return rc;
		if (done) break;
	}
	BTRY(cudaStreamSynchronize(c->stream));
	return B->est.rc;
}

}  // namespace sedi

namespace sedi {

// ---------------------------------------------------------------------------
// Autotuner.  For one (solver, precision, lanes, grid):
//   1. lane-slice width W of the Krylov fields (FP32: 8 or 4 lanes; FP64: 8,
//      4 or 2), each on a scratch context with the model's i3 split, scored
//      by the sweep time of one iteration (CUDA events, kernels alone; CG's
//      two parity forms of sweep B count half each);
//   2. the i3 split of the sweeps (the model's choice and 1, 2, 3, 4, 6, 8
//      chunks) with the best W, same score;
//   3. with flags & 1: iterations per captured graph (8, 16, 32) and, for the
//      mixed form, the reliable-update period (20, 32, 50), each scored by the
//      wall time of a real estimate of `batch` seeded probes to tol.
// The winner is recorded in the process-wide table that context creation
// reads, so contexts created afterwards (and the server's admission sizes)
// use it.  out[0..3] = W, nz (0: model), period, chunk; *score_ms = the best
// step-3 estimate time (or the step-2 sweep time without flags & 1).
// ---------------------------------------------------------------------------
static int tune_sweep_ms(sedi_ctx *h, double *ms_sum) {
	double ms[8], by[8];
	char names[8 * 32];
	int cnt = 0;
	Ctx *c = &h->c;
	const int rc = c->batched ? batched_time_kernels(c, 5, ms, by, names, &cnt)
	                          : (c->pairs ? pairs_time_kernels(c, 10, ms, by, names, &cnt) : SEDI_ERR_UNSUPPORTED);
	if (rc) return rc;
	// Time per iteration: the two parity forms of CG sweep B (cg_b, cg_bx)
	// each run every other iteration.
	bool deferred = false;
	for (int k = 0; k < cnt; k++) deferred = deferred || strncmp(names + 32 * k, "cg_bx", 5) == 0;
	*ms_sum = 0.0;
	for (int k = 0; k < cnt; k++)
		*ms_sum += (deferred && strncmp(names + 32 * k, "cg_b", 4) == 0) ? 0.5 * ms[k] : ms[k];
	return 0;
}

int batched_autotune(int solver, int precision, int batch, long long n1, long long n2, long long n3, int maxiter,
                     double tol, uint32_t seed, int flags, int *out, double *score_ms) {
	const bool mixed = precision == SEDI_PREC_MIXED;
	// One FP64 right-hand side is the single-vector form: its streaming sweeps
	// (even n1, 2^22 points or more) take the i3 split, prefetch distance and
	// narrow-sweep form; the slice width is fixed and there is no graph or
	// reliable-update choice.
	const bool single = batch < 2 && !mixed;
	if (single && (n1 % 2 != 0 || n1 * n2 * n3 < kPairsMinPoints)) return SEDI_ERR_UNSUPPORTED;
	if (single) flags &= ~1;
	const int R = pick_R(batch, mixed);
	const TuneKey key{solver, precision, R, n1, n2, n3};
	std::vector<int> Ws;
	if (single) {
		Ws.push_back(2);
	} else if (R >= 8) {
		Ws.push_back(8);
		Ws.push_back(4);
		if (!mixed) Ws.push_back(2);
	} else {
		Ws.push_back(slice_for(R, !mixed, kernel_solver(solver, mixed)));
	}
	Tuning best;
	double best_ms = -1.0;
	auto score = [&](const Tuning &t, double *ms) -> int {
		set_tuning(key, t);
		int err = 0;
		sedi_ctx *h = sedi_create(solver, (long)n1, (long)n2, (long)n3, 6.0, 1.0, 1.0, 0, precision, batch, &err);
		if (!h) return err ? err : SEDI_ERR_CUDA;
		const int rc = tune_sweep_ms(h, ms);
		sedi_destroy(h);
		return rc;
	};
	for (int W : Ws) {
		Tuning t;
		t.W = W;
		double ms = 0.0;
		const int rc = score(t, &ms);
		if (rc == SEDI_ERR_NOMEM) continue;
		if (rc) return rc;
		if (best_ms < 0 || ms < best_ms) best_ms = ms, best = t;
	}
	if (best_ms < 0) return SEDI_ERR_NOMEM;
	// i3 splits: a single vector has few tiles per plane, so it tries the
	// splits around whole waves of blocks too.
	std::vector<int> nzs = {1, 2, 3, 4, 6, 8};
	if (single)
		for (int nz : {5, 9, 10, 12, 14, 16, 18, 24, 32}) nzs.push_back(nz);
	for (int nz : nzs) {
		if (nz > n3) continue;
		Tuning t = best;
		t.nz = nz;
		double ms = 0.0;
		const int rc = score(t, &ms);
		if (rc) return rc;
		if (ms < 0.97 * best_ms) best_ms = ms, best = t;  // a clear win over the model's split
	}
	// L2 prefetch distance of the sweeps (planes ahead of the TMA loads).
	const int pfds[] = {0, 2, 4, 8};
	for (int pf : pfds) {
		Tuning t = best;
		t.pfd = pf;
		double ms = 0.0;
		const int rc = score(t, &ms);
		if (rc) return rc;
		if (ms < 0.98 * best_ms) best_ms = ms, best = t;  // a clear win over the default
	}
	// Form of CG's sweep A and BiCGStab's sweeps 2 and 3 (ring, or in place
	// with two blocks per SM or six stages).
	if (kernel_solver(solver, mixed) == SEDI_CG || kernel_solver(solver, mixed) == SEDI_BICGSTAB) {
		for (int ac = 1; ac <= 3; ac++) {
			Tuning t = best;
			t.acfg = ac;
			double ms = 0.0;
			const int rc = score(t, &ms);
			if (rc) return rc;
			if (ms < 0.98 * best_ms || (best.acfg == 0 && ac == default_form(kernel_solver(solver, mixed), single)))
				best_ms = ms, best = t;
		}
	}
	double best_est = -1.0;
	if (flags & 1) {
		set_tuning(key, best);
		int err = 0;
		sedi_ctx *h = sedi_create(solver, (long)n1, (long)n2, (long)n3, 6.0, 1.0, 1.0, 0, precision, batch, &err);
		if (!h) return err ? err : SEDI_ERR_CUDA;
		Ctx *c = &h->c;
		Batched *B = (Batched *)c->batched;
		const long long n = n1 * n2 * n3;
		double *D = nullptr;
		if (cudaMalloc(&D, sizeof(double) * n) != cudaSuccess) {
			cudaGetLastError();
			sedi_destroy(h);
			return SEDI_ERR_NOMEM;
		}
		auto timed = [&](double *ms) -> int {
			const auto t0 = std::chrono::steady_clock::now();
			const int rc = batched_estimate_src(c, batch, nullptr, seed, maxiter, tol, 1, D, nullptr, nullptr,
			                                    nullptr, nullptr, nullptr);
			*ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
			return rc < 0 ? rc : 0;
		};
		const int periods_mixed[] = {20, 32, 50}, period_fp64[] = {B->period};
		const int *periods = mixed ? periods_mixed : period_fp64;
		const int np = mixed ? 3 : 1;
		const int chunks[] = {16, 8, 32};
		int rc = 0;
		for (int ci = 0; ci < 3 && !rc; ci++) {
			if (B->graph) {
				cudaGraphExecDestroy(B->graph);
				B->graph = nullptr;
			}
			B->chunk = chunks[ci];
			for (int pi = 0; pi < np && !rc; pi++) {
				if (ci > 0 && periods[pi] != (best.period ? best.period : B->period)) continue;  // chunks at the best period
				B->period = periods[pi];
				double ms = 0.0;
				if (!B->graph && (rc = timed(&ms))) break;  // warm-up: graph capture for this chunk size
				if ((rc = timed(&ms))) break;
				if (best_est < 0 || ms < best_est) {
					best_est = ms;
					best.period = periods[pi];
					best.chunk = chunks[ci];
				}
			}
		}
		cudaFree(D);
		sedi_destroy(h);
		if (rc) return rc;
	}
	set_tuning(key, best);
	out[0] = best.W;
	out[1] = best.nz;
	out[2] = best.period;
	out[3] = best.chunk;
	out[4] = best.pfd;  // -1: the default distance
	out[5] = best.acfg ? best.acfg : default_form(kernel_solver(solver, mixed), single);
	if (score_ms) *score_ms = best_est >= 0 ? best_est : best_ms;
	return 0;
}

int batched_set_tuning(int solver, int precision, int batch, long long n1, long long n2, long long n3,
                       const int *choice) {
	const bool mixed = precision == SEDI_PREC_MIXED;
	Tuning t;
	t.W = choice[0];
	t.nz = choice[1];
	t.period = choice[2];
	t.chunk = choice[3];
	t.pfd = choice[4];
	t.acfg = choice[5];
	if (t.W < 0 || t.nz < 0 || t.period < 0 || t.chunk < 0 || t.pfd < -1 || t.pfd > 64 || t.acfg < 0 || t.acfg > 3 ||
	    (t.period > 0 && (t.period < 1 || t.period > 1000)) || t.chunk > 256)
		return SEDI_ERR_ARG;
	set_tuning(TuneKey{solver, precision, pick_R(batch, mixed), n1, n2, n3}, t);
	return 0;
}

int batched_config(const Ctx *c, int *out) {
	const Batched *B = (const Batched *)c->batched;
	if (!B) return SEDI_ERR_UNSUPPORTED;
	out[0] = B->rbT;
	out[1] = (int)B->gridT.z;
	out[2] = B->period;
	out[3] = B->chunk;
	out[4] = B->R;
	out[5] = B->gT.pfd;
	out[6] = B->acfg;
	return 0;
}

}  // namespace sedi
