// Slab (i3) domain decomposition of the FP64 solvers: the per-rank kernels.
//
// The reference decomposes the grid into blocks, one per MPI rank, with a
// ghost layer filled by a halo exchange (DomainDecomposition.hpp:51-80,
// CommHalo.hpp:84-181) and computes the stencil on the inner cells while the
// exchange is in flight, then on the border cells (DistrAsyncStencil.hpp:
// 52-100); dot products are local sums plus an allreduce
// (DistrAsyncDotProds.hpp:85-136).  Here the grid is split along i3 only:
// a rank holds a slab of nloc planes stored with one ghost plane on each
// side, [nloc + 2][n2][n1] doubles, i1 fastest, so a halo is one contiguous
// plane (no packing).  Ghost planes at the global boundary stay zero -- the
// reference's zero ghost layer (Cg.hpp:57-62).
//
// Dot products are returned per plane, each summed in a fixed order that
// depends only on n1 and n2 (the plane is cut into kSlabChunks row chunks,
// one block each, then the chunks are added in order), so a plane's partial
// sum is the same whichever rank holds the plane; the host adds the planes
// in global order.  The solution therefore does not depend on the number of
// slabs, bit for bit.  Elementwise values round as the reference's
// (operator by operator, no FMA contraction), like the single-vector form:
// a stencil input the reference stores (u = r .* iM, m = w .* iM, p_hat,
// s_hat) is formed at each neighbour read with the same rounding.
#include "sedi_internal.h"

namespace sedi {

namespace {

constexpr int kSlabThreads = 256;
constexpr int kSlabChunks = 8;  // row chunks per plane (fixed: the summation order depends on it)
constexpr int kSlabDots = 3;    // dot products per plane

struct SlabGeo {
	int n1, n2, nloc;
	long long plane;  // n1 * n2
};

__device__ __forceinline__ void chunk_rows(const SlabGeo &g, int c, int *r0, int *r1) {
	const int per = (g.n2 + kSlabChunks - 1) / kSlabChunks;
	*r0 = c * per;
	*r1 = min(g.n2, *r0 + per);
}

// 7-point stencil at ghosted plane z (1..nloc), row i2, column i1 of the
// slab, applied to f = scale .* src when `scaled` (the stencil input the
// reference stores as a vector), else to src.
__device__ __forceinline__ double slab_stencil(const SlabGeo &g, const Coef &k, const double *__restrict__ src,
                                               bool scaled, double scale, int z, int i2, int i1) {
	const long long i = (long long)z * g.plane + (long long)i2 * g.n1 + i1;
	auto f = [&](long long j) { return scaled ? mul(__ldg(src + j), scale) : __ldg(src + j); };
	const double xc = f(i);
	const double xm1 = i1 > 0 ? f(i - 1) : 0.0;
	const double xm2 = i2 > 0 ? f(i - g.n1) : 0.0;
	const double xm3 = f(i - g.plane);  // ghost plane 0 at the slab's lower side
	const double xp1 = i1 < g.n1 - 1 ? f(i + 1) : 0.0;
	const double xp2 = i2 < g.n2 - 1 ? f(i + g.n1) : 0.0;
	const double xp3 = f(i + g.plane);  // ghost plane nloc+1 at the upper side
	return stencil7(k, xc, xm1, xm2, xm3, xp1, xp2, xp3);
}

// Block-level sum of ND values in a fixed tree; result in thread 0.
template <int ND>
__device__ __forceinline__ void block_total(double (&v)[ND]) {
	__shared__ double sh[kSlabThreads / 32][ND];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	warp_sum<ND>(v);
	if (lane == 0)
#pragma unroll
		for (int d = 0; d < ND; d++) sh[warp][d] = v[d];
	__syncthreads();
	if (threadIdx.x == 0) {
#pragma unroll
		for (int d = 0; d < ND; d++) {
			double s = 0.0;
			for (int w = 0; w < kSlabThreads / 32; w++) s += sh[w][d];
			v[d] = s;
		}
	}
	__syncthreads();
}

enum SlabMode {
	SLAB_SETUP = 0,       // r = b - A src; <b,b>, <r,r>                          (Cg.hpp:112-129)
	SLAB_CG_SP = 1,       // <A src, src> (+ <r, r iM> when first)                (Cg.hpp:152-166)
	SLAB_CG_UPDATE = 2,   // x += alpha src; r -= alpha A src; <r, r iM>, <r,r>   (Cg.hpp:169-182)
	SLAB_APPLY = 3,       // y = A src                                            (Stencil.hpp:38-54)
	SLAB_PCG_SETUP = 4,   // u = r iM, w = A u, q = s = p = z = 0; <r,u>, <w,u>, <r,r>  (PipelinedCg.hpp:138-155)
	SLAB_PCG_ITER = 5,    // m = w iM, n = A m, the eight updates, w' in wn; next <r,u>, <w',u>, <r,r>
	                      //                                                      (PipelinedCg.hpp:155-223)
	SLAB_BICG_P = 6,      // p = r (first) or r + beta p + bo v                   (BiCgStab.hpp:165-173)
	SLAB_BICG_V = 7,      // v = A (p iM); <v, r_hat>                             (BiCgStab.hpp:175-187)
	SLAB_BICG_S = 8,      // s = r - alpha v                                      (BiCgStab.hpp:189)
	SLAB_BICG_T = 9,      // t = A (s iM); <s,s>, <t,s>, <t,t>                    (BiCgStab.hpp:192-212)
	SLAB_BICG_XR = 10,    // x += alpha p iM + omega s iM; r = s - omega t; <r,r>, <r, r_hat>  (:216-224)
	SLAB_BICG_X = 11,     // x += alpha p iM (early exit on s)                    (BiCgStab.hpp:193-199)
	SLAB_CG_P = 12,       // p = r iM (first) or r iM + beta p                    (Cg.hpp:144-147, :188)
	SLAB_MODES = 13
};

__host__ __device__ constexpr bool mode_stencil(int m) { return m <= 5 || m == 7 || m == 9; }
__host__ __device__ constexpr bool mode_scaled(int m) { return m == 4 || m == 5 || m == 7 || m == 9; }
__host__ __device__ constexpr int mode_dots(int m) {
	switch (m) {
	case SLAB_SETUP: case SLAB_CG_SP: case SLAB_CG_UPDATE: case SLAB_BICG_XR: return 2;
	case SLAB_PCG_SETUP: case SLAB_PCG_ITER: case SLAB_BICG_T: return 3;
	case SLAB_BICG_V: return 1;
	default: return 0;
	}
}

template <int MODE>
__global__ void __launch_bounds__(kSlabThreads) k_slab_sweep(SlabGeo g, Coef k, int z_lo, int z_hi,
                                                             sedi_slab_args a, double *chunk_part) {
	const int z = z_lo + (int)blockIdx.y;
	if (z >= z_hi) return;
	const int c = blockIdx.x;
	int r0, r1;
	chunk_rows(g, c, &r0, &r1);
	constexpr int ND = mode_dots(MODE) > 0 ? mode_dots(MODE) : 1;
	double v[ND];
#pragma unroll
	for (int d = 0; d < ND; d++) v[d] = 0.0;
	const double iM = a.iM;
	// Rows of the chunk, each by tpr threads (the smallest power of two >= n1,
	// at most the block), the block's other threads on the next rows.  Not
	// unrolled: these sweeps hide latency with resident warps, and unrolling
	// by 4 cost more in occupancy (registers) than it gained (512^3 CG 55 ->
	// 51, pipelined CG 46 -> 37 GPoint-it/s on B200).
	int tpr = 32;
	while (tpr < g.n1 && tpr < kSlabThreads) tpr <<= 1;
	const int rpi = kSlabThreads / tpr, tc = (int)threadIdx.x % tpr;
	for (int i1 = tc; i1 < g.n1; i1 += tpr) {
#pragma unroll 1
		for (int i2 = r0 + (int)threadIdx.x / tpr; i2 < r1; i2 += rpi) {
			const long long i = (long long)z * g.plane + (long long)i2 * g.n1 + i1;
			double st = 0.0;
			if (mode_stencil(MODE)) st = slab_stencil(g, k, a.src, mode_scaled(MODE), iM, z, i2, i1);
			if (MODE == SLAB_SETUP) {
				const double bi = a.b[i];
				const double ri = add(bi, mul(-1.0, st));  // combine2(1.0, b, -1.0, Ax, r)
				a.r[i] = ri;
				v[0] = fma(bi, bi, v[0]);
				v[1] = fma(ri, ri, v[1]);
			} else if (MODE == SLAB_CG_SP) {
				const double pi = a.src[i];
				v[0] = fma(st, pi, v[0]);
				if (a.first) {
					const double ri = a.r[i];
					v[1] = fma(ri, mul(ri, iM), v[1]);
				}
			} else if (MODE == SLAB_CG_UPDATE) {
				const double pi = a.src[i];
				a.x[i] = add(a.x[i], mul(a.alpha, pi));          // :169
				const double ri = add(a.r[i], mul(-a.alpha, st));  // :172
				a.r[i] = ri;
				const double ui = mul(ri, iM);                     // :175
				v[0] = fma(ri, ui, v[0]);
				v[1] = fma(ri, ri, v[1]);
			} else if (MODE == SLAB_APPLY) {
				a.y[i] = st;
			} else if (MODE == SLAB_PCG_SETUP) {
				const double ri = a.src[i];
				const double ui = mul(ri, iM);  // :138
				a.u[i] = ui;
				a.w[i] = st;                    // :141-143
				a.q[i] = a.s[i] = a.p[i] = a.z[i] = 0.0;  // :146-149
				v[0] = fma(ri, ui, v[0]);
				v[1] = fma(st, ui, v[1]);
				v[2] = fma(ri, ri, v[2]);
			} else if (MODE == SLAB_PCG_ITER) {
				const double wi = a.src[i];
				const double mi = mul(wi, iM);                            // :158
				const double qi = add(mi, mul(a.beta, a.q[i]));          // :200
				const double si = add(wi, mul(a.beta, a.s[i]));          // :203
				const double ui0 = a.u[i];
				const double pi = add(ui0, mul(a.beta, a.p[i]));         // :206
				const double zi = add(st, mul(a.beta, a.z[i]));          // :209
				const double ri = add(a.r[i], mul(-a.alpha, si));        // :212
				const double xi = add(a.x[i], mul(a.alpha, pi));         // :215
				const double ui = add(ui0, mul(-a.alpha, qi));           // :218
				const double wni = add(wi, mul(-a.alpha, zi));           // :221
				a.q[i] = qi;
				a.s[i] = si;
				a.p[i] = pi;
				a.z[i] = zi;
				a.r[i] = ri;
				a.x[i] = xi;
				a.u[i] = ui;
				a.wn[i] = wni;
				v[0] = fma(ri, ui, v[0]);   // next <r,u>
				v[1] = fma(wni, ui, v[1]);  // next <w,u>
				v[2] = fma(ri, ri, v[2]);   // next <r,r>
			} else if (MODE == SLAB_BICG_P) {
				const double ri = a.r[i];
				a.p[i] = a.first ? ri : add(add(ri, mul(a.beta, a.p[i])), mul(a.bo, a.v[i]));  // :168, :171
			} else if (MODE == SLAB_BICG_V) {
				a.v[i] = st;  // v = A p_hat (:178-180)
				v[0] = fma(st, a.rhat[i], v[0]);
			} else if (MODE == SLAB_BICG_S) {
				a.s[i] = add(a.r[i], mul(-a.alpha, a.v[i]));  // :189
			} else if (MODE == SLAB_BICG_T) {
				const double si = a.src[i];
				a.t[i] = st;  // t = A s_hat (:204-206)
				v[0] = fma(si, si, v[0]);
				v[1] = fma(st, si, v[1]);
				v[2] = fma(st, st, v[2]);
			} else if (MODE == SLAB_BICG_XR) {
				const double si = a.s[i];
				const double phi = mul(a.p[i], iM), shi = mul(si, iM);
				a.x[i] = add(add(a.x[i], mul(a.alpha, phi)), mul(a.omega, shi));  // :216
				const double ri = add(si, mul(-a.omega, a.t[i]));                   // :219
				a.r[i] = ri;
				v[0] = fma(ri, ri, v[0]);
				v[1] = fma(ri, a.rhat[i], v[1]);
			} else if (MODE == SLAB_BICG_X) {
				a.x[i] = add(a.x[i], mul(a.alpha, mul(a.p[i], iM)));  // :196
			} else {  // SLAB_CG_P
				const double ui = mul(a.r[i], iM);
				a.p[i] = a.first ? ui : add(ui, mul(a.beta, a.p[i]));
			}
		}
	}
	if (mode_dots(MODE) == 0) return;
	block_total<ND>(v);
	if (threadIdx.x == 0) {
		double *o = chunk_part + ((size_t)(z - 1) * kSlabChunks + c) * kSlabDots;
		for (int d = 0; d < kSlabDots; d++) o[d] = d < mode_dots(MODE) ? v[d < ND ? d : 0] : 0.0;
	}
}

// Per-plane sums of the chunk partials, chunks in order.
__global__ void k_slab_plane_sums(int z_lo, int z_hi, const double *chunk_part, double *plane_part) {
	const int z = z_lo + blockIdx.x * blockDim.x + threadIdx.x;
	if (z >= z_hi) return;
	for (int d = 0; d < kSlabDots; d++) {
		double s = 0.0;
		for (int c = 0; c < kSlabChunks; c++) s += chunk_part[((size_t)(z - 1) * kSlabChunks + c) * kSlabDots + d];
		plane_part[(size_t)(z - 1) * kSlabDots + d] = s;
	}
}

// t += x .* v, q += v .* v (stochastic-estimator.cc:195, :198); D = t ./ q (:216).
__global__ void __launch_bounds__(kSlabThreads) k_slab_accumulate(long long n, const double *__restrict__ x,
                                                                  const double *__restrict__ v, double *t, double *q,
                                                                  int reset) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const double vi = v[i];
		t[i] = add(reset ? 0.0 : t[i], mul(x[i], vi));
		q[i] = add(reset ? 0.0 : q[i], mul(vi, vi));
	}
}

__global__ void __launch_bounds__(kSlabThreads) k_slab_divide(long long n, const double *__restrict__ t,
                                                              const double *__restrict__ q, double *D) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		D[i] = __ddiv_rn(t[i], q[i]);
}

int blocks_for(long long n) {
	const long long b = (n + kSlabThreads - 1) / kSlabThreads;
	return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

bool slab_args(long n1, long n2, long nloc) {
	return n1 >= 1 && n2 >= 1 && nloc >= 1 && n1 <= (1L << 30) && n2 <= (1L << 30) && nloc <= (1L << 30) &&
	       (double)n1 * n2 * (nloc + 2) < 4.0e9;
}

// Pointers each mode reads or writes (src is the stencil input or the mode's
// first vector).
bool mode_args_ok(int mode, const sedi_slab_args &a) {
	switch (mode) {
	case SLAB_SETUP: return a.src && a.r && a.b;
	case SLAB_CG_SP: return a.src && (!a.first || a.r);
	case SLAB_CG_UPDATE: return a.src && a.x && a.r;
	case SLAB_APPLY: return a.src && a.y;
	case SLAB_PCG_SETUP: return a.src && a.u && a.w && a.q && a.s && a.p && a.z;
	case SLAB_PCG_ITER: return a.src && a.x && a.r && a.u && a.wn && a.q && a.s && a.p && a.z && a.wn != a.src;
	case SLAB_BICG_P: return a.r && a.p && (a.first || a.v);
	case SLAB_BICG_V: return a.src && a.v && a.rhat;
	case SLAB_BICG_S: return a.r && a.v && a.s;
	case SLAB_BICG_T: return a.src && a.t;
	case SLAB_BICG_XR: return a.x && a.p && a.s && a.t && a.r && a.rhat;
	case SLAB_BICG_X: return a.x && a.p;
	case SLAB_CG_P: return a.r && a.p;
	default: return false;
	}
}

template <int MODE>
void launch_mode(SlabGeo g, Coef k, int z_lo, int z_hi, const sedi_slab_args &a, double *chunk, cudaStream_t s) {
	constexpr int kMaxPlanes = 65535;  // grid y limit: one block row per plane
	for (int z = z_lo; z < z_hi; z += kMaxPlanes) {
		const int ze = z_hi - z > kMaxPlanes ? z + kMaxPlanes : z_hi;
		const dim3 grid(kSlabChunks, (unsigned)(ze - z));
		k_slab_sweep<MODE><<<grid, kSlabThreads, 0, s>>>(g, k, z, ze, a, chunk);
	}
}

}  // namespace

}  // namespace sedi

using namespace sedi;

extern "C" {

int sedi_slab_sweep(int mode, long n1, long n2, long nloc, double a, double b, double c, long z_lo, long z_hi,
                    const sedi_slab_args *args, double *chunk_part, double *plane_part, void *stream) {
	if (!slab_args(n1, n2, nloc) || !args || mode < 0 || mode >= SLAB_MODES || z_lo < 1 || z_hi > nloc + 1 ||
	    z_lo > z_hi)
		return SEDI_ERR_ARG;
	if (!mode_args_ok(mode, *args)) return SEDI_ERR_ARG;
	const bool dots = mode_dots(mode) > 0;
	if (dots && (!chunk_part || !plane_part)) return SEDI_ERR_ARG;
	if (z_lo == z_hi) return 0;
	SlabGeo g{(int)n1, (int)n2, (int)nloc, (long long)n1 * n2};
	const Coef k{a, b, c};
	cudaStream_t s = (cudaStream_t)stream;
	const int lo = (int)z_lo, hi = (int)z_hi;
	switch (mode) {
	case 0: launch_mode<0>(g, k, lo, hi, *args, chunk_part, s); break;
	case 1: launch_mode<1>(g, k, lo, hi, *args, chunk_part, s); break;
	case 2: launch_mode<2>(g, k, lo, hi, *args, chunk_part, s); break;
	case 3: launch_mode<3>(g, k, lo, hi, *args, chunk_part, s); break;
	case 4: launch_mode<4>(g, k, lo, hi, *args, chunk_part, s); break;
	case 5: launch_mode<5>(g, k, lo, hi, *args, chunk_part, s); break;
	case 6: launch_mode<6>(g, k, lo, hi, *args, chunk_part, s); break;
	case 7: launch_mode<7>(g, k, lo, hi, *args, chunk_part, s); break;
	case 8: launch_mode<8>(g, k, lo, hi, *args, chunk_part, s); break;
	case 9: launch_mode<9>(g, k, lo, hi, *args, chunk_part, s); break;
	case 10: launch_mode<10>(g, k, lo, hi, *args, chunk_part, s); break;
	case 11: launch_mode<11>(g, k, lo, hi, *args, chunk_part, s); break;
	default: launch_mode<12>(g, k, lo, hi, *args, chunk_part, s); break;
	}
	if (dots) k_slab_plane_sums<<<(hi - lo + 127) / 128, 128, 0, s>>>(lo, hi, chunk_part, plane_part);
	return cudaGetLastError() == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}

int sedi_slab_accumulate(long n, const double *x, const double *v, double *t, double *q, int reset, void *stream) {
	if (n < 1 || !x || !v || !t || !q) return SEDI_ERR_ARG;
	k_slab_accumulate<<<blocks_for(n), kSlabThreads, 0, (cudaStream_t)stream>>>(n, x, v, t, q, reset);
	return cudaGetLastError() == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}

int sedi_slab_divide(long n, const double *t, const double *q, double *D, void *stream) {
	if (n < 1 || !t || !q || !D) return SEDI_ERR_ARG;
	k_slab_divide<<<blocks_for(n), kSlabThreads, 0, (cudaStream_t)stream>>>(n, t, q, D);
	return cudaGetLastError() == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}

int sedi_slab_chunks(void) { return kSlabChunks; }

}  // extern "C"
