// Slab (i3) domain decomposition of the FP64 CG method: the per-rank kernels.
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
// (operator by operator, no FMA contraction), like the single-vector form.
#include "sedi_internal.h"

namespace sedi {

namespace {

constexpr int kSlabThreads = 256;
constexpr int kSlabChunks = 8;  // row chunks per plane (fixed: the summation order depends on it)

struct SlabGeo {
	int n1, n2, nloc;
	long long plane;  // n1 * n2
};

__device__ __forceinline__ void chunk_rows(const SlabGeo &g, int c, int *r0, int *r1) {
	const int per = (g.n2 + kSlabChunks - 1) / kSlabChunks;
	*r0 = c * per;
	*r1 = min(g.n2, *r0 + per);
}

// 7-point stencil at ghosted plane z (1..nloc), row i2, column i1 of the slab.
__device__ __forceinline__ double slab_stencil(const SlabGeo &g, const Coef &k, const double *__restrict__ x,
                                               int z, int i2, int i1) {
	const long long i = (long long)z * g.plane + (long long)i2 * g.n1 + i1;
	const double xc = __ldg(x + i);
	const double xm1 = i1 > 0 ? __ldg(x + i - 1) : 0.0;
	const double xm2 = i2 > 0 ? __ldg(x + i - g.n1) : 0.0;
	const double xm3 = __ldg(x + i - g.plane);  // ghost plane 0 at the slab's lower side
	const double xp1 = i1 < g.n1 - 1 ? __ldg(x + i + 1) : 0.0;
	const double xp2 = i2 < g.n2 - 1 ? __ldg(x + i + g.n1) : 0.0;
	const double xp3 = __ldg(x + i + g.plane);  // ghost plane nloc+1 at the upper side
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

// Modes of the fused stencil sweep (one block per (plane, row chunk)).
enum SlabMode {
	SLAB_SETUP = 0,  // r = b - A x; <b,b>, <r,r>            (Cg.hpp:112-129)
	SLAB_SP = 1,     // s = A p; <s,p> (+ <r,u> when first)  (Cg.hpp:152-166)
	SLAB_UPDATE = 2, // s = A p; x += alpha p; r -= alpha s; <r,u>, <r,r>  (Cg.hpp:169-182)
	SLAB_APPLY = 3,  // y = A x                                (Stencil.hpp:38-54)
};

template <int MODE>
__global__ void __launch_bounds__(kSlabThreads) k_slab_sweep(SlabGeo g, Coef k, int z_lo, int z_hi, double iM,
                                                             double alpha, int first, const double *__restrict__ src,
                                                             double *x, double *r, const double *__restrict__ b,
                                                             double *y, double *chunk_part) {
	const int z = z_lo + (int)blockIdx.y;
	if (z >= z_hi) return;
	const int c = blockIdx.x;
	int r0, r1;
	chunk_rows(g, c, &r0, &r1);
	double v[2] = {0.0, 0.0};
	const long long n_in = (long long)(r1 - r0) * g.n1;
	for (long long t = threadIdx.x; t < n_in; t += kSlabThreads) {
		const int i2 = r0 + (int)(t / g.n1), i1 = (int)(t % g.n1);
		const long long i = (long long)z * g.plane + (long long)i2 * g.n1 + i1;
		const double a = slab_stencil(g, k, src, z, i2, i1);
		if (MODE == SLAB_SETUP) {
			const double bi = b[i];
			const double ri = add(bi, mul(-1.0, a));  // combine2(1.0, b, -1.0, Ax, r)
			r[i] = ri;
			v[0] = fma(bi, bi, v[0]);
			v[1] = fma(ri, ri, v[1]);
		} else if (MODE == SLAB_SP) {
			const double pi = src[i];
			v[0] = fma(a, pi, v[0]);
			if (first) {
				const double ri = r[i];
				v[1] = fma(ri, mul(ri, iM), v[1]);
			}
		} else if (MODE == SLAB_UPDATE) {
			const double pi = src[i];
			x[i] = add(x[i], mul(alpha, pi));              // :169
			const double ri = add(r[i], mul(-alpha, a));   // :172
			r[i] = ri;
			const double ui = mul(ri, iM);                 // :175
			v[0] = fma(ri, ui, v[0]);
			v[1] = fma(ri, ri, v[1]);
		} else {
			y[i] = a;
		}
	}
	if (MODE == SLAB_APPLY) return;
	block_total<2>(v);
	if (threadIdx.x == 0) {
		double *o = chunk_part + ((size_t)(z - 1) * kSlabChunks + c) * 2;
		o[0] = v[0];
		o[1] = v[1];
	}
}

// Per-plane sums of the chunk partials, chunks in order.
__global__ void k_slab_plane_sums(int z_lo, int z_hi, const double *chunk_part, double *plane_part) {
	const int z = z_lo + blockIdx.x * blockDim.x + threadIdx.x;
	if (z >= z_hi) return;
	for (int d = 0; d < 2; d++) {
		double s = 0.0;
		for (int c = 0; c < kSlabChunks; c++) s += chunk_part[((size_t)(z - 1) * kSlabChunks + c) * 2 + d];
		plane_part[(size_t)(z - 1) * 2 + d] = s;
	}
}

// p = u + beta p with u = r .* iM (p = u on the first iteration) on the
// slab's own planes (Cg.hpp:144-147, :175, :188).
__global__ void __launch_bounds__(kSlabThreads) k_slab_p(long long n, const double *__restrict__ r, double *p,
                                                         double iM, double beta, int first) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const double u = mul(r[i], iM);
		p[i] = first ? u : add(u, mul(beta, p[i]));
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

}  // namespace

}  // namespace sedi

using namespace sedi;

extern "C" {

int sedi_slab_sweep(int mode, long n1, long n2, long nloc, double a, double b, double c, long z_lo, long z_hi,
                    double iM, double alpha, int first, const double *src, double *x, double *r, const double *bvec,
                    double *y, double *chunk_part, double *plane_part, void *stream) {
	if (!slab_args(n1, n2, nloc) || mode < 0 || mode > 3 || z_lo < 1 || z_hi > nloc + 1 || z_lo > z_hi || !src)
		return SEDI_ERR_ARG;
	if (mode != SLAB_APPLY && (!chunk_part || !plane_part)) return SEDI_ERR_ARG;
	if ((mode == SLAB_SETUP && (!r || !bvec)) || (mode == SLAB_SP && first && !r) ||
	    (mode == SLAB_UPDATE && (!x || !r)) || (mode == SLAB_APPLY && !y))
		return SEDI_ERR_ARG;
	if (z_lo == z_hi) return 0;
	SlabGeo g{(int)n1, (int)n2, (int)nloc, (long long)n1 * n2};
	const Coef k{a, b, c};
	cudaStream_t s = (cudaStream_t)stream;
	const dim3 grid(kSlabChunks, (unsigned)(z_hi - z_lo));
	switch (mode) {
	case SLAB_SETUP:
		k_slab_sweep<SLAB_SETUP><<<grid, kSlabThreads, 0, s>>>(g, k, (int)z_lo, (int)z_hi, iM, alpha, first, src, x, r,
		                                                       bvec, y, chunk_part);
		break;
	case SLAB_SP:
		k_slab_sweep<SLAB_SP><<<grid, kSlabThreads, 0, s>>>(g, k, (int)z_lo, (int)z_hi, iM, alpha, first, src, x, r,
		                                                    bvec, y, chunk_part);
		break;
	case SLAB_UPDATE:
		k_slab_sweep<SLAB_UPDATE><<<grid, kSlabThreads, 0, s>>>(g, k, (int)z_lo, (int)z_hi, iM, alpha, first, src, x,
		                                                        r, bvec, y, chunk_part);
		break;
	default:
		k_slab_sweep<SLAB_APPLY><<<grid, kSlabThreads, 0, s>>>(g, k, (int)z_lo, (int)z_hi, iM, alpha, first, src, x,
		                                                       r, bvec, y, chunk_part);
		break;
	}
	if (mode != SLAB_APPLY) {
		const int nz = (int)(z_hi - z_lo);
		k_slab_plane_sums<<<(nz + 127) / 128, 128, 0, s>>>((int)z_lo, (int)z_hi, chunk_part, plane_part);
	}
	return cudaGetLastError() == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}

int sedi_slab_p(long n, const double *r, double *p, double iM, double beta, int first, void *stream) {
	if (n < 1 || !r || !p) return SEDI_ERR_ARG;
	k_slab_p<<<blocks_for(n), kSlabThreads, 0, (cudaStream_t)stream>>>(n, r, p, iM, beta, first);
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
