// Shared device helpers for the sedi_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sedi {

constexpr int kThreads = 256;       // threads per block for the single-vector kernels
constexpr int kMaxDots = 4;         // dot products fused into one reduction

struct Geo {
	int n1, n2, n3;
	long long n;  // n1*n2*n3
};

struct Coef {
	double a, b, c;
};

// ---------------------------------------------------------------------------
// Reference-order arithmetic.  The reference evaluates every SliceOps and
// Stencil expression operator by operator (SliceOps.hpp:17-108,
// Stencil.hpp:43-50); the _rn intrinsics are never contracted into FMAs, so
// each stored value rounds exactly as the reference's does.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul(double x, double y) { return __dmul_rn(x, y); }
__device__ __forceinline__ double add(double x, double y) { return __dadd_rn(x, y); }
__device__ __forceinline__ double sub(double x, double y) { return __dsub_rn(x, y); }

// Stencil::apply_direct term order (Stencil.hpp:43-50):
//   a*x_c - c*x_{i1-1} - c*x_{i2-1} - c*x_{i3-1} - b*x_{i1+1} - b*x_{i2+1} - b*x_{i3+1}
__device__ __forceinline__ double stencil7(const Coef &k, double xc, double xm1, double xm2, double xm3,
                                           double xp1, double xp2, double xp3) {
	double y = mul(k.a, xc);
	y = sub(y, mul(k.c, xm1));
	y = sub(y, mul(k.c, xm2));
	y = sub(y, mul(k.c, xm3));
	y = sub(y, mul(k.b, xp1));
	y = sub(y, mul(k.b, xp2));
	y = sub(y, mul(k.b, xp3));
	return y;
}

// Point index -> neighbour validity and offsets.
struct Nbr {
	long long i;
	bool m1, m2, m3, p1, p2, p3;
	long long s2, s3;
};

__device__ __forceinline__ Nbr neighbours(const Geo &g, long long i) {
	Nbr q;
	q.i = i;
	const long long s2 = g.n1, s3 = (long long)g.n1 * g.n2;
	const long long t = i / g.n1;
	const int i1 = (int)(i - t * g.n1);
	const int i3 = (int)(t / g.n2);
	const int i2 = (int)(t - (long long)i3 * g.n2);
	q.m1 = i1 > 0;
	q.p1 = i1 < g.n1 - 1;
	q.m2 = i2 > 0;
	q.p2 = i2 < g.n2 - 1;
	q.m3 = i3 > 0;
	q.p3 = i3 < g.n3 - 1;
	q.s2 = s2;
	q.s3 = s3;
	return q;
}

// Apply the stencil to a field given by a functor f(index) (the field value at
// an in-grid index).  Out-of-grid neighbours are the zero ghost value 0.0.
template <class F>
__device__ __forceinline__ double apply_stencil(const Coef &k, const Nbr &q, F f) {
	const double xc = f(q.i);
	const double xm1 = q.m1 ? f(q.i - 1) : 0.0;
	const double xm2 = q.m2 ? f(q.i - q.s2) : 0.0;
	const double xm3 = q.m3 ? f(q.i - q.s3) : 0.0;
	const double xp1 = q.p1 ? f(q.i + 1) : 0.0;
	const double xp2 = q.p2 ? f(q.i + q.s2) : 0.0;
	const double xp3 = q.p3 ? f(q.i + q.s3) : 0.0;
	return stencil7(k, xc, xm1, xm2, xm3, xp1, xp2, xp3);
}

// ---------------------------------------------------------------------------
// Deterministic grid reduction of ND doubles.
//
// Every block reduces its per-thread partials in a fixed tree and stores them
// at partials[block*ND + d]; the last block to arrive (atomic ticket) sums the
// per-block partials in a fixed order.  The summation order depends only on
// the launch shape, which depends only on the grid, so results are bitwise
// reproducible run to run.  Returns true in the last block (all its threads),
// with the totals in out[0..ND) visible to every thread of that block.
// ---------------------------------------------------------------------------
template <int ND>
__device__ __forceinline__ void warp_sum(double (&v)[ND]) {
#pragma unroll
	for (int off = 16; off > 0; off >>= 1)
#pragma unroll
		for (int d = 0; d < ND; d++) v[d] += __shfl_xor_sync(0xffffffffu, v[d], off);
}

template <int ND>
__device__ __forceinline__ void block_sum(double (&v)[ND], double (*sh)[ND]) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	warp_sum<ND>(v);
	if (lane == 0)
#pragma unroll
		for (int d = 0; d < ND; d++) sh[warp][d] = v[d];
	__syncthreads();
	if (warp == 0) {
#pragma unroll
		for (int d = 0; d < ND; d++) v[d] = lane < nwarps ? sh[lane][d] : 0.0;
		warp_sum<ND>(v);
	}
	__syncthreads();
}

template <int ND>
__device__ bool grid_sum(double (&v)[ND], double *partials, unsigned int *ticket, double (&out)[ND]) {
	__shared__ double sh[32][ND];
	__shared__ bool last;
	block_sum<ND>(v, sh);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int d = 0; d < ND; d++) partials[(size_t)blockIdx.x * ND + d] = v[d];
		__threadfence();
		const unsigned int t = atomicAdd(ticket, 1u);
		last = (t == gridDim.x - 1);
	}
	__syncthreads();
	if (!last) return false;
	__threadfence();
	double w[ND];
#pragma unroll
	for (int d = 0; d < ND; d++) w[d] = 0.0;
	for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
		for (int d = 0; d < ND; d++) w[d] += __ldcg(&partials[(size_t)b * ND + d]);
	block_sum<ND>(w, sh);
	__shared__ double res[ND];
	if (threadIdx.x == 0) {
#pragma unroll
		for (int d = 0; d < ND; d++) res[d] = w[d];
		*ticket = 0u;
	}
	__syncthreads();
#pragma unroll
	for (int d = 0; d < ND; d++) out[d] = res[d];
	return true;
}

}  // namespace sedi
