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
// With b = c = 1 (the estimator's stencil) the products by 1.0 are exact and
// are left out: the same roundings with half the FP64 instructions.
__device__ __forceinline__ double stencil7(const Coef &k, double xc, double xm1, double xm2, double xm3,
                                           double xp1, double xp2, double xp3) {
	if (k.b == 1.0 && k.c == 1.0) {
		double y = mul(k.a, xc);
		y = sub(y, xm1);
		y = sub(y, xm2);
		y = sub(y, xm3);
		y = sub(y, xp1);
		y = sub(y, xp2);
		y = sub(y, xp3);
		return y;
	}
	double y = mul(k.a, xc);
	y = sub(y, mul(k.c, xm1));
	y = sub(y, mul(k.c, xm2));
	y = sub(y, mul(k.c, xm3));
	y = sub(y, mul(k.b, xp1));
	y = sub(y, mul(k.b, xp2));
	y = sub(y, mul(k.b, xp3));
	return y;
}

// ---------------------------------------------------------------------------
// 2.5-D sweep.  A block of 256 threads covers a 32 (i1) x 8 (i2) column tile
// and marches along i3 over [z0, z1); each thread keeps the stencil input at
// i3-1, i3 and i3+1 of its own column in registers, so per point it loads
// the i3+1 value and its four in-plane neighbours (L1/L2 hits) and needs no
// index division.  Block -> work assignment depends only on the grid, so the
// reductions below are bitwise reproducible.
// ---------------------------------------------------------------------------
constexpr int kTile1 = 32, kTile2 = 8;

struct Sweep {
	int i1, i2, z0, z1;
	bool active;
	long long base;  // index of (i1, i2, 0)
	long long s2, s3;
};

__device__ __forceinline__ Sweep sweep(const Geo &g, int zchunk) {
	Sweep w;
	w.i1 = blockIdx.x * kTile1 + (threadIdx.x & (kTile1 - 1));
	w.i2 = blockIdx.y * kTile2 + (threadIdx.x / kTile1);
	w.z0 = blockIdx.z * zchunk;
	w.z1 = min(w.z0 + zchunk, g.n3);
	w.active = w.i1 < g.n1 && w.i2 < g.n2 && w.z0 < w.z1;
	w.s2 = g.n1;
	w.s3 = (long long)g.n1 * g.n2;
	w.base = w.i1 + (long long)w.i2 * w.s2;
	return w;
}

// Stencil of the field f (value at an in-grid index) over the sweep; calls
// op(index, f(index), (A f)(index)) at every point of the thread's column.
template <class F, class Op>
__device__ __forceinline__ void march(const Geo &g, const Coef &k, const Sweep &w, F f, Op op) {
	if (!w.active) return;
	const bool m1 = w.i1 > 0, p1 = w.i1 < g.n1 - 1, m2 = w.i2 > 0, p2 = w.i2 < g.n2 - 1;
	long long i = w.base + (long long)w.z0 * w.s3;
	double prev = w.z0 > 0 ? f(i - w.s3) : 0.0;
	double cur = f(i);
	for (int i3 = w.z0; i3 < w.z1; i3++, i += w.s3) {
		const double next = (i3 + 1 < g.n3) ? f(i + w.s3) : 0.0;
		const double xm1 = m1 ? f(i - 1) : 0.0;
		const double xm2 = m2 ? f(i - w.s2) : 0.0;
		const double xp1 = p1 ? f(i + 1) : 0.0;
		const double xp2 = p2 ? f(i + w.s2) : 0.0;
		op(i, cur, stencil7(k, cur, xm1, xm2, prev, xp1, xp2, next));
		prev = cur;
		cur = next;
	}
}

// Pointwise visit of the sweep's column (no stencil).
template <class Op>
__device__ __forceinline__ void visit(const Geo &g, const Sweep &w, Op op) {
	if (!w.active) return;
	long long i = w.base + (long long)w.z0 * w.s3;
	for (int i3 = w.z0; i3 < w.z1; i3++, i += w.s3) op(i);
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
	const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
	const unsigned int nblk = gridDim.x * gridDim.y * gridDim.z;
	block_sum<ND>(v, sh);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int d = 0; d < ND; d++) partials[(size_t)bid * ND + d] = v[d];
		__threadfence();
		const unsigned int t = atomicAdd(ticket, 1u);
		last = (t == nblk - 1);
	}
	__syncthreads();
	if (!last) return false;
	__threadfence();
	double w[ND];
#pragma unroll
	for (int d = 0; d < ND; d++) w[d] = 0.0;
	for (unsigned int b = threadIdx.x; b < nblk; b += blockDim.x)
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
