// TMA plane streaming for the RHS-interleaved batched kernels (sm_100a).
//
// Data: a Krylov field of R right-hand sides is stored as R/W lane slices,
// each a dense [n3][n2][n1][W] grid (see SGeo).  A slice row [i1][W] is
// contiguous, so the TMA view of a field is 3-D: (W*n1, n2, n3*slices).  A
// block owns a P1 x P2 point tile, one lane slice and a chunk of i3 planes.
// Plane by plane, thread 0 issues TMA tile loads (cp.async.bulk.tensor.3d,
// each copy lands in this block's own shared memory only) of
//   - NS "source" fields with a one-point halo in i1 and i2 (box
//     W*(P1+2) x (P2+2) x 1), from which the stencil input is computed, and
//   - NQ "pointwise" fields on the tile interior (box W*P1 x P2 x 1),
// into an NST-stage shared-memory ring guarded by mbarriers.  TMA fills
// points outside the grid with zeros, which is the reference's zero ghost
// layer (Cg.hpp:57-62); planes -1 and n3 are never loaded and read as zero.
// The stencil input is computed once per halo point into a 3-plane ring, so
// each output point reads its seven stencil values from shared memory.
//
// Every wait is bounded: a block that has not seen its data after
// kWaitNs nanoseconds records an error and leaves the sweep (its remaining
// outputs are not written), so a broken descriptor cannot hang the GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sedi_common.cuh"

namespace sedi {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

struct Maps {
	CUtensorMap m[12];
};

template <class T>
struct VW;
template <>
struct VW<float> {
	static constexpr int V = 4;
	typedef float4 raw;
};
template <>
struct VW<double> {
	static constexpr int V = 2;
	typedef double2 raw;
};

template <class T>
struct Vec {
	static constexpr int V = VW<T>::V;
	T v[V];
};

template <class T>
__device__ __forceinline__ Vec<T> lds(const T *p) {
	typedef typename VW<T>::raw R;
	const R r = *reinterpret_cast<const R *>(p);
	Vec<T> o;
	memcpy(&o, &r, sizeof(R));
	return o;
}
template <class T>
__device__ __forceinline__ void sts(T *p, const Vec<T> &x) {
	typedef typename VW<T>::raw R;
	R r;
	memcpy(&r, &x, sizeof(R));
	*reinterpret_cast<R *>(p) = r;
}
template <class T>
__device__ __forceinline__ Vec<T> ldg_rw(const T *p) {
	typedef typename VW<T>::raw R;
	const R r = *reinterpret_cast<const R *>(p);
	Vec<T> o;
	memcpy(&o, &r, sizeof(R));
	return o;
}
template <class T>
__device__ __forceinline__ void stg(T *p, const Vec<T> &x) {
	typedef typename VW<T>::raw R;
	R r;
	memcpy(&r, &x, sizeof(R));
	*reinterpret_cast<R *>(p) = r;
}
template <class T>
__device__ __forceinline__ Vec<T> vzero() {
	Vec<T> o;
#pragma unroll
	for (int e = 0; e < Vec<T>::V; e++) o.v[e] = T(0);
	return o;
}

// ---------------------------------------------------------------------------
// mbarrier / TMA primitives (inline PTX).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, unsigned bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
	unsigned ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer() {
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}
// Bounded wait; false on timeout.
__device__ __forceinline__ bool mbar_wait_limit(uint64_t *bar, unsigned parity, unsigned long long limit_ns) {
	if (mbar_try(bar, parity)) return true;
	const unsigned long long t0 = gtimer();
	for (;;) {
		if (mbar_try(bar, parity)) return true;
		if (gtimer() - t0 > limit_ns) return false;
	}
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
	return mbar_wait_limit(bar, parity, kWaitNs);
}
__device__ __forceinline__ void fence_async_smem() {
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2) {
	asm volatile(
	    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
	    "[%2];" ::"r"(smem_u32(dst)),
	    "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
	    : "memory");
}

// L2 prefetch of a tensor tile (no shared memory, no barrier): the plane a
// later tma_load3 reads is already on its way from DRAM when that load is
// issued, so the ring's few stages are not the only bytes in flight.
__device__ __forceinline__ void tma_prefetch3(const CUtensorMap *map, int c0, int c1, int c2) {
	asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
	                 reinterpret_cast<uint64_t>(map)),
	             "r"(c0), "r"(c1), "r"(c2)
	             : "memory");
}

// ---------------------------------------------------------------------------
// Geometry of one batched sweep.
// ---------------------------------------------------------------------------
// Lane-sliced layout: a field of R lanes is stored as R/W slices, each a
// dense [n3][n2][n1][W] grid with W*sizeof(T) = 128 bytes (W = R when R is
// smaller), so every TMA box row and every point's lanes are contiguous.
// Element (point i, lane j) lives at ((j / W) * npts + i) * W + j % W.
struct SGeo {
	int n1, n2, n3;
	int R;          // lanes (right-hand sides, padded)
	int W;          // lanes per slice
	int zc;         // planes per block
	int tiles1;     // tiles along i1
	long long npts; // n1*n2*n3
	int pfd;        // planes the L2 prefetch runs ahead of the TMA loads (0: none)
};

__host__ __device__ __forceinline__ long long sliced(long long i, int j, int W, long long npts) {
	return ((long long)(j / W) * npts + i) * W + (j % W);
}

// PAIRS_: the two lanes of a point are two consecutive i1 points of one
// vector (a dense FP64 vector with even n1 is the 2-lane sliced layout of
// the (n1/2, n2, n3) grid); the stencil takes its i1 neighbours across the
// pair and the two lanes' sums are one reduction.
template <class T, int RB_, int P1_, int P2_, int THREADS_ = 512, int NSTR_ = 0, bool PAIRS_ = false, int MINB_ = 1>
struct Cfg {
	static constexpr int MINB = MINB_;  // blocks per SM the launch bounds ask for
	typedef T type;                              // element of the streamed fields
	static constexpr bool PAIRS = PAIRS_;
	typedef T ctype;                             // arithmetic type
	static constexpr int NSTR = NSTR_;  // stages of a transforming sweep's ring (0: SEDI_STREAM_NST_RING)
	static constexpr int V = Vec<ctype>::V;      // lanes per thread vector
	static constexpr int RB = RB_;
	static constexpr int LG = RB / V;  // lane groups per point
	static constexpr int ME = RB;      // tensor-map elements per point
	static constexpr int P1 = P1_, P2 = P2_;
	static constexpr int H1 = P1 + 2, H2 = P2 + 2;
	static constexpr int HALO = H1 * H2, INT = P1 * P2;
	static constexpr int THREADS = THREADS_;
	static constexpr int NPS = THREADS / LG;  // point slots
	static constexpr int KC = (HALO * LG + THREADS - 1) / THREADS;  // halo vectors per thread
	static constexpr int KO = (INT + NPS - 1) / NPS;                // output points per thread
	static_assert(THREADS % LG == 0, "lane groups");
	static_assert(RB * sizeof(T) % 16 == 0, "TMA inner box must be a multiple of 16 bytes");
	static_assert(ME * (P1 + 2) <= 256, "TMA box dimension limit");
};

// Pipeline of a sweep.  At step j the block computes the stencil input of
// plane j (ops that transform their sources) and the outputs of plane j-2,
// which depend only on planes j-3..j-1: the two phases are independent, so
// one barrier per plane suffices.  A stage (the TMA tiles of one plane) stays
// resident until the last step that reads it: step j+2 (its pointwise fields)
// or, when the stencil input is a raw source field read straight from the
// stages (IDENT), step j+3.
#ifndef SEDI_STREAM_NST_RING
#define SEDI_STREAM_NST_RING 5
#endif
#ifndef SEDI_STREAM_NST_IDENT
#define SEDI_STREAM_NST_IDENT 6
#endif

// Shared-memory carve-up for a kernel with NS source and NQ pointwise fields
// and ND reduced dot products.
// INPLACE: a transforming sweep that writes the stencil input over one of
// its source fields in the stage (no ring); the stencil then reads the
// stages, which live as long as a raw source's (KEEP 3).
template <class C, int NS, int NQ, int ND, bool IDENT, bool INPLACE = false>
struct Layout {
	typedef typename C::type T;
	static constexpr bool STAGED = IDENT || INPLACE;  // the stencil reads the stages
	static constexpr int NST = IDENT ? SEDI_STREAM_NST_IDENT
	                                 : (C::NSTR > 0 ? C::NSTR : (INPLACE ? SEDI_STREAM_NST_IDENT : SEDI_STREAM_NST_RING));
	static constexpr int KEEP = STAGED ? 3 : 2;  // steps a stage outlives its arrival
	static_assert(NST > KEEP + 1, "ring too shallow");
	// Every TMA destination starts on a 128-byte boundary.
	static constexpr size_t HALO_PAD = ((size_t)C::HALO * C::RB * sizeof(T) + 127) / 128 * 128;
	static constexpr size_t INT_PAD = ((size_t)C::INT * C::RB * sizeof(T) + 127) / 128 * 128;
	static constexpr size_t HALO_ELEMS = HALO_PAD / sizeof(T);  // element offset between source fields
	static constexpr size_t INT_ELEMS = INT_PAD / sizeof(T);    // element offset between pointwise fields
	static constexpr size_t STAGE_BYTES = (size_t)(NS * C::HALO + NQ * C::INT) * C::RB * sizeof(T);
	static constexpr size_t STAGE_PAD = NS * HALO_PAD + NQ * INT_PAD;
	static constexpr int RING = STAGED ? 0 : 4;  // computed stencil-input planes
	static constexpr size_t OFF_RING = NST * STAGE_PAD;
	static constexpr size_t OFF_BAR = OFF_RING + RING * HALO_PAD;
	static constexpr size_t BYTES = OFF_BAR + NST * sizeof(uint64_t);
	static_assert(BYTES <= 232448, "a sweep's shared memory must fit one block on sm_100 (227 KB)");
	// The per-lane reduction scratch reuses the stage and ring memory after
	// the sweep (both are dead once the last plane is done).
	static constexpr size_t RED_BYTES = (size_t)(ND > 0 ? ND : 1) * C::NPS * C::RB * sizeof(double);
	static_assert(RED_BYTES <= OFF_BAR, "reduction scratch must fit in the stages and the ring");
	static constexpr unsigned TX = (unsigned)STAGE_BYTES;
};

}  // namespace sedi
