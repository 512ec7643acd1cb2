// Probe generation.
//
// Host path: the reference's own generator, DistrRngStd::fill_plusminusone
// (DistrRngStd.hpp:22-42) -- std::mt19937 seeded with one value, a
// std::uniform_real_distribution<double>(0,1) draw per point, +1 when the draw
// is > 0.5 and -1 otherwise, points visited i1 fastest.  The same standard
// library code runs here, so the probes are the reference's bit for bit.
#include <random>

#include "sedi_internal.h"

namespace sedi {

void host_fill_probe(uint32_t seed, long n, double *out) {
	std::mt19937 engine(seed);
	std::uniform_real_distribution<double> dist(0.0, 1.0);
	for (long i = 0; i < n; i++) {
		const double x = dist(engine);
		out[i] = x > 0.5 ? 1.0 : -1.0;
	}
}

// Points [offset, offset + count) of the same probe: a double of
// uniform_real_distribution<double> takes two 32-bit draws of mt19937
// (generate_canonical with 53 bits from a 32-bit engine), so the engine
// skips 2 * offset draws first.
void host_fill_probe_range(uint32_t seed, long long offset, long long count, double *out) {
	std::mt19937 engine(seed);
	engine.discard((unsigned long long)offset * 2ull);
	std::uniform_real_distribution<double> dist(0.0, 1.0);
	for (long long i = 0; i < count; i++) {
		const double x = dist(engine);
		out[i] = x > 0.5 ? 1.0 : -1.0;
	}
}

// ---------------------------------------------------------------------------
// Device path.  MT19937 (Matsumoto & Nishimura 1998, ACM TOMACS 8(1)) with
// the published parameters (n=624, m=397, a=0x9908b0df, tempering
// (11,0xffffffff) (7,0x9d2c5680) (15,0xefc60000) 18, init multiplier
// 1812433253), one generator per probe, one block per probe.  A twist
// regenerates all 624 words; word i reads words i+1 and i+397 (mod 624) of
// the state as the sequential algorithm sees them, so it runs in three
// phases whose inputs are complete: [0,227) reads only old words,
// [227,454) reads new words [0,227), [454,624) reads new words [227,397) and
// (word 623) new word 0.  Each point uses two consecutive draws g1, g2:
// u = (g1 + g2*2^32) / 2^64 (the sum rounds once, the rest is exact), the
// double std::uniform_real_distribution<double>(0,1) produces with a 32-bit
// engine, and the probe value is +1 when u > 0.5, i.e. when the rounded sum
// exceeds 2^63 (DistrRngStd.hpp:32-40).
// ---------------------------------------------------------------------------
namespace {

constexpr int kMtN = 624, kMtM = 397, kMtThreads = 256;

__device__ __forceinline__ uint32_t mt_mix(uint32_t cur, uint32_t next, uint32_t far) {
	const uint32_t y = (cur & 0x80000000u) | (next & 0x7fffffffu);
	return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
	y ^= y >> 11;
	y ^= (y << 7) & 0x9d2c5680u;
	y ^= (y << 15) & 0xefc60000u;
	y ^= y >> 18;
	return y;
}

// Twist phase over words [lo, hi): every thread first reads its inputs, then
// all write.
__device__ __forceinline__ void mt_phase(uint32_t *mt, int lo, int hi) {
	uint32_t v[(kMtN + kMtThreads - 1) / kMtThreads];
	int k = 0;
	for (int i = lo + threadIdx.x; i < hi; i += kMtThreads, k++)
		v[k] = mt_mix(mt[i], mt[(i + 1) % kMtN], mt[(i + kMtM) % kMtN]);
	__syncthreads();
	k = 0;
	for (int i = lo + threadIdx.x; i < hi; i += kMtThreads, k++) mt[i] = v[k];
	__syncthreads();
}

// Probe j (seed0 + j) of a batch, written as lane j of a lane-sliced FP64
// field (element (i, j) at ((j / W) * npts + i) * W + j % W), or densely at
// out[j * npts + i] when W == 0.
__global__ void __launch_bounds__(kMtThreads) k_mt_probes(uint32_t seed0, long long npts, int W, double *out) {
	__shared__ uint32_t mt[kMtN];
	__shared__ uint32_t draw[kMtN];
	const int j = blockIdx.x;
	if (threadIdx.x == 0) {
		mt[0] = seed0 + (uint32_t)j;
		for (int i = 1; i < kMtN; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
	}
	__syncthreads();
	double *base = W ? out + ((long long)(j / W) * npts) * W + (j % W) : out + (long long)j * npts;
	const long long step = W ? W : 1;
	for (long long p0 = 0; p0 < npts; p0 += kMtN / 2) {
		mt_phase(mt, 0, kMtN - kMtM);
		mt_phase(mt, kMtN - kMtM, 2 * (kMtN - kMtM));
		mt_phase(mt, 2 * (kMtN - kMtM), kMtN);
		for (int i = threadIdx.x; i < kMtN; i += kMtThreads) draw[i] = mt_temper(mt[i]);
		__syncthreads();
		for (int k = threadIdx.x; k < kMtN / 2; k += kMtThreads) {
			const long long p = p0 + k;
			if (p >= npts) break;
			const double sum = __dadd_rn((double)draw[2 * k], __dmul_rn((double)draw[2 * k + 1], 4294967296.0));
			base[p * step] = sum > 9223372036854775808.0 ? 1.0 : -1.0;
		}
		__syncthreads();
	}
}

}  // namespace

int device_fill_probes(uint32_t seed, int nprobes, long long npts, int W, double *out, cudaStream_t s) {
	if (nprobes <= 0) return 0;
	k_mt_probes<<<nprobes, kMtThreads, 0, s>>>(seed, npts, W, out);
	return cudaGetLastError() == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}

}  // namespace sedi

extern "C" void sedi_fill_probe_range(uint32_t seed, long offset, long count, double *out) {
	if (out && offset >= 0 && count > 0) sedi::host_fill_probe_range(seed, offset, count, out);
}

extern "C" int sedi_fill_probes_dev(uint32_t seed, int nprobes, long n, double *out_dev, void *stream) {
	if (nprobes < 0 || n < 1 || !out_dev) return SEDI_ERR_ARG;
	const int rc = sedi::device_fill_probes(seed, nprobes, n, 0, out_dev, (cudaStream_t)stream);
	if (rc) return rc;
	return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? 0 : SEDI_ERR_CUDA;
}
