// Residual of A x = b without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// residual check: code running inside a memory pool or arena that owns all
// device memory, allocation-free real-time or serving loops that must not
// hit cudaMalloc latency or fail on it mid-run, and host frameworks whose
// allocator is not CUDA's.  sedi_residual_noalloc serves them: the caller
// passes the input vectors and the output vector, and the only scratch the
// kernel needs (per-block partial sums, the reduction ticket and the result)
// lives in the fixed file-scope device array below, sized for a stated
// maximum launch.  Every GPU that loads this library holds that array (about
// 64 KiB) until the process exits.
#include <mutex>

#include "sedi_internal.h"

namespace sedi {

namespace {

constexpr int kNoallocMaxBlocks = 4096;

struct NoallocScratch {
	double partials[kNoallocMaxBlocks * 2];
	double result[4];  // <b,b> (1 if 0), <r,r>, err
	unsigned int ticket;
};

// The only scratch memory of sedi_residual_noalloc.  Every call shares it
// and it keeps the last call's contents.
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// Host side: `g_noalloc_scratch` named in host code is a host-side stand-in,
// not a device address, so the device address is looked up per device.
constexpr int kMaxDevices = 64;
static NoallocScratch *g_scratch_dev[kMaxDevices];
static std::mutex g_scratch_mu;

__global__ void __launch_bounds__(kThreads) k_residual_noalloc(Geo g, Coef k, int zc, const double *__restrict__ x,
                                                               const double *__restrict__ b, double *__restrict__ r,
                                                               NoallocScratch *sc) {
	double v[2] = {0.0, 0.0};
	march(g, k, sweep(g, zc), [&](long long j) { return __ldg(x + j); }, [&](long long i, double, double ax) {
		const double bi = __ldg(b + i);
		const double ri = add(bi, -ax);  // r = b - A x (Cg.hpp:119-123)
		r[i] = ri;
		v[0] = fma(bi, bi, v[0]);
		v[1] = fma(ri, ri, v[1]);
	});
	double out[2];
	if (grid_sum<2>(v, sc->partials, &sc->ticket, out) && threadIdx.x == 0) {
		const double bb = out[0] == 0.0 ? 1.0 : out[0];  // Cg.hpp:115
		sc->result[0] = bb;
		sc->result[1] = out[1];
		sc->result[2] = sqrt(__ddiv_rn(out[1], bb));      // Cg.hpp:129
	}
}

static void shape(const Geo &g, dim3 *grid, int *zc) {
	const int gx = (g.n1 + kTile1 - 1) / kTile1, gy = (g.n2 + kTile2 - 1) / kTile2;
	long long nz = (148LL * 6 + (long long)gx * gy - 1) / ((long long)gx * gy);
	if (nz < 1) nz = 1;
	if (nz > g.n3) nz = g.n3;
	*zc = (int)((g.n3 + nz - 1) / nz);
	nz = (g.n3 + *zc - 1) / *zc;
	*grid = dim3(gx, gy, (unsigned)nz);
}

}  // namespace

}  // namespace sedi

using namespace sedi;

extern "C" int sedi_residual_noalloc(long n1, long n2, long n3, double a, double b, double c, const double *x_dev,
                                     const double *b_dev, double *r_dev, double *err_out, void *stream) {
	if (n1 < 1 || n2 < 1 || n3 < 1 || n1 > (1L << 30) || n2 > (1L << 30) || n3 > (1L << 30) || !x_dev || !b_dev ||
	    !r_dev || !err_out)
		return SEDI_ERR_ARG;
	Geo g;
	g.n1 = (int)n1;
	g.n2 = (int)n2;
	g.n3 = (int)n3;
	g.n = (long long)n1 * n2 * n3;
	// r is written while other blocks still read x (its neighbours) and b
	// through the read-only path: r may share no element with either.
	const size_t bytes = (size_t)g.n * sizeof(double);
	auto overlap = [bytes](const void *p, const void *q) {
		const char *a = static_cast<const char *>(p), *b2 = static_cast<const char *>(q);
		return a < b2 + bytes && b2 < a + bytes;
	};
	if (overlap(r_dev, x_dev) || overlap(r_dev, b_dev)) return SEDI_ERR_ARG;
	dim3 grid;
	int zc;
	shape(g, &grid, &zc);
	if ((long long)grid.x * grid.y * grid.z > kNoallocMaxBlocks) return SEDI_ERR_ARG;  // grid too large
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
		cudaGetLastError();
		return SEDI_ERR_NODEV;
	}
	NoallocScratch *sc;
	{
		// First call on a device: look up the array's device address with that
		// device current (no allocation).
		std::lock_guard<std::mutex> lk(g_scratch_mu);
		if (!g_scratch_dev[dev]) {
			void *p = nullptr;
			if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
				cudaGetLastError();
				return SEDI_ERR_CUDA;
			}
			g_scratch_dev[dev] = static_cast<NoallocScratch *>(p);
		}
		sc = g_scratch_dev[dev];
	}
	cudaStream_t s = (cudaStream_t)stream;
	// The reduction ticket must start at zero.
	if (cudaMemsetAsync(&sc->ticket, 0, sizeof(unsigned int), s) != cudaSuccess) return SEDI_ERR_CUDA;
	const Coef k{a, b, c};
	k_residual_noalloc<<<grid, kThreads, 0, s>>>(g, k, zc, x_dev, b_dev, r_dev, sc);
	if (cudaGetLastError() != cudaSuccess) return SEDI_ERR_CUDA;
	if (cudaMemcpyAsync(err_out, &sc->result[2], sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		return SEDI_ERR_CUDA;
	return 0;
}
