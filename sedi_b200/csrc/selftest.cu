// Self-test of the bounded-wait path every batched sweep relies on.
//
// The sweeps wait on mbarriers that TMA copies complete; every such wait gives
// up after a time limit, records an error and lets the block leave, so a copy
// that never lands cannot hang the GPU.  This kernel runs that wait on an
// mbarrier nothing ever arrives on (the "flag that nothing sets") with a short
// limit, and reports whether it gave up and how long it waited.  No copy is
// issued, nothing faults, and the context stays usable.
#include "sedi_internal.h"
#include "stream.cuh"

namespace sedi {
namespace {

__global__ void k_wait_selftest(unsigned long long limit_ns, int *timed_out, unsigned long long *waited_ns) {
	__shared__ uint64_t bar;
	if (threadIdx.x == 0) {
		mbar_init(&bar, 1);
		mbar_init_fence();
	}
	__syncthreads();
	bool ok = true;
	unsigned long long t0 = 0, t1 = 0;
	if (threadIdx.x == 0) {
		t0 = gtimer();
		ok = mbar_wait_limit(&bar, 0u, limit_ns);  // phase 0 never completes
		t1 = gtimer();
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		*timed_out = ok ? 0 : 1;
		*waited_ns = t1 - t0;
	}
}

}  // namespace
}  // namespace sedi

extern "C" int sedi_selftest_bounded_wait(double limit_ms, int *timed_out, double *waited_ms) {
	if (!(limit_ms > 0.0) || limit_ms > 5000.0 || !timed_out) return SEDI_ERR_ARG;
	int *d_flag = nullptr;
	unsigned long long *d_ns = nullptr;
	if (cudaMalloc(&d_flag, sizeof(int)) != cudaSuccess || cudaMalloc(&d_ns, sizeof(unsigned long long)) != cudaSuccess) {
		cudaGetLastError();
		if (d_flag) cudaFree(d_flag);
		return SEDI_ERR_NOMEM;
	}
	sedi::k_wait_selftest<<<1, 32>>>((unsigned long long)(limit_ms * 1e6), d_flag, d_ns);
	int flag = 0;
	unsigned long long ns = 0;
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) e = cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost);
	cudaFree(d_flag);
	cudaFree(d_ns);
	if (e != cudaSuccess) return SEDI_ERR_CUDA;
	*timed_out = flag;
	if (waited_ms) *waited_ms = (double)ns / 1e6;
	return 0;
}
