// Roofline denominators measured on the running GPU: FP32 and FP64 FMA
// throughput of the chip (the exact MPR stage is graded against the FP64 one).
// Every thread runs kChains independent multiply-add chains; the kernel fills
// every SM (kNumSMs x 8 blocks of 256 threads), so the pipes, not latency,
// bound it.
#include "../../include/collide_b200.h"
#include "cc_common.cuh"

namespace cc {
namespace {

constexpr int kChains = 8;
constexpr int kPeakNT = 256;

template <class T>
__global__ void __launch_bounds__(kPeakNT) k_fma_peak(T *sink, T m, T c, int iters) {
	T a[kChains];
	const T x = (T)(threadIdx.x + 1) * (T)1e-3;
#pragma unroll
	for (int j = 0; j < kChains; j++) a[j] = x + (T)j;
	for (int i = 0; i < iters; i++) {
#pragma unroll
		for (int j = 0; j < kChains; j++) a[j] = fma(a[j], m, c);
	}
	T s = 0;
#pragma unroll
	for (int j = 0; j < kChains; j++) s += a[j];
	if (s == (T)-1.25) *sink = s;  // never taken for these inputs; keeps the chains live
}

__device__ double g_peak_sink[2];

template <class T>
cudaError_t time_peak(double *flops, cudaStream_t s) {
	T *sink = nullptr;
	cudaError_t e = cudaGetSymbolAddress((void **)&sink, g_peak_sink);
	if (e != cudaSuccess) return e;
	cudaEvent_t e0, e1;
	if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
	if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
		cudaEventDestroy(e0);
		return e;
	}
	const unsigned blocks = kNumSMs * 8;
	const int iters = sizeof(T) == 8 ? 4096 : 16384;
	float best = 1e30f;
	for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {  // first run warms the clocks
		cudaEventRecord(e0, s);
		k_fma_peak<T><<<blocks, kPeakNT, 0, s>>>(sink, (T)0.9999, (T)1e-4, iters);
		cudaEventRecord(e1, s);
		e = cudaEventSynchronize(e1);
		float ms = 0.f;
		if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
		if (e == cudaSuccess && rep > 0 && ms < best) best = ms;
	}
	if (e == cudaSuccess) e = cudaGetLastError();
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (e == cudaSuccess) *flops = 2.0 * kChains * (double)iters * blocks * kPeakNT / (best * 1e-3);
	return e;
}

}  // namespace
}  // namespace cc

extern "C" cc_status cc_fma_peak(int fp64, double *flop_per_s, void *stream) {
	if (!flop_per_s) return CC_ERR_INVALID_ARGUMENT;
	*flop_per_s = 0.0;
	const cudaError_t e = fp64 ? cc::time_peak<double>(flop_per_s, (cudaStream_t)stream)
	                           : cc::time_peak<float>(flop_per_s, (cudaStream_t)stream);
	return e == cudaSuccess ? CC_OK : CC_ERR_CUDA;
}
