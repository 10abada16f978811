// Block reduction of the broadphase's first pass: scene bounds (min over all
// min corners, max over all max corners, Broadphase.cu:368-376), per-axis
// extent sums for the grid tuner, and input validation bits.
#pragma once
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"

namespace cc {

__device__ __forceinline__ bool finite3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// Every thread of the block calls this once; `have` marks threads that own a
// box. Block size NT (multiple of 32, <= 1024).
template <int NT>
__device__ __forceinline__ void accumulate_stats(float3 mn, float3 mx, bool have, DevStats *stats) {
	uint32_t e = 0;
	float3 ext = f3(0.f, 0.f, 0.f);
	if (have) {
		if (!finite3(mn) || !finite3(mx)) e |= kErrNonFinite;
		if (mn.x > mx.x || mn.y > mx.y || mn.z > mx.z) e |= kErrInverted;
		ext = mx - mn;
	} else {
		mn = f3(INFINITY, INFINITY, INFINITY);
		mx = f3(-INFINITY, -INFINITY, -INFINITY);
	}
	float v[6] = {mn.x, mn.y, mn.z, mx.x, mx.y, mx.z};
	float es[3] = {ext.x, ext.y, ext.z};
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
		for (int d = 0; d < 3; d++) {
			v[d] = fminf(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
			v[d + 3] = fmaxf(v[d + 3], __shfl_xor_sync(0xffffffffu, v[d + 3], o));
			es[d] += __shfl_xor_sync(0xffffffffu, es[d], o);
		}
		e |= __shfl_xor_sync(0xffffffffu, e, o);
	}
	__shared__ float sv[NT / 32][9];
	__shared__ uint32_t se[NT / 32];
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	if (l == 0) {
#pragma unroll
		for (int d = 0; d < 6; d++) sv[w][d] = v[d];
#pragma unroll
		for (int d = 0; d < 3; d++) sv[w][6 + d] = es[d];
		se[w] = e;
	}
	__syncthreads();
	if (threadIdx.x < 3) {
		const int d = threadIdx.x;
		float lo = sv[0][d], hi = sv[0][d + 3];
		double s = 0.0;
		for (int ww = 0; ww < NT / 32; ww++) {
			lo = fminf(lo, sv[ww][d]);
			hi = fmaxf(hi, sv[ww][d + 3]);
			s += (double)sv[ww][6 + d];
		}
		if (lo <= hi) {  // the block saw at least one box
			atomicMax(&stats->bmin_inv[d], ~f2ord(lo));
			atomicMax(&stats->bmax[d], f2ord(hi));
			atomicAdd(&stats->ext_sum[d], s);
		}
	} else if (threadIdx.x == 32) {
		uint32_t ee = 0;
		for (int ww = 0; ww < NT / 32; ww++) ee |= se[ww];
		if (ee) atomicOr(&stats->err, ee);
	}
}

}  // namespace cc
