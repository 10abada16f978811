// Block reduction of the broadphase's first pass: scene bounds (min over all
// min corners, max over all max corners, Broadphase.cu:368-376), per-axis
// extent sums for the grid tuner, and input validation bits. The last block
// to finish turns the reduced bounds into the grid plan (make_plan).
#pragma once
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"

namespace cc {

__device__ __forceinline__ bool finite3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// Grid parameters from the reduced bounds: the reference's shift and inverse
// bin size (Broadphase.cu:377-381) and the search grid of the pair test.
__device__ inline Plan make_plan(const uint32_t bmin_inv[3], const uint32_t bmax[3], uint32_t err,
                                 const double ext_sum[3], const GridParams &gp, int gx, int gy, int gz, uint64_t n) {
	Plan p;
	const int grid[3] = {gx, gy, gz};
	float mn[3], mx[3];
	p.valid = (err & (kErrNonFinite | kErrInverted | kErrBadIndex)) ? 0 : 1;
	for (int d = 0; d < 3; d++) {
		mn[d] = ord2f(~bmin_inv[d]);
		mx[d] = ord2f(bmax[d]);
		p.origin[d] = fabsf(mn[d]);                                  // :379
		p.invbin[d] = (float)grid[d] / fabsf(mx[d] + fabsf(mn[d]));  // :380-381
		p.grid[d] = grid[d];
		p.lo[d] = mn[d] + p.origin[d];  // exact minimum of the shifted coordinates
	}
	float ext[3];
	float mean_max = 0.f;
	for (int d = 0; d < 3; d++) {
		const float hi = mx[d] + p.origin[d];
		ext[d] = hi - p.lo[d];
		mean_max = fmaxf(mean_max, (float)(ext_sum[d] / (double)(n ? n : 1)));
	}
	int dim[3];
	if (gp.user_dim[0] > 0) {
		for (int d = 0; d < 3; d++) dim[d] = min(max(gp.user_dim[d], 1), kMaxDim);
	} else {
		// cell edge: the cube root of the volume that holds k_target boxes on
		// average, but at least min_ratio times the mean box extent
		double vol = 1.0;
		const float floor_len = fmaxf(mean_max, 1e-30f);
		for (int d = 0; d < 3; d++) vol *= (double)fmaxf(ext[d], floor_len);
		double c = cbrt(vol * (double)gp.k_target / (double)(n ? n : 1));
		c = fmax(c, (double)gp.min_ratio * (double)mean_max);
		for (int d = 0; d < 3; d++) {
			const double q = c > 0.0 ? (double)ext[d] / c : 1.0;
			dim[d] = (int)fmin(fmax(q, 1.0), (double)kMaxDim);
		}
	}
	while ((uint64_t)dim[0] * dim[1] * dim[2] > gp.g_max) {
		for (int d = 0; d < 3; d++) dim[d] = max(1, (int)(dim[d] * 0.8f));
	}
	for (int d = 0; d < 3; d++) {
		p.dim[d] = dim[d];
		p.inv[d] = ext[d] > 0.f ? (float)dim[d] / ext[d] : 0.f;
	}
	p.G = (uint32_t)dim[0] * dim[1] * dim[2];
	return p;
}

// Arguments the last block needs to build the plan.
struct PlanArgs {
	GridParams gp;
	int gx, gy, gz;
	uint64_t n;
};

// Every thread of the block calls this once; `have` marks threads that own a
// box. Block size NT (multiple of 32, <= 1024).
template <int NT>
__device__ __forceinline__ void accumulate_stats(float3 mn, float3 mx, bool have, DevStats *stats,
                                                 const PlanArgs &pa) {
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
	// the last block to finish builds the plan from the complete reduction
	// (only the threads that issued atomics need to fence them)
	__shared__ bool s_last;
	if (threadIdx.x < 3 || threadIdx.x == 32) __threadfence();
	__syncthreads();
	if (threadIdx.x == 0) s_last = atomicAdd(&stats->blocks_done, 1u) == gridDim.x - 1;
	__syncthreads();
	if (s_last && threadIdx.x == 0) {
		__threadfence();
		uint32_t bmin_inv[3], bmax[3];
		double ext_sum[3];
		for (int d = 0; d < 3; d++) {
			bmin_inv[d] = __ldcg(&stats->bmin_inv[d]);
			bmax[d] = __ldcg(&stats->bmax[d]);
			ext_sum[d] = __ldcg(&stats->ext_sum[d]);
		}
		const uint32_t err = __ldcg(&stats->err);
		const Plan p = make_plan(bmin_inv, bmax, err, ext_sum, pa.gp, pa.gx, pa.gy, pa.gz, pa.n);
		stats->plan = p;
		stats->cells = p.G;
	}
}

}  // namespace cc
