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
                                 const double ext_mean[3], const GridParams &gp, int gx, int gy, int gz, uint64_t n) {
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
		mean_max = fmaxf(mean_max, (float)ext_mean[d]);
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

// Every thread of the block calls this once with the bounds of the boxes it
// saw (mn/mx; `have` false if none), its error bits, and the sum of those
// boxes' extents (esum) over ecnt boxes for the grid tuner's mean extent.
// Block size NT (multiple of 32, <= 1024).
template <int NT>
__device__ __forceinline__ void accumulate_stats(float3 mn, float3 mx, bool have, DevStats *stats,
                                                 const PlanArgs &pa, uint32_t e, float3 esum, uint32_t ecnt) {
	// warp reductions on order-preserving keys: one REDUX instruction each
	uint32_t k[6];
	k[0] = have ? f2ord(mn.x) : 0xffffffffu;
	k[1] = have ? f2ord(mn.y) : 0xffffffffu;
	k[2] = have ? f2ord(mn.z) : 0xffffffffu;
	k[3] = have ? f2ord(mx.x) : 0u;
	k[4] = have ? f2ord(mx.y) : 0u;
	k[5] = have ? f2ord(mx.z) : 0u;
#pragma unroll
	for (int d = 0; d < 3; d++) {
		k[d] = __reduce_min_sync(0xffffffffu, k[d]);
		k[d + 3] = __reduce_max_sync(0xffffffffu, k[d + 3]);
	}
	e = __reduce_or_sync(0xffffffffu, e);
	ecnt = __reduce_add_sync(0xffffffffu, ecnt);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		esum.x += __shfl_xor_sync(0xffffffffu, esum.x, o);
		esum.y += __shfl_xor_sync(0xffffffffu, esum.y, o);
		esum.z += __shfl_xor_sync(0xffffffffu, esum.z, o);
	}
	__shared__ uint32_t sk[NT / 32][6];
	__shared__ float sext[NT / 32][3];
	__shared__ uint32_t se[NT / 32], sc[NT / 32];
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	if (l == 0) {
#pragma unroll
		for (int d = 0; d < 6; d++) sk[w][d] = k[d];
		sext[w][0] = esum.x;
		sext[w][1] = esum.y;
		sext[w][2] = esum.z;
		se[w] = e;
		sc[w] = ecnt;
	}
	__syncthreads();
	if (threadIdx.x < 3) {
		const int d = threadIdx.x;
		uint32_t lo = sk[0][d], hi = sk[0][d + 3];
		double s = 0.0;
		uint32_t cnt = 0;
		for (int ww = 0; ww < NT / 32; ww++) {
			lo = min(lo, sk[ww][d]);
			hi = max(hi, sk[ww][d + 3]);
			s += (double)sext[ww][d];
			cnt += sc[ww];
		}
		if (lo != 0xffffffffu) {  // the block saw at least one box
			atomicMax(&stats->bmin_inv[d], ~lo);
			atomicMax(&stats->bmax[d], hi);
			atomicAdd(&stats->ext_sum[d], s);
			if (d == 0) atomicAdd(&stats->ext_count, (unsigned long long)cnt);
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
		double ext_mean[3];
		const unsigned long long cnt = __ldcg(&stats->ext_count);
		for (int d = 0; d < 3; d++) {
			bmin_inv[d] = __ldcg(&stats->bmin_inv[d]);
			bmax[d] = __ldcg(&stats->bmax[d]);
			ext_mean[d] = __ldcg(&stats->ext_sum[d]) / (double)(cnt ? cnt : 1);
		}
		const uint32_t err = __ldcg(&stats->err);
		Plan p = make_plan(bmin_inv, bmax, err, ext_mean, pa.gp, pa.gx, pa.gy, pa.gz, pa.n);
		stats->plan = p;
		stats->cells = p.G;
	}
}

// One box per thread (k_bounds).
template <int NT>
__device__ __forceinline__ void accumulate_stats_one(float3 mn, float3 mx, bool have, DevStats *stats,
                                                     const PlanArgs &pa) {
	uint32_t e = 0;
	if (have) {
		if (!finite3(mn) || !finite3(mx)) e |= kErrNonFinite;
		if (mn.x > mx.x || mn.y > mx.y || mn.z > mx.z) e |= kErrInverted;
	}
	accumulate_stats<NT>(mn, mx, have, stats, pa, e, have ? mx - mn : f3(0.f, 0.f, 0.f), have ? 1u : 0u);
}

}  // namespace cc
