// Incremental broadphase for time-stepped scenes (cc_set_incremental): a
// candidate pair list in the manner of a Verlet list.
//
// A rebuild step searches the boxes inflated by a margin m (half on every
// side) with the full broadphase, which yields the sorted, duplicate-free list
// of candidate pairs, and keeps the step's unshifted boxes as the reference.
// Any later step whose box corners all lie within (m - delta) / 2 of the
// reference finds its pairs among the candidates: for a pair whose shifted
// boxes overlap (closed, Broadphase.cu:237), min_a - max_b <= rounding of the
// shift at that step, each corner moved by at most d, so at the reference
// min_a - max_b <= 2d + rounding < m up to the rounding of the inflation and
// the reference shift; delta bounds all of those roundings (a few units in the
// last place of the largest coordinate plus the shift). Such a step tests the
// candidates exactly on its own shifted boxes and keeps the ones that overlap,
// in order, so the result is the sorted pair list of a full search. A step
// that moved too far sets a flag and the host redoes it as a rebuild.
//
// Compiled with -fmad=false (the in-place shift must round as the reference's).
#include <algorithm>

#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"

namespace cc {

namespace {
constexpr int kNT = 256;

// The margin m: inc_margin times the largest per-axis mean box extent of this
// step (the same figure the search grid is tuned with).
__device__ __forceinline__ float margin_of(const DevStats *stats, float factor) {
	const double cnt = (double)(stats->ext_count ? stats->ext_count : 1ull);
	double mx = 0.0;
	for (int d = 0; d < 3; d++) mx = fmax(mx, stats->ext_sum[d] / cnt);
	return (float)(factor * mx);
}

// scratch = the boxes inflated by m / 2 on every side (unshifted).
__global__ void __launch_bounds__(kNT) k_vinflate(uint64_t n, const float *__restrict__ aabb,
                                                   float *__restrict__ scratch, DevStats *stats, float factor) {
	pdl_begin();
	const float m = margin_of(stats, factor), h = 0.5f * m;
	if (blockIdx.x == 0 && threadIdx.x == 0) stats->vmargin = m;
	const uint64_t total = 6 * n, step = (uint64_t)gridDim.x * kNT;
	for (uint64_t k = (uint64_t)blockIdx.x * kNT + threadIdx.x; k < total; k += step)
		scratch[k] = k < 3 * n ? aabb[k] - h : aabb[k] + h;
}

// Largest corner displacement against the reference (ordered bits into
// stats->vdisp), a copy of the unshifted boxes GenerateAABB does not write
// (RECT and TRIANGLEMESH, AABBGenerator.cu:110-111: a redo regenerates all
// others), and the in-place shift by fabs(min) (Broadphase.cu:382-386).
// Invalid input is left as it is.
__global__ void __launch_bounds__(kNT) k_vcheck(uint64_t n, float *__restrict__ aabb, const float *__restrict__ ref,
                                                 float *__restrict__ backup, const int32_t *__restrict__ T,
                                                 DevStats *stats) {
	pdl_begin();
	__shared__ float origin[3];
	__shared__ int valid;
	if (threadIdx.x < 3) origin[threadIdx.x] = stats->plan.origin[threadIdx.x];
	if (threadIdx.x == 0) valid = stats->plan.valid;
	__syncthreads();
	if (!valid) return;
	const uint64_t total = 6 * n, step = (uint64_t)gridDim.x * kNT;
	float dmax = 0.f;
	for (uint64_t k = (uint64_t)blockIdx.x * kNT + threadIdx.x; k < total; k += step) {
		const float v = aabb[k];
		dmax = fmaxf(dmax, fabsf(v - ref[k]));
		const int t = __ldg(T + (k < 3 * n ? k : k - 3 * n) / 3);
		if (t == RECT || t == TRIANGLEMESH) backup[k] = v;
		aabb[k] = v + origin[k % 3];
	}
	dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, 16));
	dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, 8));
	dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, 4));
	dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, 2));
	dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, 1));
	if ((threadIdx.x & 31) == 0 && dmax > 0.f) atomicMax(&stats->vdisp, f2ord(dmax));
}

// The step may use the candidates iff every corner moved by at most
// (m - delta) / 2; delta = 2^-19 of the largest coordinate magnitude plus the
// largest shift (16 units in the last place: the roundings of the inflation,
// the two shifts and the overlap tests, with room to spare).
__device__ __forceinline__ bool step_fits(const DevStats *stats, float margin) {
	float cmax = 0.f, omax = 0.f;
	for (int d = 0; d < 3; d++) {
		cmax = fmaxf(cmax, fmaxf(fabsf(ord2f(~stats->bmin_inv[d])), fabsf(ord2f(stats->bmax[d]))));
		omax = fmaxf(omax, stats->plan.origin[d]);
	}
	const float delta = (cmax + omax) * 0x1p-19f;
	const float limit = 0.5f * (margin - delta);
	return stats->vdisp == 0u ? limit >= 0.f : ord2f(stats->vdisp) <= limit;
}

// flags[i] = candidate i overlaps on this step's shifted boxes (all zero, and
// stats->vbad set, when the step moved too far).
// A rebuild step's own candidates always hold its pairs (no displacement).
__global__ void __launch_bounds__(kNT) k_vfilter(uint64_t nc, const unsigned long long *__restrict__ cand,
                                                  const float *__restrict__ aabb, uint64_t n, DevStats *stats,
                                                  uint32_t *__restrict__ flags, int rebuild, float margin) {
	pdl_begin();
	__shared__ int fits;
	if (threadIdx.x == 0) fits = stats->plan.valid && (rebuild || step_fits(stats, margin));
	__syncthreads();
	if (!fits && blockIdx.x == 0 && threadIdx.x == 0) stats->vbad = 1u;
	const float *mx = aabb + 3 * n;
	const uint64_t step = (uint64_t)gridDim.x * kNT;
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < nc; i += step) {
		uint32_t f = 0u;
		if (fits) {
			const unsigned long long key = cand[i];
			const uint64_t a = key >> 32, b = key & 0xffffffffull;
			if (a < n && b < n) {
				const float *pa = aabb + 3 * a, *pb = aabb + 3 * b, *qa = mx + 3 * a, *qb = mx + 3 * b;
				f = pa[0] <= qb[0] && pb[0] <= qa[0] && pa[1] <= qb[1] && pb[1] <= qa[1] && pa[2] <= qb[2] &&
				    pb[2] <= qa[2];
			}
		}
		flags[i] = f;
	}
}

// The overlapping candidates, in order, into out (if they fit its capacity).
__global__ void __launch_bounds__(kNT) k_vscatter(uint64_t nc, const unsigned long long *__restrict__ cand,
                                                   const uint32_t *__restrict__ flags,
                                                   const unsigned long long *__restrict__ pos,
                                                   unsigned long long *__restrict__ out, uint64_t out_cap,
                                                   DevStats *stats) {
	pdl_begin();
	const unsigned long long P = pos[nc];
	const bool fits = P <= out_cap;
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		stats->pairs = P;
		stats->np_n = fits ? P : 0ull;
	}
	if (!fits) return;
	const uint64_t step = (uint64_t)gridDim.x * kNT;
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < nc; i += step)
		if (flags[i]) out[pos[i]] = cand[i];
}

unsigned grid_for(uint64_t items) {
	return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kNT - 1) / kNT, (uint64_t)kNumSMs * 8));
}
}  // namespace

void launch_vinflate(uint64_t n, const float *aabb, float *scratch, DevStats *stats, float factor, cudaStream_t s) {
	if (n) launch_pdl(k_vinflate, dim3(grid_for(6 * n)), dim3(kNT), 0, s, n, aabb, scratch, stats, factor);
}

void launch_vcheck(uint64_t n, float *aabb, const float *ref, float *backup, const int32_t *T, DevStats *stats,
                   cudaStream_t s) {
	if (n) launch_pdl(k_vcheck, dim3(grid_for(6 * n)), dim3(kNT), 0, s, n, aabb, ref, backup, T, stats);
}

void launch_vfilter(uint64_t nc, const unsigned long long *cand, const float *aabb, uint64_t n, DevStats *stats,
                    uint32_t *flags, bool rebuild, float margin, cudaStream_t s) {
	launch_pdl(k_vfilter, dim3(grid_for(nc)), dim3(kNT), 0, s, nc, cand, aabb, n, stats, flags, rebuild ? 1 : 0, margin);
}

void launch_vscatter(uint64_t nc, const unsigned long long *cand, const uint32_t *flags,
                     const unsigned long long *pos, unsigned long long *out, uint64_t out_cap, DevStats *stats,
                     cudaStream_t s) {
	launch_pdl(k_vscatter, dim3(grid_for(nc)), dim3(kNT), 0, s, nc, cand, flags, pos, out, out_cap, stats);
}

}  // namespace cc
