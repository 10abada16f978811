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
	const float o0 = origin[0], o1 = origin[1], o2 = origin[2];
	float *hi = aabb + 3 * n;
	const float *rhi = ref + 3 * n;
	const uint64_t step = (uint64_t)gridDim.x * kNT;
	float dmax = 0.f;
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < n; i += step) {  // box i: both corners
		float v[6], r[6];
#pragma unroll
		for (int d = 0; d < 3; d++) {
			v[d] = aabb[3 * i + d];
			v[3 + d] = hi[3 * i + d];
			r[d] = ref[3 * i + d];
			r[3 + d] = rhi[3 * i + d];
		}
#pragma unroll
		for (int k = 0; k < 6; k++) dmax = fmaxf(dmax, fabsf(v[k] - r[k]));
		const int t = __ldg(T + i);
		if (t == RECT || t == TRIANGLEMESH) {
#pragma unroll
			for (int d = 0; d < 3; d++) {
				backup[3 * i + d] = v[d];
				backup[3 * n + 3 * i + d] = v[3 + d];
			}
		}
		aabb[3 * i] = v[0] + o0;
		aabb[3 * i + 1] = v[1] + o1;
		aabb[3 * i + 2] = v[2] + o2;
		hi[3 * i] = v[3] + o0;
		hi[3 * i + 1] = v[4] + o1;
		hi[3 * i + 2] = v[5] + o2;
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

// The candidates that overlap on this step's shifted boxes, in order, into
// out (positions past out_cap are not written): one pass over tiles of
// kVcTile candidates with a decoupled look-back for their offsets (tiles take
// their indices from a ticket, so every tile a tile waits on has started).
// The last tile writes the total (stats->pairs) and stats->np_n (0 when the
// list does not fit out). A rebuild step's own candidates always hold its
// pairs; a kept step that moved too far, or invalid input, passes nothing
// and sets stats->vbad.
constexpr int kVcIPT = 8;
constexpr uint64_t kVcTile = (uint64_t)kNT * kVcIPT;
__global__ void __launch_bounds__(kNT) k_vcompact(uint64_t nc, const unsigned long long *__restrict__ cand,
                                                   const float *__restrict__ aabb, uint64_t n, DevStats *stats,
                                                   unsigned long long *__restrict__ out, uint64_t out_cap,
                                                   uint64_t *status, uint32_t *ticket, int rebuild, float margin) {
	pdl_begin();
	__shared__ uint32_t s_tile;
	__shared__ int s_fits;
	__shared__ unsigned long long s_pre;
	__shared__ unsigned long long sm[40];
	if (threadIdx.x == 0) {
		s_tile = atomicAdd(ticket, 1u);
		s_fits = stats->plan.valid && (rebuild || step_fits(stats, margin));
	}
	__syncthreads();
	const uint32_t tile = s_tile;
	const bool fits = s_fits != 0;
	if (!fits && tile == 0 && threadIdx.x == 0) stats->vbad = 1u;
	const float *mx = aabb + 3 * n;
	const uint64_t i0 = (uint64_t)tile * kVcTile + (uint64_t)threadIdx.x * kVcIPT;
	unsigned long long key[kVcIPT];
	uint32_t keep = 0;  // bit j: candidate i0 + j overlaps
#pragma unroll
	for (int j = 0; j < kVcIPT; j++) {
		key[j] = 0ull;
		const uint64_t i = i0 + j;
		if (fits && i < nc) {
			key[j] = cand[i];
			const uint64_t a = key[j] >> 32, b = key[j] & 0xffffffffull;
			if (a < n && b < n) {
				const float *pa = aabb + 3 * a, *pb = aabb + 3 * b, *qa = mx + 3 * a, *qb = mx + 3 * b;
				if (pa[0] <= qb[0] && pb[0] <= qa[0] && pa[1] <= qb[1] && pb[1] <= qa[1] && pa[2] <= qb[2] &&
				    pb[2] <= qa[2])
					keep |= 1u << j;
			}
		}
	}
	unsigned long long total;
	const unsigned long long excl = block_excl_scan<unsigned long long, kNT>(__popc(keep), sm, &total);
	if (threadIdx.x < 32) {
		const unsigned long long pre = lookback_prefix(status, tile, total, &stats->err);
		if (threadIdx.x == 0) s_pre = pre;
	}
	__syncthreads();
	unsigned long long pos = s_pre + excl;
#pragma unroll
	for (int j = 0; j < kVcIPT; j++)
		if ((keep >> j) & 1u) {
			if (pos < out_cap) out[pos] = key[j];
			pos++;
		}
	if (tile == gridDim.x - 1 && threadIdx.x == 0) {
		const unsigned long long P = s_pre + total;
		stats->pairs = P;
		stats->np_n = P <= out_cap ? P : 0ull;
	}
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
	if (n) launch_pdl(k_vcheck, dim3(grid_for(n)), dim3(kNT), 0, s, n, aabb, ref, backup, T, stats);
}

uint64_t vcompact_status_words(uint64_t nc) { return nc / kVcTile + 2; }

void launch_vcompact(uint64_t nc, const unsigned long long *cand, const float *aabb, uint64_t n, DevStats *stats,
                     unsigned long long *out, uint64_t out_cap, uint64_t *status, uint32_t *ticket, bool rebuild,
                     float margin, cudaStream_t s) {
	const uint64_t tiles = (nc + kVcTile - 1) / kVcTile;
	cudaMemsetAsync(status, 0, sizeof(uint64_t) * vcompact_status_words(nc), s);
	cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s);
	launch_pdl(k_vcompact, dim3((unsigned)std::max<uint64_t>(tiles, 1)), dim3(kNT), 0, s, nc, cand, aabb, n, stats,
	           out, out_cap, status, ticket, rebuild ? 1 : 0, margin);
}

}  // namespace cc
