// Narrowphase: the reference's Narrowphase::DoNarrowphase
// (src/narrowphase/Narrowphase.cu:316-595) as sm_100a kernels.
//
// k_mpr: the MPR state machine of cc_mpr.cuh on persistent lanes fed from a
// queue of pair indices grouped by shape-type combination (k_np_class_*).
// Sphere-sphere pairs take the analytic branch (:382-397); every other pair
// runs Minkowski portal refinement (CollideAndFindPoint :122-314) with the
// same branch structure, iteration caps (35 discovery, 35 refinement) and
// termination rule (delta <= 1e-20, depth <= 0).
//
// Precision (the portal arithmetic is FP64 in all three):
//  0 exact  (cc_mpr_exact.cu, -fmad=false): the reference's arithmetic in
//           double, world frame — equal to the FP64 oracle, rounded to float;
//  1 fp64   (k_mpr<double>): pair-local frame (origin = body A's position),
//           rsqrt normalization, fused multiply-add;
//  2 mixed  (k_mpr<float>): as fp64 with FP32 support maps.
//
// k_np_compact: the stable hit-first ordering of :580-593 (thrust::sort_by_key
// on the 0/1 flag) as a scan + scatter; the pair keys are permuted the same way.
#include <algorithm>

#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"
#include "cc_mpr.cuh"

namespace cc {

namespace {
constexpr int kNT = 64;  // MPR: few, long-running threads; small blocks spread them over all SMs

template <class S>
__global__ void __launch_bounds__(kNT) k_mpr(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n,
                                              const int32_t *__restrict__ T, const float *__restrict__ A,
                                              const float *__restrict__ B, const float *__restrict__ C,
                                              const float *__restrict__ R, const uint32_t *__restrict__ ID,
                                              uint64_t nb, const uint8_t *__restrict__ active,
                                              const float *__restrict__ pos, const float *__restrict__ rot,
                                              float envelope, const long long *__restrict__ pairs, NpScratch sc) {
	mpr::run<S, false, kNT>(P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc,
	                        sc.classes + 2 * kNpClasses);
}

// Pairs grouped by (type A, type B) so that the threads of a warp run the
// same support maps: a counting sort of the pair indices by class.
__device__ __forceinline__ uint32_t pair_class(uint64_t i, uint64_t n, const int32_t *T, const long long *pairs) {
	const uint64_t key = (uint64_t)pairs[i];
	const uint64_t a = key >> 32, b = key & 0xffffffffull;
	if (a >= n || b >= n) return kNpClasses - 1;
	const int ta = __ldg(T + a), tb = __ldg(T + b);
	if (ta < 0 || ta > 6 || tb < 0 || tb > 6) return kNpClasses - 1;
	return (uint32_t)(ta * 7 + tb);
}

// Relative MPR cost of a shape type: smooth surfaces refine longest.
__device__ __forceinline__ int type_cost(int t) {
	switch (t) {
	case SPHERE: return 1;
	case BOX: return 2;
	case CYLINDER: return 3;
	case ELLIPSOID: return 4;
	default: return 2;
	}
}
// Sphere-sphere pairs take the analytic path and invalid pairs do nothing:
// cost 0.
__device__ __forceinline__ int class_cost(int c) {
	if (c >= 49) return 0;
	const int ta = c / 7, tb = c % 7;
	if (ta == SPHERE && tb == SPHERE) return 0;
	return type_cost(ta) + type_cost(tb);
}

__global__ void __launch_bounds__(256) k_np_class_count(uint64_t P, const unsigned long long *P_dev, uint64_t n,
                                                         const int32_t *__restrict__ T,
                                                         const long long *__restrict__ pairs, uint32_t *classes) {
	__shared__ uint32_t h[kNpClasses];
	if (threadIdx.x < kNpClasses) h[threadIdx.x] = 0;
	__syncthreads();
	const uint64_t Pn = P_dev ? min(P, (uint64_t)*P_dev) : P;
	for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < Pn; i += (uint64_t)gridDim.x * 256)
		atomicAdd(&h[pair_class(i, n, T, pairs)], 1u);
	__syncthreads();
	if (threadIdx.x < kNpClasses && h[threadIdx.x]) atomicAdd(&classes[threadIdx.x], h[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_np_class_scatter(uint64_t P, const unsigned long long *P_dev, uint64_t n,
                                                           const int32_t *__restrict__ T,
                                                           const long long *__restrict__ pairs, uint32_t *classes,
                                                           uint32_t *__restrict__ order) {
	// classes in order of descending class_cost (ties by class id), so the
	// longest pairs start first: class c begins after every class ranked
	// before it
	__shared__ uint32_t off[kNpClasses], cnt[kNpClasses];
	__shared__ int cost[kNpClasses];
	if (threadIdx.x < kNpClasses) {
		cnt[threadIdx.x] = classes[threadIdx.x];
		cost[threadIdx.x] = class_cost(threadIdx.x);
	}
	__syncthreads();
	if (threadIdx.x < kNpClasses) {
		const int c = threadIdx.x, k = cost[c];
		uint32_t acc = 0;
		for (int d = 0; d < kNpClasses; d++)
			if (cost[d] > k || (cost[d] == k && d < c)) acc += cnt[d];
		off[c] = acc;
	}
	__syncthreads();
	// per 256-pair tile: ranks within the block from shared-memory counters,
	// then one global cursor reservation per class and block (a few classes
	// hold most pairs, so per-pair global atomics would serialise on them)
	__shared__ uint32_t h[kNpClasses], base[kNpClasses];
	uint32_t *cursor = classes + kNpClasses;
	const uint64_t Pn = P_dev ? min(P, (uint64_t)*P_dev) : P;
	for (uint64_t i0 = (uint64_t)blockIdx.x * 256; i0 < Pn; i0 += (uint64_t)gridDim.x * 256) {
		if (threadIdx.x < kNpClasses) h[threadIdx.x] = 0;
		__syncthreads();
		const uint64_t i = i0 + threadIdx.x;
		uint32_t c = 0, r = 0;
		if (i < Pn) {
			c = pair_class(i, n, T, pairs);
			r = atomicAdd(&h[c], 1u);
		}
		__syncthreads();
		if (threadIdx.x < kNpClasses && h[threadIdx.x]) base[threadIdx.x] = atomicAdd(&cursor[threadIdx.x], h[threadIdx.x]);
		__syncthreads();
		if (i < Pn) order[off[c] + base[c] + r] = (uint32_t)i;
		__syncthreads();
	}
}

__device__ __forceinline__ void compact_one(uint64_t i, uint64_t P, const NpScratch &sc, long long *__restrict__ pairs,
                                            float *__restrict__ norm, float *__restrict__ cpta,
                                            float *__restrict__ cptb, float *__restrict__ depth,
                                            int32_t *__restrict__ bids);

__global__ void __launch_bounds__(256) k_np_compact(uint64_t P_cap, const unsigned long long *P_dev, NpScratch sc,
                                                     long long *__restrict__ pairs, float *__restrict__ norm,
                                                     float *__restrict__ cpta, float *__restrict__ cptb,
                                                     float *__restrict__ depth, int32_t *__restrict__ bids) {
	const uint64_t P = P_dev ? min(P_cap, (uint64_t)*P_dev) : P_cap;
	for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < P; i += (uint64_t)gridDim.x * 256)
		compact_one(i, P, sc, pairs, norm, cpta, cptb, depth, bids);
}

__device__ __forceinline__ void compact_one(uint64_t i, uint64_t P, const NpScratch &sc, long long *__restrict__ pairs,
                                            float *__restrict__ norm, float *__restrict__ cpta,
                                            float *__restrict__ cptb, float *__restrict__ depth,
                                            int32_t *__restrict__ bids) {
	const uint64_t nh = sc.pos[P];
	const uint64_t before = sc.pos[i];
	if (sc.flag[i]) {
		const uint64_t j = before;
		pairs[j] = (long long)sc.pairs[i];
		for (int d = 0; d < 3; d++) {
			norm[3 * j + d] = sc.norm[3 * i + d];
			cpta[3 * j + d] = sc.pa[3 * i + d];
			cptb[3 * j + d] = sc.pb[3 * i + d];
		}
		depth[j] = sc.depth[i];
		bids[2 * j] = sc.ids[2 * i];
		bids[2 * j + 1] = sc.ids[2 * i + 1];
	} else {
		pairs[nh + (i - before)] = (long long)sc.pairs[i];
	}
}
}  // namespace

namespace {
template <class K>
int resident(K kernel) {
	int v = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, kNT, 0) != cudaSuccess || v < 1) v = 1;
	return v;
}
// Blocks of the MPR kernel of a precision mode resident per SM.
int mpr_resident_blocks(int precision) {
	static const int b[3] = {mpr_exact_resident_blocks(), resident(k_mpr<double>), resident(k_mpr<float>)};
	return b[precision == 0 ? 0 : (precision == 2 ? 2 : 1)];
}
}  // namespace

void launch_mpr(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T, const float *A,
                const float *B, const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                const uint8_t *active, const float *pos, const float *rot, float envelope, const long long *pairs,
                const NpScratch &sc, int precision, uint64_t P_hint, cudaStream_t s) {
	if (!P_cap) return;
	{  // group the pairs by shape-type combination; the last word is the work queue
		// blocks for the expected pair count (the loops stride over the device count)
		const uint64_t Pe = std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap);
		const unsigned g = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((Pe + 255) / 256, (uint64_t)kNumSMs * 4));
		if (!sc.pre_zeroed) cudaMemsetAsync(sc.classes, 0, (2 * kNpClasses + 1) * sizeof(uint32_t), s);
		k_np_class_count<<<g, 256, 0, s>>>(P_cap, P_dev, n, T, pairs, sc.classes);
		k_np_class_scatter<<<g, 256, 0, s>>>(P_cap, P_dev, n, T, pairs, sc.classes, sc.order);
	}
	// persistent lanes: one per pair up to the resident limit, so that every
	// pair starts at once (the kernel is latency-bound: its time is the
	// longest pair's dependency chain); beyond that the queue balances
	const uint64_t want = (std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap) + kNT - 1) / kNT;
	const unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(want, kNumSMs),
	                                                   (uint64_t)kNumSMs * mpr_resident_blocks(precision));
	if (precision == 0)
		launch_mpr_exact(grid, P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc, s);
	else if (precision == 2)
		k_mpr<float><<<grid, kNT, 0, s>>>(P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs,
		                                  sc);
	else
		k_mpr<double><<<grid, kNT, 0, s>>>(P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs,
		                                   sc);
}

void launch_np_compact(uint64_t P_cap, const unsigned long long *P_dev, const NpScratch &sc, long long *pairs,
                       float *norm, float *cpta, float *cptb, float *depth, int32_t *bids,
                       unsigned long long *contacts_out, uint64_t P_hint, cudaStream_t s) {
	launch_scan_u32_to_u64(sc.flag, P_cap, sc.pos, sc.status, sc.ticket, sc.err, s, P_dev, contacts_out,
	                       sc.pre_zeroed);
	if (!P_cap) return;
	const uint64_t Pe = std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap);
	const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((Pe + 255) / 256, (uint64_t)kNumSMs * 16));
	k_np_compact<<<grid, 256, 0, s>>>(P_cap, P_dev, sc, pairs, norm, cpta, cptb, depth, bids);
}

}  // namespace cc
