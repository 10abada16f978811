// Narrowphase: the reference's Narrowphase::DoNarrowphase
// (src/narrowphase/Narrowphase.cu:316-595) as sm_100a kernels.
//
// k_mpr: the MPR state machine of cc_mpr.cuh on persistent lanes fed from a
// queue of pair indices grouped by shape-type combination (k_np_classes).
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
// k_np_classes: the pairs grouped by shape-type class (counting sort), and
// k_np_compact_coop: the stable hit-first ordering of :580-593
// (thrust::sort_by_key on the 0/1 flag) as a scan + scatter, the pair keys
// permuted the same way; each is one cooperative launch with a grid barrier.
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
	pdl_begin();
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

// The class grouping as one cooperative launch: every block counts the classes
// of its pairs (shared-memory histogram, one global atomic per class and
// block), a grid barrier, then every block derives the class offsets (longest
// classes first) and places its pairs, one cursor atomic per class and tile.
constexpr int kCoopNT = 256;
__global__ void __launch_bounds__(kCoopNT) k_np_classes(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n,
                                                         const int32_t *__restrict__ T,
                                                         const long long *__restrict__ pairs, uint32_t *classes,
                                                         uint32_t *__restrict__ order, GridBarrier *bar,
                                                         uint32_t *err) {
	__shared__ uint32_t h[kNpClasses], off[kNpClasses], base[kNpClasses];
	__shared__ int cost[kNpClasses];
	const uint64_t P = P_dev ? min(P_cap, (uint64_t)*P_dev) : P_cap;
	if (threadIdx.x < kNpClasses) h[threadIdx.x] = 0;
	__syncthreads();
	const uint64_t step = (uint64_t)gridDim.x * kCoopNT;
	for (uint64_t i = (uint64_t)blockIdx.x * kCoopNT + threadIdx.x; i < P; i += step)
		atomicAdd(&h[pair_class(i, n, T, pairs)], 1u);
	__syncthreads();
	if (threadIdx.x < kNpClasses && h[threadIdx.x]) atomicAdd(&classes[threadIdx.x], h[threadIdx.x]);
	grid_barrier(bar, err);
	if (threadIdx.x < kNpClasses) {
		h[threadIdx.x] = __ldcg(&classes[threadIdx.x]);
		cost[threadIdx.x] = class_cost(threadIdx.x);
	}
	__syncthreads();
	if (threadIdx.x < kNpClasses) {
		const int c = threadIdx.x, k = cost[c];
		uint32_t acc = 0;
		for (int d = 0; d < kNpClasses; d++)
			if (cost[d] > k || (cost[d] == k && d < c)) acc += h[d];
		off[c] = acc;
	}
	uint32_t *cursor = classes + kNpClasses;
	for (uint64_t i0 = (uint64_t)blockIdx.x * kCoopNT; i0 < P; i0 += step) {
		__syncthreads();
		if (threadIdx.x < kNpClasses) h[threadIdx.x] = 0;
		__syncthreads();
		const uint64_t i = i0 + threadIdx.x;
		uint32_t c = 0, r = 0;
		if (i < P) {
			c = pair_class(i, n, T, pairs);
			r = atomicAdd(&h[c], 1u);
		}
		__syncthreads();
		if (threadIdx.x < kNpClasses && h[threadIdx.x]) base[threadIdx.x] = atomicAdd(&cursor[threadIdx.x], h[threadIdx.x]);
		__syncthreads();
		if (i < P) order[off[c] + base[c] + r] = (uint32_t)i;
	}
}

// Hit-first stable compaction as one cooperative launch: block b owns the
// contiguous chunk b of the flags; it counts its hits, a grid barrier, then it
// adds the counts of the blocks before it and scans its chunk tile by tile,
// writing the exclusive positions (pos, pos[P] = total) and the outputs.
__device__ __forceinline__ void compact_one(uint64_t i, uint64_t P, const NpScratch &sc, long long *__restrict__ pairs,
                                            float *__restrict__ norm, float *__restrict__ cpta,
                                            float *__restrict__ cptb, float *__restrict__ depth,
                                            int32_t *__restrict__ bids, uint64_t before, uint64_t nh);

__global__ void __launch_bounds__(kCoopNT) k_np_compact_coop(uint64_t P_cap, const unsigned long long *P_dev,
                                                              NpScratch sc, long long *__restrict__ pairs,
                                                              float *__restrict__ norm, float *__restrict__ cpta,
                                                              float *__restrict__ cptb, float *__restrict__ depth,
                                                              int32_t *__restrict__ bids,
                                                              unsigned long long *contacts_out) {
	__shared__ unsigned long long sm[40];
	__shared__ unsigned long long s_pre, s_total;
	const uint64_t P = P_dev ? min(P_cap, (uint64_t)*P_dev) : P_cap;
	const uint64_t chunk = (P + gridDim.x - 1) / gridDim.x;
	const uint64_t c0 = min((uint64_t)blockIdx.x * chunk, P), c1 = min(c0 + chunk, P);
	unsigned long long cnt = 0;
	for (uint64_t i = c0 + threadIdx.x; i < c1; i += kCoopNT) cnt += sc.flag[i] ? 1ull : 0ull;
	unsigned long long tot;
	block_excl_scan<unsigned long long, kCoopNT>(cnt, sm, &tot);
	if (threadIdx.x == 0) sc.block_sums[blockIdx.x] = tot;
	grid_barrier(reinterpret_cast<GridBarrier *>(sc.bar_compact), sc.err);
	// prefix of this block and the grand total, from the per-block counts
	unsigned long long pre = 0, all = 0;
	for (uint32_t b = threadIdx.x; b < gridDim.x; b += kCoopNT) {
		const unsigned long long v = __ldcg(&sc.block_sums[b]);
		all += v;
		if (b < blockIdx.x) pre += v;
	}
	{
		unsigned long long t1, t2;
		const unsigned long long p0 = block_excl_scan<unsigned long long, kCoopNT>(pre, sm, &t1);
		const unsigned long long a0 = block_excl_scan<unsigned long long, kCoopNT>(all, sm, &t2);
		(void)p0;
		(void)a0;
		if (threadIdx.x == 0) {
			s_pre = t1;
			s_total = t2;
		}
	}
	__syncthreads();
	unsigned long long run = s_pre;
	const unsigned long long nh = s_total;
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		sc.pos[P] = nh;
		if (contacts_out) *contacts_out = nh;
	}
	for (uint64_t t0 = c0; t0 < c1; t0 += kCoopNT) {
		const uint64_t i = t0 + threadIdx.x;
		const unsigned long long f = (i < c1 && sc.flag[i]) ? 1ull : 0ull;
		unsigned long long tile_total;
		const unsigned long long ex = block_excl_scan<unsigned long long, kCoopNT>(f, sm, &tile_total);
		if (i < c1) {
			const uint64_t before = run + ex;
			sc.pos[i] = before;
			compact_one(i, P, sc, pairs, norm, cpta, cptb, depth, bids, before, nh);
		}
		run += tile_total;
	}
}

// The overlapped narrowphase's compaction (one cooperative launch): the MPR
// ran on the unsorted pairs, so each sorted key finds its result through the
// contact hash. Phase 1: block b copies its chunk of sorted keys to `tmp`,
// looks each one up and counts its hits; grid barrier; phase 2: it adds the
// counts of the blocks before it and writes the hit-first order and the
// contacts, as k_np_compact_coop does for results in sorted order.
__device__ __forceinline__ uint32_t hash_find(const NpScratch &sc, unsigned long long key) {
	const unsigned long long tag = key + 1ull;
	uint64_t h = (tag * 0x9E3779B97F4A7C15ull) >> 20;
	for (uint64_t probe = 0; probe <= sc.hmask && probe < 256; probe++, h++) {
		const unsigned long long v = __ldcg(&sc.hkeys[h & sc.hmask]);
		if (v == tag) return __ldcg(&sc.hvals[h & sc.hmask]);
		if (v == 0ull) break;
	}
	return 0xffffffffu;
}

__global__ void __launch_bounds__(kCoopNT) k_np_compact_sorted(uint64_t P_cap, const unsigned long long *P_dev,
                                                                NpScratch sc, long long *__restrict__ pairs,
                                                                unsigned long long *__restrict__ tmp,
                                                                float *__restrict__ norm, float *__restrict__ cpta,
                                                                float *__restrict__ cptb, float *__restrict__ depth,
                                                                int32_t *__restrict__ bids,
                                                                unsigned long long *contacts_out) {
	__shared__ unsigned long long sm[40];
	__shared__ unsigned long long s_pre, s_total;
	const uint64_t P = P_dev ? min(P_cap, (uint64_t)*P_dev) : P_cap;
	const uint64_t chunk = (P + gridDim.x - 1) / gridDim.x;
	const uint64_t c0 = min((uint64_t)blockIdx.x * chunk, P), c1 = min(c0 + chunk, P);
	unsigned long long cnt = 0;
	for (uint64_t i = c0 + threadIdx.x; i < c1; i += kCoopNT) {
		const unsigned long long key = (unsigned long long)pairs[i];
		tmp[i] = key;
		const uint32_t t = hash_find(sc, key);
		sc.order[i] = t;
		cnt += t != 0xffffffffu ? 1ull : 0ull;
	}
	unsigned long long tot;
	block_excl_scan<unsigned long long, kCoopNT>(cnt, sm, &tot);
	if (threadIdx.x == 0) sc.block_sums[blockIdx.x] = tot;
	grid_barrier(reinterpret_cast<GridBarrier *>(sc.bar_compact), sc.err);
	{
		unsigned long long pre = 0, all = 0, t1, t2;
		for (uint32_t b = threadIdx.x; b < gridDim.x; b += kCoopNT) {
			const unsigned long long v = __ldcg(&sc.block_sums[b]);
			all += v;
			if (b < blockIdx.x) pre += v;
		}
		block_excl_scan<unsigned long long, kCoopNT>(pre, sm, &t1);
		block_excl_scan<unsigned long long, kCoopNT>(all, sm, &t2);
		if (threadIdx.x == 0) {
			s_pre = t1;
			s_total = t2;
		}
		__syncthreads();
	}
	unsigned long long run = s_pre;
	const unsigned long long nh = s_total;
	if (blockIdx.x == 0 && threadIdx.x == 0 && contacts_out) *contacts_out = nh;
	for (uint64_t t0 = c0; t0 < c1; t0 += kCoopNT) {
		const uint64_t i = t0 + threadIdx.x;
		const uint32_t t = i < c1 ? sc.order[i] : 0xffffffffu;
		const unsigned long long f = t != 0xffffffffu ? 1ull : 0ull;
		unsigned long long tile_total;
		const unsigned long long ex = block_excl_scan<unsigned long long, kCoopNT>(f, sm, &tile_total);
		if (i < c1) {
			const uint64_t before = run + ex;
			if (f) {
				const uint64_t j = before;
				pairs[j] = (long long)tmp[i];
				for (int d = 0; d < 3; d++) {
					norm[3 * j + d] = sc.norm[3 * (uint64_t)t + d];
					cpta[3 * j + d] = sc.pa[3 * (uint64_t)t + d];
					cptb[3 * j + d] = sc.pb[3 * (uint64_t)t + d];
				}
				depth[j] = sc.depth[t];
				bids[2 * j] = sc.ids[2 * (uint64_t)t];
				bids[2 * j + 1] = sc.ids[2 * (uint64_t)t + 1];
			} else {
				pairs[nh + (i - before)] = (long long)tmp[i];
			}
		}
		run += tile_total;
	}
}

__device__ __forceinline__ void compact_one(uint64_t i, uint64_t P, const NpScratch &sc, long long *__restrict__ pairs,
                                            float *__restrict__ norm, float *__restrict__ cpta,
                                            float *__restrict__ cptb, float *__restrict__ depth,
                                            int32_t *__restrict__ bids, uint64_t before, uint64_t nh) {
	(void)P;
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

// Largest co-resident grid of a cooperative kernel of kCoopNT threads.
template <class K>
unsigned coop_blocks(K kernel) {
	int per_sm = 0, dev = 0, sms = kNumSMs;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kCoopNT, 0) != cudaSuccess || per_sm < 1)
		per_sm = 1;
	if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return (unsigned)(per_sm * sms);
}

template <class... A>
void launch_coop(void (*k)(A...), unsigned grid, cudaStream_t s, A... args) {
	void *ptrs[] = {(void *)&args...};
	cudaLaunchCooperativeKernel((const void *)k, dim3(grid), dim3(kCoopNT), ptrs, 0, s);
}
}  // namespace

unsigned np_coop_max_blocks() {
	static const unsigned m = std::min(std::min(coop_blocks(k_np_classes), coop_blocks(k_np_compact_coop)),
	                                   coop_blocks(k_np_compact_sorted));
	return m;
}

void launch_mpr(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T, const float *A,
                const float *B, const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                const uint8_t *active, const float *pos, const float *rot, float envelope, const long long *pairs,
                const NpScratch &sc, int precision, uint64_t P_hint, cudaStream_t s) {
	if (!P_cap) return;
	const uint64_t Pe = std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap);
	{  // group the pairs by shape-type combination; the last word is the work queue
		// blocks for the expected pair count (the loops stride over the device count)
		const unsigned g = (unsigned)std::max<uint64_t>(
		    1, std::min<uint64_t>((Pe + kCoopNT - 1) / kCoopNT, std::min<uint64_t>(np_coop_max_blocks(), kNpCoopBlocks)));
		if (!sc.pre_zeroed) cudaMemsetAsync(sc.classes, 0, (2 * kNpClasses + 1) * sizeof(uint32_t), s);
		launch_coop(k_np_classes, g, s, P_cap, P_dev, n, T, pairs, sc.classes, sc.order,
		            reinterpret_cast<GridBarrier *>(sc.bar_classes), sc.err);
	}
	// persistent lanes: one per pair up to the resident limit, so that every
	// pair starts at once (the kernel is latency-bound: its time is the
	// longest pair's dependency chain); beyond that the queue balances
	const uint64_t want = (Pe + kNT - 1) / kNT;
	const unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(want, kNumSMs),
	                                                   (uint64_t)kNumSMs * mpr_resident_blocks(precision));
	if (precision == 0)
		launch_mpr_exact(grid, P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc, s);
	else if (precision == 2)
		launch_pdl(k_mpr<float>, dim3(grid), dim3(kNT), 0, s, P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs,
		                                  sc);
	else
		launch_pdl(k_mpr<double>, dim3(grid), dim3(kNT), 0, s, P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs,
		                                   sc);
}

void launch_np_compact(uint64_t P_cap, const unsigned long long *P_dev, const NpScratch &sc, long long *pairs,
                       float *norm, float *cpta, float *cptb, float *depth, int32_t *bids,
                       unsigned long long *contacts_out, uint64_t P_hint, cudaStream_t s) {
	if (!P_cap) {
		cudaMemsetAsync(sc.pos, 0, sizeof(unsigned long long), s);
		if (contacts_out) cudaMemsetAsync(contacts_out, 0, sizeof(unsigned long long), s);
		return;
	}
	// one block per 256 flags of the expected count (one tile each: the scan
	// and scatter of a tile are a chain of dependent loads), within the co-resident limit
	const uint64_t Pe = std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap);
	const unsigned grid = (unsigned)std::max<uint64_t>(
	    1, std::min<uint64_t>((Pe + kCoopNT - 1) / kCoopNT, std::min<uint64_t>(np_coop_max_blocks(), kNpCoopBlocks)));
	launch_coop(k_np_compact_coop, grid, s, P_cap, P_dev, sc, pairs, norm, cpta, cptb, depth, bids, contacts_out);
}

void launch_np_compact_sorted(uint64_t P_cap, const unsigned long long *P_dev, const NpScratch &sc,
                              long long *pairs, unsigned long long *tmp, float *norm, float *cpta, float *cptb,
                              float *depth, int32_t *bids, unsigned long long *contacts_out, uint64_t P_hint,
                              cudaStream_t s) {
	if (!P_cap) {
		if (contacts_out) cudaMemsetAsync(contacts_out, 0, sizeof(unsigned long long), s);
		return;
	}
	const uint64_t Pe = std::min<uint64_t>(P_hint ? P_hint : P_cap, P_cap);
	const unsigned grid = (unsigned)std::max<uint64_t>(
	    1, std::min<uint64_t>((Pe + kCoopNT - 1) / kCoopNT, std::min<uint64_t>(np_coop_max_blocks(), kNpCoopBlocks)));
	launch_coop(k_np_compact_sorted, grid, s, P_cap, P_dev, sc, pairs, tmp, norm, cpta, cptb, depth, bids,
	            contacts_out);
}

}  // namespace cc
