// Batched scenes: many independent scenes collided by one pass of the
// pipeline. The batch is laid out as one concatenated scene (shapes
// [shape_off[s], shape_off[s+1]) and bodies [body_off[s], body_off[s+1]) of
// scene s); each scene gets the bounds, reference shift and search grid that
// a separate call would give it (Broadphase.cu:368-386 per scene), and the
// scenes' grids occupy disjoint global cell ranges, so no pair crosses scenes
// and every scene's pairs, shifted boxes and contacts equal those of a
// separate call. These kernels are the batch prologue (scene lookup, global
// body ids, per-scene bounds and plans) and epilogue (per-scene counts); the
// count, scatter and pair-test kernels take the SceneMap built here.
//
// Compiled with -fmad=false, like the single-scene bounds pass.
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"
#include "cc_stats.cuh"

namespace cc {

namespace {
constexpr int kNT = 256;

__device__ __forceinline__ uint32_t scene_lookup(const unsigned long long *off, uint32_t S, uint64_t i) {
	// largest s with off[s] <= i (off is nondecreasing, off[0] = 0, off[S] = n)
	uint32_t lo = 0, hi = S;
	while (hi - lo > 1) {
		const uint32_t mid = (lo + hi) >> 1;
		if (__ldg(off + mid) <= i) lo = mid;
		else hi = mid;
	}
	return lo;
}

// Scene of every shape and its global body id (ID[i] is local to the scene).
// A local id outside the scene's bodies becomes an id no body has, which the
// AABB kernel reports as kErrBadIndex.
__global__ void __launch_bounds__(kNT) k_batch_prep(uint64_t n, uint32_t S, const unsigned long long *shape_off,
                                                     const unsigned long long *body_off,
                                                     const uint32_t *__restrict__ ID, uint32_t *__restrict__ scene_of,
                                                     uint32_t *__restrict__ gid, uint32_t *err) {
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kNT) {
		const uint32_t s = scene_lookup(shape_off, S, i);
		scene_of[i] = s;
		const unsigned long long b0 = __ldg(body_off + s), nb_s = __ldg(body_off + s + 1) - b0;
		const uint32_t id = __ldg(ID + i);
		if ((unsigned long long)id >= nb_s) {
			atomicOr(err, (uint32_t)kErrBadIndex);
			gid[i] = 0xffffffffu;
		} else {
			gid[i] = (uint32_t)(b0 + id);
		}
	}
}

// Per-scene bounds, extent sums and validity of the (unshifted) AABBs. Warps
// whose shapes all belong to one scene reduce first (the common case).
__global__ void __launch_bounds__(kNT) k_batch_bounds(uint64_t n, const float *__restrict__ aabb,
                                                       const uint32_t *__restrict__ scene_of, SceneStats *sst,
                                                       uint32_t *err) {
	const uint32_t lane = threadIdx.x & 31;
	for (uint64_t base = (uint64_t)blockIdx.x * kNT + (threadIdx.x & ~31u); base < n;
	     base += (uint64_t)gridDim.x * kNT) {
		const uint64_t i = base + lane;
		const bool have = i < n;
		float3 mn = f3(0.f, 0.f, 0.f), mx = mn;
		uint32_t s = 0, e = 0;
		if (have) {
			mn = f3(aabb[3 * i], aabb[3 * i + 1], aabb[3 * i + 2]);
			mx = f3(aabb[3 * (n + i)], aabb[3 * (n + i) + 1], aabb[3 * (n + i) + 2]);
			s = __ldg(scene_of + i);
			if (!finite3(mn) || !finite3(mx)) e |= kErrNonFinite;
			if (mn.x > mx.x || mn.y > mx.y || mn.z > mx.z) e |= kErrInverted;
		}
		uint32_t k[6];
		k[0] = have ? ~f2ord(mn.x) : 0u;  // atomicMax on ~ord = min
		k[1] = have ? ~f2ord(mn.y) : 0u;
		k[2] = have ? ~f2ord(mn.z) : 0u;
		k[3] = have ? f2ord(mx.x) : 0u;
		k[4] = have ? f2ord(mx.y) : 0u;
		k[5] = have ? f2ord(mx.z) : 0u;
		float3 ext = have ? mx - mn : f3(0.f, 0.f, 0.f);
		const uint32_t s0 = __shfl_sync(0xffffffffu, s, 0);
		const bool uniform = __all_sync(0xffffffffu, !have || s == s0);
		if (uniform) {
#pragma unroll
			for (int d = 0; d < 6; d++) k[d] = __reduce_max_sync(0xffffffffu, k[d]);
			e = __reduce_or_sync(0xffffffffu, e);
			const uint32_t cnt = __reduce_add_sync(0xffffffffu, have ? 1u : 0u);
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				ext.x += __shfl_xor_sync(0xffffffffu, ext.x, o);
				ext.y += __shfl_xor_sync(0xffffffffu, ext.y, o);
				ext.z += __shfl_xor_sync(0xffffffffu, ext.z, o);
			}
			if (lane == 0) {
				SceneStats &t = sst[s0];
				for (int d = 0; d < 3; d++) {
					atomicMax(&t.bmin_inv[d], k[d]);
					atomicMax(&t.bmax[d], k[d + 3]);
				}
				atomicAdd(&t.ext_sum[0], (double)ext.x);
				atomicAdd(&t.ext_sum[1], (double)ext.y);
				atomicAdd(&t.ext_sum[2], (double)ext.z);
				atomicAdd(&t.count, (unsigned long long)cnt);
				if (e) {
					atomicOr(&t.err, e);
					atomicOr(err, e);
				}
			}
		} else if (have) {
			SceneStats &t = sst[s];
			for (int d = 0; d < 3; d++) {
				atomicMax(&t.bmin_inv[d], k[d]);
				atomicMax(&t.bmax[d], k[d + 3]);
			}
			atomicAdd(&t.ext_sum[0], (double)ext.x);
			atomicAdd(&t.ext_sum[1], (double)ext.y);
			atomicAdd(&t.ext_sum[2], (double)ext.z);
			atomicAdd(&t.count, 1ull);
			if (e) {
				atomicOr(&t.err, e);
				atomicOr(err, e);
			}
		}
	}
}

// One thread per scene: the plan a separate call would build (make_plan) and
// the scene's cell count G[s].
__global__ void __launch_bounds__(kNT) k_batch_plan(uint32_t S, const unsigned long long *shape_off,
                                                     const SceneStats *sst, GridParams gp, int gx, int gy, int gz,
                                                     Plan *plans, uint32_t *G) {
	const uint32_t s = blockIdx.x * kNT + threadIdx.x;
	if (s >= S) return;
	const uint64_t n_s = shape_off[s + 1] - shape_off[s];
	const SceneStats &t = sst[s];
	Plan p;
	if (n_s == 0) {
		memset(&p, 0, sizeof(p));
		plans[s] = p;
		G[s] = 0;
		return;
	}
	uint32_t bmin_inv[3], bmax[3];
	double ext_mean[3];
	for (int d = 0; d < 3; d++) {
		bmin_inv[d] = t.bmin_inv[d];
		bmax[d] = t.bmax[d];
		ext_mean[d] = t.ext_sum[d] / (double)(t.count ? t.count : 1);
	}
	GridParams g = gp;
	g.g_max = batch_scene_cells(n_s);
	p = make_plan(bmin_inv, bmax, t.err, ext_mean, g, gx, gy, gz, n_s);
	plans[s] = p;
	G[s] = p.valid ? p.G : 0u;
}

// Per-scene results: pairs of scene s (owner buckets of its shapes) and the
// contacts before its first pair in the sorted list.
__global__ void __launch_bounds__(kNT) k_batch_offsets(uint32_t S, const unsigned long long *shape_off,
                                                        const unsigned long long *owner_off,
                                                        const unsigned long long *np_pos, const DevStats *stats,
                                                        unsigned long long *scene_pairs,
                                                        unsigned long long *contact_off) {
	const uint32_t s = blockIdx.x * kNT + threadIdx.x;
	if (s > S) return;
	const bool np_ok = stats->np_n == stats->pairs;
	const unsigned long long p0 = owner_off[shape_off[s]];
	if (s < S) scene_pairs[s] = owner_off[shape_off[s + 1]] - p0;
	contact_off[s] = np_ok ? np_pos[p0] : 0ull;
}
}  // namespace

void launch_batch_prep(uint64_t n, uint32_t S, const unsigned long long *shape_off, const unsigned long long *body_off,
                       const uint32_t *ID, uint32_t *scene_of, uint32_t *gid, uint32_t *err, cudaStream_t s) {
	if (!n) return;
	const unsigned g = (unsigned)std::min<uint64_t>((n + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
	k_batch_prep<<<g, kNT, 0, s>>>(n, S, shape_off, body_off, ID, scene_of, gid, err);
}

void launch_batch_bounds(uint64_t n, const float *aabb, const uint32_t *scene_of, SceneStats *sst, uint32_t *err,
                         cudaStream_t s) {
	if (!n) return;
	const unsigned g = (unsigned)std::min<uint64_t>((n + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
	k_batch_bounds<<<g, kNT, 0, s>>>(n, aabb, scene_of, sst, err);
}

void launch_batch_plan(uint32_t S, const unsigned long long *shape_off, const SceneStats *sst, const GridParams &gp,
                       const int grid[3], Plan *plans, uint32_t *G, cudaStream_t s) {
	k_batch_plan<<<(S + kNT - 1) / kNT, kNT, 0, s>>>(S, shape_off, sst, gp, grid[0], grid[1], grid[2], plans, G);
}

void launch_batch_offsets(uint32_t S, const unsigned long long *shape_off, const unsigned long long *owner_off,
                          const unsigned long long *np_pos, const DevStats *stats, unsigned long long *scene_pairs,
                          unsigned long long *contact_off, cudaStream_t s) {
	k_batch_offsets<<<(S + 1 + kNT - 1) / kNT, kNT, 0, s>>>(S, shape_off, owner_off, np_pos, stats, scene_pairs,
	                                                        contact_off);
}

}  // namespace cc
