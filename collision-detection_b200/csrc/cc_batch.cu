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

// Gathers scenes held in separate allocations into the concatenated layout:
// one thread per shape (kBodies false) or per body (true).
template <bool kBodies>
__global__ void __launch_bounds__(kNT) k_gather(uint64_t n, uint32_t S, const unsigned long long *off,
                                                 const SceneSrc *src, SceneDst dst) {
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kNT) {
		const uint32_t s = scene_lookup(off, S, i);
		const uint64_t j = i - __ldg(off + s);
		const SceneSrc &c = src[s];
		if constexpr (kBodies) {
			for (int d = 0; d < 3; d++) dst.pos[3 * i + d] = c.pos[3 * j + d];
			reinterpret_cast<float4 *>(dst.rot)[i] = reinterpret_cast<const float4 *>(c.rot)[j];
			dst.active[i] = c.active[j];
		} else {
			dst.T[i] = c.T[j];
			for (int d = 0; d < 3; d++) {
				dst.A[3 * i + d] = c.A[3 * j + d];
				dst.B[3 * i + d] = c.B[3 * j + d];
				dst.C[3 * i + d] = c.C[3 * j + d];
			}
			reinterpret_cast<float4 *>(dst.R)[i] = reinterpret_cast<const float4 *>(c.R)[j];
			dst.ID[i] = c.ID[j];
		}
	}
}

// The third shape array (C) of the shapes that read it: CONE, which GenerateAABB
// bounds as a triangle (AABBGenerator.cu:103-107), and TRIANGLEMESH, whose
// third vertex the support map and centre use (Narrowphase.cu:11-17, 44-47).
// `src` is the caller's pinned host array, read through its device mapping, so
// a scene without such shapes moves none of its bytes over PCIe.
__global__ void __launch_bounds__(kNT) k_gather_c(uint64_t n, const int32_t *__restrict__ T,
                                                   const float *__restrict__ src, float *__restrict__ dst) {
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kNT) {
		const int t = __ldg(T + i);
		if (t == CONE || t == TRIANGLEMESH) {
			const float x = src[3 * i], y = src[3 * i + 1], z = src[3 * i + 2];
			dst[3 * i] = x;
			dst[3 * i + 1] = y;
			dst[3 * i + 2] = z;
		}
	}
}

// Counter-based random numbers for the time-step update: SplitMix64's output
// function (Steele, Lea, Flood 2014) applied to seed + counter, so every body
// draws the same numbers whatever the launch shape.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}
__device__ __forceinline__ float unit_open(uint64_t h) {  // (0, 1)
	return ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
}
// Two standard normals by the Box-Muller transform (Box and Muller, 1958).
__device__ __forceinline__ float2 normal2(uint64_t key) {
	const float u1 = unit_open(mix64(key)), u2 = unit_open(mix64(key ^ 0x5851f42d4c957f2dull));
	const float r = sqrtf(-2.0f * logf(u1));
	float s, c;
	sincosf(6.283185307179586f * u2, &s, &c);
	return make_float2(r * c, r * s);
}

// pos += N(0, sigma^2); rot = normalize(dq * rot), dq = (cos(a/2), u sin(a/2))
// with u uniform on the sphere and a ~ U[0, max_angle]. Quaternions (w,x,y,z).
// Body i of a scene updated with `seed` (the random numbers are a function of
// (seed, i) alone).
__device__ __forceinline__ void perturb_one(float *__restrict__ pos, float *__restrict__ rot, uint64_t i,
                                            uint64_t seed, float sigma, float max_angle) {
	{
		const uint64_t key = mix64(seed) + 8 * i;
		const float2 n01 = normal2(key), n23 = normal2(key + 1), n45 = normal2(key + 2);
		pos[3 * i] += sigma * n01.x;
		pos[3 * i + 1] += sigma * n01.y;
		pos[3 * i + 2] += sigma * n23.x;
		float ux = n23.y, uy = n45.x, uz = n45.y;
		const float ul = sqrtf(ux * ux + uy * uy + uz * uz);
		if (ul > 0.f) {
			ux /= ul; uy /= ul; uz /= ul;
		} else {
			ux = 1.f; uy = 0.f; uz = 0.f;
		}
		const float h = 0.5f * max_angle * unit_open(mix64(key + 3));
		float sh, ch;
		sincosf(h, &sh, &ch);
		const float bx = ux * sh, by = uy * sh, bz = uz * sh;
		float4 q = reinterpret_cast<float4 *>(rot)[i];
		float4 r;
		r.x = ch * q.x - bx * q.y - by * q.z - bz * q.w;
		r.y = ch * q.y + bx * q.x + by * q.w - bz * q.z;
		r.z = ch * q.z - bx * q.w + by * q.x + bz * q.y;
		r.w = ch * q.w + bx * q.z - by * q.y + bz * q.x;
		const float rl = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
		reinterpret_cast<float4 *>(rot)[i] = make_float4(r.x / rl, r.y / rl, r.z / rl, r.w / rl);
	}
}

__global__ void __launch_bounds__(kNT) k_perturb(uint64_t nb, float *__restrict__ pos, float *__restrict__ rot,
                                                  uint64_t seed, float sigma, float max_angle) {
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < nb; i += (uint64_t)gridDim.x * kNT)
		perturb_one(pos, rot, i, seed, sigma, max_angle);
}

// Several scenes in one launch: the bodies of all scenes as one index range,
// scene k owning [d[k].first, d[k].first + d[k].nb) (found by binary search).
__global__ void __launch_bounds__(kNT) k_perturb_scenes(uint32_t count, uint64_t total,
                                                         const PerturbScene *__restrict__ d, float sigma,
                                                         float max_angle) {
	for (uint64_t g = (uint64_t)blockIdx.x * kNT + threadIdx.x; g < total; g += (uint64_t)gridDim.x * kNT) {
		uint32_t lo = 0, hi = count;  // last scene with first <= g
		while (hi - lo > 1) {
			const uint32_t mid = (lo + hi) >> 1;
			if (d[mid].first <= g) lo = mid;
			else hi = mid;
		}
		const PerturbScene sc = d[lo];
		perturb_one(sc.pos, sc.rot, g - sc.first, sc.seed, sigma, max_angle);
	}
}
}  // namespace

// Small host tables go to the device inside kernel parameters: the driver
// copies a launch's parameters with the launch, so the table needs no copy
// engine and no staging of pageable memory, and cannot queue behind bulk
// uploads running on another stream.
struct ParamChunk {
	uint32_t words[kParamChunkBytes / 4];
};
__global__ void k_param_copy(uint32_t *__restrict__ dst, uint32_t nwords, ParamChunk c) {
	for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = c.words[i];
}

cudaError_t copy_small_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) {
	if (bytes > kParamCopyMax || (bytes & 3) || (reinterpret_cast<uintptr_t>(dst) & 3))
		return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
	const unsigned char *from = static_cast<const unsigned char *>(src);
	uint32_t *to = static_cast<uint32_t *>(dst);
	for (size_t off = 0; off < bytes; off += kParamChunkBytes) {
		const size_t n = std::min<size_t>(kParamChunkBytes, bytes - off);
		ParamChunk c;
		memcpy(c.words, from + off, n);
		k_param_copy<<<1, 256, 0, s>>>(to + off / 4, (uint32_t)(n / 4), c);
	}
	return cudaGetLastError();
}

void launch_perturb_scenes(uint32_t count, uint64_t total, const PerturbScene *d, float sigma, float max_angle,
                           cudaStream_t s) {
	if (!count || !total) return;
	const unsigned g = (unsigned)std::min<uint64_t>((total + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
	k_perturb_scenes<<<g, kNT, 0, s>>>(count, total, d, sigma, max_angle);
}

void launch_perturb(uint64_t nb, float *pos, float *rot, uint64_t seed, float sigma, float max_angle, cudaStream_t s) {
	if (!nb) return;
	const unsigned g = (unsigned)std::min<uint64_t>((nb + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
	k_perturb<<<g, kNT, 0, s>>>(nb, pos, rot, seed, sigma, max_angle);
}

void launch_gather(uint64_t n, uint64_t nb, uint32_t S, const unsigned long long *shape_off,
                   const unsigned long long *body_off, const SceneSrc *src, const SceneDst &dst, cudaStream_t s) {
	if (n) {
		const unsigned g = (unsigned)std::min<uint64_t>((n + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
		k_gather<false><<<g, kNT, 0, s>>>(n, S, shape_off, src, dst);
	}
	if (nb) {
		const unsigned g = (unsigned)std::min<uint64_t>((nb + kNT - 1) / kNT, (uint64_t)kNumSMs * 16);
		k_gather<true><<<g, kNT, 0, s>>>(nb, S, body_off, src, dst);
	}
}

void launch_gather_c(uint64_t n, const int32_t *T, const float *src, float *dst, cudaStream_t s) {
	if (!n) return;
	const unsigned g = (unsigned)std::min<uint64_t>((n + kNT - 1) / kNT, (uint64_t)kNumSMs * 8);
	k_gather_c<<<g, kNT, 0, s>>>(n, T, src, dst);
}

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
