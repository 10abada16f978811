// AABB generation: AABBGenerator::GenerateAABB of the reference
// (src/aabb/AABBGenerator.cu:84-188) as one sm_100a kernel, one thread per
// shape, optionally fused with the broadphase's first pass (scene bounds,
// extent sums and input validation) so the pipeline reads each shape once.
// Compiled with -fmad=false: results are bit-identical to the reference's
// host build.
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"
#include "cc_stats.cuh"

namespace cc {

namespace {
constexpr int kNT = 256;

__device__ __forceinline__ float3 ld3(const float *p, uint64_t i) {
	return f3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
__device__ __forceinline__ float4 ld4(const float *p, uint64_t i) {
	return __ldg(reinterpret_cast<const float4 *>(p) + i);
}
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }  // std::max

// function_ComputeAABB (AABBGenerator.cu:84-116). Returns false for the types
// the reference skips (:110-111): nothing is written for them.
__device__ __forceinline__ bool shape_aabb(uint64_t i, const int32_t *T, const float *A, const float *B,
                                           const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                                           const float *pos, const float *rot, float3 &mn, float3 &mx,
                                           uint32_t *err) {
	const int type = __ldg(T + i);
	const uint32_t id = __ldg(ID + i);
	if (id >= nb) {
		atomicOr(err, (uint32_t)kErrBadIndex);
		return false;
	}
	float3 a = ld3(A, i), b = ld3(B, i);
	const float3 position = ld3(pos, id);
	const float4 brot = ld4(rot, id);
	const float4 lrot = ld4(R, i);
	if (type == SPHERE) {  // :96-98, ComputeAABBSphere :11-14
		const float3 p = qrot(a, brot) + position;
		const float3 r = f3(b.x, b.x, b.x);
		mn = p - r;
		mx = p + r;
		return true;
	}
	if (type == CONE) {  // :103-107: the reference treats type 5 as a triangle
		const float4 rotation = qmul(brot, lrot);
		const float3 c = ld3(C, i);
		a = qrot(a + position, rotation);
		b = qrot(b + position, rotation);
		const float3 cc = qrot(c + position, rotation);
		mn = f3(smin(a.x, smin(b.x, cc.x)), smin(a.y, smin(b.y, cc.y)), smin(a.z, smin(b.z, cc.z)));
		mx = f3(smax(a.x, smax(b.x, cc.x)), smax(a.y, smax(b.y, cc.y)), smax(a.z, smax(b.z, cc.z)));
		return true;
	}
	if (type == ELLIPSOID || type == BOX || type == CYLINDER) {  // :108-109, ComputeAABBBox :25-35
		const Rot m = rot_rows(qmul(brot, lrot));
		const float3 half = f3(dot(abs3(m.r0), b), dot(abs3(m.r1), b), dot(abs3(m.r2), b));
		const float3 p = qrot(a, brot) + position;
		mn = p - half;
		mx = p + half;
		return true;
	}
	return false;
}

template <bool kStats>
__global__ void __launch_bounds__(kNT) k_aabb(uint64_t n, const int32_t *__restrict__ T, const float *__restrict__ A,
                                               const float *__restrict__ B, const float *__restrict__ C,
                                               const float *__restrict__ R, const uint32_t *__restrict__ ID,
                                               uint64_t nb, const float *__restrict__ pos,
                                               const float *__restrict__ rot, float *__restrict__ aabb,
                                               DevStats *stats, uint32_t *err, PlanArgs pa) {
	const uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	float3 mn = f3(INFINITY, INFINITY, INFINITY), mx = f3(-INFINITY, -INFINITY, -INFINITY);
	bool have = false;
	if (i < n) {
		if (shape_aabb(i, T, A, B, C, R, ID, nb, pos, rot, mn, mx, err)) {
			float *o = aabb + 3 * i, *o2 = aabb + 3 * (i + n);
			o[0] = mn.x; o[1] = mn.y; o[2] = mn.z;
			o2[0] = mx.x; o2[1] = mx.y; o2[2] = mx.z;
		} else if (kStats) {  // skipped shape: the broadphase sees the caller's old values
			const float *o = aabb + 3 * i, *o2 = aabb + 3 * (i + n);
			mn = f3(o[0], o[1], o[2]);
			mx = f3(o2[0], o2[1], o2[2]);
		}
		have = true;
	}
	if constexpr (kStats) accumulate_stats<kNT>(mn, mx, have, stats, pa);
}
}  // namespace

void launch_aabb(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                 const uint32_t *ID, uint64_t nb, const float *pos, const float *rot, float *aabb, DevStats *stats,
                 uint32_t *err, const GridParams &gp, const int grid[3], cudaStream_t s) {
	if (n == 0) return;
	const unsigned blocks = (unsigned)((n + kNT - 1) / kNT);
	PlanArgs pa;
	pa.gp = gp;
	pa.gx = grid ? grid[0] : 1;
	pa.gy = grid ? grid[1] : 1;
	pa.gz = grid ? grid[2] : 1;
	pa.n = n;
	if (stats)
		k_aabb<true><<<blocks, kNT, 0, s>>>(n, T, A, B, C, R, ID, nb, pos, rot, aabb, stats, err, pa);
	else
		k_aabb<false><<<blocks, kNT, 0, s>>>(n, T, A, B, C, R, ID, nb, pos, rot, aabb, nullptr, err, pa);
}

}  // namespace cc
