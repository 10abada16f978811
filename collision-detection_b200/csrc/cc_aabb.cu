// AABB generation: AABBGenerator::GenerateAABB of the reference
// (src/aabb/AABBGenerator.cu:84-188) as one sm_100a kernel, one thread per
// shape, optionally fused with the broadphase's first pass (scene bounds,
// extent sums and input validation) so the pipeline reads each shape once.
// Compiled with -fmad=false: results are bit-identical to the reference's
// host build.
#include <algorithm>

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
	// A zero local offset rotates to (+-0, +-0, +-0) and an identity local
	// rotation leaves body_rot unchanged up to the sign of zero terms; neither
	// sign survives (p +- r rounds the same, |R| drops it), so skipping that
	// arithmetic gives bit-identical boxes.
	const bool a_zero = a.x == 0.f && a.y == 0.f && a.z == 0.f;
	const bool r_ident = lrot.x == 1.f && lrot.y == 0.f && lrot.z == 0.f && lrot.w == 0.f;
	if (type == SPHERE) {  // :96-98, ComputeAABBSphere :11-14
		const float3 p = a_zero ? position : qrot(a, brot) + position;
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
		const Rot m = rot_rows(r_ident ? brot : qmul(brot, lrot));
		const float3 half = f3(dot(abs3(m.r0), b), dot(abs3(m.r1), b), dot(abs3(m.r2), b));
		const float3 p = a_zero ? position : qrot(a, brot) + position;
		mn = p - half;
		mx = p + half;
		return true;
	}
	return false;
}

// Persistent: each thread walks shapes blockIdx*kNT + tid, step gridDim*kNT,
// keeping its share of the bounds in registers, so the block reduces once.
template <bool kStats>
__global__ void __launch_bounds__(kNT) k_aabb(uint64_t n, const int32_t *__restrict__ T, const float *__restrict__ A,
                                               const float *__restrict__ B, const float *__restrict__ C,
                                               const float *__restrict__ R, const uint32_t *__restrict__ ID,
                                               uint64_t nb, const float *__restrict__ pos,
                                               const float *__restrict__ rot, float *__restrict__ aabb,
                                               DevStats *stats, uint32_t *err, PlanArgs pa, ZeroList zero) {
	pdl_begin();
	zero_ranges(zero);
	float3 bmn = f3(INFINITY, INFINITY, INFINITY), bmx = f3(-INFINITY, -INFINITY, -INFINITY);
	float3 esum = f3(0.f, 0.f, 0.f);  // extent sum for the grid tuner's mean box size
	bool have = false;
	uint32_t e = 0, ecnt = 0;
	for (uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kNT) {
		float3 mn, mx;
		if (shape_aabb(i, T, A, B, C, R, ID, nb, pos, rot, mn, mx, err)) {
			float *o = aabb + 3 * i, *o2 = aabb + 3 * (i + n);
			o[0] = mn.x; o[1] = mn.y; o[2] = mn.z;
			o2[0] = mx.x; o2[1] = mx.y; o2[2] = mx.z;
		} else if (kStats) {  // skipped shape: the broadphase sees the caller's old values
			const float *o = aabb + 3 * i, *o2 = aabb + 3 * (i + n);
			mn = f3(o[0], o[1], o[2]);
			mx = f3(o2[0], o2[1], o2[2]);
		}
		if constexpr (kStats) {
			if (!finite3(mn) || !finite3(mx)) e |= kErrNonFinite;
			if (mn.x > mx.x || mn.y > mx.y || mn.z > mx.z) e |= kErrInverted;
			bmn = f3(fminf(bmn.x, mn.x), fminf(bmn.y, mn.y), fminf(bmn.z, mn.z));
			bmx = f3(fmaxf(bmx.x, mx.x), fmaxf(bmx.y, mx.y), fmaxf(bmx.z, mx.z));
			esum = esum + (mx - mn);
			ecnt++;
			have = true;
		}
	}
	if constexpr (kStats) accumulate_stats<kNT>(bmn, bmx, have, stats, pa, e, esum, ecnt);
}
template <class K>
int resident_blocks(K kernel) {
	int b = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kNT, 0) != cudaSuccess || b < 1) b = 1;
	return b;
}
}  // namespace

void launch_aabb(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                 const uint32_t *ID, uint64_t nb, const float *pos, const float *rot, float *aabb, DevStats *stats,
                 uint32_t *err, const GridParams &gp, const int grid[3], cudaStream_t s, const ZeroList &zero) {
	if (n == 0) return;
	// persistent grid: as many blocks as are resident at once
	static const int per_sm[2] = {resident_blocks(k_aabb<false>), resident_blocks(k_aabb<true>)};
	const unsigned blocks =
	    (unsigned)std::min<uint64_t>((n + kNT - 1) / kNT, (uint64_t)kNumSMs * per_sm[stats ? 1 : 0]);
	PlanArgs pa;
	pa.gp = gp;
	pa.gx = grid ? grid[0] : 1;
	pa.gy = grid ? grid[1] : 1;
	pa.gz = grid ? grid[2] : 1;
	pa.n = n;
	if (stats)
		launch_pdl(k_aabb<true>, dim3(blocks), dim3(kNT), 0, s, n, T, A, B, C, R, ID, nb, pos, rot, aabb, stats, err, pa, zero);
	else
		launch_pdl(k_aabb<false>, dim3(blocks), dim3(kNT), 0, s, n, T, A, B, C, R, ID, nb, pos, rot, aabb, nullptr, err, pa, zero);
}

}  // namespace cc
