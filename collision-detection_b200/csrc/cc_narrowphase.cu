// Narrowphase: the reference's Narrowphase::DoNarrowphase
// (src/narrowphase/Narrowphase.cu:316-595) as sm_100a kernels.
//
// k_mpr: one thread per candidate pair. Sphere-sphere pairs take the analytic
// branch (:382-397); every other pair runs Minkowski portal refinement
// (CollideAndFindPoint :122-314) with the same branch structure, iteration
// caps (35 discovery, 35 refinement) and termination rule (delta <= 1e-20,
// depth <= 0).
//
// Precision: support maps (SupportFunctions.cuh:11-99 via TransformSupportVert
// :19-52) run in FP32 in a pair-local frame whose origin is body A's position,
// so mm-sized shapes at coordinates ~10 keep ~1e-10 absolute resolution. The
// portal arithmetic (zero tests, orientation signs, face normals, the
// termination test and the barycentric contact point) runs in FP64 on the
// FP32 support points. Contact points are translated back to world
// coordinates at the end.
//
// k_np_compact: the stable hit-first ordering of :580-593 (thrust::sort_by_key
// on the 0/1 flag) as a scan + scatter; the pair keys are permuted the same way.
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"

namespace cc {

namespace {
constexpr int kNT = 128;
constexpr float kEps = 1.1920928955078125e-07f;  // FLT_EPSILON (collision_detection.h:54)

// the FP64 operators below would hide cc's float3 operators otherwise
using cc::operator+;
using cc::operator-;
using cc::operator*;

struct d3 {
	double x, y, z;
};
__device__ __forceinline__ d3 D(float3 a) { return {(double)a.x, (double)a.y, (double)a.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 dcross(d3 a, d3 b) {
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 dnormalize(d3 a) {
	const double l = sqrt(ddot(a, a));
	return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ bool dzero(d3 a) {
	return fabs(a.x) < (double)kEps && fabs(a.y) < (double)kEps && fabs(a.z) < (double)kEps;
}
__device__ __forceinline__ float3 F(d3 a) { return f3((float)a.x, (float)a.y, (float)a.z); }

// A shape placed in the pair-local frame.
struct Shape {
	int type;
	float3 X, Y, Z;  // centre (or triangle vertex 0), parameters B (or vertex 1), C (or vertex 2)
	Rot m;           // rotation body_rot * local_rot (:356-357)
};

// Local support map: SupportFunctions.cuh:11-99.
__device__ __forceinline__ float3 support_local(int type, float3 B, float3 n) {
	switch (type) {
	case SPHERE:
		return B.x * n;
	case ELLIPSOID: {
		const float3 nn = normalize(n);
		return divs(mulv(mulv(B, B), nn), length(mulv(B, nn)));
	}
	case BOX:
		return f3(signf(n.x) * B.x, signf(n.y) * B.y, signf(n.z) * B.z);
	case CYLINDER: {
		const float3 u = f3(0.f, 1.f, 0.f);
		const float3 w = n - dot(u, n) * u;
		const float sy = signf(dot(u, n)) * B.y;
		if (length(w) != 0.f) return sy * u + B.x * normalize(w);
		return sy * u;
	}
	case RECT: {
		float3 r = B;
		if (n.x < 0.f) r.x = -r.x;
		if (n.y < 0.f) r.y = -r.y;
		return r;
	}
	case CONE: {
		const float radius = B.x, height = B.y;
		const float sa = radius / sqrtf(radius * radius + height * height);
		if (n.y > length(n) * sa) return f3(0.f, (float)(height / 2.0), 0.f);
		const float s = sqrtf(n.x * n.x + n.z * n.z);
		if (s > 1e-9f) {
			const float d = radius / s;
			return f3(n.x * d, (float)(-height / 2.0), n.z * d);
		}
		return f3(0.f, (float)(-height / 2.0), 0.f);
	}
	}
	return f3(0.f, 0.f, 0.f);
}

// TransformSupportVert (:19-52): world support point along direction b.
__device__ __forceinline__ float3 support(const Shape &s, d3 b) {
	const float3 n = normalize(F(b));
	if (s.type == TRIANGLEMESH) {
		float dist = dot(s.X, n);
		float3 p = s.X;
		if (dot(s.Y, n) > dist) { dist = dot(s.Y, n); p = s.Y; }
		if (dot(s.Z, n) > dist) { p = s.Z; }
		return p;
	}
	const float3 rn = mat_t_vec(s.m, n);
	return mat_vec(s.m, support_local(s.type, s.Y, rn)) + s.X;
}

__device__ __forceinline__ d3 centre(const Shape &s) {  // GetCenter :11-17
	if (s.type == TRIANGLEMESH)
		return {((double)s.X.x + s.Y.x + s.Z.x) / 3.0, ((double)s.X.y + s.Y.y + s.Z.y) / 3.0,
		        ((double)s.X.z + s.Y.z + s.Z.z) / 3.0};
	return D(s.X);
}

// CollideAndFindPoint (:122-314). Support points are FP32; the portal
// vertices v_i = v_i2 - v_i1 are formed exactly in FP64.
__device__ bool mpr(const Shape &A, const Shape &B, d3 &out_n, d3 &out_p) {
	const d3 v01 = centre(A), v02 = centre(B);
	d3 v0 = v02 - v01;
	if (dzero(v0)) v0 = {1.0, 0.0, 0.0};
	d3 n = -v0;
	float3 v11 = support(A, -n), v12 = support(B, n);
	d3 v1 = D(v12) - D(v11);
	if (ddot(v1, n) <= 0.0) return false;
	n = dcross(v1, v0);
	if (dzero(n)) {
		n = dnormalize(v1 - v0);
		out_n = n;
		out_p = 0.5 * (D(v11) + D(v12));
		return true;
	}
	float3 v21 = support(A, -n), v22 = support(B, n);
	d3 v2 = D(v22) - D(v21);
	if (ddot(v2, n) <= 0.0) return false;
	n = dcross(v1 - v0, v2 - v0);
	if (ddot(n, v0) > 0.0) {
		d3 t = v1; v1 = v2; v2 = t;
		float3 u = v11; v11 = v21; v21 = u;
		u = v12; v12 = v22; v22 = u;
		n = -n;
	}
	float3 v31, v32;
	d3 v3;
	bool hit = false;
	int phase1 = 0, phase2 = 0;
	const int max_iterations = 34;
	while (true) {
		if (phase1 > max_iterations) return false;
		phase1++;
		v31 = support(A, -n);
		v32 = support(B, n);
		v3 = D(v32) - D(v31);
		if (ddot(v3, n) <= 0.0) return false;
		if (ddot(dcross(v1, v3), v0) < 0.0) {
			v2 = v3; v21 = v31; v22 = v32;
			n = dcross(v1 - v0, v3 - v0);
			continue;
		}
		if (ddot(dcross(v3, v2), v0) < 0.0) {
			v1 = v3; v11 = v31; v12 = v32;
			n = dcross(v3 - v0, v2 - v0);
			continue;
		}
		while (true) {
			phase2++;
			n = dnormalize(dcross(v2 - v1, v3 - v1));
			if (ddot(n, v1) >= 0.0 && !hit) hit = true;
			const float3 v41 = support(A, -n), v42 = support(B, n);
			const d3 v4 = D(v42) - D(v41);
			const double delta = ddot(v4 - v3, n);
			const double depth = ddot(v4, n);
			if (delta <= 1e-20 || depth <= 0.0 || phase2 > max_iterations) {
				if (hit) {
					double b0 = ddot(dcross(v1, v2), v3);
					double b1 = ddot(dcross(v3, v2), v0);
					double b2 = ddot(dcross(v0, v1), v3);
					double b3 = ddot(dcross(v2, v1), v0);
					double sum = b0 + b1 + b2 + b3;
					if (sum <= 0.0) {
						b0 = 0.0;
						b1 = ddot(dcross(v2, v3), n);
						b2 = ddot(dcross(v3, v1), n);
						b3 = ddot(dcross(v1, v2), n);
						sum = b1 + b2 + b3;
					}
					const double inv = 1.0 / sum;
					const d3 p = b0 * v01 + b1 * D(v11) + b2 * D(v21) + b3 * D(v31);
					const d3 q = b0 * v02 + b1 * D(v12) + b2 * D(v22) + b3 * D(v32);
					out_p = (0.5 * inv) * (p + q);
					out_n = dnormalize(n);
				}
				return hit;
			}
			if (ddot(dcross(v4, v1), v0) < 0.0) {
				if (ddot(dcross(v4, v2), v0) < 0.0) { v1 = v4; v11 = v41; v12 = v42; }
				else { v3 = v4; v31 = v41; v32 = v42; }
			} else {
				if (ddot(dcross(v4, v3), v0) < 0.0) { v2 = v4; v21 = v41; v22 = v42; }
				else { v1 = v4; v11 = v41; v12 = v42; }
			}
		}
	}
}

__device__ __forceinline__ float3 ld3(const float *p, uint64_t i) {
	return f3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
__device__ __forceinline__ float4 ld4(const float *p, uint64_t i) {
	return __ldg(reinterpret_cast<const float4 *>(p) + i);
}
__device__ __forceinline__ void st3(float *p, uint64_t i, d3 v) {
	p[3 * i] = (float)v.x; p[3 * i + 1] = (float)v.y; p[3 * i + 2] = (float)v.z;
}

// Shape of one side of a pair in the frame centred at `org` (:351-377).
__device__ __forceinline__ Shape load_shape(uint32_t s, uint32_t id, const int32_t *T, const float *A, const float *B,
                                            const float *C, const float *R, const float *pos, const float *rot,
                                            float3 org, int &type_out) {
	Shape sh;
	sh.type = __ldg(T + s);
	type_out = sh.type;
	const float3 p = ld3(pos, id);
	const float4 q = ld4(rot, id);
	const float4 qr = qmul(q, ld4(R, s));
	sh.m = rot_rows(qr);
	sh.X = ld3(A, s);
	sh.Y = ld3(B, s);
	sh.Z = ld3(C, s);
	if (sh.type == SPHERE || sh.type == ELLIPSOID || sh.type == BOX || sh.type == CYLINDER) {
		sh.X = qrot(sh.X, q) + (p - org);
	} else if (sh.type == TRIANGLEMESH) {
		sh.X = qrot(sh.X + p, qr) - org;
		sh.Y = qrot(sh.Y + p, qr) - org;
		sh.Z = qrot(sh.Z + p, qr) - org;
	}
	return sh;
}

__global__ void __launch_bounds__(kNT) k_mpr(uint64_t P, uint64_t n, const int32_t *__restrict__ T,
                                              const float *__restrict__ A, const float *__restrict__ B,
                                              const float *__restrict__ C, const float *__restrict__ R,
                                              const uint32_t *__restrict__ ID, uint64_t nb,
                                              const uint8_t *__restrict__ active, const float *__restrict__ pos,
                                              const float *__restrict__ rot, float envelope,
                                              const long long *__restrict__ pairs, NpScratch sc) {
	const uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	if (i >= P) return;
	const long long key = pairs[i];
	sc.pairs[i] = (unsigned long long)key;
	sc.flag[i] = 0u;
	const uint64_t sa64 = (uint64_t)key >> 32, sb64 = (uint64_t)key & 0xffffffffull;
	if (sa64 >= n || sb64 >= n) {
		atomicOr(sc.err, (uint32_t)kErrBadIndex);
		return;
	}
	const uint32_t sa = (uint32_t)sa64, sb = (uint32_t)sb64;
	const uint32_t ida = __ldg(ID + sa), idb = __ldg(ID + sb);
	if (ida >= nb || idb >= nb) {
		atomicOr(sc.err, (uint32_t)kErrBadIndex);
		return;
	}
	if (!active[ida] && !active[idb]) return;  // :344-346
	if (ida == idb) return;                     // :347-349
	const float3 org = ld3(pos, ida);
	int ta, tb;
	const Shape SA = load_shape(sa, ida, T, A, B, C, R, pos, rot, org, ta);
	const Shape SB = load_shape(sb, idb, T, A, B, C, R, pos, rot, org, tb);
	double env = envelope;
	if (ta == TRIANGLEMESH || tb == TRIANGLEMESH) env = 0.0;
	d3 N = {1.0, 0.0, 0.0}, p1, p2;
	if (ta == SPHERE && tb == SPHERE) {  // :382-397
		const d3 xa = D(SA.X), xb = D(SB.X);
		const d3 rel = xb - xa;
		const double d2 = ddot(rel, rel);
		const double cd = (double)SA.Y.x + (double)SB.Y.x;
		if (!(d2 <= cd * cd)) return;
		N = dnormalize(rel);
		p1 = xa + (double)SA.Y.x * N;
		p2 = xb - (double)SB.Y.x * N;
	} else {  // :400-406
		d3 p0;
		if (!mpr(SA, SB, N, p0)) return;
		p1 = ddot(D(support(SA, -N)) - p0, N) * N + p0;
		p2 = ddot(D(support(SB, N)) - p0, N) * N + p0;
		N = -N;
	}
	p1 = p1 - env * N;  // :412-415
	p2 = p2 + env * N;
	const double depth = ddot(N, p2 - p1);
	const d3 o = D(org);
	st3(sc.norm, i, N);
	st3(sc.pa, i, p1 + o);
	st3(sc.pb, i, p2 + o);
	sc.depth[i] = (float)depth;
	sc.ids[2 * i] = (int32_t)ida;
	sc.ids[2 * i + 1] = (int32_t)idb;
	sc.flag[i] = 1u;
}

__global__ void __launch_bounds__(256) k_np_compact(uint64_t P, NpScratch sc, long long *__restrict__ pairs,
                                                     float *__restrict__ norm, float *__restrict__ cpta,
                                                     float *__restrict__ cptb, float *__restrict__ depth,
                                                     int32_t *__restrict__ bids) {
	const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
	if (i >= P) return;
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

void launch_mpr(uint64_t P, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *pos,
                const float *rot, float envelope, const long long *pairs, const NpScratch &sc, cudaStream_t s) {
	if (P)
		k_mpr<<<(unsigned)((P + kNT - 1) / kNT), kNT, 0, s>>>(P, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope,
		                                                      pairs, sc);
}

void launch_np_compact(uint64_t P, const NpScratch &sc, long long *pairs, float *norm, float *cpta, float *cptb,
                       float *depth, int32_t *bids, cudaStream_t s) {
	launch_scan_u32_to_u64(sc.flag, P, sc.pos, sc.status, sc.ticket, sc.err, s);
	if (P) k_np_compact<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(P, sc, pairs, norm, cpta, cptb, depth, bids);
}

}  // namespace cc
