// Minkowski portal refinement (the reference's CollideAndFindPoint,
// src/narrowphase/Narrowphase.cu:122-314, inside function_MPR_Store :316-423)
// as a per-lane state machine with warp-level work stealing.
//
// Every loop iteration, each busy lane evaluates exactly ONE support pair
// (support(A, -d), support(B, d)) and then updates its MPR state; a lane whose
// pair is finished writes its contact and takes the next pair from a global
// queue (pairs pre-grouped by shape-type combination). The warp therefore runs
// the same support code on most of its lanes in every iteration instead of
// idling while a few pairs refine to the iteration cap.
//
// Template parameters:
//   S       scalar of the support maps (double or float)
//   kExact  true:  the FP64 oracle's arithmetic exactly — world coordinates,
//                  every direction normalized before the support map,
//                  normalize = v / sqrt(v.v), the reference's operation order;
//                  the including translation unit is compiled with
//                  -fmad=false, so results equal the reference compiled with
//                  real = double, rounded to float on output.
//           false: pair-local frame (origin = body A's position), one
//                  reciprocal square root per normalization, fused
//                  multiply-add allowed.
// Portal arithmetic is FP64 in every variant.
#pragma once
#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"

namespace cc {
namespace mpr {

constexpr double kEps = 1.1920928955078125e-07;  // FLT_EPSILON (collision_detection.h:54)
constexpr int kMaxIter = 34;                      // Narrowphase.cu:198

template <class T>
struct vec {
	T x, y, z;
};
template <class T>
__device__ __forceinline__ vec<T> mk(T x, T y, T z) { return {x, y, z}; }
template <class T, class U>
__device__ __forceinline__ vec<T> cvt(vec<U> a) { return {(T)a.x, (T)a.y, (T)a.z}; }
template <class T>
__device__ __forceinline__ vec<T> cvt3(float3 a) { return {(T)a.x, (T)a.y, (T)a.z}; }
template <class T>
__device__ __forceinline__ vec<T> add(vec<T> a, vec<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
__device__ __forceinline__ vec<T> sub(vec<T> a, vec<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
__device__ __forceinline__ vec<T> neg(vec<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T>
__device__ __forceinline__ vec<T> scl(T s, vec<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T>
__device__ __forceinline__ vec<T> mulv(vec<T> a, vec<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T>
__device__ __forceinline__ T dotp(vec<T> a, vec<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
__device__ __forceinline__ vec<T> crossp(vec<T> a, vec<T> b) {
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
__device__ __forceinline__ T len(vec<T> a) { return sqrt(dotp(a, a)); }
// One FP64 quotient a / l from y = RN(1/l), equal to the IEEE quotient:
// q = a*y corrected once is a faithful quotient, and one more correction
// q + (a - l*q)*y, with the residual exact in an FMA, rounds to RN(a / l)
// (Markstein's theorem: P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990). The
// corrections are written as -fma(-r, y, -q) so that a = -0 keeps its sign.
// Valid without underflow or overflow: l and a nonzero |a| in [2^-500, 2^500].
__device__ __forceinline__ double quot_rcp(double a, double l, double y) {
	const double q0 = a * y;
	const double q1 = -fma(-fma(-l, q0, a), y, -q0);
	return -fma(-fma(-l, q1, a), y, -q1);
}
__device__ __forceinline__ bool quot_range(double x) {
	const double m = fabs(x);
	return m == 0.0 || (m >= 0x1p-500 && m <= 0x1p500);
}
// a / l componentwise with IEEE results. In double, one correctly rounded
// reciprocal (__drcp_rn) serves the three components: an FP64 division is a
// dependent sequence of ~120 cycles and three of them run one after the
// other, while the three corrections overlap (~2x faster normalization).
template <class T>
__device__ __forceinline__ vec<T> div3(vec<T> a, T l) {
	if constexpr (sizeof(T) == 8) {
		if (l >= 0x1p-500 && l <= 0x1p500 && quot_range(a.x) && quot_range(a.y) && quot_range(a.z)) {
			const double y = __drcp_rn(l);
			return {quot_rcp(a.x, l, y), quot_rcp(a.y, l, y), quot_rcp(a.z, l, y)};
		}
	}
	return {a.x / l, a.y / l, a.z / l};
}
// normalize: the reference's a / |a| (exact) or a * rsqrt(a.a) (fast)
template <class T, bool kExact>
__device__ __forceinline__ vec<T> unit(vec<T> a) {
	if constexpr (kExact) {
		const T l = len(a);
		return div3(a, l);
	} else {
		const T il = rsqrt(dotp(a, a));
		return {a.x * il, a.y * il, a.z * il};
	}
}

// a / sqrt(a.a) in double with IEEE results, without the square root and the
// reciprocal when a.a lies within 2^20 units in the last place of 1 (a vector
// normalized once already). With s = a.a whose bits are bits(1) + e:
//  * sqrt(s) has the bits bits(1) + floor(e / 2). For s = 1 + t, sqrt(s) lies
//    strictly below 1 + t/2 (concavity) and above 1 + t/2 - t^2/8. Above 1
//    (t = e 2^-52) 1 + t/2 is representable for even e and a midpoint for odd
//    e; below 1 (t = e 2^-53, spacing 2^-53) the same holds with the halved
//    spacing. Either way the correctly rounded root is the representable
//    number at or just below 1 + t/2, t^2/8 being far below half a spacing.
//  * RN(1 / l) for l with the bits bits(1) + f: for f >= 0, 1/l lies above
//    1 - f 2^-52 (representable, bits(1) - 2f) by less than f^2 2^-104, under
//    half the spacing 2^-53 below 1; for f < 0, 1/l lies strictly above
//    1 - f 2^-53, which is representable (bits(1) - f/2) for even f and a
//    midpoint for odd f, so RN gives bits(1) + ceil(-f / 2) = bits(1) -
//    floor(f / 2).
// The quotients then follow quot_rcp (Markstein) as in div3, so the result is
// bit for bit unit<double, true>(a).
__device__ __forceinline__ vec<double> unit_again(vec<double> a) {
	constexpr long long kOne = 0x3FF0000000000000ll, kNear = 1ll << 20;
	const long long e = __double_as_longlong(dotp(a, a)) - kOne;
	if (e >= -kNear && e <= kNear && quot_range(a.x) && quot_range(a.y) && quot_range(a.z)) {
		const long long f = e >> 1;  // arithmetic shift: floor(e / 2)
		const double l = __longlong_as_double(kOne + f);
		const double y = __longlong_as_double(f >= 0 ? kOne - 2 * f : kOne - (f >> 1));
		return {quot_rcp(a.x, l, y), quot_rcp(a.y, l, y), quot_rcp(a.z, l, y)};
	}
	return unit<double, true>(a);
}

template <class T>
__device__ __forceinline__ T sgn(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0)); }
template <class T>
__device__ __forceinline__ bool is_zero(vec<T> a) {
	return fabs((double)a.x) < kEps && fabs((double)a.y) < kEps && fabs((double)a.z) < kEps;
}

// A shape placed in the frame of the pair, with the rows of its rotation
// body_rot * local_rot (Narrowphase.cu:356-357).
template <class S>
struct Shape {
	int type;
	vec<S> X, Y, Z;  // centre (or triangle vertex 0), B (or vertex 1), C (or vertex 2)
	vec<S> r0, r1, r2;
};

template <class S>
__device__ __forceinline__ void rows_of(S w, S x, S y, S z, vec<S> &r0, vec<S> &r1, vec<S> &r2) {
	const S xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y,
	        wz = w * z;
	r0 = mk<S>(S(1) - S(2) * (yy + zz), S(2) * (xy - wz), S(2) * (xz + wy));
	r1 = mk<S>(S(2) * (xy + wz), S(1) - S(2) * (xx + zz), S(2) * (yz - wx));
	r2 = mk<S>(S(2) * (xz - wy), S(2) * (yz + wx), S(1) - S(2) * (xx + yy));
}
template <class S>
__device__ __forceinline__ vec<S> mrow(vec<S> r0, vec<S> r1, vec<S> r2, vec<S> v) {
	return {dotp(r0, v), dotp(r1, v), dotp(r2, v)};
}
template <class S>
__device__ __forceinline__ vec<S> mcol(vec<S> r0, vec<S> r1, vec<S> r2, vec<S> v) {
	return {r0.x * v.x + r1.x * v.y + r2.x * v.z, r0.y * v.x + r1.y * v.y + r2.y * v.z,
	        r0.z * v.x + r1.z * v.y + r2.z * v.z};
}

// Local support maps (SupportFunctions.cuh:11-99), on a unit direction in the
// exact variant; the fast variant uses that every map but the sphere's is
// invariant to the length of n. support_local_t: the four round and boxy
// types by compile-time type.
template <class S, bool kExact, int TYPE>
__device__ __forceinline__ vec<S> support_local_t(vec<S> B, vec<S> n) {
	if constexpr (TYPE == SPHERE) {
		if constexpr (kExact) return scl(B.x, n);
		else return scl(B.x, unit<S, false>(n));
	} else if constexpr (TYPE == ELLIPSOID) {
		if constexpr (kExact) {
			const vec<S> nn = unit<S, true>(n);
			const vec<S> bbn = mulv(mulv(B, B), nn);
			const S l = len(mulv(B, nn));
			return div3(bbn, l);
		} else {  // B*B*n / |B*n|
			const vec<S> bn = mulv(B, n);
			const S il = rsqrt(dotp(bn, bn));
			return {B.x * bn.x * il, B.y * bn.y * il, B.z * bn.z * il};
		}
	} else if constexpr (TYPE == BOX) {
		return {sgn(n.x) * B.x, sgn(n.y) * B.y, sgn(n.z) * B.z};
	} else {
		static_assert(TYPE == CYLINDER, "sphere, ellipsoid, box or cylinder");
		// axis = local y: w = n - (u.n) u = (n.x, 0, n.z)
		const vec<S> w = mk<S>(n.x, S(0), n.z);
		const S sy = sgn(n.y) * B.y;
		if (len(w) != S(0)) {
			const vec<S> wn = unit<S, kExact>(w);
			return {B.x * wn.x, sy + B.x * wn.y, B.x * wn.z};
		}
		return mk<S>(S(0), sy, S(0));
	}
}
template <class S, bool kExact>
__device__ __forceinline__ vec<S> support_local(int type, vec<S> B, vec<S> n) {
	switch (type) {
	case SPHERE: return support_local_t<S, kExact, SPHERE>(B, n);
	case ELLIPSOID: return support_local_t<S, kExact, ELLIPSOID>(B, n);
	case BOX: return support_local_t<S, kExact, BOX>(B, n);
	case CYLINDER: return support_local_t<S, kExact, CYLINDER>(B, n);
	case RECT: {
		vec<S> r = B;
		if (n.x < S(0)) r.x = -r.x;
		if (n.y < S(0)) r.y = -r.y;
		return r;
	}
	case CONE: {
		const S radius = B.x, height = B.y;
		const S sa = radius / sqrt(radius * radius + height * height);
		if (n.y > len(n) * sa) return mk<S>(S(0), height / S(2), S(0));
		const S s = sqrt(n.x * n.x + n.z * n.z);
		if (s > S(1e-9)) {
			const S d = radius / s;
			return mk<S>(n.x * d, -height / S(2), n.z * d);
		}
		return mk<S>(S(0), -height / S(2), S(0));
	}
	}
	return mk<S>(S(0), S(0), S(0));
}

// TransformSupportVert (:19-52) along direction d. The reference normalizes
// d first (exact variant); the caller does that once for both shapes of the
// pair, since d / |d| for -d is exactly -(d / |d|) in IEEE arithmetic.
template <class S, bool kExact>
__device__ __forceinline__ vec<S> support(const Shape<S> &s, vec<S> d) {
	if (s.type == TRIANGLEMESH) {  // SupportFunctions.cuh:14-29, world frame
		S dist = dotp(s.X, d);
		vec<S> p = s.X;
		if (dotp(s.Y, d) > dist) { dist = dotp(s.Y, d); p = s.Y; }
		if (dotp(s.Z, d) > dist) { p = s.Z; }
		return p;
	}
	const vec<S> rn = mcol(s.r0, s.r1, s.r2, d);
	return add(mrow(s.r0, s.r1, s.r2, support_local<S, kExact>(s.type, s.Y, rn)), s.X);
}

typedef vec<double> D3;

template <class S>
__device__ __forceinline__ D3 centre(const Shape<S> &s) {  // GetCenter :11-17
	if (s.type == TRIANGLEMESH)
		return {((double)s.X.x + s.Y.x + s.Z.x) / 3.0, ((double)s.X.y + s.Y.y + s.Z.y) / 3.0,
		        ((double)s.X.z + s.Y.z + s.Z.z) / 3.0};
	return {(double)s.X.x + 0.0, (double)s.X.y + 0.0, (double)s.X.z + 0.0};  // R3(0,0,0) + A
}

__device__ __forceinline__ float3 ld3(const float *p, uint64_t i) {
	return f3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
__device__ __forceinline__ float4 ld4(const float *p, uint64_t i) {
	return __ldg(reinterpret_cast<const float4 *>(p) + i);
}

// One side of a pair in the frame centred at `org` (:351-377).
template <class S>
__device__ __forceinline__ Shape<S> load_shape(uint32_t s, uint32_t id, const int32_t *T, const float *A,
                                               const float *B, const float *C, const float *R, const float *pos,
                                               const float *rot, vec<S> org) {
	Shape<S> sh;
	sh.type = __ldg(T + s);
	const float3 p = ld3(pos, id);
	const float4 q = ld4(rot, id);
	const float4 lq = ld4(R, s);
	// mult(body_rot, local_rot) (Hamilton product, terms left to right)
	const S w1 = q.x, x1 = q.y, y1 = q.z, z1 = q.w, w2 = lq.x, x2 = lq.y, y2 = lq.z, z2 = lq.w;
	const S qw = w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2;
	const S qx = w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2;
	const S qy = w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2;
	const S qz = w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2;
	rows_of<S>(qw, qx, qy, qz, sh.r0, sh.r1, sh.r2);
	sh.X = cvt3<S>(ld3(A, s));
	sh.Y = cvt3<S>(ld3(B, s));
	sh.Z = cvt3<S>(ld3(C, s));
	const vec<S> po = sub(cvt3<S>(p), org);
	if (sh.type == SPHERE || sh.type == ELLIPSOID || sh.type == BOX || sh.type == CYLINDER) {
		vec<S> b0, b1, b2;
		rows_of<S>((S)q.x, (S)q.y, (S)q.z, (S)q.w, b0, b1, b2);
		sh.X = add(mrow(b0, b1, b2, sh.X), po);  // quatRotate(A, body_rot) + pos
	} else if (sh.type == TRIANGLEMESH) {
		const vec<S> pw = cvt3<S>(p);  // quatRotate(v + pos, body_rot * local_rot), then into the frame
		sh.X = sub(mrow(sh.r0, sh.r1, sh.r2, add(sh.X, pw)), org);
		sh.Y = sub(mrow(sh.r0, sh.r1, sh.r2, add(sh.Y, pw)), org);
		sh.Z = sub(mrow(sh.r0, sh.r1, sh.r2, add(sh.Z, pw)), org);
	}
	return sh;
}

// Per-lane MPR state.
// kParked: the refinement has ended with a hit and the lane waits, its portal
// kept, for the warp to finish all such pairs together (run()).
enum State : int { kIdle = 0, kS1, kS2, kDisc, kRefine, kPost, kParked };

template <class S, bool kExact>
struct Lane {
	uint32_t pair;  // index of the pair being worked on
	int st;
	int phase1, phase2;
	bool hit;
	Shape<S> A, B;
	D3 v0, v1, v2, v3;
	vec<S> v11, v12, v21, v22, v31, v32;
	D3 n;      // direction of the next support pair
	D3 N, p0;  // contact normal and point (post stage)
	D3 org;    // frame origin
	double env;
};

template <class S>
__device__ __forceinline__ D3 vd(vec<S> pb, vec<S> pa) { return sub(cvt<double>(pb), cvt<double>(pa)); }
template <class S>
__device__ __forceinline__ D3 dd(vec<S> a) { return cvt<double>(a); }

struct Outputs {
	const NpScratch *sc;
};

__device__ __forceinline__ void st3(float *p, uint64_t i, D3 v) {
	p[3 * i] = (float)v.x;
	p[3 * i + 1] = (float)v.y;
	p[3 * i + 2] = (float)v.z;
}

// function_MPR_Store :404-422 once the contact normal N and point p0 (or the
// sphere-sphere p1/p2) are known: envelope, depth, outputs.
template <class S, bool kExact>
__device__ __forceinline__ void write_contact(const Lane<S, kExact> &L, D3 N, D3 p1, D3 p2, uint32_t ida, uint32_t idb,
                                              const NpScratch &sc) {
	p1 = sub(p1, scl(L.env, N));  // :412-415
	p2 = add(p2, scl(L.env, N));
	const double depth = dotp(N, sub(p2, p1));
	const uint64_t i = L.pair;
	st3(sc.norm, i, N);
	st3(sc.pa, i, add(p1, L.org));
	st3(sc.pb, i, add(p2, L.org));
	sc.depth[i] = (float)depth;
	sc.ids[2 * i] = (int32_t)ida;
	sc.ids[2 * i + 1] = (int32_t)idb;
	sc.flag[i] = 1u;
	if (sc.hkeys) {  // overlapped narrowphase: key -> i for the compaction in sorted order
		const unsigned long long tag = sc.pairs[i] + 1ull;
		uint64_t h = (tag * 0x9E3779B97F4A7C15ull) >> 20;
		bool placed = false;
		for (uint64_t probe = 0; probe <= sc.hmask && probe < 256; probe++, h++) {
			const uint64_t slot = h & sc.hmask;
			if (atomicCAS(&sc.hkeys[slot], 0ull, tag) == 0ull) {
				sc.hvals[slot] = (uint32_t)i;
				placed = true;
				break;
			}
		}
		if (!placed) atomicOr(sc.err, (uint32_t)kErrHashFull);
	}
}

// Starts pair i: the checks and transforms of :338-377; sphere-sphere pairs
// (:382-397) and skipped pairs finish here. Returns true if the lane now runs
// the MPR state machine.
template <class S, bool kExact>
__device__ __forceinline__ bool start_pair(Lane<S, kExact> &L, uint32_t i, uint64_t n, const int32_t *T,
                                           const float *A, const float *B, const float *C, const float *R,
                                           const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *pos,
                                           const float *rot, float envelope, const long long *pairs,
                                           const NpScratch &sc) {
	L.pair = i;
	const long long key = pairs[i];
	sc.pairs[i] = (unsigned long long)key;
	sc.flag[i] = 0u;
	const uint64_t sa64 = (uint64_t)key >> 32, sb64 = (uint64_t)key & 0xffffffffull;
	if (sa64 >= n || sb64 >= n) {
		atomicOr(sc.err, (uint32_t)kErrBadIndex);
		return false;
	}
	const uint32_t sa = (uint32_t)sa64, sb = (uint32_t)sb64;
	const uint32_t ida = __ldg(ID + sa), idb = __ldg(ID + sb);
	if (ida >= nb || idb >= nb) {
		atomicOr(sc.err, (uint32_t)kErrBadIndex);
		return false;
	}
	if (!active[ida] && !active[idb]) return false;  // :344-346
	if (ida == idb) return false;                     // :347-349
	if constexpr (kExact) {
		L.org = mk(0.0, 0.0, 0.0);
	} else {
		const float3 o = ld3(pos, ida);
		L.org = mk((double)o.x, (double)o.y, (double)o.z);
	}
	const vec<S> org = cvt<S>(L.org);
	L.A = load_shape<S>(sa, ida, T, A, B, C, R, pos, rot, org);
	L.B = load_shape<S>(sb, idb, T, A, B, C, R, pos, rot, org);
	L.env = envelope;
	if (L.A.type == TRIANGLEMESH || L.B.type == TRIANGLEMESH) L.env = 0.0;
	if (L.A.type == SPHERE && L.B.type == SPHERE) {  // :382-397
		const D3 xa = dd(L.A.X), xb = dd(L.B.X);
		const D3 rel = sub(xb, xa);
		const double d2 = dotp(rel, rel);
		const double ra = (double)L.A.Y.x, rb = (double)L.B.Y.x;
		const double cd = ra + rb;
		if (!(d2 <= cd * cd)) return false;
		const D3 N = unit<double, kExact>(rel);
		write_contact(L, N, add(xa, scl(ra, N)), sub(xb, scl(rb, N)), ida, idb, sc);
		return false;
	}
	// CollideAndFindPoint :137-144
	const D3 v01 = centre(L.A), v02 = centre(L.B);
	L.v0 = sub(v02, v01);
	if (is_zero(L.v0)) L.v0 = mk(1.0, 0.0, 0.0);
	L.n = neg(L.v0);
	L.st = kS1;
	return true;
}

// Finishes a hit: the contact points of :404-406 need one more support pair
// along the normal; N, p0 are set here and the post stage evaluates it.
template <class S, bool kExact>
__device__ __forceinline__ void to_post(Lane<S, kExact> &L, D3 N, D3 p0) {
	L.N = N;
	L.p0 = p0;
	L.n = N;
	L.st = kPost;
}

// Work that happens before a lane's next support evaluation; may finish the
// pair (returns false) without evaluating a support pair.
template <class S, bool kExact>
__device__ __forceinline__ bool pre_step(Lane<S, kExact> &L) {
	if (L.st == kDisc) {  // :201-205
		if (L.phase1 > kMaxIter) return false;
		L.phase1++;
	} else if (L.st == kRefine) {  // :240-253
		L.phase2++;
		L.n = unit<double, kExact>(crossp(sub(L.v2, L.v1), sub(L.v3, L.v1)));
		if (dotp(L.n, L.v1) >= 0.0 && !L.hit) L.hit = true;
	}
	return true;
}

// The end of a refinement with a hit (:256-283 once the portal is final): the
// barycentric contact point and the normal; the post stage then evaluates one
// more support pair along the normal.
template <class S, bool kExact>
__device__ __forceinline__ void finish_refine(Lane<S, kExact> &L) {
	const D3 v1 = L.v1, v2 = L.v2, v3v = L.v3, v0 = L.v0, n = L.n;
	double b0 = dotp(crossp(v1, v2), v3v);
	double b1 = dotp(crossp(v3v, v2), v0);
	double b2 = dotp(crossp(v0, v1), v3v);
	double b3 = dotp(crossp(v2, v1), v0);
	double sum = b0 + b1 + b2 + b3;
	if (sum <= 0.0) {
		b0 = 0.0;
		b1 = dotp(crossp(v2, v3v), n);
		b2 = dotp(crossp(v3v, v1), n);
		b3 = dotp(crossp(v1, v2), n);
		sum = b1 + b2 + b3;
	}
	const double inv = 1.0 / sum;
	const D3 v01 = centre(L.A), v02 = centre(L.B);
	const D3 p = add(add(add(scl(b0, v01), scl(b1, dd(L.v11))), scl(b2, dd(L.v21))), scl(b3, dd(L.v31)));
	const D3 q = add(add(add(scl(b0, v02), scl(b1, dd(L.v12))), scl(b2, dd(L.v22))), scl(b3, dd(L.v32)));
	const D3 pq = add(p, q);
	const D3 pt = mk(pq.x * inv * 0.5, pq.y * inv * 0.5, pq.z * inv * 0.5);
	to_post(L, unit<double, kExact>(n), pt);
}

// State update after the support pair (pa = support(A,-n), pb = support(B,n)).
// Returns false when the pair is finished. park: a refinement that ends with a
// hit leaves its portal as it is (kParked) instead of finishing it here.
template <class S, bool kExact>
__device__ __forceinline__ bool post_step(Lane<S, kExact> &L, vec<S> pa, vec<S> pb, const NpScratch &sc,
                                          uint32_t ida, uint32_t idb, bool park) {
	switch (L.st) {
	case kS1: {  // :146-171
		L.v11 = pa;
		L.v12 = pb;
		L.v1 = vd(pb, pa);
		if (dotp(L.v1, L.n) <= 0.0) return false;
		L.n = crossp(L.v1, L.v0);
		if (is_zero(L.n)) {
			const D3 N = unit<double, kExact>(sub(L.v1, L.v0));
			const D3 s12 = add(dd(L.v11), dd(L.v12));
			to_post(L, N, kExact ? mk(s12.x * 0.5, s12.y * 0.5, s12.z * 0.5) : scl(0.5, s12));
			return true;
		}
		L.st = kS2;
		return true;
	}
	case kS2: {  // :173-191
		L.v21 = pa;
		L.v22 = pb;
		L.v2 = vd(pb, pa);
		if (dotp(L.v2, L.n) <= 0.0) return false;
		L.n = crossp(sub(L.v1, L.v0), sub(L.v2, L.v0));
		if (dotp(L.n, L.v0) > 0.0) {
			D3 t = L.v1; L.v1 = L.v2; L.v2 = t;
			vec<S> u = L.v11; L.v11 = L.v21; L.v21 = u;
			u = L.v12; L.v12 = L.v22; L.v22 = u;
			L.n = neg(L.n);
		}
		L.phase1 = 0;
		L.phase2 = 0;
		L.hit = false;
		L.st = kDisc;
		return true;
	}
	case kDisc: {  // :209-232
		L.v31 = pa;
		L.v32 = pb;
		L.v3 = vd(pb, pa);
		if (dotp(L.v3, L.n) <= 0.0) return false;
		// both side tests evaluated up front (independent; same arithmetic)
		const double s13 = dotp(crossp(L.v1, L.v3), L.v0), s32 = dotp(crossp(L.v3, L.v2), L.v0);
		if (s13 < 0.0) {
			L.v2 = L.v3; L.v21 = L.v31; L.v22 = L.v32;
			L.n = crossp(sub(L.v1, L.v0), sub(L.v3, L.v0));
			return true;
		}
		if (s32 < 0.0) {
			L.v1 = L.v3; L.v11 = L.v31; L.v12 = L.v32;
			L.n = crossp(sub(L.v3, L.v0), sub(L.v2, L.v0));
			return true;
		}
		L.st = kRefine;
		return true;
	}
	case kRefine: {  // :256-311
		const D3 v4 = vd(pb, pa);
		const double delta = dotp(sub(v4, L.v3), L.n);
		const double depth = dotp(v4, L.n);
		// the three side tests of the portal update (:295-310), evaluated up
		// front beside the termination test (independent; same arithmetic)
		const double s41 = dotp(crossp(v4, L.v1), L.v0), s42 = dotp(crossp(v4, L.v2), L.v0),
		             s43 = dotp(crossp(v4, L.v3), L.v0);
		if (delta <= 1e-20 || depth <= 0.0 || L.phase2 > kMaxIter) {
			if (!L.hit) return false;
			if (park) L.st = kParked;
			else finish_refine(L);
			return true;
		}
		if (s41 < 0.0) {
			if (s42 < 0.0) { L.v1 = v4; L.v11 = pa; L.v12 = pb; }
			else { L.v3 = v4; L.v31 = pa; L.v32 = pb; }
		} else {
			if (s43 < 0.0) { L.v2 = v4; L.v21 = pa; L.v22 = pb; }
			else { L.v1 = v4; L.v11 = pa; L.v12 = pb; }
		}
		return true;
	}
	case kPost: {  // :404-406
		const D3 N = L.N, p0 = L.p0;
		const D3 p1 = add(scl(dotp(sub(dd(pa), p0), N), N), p0);
		const D3 p2 = add(scl(dotp(sub(dd(pb), p0), N), N), p0);
		write_contact(L, neg(N), p1, p2, ida, idb, sc);
		return false;
	}
	}
	return false;
}

// Persistent kernel: lanes take pairs from the global queue `order`
// (P = min(P_cap, *P_dev) entries), one support pair per busy lane per
// iteration. Once the warp has seen the queue drained, a refinement that ends
// with a hit parks, and the parked pairs of the warp are finished together
// when none of its lanes runs any more: the warp then runs the finishing code
// (barycentric point, normal, one more support pair, the contact) once instead
// of once for every pair that ends at a different iteration. The finishing
// arithmetic reads only the parked portal, so the contacts are the same.
template <class S, bool kExact, int NT>
__device__ __forceinline__ void run(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T,
                                    const float *A, const float *B, const float *C, const float *R, const uint32_t *ID,
                                    uint64_t nb, const uint8_t *active, const float *pos, const float *rot,
                                    float envelope, const long long *pairs, const NpScratch &sc, uint32_t *queue) {
	const uint64_t P = P_dev ? min(P_cap, (uint64_t)*P_dev) : P_cap;
	Lane<S, kExact> L;
	L.st = kIdle;
	bool done = false;     // the queue is exhausted for this lane
	bool drained = false;  // the warp has taken the last queue entries (warp-uniform)
	uint32_t ida = 0, idb = 0;
	const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
	while (true) {
		// lanes without a pair take the next ones from the queue (one atomic per warp)
		const bool want = L.st == kIdle && !done;
		const uint32_t m = __ballot_sync(0xffffffffu, want);
		if (m) {
			uint32_t base = 0;
			const int leader = __ffs(m) - 1;
			if ((int)lane == leader) base = atomicAdd(queue, (uint32_t)__popc(m));
			base = __shfl_sync(0xffffffffu, base, leader);
			drained = drained || (uint64_t)base + __popc(m) >= P;
			if (want) {
				const uint64_t j = (uint64_t)base + __popc(m & lt);
				if (j >= P) {
					done = true;
				} else {
					const uint32_t i = sc.order[j];
					if (start_pair(L, i, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc)) {
						const uint64_t key = (uint64_t)pairs[i];
						ida = __ldg(ID + (uint32_t)(key >> 32));
						idb = __ldg(ID + (uint32_t)(key & 0xffffffffull));
					} else {
						L.st = kIdle;
					}
				}
			}
		}
		done = done || drained;
		const bool running = L.st != kIdle && L.st != kParked;
		if (!__any_sync(0xffffffffu, running || !done)) {
			const bool parked = L.st == kParked;
			if (!__any_sync(0xffffffffu, parked)) break;
			if (parked) finish_refine(L);  // -> kPost: the next iteration writes the contact
			continue;
		}
		if (!running) continue;
		if (!pre_step(L)) {
			L.st = kIdle;
			continue;
		}
		// the support pair: support(A, -n), support(B, n)
		vec<S> d = cvt<S>(L.n);
		if constexpr (kExact && sizeof(S) == 8) d = unit_again(d);  // n is a unit vector when refining
		else if constexpr (kExact) d = unit<S, true>(d);
		const vec<S> pa = support<S, kExact>(L.A, neg(d));
		const vec<S> pb = support<S, kExact>(L.B, d);
		if (!post_step(L, pa, pb, sc, ida, idb, drained)) L.st = kIdle;
	}
}

}  // namespace mpr
}  // namespace cc
