/*
 * Test infrastructure (oracle only; never linked into the product library).
 *
 * Stand-in for the reference's missing git submodule `includes`
 * (hmazhar/gpu_math, declared in .gitmodules:4-6 of uwsbel/collision-detection;
 * the directory is empty in the reference checkout and no commit is pinned, so
 * the version is UNKNOWN). Every reference source includes it:
 * src/aabb/AABBGenerator.cuh:12, src/broadphase/Broadphase.cuh:11,
 * src/narrowphase/Narrowphase.cuh:11, src/SupportFunctions.cuh:9.
 *
 * This header restates, from the mathematics, the vector / quaternion
 * primitives those call sites use. It fixes the operation order of every
 * primitive (no fused multiply-add; build with -ffp-contract=off) because that
 * order defines "the reference's own result" for AABBs bit for bit:
 *
 *   real           float (CC_SHIM_DOUBLE: double, the FP64 MPR oracle)
 *   real4 as quat  (.x,.y,.z,.w) = (w,i,j,k)            AABBGenerator.cuh:57
 *   dot(a,b)       (a.x*b.x + a.y*b.y) + a.z*b.z
 *   cross(a,b)     (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
 *   length(a)      sqrt(dot(a,a))
 *   normalize(a)   a / length(a), per component (IEEE division)
 *   sign(x)        +1 for x>0, -1 for x<0, 0 for x==0
 *   IsZero(x)      |x| < FLT_EPSILON (collision_detection.h:54 EPS)
 *   mult(p,q)      Hamilton product p*q, terms summed left to right
 *   AMat(q)        textbook unit-quaternion rotation matrix, rows r0,r1,r2:
 *                  r0 = (1-2(yy+zz), 2(xy-wz),   2(xz+wy))
 *                  r1 = (2(xy+wz),   1-2(xx+zz), 2(yz-wx))
 *                  r2 = (2(xz-wy),   2(yz+wx),   1-2(xx+yy))
 *   quatRotate(v,q) = quatRotateMat(v,q) = AMat(q) * v   (row dots)
 *   quatRotateMatT(v,q) = AMat(q)^T * v
 *   MatMult(M,v)   row dots;  AbsMat(M) elementwise fabs
 *
 * The product's own math header (collision-detection_b200/csrc/cc_math.cuh)
 * implements the same definitions independently; the parity tests prove that
 * the two agree bit for bit on AABBs.
 */
#ifndef CC_ORACLE_GPU_MATH_SHIM_H
#define CC_ORACLE_GPU_MATH_SHIM_H

#include <cmath>
#include <cfloat>
#include <vector_types.h>
#include <vector_functions.h>

#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif

#define CCS_HD __host__ __device__ inline

#ifdef CC_SHIM_DOUBLE
typedef double real;
struct real3 { double x, y, z; };
struct real4 { double x, y, z, w; };
#else
typedef float real;
typedef float3 real3;
typedef float4 real4;
#endif

typedef unsigned int uint;

struct M33 {
	real3 U, V, W;  // rows
};

CCS_HD real3 R3(real a) { real3 r; r.x = a; r.y = a; r.z = a; return r; }
CCS_HD real3 R3(real a, real b, real c) { real3 r; r.x = a; r.y = b; r.z = c; return r; }
CCS_HD real4 R4(real a, real b, real c, real d) { real4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r; }
CCS_HD real3 make_real3(real a, real b, real c) { return R3(a, b, c); }
CCS_HD real4 make_real4(real a, real b, real c, real d) { return R4(a, b, c, d); }
CCS_HD int2 I2(int a, int b) { int2 r; r.x = a; r.y = b; return r; }
CCS_HD int3 I3(int a, int b, int c) { int3 r; r.x = a; r.y = b; r.z = c; return r; }
CCS_HD uint3 U3(uint a, uint b, uint c) { uint3 r; r.x = a; r.y = b; r.z = c; return r; }

#define ZERO_VECTOR R3(0)

CCS_HD real3 operator+(const real3 &a, const real3 &b) { return R3(a.x + b.x, a.y + b.y, a.z + b.z); }
CCS_HD real3 operator-(const real3 &a, const real3 &b) { return R3(a.x - b.x, a.y - b.y, a.z - b.z); }
CCS_HD real3 operator*(const real3 &a, const real3 &b) { return R3(a.x * b.x, a.y * b.y, a.z * b.z); }
CCS_HD real3 operator/(const real3 &a, const real3 &b) { return R3(a.x / b.x, a.y / b.y, a.z / b.z); }
CCS_HD real3 operator*(const real3 &a, real s) { return R3(a.x * s, a.y * s, a.z * s); }
CCS_HD real3 operator*(real s, const real3 &a) { return R3(s * a.x, s * a.y, s * a.z); }
CCS_HD real3 operator/(const real3 &a, real s) { return R3(a.x / s, a.y / s, a.z / s); }
CCS_HD real3 operator-(const real3 &a) { return R3(-a.x, -a.y, -a.z); }
CCS_HD real3 &operator+=(real3 &a, const real3 &b) { a = a + b; return a; }
CCS_HD real3 &operator-=(real3 &a, const real3 &b) { a = a - b; return a; }

CCS_HD real dot(const real3 &a, const real3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CCS_HD real3 cross(const real3 &a, const real3 &b) {
	return R3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
CCS_HD real length(const real3 &a) { return sqrt(dot(a, a)); }
CCS_HD real3 normalize(const real3 &a) { real l = length(a); return R3(a.x / l, a.y / l, a.z / l); }
CCS_HD real3 fabs(const real3 &a) { return R3(fabs(a.x), fabs(a.y), fabs(a.z)); }
CCS_HD real sign(real x) { return x > 0 ? real(1) : (x < 0 ? real(-1) : real(0)); }
CCS_HD bool IsZero(real x) { return fabs(x) < real(FLT_EPSILON); }
CCS_HD bool IsZero(const real3 &a) { return IsZero(a.x) && IsZero(a.y) && IsZero(a.z); }
CCS_HD bool isEqual(real a, real b) { return IsZero(a - b); }
template <class T> CCS_HD void Swap(T &a, T &b) { T t = a; a = b; b = t; }

/* Hamilton product, quaternions stored (w,i,j,k) in (.x,.y,.z,.w). */
CCS_HD real4 mult(const real4 &p, const real4 &q) {
	real4 r;
	r.x = p.x * q.x - p.y * q.y - p.z * q.z - p.w * q.w;
	r.y = p.x * q.y + p.y * q.x + p.z * q.w - p.w * q.z;
	r.z = p.x * q.z - p.y * q.w + p.z * q.x + p.w * q.y;
	r.w = p.x * q.w + p.y * q.z - p.z * q.y + p.w * q.x;
	return r;
}

CCS_HD M33 AMat(const real4 &q) {
	const real w = q.x, x = q.y, y = q.z, z = q.w;
	const real xx = x * x, yy = y * y, zz = z * z;
	const real xy = x * y, xz = x * z, yz = y * z;
	const real wx = w * x, wy = w * y, wz = w * z;
	M33 m;
	m.U = R3(real(1) - real(2) * (yy + zz), real(2) * (xy - wz), real(2) * (xz + wy));
	m.V = R3(real(2) * (xy + wz), real(1) - real(2) * (xx + zz), real(2) * (yz - wx));
	m.W = R3(real(2) * (xz - wy), real(2) * (yz + wx), real(1) - real(2) * (xx + yy));
	return m;
}
CCS_HD M33 AMatT(const real4 &q) {
	M33 m = AMat(q), t;
	t.U = R3(m.U.x, m.V.x, m.W.x);
	t.V = R3(m.U.y, m.V.y, m.W.y);
	t.W = R3(m.U.z, m.V.z, m.W.z);
	return t;
}
CCS_HD M33 AbsMat(const M33 &m) {
	M33 r;
	r.U = fabs(m.U);
	r.V = fabs(m.V);
	r.W = fabs(m.W);
	return r;
}
CCS_HD real3 MatMult(const M33 &m, const real3 &v) { return R3(dot(m.U, v), dot(m.V, v), dot(m.W, v)); }
CCS_HD real3 quatRotateMat(const real3 &v, const real4 &q) { return MatMult(AMat(q), v); }
CCS_HD real3 quatRotate(const real3 &v, const real4 &q) { return quatRotateMat(v, q); }
CCS_HD real3 quatRotateMatT(const real3 &v, const real4 &q) { return MatMult(AMatT(q), v); }

#endif
