// Vector / quaternion arithmetic of the collision path.
//
// The reference takes these primitives from its gpu_math submodule
// (hmazhar/gpu_math, absent from the reference checkout, version unknown);
// they are defined here from the mathematics with a fixed operation order:
//
//   quaternion     float4 (w, x, y, z) in (.x, .y, .z, .w)  (AABBGenerator.cuh:57)
//   dot(a, b)      (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a, b)    (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   qmul(p, q)     Hamilton product, terms summed left to right
//   rot_rows(q)    rows of the unit-quaternion rotation matrix
//                  (1-2(yy+zz), 2(xy-wz), 2(xz+wy)) / (2(xy+wz), 1-2(xx+zz), 2(yz-wx))
//                  / (2(xz-wy), 2(yz+wx), 1-2(xx+yy))
//   qrot(v, q)     rotation matrix times v (row dots)
//   sign(x)        +1 / -1 / 0
//
// AABB and broadphase kernels are compiled with -fmad=false so every product
// and sum rounds separately: that is what makes their results bit-identical to
// the reference's host build. The narrowphase is tolerance-checked and keeps
// fused multiply-add.
#pragma once
#include <cuda_runtime.h>

namespace cc {

__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ float3 mulv(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float3 divs(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross(float3 a, float3 b) {
	return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ float3 normalize(float3 a) { float l = length(a); return f3(a.x / l, a.y / l, a.z / l); }
__host__ __device__ __forceinline__ float3 abs3(float3 a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__host__ __device__ __forceinline__ float signf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

__host__ __device__ __forceinline__ float4 qmul(float4 p, float4 q) {
	return make_float4(p.x * q.x - p.y * q.y - p.z * q.z - p.w * q.w,
	                   p.x * q.y + p.y * q.x + p.z * q.w - p.w * q.z,
	                   p.x * q.z - p.y * q.w + p.z * q.x + p.w * q.y,
	                   p.x * q.w + p.y * q.z - p.z * q.y + p.w * q.x);
}

struct Rot {
	float3 r0, r1, r2;  // rows
};

__host__ __device__ __forceinline__ Rot rot_rows(float4 q) {
	const float w = q.x, x = q.y, y = q.z, z = q.w;
	const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
	const float wx = w * x, wy = w * y, wz = w * z;
	Rot m;
	m.r0 = f3(1.f - 2.f * (yy + zz), 2.f * (xy - wz), 2.f * (xz + wy));
	m.r1 = f3(2.f * (xy + wz), 1.f - 2.f * (xx + zz), 2.f * (yz - wx));
	m.r2 = f3(2.f * (xz - wy), 2.f * (yz + wx), 1.f - 2.f * (xx + yy));
	return m;
}
__host__ __device__ __forceinline__ float3 mat_vec(const Rot &m, float3 v) { return f3(dot(m.r0, v), dot(m.r1, v), dot(m.r2, v)); }
__host__ __device__ __forceinline__ float3 mat_t_vec(const Rot &m, float3 v) {
	return f3(dot(f3(m.r0.x, m.r1.x, m.r2.x), v), dot(f3(m.r0.y, m.r1.y, m.r2.y), v), dot(f3(m.r0.z, m.r1.z, m.r2.z), v));
}
__host__ __device__ __forceinline__ float3 qrot(float3 v, float4 q) { return mat_vec(rot_rows(q), v); }

// Shape codes of the reference (collision_detection.h:57).
enum ShapeType : int { SPHERE = 0, ELLIPSOID = 1, BOX = 2, CYLINDER = 3, RECT = 4, CONE = 5, TRIANGLEMESH = 6 };

}  // namespace cc
