/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement, on the CPU, of the reference's collision path
 * (uwsbel/collision-detection: AABB generation -> uniform-grid broadphase ->
 * MPR narrowphase). Only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py may load it, and only as the checker: the product library
 * (collision-detection_b200/) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates. The vector and
 * quaternion primitives follow oracle/shim/includes/gpu_math.h, the stand-in
 * for the reference's missing gpu_math submodule (version unknown), with the
 * same operation order and no fused multiply-add (build with
 * -ffp-contract=off). The restatement is pinned against the reference's own
 * sources compiled in host mode (oracle/_ref, built by oracle/Makefile) and
 * against the reference tests' known answers (tests/test_oracle.py).
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CCO_API __attribute__((visibility("default")))
#define CCO_API_DEFINED

/* shape_type, collision_detection.h:57 */
enum { CCO_SPHERE, CCO_ELLIPSOID, CCO_BOX, CCO_CYLINDER, CCO_RECT, CCO_CONE, CCO_TRIANGLEMESH };

#define CCO_R float
#define CCO_SFX _f32
#define CCO_SQRT sqrtf
#include "cco_mpr.inc.h"
#undef CCO_R
#undef CCO_SFX
#undef CCO_SQRT
#define CCO_R double
#define CCO_SFX _f64
#define CCO_SQRT sqrt
#include "cco_mpr.inc.h"
#undef CCO_R
#undef CCO_SFX
#undef CCO_SQRT

CCO_API int64_t cco_narrowphase_f32_api(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                                        const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active,
                                        const float *pos, const float *rot, float envelope, int64_t *pairs, uint64_t P,
                                        double *norm, double *cpta, double *cptb, double *depth, int32_t *bids) {
	return cco_narrowphase_f32(n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, P, norm, cpta, cptb, depth,
	                           bids);
}
CCO_API int64_t cco_narrowphase_f64_api(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                                        const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active,
                                        const float *pos, const float *rot, float envelope, int64_t *pairs, uint64_t P,
                                        double *norm, double *cpta, double *cptb, double *depth, int32_t *bids) {
	return cco_narrowphase_f64(n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, P, norm, cpta, cptb, depth,
	                           bids);
}

/* ------------------------------------------------------------------------ */
/* AABB generation                                                           */
/* ------------------------------------------------------------------------ */
typedef cco_v3_f32 v3f;
typedef cco_q4_f32 q4f;

/* std::min / std::max on floats (the triangle branch calls min/max under
 * `using namespace std`, AABBGenerator.cu:17-22). */
static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float smax(float a, float b) { return (a < b) ? b : a; }

/* One shape: function_ComputeAABB, AABBGenerator.cu:84-116, with
 * ComputeAABBSphere :11-14, ComputeAABBTriangle :16-23 and the live part of
 * ComputeAABBBox :25-35. Returns 0 (and writes nothing) for the types the
 * reference skips (:110-111). Type 5 is treated as a triangle, as at :103. */
static int aabb_one(uint64_t i, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                    const uint32_t *ID, const float *pos, const float *rot, v3f *mn, v3f *mx) {
	int type = T[i];
	uint32_t id = ID[i];
	v3f a = ld3_f32(A, i), b = ld3_f32(B, i), c = ld3_f32(C, i);
	v3f position = ld3_f32(pos, id);
	q4f brot = ld4_f32(rot, id), lrot = ld4_f32(R, i);
	q4f rotation = qmult_f32(brot, lrot);
	if (type == 0) {
		a = qrot_f32(a, brot);
		v3f p = add_f32(a, position);
		*mn = sub_f32(p, v3_f32(b.x, b.x, b.x));
		*mx = add_f32(p, v3_f32(b.x, b.x, b.x));
	} else if (type == 5) {
		a = qrot_f32(add_f32(a, position), rotation);
		b = qrot_f32(add_f32(b, position), rotation);
		c = qrot_f32(add_f32(c, position), rotation);
		mn->x = smin(a.x, smin(b.x, c.x)); mn->y = smin(a.y, smin(b.y, c.y)); mn->z = smin(a.z, smin(b.z, c.z));
		mx->x = smax(a.x, smax(b.x, c.x)); mx->y = smax(a.y, smax(b.y, c.y)); mx->z = smax(a.z, smax(b.z, c.z));
	} else if (type == 1 || type == 2 || type == 3) {
		/* ComputeAABBBox(B, A, position, R_local, body_rot): q1 = body_rot*R_local,
		 * half extents |AMat(q1)| * B, centre quatRotate(A, body_rot) + position */
		q4f q1 = qmult_f32(brot, lrot);
		v3f r0, r1, r2;
		amat_f32(q1, &r0, &r1, &r2);
		r0 = v3_f32(fabsf(r0.x), fabsf(r0.y), fabsf(r0.z));
		r1 = v3_f32(fabsf(r1.x), fabsf(r1.y), fabsf(r1.z));
		r2 = v3_f32(fabsf(r2.x), fabsf(r2.y), fabsf(r2.z));
		v3f half = v3_f32(dot_f32(r0, b), dot_f32(r1, b), dot_f32(r2, b));
		v3f p = add_f32(qrot_f32(a, brot), position);
		*mn = sub_f32(p, half);
		*mx = add_f32(p, half);
	} else {
		return 0;
	}
	return 1;
}

/* AABBGenerator::GenerateAABB, AABBGenerator.cu:135-188: aabb[i] = min,
 * aabb[i + n] = max (float3 each); skipped shapes leave aabb untouched. */
CCO_API void cco_aabb(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                      const uint32_t *ID, const float *pos, const float *rot, float *aabb) {
	for (uint64_t i = 0; i < n; i++) {
		v3f mn, mx;
		if (!aabb_one(i, T, A, B, C, R, ID, pos, rot, &mn, &mx)) continue;
		aabb[3 * i] = mn.x; aabb[3 * i + 1] = mn.y; aabb[3 * i + 2] = mn.z;
		aabb[3 * (i + n)] = mx.x; aabb[3 * (i + n) + 1] = mx.y; aabb[3 * (i + n) + 2] = mx.z;
	}
}

/* ------------------------------------------------------------------------ */
/* Broadphase                                                                */
/* ------------------------------------------------------------------------ */

/* float -> int truncation as the reference's host build performs it
 * (HashMin, Broadphase.cu:125-133, assigns a float product to an int; on
 * x86-64 that is cvttss2si, which yields INT_MIN for NaN and for values
 * outside the int range). Written out so the C compiler cannot exploit the
 * undefined behaviour of the plain cast. */
static inline int32_t trunc_i32(float v) {
	if (!(v >= -2147483648.0f && v < 2147483648.0f)) return INT32_MIN;
	return (int32_t)v;
}

/* Grid parameters of Broadphase.cu:368-386: bounds over all 2n corners
 * (fminf/fmaxf, :15-21), origin = fabs(min) (:379), inverse bin size
 * grid / fabs(max + fabs(min)) (:380-381), and the in-place shift
 * aabb += origin (:382-386). */
CCO_API void cco_bounds_shift(uint64_t n, float *aabb, const int32_t *grid, float *origin_out, float *inv_bin_out) {
	float mn[3] = {aabb[0], aabb[1], aabb[2]}, mx[3] = {aabb[0], aabb[1], aabb[2]};
	for (uint64_t i = 0; i < 2 * n; i++)
		for (int d = 0; d < 3; d++) {
			mn[d] = fminf(mn[d], aabb[3 * i + d]);
			mx[d] = fmaxf(mx[d], aabb[3 * i + d]);
		}
	float o[3], s[3];
	for (int d = 0; d < 3; d++) {
		o[d] = fabsf(mn[d]);
		s[d] = fabsf(mx[d] + fabsf(mn[d]));
		s[d] = (float)grid[d] / s[d];
	}
	for (uint64_t i = 0; i < 2 * n; i++)
		for (int d = 0; d < 3; d++) aabb[3 * i + d] = aabb[3 * i + d] + o[d];
	for (int d = 0; d < 3; d++) { origin_out[d] = o[d]; inv_bin_out[d] = s[d]; }
}

/* HashMin (Broadphase.cu:125-133) for one corner. */
static inline void hash_min(const float *p, const float *s, int32_t *g) {
	for (int d = 0; d < 3; d++) g[d] = trunc_i32(p[d] * s[d]);
}

/* Cells per body: function_Count_AABB_BIN_Intersection, Broadphase.cu:150-154
 * (int product, stored as uint). */
static inline uint32_t body_cells(const float *aabb, uint64_t n, uint64_t i, const float *s) {
	int32_t g0[3], g1[3];
	hash_min(aabb + 3 * i, s, g0);
	hash_min(aabb + 3 * (i + n), s, g1);
	int32_t c = (int32_t)((uint32_t)(g1[0] - g0[0] + 1) * (uint32_t)(g1[1] - g0[1] + 1) * (uint32_t)(g1[2] - g0[2] + 1));
	return (uint32_t)c;
}

/* Stable LSD radix sort of (key, value) by key, 8 bits per pass. */
static void radix_sort_kv32(uint32_t *key, uint32_t *val, uint64_t m) {
	uint32_t *k2 = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
	uint32_t *v2 = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
	for (int shift = 0; shift < 32; shift += 8) {
		uint64_t cnt[257] = {0};
		for (uint64_t i = 0; i < m; i++) cnt[((key[i] >> shift) & 255) + 1]++;
		for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
		for (uint64_t i = 0; i < m; i++) {
			uint64_t d = cnt[(key[i] >> shift) & 255]++;
			k2[d] = key[i]; v2[d] = val[i];
		}
		memcpy(key, k2, sizeof(uint32_t) * m);
		memcpy(val, v2, sizeof(uint32_t) * m);
	}
	free(k2); free(v2);
}

static void radix_sort_u64(uint64_t *key, uint64_t m) {
	uint64_t *k2 = (uint64_t *)malloc(sizeof(uint64_t) * (m ? m : 1));
	for (int shift = 0; shift < 64; shift += 8) {
		uint64_t cnt[257] = {0};
		for (uint64_t i = 0; i < m; i++) cnt[((key[i] >> shift) & 255) + 1]++;
		if (cnt[1] == m) continue; /* every digit 0 */
		for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
		for (uint64_t i = 0; i < m; i++) k2[cnt[(key[i] >> shift) & 255]++] = key[i];
		memcpy(key, k2, sizeof(uint64_t) * m);
	}
	free(k2);
}

/* The sorted bin list of Broadphase.cu:394-480 for already-shifted AABBs and
 * inverse bin size s: per-body counts (:150-154), inclusive scan (:403-407),
 * body-major emission with the x-outer / z-inner loop and the unclamped linear
 * index (uint arithmetic) of Hash_Index (:140-147, :172-195), stable
 * sort_by_key (:428-432), reduce_by_key into unique bins (:439-443) and the
 * inclusive end offsets (:476-480).
 * Outputs (each may be NULL to skip): bins[E], bodies[E] in sorted order,
 * active[A], bin_end[A]. Returns E; *n_active = A. Caller sizes arrays from a
 * first call with NULL outputs. */
CCO_API int64_t cco_bins(uint64_t n, const float *aabb, const float *s, const int32_t *grid, uint32_t *bins,
                         uint32_t *bodies, uint32_t *active, uint32_t *bin_end, uint64_t *n_active) {
	uint64_t E = 0;
	for (uint64_t i = 0; i < n; i++) E += body_cells(aabb, n, i, s);
	*n_active = 0;
	uint32_t *bk = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
	uint32_t *bv = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
	uint64_t w = 0;
	const uint32_t gx = (uint32_t)grid[0], gy = (uint32_t)grid[1];
	for (uint64_t i = 0; i < n; i++) {
		int32_t g0[3], g1[3];
		hash_min(aabb + 3 * i, s, g0);
		hash_min(aabb + 3 * (i + n), s, g1);
		for (uint32_t x = (uint32_t)g0[0]; x <= (uint32_t)g1[0]; x++)
			for (uint32_t y = (uint32_t)g0[1]; y <= (uint32_t)g1[1]; y++)
				for (uint32_t z = (uint32_t)g0[2]; z <= (uint32_t)g1[2] && w < E; z++) {
					bk[w] = z * gy * gx + y * gx + x;
					bv[w] = (uint32_t)i;
					w++;
				}
	}
	radix_sort_kv32(bk, bv, E);
	uint64_t A = 0;
	for (uint64_t e = 0; e < E; e++) {
		if (e == 0 || bk[e] != bk[e - 1]) {
			if (active) active[A] = bk[e];
			A++;
		}
		if (bin_end) bin_end[A - 1] = (uint32_t)(e + 1);
	}
	if (bins) memcpy(bins, bk, sizeof(uint32_t) * E);
	if (bodies) memcpy(bodies, bv, sizeof(uint32_t) * E);
	*n_active = A;
	free(bk); free(bv);
	return (int64_t)E;
}

/* Closed AABB overlap, Broadphase.cu:237 / :296. */
static inline int overlap(const float *aabb, uint64_t n, uint32_t a, uint32_t b) {
	const float *amn = aabb + 3 * (uint64_t)a, *amx = aabb + 3 * ((uint64_t)a + n);
	const float *bmn = aabb + 3 * (uint64_t)b, *bmx = aabb + 3 * ((uint64_t)b + n);
	return (amn[0] <= bmx[0] && bmn[0] <= amx[0]) && (amn[1] <= bmx[1] && bmn[1] <= amx[1]) &&
	       (amn[2] <= bmx[2] && bmn[2] <= amx[2]);
}

/* Broadphase::detectPossibleCollisions, Broadphase.cu:344-545: bounds and
 * in-place shift (:368-386), sorted bin list (:394-480), per-bin pair tests
 * over i < k with distinct bodies (:215-246, :265-314) emitting
 * (min << 32) | max, then sort + unique (:522-535). `aabb` is shifted in
 * place. Writes min(P, cap) sorted unique keys and returns P. n == 0 returns
 * 0 (the reference reads aabb_data[0] there, Broadphase.cu:368). */
CCO_API int64_t cco_broadphase(uint64_t n, float *aabb, const int32_t *grid, int64_t *pairs, uint64_t cap) {
	if (n == 0) return 0;
	float o[3], s[3];
	cco_bounds_shift(n, aabb, grid, o, s);
	uint64_t A = 0;
	int64_t E = cco_bins(n, aabb, s, grid, NULL, NULL, NULL, NULL, &A);
	uint32_t *bins = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
	uint32_t *bodies = (uint32_t *)malloc(sizeof(uint32_t) * (E ? E : 1));
	uint32_t *bend = (uint32_t *)malloc(sizeof(uint32_t) * (A ? A : 1));
	cco_bins(n, aabb, s, grid, bins, bodies, NULL, bend, &A);
	uint64_t cap_c = 1024, C = 0;
	uint64_t *cand = (uint64_t *)malloc(sizeof(uint64_t) * cap_c);
	for (uint64_t b = 0; b < A; b++) {
		uint64_t beg = b ? bend[b - 1] : 0, end = bend[b];
		for (uint64_t i = beg; i < end; i++) {
			uint32_t ta = bodies[i];
			for (uint64_t k = i + 1; k < end; k++) {
				uint32_t tb = bodies[k];
				if (ta == tb || !overlap(aabb, n, ta, tb)) continue;
				uint32_t lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
				if (C == cap_c) { cap_c *= 2; cand = (uint64_t *)realloc(cand, sizeof(uint64_t) * cap_c); }
				cand[C++] = ((uint64_t)lo << 32) | hi;
			}
		}
	}
	radix_sort_u64(cand, C);
	uint64_t P = 0;
	for (uint64_t i = 0; i < C; i++)
		if (i == 0 || cand[i] != cand[i - 1]) cand[P++] = cand[i];
	for (uint64_t i = 0; i < P && i < cap; i++) pairs[i] = (int64_t)cand[i];
	free(cand); free(bins); free(bodies); free(bend);
	return (int64_t)P;
}

/* All-pairs closed-overlap test on already-shifted AABBs, without any grid:
 * the set the reference's pair list equals for valid boxes (two overlapping
 * boxes always share a cell because truncation is monotone, and every
 * candidate is re-tested and deduplicated, Broadphase.cu:237, 296, 522-533).
 * Returns P; writes min(P, cap) sorted keys. O(n^2): small n only. */
CCO_API int64_t cco_pairs_bruteforce(uint64_t n, const float *aabb, int64_t *pairs, uint64_t cap) {
	uint64_t P = 0;
	for (uint64_t a = 0; a < n; a++)
		for (uint64_t b = a + 1; b < n; b++)
			if (overlap(aabb, n, (uint32_t)a, (uint32_t)b)) {
				if (P < cap) pairs[P] = (int64_t)((a << 32) | b);
				P++;
			}
	return (int64_t)P;
}
