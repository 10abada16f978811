/*
 * Test infrastructure (oracle only). Narrowphase restatement, included twice
 * by oracle/cc_oracle.c: once with CCO_R=float / CCO_SFX=_f32 / CCO_SQRT=sqrtf
 * and once with CCO_R=double / CCO_SFX=_f64 / CCO_SQRT=sqrt (the FP64 MPR
 * oracle). Operation order follows
 * the reference line by line with the vector primitives of
 * oracle/shim/includes/gpu_math.h (no fused multiply-add).
 */
#define CCO_CAT2(a, b) a##b
#define CCO_CAT(a, b) CCO_CAT2(a, b)
#define F(name) CCO_CAT(name, CCO_SFX)
#define V3 F(cco_v3)
#define Q4 F(cco_q4)

typedef struct { CCO_R x, y, z; } V3;
typedef struct { CCO_R x, y, z, w; } Q4;  /* (w,i,j,k) in (.x,.y,.z,.w) */

static inline V3 F(v3)(CCO_R x, CCO_R y, CCO_R z) { V3 r = {x, y, z}; return r; }
static inline V3 F(add)(V3 a, V3 b) { return F(v3)(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 F(sub)(V3 a, V3 b) { return F(v3)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 F(mulv)(V3 a, V3 b) { return F(v3)(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 F(muls)(V3 a, CCO_R s) { return F(v3)(a.x * s, a.y * s, a.z * s); }
static inline V3 F(smul)(CCO_R s, V3 a) { return F(v3)(s * a.x, s * a.y, s * a.z); }
static inline V3 F(divs)(V3 a, CCO_R s) { return F(v3)(a.x / s, a.y / s, a.z / s); }
static inline V3 F(neg)(V3 a) { return F(v3)(-a.x, -a.y, -a.z); }
static inline CCO_R F(dot)(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 F(cross)(V3 a, V3 b) {
	return F(v3)(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline CCO_R F(len)(V3 a) { return CCO_SQRT(F(dot)(a, a)); }
static inline V3 F(normalize)(V3 a) { CCO_R l = F(len)(a); return F(v3)(a.x / l, a.y / l, a.z / l); }
static inline CCO_R F(sign)(CCO_R x) { return x > 0 ? (CCO_R)1 : (x < 0 ? (CCO_R)-1 : (CCO_R)0); }
static inline int F(iszero)(CCO_R x) { return fabs((double)x) < (double)FLT_EPSILON; }
static inline int F(iszero3)(V3 a) { return F(iszero)(a.x) && F(iszero)(a.y) && F(iszero)(a.z); }

static inline Q4 F(qmult)(Q4 p, Q4 q) {
	Q4 r;
	r.x = p.x * q.x - p.y * q.y - p.z * q.z - p.w * q.w;
	r.y = p.x * q.y + p.y * q.x + p.z * q.w - p.w * q.z;
	r.z = p.x * q.z - p.y * q.w + p.z * q.x + p.w * q.y;
	r.w = p.x * q.w + p.y * q.z - p.z * q.y + p.w * q.x;
	return r;
}
/* Rows of the rotation matrix of q. */
static inline void F(amat)(Q4 q, V3 *r0, V3 *r1, V3 *r2) {
	const CCO_R w = q.x, x = q.y, y = q.z, z = q.w;
	const CCO_R xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
	const CCO_R wx = w * x, wy = w * y, wz = w * z;
	const CCO_R one = 1, two = 2;
	*r0 = F(v3)(one - two * (yy + zz), two * (xy - wz), two * (xz + wy));
	*r1 = F(v3)(two * (xy + wz), one - two * (xx + zz), two * (yz - wx));
	*r2 = F(v3)(two * (xz - wy), two * (yz + wx), one - two * (xx + yy));
}
static inline V3 F(qrot)(V3 v, Q4 q) {
	V3 r0, r1, r2;
	F(amat)(q, &r0, &r1, &r2);
	return F(v3)(F(dot)(r0, v), F(dot)(r1, v), F(dot)(r2, v));
}
static inline V3 F(qrotT)(V3 v, Q4 q) {
	V3 r0, r1, r2;
	F(amat)(q, &r0, &r1, &r2);
	V3 c0 = F(v3)(r0.x, r1.x, r2.x), c1 = F(v3)(r0.y, r1.y, r2.y), c2 = F(v3)(r0.z, r1.z, r2.z);
	return F(v3)(F(dot)(c0, v), F(dot)(c1, v), F(dot)(c2, v));
}

/* Support maps in the shape's local frame: SupportFunctions.cuh:11-99. */
static V3 F(support_local)(int type, V3 B, V3 n) {
	switch (type) {
	case CCO_SPHERE:  /* :11-13 */
		return F(smul)(B.x, n);
	case CCO_ELLIPSOID: { /* :37-50 */
		V3 nn = F(normalize)(n);
		return F(divs)(F(mulv)(F(mulv)(B, B), nn), F(len)(F(mulv)(B, nn)));
	}
	case CCO_BOX:  /* :30-36 */
		return F(v3)(F(sign)(n.x) * B.x, F(sign)(n.y) * B.y, F(sign)(n.z) * B.z);
	case CCO_CYLINDER: { /* :52-64, axis = local y */
		V3 u = F(v3)(0, 1, 0);
		V3 w = F(sub)(n, F(smul)(F(dot)(u, n), u));
		if (F(len)(w) != 0)
			return F(add)(F(smul)(F(sign)(F(dot)(u, n)) * B.y, u), F(smul)(B.x, F(normalize)(w)));
		return F(smul)(F(sign)(F(dot)(u, n)) * B.y, u);
	}
	case CCO_RECT: { /* :65-73 */
		V3 r = B;
		if (n.x < 0) r.x = -r.x;
		if (n.y < 0) r.y = -r.y;
		return r;
	}
	case CCO_CONE: { /* :74-99 */
		CCO_R radius = B.x, height = B.y;
		CCO_R sa = radius / CCO_SQRT(radius * radius + height * height);
		if (n.y > F(len)(n) * sa) return F(v3)(0, (CCO_R)(height / 2.0), 0);
		CCO_R s = CCO_SQRT(n.x * n.x + n.z * n.z);
		if (s > 1e-9) {
			CCO_R d = radius / s;
			return F(v3)(n.x * d, (CCO_R)(-height / 2.0), n.z * d);
		}
		return F(v3)(0, (CCO_R)(-height / 2.0), 0);
	}
	}
	return F(v3)(0, 0, 0);
}

/* Narrowphase.cu:11-17 */
static V3 F(center)(int type, V3 A, V3 B, V3 C) {
	if (type == CCO_TRIANGLEMESH)
		return F(v3)((A.x + B.x + C.x) / 3.0f, (A.y + B.y + C.y) / 3.0f, (A.z + B.z + C.z) / 3.0f);
	return F(add)(F(v3)(0, 0, 0), A);
}

/* Narrowphase.cu:19-52 (TRIANGLEMESH: SupportFunctions.cuh:14-29 in world frame) */
static V3 F(support)(int type, V3 A, V3 B, V3 C, Q4 R, V3 b) {
	V3 n = F(normalize)(b);
	if (type == CCO_TRIANGLEMESH) {
		CCO_R dist = F(dot)(A, n);
		V3 p = A;
		if (F(dot)(B, n) > dist) { dist = F(dot)(B, n); p = B; }
		if (F(dot)(C, n) > dist) { dist = F(dot)(C, n); p = C; }
		return p;
	}
	V3 rn = F(qrotT)(n, R);
	V3 ls = F(support_local)(type, B, rn);
	return F(add)(F(qrot)(ls, R), A);
}

#define SUP_A(d) F(support)(tA, AX, AY, AZ, AR, (d))
#define SUP_B(d) F(support)(tB, BX, BY, BZ, BR, (d))
#define SWAP3(a, b) do { V3 t_ = (a); (a) = (b); (b) = t_; } while (0)

/* Optional iteration record (test diagnostics): when set, each MPR call
 * stores phase1 * 1000 + phase2 at the sink's cursor (0 for a call that ends
 * before the discovery loop). */
static int32_t *F(g_iter_sink) = 0;
static uint64_t F(g_iter_n) = 0;
#define CCO_ITERS(p1, p2) do { if (F(g_iter_sink)) F(g_iter_sink)[F(g_iter_n)++] = (p1) * 1000 + (p2); } while (0)

/* Minkowski portal refinement: Narrowphase.cu:122-314. Returns hit. */
static int F(mpr)(int tA, V3 AX, V3 AY, V3 AZ, Q4 AR, int tB, V3 BX, V3 BY, V3 BZ, Q4 BR, V3 *rn, V3 *pt, CCO_R *depth) {
	V3 v01 = F(center)(tA, AX, AY, AZ), v02 = F(center)(tB, BX, BY, BZ);
	V3 v0 = F(sub)(v02, v01);
	if (F(iszero3)(v0)) v0 = F(v3)(1, 0, 0);
	V3 n = F(neg)(v0);
	V3 v11 = SUP_A(F(neg)(n)), v12 = SUP_B(n);
	V3 v1 = F(sub)(v12, v11);
	if (F(dot)(v1, n) <= 0.0) { CCO_ITERS(0, 0); return 0; }
	n = F(cross)(v1, v0);
	if (F(iszero3)(n)) {
		CCO_ITERS(0, 0);
		n = F(sub)(v1, v0);
		n = F(normalize)(n);
		*rn = n;
		*pt = F(muls)(F(add)(v11, v12), (CCO_R).5);
		*depth = F(dot)(F(sub)(v12, v11), n);
		return 1;
	}
	V3 v21 = SUP_A(F(neg)(n)), v22 = SUP_B(n);
	V3 v2 = F(sub)(v22, v21);
	if (F(dot)(v2, n) <= 0.0) { CCO_ITERS(0, 0); return 0; }
	n = F(cross)(F(sub)(v1, v0), F(sub)(v2, v0));
	if (F(dot)(n, v0) > 0.0) {
		SWAP3(v1, v2); SWAP3(v11, v21); SWAP3(v12, v22);
		n = F(neg)(n);
	}
	V3 v31, v32, v3;
	int hit = 0, phase1 = 0, phase2 = 0;
	const int max_iterations = 34;
	for (;;) {
		if (phase1 > max_iterations) { CCO_ITERS(phase1, phase2); return 0; }
		phase1++;
		v31 = SUP_A(F(neg)(n)); v32 = SUP_B(n);
		v3 = F(sub)(v32, v31);
		if (F(dot)(v3, n) <= 0.0) { CCO_ITERS(phase1, phase2); return 0; }
		if (F(dot)(F(cross)(v1, v3), v0) < 0.0) {
			v2 = v3; v21 = v31; v22 = v32;
			n = F(cross)(F(sub)(v1, v0), F(sub)(v3, v0));
			continue;
		}
		if (F(dot)(F(cross)(v3, v2), v0) < 0.0) {
			v1 = v3; v11 = v31; v12 = v32;
			n = F(cross)(F(sub)(v3, v0), F(sub)(v2, v0));
			continue;
		}
		for (;;) {
			phase2++;
			n = F(cross)(F(sub)(v2, v1), F(sub)(v3, v1));
			n = F(normalize)(n);
			if (F(dot)(n, v1) >= 0.0 && !hit) hit = 1;
			V3 v41 = SUP_A(F(neg)(n)), v42 = SUP_B(n);
			V3 v4 = F(sub)(v42, v41);
			CCO_R delta = F(dot)(F(sub)(v4, v3), n);
			*depth = F(dot)(v4, n);
			if (delta <= 1e-20 || *depth <= 0.0 || phase2 > max_iterations) {
				if (hit) {
					CCO_R b0 = F(dot)(F(cross)(v1, v2), v3);
					CCO_R b1 = F(dot)(F(cross)(v3, v2), v0);
					CCO_R b2 = F(dot)(F(cross)(v0, v1), v3);
					CCO_R b3 = F(dot)(F(cross)(v2, v1), v0);
					CCO_R sum = b0 + b1 + b2 + b3;
					if (sum <= 0.) {
						b0 = 0;
						b1 = F(dot)(F(cross)(v2, v3), n);
						b2 = F(dot)(F(cross)(v3, v1), n);
						b3 = F(dot)(F(cross)(v1, v2), n);
						sum = b1 + b2 + b3;
					}
					CCO_R inv = 1.0f / sum;
					V3 p = F(add)(F(add)(F(add)(F(smul)(b0, v01), F(smul)(b1, v11)), F(smul)(b2, v21)), F(smul)(b3, v31));
					V3 q = F(add)(F(add)(F(add)(F(smul)(b0, v02), F(smul)(b1, v12)), F(smul)(b2, v22)), F(smul)(b3, v32));
					*pt = F(muls)(F(muls)(F(add)(p, q), inv), (CCO_R).5);
					*rn = F(normalize)(n);
				}
				CCO_ITERS(phase1, phase2);
				return hit;
			}
			if (F(dot)(F(cross)(v4, v1), v0) < 0) {
				if (F(dot)(F(cross)(v4, v2), v0) < 0) { v1 = v4; v11 = v41; v12 = v42; }
				else { v3 = v4; v31 = v41; v32 = v42; }
			} else {
				if (F(dot)(F(cross)(v4, v3), v0) < 0) { v2 = v4; v21 = v41; v22 = v42; }
				else { v1 = v4; v11 = v41; v12 = v42; }
			}
		}
	}
}
#undef SUP_A
#undef SUP_B
#undef SWAP3
#undef CCO_ITERS

CCO_API void F(cco_iter_sink)(int32_t *buf) { F(g_iter_sink) = buf; F(g_iter_n) = 0; }
CCO_API uint64_t F(cco_iter_count)(void) { return F(g_iter_n); }

static inline V3 F(ld3)(const float *p, uint64_t i) { return F(v3)(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline Q4 F(ld4)(const float *p, uint64_t i) {
	Q4 q = {p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]};
	return q;
}

/* Per-pair contact: Narrowphase.cu:316-423. Returns 1 and fills the outputs
 * when the pair is a contact (the reference's contact_active == 0). */
static int F(pair_contact)(int64_t key, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                           const uint32_t *ID, const uint8_t *active, const float *pos, const float *rot,
                           CCO_R envelope_in, V3 *norm, V3 *pa, V3 *pb, CCO_R *depth_out, int32_t *ida, int32_t *idb) {
	int px = (int)(key >> 32), py = (int)(key & 0xffffffff);
	int tA = T[px], tB = T[py];
	uint32_t IDA = ID[px], IDB = ID[py];
	int actA = active ? active[IDA] != 0 : 1, actB = active ? active[IDB] != 0 : 1;
	if (!actA && !actB) return 0;
	if (IDA == IDB) return 0;
	V3 posA = F(ld3)(pos, IDA), posB = F(ld3)(pos, IDB);
	Q4 rotA = F(ld4)(rot, IDA), rotB = F(ld4)(rot, IDB);
	V3 AX = F(ld3)(A, px), BX = F(ld3)(A, py);
	V3 AY = F(ld3)(B, px), BY = F(ld3)(B, py);
	V3 AZ = F(ld3)(C, px), BZ = F(ld3)(C, py);
	Q4 AR = F(qmult)(rotA, F(ld4)(R, px));
	Q4 BR = F(qmult)(rotB, F(ld4)(R, py));
	CCO_R envelope = envelope_in;
	if (tA == CCO_SPHERE || tA == CCO_ELLIPSOID || tA == CCO_BOX || tA == CCO_CYLINDER) {
		AX = F(add)(F(qrot)(AX, rotA), posA);
	} else if (tA == CCO_TRIANGLEMESH) {
		envelope = 0;
		AX = F(qrot)(F(add)(AX, posA), AR);
		AY = F(qrot)(F(add)(AY, posA), AR);
		AZ = F(qrot)(F(add)(AZ, posA), AR);
	}
	if (tB == CCO_SPHERE || tB == CCO_ELLIPSOID || tB == CCO_BOX || tB == CCO_CYLINDER) {
		BX = F(add)(F(qrot)(BX, rotB), posB);
	} else if (tB == CCO_TRIANGLEMESH) {
		envelope = 0;
		BX = F(qrot)(F(add)(BX, posB), BR);
		BY = F(qrot)(F(add)(BY, posB), BR);
		BZ = F(qrot)(F(add)(BZ, posB), BR);
	}
	V3 N = F(v3)(1, 0, 0), p1 = F(v3)(0, 0, 0), p2 = F(v3)(0, 0, 0), p0 = F(v3)(0, 0, 0);
	CCO_R depth = 0;
	if (tA == CCO_SPHERE && tB == CCO_SPHERE) {
		V3 relpos = F(sub)(BX, AX);
		CCO_R d2 = F(dot)(relpos, relpos);
		CCO_R cd = AY.x + BY.x;
		if (!(d2 <= cd * cd)) return 0;
		N = F(normalize)(relpos);
		p1 = F(add)(AX, F(muls)(N, AY.x));
		p2 = F(sub)(BX, F(muls)(N, BY.x));
	} else {
		if (!F(mpr)(tA, AX, AY, AZ, AR, tB, BX, BY, BZ, BR, &N, &p0, &depth)) return 0;
		p1 = F(add)(F(smul)(F(dot)(F(sub)(F(support)(tA, AX, AY, AZ, AR, F(neg)(N)), p0), N), N), p0);
		p2 = F(add)(F(smul)(F(dot)(F(sub)(F(support)(tB, BX, BY, BZ, BR, N), p0), N), N), p0);
		N = F(neg)(N);
	}
	p1 = F(sub)(p1, F(muls)(N, envelope));
	p2 = F(add)(p2, F(muls)(N, envelope));
	depth = F(dot)(N, F(sub)(p2, p1));
	*norm = N; *pa = p1; *pb = p2; *depth_out = depth;
	*ida = (int32_t)IDA; *idb = (int32_t)IDB;
	return 1;
}

/* DoNarrowphase (Narrowphase.cu:511-595): every pair is evaluated, then the
 * contacts are moved to the front in pair order (the stable sort by the
 * 0/1 flag at :584-588) and `pairs` is permuted the same way. Outputs are
 * doubles (3 per vector). Returns the number of contacts. */
int64_t F(cco_narrowphase)(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                           const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *pos,
                           const float *rot, float envelope, int64_t *pairs, uint64_t P, double *norm, double *cpta,
                           double *cptb, double *depth, int32_t *bids) {
	(void)n; (void)nb;
	int64_t *miss = (int64_t *)malloc(sizeof(int64_t) * (P ? P : 1));
	uint64_t nc = 0, nm = 0;
	for (uint64_t i = 0; i < P; i++) {
		V3 N, pa, pb; CCO_R d; int32_t ia, ib;
		if (F(pair_contact)(pairs[i], T, A, B, C, R, ID, active, pos, rot, (CCO_R)envelope, &N, &pa, &pb, &d, &ia, &ib)) {
			norm[3 * nc] = N.x; norm[3 * nc + 1] = N.y; norm[3 * nc + 2] = N.z;
			cpta[3 * nc] = pa.x; cpta[3 * nc + 1] = pa.y; cpta[3 * nc + 2] = pa.z;
			cptb[3 * nc] = pb.x; cptb[3 * nc + 1] = pb.y; cptb[3 * nc + 2] = pb.z;
			depth[nc] = d; bids[2 * nc] = ia; bids[2 * nc + 1] = ib;
			pairs[nc++] = pairs[i];
		} else {
			miss[nm++] = pairs[i];
		}
	}
	for (uint64_t i = 0; i < nm; i++) pairs[nc + i] = miss[i];
	free(miss);
	return (int64_t)nc;
}

#undef V3
#undef Q4
#undef F
