/*
 * Test infrastructure (oracle only). Built by oracle/Makefile into
 * oracle/_ref/libccref_f32.so (real=float) and oracle/_ref/libccref_f64.so
 * (real=double, narrowphase only: the FP64 MPR oracle).
 *
 * This translation unit compiles the reference's OWN sources where they lie
 * (src/aabb/AABBGenerator.cu, src/broadphase/Broadphase.cu,
 * src/narrowphase/Narrowphase.cu of uwsbel/collision-detection) in host/OpenMP
 * mode (SIM_ENABLE_GPU_MODE undefined, so custom_vector = thrust::host_vector
 * and EXEC_POLICY = thrust::omp::par, collision_detection.h:60-69) against the
 * gpu_math stand-in in oracle/shim, and wraps the three public classes in a
 * plain C ABI so Python tests, fixture generators and the CPU baseline can
 * call them. Nothing here runs on a GPU.
 */
#include <cstdint>
#include <cstring>
#include <omp.h>

#ifndef CC_SHIM_DOUBLE
/* AABBGenerator.cu is its own translation unit (it defines numAABB_const, as
 * Broadphase.cu:8 does); only its header is needed here. */
#include "Broadphase.cu"
#endif
#include "Narrowphase.cu"

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int ccref_real_bytes() { return (int)sizeof(real); }
REF_API void ccref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
REF_API int ccref_max_threads() { return omp_get_max_threads(); }

template <class V, class S>
static void fill_vec(V &v, const S *src, size_t n) {
	v.resize(n);
	for (size_t i = 0; i < n; i++) v[i] = src[i];
}

static real3 to_r3(const float *p) { return R3(real(p[0]), real(p[1]), real(p[2])); }
static real4 to_r4(const float *p) { return R4(real(p[0]), real(p[1]), real(p[2]), real(p[3])); }

struct RefScene {
	custom_vector<shape_type> T;
	custom_vector<real3> A, B, C;
	custom_vector<real4> R;
	custom_vector<uint> ID;
	custom_vector<bool> active;
	custom_vector<real3> pos;
	custom_vector<real4> rot;
};

static void load_scene(RefScene &s, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                       const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *pos,
                       const float *rot) {
	s.T.resize(n); s.A.resize(n); s.B.resize(n); s.C.resize(n); s.R.resize(n); s.ID.resize(n);
	for (uint64_t i = 0; i < n; i++) {
		s.T[i] = (shape_type)T[i];
		s.A[i] = to_r3(A + 3 * i);
		s.B[i] = to_r3(B + 3 * i);
		s.C[i] = to_r3(C + 3 * i);
		s.R[i] = to_r4(R + 4 * i);
		s.ID[i] = ID[i];
	}
	s.pos.resize(nb); s.rot.resize(nb); s.active.resize(nb);
	for (uint64_t i = 0; i < nb; i++) {
		s.pos[i] = to_r3(pos + 3 * i);
		s.rot[i] = to_r4(rot + 4 * i);
		s.active[i] = active ? (active[i] != 0) : true;
	}
}

#ifndef CC_SHIM_DOUBLE
/* AABBGenerator::GenerateAABB (AABBGenerator.cu:135-188). `aabb` (2n float3,
 * mins then maxs) is read first so that shapes the reference skips
 * (AABBGenerator.cu:110-111) keep the caller's previous values. */
REF_API int ccref_generate_aabb(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                                const float *R, const uint32_t *ID, uint64_t nb, const float *pos, const float *rot,
                                float *aabb) {
	RefScene s;
	load_scene(s, n, T, A, B, C, R, ID, nb, nullptr, pos, rot);
	custom_vector<real3> out(2 * n);
	for (uint64_t i = 0; i < 2 * n; i++) out[i] = to_r3(aabb + 3 * i);
	AABBGenerator gen;
	gen.GenerateAABB(s.T, s.A, s.B, s.C, s.R, s.ID, s.pos, s.rot, out);
	for (uint64_t i = 0; i < 2 * n; i++) {
		aabb[3 * i] = out[i].x; aabb[3 * i + 1] = out[i].y; aabb[3 * i + 2] = out[i].z;
	}
	return 0;
}

/* Broadphase::detectPossibleCollisions (Broadphase.cu:344-545). `aabb` is
 * shifted in place exactly as the reference does (Broadphase.cu:382-386).
 * Returns the number of unique pairs; copies min(P, cap) of them. An empty
 * input returns 0 here: the reference itself reads aabb_data[0]
 * (Broadphase.cu:368) on an empty vector. `par` holds the ten
 * setParallelConfiguration flags (Broadphase.cu:69-90); NULL keeps the
 * constructor default. */
REF_API int64_t ccref_broadphase(uint64_t n, float *aabb, int gx, int gy, int gz, const int32_t *par,
                                 int64_t *pairs, uint64_t cap) {
	if (n == 0) return 0;
	custom_vector<real3> ad(2 * n);
	for (uint64_t i = 0; i < 2 * n; i++) ad[i] = to_r3(aabb + 3 * i);
	custom_vector<long long> pc;
	Broadphase bp;
	bp.setBinsPerAxis(I3(gx, gy, gz));
	if (par) bp.setParallelConfiguration(par[0], par[1], par[2], par[3], par[4], par[5], par[6], par[7], par[8], par[9]);
	bp.detectPossibleCollisions(ad, pc);
	for (uint64_t i = 0; i < 2 * n; i++) {
		aabb[3 * i] = ad[i].x; aabb[3 * i + 1] = ad[i].y; aabb[3 * i + 2] = ad[i].z;
	}
	uint64_t P = bp.getNumPossibleContacts();
	for (uint64_t i = 0; i < P && i < cap; i++) pairs[i] = pc[i];
	return (int64_t)P;
}

/* The reference keeps its sorted bin list in locals of
 * detectPossibleCollisions (Broadphase.cu:345-349). This entry replays
 * steps 2-4 of that function (Broadphase.cu:368-443, 470-480) with the
 * reference's own per-body functions (function_Count_AABB_BIN_Intersection
 * :150, function_Store_AABB_BIN_Intersection :172) and the same Thrust calls,
 * and returns the sorted (bin, body) list, the unique bins and the inclusive
 * end offsets. Sizes: returns E; *n_active receives A. Arrays are filled up to
 * their caps. `aabb` is shifted in place like the reference. */
REF_API int64_t ccref_bins(uint64_t n, float *aabb, int gx, int gy, int gz, uint32_t *bin_number,
                           uint32_t *body_number, uint64_t cap_e, uint32_t *active_bins, uint32_t *bin_end,
                           uint64_t cap_a, uint64_t *n_active) {
	*n_active = 0;
	if (n == 0) return 0;
	custom_vector<real3> ad(2 * n);
	for (uint64_t i = 0; i < 2 * n; i++) ad[i] = to_r3(aabb + 3 * i);
	int3 grid_size = I3(gx, gy, gz);
	uint numAABB = (uint)n;
	bbox init = bbox(ad[0], ad[0]);
	bbox result = thrust::transform_reduce(ad.begin(), ad.end(), bbox_transformation(), init, bbox_reduction());
	real3 global_origin = fabs(result.first);
	real3 bin_size_vec = fabs(result.second + fabs(result.first));
	bin_size_vec = R3(grid_size.x, grid_size.y, grid_size.z) / bin_size_vec;
	thrust::transform(ad.begin(), ad.end(), thrust::constant_iterator<real3>(global_origin), ad.begin(),
	                  thrust::plus<real3>());
	custom_vector<uint> Bins_Intersected(numAABB);
	for (uint i = 0; i < numAABB; i++)
		function_Count_AABB_BIN_Intersection(i, ad.data(), bin_size_vec, numAABB, Bins_Intersected.data());
	thrust::inclusive_scan(Bins_Intersected.begin(), Bins_Intersected.end(), Bins_Intersected.begin());
	uint E = Bins_Intersected.back();
	custom_vector<uint> bn(E), bd(E), bsi(E);
	for (uint i = 0; i < numAABB; i++)
		function_Store_AABB_BIN_Intersection(i, ad.data(), Bins_Intersected.data(), bin_size_vec, grid_size, numAABB,
		                                     bn.data(), bd.data());
	thrust::sort_by_key(bn.begin(), bn.end(), bd.begin());
	for (uint64_t i = 0; i < E && i < cap_e; i++) { bin_number[i] = bn[i]; body_number[i] = bd[i]; }
	uint A = thrust::reduce_by_key(bn.begin(), bn.end(), thrust::constant_iterator<uint>(1), bn.begin(), bsi.begin())
	             .second - bsi.begin();
	bsi.resize(A);
	thrust::inclusive_scan(bsi.begin(), bsi.end(), bsi.begin());
	for (uint64_t i = 0; i < A && i < cap_a; i++) { active_bins[i] = bn[i]; bin_end[i] = bsi[i]; }
	*n_active = A;
	for (uint64_t i = 0; i < 2 * n; i++) {
		aabb[3 * i] = ad[i].x; aabb[3 * i + 1] = ad[i].y; aabb[3 * i + 2] = ad[i].z;
	}
	return (int64_t)E;
}
#endif

/* Narrowphase::DoNarrowphase (Narrowphase.cu:511-595) in the `real` type this file is compiled with.
 * Inputs are float arrays converted to `real`. `pairs` (P keys) is permuted in
 * place like the reference does (Narrowphase.cu:584-588). Contact outputs
 * (norm, cpta, cptb as 3 doubles each, depth, bids as 2 int32) are written
 * for the first n_contacts entries; returns n_contacts. */
REF_API int64_t ccref_narrowphase(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                                  const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active,
                                  const float *pos, const float *rot, float envelope, int64_t *pairs, uint64_t P,
                                  double *norm, double *cpta, double *cptb, double *depth, int32_t *bids) {
	RefScene s;
	load_scene(s, n, T, A, B, C, R, ID, nb, active, pos, rot);
	custom_vector<long long> pc(P);
	for (uint64_t i = 0; i < P; i++) pc[i] = pairs[i];
	custom_vector<real3> nd, ca, cb;
	custom_vector<real> dd;
	custom_vector<int2> bd;
	uint nc = 0;
	Narrowphase np;
	np.SetCollisionEnvelope(real(envelope));
	np.DoNarrowphase(s.T, s.A, s.B, s.C, s.R, s.ID, s.active, s.pos, s.rot, pc, nd, ca, cb, dd, bd, nc);
	for (uint64_t i = 0; i < P; i++) pairs[i] = pc[i];
	for (uint64_t i = 0; i < nc; i++) {
		norm[3 * i] = nd[i].x; norm[3 * i + 1] = nd[i].y; norm[3 * i + 2] = nd[i].z;
		cpta[3 * i] = ca[i].x; cpta[3 * i + 1] = ca[i].y; cpta[3 * i + 2] = ca[i].z;
		cptb[3 * i] = cb[i].x; cptb[3 * i + 1] = cb[i].y; cptb[3 * i + 2] = cb[i].z;
		depth[i] = dd[i];
		bids[2 * i] = bd[i].x; bids[2 * i + 1] = bd[i].y;
	}
	return (int64_t)nc;
}

#ifndef CC_SHIM_DOUBLE
/* A resident scene for timing the reference's CPU path: the host vectors are
 * built once, then each ccref_session_run calls GenerateAABB,
 * detectPossibleCollisions and DoNarrowphase exactly as a Chrono caller would
 * and reports each stage's omp_get_wtime duration. */
struct RefSession {
	RefScene s;
	custom_vector<real3> aabb;
	custom_vector<long long> pairs;
	custom_vector<real3> norm, cpta, cptb;
	custom_vector<real> depth;
	custom_vector<int2> bids;
	AABBGenerator gen;
	Broadphase bp;
	Narrowphase np;
	uint n_contacts;
};

REF_API void *ccref_session_create(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                                   const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active,
                                   const float *pos, const float *rot, int gx, int gy, int gz, int all_parallel) {
	RefSession *s = new RefSession();
	load_scene(s->s, n, T, A, B, C, R, ID, nb, active, pos, rot);
	s->bp.setBinsPerAxis(I3(gx, gy, gz));
	if (all_parallel) s->bp.setParallelConfiguration(1, 1, 1, 1, 1, 1, 1, 1, 1, 1);
	s->n_contacts = 0;
	return s;
}

/* Runs the three stages once. times[0..2] = seconds in GenerateAABB,
 * detectPossibleCollisions, DoNarrowphase. counts[0] = pairs, counts[1] =
 * contacts. */
REF_API int ccref_session_run(void *h, double *times, uint64_t *counts) {
	RefSession *s = (RefSession *)h;
	double t0 = omp_get_wtime();
	s->gen.GenerateAABB(s->s.T, s->s.A, s->s.B, s->s.C, s->s.R, s->s.ID, s->s.pos, s->s.rot, s->aabb);
	double t1 = omp_get_wtime();
	s->bp.detectPossibleCollisions(s->aabb, s->pairs);
	double t2 = omp_get_wtime();
	s->np.DoNarrowphase(s->s.T, s->s.A, s->s.B, s->s.C, s->s.R, s->s.ID, s->s.active, s->s.pos, s->s.rot, s->pairs,
	                    s->norm, s->cpta, s->cptb, s->depth, s->bids, s->n_contacts);
	double t3 = omp_get_wtime();
	times[0] = t1 - t0; times[1] = t2 - t1; times[2] = t3 - t2;
	counts[0] = s->bp.getNumPossibleContacts();
	counts[1] = s->n_contacts;
	return 0;
}

REF_API void ccref_session_destroy(void *h) { delete (RefSession *)h; }
#endif
