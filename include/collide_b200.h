/*
 * collide_b200 — C ABI of the B200 (sm_100a) collision pipeline.
 *
 * Drop-in for the collision path of uwsbel/collision-detection
 * ("Chrono::Collide"): AABB generation -> uniform-grid broadphase -> MPR
 * narrowphase. Each entry point below replaces one public method of the
 * reference's C++ classes (cited per function, paths relative to the
 * reference repository). Arguments are plain pointers and sizes; no CUDA or
 * C++ types appear in the signatures.
 *
 * Conventions
 *  - Array pointers are DEVICE pointers (cudaMalloc / thrust::device_vector
 *    storage) unless the function name ends in _host.
 *  - real3 arrays are packed float[3] (12-byte stride, the layout of the
 *    reference's real3 = float3); real4 arrays are float[4] (w, x, y, z) and
 *    must be 16-byte aligned (float4).
 *  - An AABB array holds 2n real3: aabb[i] = min corner, aabb[i + n] = max
 *    corner (AABBGenerator.cu:114-115).
 *  - A pair is the int64 key (min_index << 32) | max_index
 *    (Broadphase.cu:299-308); pair lists are sorted and duplicate-free.
 *  - `stream` is a cudaStream_t (NULL = the legacy default stream). Calls are
 *    stream-ordered and return once their results are complete.
 *  - One cc_ctx must not be used by two host threads at the same time;
 *    distinct contexts are independent.
 *  - Every call returns a cc_status. On CC_ERR_CAPACITY the required count is
 *    stored in the count out-parameter and the result is retained by the
 *    context (see cc_broadphase_fetch).
 */
#ifndef COLLIDE_B200_H
#define COLLIDE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CC_API __attribute__((visibility("default")))
#else
#define CC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cc_ctx cc_ctx;

typedef enum cc_status {
	CC_OK = 0,
	CC_ERR_INVALID_ARGUMENT = 1, /* null pointer with n > 0, misaligned real4 array, negative grid */
	CC_ERR_INVALID_INPUT = 2,    /* an AABB corner is NaN/Inf or has min > max on some axis */
	CC_ERR_CAPACITY = 3,         /* output too small; the required count is returned */
	CC_ERR_CUDA = 4,             /* CUDA runtime error (cc_last_error has the text) */
	CC_ERR_OUT_OF_MEMORY = 5,    /* device allocation failed */
	CC_ERR_INTERNAL = 6,         /* a bounded device-side wait expired */
	CC_ERR_NO_RESULT = 7         /* cc_broadphase_fetch without a retained result */
} cc_status;

/* shape_type of the reference (src/collision_detection.h:57). */
enum {
	CC_SPHERE = 0,
	CC_ELLIPSOID = 1,
	CC_BOX = 2,
	CC_CYLINDER = 3,
	CC_RECT = 4,
	CC_CONE = 5,
	CC_TRIANGLEMESH = 6
};

/* ---- context ------------------------------------------------------------ */

/* Creates a context on CUDA device `device` (the library's scratch memory and
 * tuning state live here). No reference counterpart: the reference classes
 * allocate temporaries inside every call (Broadphase.cu:345-349). */
CC_API cc_status cc_ctx_create(cc_ctx **ctx, int device);
CC_API void cc_ctx_destroy(cc_ctx *ctx);
CC_API const char *cc_status_string(cc_status s);
/* Detail of the last error on this context ("" if none). */
CC_API const char *cc_last_error(const cc_ctx *ctx);
CC_API const char *cc_version(void);

/* Search grid of the pair test. The pair list does not depend on it (two
 * overlapping boxes share a cell of any grid), so by default (0,0,0) the
 * library picks it from the scene bounds, the body count and the mean box
 * extent: cells hold about `cell_target` boxes and are at least `min_ratio`
 * mean box extents wide. (gx,gy,gz) > 0 pins the grid. */
CC_API cc_status cc_set_search_grid(cc_ctx *ctx, int gx, int gy, int gz);
CC_API cc_status cc_set_tuning(cc_ctx *ctx, float cell_target, float min_ratio);
/* Incremental broadphase for time-step updates (default off; the reference
 * rebuilds every step, Broadphase.cu:344-545). A rebuild step of cc_collide
 * (and cc_collide_host) searches the boxes inflated by `margin` (> 0) mean box
 * extents into a sorted candidate pair list and keeps its boxes; a later step
 * whose box corners all moved by less than half the inflation (minus a
 * rounding allowance) tests only those candidates, exactly, on its own
 * shifted boxes and keeps the overlapping ones in order: the sorted pair list
 * of a full search, so results are identical with it on or off. A step that
 * moved too far is redone as a rebuild; a rebuild also happens when the shape
 * count changes and, ahead of time, after a step that used more than half
 * of the allowance. Larger margins rebuild less often and test more
 * candidates. The pipelined host calls (cc_collide_host_submit) do not use
 * it. No reference counterpart. */
CC_API cc_status cc_set_incremental(cc_ctx *ctx, int on, float margin);
/* 1 if the last incremental step rebuilt its candidate list, 0 if it used the
 * kept one, -1 before any incremental step. */
CC_API int cc_last_step_rebuilt(const cc_ctx *ctx);
/* Cells of the search grid holding more than `entries` entries (default 128,
 * at least 128; 0 = never) are tested by the tiled dense-cell kernel instead
 * of lane per entry. Pairs do not depend on it; the tuner picks it with the
 * grid. No reference counterpart. */
CC_API cc_status cc_set_dense_cell(cc_ctx *ctx, uint32_t entries);
/* Launch shape of the sparse pair test: `window` entries staged per warp in
 * shared memory (64, 96 = default, or 128) and a grid cap of `blocks_per_sm`
 * blocks per SM (1..16, default 8). Pairs do not depend on it; the tuner
 * picks it. No reference counterpart. */
CC_API cc_status cc_set_pair_test_shape(cc_ctx *ctx, int window, int blocks_per_sm);
/* Narrowphase precision. The reference runs MPR in `real` (float). Here:
 *  CC_NP_EXACT (default): the reference's MPR arithmetic in FP64 in world
 *    coordinates, operation for operation — contacts equal those of the
 *    reference built with real = double, rounded to float;
 *  CC_NP_FP64: FP64 in a pair-local frame with fused multiply-add (faster,
 *    ~1e-5 p99 normal difference from the exact result on box contacts);
 *  CC_NP_MIXED: as CC_NP_FP64 but FP32 support maps. */
enum { CC_NP_EXACT = 0, CC_NP_FP64 = 1, CC_NP_MIXED = 2 };
CC_API cc_status cc_set_narrowphase_precision(cc_ctx *ctx, int mode);
/* Overlapped narrowphase for cc_collide (default on): after the pair test
 * the MPR runs on the unsorted pair list on a second stream while the list is
 * sorted, and the compaction joins both in sorted order, finding each pair's
 * result through a hash of the contacts. Results are identical either way
 * (a step whose contacts overflow the hash is redone in order). Applies to
 * outputs of at most 2^24 pairs. No reference counterpart. */
CC_API cc_status cc_set_narrowphase_overlap(cc_ctx *ctx, int on);
/* CUDA-graph replay of cc_collide (default on; environment CC_GRAPH_REPLAY=0
 * turns it off at context creation). When the same configuration (sizes,
 * pointers, grid, precision, envelope, tuning) reaches cc_collide twice in a
 * row, its launches are captured once and replayed by one graph launch per
 * call from then on. Results are identical either way. No reference
 * counterpart. */
CC_API cc_status cc_set_graph_replay(cc_ctx *ctx, int on);
/* The grid the last broadphase searched on, and its entry count. */
CC_API cc_status cc_get_last_grid(const cc_ctx *ctx, int *dims3, uint64_t *entries);

/* ---- AABBGenerator::GenerateAABB (src/aabb/AABBGenerator.cuh:21-30,
 *      AABBGenerator.cu:135-188) --------------------------------------------
 * n shapes: T (shape type), A (local position), B (radius / half extents),
 * C, R (local rotation, real4), ID (body of each shape); nb bodies: body_pos,
 * body_rot (real4). Writes aabb[0..2n). Shapes of a type the reference does
 * not bound (RECT, TRIANGLEMESH; AABBGenerator.cu:110-111) are left untouched;
 * type 5 (CONE) is bounded as a triangle, as the reference does (:103-107). */
CC_API cc_status cc_generate_aabb(cc_ctx *ctx, uint64_t n, const int32_t *T, const float *A, const float *B,
                           const float *C, const float *R, const uint32_t *ID, uint64_t nb, const float *body_pos,
                           const float *body_rot, float *aabb, void *stream);

/* ---- Broadphase::detectPossibleCollisions (src/broadphase/Broadphase.cuh:17,
 *      Broadphase.cu:344-545) + setBinsPerAxis (:57-60) + getNumPossibleContacts
 *      (:66-68) ------------------------------------------------------------
 * Shifts `aabb` in place by fabs(min corner) exactly as the reference does
 * (Broadphase.cu:379-386) and writes the sorted unique pair list. (gx,gy,gz)
 * is the reference's bins per axis; it fixes the bin list
 * (cc_broadphase_bins) and the shift, not the pairs. *n_pairs receives the
 * pair count. If pairs_cap < count: returns CC_ERR_CAPACITY, writes nothing,
 * and keeps the result for one cc_broadphase_fetch. On CC_ERR_INVALID_INPUT
 * `aabb` is not modified. n == 0 yields 0 pairs (the reference reads
 * aabb_data[0] there, Broadphase.cu:368). */
CC_API cc_status cc_broadphase(cc_ctx *ctx, uint64_t n, float *aabb, int gx, int gy, int gz, int64_t *pairs,
                        uint64_t pairs_cap, uint64_t *n_pairs, void *stream);
/* Writes the pair list retained by the last cc_broadphase / cc_collide that
 * returned CC_ERR_CAPACITY (once). */
CC_API cc_status cc_broadphase_fetch(cc_ctx *ctx, int64_t *pairs, uint64_t pairs_cap, void *stream);

/* The reference's internal sorted bin list (locals of detectPossibleCollisions,
 * Broadphase.cu:394-480) on grid (gx,gy,gz): bin_number / body_number sorted by
 * bin, then body (:428-432); active_bins = unique bins and bin_end = inclusive
 * end offsets (reduce_by_key :439-443 and scan :476-480). Shifts `aabb` in
 * place like cc_broadphase. Any output may be NULL. Counts are always
 * returned; CC_ERR_CAPACITY if a non-NULL output is too small. */
CC_API cc_status cc_broadphase_bins(cc_ctx *ctx, uint64_t n, float *aabb, int gx, int gy, int gz, uint32_t *bin_number,
                             uint32_t *body_number, uint64_t entries_cap, uint64_t *n_entries, uint32_t *active_bins,
                             uint32_t *bin_end, uint64_t active_cap, uint64_t *n_active, void *stream);

/* ---- Narrowphase::DoNarrowphase (src/narrowphase/Narrowphase.cuh:19-34,
 *      Narrowphase.cu:511-595) + SetCollisionEnvelope (:53-55) --------------
 * Shape and body arrays as in cc_generate_aabb; active[nb] is the body
 * active flag (bool). For each of the n_pairs candidate keys: sphere-sphere
 * analytic contact or MPR. Contacts are written in pair order to
 * norm/cpta/cptb (real3), depth and bids (int32 pairs of body ids); all five
 * outputs need room for n_pairs entries. `pairs` is permuted in place so its
 * first *n_contacts keys are the contacts' pairs (Narrowphase.cu:584-588). */
CC_API cc_status cc_narrowphase(cc_ctx *ctx, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                         const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *body_pos,
                         const float *body_rot, float envelope, int64_t *pairs, uint64_t n_pairs, float *norm,
                         float *cpta, float *cptb, float *depth, int32_t *bids, uint64_t *n_contacts, void *stream);

/* ---- whole pipeline ------------------------------------------------------ */

/* A scene in the reference's shape-array layout. */
typedef struct cc_scene {
	uint64_t n;          /* shapes */
	const int32_t *T;
	const float *A, *B, *C; /* real3[n] */
	const float *R;      /* real4[n] */
	const uint32_t *ID;
	uint64_t nb;         /* bodies */
	const float *body_pos; /* real3[nb] */
	const float *body_rot; /* real4[nb] */
	const uint8_t *active; /* bool[nb] */
} cc_scene;

typedef struct cc_result {
	float *aabb;         /* real3[2n] (shifted, as after detectPossibleCollisions) */
	int64_t *pairs;      /* pairs_cap keys; contacts' pairs first on return */
	uint64_t pairs_cap;
	float *norm, *cpta, *cptb; /* real3[pairs_cap] */
	float *depth;        /* [pairs_cap] */
	int32_t *bids;       /* int32[2 * pairs_cap] */
	uint64_t n_pairs;    /* out */
	uint64_t n_contacts; /* out */
} cc_result;

/* GenerateAABB -> detectPossibleCollisions -> DoNarrowphase, the sequence a
 * Chrono time step runs, with the AABB pass fused into the broadphase's
 * bounds reduction. Device pointers. */
CC_API cc_status cc_collide(cc_ctx *ctx, const cc_scene *scene, int gx, int gy, int gz, float envelope, cc_result *res,
                     void *stream);

/* A batch of independent scenes in one call. The scenes are concatenated:
 * shapes [shape_offsets[s], shape_offsets[s+1]) and bodies
 * [body_offsets[s], body_offsets[s+1]) belong to scene s, and ID holds body
 * indices local to each scene. Offsets are HOST arrays of num_scenes + 1
 * entries starting at 0 and ending at scene.n / scene.nb; all other arrays
 * are on the device. No reference counterpart: it replaces one
 * GenerateAABB -> detectPossibleCollisions -> DoNarrowphase sequence
 * (AABBGenerator.cuh:21-30, Broadphase.cuh:17, Narrowphase.cuh:19-34) per
 * scene. Every scene gets its own bounds, shift and grid, exactly as a
 * separate cc_collide would, and no pair crosses scenes. */
typedef struct cc_batch {
	uint64_t num_scenes;
	const uint64_t *shape_offsets; /* host, num_scenes + 1 */
	const uint64_t *body_offsets;  /* host, num_scenes + 1 */
	cc_scene scene;                /* the concatenated scenes (device) */
} cc_batch;

/* cc_collide over a batch. Outputs use the concatenated numbering:
 * res->aabb holds the mins of all shapes then their maxs (each scene shifted
 * by its own origin), pair keys are (global a << 32 | global b) with
 * a = shape_offsets[s] + local index, bids are global body indices. The pair
 * list is sorted, so it is grouped by scene; contacts come first (stable), so
 * scene s's contacts are [contact_offsets[s], contact_offsets[s+1]).
 * scene_pairs (host, num_scenes) receives each scene's pair count;
 * scene_pairs and contact_offsets (host, num_scenes + 1) may be NULL. On
 * CC_ERR_CAPACITY res->n_pairs is the size needed (call again). */
CC_API cc_status cc_collide_batch(cc_ctx *ctx, const cc_batch *batch, int gx, int gy, int gz, float envelope,
                                  cc_result *res, uint64_t *scene_pairs, uint64_t *contact_offsets, void *stream);

/* cc_collide_batch over scenes that live in separate device allocations
 * (scenes[s] holds scene s's device pointers, IDs local to the scene): the
 * library gathers them into its own concatenated arena with one kernel, then
 * runs the batch. Outputs as cc_collide_batch. No reference counterpart. */
CC_API cc_status cc_collide_scenes(cc_ctx *ctx, uint64_t num_scenes, const cc_scene *scenes, int gx, int gy, int gz,
                                   float envelope, cc_result *res, uint64_t *scene_pairs, uint64_t *contact_offsets,
                                   void *stream);

/* A time-step update of device-resident bodies, as a served simulation sends
 * it: every position component moves by N(0, sigma^2) and every orientation
 * turns by an angle U[0, max_angle] about a uniform random axis
 * (rot = normalize(dq * rot)). The random numbers are a pure function of
 * (seed, body index): the same call gives the same bodies on any launch.
 * Asynchronous on `stream`. No reference counterpart. */
CC_API cc_status cc_perturb_bodies(cc_ctx *ctx, uint64_t nb, float *body_pos, float *body_rot, uint64_t seed,
                                   float sigma, float max_angle, void *stream);

/* The updates of `count` scenes in one launch (a serving pass's time-step
 * queries): scene k's nb[k] bodies at the device arrays body_pos[k] and
 * body_rot[k] move exactly as cc_perturb_bodies(ctx, nb[k], body_pos[k],
 * body_rot[k], seeds[k], sigma, max_angle) moves them. The four argument
 * arrays are host memory and may be reused once the call returns. Entries
 * are applied concurrently, so their body ranges must not overlap: a scene
 * updated twice takes two calls. No reference counterpart. */
CC_API cc_status cc_perturb_scenes(cc_ctx *ctx, uint64_t count, const uint64_t *nb, float *const *body_pos,
                                   float *const *body_rot, const uint64_t *seeds, float sigma, float max_angle,
                                   void *stream);

/* Same with HOST pointers in `scene` and `res` (pinned memory recommended):
 * the inputs are copied to context-owned device buffers, the pipeline runs,
 * and aabb (if non-NULL), pairs and contacts are copied back. The third shape
 * array C is read only for CONE (bounded as a triangle) and TRIANGLEMESH
 * shapes: from a pinned host array a kernel fetches C for those shapes alone
 * through its device mapping (no bytes for a scene without them); a pageable C
 * is copied whole (environment CC_GATHER_C=0 copies it whole always). */
CC_API cc_status cc_collide_host(cc_ctx *ctx, const cc_scene *scene, int gx, int gy, int gz, float envelope,
                          cc_result *res, void *stream);

/* Pipelined form of cc_collide_host for a stream of time steps: submit
 * enqueues one step (copies in on one stream, the pipeline on another, the
 * small counter read-back) and returns at once, so the copy of step k+1 runs
 * while step k computes; wait finishes the OLDEST submitted step: waits for
 * it, copies its pairs and contacts into `res` (the same cc_result that was
 * submitted) and sets res->n_pairs / n_contacts. At most two steps are in
 * flight per context; host buffers must stay untouched until their wait.
 * Work is ordered after the caller's `stream` at submit, and `stream` waits
 * for the step's copies at wait. A step that needs more scratch or more
 * output than the submit provided is redone on the blocking path inside
 * wait, with cc_collide_host's results and status. Stage profiling is not
 * recorded for these calls. No reference counterpart. */
CC_API cc_status cc_collide_host_submit(cc_ctx *ctx, const cc_scene *scene, int gx, int gy, int gz, float envelope,
                                        cc_result *res, void *stream);
CC_API cc_status cc_collide_host_wait(cc_ctx *ctx, cc_result *res, void *stream);
/* Static shapes for host steps (cc_collide_host, cc_collide_host_submit).
 * In a simulation the shape arrays T, A, B, C, R, ID (60 of the 89 bytes per
 * shape and body) stay the same from step to step while the body poses move.
 * With on != 0 a host step copies those six arrays only when their host
 * pointers or the shape count differ from the last copy into the same device
 * buffers; body_pos, body_rot and active are copied every step. The caller
 * must not change the shape arrays' contents in place while this is on, or
 * must call cc_set_static_shapes(ctx, 1) again after doing so: every call of
 * this function drops the kept copies. Off by default; results are identical
 * either way. No reference counterpart (the reference takes device vectors
 * that its caller keeps up to date). */
CC_API cc_status cc_set_static_shapes(cc_ctx *ctx, int on);

/* Number of kernels the last call on this context launched. */
CC_API uint64_t cc_last_launch_count(const cc_ctx *ctx);

/* Stage timing (no reference counterpart). With mode 1, every call brackets
 * each kernel stage with CUDA events on the caller's stream and accumulates
 * the device time per stage. With mode 2, a cc_collide step with the
 * narrowphase in order (cc_set_narrowphase_overlap off) records only two
 * spans, "broadphase_span" (cell count through the sorted pair list) and
 * "narrowphase_span" (MPR and compaction), one event pair each, so that the
 * kernels inside a span run back to back as they do unprofiled. Mode 0 turns
 * timing off. cc_stage_times fills up to `cap` totals in milliseconds and
 * launch counts, indexed by stage id; stage names come from cc_stage_name.
 * cc_reset_stage_times zeroes the totals. */
CC_API cc_status cc_set_profiling(cc_ctx *ctx, int on);
CC_API int cc_stage_count(void);
CC_API const char *cc_stage_name(int stage);
CC_API cc_status cc_stage_times(const cc_ctx *ctx, double *ms, uint64_t *launches, int cap);
CC_API cc_status cc_reset_stage_times(cc_ctx *ctx);

/* Roofline denominator (no reference counterpart): the FP32 (fp64 = 0) or
 * FP64 (fp64 = 1) multiply-add throughput of the current device in FLOP/s,
 * timed with CUDA events on `stream` over a kernel that fills every SM with
 * independent FMA chains (best of three runs after one warm-up). */
CC_API cc_status cc_fma_peak(int fp64, double *flop_per_s, void *stream);

/* ---- broadphase without allocation ---------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory while they run. A real-time step loop cannot
 * afford cudaMalloc/cudaFree, which may synchronize the whole device and take
 * unbounded time; a framework that hands out all device memory from its own
 * pool cannot let a library allocate behind its back. Same contract as cc_broadphase (shifts
 * `aabb` in place, writes the sorted unique pair list, *n_pairs = count), but
 * it needs no context and allocates nothing: its scratch is one fixed
 * CC_NOALLOC_SCRATCH_BYTES device array that every GPU loading the library
 * holds until exit. Limits: n <= CC_NOALLOC_MAX_BODIES, search-grid entries <=
 * CC_NOALLOC_MAX_ENTRIES, pairs <= CC_NOALLOC_MAX_PAIRS; beyond them it returns
 * CC_ERR_CAPACITY (with *n_pairs set once the count is known). pairs_cap below
 * the count also returns CC_ERR_CAPACITY; nothing is retained. The first call
 * on each device looks up the scratch array's device address (once per
 * device, with that device current). The call waits for its stream twice (to
 * read the entry and pair counts). All calls share the one scratch array, which
 * keeps the last call's contents: calls that overlap on the GPU, or that come
 * from two host threads at once, race. */
#define CC_NOALLOC_MAX_BODIES 65536u
#define CC_NOALLOC_MAX_ENTRIES (4u * CC_NOALLOC_MAX_BODIES)
#define CC_NOALLOC_MAX_PAIRS (4u * CC_NOALLOC_MAX_BODIES)
#define CC_NOALLOC_SCRATCH_BYTES (16u << 20)
CC_API cc_status cc_broadphase_noalloc(uint64_t n, float *aabb, int gx, int gy, int gz, int64_t *pairs,
                                       uint64_t pairs_cap, uint64_t *n_pairs, void *stream);

#ifdef __cplusplus
}
#endif

#endif
