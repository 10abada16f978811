// Internal interfaces between the translation units of libcollide_b200.so.
// Host code only sees launchers (each .cu file owns its kernels); nothing here
// is part of the public C ABI (include/collide_b200.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace cc {

// Uniform search grid of the pair test (chosen on the device from the bounds,
// see make_plan in cc_broadphase.cu). Any monotone cell map finds the same
// pairs, so this grid is free to differ from the caller's bins-per-axis.
struct Plan {
	float lo[3];      // shifted minimum corner of the scene
	float inv[3];     // cells per unit length per axis
	int dim[3];       // cells per axis (1..kMaxDim)
	uint32_t G;       // dim[0] * dim[1] * dim[2]
	float origin[3];  // reference shift: fabs(min) (Broadphase.cu:379)
	float invbin[3];  // reference inverse bin size: grid / fabs(max + fabs(min)) (:380-381)
	int grid[3];      // reference bins per axis
	int valid;        // bounds were finite and every box had min <= max
};

// Per-call device state; zeroed (one memset) at the start of every call.
struct DevStats {
	uint32_t bmin_inv[3];  // ~f2ord(min) accumulated with atomicMax (0 = neutral)
	uint32_t bmax[3];      // f2ord(max) accumulated with atomicMax (0 = neutral)
	uint32_t err;          // DeviceError bits
	uint32_t max_bin;      // largest reference bin id emitted (bin-list path)
	double ext_sum[3];     // sum of sampled AABB extents per axis (tuner input)
	unsigned long long ext_count;  // number of sampled boxes
	unsigned long long pairs;     // unique pairs emitted by the tile test (may exceed capacity)
	unsigned long long entries;   // (cell, body) entries of the search grid
	unsigned long long ref_entries;
	unsigned long long contacts;
	unsigned long long big_segments;  // owner buckets of 33..1024 pairs (listed from the front)
	unsigned long long max_segment;
	unsigned long long seg_big;       // owner buckets of 1025..16384 pairs (listed from the back)
	unsigned long long cells;     // plan.G as a 64-bit scan count
	unsigned long long np_n;      // pairs handed to the narrowphase (0 if an output was too small)
	unsigned long long dense_items;  // (cell, row chunk) work items of the dense-cell pair test
	uint32_t blocks_done;         // last-block detection of the bounds reduction
	uint32_t pad_;
	Plan plan;
	// grid barriers of the cooperative kernels (GridBarrier: arrived, gen),
	// zeroed with the rest at the start of a pass
	uint32_t bar_emit[2];  // k_owner_sort_fused
	uint32_t bar_np[2];
	uint32_t bar_compact[2];
	uint32_t bar_scan[2];  // k_scan_cells_coop
	// incremental steps (candidate lists): largest corner displacement since
	// the rebuild (ordered bits), a step that moved too far, the margin
	uint32_t vdisp;
	uint32_t vbad;
	float vmargin;
	uint32_t pad3_;
};

constexpr int kMaxDim = 1024;  // cells per axis (10-bit packed cell coordinates)

// Tuner parameters of the search grid.
struct GridParams {
	float k_target;   // target mean entries per cell
	float min_ratio;  // minimum cell edge as a multiple of the mean box extent
	int user_dim[3];  // > 0: search on exactly this grid (tuner bypassed)
	uint32_t g_max;   // capacity of the per-cell arrays
	uint32_t dense_cell;  // cells holding more entries go to the tiled dense-cell pair test
	int pair_window;        // sparse pair test: entries staged per warp (64, 96, 128)
	int pair_blocks_per_sm; // sparse pair test: grid cap in blocks per SM
};

// Word ranges the first kernel of a pass zeroes (scan control words, class
// counters, cell counts), replacing a chain of memset launches.
struct ZeroList {
	uint32_t *p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
	uint64_t words[5] = {0, 0, 0, 0, 0};
};

// ------------------------------------------------------------------ scan
// Exclusive scan of `n` uint32 counts into uint64 offsets out[0..n] (out[n] =
// total) with one decoupled look-back pass. status: >= scan_tiles(n) words.
// With n_dev the count is min(n, *n_dev), read on the device; total_out
// (optional) receives the sum.
size_t scan_tiles(uint64_t n);
void launch_scan_u32_to_u64(const uint32_t *in, uint64_t n, unsigned long long *out, uint64_t *status,
                            uint32_t *ticket, uint32_t *err, cudaStream_t s,
                            const unsigned long long *n_dev = nullptr, unsigned long long *total_out = nullptr,
                            bool pre_zeroed = false);
// Same, 32-bit output (caller guarantees total < 2^32). zero_in: the scan
// stores 0 over every input word it read (the cell counts become the
// scatter's cursors without a memset).
void launch_scan_u32_to_u32(const uint32_t *in, uint64_t n, uint32_t *out, uint64_t *status, uint32_t *ticket,
                            uint32_t *err, cudaStream_t s, const unsigned long long *n_dev = nullptr,
                            unsigned long long *total_out = nullptr, bool pre_zeroed = false,
                            uint32_t *zero_in = nullptr);

// ------------------------------------------------------------------ radix sort
// Stable LSD radix sort of 64-bit keys on bits [bit_lo, bit_hi). `keys` and
// `tmp` are n-element buffers; the result ends in `keys`. `hist` needs
// radix_hist_words(n) words, `status` scan_tiles(radix_hist_words(n)) words.
size_t radix_hist_words(uint64_t n);
void radix_sort_u64(unsigned long long *keys, unsigned long long *tmp, uint64_t n, int bit_lo, int bit_hi,
                    uint32_t *hist, unsigned long long *hoff, uint64_t *status, uint32_t *ticket, uint32_t *err,
                    cudaStream_t s);

// ------------------------------------------------------------------ AABB
// GenerateAABB. With `stats` non-null the kernel also accumulates the scene
// bounds, extent sums and validity (the broadphase's first pass) and its last
// block writes the grid plan (stats->plan) for grid dims `grid` and tuning gp.
// Body ids >= nb set kErrBadIndex in *err and leave that shape's AABB unwritten.
void launch_aabb(uint64_t n, const int32_t *T, const float *A, const float *B, const float *C, const float *R,
                 const uint32_t *ID, uint64_t nb, const float *pos, const float *rot, float *aabb, DevStats *stats,
                 uint32_t *err, const GridParams &gp, const int grid[3], cudaStream_t s,
                 const ZeroList &zero = ZeroList());

// ------------------------------------------------------------------ broadphase
// A batch of independent scenes laid out as one concatenated scene: every
// scene has its own bounds, reference shift and search grid (plans[s]); the
// grids occupy disjoint global cell ranges starting at cell_base[s]. Null
// pointers: a single scene whose plan is DevStats::plan.
struct SceneMap {
	const uint32_t *scene_of = nullptr;   // n: scene of every shape
	const Plan *plans = nullptr;          // per scene
	const uint32_t *cell_base = nullptr;  // per scene + 1
};

struct BpBuffers {
	DevStats *stats;
	uint32_t *cell_count;    // g_max
	uint32_t *cell_start;    // g_max + 1
	uint32_t g_max;
	float4 *entries;         // entry_cap * 2 (lo+id, hi+packed cell)
	uint64_t entry_cap;
	uint32_t *owner_count;   // n
	unsigned long long *owner_off;  // n + 1
	unsigned long long *pairs_tmp;  // pair_cap
	uint64_t pair_cap;
	uint64_t *status;        // look-back tiles of the cell scan
	uint32_t *ticket;        // its tile counter
	uint32_t *big_list;      // big segment owners
	uint64_t big_cap;
	uint64_t *status2 = nullptr;  // look-back tiles of the owner scan (null: shares status)
	uint32_t *ticket2 = nullptr;
	bool pre_zeroed = false;      // status/ticket regions were zeroed by the pass's first kernel
	SceneMap sm;                  // batch layout (empty: one scene)
	uint2 *dense = nullptr;       // dense-cell work items (cell, first row)
	uint64_t dense_cap = 0;
	uint32_t dense_cell = 128;    // threshold (entries) of a dense cell
	// Pairs are bucketed by owner (the smaller index a) coarsened to a >> owner_shift:
	// ceil(n / 2^owner_shift) buckets. Inside a bucket the sort keys are packed to
	// 32 bits as ((a mod 2^owner_shift) << key_bits) | b, with key_bits the bits of
	// n - 1 (owner_shift + key_bits <= 32). owner_shift 0: one bucket per body, keys
	// are the partner halves b (batches, incremental steps, the clustered scenes).
	int owner_shift = 0;
	int key_bits = 32;
	// launch shape of the sparse pair test: entries staged per warp (64, 96 or
	// 128) and the grid cap in blocks per SM
	int pair_window = 96;
	int pair_blocks_per_sm = 8;
	// non-null: the fused owner sort (k_owner_sort_fused) emits this call's
	// pairs; k_count zeroes these per-bucket cursors (owner_buckets(n,
	// owner_shift) words, in the owner_off scratch) beside the counts
	uint32_t *owner_cursor = nullptr;
	// non-null: the cell offsets come from the cooperative scan
	// (k_scan_cells_coop), these kScanCoopBlocks words hold its block sums
	unsigned long long *scan_bsum = nullptr;
	// g_max words (start << 32 | cursor) the cooperative scan writes with
	// cursor 0: the scatter takes a slot with one 64-bit atomic instead of a
	// start load plus a cursor atomic (launch_scatter with packed = true)
	unsigned long long *cell_cs = nullptr;
};
constexpr uint32_t kScanCoopBlocks = 2048;
// Owner buckets of n bodies at a shift.
__host__ __device__ inline uint64_t owner_buckets(uint64_t n, int shift) {
	return n ? ((n - 1) >> shift) + 1 : 0;
}

// Bounds pass over caller AABBs; its last block writes stats->plan.
void launch_bounds(uint64_t n, const float *aabb, DevStats *stats, const GridParams &gp, const int grid[3],
                   cudaStream_t s, const ZeroList &zero = ZeroList());
// In-place shift + per-cell counts on the plan's search grid.
void launch_count(uint64_t n, float *aabb, const BpBuffers &b, cudaStream_t s);
void launch_scan_cells(const BpBuffers &b, uint32_t g_max, cudaStream_t s);
void launch_scatter(uint64_t n, const float *aabb, const BpBuffers &b, cudaStream_t s, bool packed = false);
void launch_pair_test(uint64_t n, const BpBuffers &b, uint64_t entries_hint, cudaStream_t s);
void launch_scan_owner(uint64_t n, const BpBuffers &b, cudaStream_t s);
// Cells holding more than b.dense_cell entries are left out of the
// lane-per-entry pair test and tested here instead, tile by tile (N-body
// style); kDenseCell is the default threshold and the smallest sizing unit of
// the work list.
constexpr uint32_t kDenseCell = 128;
void launch_pair_test_dense(const BpBuffers &b, cudaStream_t s);
// Device-driven emission: P is read from stats->pairs. If P exceeds the
// scratch (pair_cap) or out_cap nothing is written and stats->np_n = 0, else
// stats->np_n = P.
void launch_owner_scatter(uint64_t out_cap, unsigned long long *out, const BpBuffers &b, cudaStream_t s);
void launch_segsort(uint64_t n, unsigned long long *out, const BpBuffers &b, cudaStream_t s);
void launch_segsort_mid(unsigned long long *out, const BpBuffers &b, cudaStream_t s);
void launch_segsort_big(unsigned long long *out, const BpBuffers &b, cudaStream_t s);
// The owner scan, bucketing and bucket sorts above as one cooperative kernel,
// for at most 8191 owner buckets (fused_sort_fits); b.owner_cursor must be set
// (and was zeroed by this call's launch_count). Same device-driven contract as
// launch_owner_scatter; P_hint sizes the grid only.
bool fused_sort_fits(uint64_t buckets);
// Environment CC_FUSED_SORT=0 keeps the five-launch owner path everywhere.
bool fused_sort_enabled();
void launch_owner_sort_fused(uint64_t n, uint64_t out_cap, unsigned long long *out, uint64_t P_hint, const BpBuffers &b,
                             cudaStream_t s);

// ------------------------------------------------------------------ incremental steps
// Candidate lists for time-stepped scenes (cc_verlet.cu): the boxes inflated
// by factor x the mean box extent (stats->vmargin receives the margin); the
// largest corner displacement against the rebuild's reference boxes plus a
// copy of the unshifted RECT / TRIANGLEMESH boxes and the in-place shift; the
// candidates that overlap on the shifted boxes, in order, into out
// (stats->pairs and stats->np_n as the pair test and emission set them;
// nothing, and stats->vbad set, when the step moved farther than the
// rebuild's margin allows; a rebuild step always passes).
void launch_vinflate(uint64_t n, const float *aabb, float *scratch, DevStats *stats, float factor, cudaStream_t s);
void launch_vcheck(uint64_t n, float *aabb, const float *ref, float *backup, const int32_t *T, DevStats *stats,
                   cudaStream_t s);
// Words of the status region launch_vcompact needs for nc candidates.
uint64_t vcompact_status_words(uint64_t nc);
void launch_vcompact(uint64_t nc, const unsigned long long *cand, const float *aabb, uint64_t n, DevStats *stats,
                     unsigned long long *out, uint64_t out_cap, uint64_t *status, uint32_t *ticket, bool rebuild,
                     float margin, cudaStream_t s);

// ------------------------------------------------------------------ batches
// Per-scene accumulators of the batch bounds pass (zeroed per call).
struct SceneStats {
	uint32_t bmin_inv[3];  // ~f2ord(min), atomicMax
	uint32_t bmax[3];      // f2ord(max), atomicMax
	uint32_t err;
	uint32_t pad_;
	double ext_sum[3];
	unsigned long long count;
};
// Cells a scene of n_s shapes may use (the single-scene g_max rule).
__host__ __device__ inline uint32_t batch_scene_cells(uint64_t n_s) {
	if (n_s == 0) return 0;
	const uint64_t g = n_s > 4096 ? n_s : 4096;
	return (uint32_t)(g < ((uint64_t)1 << 28) ? g : ((uint64_t)1 << 28));
}
// Device pointers of one scene held in its own allocations, and the
// concatenated destination (16-byte aligned real4 arrays on both sides).
struct SceneSrc {
	const int32_t *T;
	const float *A, *B, *C, *R;
	const uint32_t *ID;
	const float *pos, *rot;
	const uint8_t *active;
};
struct SceneDst {
	int32_t *T;
	float *A, *B, *C, *R;
	uint32_t *ID;
	float *pos, *rot;
	uint8_t *active;
};
void launch_perturb(uint64_t nb, float *pos, float *rot, uint64_t seed, float sigma, float max_angle, cudaStream_t s);
// One scene of a multi-scene update: its bodies are [first, first + nb) of the
// launch's body range (scenes in order, first[0] = 0).
struct PerturbScene {
	float *pos, *rot;
	uint64_t nb, first, seed;
};
void launch_perturb_scenes(uint32_t count, uint64_t total, const PerturbScene *d, float sigma, float max_angle,
                           cudaStream_t s);
// Host -> device copy of a small table (bytes a multiple of 4, at most
// kParamCopyMax) through kernel parameters, in chunks of kParamChunkBytes;
// larger or unaligned tables fall back to cudaMemcpyAsync. The host table may
// be reused as soon as the call returns.
constexpr size_t kParamChunkBytes = 8192;
constexpr size_t kParamCopyMax = 64 * 1024;
cudaError_t copy_small_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s);
void launch_gather(uint64_t n, uint64_t nb, uint32_t S, const unsigned long long *shape_off,
                   const unsigned long long *body_off, const SceneSrc *src, const SceneDst &dst, cudaStream_t s);
// dst[i] = src[i] (3 floats) for the shapes of type CONE or TRIANGLEMESH, the
// only ones whose C is read; T is on the device, src a device-accessible
// (pinned, mapped) host array.
void launch_gather_c(uint64_t n, const int32_t *T, const float *src, float *dst, cudaStream_t s);
void launch_batch_prep(uint64_t n, uint32_t S, const unsigned long long *shape_off, const unsigned long long *body_off,
                       const uint32_t *ID, uint32_t *scene_of, uint32_t *gid, uint32_t *err, cudaStream_t s);
void launch_batch_bounds(uint64_t n, const float *aabb, const uint32_t *scene_of, SceneStats *sst, uint32_t *err,
                         cudaStream_t s);
void launch_batch_plan(uint32_t S, const unsigned long long *shape_off, const SceneStats *sst, const GridParams &gp,
                       const int grid[3], Plan *plans, uint32_t *G, cudaStream_t s);
void launch_batch_offsets(uint32_t S, const unsigned long long *shape_off, const unsigned long long *owner_off,
                          const unsigned long long *np_pos, const DevStats *stats, unsigned long long *scene_pairs,
                          unsigned long long *contact_off, cudaStream_t s);

// Reference-grid bin list (the reference's internal sorted (bin, body) list).
void launch_ref_count(uint64_t n, const float *aabb_shifted, const DevStats *stats, uint32_t *cnt, cudaStream_t s);
void launch_ref_emit(uint64_t n, const float *aabb_shifted, DevStats *stats, const unsigned long long *off,
                     unsigned long long *keys, uint64_t cap, cudaStream_t s);
// Run boundaries of the sorted keys: flags[e] = 1 where a new bin starts.
void launch_ref_flags(const unsigned long long *keys, uint64_t E, uint32_t *flags, cudaStream_t s);
void launch_ref_split(const unsigned long long *keys, uint64_t E, const uint32_t *run_pos, uint32_t *bin_number,
                      uint32_t *body_number, uint32_t *active_bins, uint32_t *bin_end, uint64_t cap_a,
                      cudaStream_t s);

// ------------------------------------------------------------------ narrowphase
struct NpScratch {
	float *norm, *pa, *pb;  // 3 * P each
	float *depth;           // P
	int32_t *ids;           // 2 * P
	unsigned long long *pairs;  // P (copy of the input keys)
	uint32_t *flag;         // P
	unsigned long long *pos;  // P + 1
	uint64_t *status;       // look-back tiles of the flag scan
	uint32_t *ticket;
	uint32_t *err;
	uint32_t *order;        // P: pair indices grouped by (type A, type B)
	uint32_t *classes;      // 2 * kNpClasses counters + the work-queue counter (zeroed per call)
	bool pre_zeroed = false;  // classes, status and ticket already zeroed for this pass
	void *bar_classes = nullptr;  // grid barriers (GridBarrier) of the cooperative class sort and compaction,
	void *bar_compact = nullptr;  // zeroed at the start of the call
	unsigned long long *block_sums = nullptr;  // per-block flag counts of the compaction (>= its grid)
	// Overlapped narrowphase (the MPR on the unsorted pairs while they are
	// sorted): every contact's key -> its pair index, open addressing with
	// linear probing over hmask + 1 slots (0 = empty, else key + 1), zeroed at
	// the start of the pass. Null: the MPR runs on the sorted list.
	unsigned long long *hkeys = nullptr;
	uint32_t *hvals = nullptr;
	uint64_t hmask = 0;
};
constexpr int kNpClasses = 64;  // 7 x 7 shape-type combinations + one for invalid keys
// Grid bound of the narrowphase's cooperative kernels (and the size of
// NpScratch::block_sums).
constexpr unsigned kNpCoopBlocks = 148 * 8;

// Pair indices >= n and body ids >= nb set kErrBadIndex in *sc.err; such a
// pair is reported as no contact. precision: 0 exact (the reference's FP64
// arithmetic), 1 fp64 (pair-local frame), 2 mixed (FP32 support maps).
// P_cap: host bound on the pair count; with P_dev the count is min(P_cap,
// *P_dev), read on the device. P_hint sizes the persistent grid.
void launch_mpr(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T, const float *A,
                const float *B, const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                const uint8_t *active, const float *pos, const float *rot, float envelope, const long long *pairs,
                const NpScratch &sc, int precision, uint64_t P_hint, cudaStream_t s);
// The exact variant lives in its own -fmad=false translation unit.
// Blocks of the exact MPR kernel resident per SM.
int mpr_exact_resident_blocks();
void launch_mpr_exact(unsigned grid, uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T,
                      const float *A, const float *B, const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                      const uint8_t *active, const float *pos, const float *rot, float envelope,
                      const long long *pairs, const NpScratch &sc, cudaStream_t s);
void launch_np_compact(uint64_t P_cap, const unsigned long long *P_dev, const NpScratch &sc, long long *pairs,
                       float *norm, float *cpta, float *cptb, float *depth, int32_t *bids,
                       unsigned long long *contacts_out, uint64_t P_hint, cudaStream_t s);
// The overlapped narrowphase's compaction: the MPR ran on the unsorted pairs
// (results at their unsorted index, contacts in sc's hash); `pairs` holds the
// sorted list of *P_dev keys. Writes the hit-first order into `pairs` and the
// contacts in that order, exactly as launch_np_compact does after an MPR on
// the sorted list. tmp: P_cap keys of scratch.
void launch_np_compact_sorted(uint64_t P_cap, const unsigned long long *P_dev, const NpScratch &sc,
                              long long *pairs, unsigned long long *tmp, float *norm, float *cpta, float *cptb,
                              float *depth, int32_t *bids, unsigned long long *contacts_out, uint64_t P_hint,
                              cudaStream_t s);

}  // namespace cc
