// C ABI of libcollide_b200.so (include/collide_b200.h): context, scratch
// management and the host-side orchestration of the kernels. No kernels live
// here; every device pass is a launcher from cc_aabb.cu, cc_broadphase.cu,
// cc_narrowphase.cu or cc_sort.cu.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/collide_b200.h"
#include "cc_common.cuh"
#include "cc_internal.h"

using namespace cc;

namespace {

struct Buf {
	void *p = nullptr;
	size_t bytes = 0;
	uint64_t allocs = 0;  // times allocated (a new allocation may reuse the old address)
};

// Kernel stages timed by the optional profiler.
enum Stage : int {
	ST_AABB, ST_BOUNDS, ST_COUNT, ST_SCAN_CELLS, ST_SCATTER, ST_PAIR_TEST, ST_SCAN_OWNER, ST_OWNER_SCATTER,
	ST_SEGSORT, ST_MPR, ST_NP_COMPACT, ST_BINS, ST_COPY_IN, ST_COPY_OUT, ST_SEGSORT_MID, ST_SEGSORT_BIG,
	ST_SPAN_BROADPHASE, ST_SPAN_NARROWPHASE, ST_COUNT_
};
const char *kStageNames[ST_COUNT_] = {"aabb", "bounds", "count", "scan_cells", "scatter", "pair_test",
                                      "scan_owner", "owner_scatter", "segsort", "mpr", "np_compact", "bins",
                                      "copy_in", "copy_out", "segsort_mid", "segsort_big",
                                      "broadphase_span", "narrowphase_span"};
// Profiling modes (cc_set_profiling): events around every stage, or only
// around the two spans (one event pair each, so that the kernels inside run
// back to back as they do unprofiled).
constexpr int kProfStages = 1, kProfSpans = 2;
constexpr int kMaxMarks = 64;

// A CUDA graph of one kind of call, replayed while the call's configuration
// (its key: everything its launches depend on) repeats.
struct GraphSlot {
	cudaGraphExec_t exec = nullptr;
	unsigned char key[512] = {};
	unsigned char pending[512] = {};
	size_t key_size = 0;
	bool have_pending = false;
	uint64_t launches = 0;
	void drop() {
		if (exec) cudaGraphExecDestroy(exec);
		exec = nullptr;
		have_pending = false;
		key_size = 0;
	}
};

}  // namespace

struct cc_ctx {
	int device = 0;
	std::string err;
	GridParams gp{};
	cudaError_t cuda_err = cudaSuccess;
	// device scratch
	Buf stats, cell_count, cell_start, entries, owner_count, owner_off, pairs_tmp, status, ticket, big_list, dense;
	Buf ref_cnt, ref_off, ref_keys, ref_tmp, ref_flags, ref_runpos, rx_hist, rx_hoff;
	Buf np_norm, np_pa, np_pb, np_depth, np_ids, np_pairs, np_flag, np_pos, np_order, np_classes, np_bsum;
	Buf bp_bsum;  // block sums of the cooperative cell scan
	Buf cell_cs;  // packed (start, cursor) words of the cells
	Buf in_T, in_A, in_B, in_C, in_R, in_ID, in_pos, in_rot, in_act, out_aabb, out_pairs, out_norm, out_pa, out_pb,
	    out_depth, out_bids;
	// batch scratch: offsets, scene of each shape, global body ids, per-scene
	// stats and plans, scene cell counts and bases, G-scan control, results
	Buf b_off, b_scene_of, b_gid, b_sst, b_plans, b_G, b_base, b_status, b_ticket, b_res;
	// descriptor table of cc_perturb_scenes
	Buf pt_desc;
	// overlapped narrowphase (cc_set_narrowphase_overlap): the MPR on the
	// unsorted pairs on np_stream while the main stream sorts them; the
	// contact hash (keys, values) sized for 4x the expected pair count
	bool np_overlap = true;
	cudaStream_t np_stream = nullptr;
	cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
	Buf np_hkeys, np_hvals;
	uint64_t np_hslots = 0;
	// gather arena of cc_collide_scenes
	Buf g_T, g_A, g_B, g_C, g_R, g_ID, g_pos, g_rot, g_act, g_src, g_off;
	SceneMap sm;  // set while a batch call runs
	DevStats *h_stats = nullptr;  // pinned
	uint64_t *h_word = nullptr;   // pinned scratch words
	// retained broadphase result (owner buckets not yet scattered)
	bool retained = false;
	uint64_t retained_n = 0, retained_P = 0;
	bool retained_fused = false;
	// this call's pairs are emitted by the fused owner sort (one scene, not
	// incremental, few owner buckets); set by prepare and the call
	bool fused_now = false;
	// one scene whose last call found no dense cell: the dense-cell pair test is
	// not launched (the sparse one tests every cell and counts dense ones)
	bool dense_skip = false;
	uint64_t last_dense = 1;  // dense cells of the last call (1: none seen yet)
	uint64_t last_E = 0, last_P = 0;
	int last_dim[3] = {0, 0, 0};
	// owner buckets of the pair sort (BpBuffers::owner_shift / key_bits), chosen
	// per call from the last call's pairs per body
	int owner_shift = 0, key_bits = 32;
	uint64_t launches = 0;
	int np_precision = CC_NP_EXACT;
	// scratch generation: bumped whenever ensure() moves a buffer
	uint64_t buf_gen = 0;
	// ensure() in dry-run mode records would_grow instead of reallocating
	bool dry_run = false, would_grow = false;
	// host steps with static shapes (cc_set_static_shapes): which host arrays
	// of which size each device copy of the six shape arrays holds; a copy is
	// reused while on, the same and of the current generation (every setter
	// call starts a new one)
	struct ShapeCopy {
		const void *src[6] = {};
		void *dst[6] = {};
		uint64_t allocs[6] = {};  // the device buffers' allocation counts at the copy
		uint64_t n = 0, gen = 0;
	};
	bool static_shapes = false;
	uint64_t shapes_gen = 1;
	ShapeCopy in_shapes, hs_shapes[2];
	// pipelined host steps (cc_collide_host_submit / _wait): two slots of
	// device inputs and outputs; copies in on one stream, the pipeline on
	// another, copies out on a third
	struct HostSlot {
		Buf T, A, B, C, R, ID, pos, rot, act, aabb, pairs, norm, pa, pb, depth, bids;
		cudaEvent_t in_done = nullptr, done = nullptr;
		DevStats *h_stats = nullptr;  // pinned copy of the step's counters
		cc_scene dev{};
		cc_result *res = nullptr;
		int grid[3] = {0, 0, 0};
		float env = 0.f;
		uint64_t cap = 0, entry_cap = 0, pair_cap = 0;
	} hs[2];
	cudaStream_t hs_copy = nullptr, hs_comp = nullptr, hs_out = nullptr;
	cudaEvent_t hs_user = nullptr, hs_back = nullptr;
	int hs_next = 0, hs_oldest = 0, hs_inflight = 0;
	// look-back status regions (words) of the cell, owner and contact-flag
	// scans, laid out back to back in `status`
	uint64_t st_words[3] = {0, 0, 0};
	// incremental broadphase (cc_set_incremental, cc_verlet.cu): the sorted
	// candidate pairs of the boxes inflated by inc_margin mean extents, the
	// rebuild's unshifted boxes, a copy of the current step's unshifted boxes,
	// and the compaction's look-back words; the candidates are used while the
	// scene keeps its size (and the buffers holding them were not moved)
	bool incremental = false, inc_valid = false;
	float inc_margin = 0.5f;
	uint64_t inc_n = 0, inc_allocs = 0, inc_nc = 0;
	float inc_m = 0.f, inc_disp = 0.f;  // the rebuild's margin; the last step's largest displacement
	int last_rebuilt = -1;
	Buf v_ref, v_backup, v_scratch, v_cand, v_status;
	// the current pass's first kernel zeroed the scan control words, the
	// narrowphase class counters and the cell counts (ZeroList)
	bool pass_zeroed = false;
	// CUDA graph of the whole device pipeline (cc_collide), replayed while its
	// configuration (GraphKey) is unchanged
	cudaStream_t cap_stream = nullptr;
	bool graph_off = false;
	GraphSlot g_collide, g_batch;  // cc_collide's step and the batch pass
	// stage profiler
	int prof = 0;  // 0, kProfStages or kProfSpans
	cudaEvent_t ev[2 * kMaxMarks] = {};
	int mark_stage[kMaxMarks] = {};
	int nmarks = 0;
	double stage_ms[ST_COUNT_] = {};
	uint64_t stage_n[ST_COUNT_] = {};
};

namespace {

cc_status set_err(cc_ctx *c, cc_status st, const char *fmt, ...) {
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	c->err = buf;
	return st;
}

#define CC_CUDA(c, expr)                                                                                 \
	do {                                                                                                 \
		cudaError_t e_ = (expr);                                                                         \
		if (e_ != cudaSuccess) {                                                                         \
			(c)->cuda_err = e_;                                                                          \
			return set_err((c), e_ == cudaErrorMemoryAllocation ? CC_ERR_OUT_OF_MEMORY : CC_ERR_CUDA,   \
			               "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);        \
		}                                                                                                \
	} while (0)

#define CC_TRY(expr)                    \
	do {                                \
		cc_status s_ = (expr);          \
		if (s_ != CC_OK) return s_;     \
	} while (0)

cc_status ensure(cc_ctx *c, Buf &b, size_t bytes) {
	if (bytes <= b.bytes) return CC_OK;
	if (c->dry_run) {  // only report that this call would reallocate
		c->would_grow = true;
		return CC_OK;
	}
	size_t nb = std::max(bytes, b.bytes + b.bytes / 2);
	nb = (nb + 255) & ~size_t(255);
	if (b.p) {
		CC_CUDA(c, cudaFree(b.p));
		b.p = nullptr;
		b.bytes = 0;
	}
	CC_CUDA(c, cudaMalloc(&b.p, nb));
	b.bytes = nb;
	b.allocs++;
	c->buf_gen++;
	return CC_OK;
}

template <class T>
T *ptr(const Buf &b) { return reinterpret_cast<T *>(b.p); }

// Brackets one stage with events when profiling is on (RAII).
struct StageMark {
	cc_ctx *c;
	int slot = -1;
	cudaStream_t s;
	StageMark(cc_ctx *c_, int stage, cudaStream_t s_) : c(c_), s(s_) {
		const bool span = stage == ST_SPAN_BROADPHASE || stage == ST_SPAN_NARROWPHASE;
		if (c->prof != (span ? kProfSpans : kProfStages) || c->nmarks >= kMaxMarks) return;
		slot = c->nmarks++;
		c->mark_stage[slot] = stage;
		cudaEventRecord(c->ev[2 * slot], s);
	}
	~StageMark() {
		if (slot >= 0) cudaEventRecord(c->ev[2 * slot + 1], s);
	}
};

void prof_collect(cc_ctx *c);

// Collects a call's stage marks on every return path.
struct ProfGuard {
	cc_ctx *c;
	cudaStream_t s;
	ProfGuard(cc_ctx *c_, void *s_) : c(c_), s((cudaStream_t)s_) { c->nmarks = 0; }
	~ProfGuard() {
		if (c->prof && c->nmarks) {
			cudaStreamSynchronize(s);
			prof_collect(c);
		}
	}
};

// Folds the completed marks of a call into the totals (after its final sync).
void prof_collect(cc_ctx *c) {
	for (int i = 0; i < c->nmarks; i++) {
		float ms = 0.f;
		if (cudaEventElapsedTime(&ms, c->ev[2 * i], c->ev[2 * i + 1]) == cudaSuccess) {
			c->stage_ms[c->mark_stage[i]] += ms;
			c->stage_n[c->mark_stage[i]] += 1;
		}
	}
	c->nmarks = 0;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

cc_status check_launch(cc_ctx *c) {
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) {
		c->cuda_err = e;
		return set_err(c, CC_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
	}
	return CC_OK;
}

cc_status read_stats(cc_ctx *c, cudaStream_t s) {
	CC_CUDA(c, cudaMemcpyAsync(c->h_stats, c->stats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, s));
	CC_CUDA(c, cudaStreamSynchronize(s));
	return CC_OK;
}

cc_status device_err(cc_ctx *c) {
	const uint32_t e = c->h_stats->err;
	if (e & (kErrNonFinite | kErrInverted))
		return set_err(c, CC_ERR_INVALID_INPUT, "AABB input has %s%s", (e & kErrNonFinite) ? "non-finite corners " : "",
		               (e & kErrInverted) ? "boxes with min > max" : "");
	if (e & kErrBadIndex) return set_err(c, CC_ERR_INVALID_INPUT, "a body id is >= nb");
	if (e & kErrSpinLimit) return set_err(c, CC_ERR_INTERNAL, "device-side look-back wait gave up");
	return CC_OK;
}

uint32_t g_max_for(uint64_t n) {
	uint64_t g = std::max<uint64_t>(4096, n);
	return (uint32_t)std::min<uint64_t>(g, (uint64_t)1 << 28);
}

BpBuffers bp_buffers(cc_ctx *c) {
	BpBuffers b;
	b.stats = ptr<DevStats>(c->stats);
	b.cell_count = ptr<uint32_t>(c->cell_count);
	b.cell_start = ptr<uint32_t>(c->cell_start);
	b.g_max = c->gp.g_max;
	b.entries = ptr<float4>(c->entries);
	b.entry_cap = c->entries.bytes / (2 * sizeof(float4));
	b.owner_count = ptr<uint32_t>(c->owner_count);
	b.owner_off = ptr<unsigned long long>(c->owner_off);
	b.pairs_tmp = ptr<unsigned long long>(c->pairs_tmp);
	b.pair_cap = c->pairs_tmp.bytes / sizeof(unsigned long long);
	b.status = ptr<uint64_t>(c->status);
	b.ticket = ptr<uint32_t>(c->ticket);
	b.status2 = b.status + c->st_words[0];
	b.ticket2 = b.ticket + 4;
	b.big_list = ptr<uint32_t>(c->big_list);
	b.big_cap = c->big_list.bytes / sizeof(uint32_t);
	b.pre_zeroed = c->pass_zeroed;
	b.owner_cursor = c->fused_now ? ptr<uint32_t>(c->owner_off) : nullptr;
	b.scan_bsum = c->bp_bsum.p ? ptr<unsigned long long>(c->bp_bsum) : nullptr;
	b.cell_cs = c->cell_cs.p && c->cell_cs.bytes >= sizeof(unsigned long long) * c->gp.g_max
	                ? ptr<unsigned long long>(c->cell_cs)
	                : nullptr;
	b.sm = c->sm;
	b.dense = c->dense_skip ? nullptr : ptr<uint2>(c->dense);
	b.dense_cap = c->dense.bytes / sizeof(uint2);
	b.dense_cell = c->gp.dense_cell;
	b.owner_shift = c->owner_shift;
	b.key_bits = c->key_bits;
	b.pair_window = c->gp.pair_window;
	b.pair_blocks_per_sm = c->gp.pair_blocks_per_sm;
	return b;
}

// Owner buckets of the pair sort for n bodies: about 8 pairs per bucket at the
// last call's pair count (n / 4 before any), so that the bucket scan and the
// per-bucket sorts touch ~P/8 buckets instead of n owners. A sparse scene
// (1M mixed shapes, 0.026 pairs per body) gets 2^8 owners per bucket, a dense
// one (hundreds of pairs per body) one owner per bucket. The shift moves only
// when the ideal differs by two or more, so a captured graph stays valid while
// the pair count drifts. The packed in-bucket keys need shift + bits(n - 1) <= 32.
void choose_owner_shift(cc_ctx *c, uint64_t n) {
	int kb = 1;
	while (kb < 32 && ((uint64_t)1 << kb) < n) kb++;
	const double P = (double)std::max<uint64_t>(c->last_P ? c->last_P : n / 4, 1);
	int ideal = (int)std::floor(std::log2(8.0 * (double)std::max<uint64_t>(n, 1) / P));
	ideal = std::max(0, std::min(ideal, std::min(16, 32 - kb)));
	int cur = std::min(c->owner_shift, 32 - kb);
	if (std::abs(ideal - cur) >= 2 || c->key_bits != kb) cur = ideal;
	c->owner_shift = n < 2 ? 0 : cur;
	c->key_bits = kb;
}

// Words of a look-back status region for a scan over n elements (rounded to
// 256 bytes).
size_t status_words_for(uint64_t n) { return (scan_tiles(n) + 8 + 31) & ~size_t(31); }
cc_status ensure_status(cc_ctx *c) {
	return ensure(c, c->status, sizeof(uint64_t) * (c->st_words[0] + c->st_words[1] + c->st_words[2]));
}

// Narrowphase scratch for up to P pairs.
cc_status np_prepare(cc_ctx *c, uint64_t P) {
	P = std::max<uint64_t>(P, 1);
	CC_TRY(ensure(c, c->np_norm, 12 * P));
	CC_TRY(ensure(c, c->np_pa, 12 * P));
	CC_TRY(ensure(c, c->np_pb, 12 * P));
	CC_TRY(ensure(c, c->np_depth, 4 * P));
	CC_TRY(ensure(c, c->np_ids, 8 * P));
	CC_TRY(ensure(c, c->np_pairs, 8 * P));
	CC_TRY(ensure(c, c->np_flag, 4 * P));
	CC_TRY(ensure(c, c->np_pos, 8 * (P + 1)));
	CC_TRY(ensure(c, c->np_order, 4 * P));
	CC_TRY(ensure(c, c->np_classes, (2 * kNpClasses + 32) * sizeof(uint32_t)));
	CC_TRY(ensure(c, c->np_bsum, kNpCoopBlocks * sizeof(unsigned long long)));
	CC_TRY(ensure(c, c->stats, sizeof(DevStats)));
	c->st_words[2] = std::max<uint64_t>(c->st_words[2], status_words_for(P + 1));
	CC_TRY(ensure_status(c));
	CC_TRY(ensure(c, c->ticket, 64));
	return CC_OK;
}

// Allocates the n-dependent broadphase scratch and, if np_cap > 0, the
// narrowphase scratch for np_cap pairs. Buffers only grow; every public call
// ends with a synchronize, so nothing in flight uses a buffer replaced here.
cc_status prepare(cc_ctx *c, uint64_t n, uint64_t np_cap, uint64_t g_override = 0) {
	c->gp.g_max = g_override ? (uint32_t)g_override : g_max_for(n);
	if (g_override) {  // a batch: its per-scene pair counts are read at scene boundaries of the owner offsets
		c->owner_shift = 0;
		c->key_bits = 32;
	} else {
		choose_owner_shift(c, n);
	}
	c->fused_now = !g_override && fused_sort_enabled() && fused_sort_fits(owner_buckets(n, c->owner_shift));
	c->dense_skip = !g_override && c->last_dense == 0;
	CC_TRY(ensure(c, c->stats, sizeof(DevStats)));
	CC_TRY(ensure(c, c->bp_bsum, sizeof(unsigned long long) * kScanCoopBlocks));
	CC_TRY(ensure(c, c->cell_cs, sizeof(unsigned long long) * c->gp.g_max));
	CC_TRY(ensure(c, c->cell_count, sizeof(uint32_t) * c->gp.g_max));
	CC_TRY(ensure(c, c->cell_start, sizeof(uint32_t) * (c->gp.g_max + 1)));
	CC_TRY(ensure(c, c->owner_count, sizeof(uint32_t) * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->owner_off, sizeof(unsigned long long) * (n + 1)));
	const uint64_t e_guess = std::max<uint64_t>(c->last_E + c->last_E / 4, 2 * n + 1024);
	CC_TRY(ensure(c, c->entries, 2 * sizeof(float4) * e_guess));
	const uint64_t p_guess = std::max<uint64_t>(c->last_P + c->last_P / 4, n / 4 + 1024);
	CC_TRY(ensure(c, c->pairs_tmp, sizeof(unsigned long long) * p_guess));
	c->st_words[0] = std::max<uint64_t>(c->st_words[0], status_words_for(c->gp.g_max));
	c->st_words[1] = std::max<uint64_t>(c->st_words[1], status_words_for(n + 1));
	CC_TRY(ensure_status(c));
	CC_TRY(ensure(c, c->ticket, 64));
	CC_TRY(ensure(c, c->big_list, sizeof(uint32_t) * (n + 1024)));
	CC_TRY(ensure(c, c->dense, sizeof(uint2) * (c->entries.bytes / (2 * sizeof(float4)) / kDenseCell + 1024)));
	if (np_cap) CC_TRY(np_prepare(c, np_cap));
	return CC_OK;
}

NpScratch np_scratch(cc_ctx *c) {
	NpScratch sc;
	sc.norm = ptr<float>(c->np_norm);
	sc.pa = ptr<float>(c->np_pa);
	sc.pb = ptr<float>(c->np_pb);
	sc.depth = ptr<float>(c->np_depth);
	sc.ids = ptr<int32_t>(c->np_ids);
	sc.pairs = ptr<unsigned long long>(c->np_pairs);
	sc.flag = ptr<uint32_t>(c->np_flag);
	sc.pos = ptr<unsigned long long>(c->np_pos);
	sc.status = ptr<uint64_t>(c->status) + c->st_words[0] + c->st_words[1];
	sc.ticket = ptr<uint32_t>(c->ticket) + 8;
	sc.bar_classes = ptr<DevStats>(c->stats)->bar_np;
	sc.bar_compact = ptr<DevStats>(c->stats)->bar_compact;
	sc.block_sums = ptr<unsigned long long>(c->np_bsum);
	sc.err = &ptr<DevStats>(c->stats)->err;
	sc.order = ptr<uint32_t>(c->np_order);
	sc.classes = ptr<uint32_t>(c->np_classes);
	sc.pre_zeroed = c->pass_zeroed;
	return sc;
}

// Arguments of the narrowphase stage.
struct NpArgs {
	uint64_t n, nb;
	const int32_t *T;
	const float *A, *B, *C, *R;
	const uint32_t *ID;
	const uint8_t *active;
	const float *pos, *rot;
	float envelope;
	int64_t *pairs;
	float *norm, *cpta, *cptb, *depth;
	int32_t *bids;
};

// Launch-shape hints from the previous call's sizes, rounded up to a power of
// two so that a captured graph stays valid while sizes drift (every kernel
// loops over the device-side count, so any launch shape is correct).
uint64_t pow2ceil(uint64_t v) {
	uint64_t p = 1;
	while (p < v) p <<= 1;
	return p;
}
uint64_t hint_E(const cc_ctx *c, uint64_t n) { return pow2ceil(std::max<uint64_t>(c->last_E, n)); }
uint64_t hint_P(const cc_ctx *c) { return pow2ceil(std::max<uint64_t>(c->last_P, 1)); }

// count .. owner scan: needs stats zeroed and the plan from the bounds pass.
void enqueue_search(cc_ctx *c, uint64_t n, float *aabb, cudaStream_t s, bool owner_scan = true) {
	BpBuffers b = bp_buffers(c);
	const uint32_t gmax = c->gp.g_max;
	{
		StageMark m(c, ST_COUNT, s);
		if (!b.pre_zeroed) cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * gmax, s);
		launch_count(n, aabb, b, s);
	}
	{
		StageMark m(c, ST_SCAN_CELLS, s);
		launch_scan_cells(b, gmax, s);
	}
	{
		StageMark m(c, ST_SCATTER, s);
		launch_scatter(n, aabb, b, s, b.scan_bsum && b.cell_cs);  // the cell scan wrote the packed cursors
	}
	{
		StageMark m(c, ST_PAIR_TEST, s);
		launch_pair_test(n, b, hint_E(c, n), s);
	}
	owner_scan = owner_scan && !c->fused_now;  // the fused owner sort scans the buckets itself
	if (owner_scan) {
		StageMark m(c, ST_SCAN_OWNER, s);
		launch_scan_owner(n, b, s);
	}
	// count, cell scan, scatter, sparse + dense pair test, owner scan
	c->launches += (owner_scan ? 6 : 5) - (c->dense_skip ? 1 : 0);
}

// Sorted pair list into `out` (device-driven: writes nothing if the pair
// count exceeds out_cap or the scratch).
void enqueue_emit(cc_ctx *c, uint64_t n, unsigned long long *out, uint64_t out_cap, cudaStream_t s) {
	BpBuffers b = bp_buffers(c);
	if (c->fused_now) {
		StageMark m(c, ST_SEGSORT, s);
		launch_owner_sort_fused(n, out_cap, out, hint_P(c), b, s);
		c->launches += 1;
		return;
	}
	{
		StageMark m(c, ST_OWNER_SCATTER, s);
		launch_owner_scatter(out_cap, out, b, s);
	}
	{
		StageMark m(c, ST_SEGSORT, s);
		launch_segsort(n, out, b, s);
	}
	{
		StageMark m(c, ST_SEGSORT_MID, s);
		launch_segsort_mid(out, b, s);
	}
	{
		StageMark m(c, ST_SEGSORT_BIG, s);
		launch_segsort_big(out, b, s);
	}
	c->launches += 4;
}

// Narrowphase over min(P_cap, *P_dev) pairs (P_dev null: exactly P_cap).
void enqueue_np(cc_ctx *c, const NpArgs &a, uint64_t P_cap, const unsigned long long *P_dev, cudaStream_t s) {
	if (!P_cap) return;
	NpScratch sc = np_scratch(c);
	{
		StageMark m(c, ST_MPR, s);
		launch_mpr(P_cap, P_dev, a.n, a.T, a.A, a.B, a.C, a.R, a.ID, a.nb, a.active, a.pos, a.rot, a.envelope,
		           reinterpret_cast<const long long *>(a.pairs), sc, c->np_precision,
		           P_dev ? hint_P(c) : P_cap, s);
	}
	{
		StageMark m(c, ST_NP_COMPACT, s);
		launch_np_compact(P_cap, P_dev, sc, reinterpret_cast<long long *>(a.pairs), a.norm, a.cpta, a.cptb, a.depth,
		                  a.bids, &ptr<DevStats>(c->stats)->contacts, P_dev ? hint_P(c) : P_cap, s);
	}
	c->launches += 3;  // class grouping, MPR, compaction
}

// The step after the pair test with the narrowphase overlapped (one scene):
// the MPR runs on the unsorted pairs on c->np_stream (forked after the pair
// test) while `s` sorts them into a.pairs; the compaction joins both and
// finds each sorted key's result through the contact hash.
cc_status enqueue_sort_and_np_overlapped(cc_ctx *c, uint64_t n, const NpArgs &a, uint64_t pairs_cap,
                                         cudaStream_t s) {
	DevStats *d = ptr<DevStats>(c->stats);
	BpBuffers b = bp_buffers(c);
	NpScratch sc = np_scratch(c);
	sc.hkeys = ptr<unsigned long long>(c->np_hkeys);
	sc.hvals = ptr<uint32_t>(c->np_hvals);
	sc.hmask = c->np_hslots - 1;
	CC_CUDA(c, cudaEventRecord(c->ev_fork, s));
	CC_CUDA(c, cudaStreamWaitEvent(c->np_stream, c->ev_fork, 0));
	{
		StageMark m(c, ST_MPR, c->np_stream);
		launch_mpr(std::min<uint64_t>(pairs_cap, b.pair_cap), &d->pairs, a.n, a.T, a.A, a.B, a.C, a.R, a.ID, a.nb,
		           a.active, a.pos, a.rot, a.envelope, reinterpret_cast<const long long *>(b.pairs_tmp), sc,
		           c->np_precision, hint_P(c), c->np_stream);
	}
	CC_CUDA(c, cudaEventRecord(c->ev_join, c->np_stream));
	if (!c->fused_now) {
		StageMark m(c, ST_SCAN_OWNER, s);
		launch_scan_owner(n, b, s);
		c->launches += 1;
	}
	c->launches += 2;  // class grouping, MPR
	enqueue_emit(c, n, reinterpret_cast<unsigned long long *>(a.pairs), pairs_cap, s);
	CC_CUDA(c, cudaStreamWaitEvent(s, c->ev_join, 0));
	{
		StageMark m(c, ST_NP_COMPACT, s);
		launch_np_compact_sorted(pairs_cap, &d->np_n, sc, reinterpret_cast<long long *>(a.pairs), b.pairs_tmp,
		                         a.norm, a.cpta, a.cptb, a.depth, a.bids, &d->contacts, hint_P(c), s);
	}
	c->launches += 1;
	return CC_OK;
}

// Zeroes the per-pass counters before the passes after the count are redone.
cc_status reset_pass_counters(cc_ctx *c, uint64_t n, cudaStream_t s) {
	DevStats *d = ptr<DevStats>(c->stats);
	CC_CUDA(c, cudaMemsetAsync(c->cell_count.p, 0, sizeof(uint32_t) * c->gp.g_max, s));
	CC_CUDA(c, cudaMemsetAsync(c->owner_count.p, 0, sizeof(uint32_t) * n, s));
	if (c->fused_now) CC_CUDA(c, cudaMemsetAsync(c->owner_off.p, 0, sizeof(uint32_t) * n, s));  // the cursors
	CC_CUDA(c, cudaMemsetAsync(&d->err, 0, sizeof(uint32_t), s));
	CC_CUDA(c, cudaMemsetAsync(&d->pairs, 0, sizeof(unsigned long long), s));
	CC_CUDA(c, cudaMemsetAsync(&d->contacts, 0, sizeof(unsigned long long), s));
	CC_CUDA(c, cudaMemsetAsync(&d->big_segments, 0, 3 * sizeof(unsigned long long), s));
	CC_CUDA(c, cudaMemsetAsync(&d->np_n, 0, sizeof(unsigned long long), s));
	CC_CUDA(c, cudaMemsetAsync(&d->dense_items, 0, sizeof(unsigned long long), s));
	return CC_OK;
}

// After the synchronize: if a scratch guess (entries, unsorted pairs) was too
// small, grow it and redo the passes after the count (rare: the guesses
// follow the previous call). h_stats is current on return.
cc_status settle(cc_ctx *c, uint64_t n, float *aabb, unsigned long long *out, uint64_t out_cap, const NpArgs *np,
                 cudaStream_t s) {
	for (int round = 0; round < 3; round++) {
		const uint64_t E = c->h_stats->entries, P = c->h_stats->pairs;
		BpBuffers b = bp_buffers(c);
		if (E <= b.entry_cap && P <= b.pair_cap) return CC_OK;
		if (E >= 0xffffffffull)
			return set_err(c, CC_ERR_CAPACITY, "search grid needs %llu entries (>= 2^32)", (unsigned long long)E);
		if (E > b.entry_cap) {
			CC_TRY(ensure(c, c->entries, 2 * sizeof(float4) * (E + E / 8)));
			CC_TRY(ensure(c, c->dense, sizeof(uint2) * ((E + E / 8) / kDenseCell + 1024)));
		}
		if (P > b.pair_cap) CC_TRY(ensure(c, c->pairs_tmp, sizeof(unsigned long long) * (P + P / 8)));
		CC_TRY(reset_pass_counters(c, n, s));
		b = bp_buffers(c);
		launch_scatter(n, aabb, b, s);
		launch_pair_test(n, b, E, s);
		if (!c->fused_now) launch_scan_owner(n, b, s);
		c->launches += 4 - (c->fused_now ? 1 : 0) - (c->dense_skip ? 1 : 0);
		if (out) enqueue_emit(c, n, out, out_cap, s);
		if (np) enqueue_np(c, *np, out_cap, &ptr<DevStats>(c->stats)->np_n, s);
		CC_TRY(check_launch(c));
		CC_TRY(read_stats(c, s));
		CC_TRY(device_err(c));
	}
	return set_err(c, CC_ERR_INTERNAL, "broadphase scratch did not converge");
}

// A bucket longer than the block sort handles: sort the whole list (rare).
cc_status sort_fallback(cc_ctx *c, uint64_t n, uint64_t P, unsigned long long *out, cudaStream_t s) {
	const size_t hw = radix_hist_words(P);
	CC_TRY(ensure(c, c->ref_tmp, sizeof(unsigned long long) * P));
	CC_TRY(ensure(c, c->rx_hist, sizeof(uint32_t) * hw));
	CC_TRY(ensure(c, c->rx_hoff, sizeof(unsigned long long) * (hw + 1)));
	CC_TRY(ensure(c, c->status, sizeof(uint64_t) * status_words_for(hw + 1)));
	int bits = 1;
	while (bits < 32 && ((uint64_t)1 << bits) < n) bits++;
	{
		StageMark m(c, ST_SEGSORT, s);
		radix_sort_u64(out, ptr<unsigned long long>(c->ref_tmp), P, 0, 32 + bits, ptr<uint32_t>(c->rx_hist),
		               ptr<unsigned long long>(c->rx_hoff), ptr<uint64_t>(c->status), ptr<uint32_t>(c->ticket),
		               &ptr<DevStats>(c->stats)->err, s);
	}
	c->launches += 3 * ((32 + bits + 7) / 8);
	CC_TRY(check_launch(c));
	CC_CUDA(c, cudaStreamSynchronize(s));
	return CC_OK;
}

void remember(cc_ctx *c) {
	c->last_E = c->h_stats->entries;
	c->last_P = c->h_stats->pairs;
	c->last_dense = c->h_stats->dense_items;
	for (int d = 0; d < 3; d++) c->last_dim[d] = c->h_stats->plan.dim[d];
}

void retain(cc_ctx *c, uint64_t n, uint64_t P) {
	c->retained = true;
	c->retained_n = n;
	c->retained_P = P;
	c->retained_fused = c->fused_now;
}

// Writes the retained pair list into `out` (cap >= P checked by the caller).
cc_status emit_retained(cc_ctx *c, unsigned long long *out, uint64_t cap, cudaStream_t s) {
	PdlScope pdl_(c->retained_n);
	DevStats *d = ptr<DevStats>(c->stats);
	c->h_word[0] = c->retained_P;
	CC_CUDA(c, cudaMemcpyAsync(&d->pairs, c->h_word, sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
	CC_CUDA(c, cudaMemsetAsync(&d->big_segments, 0, 3 * sizeof(unsigned long long), s));
	CC_CUDA(c, cudaMemsetAsync(&d->err, 0, sizeof(uint32_t), s));
	c->fused_now = c->retained_fused;
	enqueue_emit(c, c->retained_n, out, cap, s);
	CC_TRY(check_launch(c));
	CC_TRY(read_stats(c, s));
	c->retained = false;
	if (c->h_stats->err & kErrSegmentTooLong) CC_TRY(sort_fallback(c, c->retained_n, c->retained_P, out, s));
	return CC_OK;
}

cc_status check_scene(cc_ctx *c, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                      const float *R, const uint32_t *ID, uint64_t nb, const float *pos, const float *rot) {
	if (n == 0) return CC_OK;
	if (!T || !A || !B || !C || !R || !ID || !pos || !rot || nb == 0)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "null shape/body array with n = %llu", (unsigned long long)n);
	if (!aligned16(R) || !aligned16(rot))
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "real4 arrays (R, body_rot) must be 16-byte aligned");
	return CC_OK;
}

cc_status check_grid(cc_ctx *c, int gx, int gy, int gz) {
	if (gx < 0 || gy < 0 || gz < 0) return set_err(c, CC_ERR_INVALID_ARGUMENT, "negative bins per axis");
	return CC_OK;
}

// Runs enqueue_all on `s`, or replays its graph: a configuration (key) that
// reaches the slot twice in a row is captured on the context's capture stream
// and replayed by one graph launch from then on. Where capture fails the
// context stays on stream launches.
template <class F>
cc_status run_graphed(cc_ctx *c, GraphSlot &g, const void *key, size_t ksize, F &&enqueue_all, cudaStream_t s) {
	bool replayed = false;
	if (!c->prof && !c->graph_off && ksize <= sizeof(g.key)) {
		if (g.exec && g.key_size == ksize && memcmp(key, g.key, ksize) == 0) {
			replayed = true;
		} else if (g.have_pending && memcmp(key, g.pending, ksize) == 0) {
			if (!c->cap_stream) CC_CUDA(c, cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
			const uint64_t l0 = c->launches;
			cudaGraph_t gr = nullptr;
			cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeRelaxed);
			cc_status st = CC_OK;
			if (e == cudaSuccess) {
				st = enqueue_all(c->cap_stream);
				e = cudaStreamEndCapture(c->cap_stream, &gr);
			}
			if (st != CC_OK) {
				if (gr) cudaGraphDestroy(gr);
				c->launches = l0;
				g.have_pending = false;
				return st;
			}
			g.launches = c->launches - l0;
			c->launches = l0;
			g.drop();
			if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, gr, 0);
			if (gr) cudaGraphDestroy(gr);
			if (e == cudaSuccess) {
				memcpy(g.key, key, ksize);
				g.key_size = ksize;
				replayed = true;
			} else {  // not capturable here: stay on stream launches
				cudaGetLastError();
				g.exec = nullptr;
				c->graph_off = true;
			}
		} else {
			memcpy(g.pending, key, ksize);
			g.have_pending = true;
		}
	}
	if (replayed) {
		CC_CUDA(c, cudaGraphLaunch(g.exec, s));
		c->launches += g.launches;
	} else {
		CC_TRY(enqueue_all(s));
	}
	return check_launch(c);
}

// The first half of collide_dev: sizes the scratch and enqueues the whole step
// on `s` (or replays its graph when `graphs`), without waiting.
cc_status collide_enqueue(cc_ctx *c, const cc_scene &sc, int gx, int gy, int gz, float envelope, float *aabb,
                          int64_t *pairs, uint64_t pairs_cap, float *norm, float *cpta, float *cptb, float *depth,
                          int32_t *bids, cudaStream_t s, bool graphs) {
	c->retained = false;
	const uint64_t n = sc.n;
	PdlScope pdl_(n);
	CC_TRY(prepare(c, n, pairs_cap));
	// overlapped narrowphase: one scene, an output of at most 2^24 pairs
	const bool ov = c->np_overlap && pairs_cap > 0 && pairs_cap <= ((uint64_t)1 << 24);
	if (ov) {
		if (!c->np_stream) CC_CUDA(c, cudaStreamCreateWithFlags(&c->np_stream, cudaStreamNonBlocking));
		if (!c->ev_fork) CC_CUDA(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
		if (!c->ev_join) CC_CUDA(c, cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
		c->np_hslots = pow2ceil(std::max<uint64_t>(4 * std::min<uint64_t>(hint_P(c), pairs_cap), 4096));
		CC_TRY(ensure(c, c->np_hkeys, sizeof(unsigned long long) * c->np_hslots));
		CC_TRY(ensure(c, c->np_hvals, sizeof(uint32_t) * c->np_hslots));
	}
	DevStats *d = ptr<DevStats>(c->stats);
	const int grid[3] = {gx, gy, gz};
	unsigned long long *out = reinterpret_cast<unsigned long long *>(pairs);
	const NpArgs a = {n, sc.nb, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.active, sc.body_pos, sc.body_rot, envelope,
	                  pairs, norm, cpta, cptb, depth, bids};
	// the AABB kernel also zeroes the pass's scan control words, class
	// counters and cell counts
	ZeroList zero;
	zero.p[0] = ptr<uint32_t>(c->status);
	zero.words[0] = 2 * (c->st_words[0] + c->st_words[1] + c->st_words[2]);
	zero.p[1] = ptr<uint32_t>(c->ticket);
	zero.words[1] = 16;
	zero.p[2] = ptr<uint32_t>(c->np_classes);
	zero.words[2] = 2 * kNpClasses + 1;
	zero.p[3] = ptr<uint32_t>(c->cell_count);
	zero.words[3] = c->gp.g_max;
	if (ov) {  // the contact hash starts empty
		zero.p[4] = ptr<uint32_t>(c->np_hkeys);
		zero.words[4] = 2 * c->np_hslots;
	}
	for (int r = 0; r < 5; r++)
		if (!zero.p[r]) zero.words[r] = 0;
	auto enqueue_all = [&](cudaStream_t st) -> cc_status {
		{
			StageMark m(c, ST_AABB, st);
			CC_CUDA(c, cudaMemsetAsync(d, 0, sizeof(DevStats), st));
			launch_aabb(n, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.nb, sc.body_pos, sc.body_rot, aabb, d, &d->err,
			            c->gp, grid, st, zero);
		}
		c->launches += 1;
		c->pass_zeroed = true;
		if (ov) {
			enqueue_search(c, n, aabb, st, false);
			const cc_status r = enqueue_sort_and_np_overlapped(c, n, a, pairs_cap, st);
			c->pass_zeroed = false;
			return r;
		}
		{
			StageMark m(c, ST_SPAN_BROADPHASE, st);
			enqueue_search(c, n, aabb, st);
			enqueue_emit(c, n, out, pairs_cap, st);
		}
		{
			StageMark m(c, ST_SPAN_NARROWPHASE, st);
			enqueue_np(c, a, pairs_cap, &d->np_n, st);
		}
		c->pass_zeroed = false;
		return CC_OK;
	};
	if (!graphs) {
		CC_TRY(enqueue_all(s));
		return check_launch(c);
	}
	// everything the captured launches depend on
	struct {
		uint64_t n, nb, pairs_cap, hE, hP, gen, st[3];
		const void *p[18];
		int dims[3], prec, oshift, kbits, ov, fused, dense_skip;
		float env;
		GridParams gp;
		uint64_t hslots;
	} k;
	memset(&k, 0, sizeof(k));
	k.n = n; k.nb = sc.nb; k.pairs_cap = pairs_cap; k.hE = hint_E(c, n); k.hP = hint_P(c); k.gen = c->buf_gen;
	for (int r = 0; r < 3; r++) k.st[r] = c->st_words[r];
	const void *ps[18] = {sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.active, sc.body_pos, sc.body_rot, aabb,
	                      pairs, norm, cpta, cptb, depth, bids, nullptr, nullptr};
	memcpy(k.p, ps, sizeof(ps));
	k.dims[0] = gx; k.dims[1] = gy; k.dims[2] = gz; k.prec = c->np_precision; k.env = envelope; k.gp = c->gp;
	k.oshift = c->owner_shift; k.kbits = c->key_bits; k.ov = ov ? 1 : 0; k.hslots = ov ? c->np_hslots : 0;
	k.fused = c->fused_now ? 1 : 0;
	k.dense_skip = c->dense_skip ? 1 : 0;
	return run_graphed(c, c->g_collide, &k, sizeof(k), enqueue_all, s);
}

// The second half: with c->h_stats current (the step's DevStats), checks
// errors, redoes passes whose scratch was too small, and reports the counts.
cc_status collide_finish(cc_ctx *c, const cc_scene &sc, float envelope, float *aabb, int64_t *pairs,
                         uint64_t pairs_cap, float *norm, float *cpta, float *cptb, float *depth, int32_t *bids,
                         uint64_t *n_pairs, uint64_t *n_contacts, cudaStream_t s) {
	const uint64_t n = sc.n;
	DevStats *d = ptr<DevStats>(c->stats);
	unsigned long long *out = reinterpret_cast<unsigned long long *>(pairs);
	const NpArgs a = {n, sc.nb, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.active, sc.body_pos, sc.body_rot, envelope,
	                  pairs, norm, cpta, cptb, depth, bids};
	CC_TRY(device_err(c));
	CC_TRY(settle(c, n, aabb, out, pairs_cap, &a, s));
	remember(c);
	const uint64_t P = c->h_stats->pairs;
	*n_pairs = P;
	if (P > pairs_cap) {
		retain(c, n, P);
		return set_err(c, CC_ERR_CAPACITY, "pair list needs %llu entries, capacity %llu", (unsigned long long)P,
		               (unsigned long long)pairs_cap);
	}
	if (c->h_stats->err & kErrSegmentTooLong) {
		// the list was sorted bucket-wise only up to 4096 per bucket: sort it whole, redo the narrowphase
		CC_TRY(sort_fallback(c, n, P, out, s));
		CC_CUDA(c, cudaMemsetAsync(&d->contacts, 0, sizeof(unsigned long long), s));
		enqueue_np(c, a, pairs_cap, &d->np_n, s);
		CC_TRY(check_launch(c));
		CC_TRY(read_stats(c, s));
	} else if (c->h_stats->err & kErrHashFull) {
		// more contacts than the overlapped narrowphase's hash took: run it again on the sorted list,
		// which its compaction kept in the unsorted-pair scratch before permuting the output
		CC_CUDA(c, cudaMemcpyAsync(out, c->pairs_tmp.p, sizeof(unsigned long long) * P, cudaMemcpyDeviceToDevice, s));
		CC_CUDA(c, cudaMemsetAsync(&d->contacts, 0, sizeof(unsigned long long), s));
		enqueue_np(c, a, pairs_cap, &d->np_n, s);
		CC_TRY(check_launch(c));
		CC_TRY(read_stats(c, s));
	}
	if (c->h_stats->err & kErrBadIndex)
		return set_err(c, CC_ERR_INVALID_INPUT, "a pair index is >= n or a body id is >= nb");
	*n_contacts = c->h_stats->contacts;
	return CC_OK;
}

// One incremental step of one scene (cc_set_incremental; cc_verlet.cu). A
// rebuild step (the first, a new size, moved candidate buffers, a step that
// used more than half of the margin last time, or a redo) searches the boxes
// inflated by the margin with the full broadphase into the sorted candidate
// list and keeps the unshifted boxes as the reference; every step then checks
// the displacement, shifts the boxes in place, keeps the candidates that
// overlap (in order) and runs the narrowphase on them. A step that moved too
// far is redone as a rebuild from its unshifted boxes. Two synchronizes in a
// rebuild step, one otherwise.
cc_status collide_verlet(cc_ctx *c, const cc_scene &sc, int gx, int gy, int gz, float envelope, float *aabb,
                         int64_t *pairs, uint64_t pairs_cap, float *norm, float *cpta, float *cptb, float *depth,
                         int32_t *bids, uint64_t *n_pairs, uint64_t *n_contacts, cudaStream_t s) {
	const uint64_t n = sc.n;
	PdlScope pdl_(n);
	const int grid[3] = {gx, gy, gz};
	unsigned long long *out = reinterpret_cast<unsigned long long *>(pairs);
	const NpArgs a = {n, sc.nb, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.active, sc.body_pos, sc.body_rot, envelope,
	                  pairs, norm, cpta, cptb, depth, bids};
	for (int attempt = 0; attempt < 2; attempt++) {
		CC_TRY(prepare(c, n, pairs_cap));
		DevStats *d = ptr<DevStats>(c->stats);  // (allocated by the first prepare)
		c->pass_zeroed = false;
		CC_TRY(ensure(c, c->v_ref, 24 * n));
		CC_TRY(ensure(c, c->v_backup, 24 * n));
		const uint64_t allocs = c->v_ref.allocs + c->v_cand.allocs;
		const bool rebuild = attempt > 0 || !c->inc_valid || c->inc_n != n || c->inc_allocs != allocs ||
		                     c->inc_disp > 0.25f * c->inc_m;
		const auto enqueue_front = [&](cudaStream_t st) -> cc_status {
			CC_CUDA(c, cudaMemsetAsync(d, 0, sizeof(DevStats), st));
			launch_aabb(n, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.nb, sc.body_pos, sc.body_rot, aabb, d, &d->err,
			            c->gp, grid, st);
			c->launches += 1;
			return CC_OK;
		};
		if (rebuild) {
			CC_TRY(enqueue_front(s));
			c->inc_valid = false;
			CC_TRY(ensure(c, c->v_scratch, 24 * n));
			const uint64_t want = std::max<uint64_t>(2 * c->inc_nc, std::max<uint64_t>(c->last_P, n / 4) + 1024);
			CC_TRY(ensure(c, c->v_cand, sizeof(unsigned long long) * want));
			// the compaction's look-back words sized with the list, so that a
			// slightly longer list next time allocates nothing
			CC_TRY(ensure(c, c->v_status,
			              sizeof(uint64_t) * vcompact_status_words(c->v_cand.bytes / sizeof(unsigned long long))));
			float *scratch = ptr<float>(c->v_scratch);
			unsigned long long *cand = ptr<unsigned long long>(c->v_cand);
			CC_CUDA(c, cudaMemcpyAsync(c->v_ref.p, aabb, 24 * n, cudaMemcpyDeviceToDevice, s));
			launch_vinflate(n, aabb, scratch, d, c->inc_margin, s);
			uint64_t cap = c->v_cand.bytes / sizeof(unsigned long long);
			enqueue_search(c, n, scratch, s);
			enqueue_emit(c, n, cand, cap, s);
			c->launches += 1;
			CC_TRY(check_launch(c));
			CC_TRY(read_stats(c, s));
			CC_TRY(device_err(c));
			CC_TRY(settle(c, n, scratch, cand, cap, nullptr, s));
			uint64_t nc = c->h_stats->pairs;
			if (nc > cap) {  // more candidates than the list holds: grow it and emit the retained pairs
				CC_TRY(ensure(c, c->v_cand, sizeof(unsigned long long) * (nc + nc / 8)));
				cand = ptr<unsigned long long>(c->v_cand);
				cap = c->v_cand.bytes / sizeof(unsigned long long);
				retain(c, n, nc);
				CC_TRY(emit_retained(c, cand, cap, s));
				c->retained = false;
				CC_TRY(check_launch(c));
				CC_TRY(read_stats(c, s));
			}
			if (c->h_stats->err & kErrSegmentTooLong) CC_TRY(sort_fallback(c, n, nc, cand, s));
			c->inc_nc = nc;
			c->inc_m = c->h_stats->vmargin;
			// the step goes on with its own counters: clear what the search left
			CC_CUDA(c, cudaMemsetAsync(&d->err, 0, sizeof(uint32_t), s));
			CC_CUDA(c, cudaMemsetAsync(&d->pairs, 0, sizeof(unsigned long long), s));
			CC_CUDA(c, cudaMemsetAsync(&d->np_n, 0, sizeof(unsigned long long), s));
			CC_CUDA(c, cudaMemsetAsync(&d->contacts, 0, sizeof(unsigned long long), s));
			CC_CUDA(c, cudaMemsetAsync(&d->big_segments, 0, 3 * sizeof(unsigned long long), s));
		}
		const uint64_t nc = c->inc_nc;
		CC_TRY(ensure(c, c->v_status, sizeof(uint64_t) * vcompact_status_words(nc)));
		const auto enqueue_tail = [&](cudaStream_t st) -> cc_status {
			{
				StageMark m(c, ST_COUNT, st);
				launch_vcheck(n, aabb, ptr<float>(c->v_ref), ptr<float>(c->v_backup), sc.T, d, st);
			}
			{
				StageMark m(c, ST_PAIR_TEST, st);
				launch_vcompact(nc, ptr<unsigned long long>(c->v_cand), aabb, n, d, out, pairs_cap,
				                ptr<uint64_t>(c->v_status), ptr<uint32_t>(c->ticket) + 12, rebuild, c->inc_m, st);
			}
			c->launches += 2;
			enqueue_np(c, a, pairs_cap, &d->np_n, st);
			return CC_OK;
		};
		if (!rebuild) CC_TRY(enqueue_front(s));
		CC_TRY(enqueue_tail(s));
		CC_TRY(check_launch(c));
		CC_TRY(read_stats(c, s));
		CC_TRY(device_err(c));
		if (c->h_stats->vbad) {
			// moved too far: redo as a rebuild, from the caller's RECT / TRIANGLEMESH boxes (the
			// backup's other entries are stale; GenerateAABB rewrites those boxes first)
			CC_CUDA(c, cudaMemcpyAsync(aabb, c->v_backup.p, 24 * n, cudaMemcpyDeviceToDevice, s));
			continue;
		}
		c->last_rebuilt = rebuild ? 1 : 0;
		c->inc_disp = c->h_stats->vdisp ? ord2f_host(c->h_stats->vdisp) : 0.f;
		c->inc_valid = true;
		c->inc_n = n;
		c->inc_allocs = c->v_ref.allocs + c->v_cand.allocs;
		const uint64_t P = c->h_stats->pairs;
		c->last_P = P;
		*n_pairs = P;
		if (P > pairs_cap)
			return set_err(c, CC_ERR_CAPACITY, "pair list needs %llu entries, capacity %llu", (unsigned long long)P,
			               (unsigned long long)pairs_cap);
		if (c->h_stats->err & kErrBadIndex)
			return set_err(c, CC_ERR_INVALID_INPUT, "a pair index is >= n or a body id is >= nb");
		*n_contacts = c->h_stats->contacts;
		return CC_OK;
	}
	return set_err(c, CC_ERR_INTERNAL, "incremental step did not settle");
}

// GenerateAABB -> broadphase -> narrowphase on device pointers with one
// synchronize in the common case.
cc_status collide_dev(cc_ctx *c, const cc_scene &sc, int gx, int gy, int gz, float envelope, float *aabb,
                      int64_t *pairs, uint64_t pairs_cap, float *norm, float *cpta, float *cptb, float *depth,
                      int32_t *bids, uint64_t *n_pairs, uint64_t *n_contacts, cudaStream_t s) {
	*n_pairs = 0;
	*n_contacts = 0;
	c->retained = false;
	if (sc.n == 0) return CC_OK;
	if (c->incremental)
		return collide_verlet(c, sc, gx, gy, gz, envelope, aabb, pairs, pairs_cap, norm, cpta, cptb, depth, bids,
		                      n_pairs, n_contacts, s);
	CC_TRY(collide_enqueue(c, sc, gx, gy, gz, envelope, aabb, pairs, pairs_cap, norm, cpta, cptb, depth, bids, s,
	                       true));
	const uint64_t gen = c->buf_gen;
	CC_TRY(read_stats(c, s));
	const cc_status st = collide_finish(c, sc, envelope, aabb, pairs, pairs_cap, norm, cpta, cptb, depth, bids,
	                                    n_pairs, n_contacts, s);
	(void)gen;
	return st;
}

}  // namespace

extern "C" {

cc_status cc_ctx_create(cc_ctx **out, int device) {
	if (!out) return CC_ERR_INVALID_ARGUMENT;
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CC_ERR_CUDA;
	cc_ctx *c = new cc_ctx();
	c->device = device;
	c->gp.k_target = 4.0f;
	c->gp.min_ratio = 2.0f;
	c->gp.dense_cell = kDenseCell;
	c->gp.pair_window = 96;
	c->gp.pair_blocks_per_sm = 8;
	c->np_overlap = true;
	c->gp.user_dim[0] = c->gp.user_dim[1] = c->gp.user_dim[2] = 0;
	if (const char *v = getenv("CC_GRAPH_REPLAY")) c->graph_off = v[0] == '0';
	if (cudaSetDevice(device) != cudaSuccess || cudaMallocHost(&c->h_stats, sizeof(DevStats)) != cudaSuccess ||
	    cudaMallocHost(&c->h_word, 64) != cudaSuccess) {
		delete c;
		return CC_ERR_CUDA;
	}
	*out = c;
	return CC_OK;
}

void cc_ctx_destroy(cc_ctx *c) {
	if (!c) return;
	cudaSetDevice(c->device);
	Buf *bufs[] = {&c->stats,    &c->cell_count, &c->cell_start, &c->entries,  &c->owner_count, &c->owner_off,
	               &c->pairs_tmp, &c->status,    &c->ticket,     &c->big_list, &c->dense,       &c->ref_cnt,
	               &c->ref_off,
	               &c->ref_keys, &c->ref_tmp,    &c->ref_flags,  &c->ref_runpos, &c->rx_hist,   &c->rx_hoff,
	               &c->np_norm,  &c->np_pa,      &c->np_pb,      &c->np_depth, &c->np_ids,      &c->np_pairs,
	               &c->np_flag,  &c->np_pos,     &c->np_order, &c->np_classes, &c->in_T,       &c->in_A,     &c->in_B,        &c->in_C,
	               &c->in_R,     &c->in_ID,      &c->in_pos,     &c->in_rot,   &c->in_act,      &c->out_aabb,
	               &c->out_pairs, &c->out_norm,  &c->out_pa,     &c->out_pb,   &c->out_depth,   &c->out_bids,
	               &c->b_off,    &c->b_scene_of, &c->b_gid,      &c->b_sst,    &c->b_plans,     &c->b_G,
	               &c->b_base,   &c->b_status,   &c->b_ticket,   &c->b_res,    &c->g_T,         &c->g_A,
	               &c->g_B,      &c->g_C,        &c->g_R,        &c->g_ID,     &c->g_pos,       &c->g_rot,
	               &c->g_act,    &c->g_src,      &c->g_off,      &c->v_ref,    &c->v_backup,   &c->v_scratch, &c->v_cand,   &c->v_status,
	               &c->np_bsum,  &c->pt_desc,    &c->np_hkeys,   &c->np_hvals,   &c->bp_bsum,    &c->cell_cs};
	for (Buf *b : bufs)
		if (b->p) cudaFree(b->p);
	c->g_collide.drop();
	c->g_batch.drop();
	if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
	if (c->np_stream) cudaStreamDestroy(c->np_stream);
	if (c->ev_fork) cudaEventDestroy(c->ev_fork);
	if (c->ev_join) cudaEventDestroy(c->ev_join);
	for (auto &h : c->hs) {
		Buf *hb[] = {&h.T, &h.A, &h.B, &h.C, &h.R, &h.ID, &h.pos, &h.rot, &h.act, &h.aabb, &h.pairs, &h.norm, &h.pa,
		             &h.pb, &h.depth, &h.bids};
		for (Buf *b : hb)
			if (b->p) cudaFree(b->p);
		if (h.in_done) cudaEventDestroy(h.in_done);
		if (h.done) cudaEventDestroy(h.done);
		if (h.h_stats) cudaFreeHost(h.h_stats);
	}
	for (cudaStream_t t : {c->hs_copy, c->hs_comp, c->hs_out})
		if (t) cudaStreamDestroy(t);
	if (c->hs_user) cudaEventDestroy(c->hs_user);
	if (c->hs_back) cudaEventDestroy(c->hs_back);
	if (c->h_stats) cudaFreeHost(c->h_stats);
	if (c->h_word) cudaFreeHost(c->h_word);
	for (int i = 0; i < 2 * kMaxMarks; i++)
		if (c->ev[i]) cudaEventDestroy(c->ev[i]);
	delete c;
}

const char *cc_status_string(cc_status s) {
	switch (s) {
	case CC_OK: return "ok";
	case CC_ERR_INVALID_ARGUMENT: return "invalid argument";
	case CC_ERR_INVALID_INPUT: return "invalid input (non-finite or inverted AABB)";
	case CC_ERR_CAPACITY: return "output capacity too small";
	case CC_ERR_CUDA: return "CUDA error";
	case CC_ERR_OUT_OF_MEMORY: return "out of device memory";
	case CC_ERR_INTERNAL: return "internal error (device wait limit)";
	case CC_ERR_NO_RESULT: return "no retained result";
	}
	return "unknown status";
}

const char *cc_last_error(const cc_ctx *c) { return c ? c->err.c_str() : ""; }
const char *cc_version(void) { return "collide_b200 0.1 (sm_100a)"; }

cc_status cc_set_search_grid(cc_ctx *c, int gx, int gy, int gz) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (gx < 0 || gy < 0 || gz < 0 || gx > kMaxDim || gy > kMaxDim || gz > kMaxDim)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "search grid dims must be in [0, %d]", kMaxDim);
	const bool pin = gx > 0 && gy > 0 && gz > 0;
	c->gp.user_dim[0] = pin ? gx : 0;
	c->gp.user_dim[1] = pin ? gy : 0;
	c->gp.user_dim[2] = pin ? gz : 0;
	return CC_OK;
}

int cc_last_step_rebuilt(const cc_ctx *c) { return c ? c->last_rebuilt : -1; }

cc_status cc_set_incremental(cc_ctx *c, int on, float margin) {
	if (!c || !(margin > 0.f)) return CC_ERR_INVALID_ARGUMENT;
	c->incremental = on != 0;
	c->inc_margin = margin;
	c->inc_valid = false;
	return CC_OK;
}

cc_status cc_set_narrowphase_overlap(cc_ctx *c, int on) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	c->np_overlap = on != 0;
	return CC_OK;
}

cc_status cc_set_pair_test_shape(cc_ctx *c, int window, int blocks_per_sm) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (window != 64 && window != 96 && window != 128)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "pair-test window must be 64, 96 or 128");
	if (blocks_per_sm < 1 || blocks_per_sm > 16)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "pair-test blocks per SM must be 1..16");
	c->gp.pair_window = window;
	c->gp.pair_blocks_per_sm = blocks_per_sm;
	return CC_OK;
}

cc_status cc_set_dense_cell(cc_ctx *c, uint32_t entries) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	c->gp.dense_cell = entries ? std::max<uint32_t>(entries, kDenseCell) : 0xffffffffu;
	c->last_dense = 1;  // the next call launches the dense-cell kernel and counts again
	return CC_OK;
}

cc_status cc_set_tuning(cc_ctx *c, float cell_target, float min_ratio) {
	if (!c || !(cell_target > 0.f) || !(min_ratio >= 0.f)) return CC_ERR_INVALID_ARGUMENT;
	c->gp.k_target = cell_target;
	c->gp.min_ratio = min_ratio;
	return CC_OK;
}

cc_status cc_set_narrowphase_precision(cc_ctx *c, int mode) {
	if (!c || (mode != CC_NP_EXACT && mode != CC_NP_FP64 && mode != CC_NP_MIXED)) return CC_ERR_INVALID_ARGUMENT;
	c->np_precision = mode;
	return CC_OK;
}

cc_status cc_set_static_shapes(cc_ctx *c, int on) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	c->static_shapes = on != 0;
	c->shapes_gen++;  // every call drops the kept copies
	return CC_OK;
}

cc_status cc_get_last_grid(const cc_ctx *c, int *dims3, uint64_t *entries) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (dims3)
		for (int d = 0; d < 3; d++) dims3[d] = c->last_dim[d];
	if (entries) *entries = c->last_E;
	return CC_OK;
}

uint64_t cc_last_launch_count(const cc_ctx *c) { return c ? c->launches : 0; }

cc_status cc_set_graph_replay(cc_ctx *c, int on) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	c->graph_off = !on;
	c->g_collide.have_pending = c->g_batch.have_pending = false;
	if (!on) {
		c->g_collide.drop();
		c->g_batch.drop();
		}
	return CC_OK;
}

cc_status cc_set_profiling(cc_ctx *c, int on) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (on && !c->ev[0]) {
		CC_CUDA(c, cudaSetDevice(c->device));
		for (int i = 0; i < 2 * kMaxMarks; i++) CC_CUDA(c, cudaEventCreate(&c->ev[i]));
	}
	if (on < 0 || on > kProfSpans) return set_err(c, CC_ERR_INVALID_ARGUMENT, "profiling mode %d (0, 1 or 2)", on);
	c->prof = on;
	return CC_OK;
}

int cc_stage_count(void) { return ST_COUNT_; }

const char *cc_stage_name(int st) { return (st >= 0 && st < ST_COUNT_) ? kStageNames[st] : ""; }

cc_status cc_stage_times(const cc_ctx *c, double *ms, uint64_t *launches, int cap) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	for (int i = 0; i < cap && i < ST_COUNT_; i++) {
		if (ms) ms[i] = c->stage_ms[i];
		if (launches) launches[i] = c->stage_n[i];
	}
	return CC_OK;
}

cc_status cc_reset_stage_times(cc_ctx *c) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	for (int i = 0; i < ST_COUNT_; i++) {
		c->stage_ms[i] = 0.0;
		c->stage_n[i] = 0;
	}
	return CC_OK;
}

cc_status cc_generate_aabb(cc_ctx *c, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                           const float *R, const uint32_t *ID, uint64_t nb, const float *pos, const float *rot,
                           float *aabb, void *stream) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	CC_TRY(check_scene(c, n, T, A, B, C, R, ID, nb, pos, rot));
	if (n && !aabb) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null aabb");
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	if (n == 0) return CC_OK;
	CC_TRY(ensure(c, c->stats, sizeof(DevStats)));
	uint32_t *err = &ptr<DevStats>(c->stats)->err;
	{
		StageMark m(c, ST_AABB, s);
		CC_CUDA(c, cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
		launch_aabb(n, T, A, B, C, R, ID, nb, pos, rot, aabb, nullptr, err, c->gp, nullptr, s);
	}
	c->launches += 1;
	CC_TRY(check_launch(c));
	CC_CUDA(c, cudaMemcpyAsync(c->h_word, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
	CC_CUDA(c, cudaStreamSynchronize(s));
	if ((uint32_t)c->h_word[0] & kErrBadIndex) return set_err(c, CC_ERR_INVALID_INPUT, "a body id is >= nb");
	return CC_OK;
}

cc_status cc_broadphase(cc_ctx *c, uint64_t n, float *aabb, int gx, int gy, int gz, int64_t *pairs,
                        uint64_t pairs_cap, uint64_t *n_pairs, void *stream) {
	if (!c || !n_pairs) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	*n_pairs = 0;
	c->retained = false;
	CC_TRY(check_grid(c, gx, gy, gz));
	if (n == 0) return CC_OK;
	if (!aabb) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null aabb");
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	CC_TRY(prepare(c, n, 0));
	PdlScope pdl_(n);
	const int grid[3] = {gx, gy, gz};
	{
		StageMark m(c, ST_BOUNDS, s);
		CC_CUDA(c, cudaMemsetAsync(c->stats.p, 0, sizeof(DevStats), s));
		launch_bounds(n, aabb, ptr<DevStats>(c->stats), c->gp, grid, s);
	}
	c->launches += 1;
	enqueue_search(c, n, aabb, s);
	unsigned long long *out = reinterpret_cast<unsigned long long *>(pairs);
	const uint64_t cap = pairs ? pairs_cap : 0;
	if (cap) enqueue_emit(c, n, out, cap, s);
	CC_TRY(check_launch(c));
	CC_TRY(read_stats(c, s));
	CC_TRY(device_err(c));
	CC_TRY(settle(c, n, aabb, cap ? out : nullptr, cap, nullptr, s));
	remember(c);
	const uint64_t P = c->h_stats->pairs;
	*n_pairs = P;
	if (P > cap) {
		retain(c, n, P);
		return set_err(c, CC_ERR_CAPACITY, "pair list needs %llu entries, capacity %llu", (unsigned long long)P,
		               (unsigned long long)cap);
	}
	if (c->h_stats->err & kErrSegmentTooLong) CC_TRY(sort_fallback(c, n, P, out, s));
	return CC_OK;
}

cc_status cc_broadphase_fetch(cc_ctx *c, int64_t *pairs, uint64_t pairs_cap, void *stream) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	if (!c->retained) return set_err(c, CC_ERR_NO_RESULT, "no retained pair list");
	if (c->retained_P > pairs_cap || (!pairs && c->retained_P))
		return set_err(c, CC_ERR_CAPACITY, "pair list needs %llu entries", (unsigned long long)c->retained_P);
	CC_CUDA(c, cudaSetDevice(c->device));
	if (c->retained_P == 0) {
		c->retained = false;
		return CC_OK;
	}
	return emit_retained(c, reinterpret_cast<unsigned long long *>(pairs), pairs_cap, (cudaStream_t)stream);
}

cc_status cc_broadphase_bins(cc_ctx *c, uint64_t n, float *aabb, int gx, int gy, int gz, uint32_t *bin_number,
                             uint32_t *body_number, uint64_t entries_cap, uint64_t *n_entries, uint32_t *active_bins,
                             uint32_t *bin_end, uint64_t active_cap, uint64_t *n_active, void *stream) {
	if (!c || !n_entries || !n_active) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	*n_entries = 0;
	*n_active = 0;
	c->retained = false;
	CC_TRY(check_grid(c, gx, gy, gz));
	if (n == 0) return CC_OK;
	if (!aabb) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null aabb");
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	CC_TRY(prepare(c, n, 0));
	StageMark bins_mark(c, ST_BINS, s);
	BpBuffers b = bp_buffers(c);
	const int grid[3] = {gx, gy, gz};
	CC_CUDA(c, cudaMemsetAsync(c->stats.p, 0, sizeof(DevStats), s));
	launch_bounds(n, aabb, b.stats, c->gp, grid, s);  // + plan
	CC_CUDA(c, cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * c->gp.g_max, s));
	launch_count(n, aabb, b, s);  // in-place shift
	// per-body bin counts -> offsets
	CC_TRY(ensure(c, c->ref_cnt, sizeof(uint32_t) * n));
	CC_TRY(ensure(c, c->ref_off, sizeof(unsigned long long) * (n + 1)));
	launch_ref_count(n, aabb, b.stats, ptr<uint32_t>(c->ref_cnt), s);
	launch_scan_u32_to_u64(ptr<uint32_t>(c->ref_cnt), n, ptr<unsigned long long>(c->ref_off), b.status, b.ticket,
	                       &b.stats->err, s);
	c->launches += 5;
	CC_TRY(check_launch(c));
	CC_CUDA(c, cudaMemcpyAsync(c->h_word, ptr<unsigned long long>(c->ref_off) + n, 8, cudaMemcpyDeviceToHost, s));
	CC_TRY(read_stats(c, s));
	CC_TRY(device_err(c));
	const uint64_t E = c->h_word[0];
	*n_entries = E;
	// emit (bin << 32 | body) body-major, stable sort on the bin half
	CC_TRY(ensure(c, c->ref_keys, sizeof(unsigned long long) * std::max<uint64_t>(E, 1)));
	CC_TRY(ensure(c, c->ref_tmp, sizeof(unsigned long long) * std::max<uint64_t>(E, 1)));
	launch_ref_emit(n, aabb, b.stats, ptr<unsigned long long>(c->ref_off), ptr<unsigned long long>(c->ref_keys), E, s);
	c->launches += 1;
	CC_TRY(read_stats(c, s));
	if (c->h_stats->err & kErrBinCount) return set_err(c, CC_ERR_INTERNAL, "bin count/emit mismatch");
	int bits = 0;
	while (bits < 32 && ((uint64_t)c->h_stats->max_bin >> bits) != 0) bits++;
	unsigned long long *keys = ptr<unsigned long long>(c->ref_keys);
	// size all remaining scratch first: nothing may be reallocated while
	// kernels that use it are in flight
	const size_t hw = radix_hist_words(E);
	CC_TRY(ensure(c, c->rx_hist, sizeof(uint32_t) * hw));
	CC_TRY(ensure(c, c->rx_hoff, sizeof(unsigned long long) * (hw + 1)));
	CC_TRY(ensure(c, c->status, sizeof(uint64_t) * status_words_for(std::max<uint64_t>(hw, E) + 1)));
	CC_TRY(ensure(c, c->ref_flags, sizeof(uint32_t) * std::max<uint64_t>(E, 1)));
	CC_TRY(ensure(c, c->ref_runpos, sizeof(uint32_t) * (E + 1)));
	b = bp_buffers(c);
	if (E > 1 && bits > 0) {
		radix_sort_u64(keys, ptr<unsigned long long>(c->ref_tmp), E, 32, 32 + bits, ptr<uint32_t>(c->rx_hist),
		               ptr<unsigned long long>(c->rx_hoff), b.status, b.ticket, &b.stats->err, s);
		c->launches += 3 * ((bits + 7) / 8);
	}
	// runs of equal bins
	launch_ref_flags(keys, E, ptr<uint32_t>(c->ref_flags), s);
	launch_scan_u32_to_u32(ptr<uint32_t>(c->ref_flags), E, ptr<uint32_t>(c->ref_runpos), b.status, b.ticket,
	                       &b.stats->err, s);
	c->launches += 2;
	CC_TRY(check_launch(c));
	CC_CUDA(c, cudaMemcpyAsync(c->h_word, ptr<uint32_t>(c->ref_runpos) + E, 4, cudaMemcpyDeviceToHost, s));
	CC_CUDA(c, cudaStreamSynchronize(s));
	const uint64_t A = (uint32_t)c->h_word[0];
	*n_active = A;
	if ((bin_number || body_number) && E > entries_cap)
		return set_err(c, CC_ERR_CAPACITY, "bin list needs %llu entries", (unsigned long long)E);
	if ((active_bins || bin_end) && A > active_cap)
		return set_err(c, CC_ERR_CAPACITY, "active-bin list needs %llu entries", (unsigned long long)A);
	launch_ref_split(keys, E, ptr<uint32_t>(c->ref_runpos), bin_number, body_number, active_bins, bin_end, A, s);
	c->launches += 1;
	CC_TRY(check_launch(c));
	CC_CUDA(c, cudaStreamSynchronize(s));
	return CC_OK;
}

cc_status cc_narrowphase(cc_ctx *c, uint64_t n, const int32_t *T, const float *A, const float *B, const float *C,
                         const float *R, const uint32_t *ID, uint64_t nb, const uint8_t *active, const float *pos,
                         const float *rot, float envelope, int64_t *pairs, uint64_t n_pairs, float *norm, float *cpta,
                         float *cptb, float *depth, int32_t *bids, uint64_t *n_contacts, void *stream) {
	if (!c || !n_contacts) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	*n_contacts = 0;
	CC_TRY(check_scene(c, n, T, A, B, C, R, ID, nb, pos, rot));
	if (n_pairs && (!pairs || !norm || !cpta || !cptb || !depth || !bids || !active))
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "null pair/contact/active array");
	CC_CUDA(c, cudaSetDevice(c->device));
	if (n_pairs == 0) return CC_OK;
	cudaStream_t s = (cudaStream_t)stream;
	CC_TRY(np_prepare(c, n_pairs));
	CC_CUDA(c, cudaMemsetAsync(c->stats.p, 0, sizeof(DevStats), s));
	const NpArgs a = {n, nb, T, A, B, C, R, ID, active, pos, rot, envelope, pairs, norm, cpta, cptb, depth, bids};
	enqueue_np(c, a, n_pairs, nullptr, s);
	CC_TRY(check_launch(c));
	CC_TRY(read_stats(c, s));
	if (c->h_stats->err & kErrBadIndex)
		return set_err(c, CC_ERR_INVALID_INPUT, "a pair index is >= n or a body id is >= nb");
	if (c->h_stats->err & kErrSpinLimit) return set_err(c, CC_ERR_INTERNAL, "device-side look-back wait gave up");
	*n_contacts = c->h_stats->contacts;
	return CC_OK;
}

}  // extern "C"

namespace {
cc_status batch_impl(cc_ctx *c, const cc_batch *bt, int gx, int gy, int gz, float envelope, cc_result *res,
                     uint64_t *scene_pairs, uint64_t *contact_offsets, void *stream) {
	res->n_pairs = res->n_contacts = 0;
	c->retained = false;
	const uint64_t S = bt->num_scenes;
	if (S == 0) return CC_OK;
	if (S >= 0xffffffffull || !bt->shape_offsets || !bt->body_offsets)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "num_scenes out of range or null offsets");
	const cc_scene &sc = bt->scene;
	if (bt->shape_offsets[0] != 0 || bt->body_offsets[0] != 0 || bt->shape_offsets[S] != sc.n ||
	    bt->body_offsets[S] != sc.nb)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "offsets must start at 0 and end at scene.n / scene.nb");
	uint64_t g_total = 0;
	for (uint64_t s = 0; s < S; s++) {
		if (bt->shape_offsets[s + 1] < bt->shape_offsets[s] || bt->body_offsets[s + 1] < bt->body_offsets[s])
			return set_err(c, CC_ERR_INVALID_ARGUMENT, "offsets decrease at scene %llu", (unsigned long long)s);
		g_total += batch_scene_cells(bt->shape_offsets[s + 1] - bt->shape_offsets[s]);
	}
	if (g_total >= ((uint64_t)1 << 31))
		return set_err(c, CC_ERR_CAPACITY, "batch needs %llu grid cells (>= 2^31)", (unsigned long long)g_total);
	CC_TRY(check_grid(c, gx, gy, gz));
	CC_TRY(check_scene(c, sc.n, sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.nb, sc.body_pos, sc.body_rot));
	const uint64_t n = sc.n;
	if (n == 0) return CC_OK;
	if (!res->aabb || !sc.active) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null aabb or active array");
	PdlScope pdl_(n);
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	const uint64_t pairs_cap = res->pairs_cap;
	CC_TRY(prepare(c, n, pairs_cap, std::max<uint64_t>(g_total, 1)));
	CC_TRY(ensure(c, c->b_off, sizeof(unsigned long long) * 2 * (S + 1)));
	CC_TRY(ensure(c, c->b_scene_of, sizeof(uint32_t) * n));
	CC_TRY(ensure(c, c->b_gid, sizeof(uint32_t) * n));
	CC_TRY(ensure(c, c->b_sst, sizeof(SceneStats) * S));
	CC_TRY(ensure(c, c->b_plans, sizeof(Plan) * S));
	CC_TRY(ensure(c, c->b_G, sizeof(uint32_t) * (S + 1)));
	CC_TRY(ensure(c, c->b_base, sizeof(uint32_t) * (S + 2)));
	CC_TRY(ensure(c, c->b_status, sizeof(uint64_t) * status_words_for(S + 1)));
	CC_TRY(ensure(c, c->b_ticket, 64));
	CC_TRY(ensure(c, c->b_res, sizeof(unsigned long long) * (2 * S + 2)));
	unsigned long long *d_shape = ptr<unsigned long long>(c->b_off), *d_body = d_shape + (S + 1);
	CC_CUDA(c, copy_small_h2d(d_shape, bt->shape_offsets, sizeof(uint64_t) * (S + 1), s));
	CC_CUDA(c, copy_small_h2d(d_body, bt->body_offsets, sizeof(uint64_t) * (S + 1), s));
	DevStats *d = ptr<DevStats>(c->stats);
	const int grid[3] = {gx, gy, gz};
	uint32_t *scene_of = ptr<uint32_t>(c->b_scene_of), *gid = ptr<uint32_t>(c->b_gid);
	SceneStats *sst = ptr<SceneStats>(c->b_sst);
	Plan *plans = ptr<Plan>(c->b_plans);
	uint32_t *G = ptr<uint32_t>(c->b_G), *base = ptr<uint32_t>(c->b_base);
	unsigned long long *d_pairs_s = ptr<unsigned long long>(c->b_res), *d_coff = d_pairs_s + S;
	unsigned long long *out = reinterpret_cast<unsigned long long *>(res->pairs);
	// the rest of the pipeline sees one scene of n shapes with global body ids
	struct SmGuard {
		cc_ctx *c;
		~SmGuard() {
			c->sm = SceneMap();
			c->pass_zeroed = false;
		}
	} smg_{c};
	const NpArgs a = {n, sc.nb, sc.T, sc.A, sc.B, sc.C, sc.R, gid, sc.active, sc.body_pos, sc.body_rot, envelope,
	                  res->pairs, res->norm, res->cpta, res->cptb, res->depth, res->bids};
	ZeroList zero;
	zero.p[0] = ptr<uint32_t>(c->status);
	zero.words[0] = 2 * (c->st_words[0] + c->st_words[1] + c->st_words[2]);
	zero.p[1] = ptr<uint32_t>(c->ticket);
	zero.words[1] = 16;
	zero.p[2] = ptr<uint32_t>(c->np_classes);
	zero.words[2] = 2 * kNpClasses + 1;
	zero.p[3] = ptr<uint32_t>(c->cell_count);
	zero.words[3] = c->gp.g_max;
	for (int r = 0; r < 4; r++)
		if (!zero.p[r]) zero.words[r] = 0;
	// the rest of the pipeline takes each shape's plan from the scene map
	c->sm.scene_of = scene_of;
	c->sm.plans = plans;
	c->sm.cell_base = base;
	const bool want_offsets = scene_pairs || contact_offsets;
	auto enqueue_all = [&](cudaStream_t st) -> cc_status {
		{
			StageMark m(c, ST_AABB, st);
			CC_CUDA(c, cudaMemsetAsync(d, 0, sizeof(DevStats), st));
			CC_CUDA(c, cudaMemsetAsync(sst, 0, sizeof(SceneStats) * S, st));
			launch_batch_prep(n, (uint32_t)S, d_shape, d_body, sc.ID, scene_of, gid, &d->err, st);
			launch_aabb(n, sc.T, sc.A, sc.B, sc.C, sc.R, gid, sc.nb, sc.body_pos, sc.body_rot, res->aabb, nullptr,
			            &d->err, c->gp, grid, st, zero);
		}
		{
			StageMark m(c, ST_BOUNDS, st);
			launch_batch_bounds(n, res->aabb, scene_of, sst, &d->err, st);
			launch_batch_plan((uint32_t)S, d_shape, sst, c->gp, grid, plans, G, st);
			launch_scan_u32_to_u32(G, S, base, ptr<uint64_t>(c->b_status), ptr<uint32_t>(c->b_ticket), &d->err, st,
			                       nullptr, &d->cells);
		}
		c->launches += 6;
		c->pass_zeroed = true;
		enqueue_search(c, n, res->aabb, st);
		enqueue_emit(c, n, out, pairs_cap, st);
		enqueue_np(c, a, pairs_cap, &d->np_n, st);
		c->pass_zeroed = false;
		// per-scene pair counts and contact offsets, read back behind the pass
		if (want_offsets) {
			launch_batch_offsets((uint32_t)S, d_shape, ptr<unsigned long long>(c->owner_off),
			                     ptr<unsigned long long>(c->np_pos), d, d_pairs_s, d_coff, st);
			c->launches += 1;
		}
		return CC_OK;
	};
	// everything the pass's launches depend on (the offsets' contents are
	// copied in before every pass, outside the graph)
	struct {
		uint64_t n, nb, S, pairs_cap, hE, hP, gen, st[3];
		const void *p[16];
		int dims[3], prec, want;
		float env;
		GridParams gp;
	} k;
	memset(&k, 0, sizeof(k));
	k.n = n; k.nb = sc.nb; k.S = S; k.pairs_cap = pairs_cap; k.hE = hint_E(c, n); k.hP = hint_P(c);
	k.gen = c->buf_gen;
	for (int r = 0; r < 3; r++) k.st[r] = c->st_words[r];
	const void *ps[16] = {sc.T, sc.A, sc.B, sc.C, sc.R, sc.ID, sc.active, sc.body_pos, sc.body_rot, res->aabb,
	                      res->pairs, res->norm, res->cpta, res->cptb, res->depth, res->bids};
	memcpy(k.p, ps, sizeof(ps));
	k.dims[0] = gx; k.dims[1] = gy; k.dims[2] = gz; k.prec = c->np_precision; k.want = want_offsets ? 1 : 0;
	k.env = envelope; k.gp = c->gp;
	CC_TRY(run_graphed(c, c->g_batch, &k, sizeof(k), enqueue_all, s));
	auto copy_back = [&]() -> cc_status {
		if (scene_pairs)
			CC_CUDA(c, cudaMemcpyAsync(scene_pairs, d_pairs_s, sizeof(uint64_t) * S, cudaMemcpyDeviceToHost, s));
		if (contact_offsets)
			CC_CUDA(c, cudaMemcpyAsync(contact_offsets, d_coff, sizeof(uint64_t) * (S + 1), cudaMemcpyDeviceToHost, s));
		return CC_OK;
	};
	auto copy_offsets = [&]() -> cc_status {
		launch_batch_offsets((uint32_t)S, d_shape, ptr<unsigned long long>(c->owner_off),
		                     ptr<unsigned long long>(c->np_pos), d, d_pairs_s, d_coff, s);
		CC_TRY(check_launch(c));
		return copy_back();
	};
	if (want_offsets) CC_TRY(copy_back());
	CC_TRY(check_launch(c));
	CC_TRY(read_stats(c, s));
	CC_TRY(device_err(c));
	bool redone = c->h_stats->entries > c->entries.bytes / (2 * sizeof(float4)) ||
	              c->h_stats->pairs > c->pairs_tmp.bytes / sizeof(unsigned long long);
	CC_TRY(settle(c, n, res->aabb, out, pairs_cap, &a, s));
	remember(c);
	const uint64_t P = c->h_stats->pairs;
	res->n_pairs = P;
	if (P > pairs_cap)
		return set_err(c, CC_ERR_CAPACITY, "pair list needs %llu entries, capacity %llu", (unsigned long long)P,
		               (unsigned long long)pairs_cap);
	if (c->h_stats->err & kErrSegmentTooLong) {
		CC_TRY(sort_fallback(c, n, P, out, s));
		CC_CUDA(c, cudaMemsetAsync(&d->contacts, 0, sizeof(unsigned long long), s));
		enqueue_np(c, a, pairs_cap, &d->np_n, s);
		CC_TRY(check_launch(c));
		CC_TRY(read_stats(c, s));
		redone = true;
	}
	if (c->h_stats->err & kErrBadIndex)
		return set_err(c, CC_ERR_INVALID_INPUT, "a pair index is >= n or a body id is outside its scene");
	res->n_contacts = c->h_stats->contacts;
	if (want_offsets && redone) {
		CC_TRY(copy_offsets());
		CC_CUDA(c, cudaStreamSynchronize(s));
	}
	return CC_OK;
}
}  // namespace

extern "C" {

cc_status cc_collide_batch(cc_ctx *c, const cc_batch *bt, int gx, int gy, int gz, float envelope, cc_result *res,
                           uint64_t *scene_pairs, uint64_t *contact_offsets, void *stream) {
	if (!c || !bt || !res) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	return batch_impl(c, bt, gx, gy, gz, envelope, res, scene_pairs, contact_offsets, stream);
}

cc_status cc_collide_scenes(cc_ctx *c, uint64_t num_scenes, const cc_scene *scenes, int gx, int gy, int gz,
                            float envelope, cc_result *res, uint64_t *scene_pairs, uint64_t *contact_offsets,
                            void *stream) {
	if (!c || !res || (num_scenes && !scenes)) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	res->n_pairs = res->n_contacts = 0;
	if (num_scenes == 0) return CC_OK;
	if (num_scenes >= 0xffffffffull) return set_err(c, CC_ERR_INVALID_ARGUMENT, "too many scenes");
	std::vector<uint64_t> so(num_scenes + 1, 0), bo(num_scenes + 1, 0);
	std::vector<SceneSrc> src(num_scenes);
	for (uint64_t s = 0; s < num_scenes; s++) {
		const cc_scene &x = scenes[s];
		CC_TRY(check_scene(c, x.n, x.T, x.A, x.B, x.C, x.R, x.ID, x.nb, x.body_pos, x.body_rot));
		if ((x.n || x.nb) && (!x.active || !x.body_pos || !x.body_rot))
			return set_err(c, CC_ERR_INVALID_ARGUMENT, "scene %llu: null body arrays", (unsigned long long)s);
		so[s + 1] = so[s] + x.n;
		bo[s + 1] = bo[s] + x.nb;
		src[s] = SceneSrc{x.T, x.A, x.B, x.C, x.R, x.ID, x.body_pos, x.body_rot, x.active};
	}
	const uint64_t n = so[num_scenes], nb = bo[num_scenes];
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	CC_TRY(ensure(c, c->g_T, 4 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_A, 12 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_B, 12 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_C, 12 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_R, 16 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_ID, 4 * std::max<uint64_t>(n, 1)));
	CC_TRY(ensure(c, c->g_pos, 12 * std::max<uint64_t>(nb, 1)));
	CC_TRY(ensure(c, c->g_rot, 16 * std::max<uint64_t>(nb, 1)));
	CC_TRY(ensure(c, c->g_act, std::max<uint64_t>(nb, 1)));
	CC_TRY(ensure(c, c->g_src, sizeof(SceneSrc) * num_scenes));
	CC_TRY(ensure(c, c->g_off, sizeof(unsigned long long) * 2 * (num_scenes + 1)));
	unsigned long long *d_so = ptr<unsigned long long>(c->g_off), *d_bo = d_so + (num_scenes + 1);
	CC_CUDA(c, copy_small_h2d(c->g_src.p, src.data(), sizeof(SceneSrc) * num_scenes, s));
	CC_CUDA(c, copy_small_h2d(d_so, so.data(), sizeof(uint64_t) * (num_scenes + 1), s));
	CC_CUDA(c, copy_small_h2d(d_bo, bo.data(), sizeof(uint64_t) * (num_scenes + 1), s));
	SceneDst dst{ptr<int32_t>(c->g_T), ptr<float>(c->g_A), ptr<float>(c->g_B), ptr<float>(c->g_C), ptr<float>(c->g_R),
	             ptr<uint32_t>(c->g_ID), ptr<float>(c->g_pos), ptr<float>(c->g_rot), ptr<uint8_t>(c->g_act)};
	{
		StageMark m(c, ST_COPY_IN, s);
		launch_gather(n, nb, (uint32_t)num_scenes, d_so, d_bo, ptr<SceneSrc>(c->g_src), dst, s);
	}
	c->launches += 2;
	cc_batch bt;
	bt.num_scenes = num_scenes;
	bt.shape_offsets = so.data();
	bt.body_offsets = bo.data();
	bt.scene = cc_scene{n, dst.T, dst.A, dst.B, dst.C, dst.R, dst.ID, nb, dst.pos, dst.rot, dst.active};
	return batch_impl(c, &bt, gx, gy, gz, envelope, res, scene_pairs, contact_offsets, stream);
}

cc_status cc_perturb_bodies(cc_ctx *c, uint64_t nb, float *body_pos, float *body_rot, uint64_t seed, float sigma,
                            float max_angle, void *stream) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (nb == 0) return CC_OK;
	if (!body_pos || !body_rot) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null body arrays");
	if (!aligned16(body_rot)) return set_err(c, CC_ERR_INVALID_ARGUMENT, "body_rot must be 16-byte aligned");
	CC_CUDA(c, cudaSetDevice(c->device));
	launch_perturb(nb, body_pos, body_rot, seed, sigma, max_angle, (cudaStream_t)stream);
	return check_launch(c);
}

cc_status cc_perturb_scenes(cc_ctx *c, uint64_t count, const uint64_t *nb, float *const *body_pos,
                            float *const *body_rot, const uint64_t *seeds, float sigma, float max_angle, void *stream) {
	if (!c) return CC_ERR_INVALID_ARGUMENT;
	if (count == 0) return CC_OK;
	if (!nb || !body_pos || !body_rot || !seeds) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null argument array");
	if (count >= 0xffffffffull) return set_err(c, CC_ERR_INVALID_ARGUMENT, "too many scenes");
	std::vector<PerturbScene> d;
	d.reserve(count);
	uint64_t total = 0;
	for (uint64_t k = 0; k < count; k++) {
		if (nb[k] == 0) continue;
		if (!body_pos[k] || !body_rot[k])
			return set_err(c, CC_ERR_INVALID_ARGUMENT, "scene %llu: null body arrays", (unsigned long long)k);
		if (!aligned16(body_rot[k]))
			return set_err(c, CC_ERR_INVALID_ARGUMENT, "scene %llu: body_rot must be 16-byte aligned",
			               (unsigned long long)k);
		d.push_back(PerturbScene{body_pos[k], body_rot[k], nb[k], total, seeds[k]});
		total += nb[k];
	}
	if (d.empty()) return CC_OK;
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	CC_TRY(ensure(c, c->pt_desc, sizeof(PerturbScene) * d.size()));
	// the descriptor table travels in kernel parameters (or a staged copy when
	// large): the host vector may go away once the call returns
	CC_CUDA(c, copy_small_h2d(c->pt_desc.p, d.data(), sizeof(PerturbScene) * d.size(), s));
	launch_perturb_scenes((uint32_t)d.size(), total, ptr<PerturbScene>(c->pt_desc), sigma, max_angle, s);
	return check_launch(c);
}

cc_status cc_collide(cc_ctx *c, const cc_scene *sc, int gx, int gy, int gz, float envelope, cc_result *res,
                     void *stream) {
	if (!c || !sc || !res) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	CC_TRY(check_grid(c, gx, gy, gz));
	CC_TRY(check_scene(c, sc->n, sc->T, sc->A, sc->B, sc->C, sc->R, sc->ID, sc->nb, sc->body_pos, sc->body_rot));
	if (sc->n && (!res->aabb || !sc->active))
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "null aabb or active array");
	CC_CUDA(c, cudaSetDevice(c->device));
	return collide_dev(c, *sc, gx, gy, gz, envelope, res->aabb, res->pairs, res->pairs_cap, res->norm, res->cpta,
	                   res->cptb, res->depth, res->bids, &res->n_pairs, &res->n_contacts, (cudaStream_t)stream);
}

}  // extern "C"

namespace {
// Turns stage profiling off for the scope of a call.
struct NoProfile {
	cc_ctx *c;
	int was;
	explicit NoProfile(cc_ctx *c_) : c(c_), was(c_->prof) { c->prof = 0; }
	~NoProfile() { c->prof = was; }
};

// Copies a finished step's outputs (P pairs, nc contacts) from its slot to the
// caller's host buffers and waits for them.
cc_status host_copy_out(cc_ctx *c, cc_ctx::HostSlot &h, cc_result *res, uint64_t P, uint64_t nc, cudaStream_t s) {
	StageMark m(c, ST_COPY_OUT, s);
	const uint64_t n = h.dev.n;
	if (res->aabb) CC_CUDA(c, cudaMemcpyAsync(res->aabb, h.aabb.p, 24 * n, cudaMemcpyDeviceToHost, s));
	if (res->pairs && P) CC_CUDA(c, cudaMemcpyAsync(res->pairs, h.pairs.p, 8 * P, cudaMemcpyDeviceToHost, s));
	if (nc) {
		if (res->norm) CC_CUDA(c, cudaMemcpyAsync(res->norm, h.norm.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->cpta) CC_CUDA(c, cudaMemcpyAsync(res->cpta, h.pa.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->cptb) CC_CUDA(c, cudaMemcpyAsync(res->cptb, h.pb.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->depth) CC_CUDA(c, cudaMemcpyAsync(res->depth, h.depth.p, 4 * nc, cudaMemcpyDeviceToHost, s));
		if (res->bids) CC_CUDA(c, cudaMemcpyAsync(res->bids, h.bids.p, 8 * nc, cudaMemcpyDeviceToHost, s));
	}
	CC_CUDA(c, cudaStreamSynchronize(s));
	return CC_OK;
}

// The six shape arrays of a host step (T, A, B, C, R, ID) into dst, unless
// static shapes are on and dst already holds these host arrays' contents.
// The device address of a pinned, mapped host array; null for pageable memory.
const void *mapped_host(const void *p) {
	static const bool off = [] {
		const char *v = getenv("CC_GATHER_C");
		return v && v[0] == '0';
	}();
	if (off) return nullptr;
	cudaPointerAttributes a;
	if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return nullptr;
	}
	return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// The six shape arrays to the device. C is read only for CONE and
// TRIANGLEMESH shapes, so from a pinned host array it is not copied whole:
// *gather_c receives its device mapping and the caller gathers those shapes'
// C with launch_gather_c once T is on the device, on its compute stream (a
// kernel on the copy stream would hold the later copies until the SMs are free).
cc_status upload_shapes(cc_ctx *c, cc_ctx::ShapeCopy &sh, Buf *const dst[6], const cc_scene *sc, cudaStream_t t,
                        const float **gather_c) {
	*gather_c = nullptr;
	const void *src[6] = {sc->T, sc->A, sc->B, sc->C, sc->R, sc->ID};
	static const uint64_t bytes[6] = {4, 12, 12, 12, 16, 4};
	bool same = c->static_shapes && sh.gen == c->shapes_gen && sh.n == sc->n;
	for (int k = 0; k < 6; k++)
		same = same && sh.src[k] == src[k] && sh.dst[k] == dst[k]->p && sh.allocs[k] == dst[k]->allocs;
	if (same) return CC_OK;
	sh.gen = 0;  // not valid until every copy is enqueued
	const float *c_mapped = sc->n ? static_cast<const float *>(mapped_host(sc->C)) : nullptr;
	for (int k = 0; k < 6; k++) {
		if (k == 3 && c_mapped)
			*gather_c = c_mapped;
		else
			CC_CUDA(c, cudaMemcpyAsync(dst[k]->p, src[k], bytes[k] * sc->n, cudaMemcpyHostToDevice, t));
		sh.src[k] = src[k];
		sh.dst[k] = dst[k]->p;
		sh.allocs[k] = dst[k]->allocs;
	}
	sh.n = sc->n;
	sh.gen = c->shapes_gen;
	return CC_OK;
}

// Sizes one slot for a scene of n shapes / nb bodies and cap pairs and points
// its device view at it.
cc_status host_slot_prepare(cc_ctx *c, cc_ctx::HostSlot &h, uint64_t n, uint64_t nb, uint64_t cap) {
	const uint64_t k = std::max<uint64_t>(cap, 1);
	CC_TRY(ensure(c, h.T, 4 * n));
	CC_TRY(ensure(c, h.A, 12 * n));
	CC_TRY(ensure(c, h.B, 12 * n));
	CC_TRY(ensure(c, h.C, 12 * n));
	CC_TRY(ensure(c, h.R, 16 * n));
	CC_TRY(ensure(c, h.ID, 4 * n));
	CC_TRY(ensure(c, h.pos, 12 * nb));
	CC_TRY(ensure(c, h.rot, 16 * nb));
	CC_TRY(ensure(c, h.act, nb));
	CC_TRY(ensure(c, h.aabb, 24 * n));
	CC_TRY(ensure(c, h.pairs, 8 * k));
	CC_TRY(ensure(c, h.norm, 12 * k));
	CC_TRY(ensure(c, h.pa, 12 * k));
	CC_TRY(ensure(c, h.pb, 12 * k));
	CC_TRY(ensure(c, h.depth, 4 * k));
	CC_TRY(ensure(c, h.bids, 8 * k));
	h.dev = cc_scene{n, ptr<int32_t>(h.T), ptr<float>(h.A), ptr<float>(h.B), ptr<float>(h.C), ptr<float>(h.R),
	                 ptr<uint32_t>(h.ID), nb, ptr<float>(h.pos), ptr<float>(h.rot), ptr<uint8_t>(h.act)};
	return CC_OK;
}
}  // namespace

extern "C" {

cc_status cc_collide_host_submit(cc_ctx *c, const cc_scene *sc, int gx, int gy, int gz, float envelope,
                                 cc_result *res, void *stream) {
	if (!c || !sc || !res) return CC_ERR_INVALID_ARGUMENT;
	NoProfile np_(c);  // stage events would span three streams: not recorded here
	c->launches = 0;
	if (c->hs_inflight == 2)
		return set_err(c, CC_ERR_INVALID_ARGUMENT, "two steps in flight: call cc_collide_host_wait first");
	CC_TRY(check_grid(c, gx, gy, gz));
	CC_TRY(check_scene(c, sc->n, sc->T, sc->A, sc->B, sc->C, sc->R, sc->ID, sc->nb, sc->body_pos, sc->body_rot));
	if (sc->n && !sc->active) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null active array");
	CC_CUDA(c, cudaSetDevice(c->device));
	if (!c->hs_copy) {
		CC_CUDA(c, cudaStreamCreateWithFlags(&c->hs_copy, cudaStreamNonBlocking));
		CC_CUDA(c, cudaStreamCreateWithFlags(&c->hs_comp, cudaStreamNonBlocking));
		CC_CUDA(c, cudaStreamCreateWithFlags(&c->hs_out, cudaStreamNonBlocking));
		CC_CUDA(c, cudaEventCreateWithFlags(&c->hs_user, cudaEventDisableTiming));
		CC_CUDA(c, cudaEventCreateWithFlags(&c->hs_back, cudaEventDisableTiming));
		for (auto &h : c->hs) {
			CC_CUDA(c, cudaEventCreateWithFlags(&h.in_done, cudaEventDisableTiming));
			CC_CUDA(c, cudaEventCreateWithFlags(&h.done, cudaEventDisableTiming));
			CC_CUDA(c, cudaMallocHost(&h.h_stats, sizeof(DevStats)));
		}
	}
	cc_ctx::HostSlot &h = c->hs[c->hs_next];
	const uint64_t n = sc->n, nb = sc->nb, cap = res->pairs_cap;
	// growing a buffer frees the old one: never while another step may use it
	if (c->hs_inflight) {
		c->dry_run = true;
		c->would_grow = false;
		const cc_status d1 = host_slot_prepare(c, h, n, nb, cap);
		const cc_status d2 = n ? prepare(c, n, cap) : CC_OK;
		c->dry_run = false;
		if (d1 != CC_OK || d2 != CC_OK || c->would_grow) CC_CUDA(c, cudaStreamSynchronize(c->hs_comp));
	}
	CC_TRY(host_slot_prepare(c, h, n, nb, cap));
	if (n) CC_TRY(prepare(c, n, cap));
	// after the caller's prior work on `stream`
	const float *gather_c = nullptr;
	CC_CUDA(c, cudaEventRecord(c->hs_user, (cudaStream_t)stream));
	CC_CUDA(c, cudaStreamWaitEvent(c->hs_copy, c->hs_user, 0));
	{
		StageMark m(c, ST_COPY_IN, c->hs_copy);
		cudaStream_t t = c->hs_copy;
		Buf *const dst[6] = {&h.T, &h.A, &h.B, &h.C, &h.R, &h.ID};
		CC_TRY(upload_shapes(c, c->hs_shapes[c->hs_next], dst, sc, t, &gather_c));
		CC_CUDA(c, cudaMemcpyAsync(h.pos.p, sc->body_pos, 12 * nb, cudaMemcpyHostToDevice, t));
		CC_CUDA(c, cudaMemcpyAsync(h.rot.p, sc->body_rot, 16 * nb, cudaMemcpyHostToDevice, t));
		CC_CUDA(c, cudaMemcpyAsync(h.act.p, sc->active, nb, cudaMemcpyHostToDevice, t));
		if (res->aabb) CC_CUDA(c, cudaMemcpyAsync(h.aabb.p, res->aabb, 24 * n, cudaMemcpyHostToDevice, t));
		CC_CUDA(c, cudaEventRecord(h.in_done, t));
	}
	CC_CUDA(c, cudaStreamWaitEvent(c->hs_comp, h.in_done, 0));
	if (gather_c) {
		launch_gather_c(n, ptr<int32_t>(h.T), gather_c, ptr<float>(h.C), c->hs_comp);
		c->launches += 1;
	}
	if (n) {
		CC_TRY(collide_enqueue(c, h.dev, gx, gy, gz, envelope, ptr<float>(h.aabb), ptr<int64_t>(h.pairs), cap,
		                       ptr<float>(h.norm), ptr<float>(h.pa), ptr<float>(h.pb), ptr<float>(h.depth),
		                       ptr<int32_t>(h.bids), c->hs_comp, false));
		CC_CUDA(c, cudaMemcpyAsync(h.h_stats, c->stats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, c->hs_comp));
		const BpBuffers b = bp_buffers(c);
		h.entry_cap = b.entry_cap;
		h.pair_cap = b.pair_cap;
	} else {
		memset(h.h_stats, 0, sizeof(DevStats));
	}
	CC_CUDA(c, cudaEventRecord(h.done, c->hs_comp));
	h.res = res;
	h.grid[0] = gx;
	h.grid[1] = gy;
	h.grid[2] = gz;
	h.env = envelope;
	h.cap = cap;
	c->hs_next ^= 1;
	c->hs_inflight++;
	return CC_OK;
}

cc_status cc_collide_host_wait(cc_ctx *c, cc_result *res, void *stream) {
	if (!c || !res) return CC_ERR_INVALID_ARGUMENT;
	NoProfile np_(c);
	if (c->hs_inflight == 0) return set_err(c, CC_ERR_NO_RESULT, "no step in flight");
	cc_ctx::HostSlot &h = c->hs[c->hs_oldest];
	// a mismatched wait leaves the oldest step in flight for the right one
	if (res != h.res) return set_err(c, CC_ERR_INVALID_ARGUMENT, "wait with a different result than the oldest submit");
	c->hs_oldest ^= 1;
	c->hs_inflight--;
	CC_CUDA(c, cudaSetDevice(c->device));
	CC_CUDA(c, cudaEventSynchronize(h.done));
	res->n_pairs = res->n_contacts = 0;
	if (h.dev.n == 0) return CC_OK;
	const DevStats &st = *h.h_stats;
	const bool fast = st.err == 0 && st.entries <= h.entry_cap && st.pairs <= h.pair_cap && st.pairs <= h.cap &&
	                  st.np_n == st.pairs;
	uint64_t P = st.pairs, nc = st.contacts;
	if (fast) {
		memcpy(c->h_stats, h.h_stats, sizeof(DevStats));
		remember(c);
	} else {
		// rare: an error, a scratch overflow or a full output. Let the steps in
		// flight finish, then run this one again on the blocking path, which
		// regrows scratch, reports the error or retains the result.
		CC_CUDA(c, cudaStreamSynchronize(c->hs_comp));
		// the first run shifted the boxes in place; GenerateAABB keeps the
		// caller's boxes of RECT/TRIANGLEMESH shapes, so start from them again
		if (res->aabb)
			CC_CUDA(c, cudaMemcpy(h.aabb.p, res->aabb, 24 * h.dev.n, cudaMemcpyHostToDevice));
		const cc_status r = collide_dev(c, h.dev, h.grid[0], h.grid[1], h.grid[2], h.env, ptr<float>(h.aabb),
		                                ptr<int64_t>(h.pairs), h.cap, ptr<float>(h.norm), ptr<float>(h.pa),
		                                ptr<float>(h.pb), ptr<float>(h.depth), ptr<int32_t>(h.bids), &P, &nc,
		                                c->hs_comp);
		res->n_pairs = P;
		res->n_contacts = nc;
		if (r != CC_OK) return r;
	}
	res->n_pairs = P;
	res->n_contacts = nc;
	CC_TRY(host_copy_out(c, h, res, P, nc, c->hs_out));
	// the caller's stream sees the step as done
	CC_CUDA(c, cudaEventRecord(c->hs_back, c->hs_out));
	CC_CUDA(c, cudaStreamWaitEvent((cudaStream_t)stream, c->hs_back, 0));
	return CC_OK;
}

cc_status cc_collide_host(cc_ctx *c, const cc_scene *sc, int gx, int gy, int gz, float envelope, cc_result *res,
                          void *stream) {
	if (!c || !sc || !res) return CC_ERR_INVALID_ARGUMENT;
	ProfGuard pg_(c, stream);
	c->launches = 0;
	CC_TRY(check_grid(c, gx, gy, gz));
	CC_TRY(check_scene(c, sc->n, sc->T, sc->A, sc->B, sc->C, sc->R, sc->ID, sc->nb, sc->body_pos, sc->body_rot));
	if (sc->n && !sc->active) return set_err(c, CC_ERR_INVALID_ARGUMENT, "null active array");
	CC_CUDA(c, cudaSetDevice(c->device));
	cudaStream_t s = (cudaStream_t)stream;
	const uint64_t n = sc->n, nb = sc->nb;
	res->n_pairs = res->n_contacts = 0;
	if (n == 0) return CC_OK;
	CC_TRY(ensure(c, c->in_T, 4 * n));
	CC_TRY(ensure(c, c->in_A, 12 * n));
	CC_TRY(ensure(c, c->in_B, 12 * n));
	CC_TRY(ensure(c, c->in_C, 12 * n));
	CC_TRY(ensure(c, c->in_R, 16 * n));
	CC_TRY(ensure(c, c->in_ID, 4 * n));
	CC_TRY(ensure(c, c->in_pos, 12 * nb));
	CC_TRY(ensure(c, c->in_rot, 16 * nb));
	CC_TRY(ensure(c, c->in_act, nb));
	CC_TRY(ensure(c, c->out_aabb, 24 * n));
	const uint64_t cap = res->pairs_cap;
	CC_TRY(ensure(c, c->out_pairs, 8 * std::max<uint64_t>(cap, 1)));
	CC_TRY(ensure(c, c->out_norm, 12 * std::max<uint64_t>(cap, 1)));
	CC_TRY(ensure(c, c->out_pa, 12 * std::max<uint64_t>(cap, 1)));
	CC_TRY(ensure(c, c->out_pb, 12 * std::max<uint64_t>(cap, 1)));
	CC_TRY(ensure(c, c->out_depth, 4 * std::max<uint64_t>(cap, 1)));
	CC_TRY(ensure(c, c->out_bids, 8 * std::max<uint64_t>(cap, 1)));
	std::unique_ptr<StageMark> cin(new StageMark(c, ST_COPY_IN, s));
	{
		Buf *const dst[6] = {&c->in_T, &c->in_A, &c->in_B, &c->in_C, &c->in_R, &c->in_ID};
		const float *gather_c = nullptr;
		CC_TRY(upload_shapes(c, c->in_shapes, dst, sc, s, &gather_c));
		if (gather_c) {
			launch_gather_c(n, ptr<int32_t>(c->in_T), gather_c, ptr<float>(c->in_C), s);
			c->launches += 1;
		}
	}
	CC_CUDA(c, cudaMemcpyAsync(c->in_pos.p, sc->body_pos, 12 * nb, cudaMemcpyHostToDevice, s));
	CC_CUDA(c, cudaMemcpyAsync(c->in_rot.p, sc->body_rot, 16 * nb, cudaMemcpyHostToDevice, s));
	CC_CUDA(c, cudaMemcpyAsync(c->in_act.p, sc->active, nb, cudaMemcpyHostToDevice, s));
	if (res->aabb) CC_CUDA(c, cudaMemcpyAsync(c->out_aabb.p, res->aabb, 24 * n, cudaMemcpyHostToDevice, s));
	cin.reset();
	cc_scene d;
	d.n = n;
	d.nb = nb;
	d.T = ptr<int32_t>(c->in_T);
	d.A = ptr<float>(c->in_A);
	d.B = ptr<float>(c->in_B);
	d.C = ptr<float>(c->in_C);
	d.R = ptr<float>(c->in_R);
	d.ID = ptr<uint32_t>(c->in_ID);
	d.body_pos = ptr<float>(c->in_pos);
	d.body_rot = ptr<float>(c->in_rot);
	d.active = ptr<uint8_t>(c->in_act);
	uint64_t P = 0, nc = 0;
	cc_status st = collide_dev(c, d, gx, gy, gz, envelope, ptr<float>(c->out_aabb), ptr<int64_t>(c->out_pairs), cap,
	                           ptr<float>(c->out_norm), ptr<float>(c->out_pa), ptr<float>(c->out_pb),
	                           ptr<float>(c->out_depth), ptr<int32_t>(c->out_bids), &P, &nc, s);
	res->n_pairs = P;
	res->n_contacts = nc;
	if (st != CC_OK) return st;
	StageMark cout_mark(c, ST_COPY_OUT, s);
	if (res->aabb) CC_CUDA(c, cudaMemcpyAsync(res->aabb, c->out_aabb.p, 24 * n, cudaMemcpyDeviceToHost, s));
	if (res->pairs && P) CC_CUDA(c, cudaMemcpyAsync(res->pairs, c->out_pairs.p, 8 * P, cudaMemcpyDeviceToHost, s));
	if (nc) {
		if (res->norm) CC_CUDA(c, cudaMemcpyAsync(res->norm, c->out_norm.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->cpta) CC_CUDA(c, cudaMemcpyAsync(res->cpta, c->out_pa.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->cptb) CC_CUDA(c, cudaMemcpyAsync(res->cptb, c->out_pb.p, 12 * nc, cudaMemcpyDeviceToHost, s));
		if (res->depth) CC_CUDA(c, cudaMemcpyAsync(res->depth, c->out_depth.p, 4 * nc, cudaMemcpyDeviceToHost, s));
		if (res->bids) CC_CUDA(c, cudaMemcpyAsync(res->bids, c->out_bids.p, 8 * nc, cudaMemcpyDeviceToHost, s));
	}
	CC_CUDA(c, cudaStreamSynchronize(s));
	return CC_OK;
}

}  // extern "C"
