// cc_broadphase_noalloc: the broadphase for callers that cannot allocate
// device memory.
//
// Some callers of a collision step cannot call cudaMalloc or cudaFree, or let
// a library do it for them: hard real-time simulation loops (cudaMalloc and
// cudaFree can synchronize the whole device and take unbounded time), and host
// frameworks that hand out every byte of device memory from their own pool and
// forbid side allocations. For them this entry point takes its scratch from
// one file-scope device array of fixed size (kScratchBytes, 16 MiB) that every
// GPU loading the library holds until the process exits, and it calls no
// allocating routine: no cudaMalloc/cudaFree, no pinned host memory, no
// library that allocates. The caller passes the AABBs (shifted in place, as
// detectPossibleCollisions does) and the pair output buffer.
//
// Limits: n <= CC_NOALLOC_MAX_BODIES; the search-grid entries and the pair
// count must fit the scratch (CC_NOALLOC_MAX_ENTRIES, CC_NOALLOC_MAX_PAIRS);
// larger inputs are rejected with CC_ERR_CAPACITY (the limits are constants in
// include/collide_b200.h).
//
// Set-up: the first call on each device (with that device current) looks up
// the device address of the scratch array with cudaGetSymbolAddress. Each call
// waits for its stream twice, to read the entry and pair counts. Every call
// shares the one array (and one host-side staging block), which keeps the last
// call's contents: calls that overlap on the GPU, or come from two host
// threads at once, race. Each call zeroes what must start at zero, so stale
// contents from the previous call never leak into the result.
#include <mutex>

#include "../../include/collide_b200.h"
#include "cc_common.cuh"
#include "cc_internal.h"

namespace cc {
namespace {

constexpr uint64_t kMaxBodies = CC_NOALLOC_MAX_BODIES;
constexpr uint64_t kMaxEntries = CC_NOALLOC_MAX_ENTRIES;
constexpr uint64_t kMaxPairs = CC_NOALLOC_MAX_PAIRS;
constexpr uint32_t kGMax = (uint32_t)kMaxBodies;  // per-cell arrays (>= 4096)
constexpr uint64_t kBigCap = kMaxBodies + 1024;
constexpr size_t kScratchBytes = CC_NOALLOC_SCRATCH_BYTES;

// The scratch. In host code `g_scratch` is only a stand-in symbol, never a
// device address: kernels receive the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Carve-out of the scratch array (byte offsets).
struct Layout {
	size_t stats, cell_count, cell_start, owner_count, owner_off, entries, pairs_tmp, rx_tmp, rx_hist, rx_hoff,
	    status, ticket, big_list, end;
	size_t hist_words, status_words;
};

constexpr Layout make_layout() {
	Layout L{};
	size_t o = 0;
	L.stats = o; o += align256(sizeof(DevStats));
	L.cell_count = o; o += align256(sizeof(uint32_t) * kGMax);
	L.cell_start = o; o += align256(sizeof(uint32_t) * (kGMax + 1));
	L.owner_count = o; o += align256(sizeof(uint32_t) * kMaxBodies);
	L.owner_off = o; o += align256(sizeof(unsigned long long) * (kMaxBodies + 1));
	L.entries = o; o += align256(2 * sizeof(float4) * kMaxEntries);
	L.pairs_tmp = o; o += align256(sizeof(unsigned long long) * kMaxPairs);
	L.rx_tmp = o; o += align256(sizeof(unsigned long long) * kMaxPairs);
	// radix_hist_words(kMaxPairs): 256 digits x (tiles of 2048 keys + 1)
	L.hist_words = 256 * ((kMaxPairs + 2047) / 2048 + 1);
	L.rx_hist = o; o += align256(sizeof(uint32_t) * L.hist_words);
	L.rx_hoff = o; o += align256(sizeof(unsigned long long) * (L.hist_words + 1));
	// look-back tiles for the largest scan (4096 items per tile) + slack
	L.status_words = (L.hist_words > kMaxBodies + 1 ? L.hist_words : kMaxBodies + 1) / 4096 + 16;
	L.status = o; o += align256(sizeof(uint64_t) * L.status_words);
	L.ticket = o; o += 256;
	L.big_list = o; o += align256(sizeof(uint32_t) * kBigCap);
	L.end = o;
	return L;
}
constexpr Layout kL = make_layout();
static_assert(kL.end <= kScratchBytes, "scratch layout exceeds the static array");

std::mutex g_setup_mu;
void *g_dev_ptr[64] = {};          // scratch address per device (set up once)
DevStats g_host_stats;             // host staging of the device stats (pageable)
unsigned long long g_host_word[2];

// The status code is the whole error report (there is no context to hold a
// message); `msg` documents the cause at each call site.
cc_status fail(cc_status st, const char *msg) {
	(void)msg;
	return st;
}

// The first call on a device looks up the scratch address (device current).
cc_status scratch_for_current_device(unsigned char **out) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(CC_ERR_CUDA, "no current device");
	std::lock_guard<std::mutex> lk(g_setup_mu);
	if (!g_dev_ptr[dev]) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
		if (e != cudaSuccess || !p) return fail(CC_ERR_CUDA, cudaGetErrorString(e));
		g_dev_ptr[dev] = p;
	}
	*out = static_cast<unsigned char *>(g_dev_ptr[dev]);
	return CC_OK;
}

#define NA_CUDA(expr)                                                      \
	do {                                                                   \
		const cudaError_t e_ = (expr);                                     \
		if (e_ != cudaSuccess) return fail(CC_ERR_CUDA, cudaGetErrorString(e_)); \
	} while (0)

cc_status read_stats(const DevStats *dstats, cudaStream_t s) {
	NA_CUDA(cudaMemcpyAsync(&g_host_stats, dstats, sizeof(DevStats), cudaMemcpyDeviceToHost, s));
	NA_CUDA(cudaStreamSynchronize(s));
	return CC_OK;
}

}  // namespace
}  // namespace cc

using namespace cc;

extern "C" cc_status cc_broadphase_noalloc(uint64_t n, float *aabb, int gx, int gy, int gz, int64_t *pairs,
                                           uint64_t pairs_cap, uint64_t *n_pairs, void *stream) {
	if (!n_pairs) return fail(CC_ERR_INVALID_ARGUMENT, "n_pairs is NULL");
	*n_pairs = 0;
	if (gx < 0 || gy < 0 || gz < 0) return fail(CC_ERR_INVALID_ARGUMENT, "negative bins per axis");
	if (n == 0) return CC_OK;
	if (!aabb) return fail(CC_ERR_INVALID_ARGUMENT, "aabb is NULL");
	if (n > kMaxBodies) return fail(CC_ERR_CAPACITY, "more bodies than CC_NOALLOC_MAX_BODIES");
	unsigned char *base = nullptr;
	cc_status st = scratch_for_current_device(&base);
	if (st != CC_OK) return st;
	cudaStream_t s = (cudaStream_t)stream;

	BpBuffers b;
	b.stats = reinterpret_cast<DevStats *>(base + kL.stats);
	b.cell_count = reinterpret_cast<uint32_t *>(base + kL.cell_count);
	b.cell_start = reinterpret_cast<uint32_t *>(base + kL.cell_start);
	b.g_max = (uint32_t)(n > 4096 ? n : 4096);  // the same per-cell budget the context path uses
	b.entries = reinterpret_cast<float4 *>(base + kL.entries);
	b.entry_cap = kMaxEntries;
	b.owner_count = reinterpret_cast<uint32_t *>(base + kL.owner_count);
	b.owner_off = reinterpret_cast<unsigned long long *>(base + kL.owner_off);
	b.pairs_tmp = reinterpret_cast<unsigned long long *>(base + kL.pairs_tmp);
	b.pair_cap = kMaxPairs;
	b.status = reinterpret_cast<uint64_t *>(base + kL.status);
	b.ticket = reinterpret_cast<uint32_t *>(base + kL.ticket);
	b.big_list = reinterpret_cast<uint32_t *>(base + kL.big_list);
	b.big_cap = kBigCap;
	GridParams gp;
	gp.k_target = 4.0f;
	gp.min_ratio = 2.0f;
	gp.user_dim[0] = gp.user_dim[1] = gp.user_dim[2] = 0;
	gp.g_max = b.g_max;
	gp.dense_cell = kDenseCell;
	gp.pair_window = b.pair_window;
	gp.pair_blocks_per_sm = b.pair_blocks_per_sm;
	const int grid[3] = {gx, gy, gz};

	// everything that accumulates starts at zero (the array keeps the last call's contents)
	NA_CUDA(cudaMemsetAsync(b.stats, 0, sizeof(DevStats), s));
	NA_CUDA(cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * b.g_max, s));
	launch_bounds(n, aabb, b.stats, gp, grid, s);  // + the grid plan
	launch_count(n, aabb, b, s);
	launch_scan_cells(b, b.g_max, s);  // leaves the counts zeroed for the scatter
	launch_scatter(n, aabb, b, s);
	launch_pair_test(n, b, n, s);
	launch_scan_owner(n, b, s);
	NA_CUDA(cudaGetLastError());
	if ((st = read_stats(b.stats, s)) != CC_OK) return st;
	const uint32_t e = g_host_stats.err;
	if (e & (kErrNonFinite | kErrInverted)) return fail(CC_ERR_INVALID_INPUT, "non-finite or inverted AABB");
	if (e & kErrSpinLimit) return fail(CC_ERR_INTERNAL, "device-side look-back wait gave up");
	const uint64_t E = g_host_stats.entries, P = g_host_stats.pairs;
	if (E > kMaxEntries) return fail(CC_ERR_CAPACITY, "search-grid entries exceed CC_NOALLOC_MAX_ENTRIES");
	*n_pairs = P;
	if (P > kMaxPairs) return fail(CC_ERR_CAPACITY, "pair count exceeds CC_NOALLOC_MAX_PAIRS");
	if (P > pairs_cap || (!pairs && P)) return fail(CC_ERR_CAPACITY, "pairs_cap is smaller than the pair count");
	if (P == 0) return CC_OK;

	unsigned long long *out = reinterpret_cast<unsigned long long *>(pairs);
	launch_owner_scatter(pairs_cap, out, b, s);
	launch_segsort(n, out, b, s);
	launch_segsort_mid(out, b, s);
	launch_segsort_big(out, b, s);
	NA_CUDA(cudaGetLastError());
	if ((st = read_stats(b.stats, s)) != CC_OK) return st;
	if (g_host_stats.err & kErrSegmentTooLong) {
		int bits = 1;
		while (bits < 32 && ((uint64_t)1 << bits) < n) bits++;
		radix_sort_u64(out, reinterpret_cast<unsigned long long *>(base + kL.rx_tmp), P, 0, 32 + bits,
		               reinterpret_cast<uint32_t *>(base + kL.rx_hist),
		               reinterpret_cast<unsigned long long *>(base + kL.rx_hoff), b.status, b.ticket,
		               &b.stats->err, s);
	}
	NA_CUDA(cudaGetLastError());
	NA_CUDA(cudaMemcpyAsync(g_host_word, &b.stats->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
	NA_CUDA(cudaStreamSynchronize(s));
	if ((uint32_t)g_host_word[0] & kErrSpinLimit) return fail(CC_ERR_INTERNAL, "device-side look-back wait gave up");
	return CC_OK;
}
