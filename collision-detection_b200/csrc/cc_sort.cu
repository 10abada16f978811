// Single-pass exclusive scan (decoupled look-back) and a stable LSD radix sort
// of 64-bit keys. Integer-only; used by the broadphase (cell offsets, pair
// owner offsets, the reference-grid bin list) and the narrowphase compaction.
#include "cc_common.cuh"
#include "cc_internal.h"

namespace cc {

namespace {
constexpr int kScanNT = 256, kScanIPT = 16;
constexpr uint64_t kScanTile = (uint64_t)kScanNT * kScanIPT;

template <class OutT>
__global__ void __launch_bounds__(kScanNT) k_scan(const uint32_t *__restrict__ in, uint64_t n_host,
                                                  const unsigned long long *__restrict__ n_dev,
                                                  OutT *__restrict__ out,
                                                  unsigned long long *total_out, uint64_t *status, uint32_t *ticket,
                                                  uint32_t *err, uint32_t *zero_in) {
	pdl_begin();
	__shared__ uint32_t s_tile;
	__shared__ unsigned long long s_pre;
	__shared__ unsigned long long sm[40];
	if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
	__syncthreads();
	const uint32_t tile = s_tile;
	// the element count may live on the device (<= n_host); tiles past it have
	// no successor that waits on them and leave at once
	const uint64_t n = n_dev ? min(n_host, (uint64_t)*n_dev) : n_host;
	if ((uint64_t)tile > n / kScanTile) return;
	const uint64_t i0 = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanIPT;
	uint32_t v[kScanIPT];
	if (i0 + kScanIPT <= n && ((reinterpret_cast<uintptr_t>(in) & 15) == 0)) {
		const uint4 *p = reinterpret_cast<const uint4 *>(in + i0);
#pragma unroll
		for (int q = 0; q < kScanIPT / 4; q++) {
			uint4 t = __ldcs(p + q);
			v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
		}
		if (zero_in && (reinterpret_cast<uintptr_t>(zero_in) & 15) == 0) {
			uint4 *z = reinterpret_cast<uint4 *>(zero_in + i0);
#pragma unroll
			for (int q = 0; q < kScanIPT / 4; q++) z[q] = make_uint4(0u, 0u, 0u, 0u);
		} else if (zero_in) {
#pragma unroll
			for (int j = 0; j < kScanIPT; j++) zero_in[i0 + j] = 0u;
		}
	} else {
#pragma unroll
		for (int j = 0; j < kScanIPT; j++) v[j] = (i0 + j < n) ? in[i0 + j] : 0u;
		if (zero_in)
			for (int j = 0; j < kScanIPT; j++)
				if (i0 + j < n) zero_in[i0 + j] = 0u;
	}
	unsigned long long sum = 0;
#pragma unroll
	for (int j = 0; j < kScanIPT; j++) sum += v[j];
	unsigned long long total;
	unsigned long long excl = block_excl_scan<unsigned long long, kScanNT>(sum, sm, &total);
	if (threadIdx.x < 32) {
		unsigned long long p = lookback_prefix(status, tile, total, err);
		if (threadIdx.x == 0) s_pre = p;
	}
	__syncthreads();
	unsigned long long run = s_pre + excl;
#pragma unroll
	for (int j = 0; j < kScanIPT; j++) {
		if (i0 + j < n) out[i0 + j] = (OutT)run;
		run += v[j];
	}
	if (i0 <= n && n < i0 + kScanIPT) {
		out[n] = (OutT)run;
		if (total_out) *total_out = run;
	}
}

template <class OutT>
void scan_impl(const uint32_t *in, uint64_t n, OutT *out, uint64_t *status, uint32_t *ticket, uint32_t *err,
               cudaStream_t s, const unsigned long long *n_dev, unsigned long long *total_out, bool pre_zeroed,
               uint32_t *zero_in) {
	const uint64_t tiles = n / kScanTile + 1;
	if (!pre_zeroed) {
		cudaMemsetAsync(status, 0, tiles * sizeof(uint64_t), s);
		cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s);
	}
	launch_pdl(k_scan<OutT>, dim3((unsigned)tiles), dim3(kScanNT), 0, s, in, n, n_dev, out, total_out, status, ticket, err, zero_in);
}
}  // namespace

size_t scan_tiles(uint64_t n) { return (size_t)(n / kScanTile + 1); }

void launch_scan_u32_to_u64(const uint32_t *in, uint64_t n, unsigned long long *out, uint64_t *status,
                            uint32_t *ticket, uint32_t *err, cudaStream_t s, const unsigned long long *n_dev,
                            unsigned long long *total_out, bool pre_zeroed) {
	scan_impl(in, n, out, status, ticket, err, s, n_dev, total_out, pre_zeroed, (uint32_t *)nullptr);
}
void launch_scan_u32_to_u32(const uint32_t *in, uint64_t n, uint32_t *out, uint64_t *status, uint32_t *ticket,
                            uint32_t *err, cudaStream_t s, const unsigned long long *n_dev,
                            unsigned long long *total_out, bool pre_zeroed, uint32_t *zero_in) {
	scan_impl(in, n, out, status, ticket, err, s, n_dev, total_out, pre_zeroed, zero_in);
}

// --------------------------------------------------------------------------
// Radix sort. Tile = 8 warps x 8 items x 32 lanes = 2048 keys, striped inside
// each warp (item j of lane l is key w*256 + j*32 + l), so processing j in
// order and lanes in order visits keys in their original order: ranking with
// __match_any_sync is therefore stable.
// --------------------------------------------------------------------------
namespace {
constexpr int kRxNT = 256, kRxIPT = 8, kRxWarps = kRxNT / 32;
constexpr uint64_t kRxTile = (uint64_t)kRxNT * kRxIPT;

__global__ void __launch_bounds__(kRxNT) k_radix_hist(const unsigned long long *__restrict__ keys, uint64_t n,
                                                      int shift, uint32_t ntiles, uint32_t *__restrict__ hist) {
	__shared__ uint32_t h[256];
	h[threadIdx.x] = 0;
	__syncthreads();
	const uint64_t base = (uint64_t)blockIdx.x * kRxTile;
	for (int j = 0; j < kRxIPT; j++) {
		uint64_t i = base + (uint64_t)j * kRxNT + threadIdx.x;
		if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1u);
	}
	__syncthreads();
	hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kRxNT) k_radix_scatter(const unsigned long long *__restrict__ keys, uint64_t n,
                                                         int shift, uint32_t ntiles,
                                                         const unsigned long long *__restrict__ hoff,
                                                         unsigned long long *__restrict__ out) {
	__shared__ uint32_t cnt[kRxWarps][256];
	__shared__ uint32_t woff[kRxWarps][256];
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	for (int d = l; d < 256; d += 32) cnt[w][d] = 0;
	__syncwarp();
	const uint64_t wbase = (uint64_t)blockIdx.x * kRxTile + (uint64_t)w * (kRxIPT * 32);
	unsigned long long k[kRxIPT];
	uint32_t rank[kRxIPT];
	const uint32_t lt = (1u << l) - 1u;
#pragma unroll
	for (int j = 0; j < kRxIPT; j++) {
		uint64_t i = wbase + (uint64_t)j * 32 + l;
		bool valid = i < n;
		k[j] = valid ? keys[i] : 0ull;
		uint32_t d = valid ? (uint32_t)((k[j] >> shift) & 255) : 256u;
		uint32_t peers = __match_any_sync(0xffffffffu, d);
		uint32_t r = __popc(peers & lt);
		uint32_t b = valid ? cnt[w][d] : 0u;
		__syncwarp();
		if (valid && r == 0) cnt[w][d] = b + __popc(peers);
		__syncwarp();
		rank[j] = b + r;
	}
	__syncthreads();
	{
		const int d = threadIdx.x;  // one digit per thread
		uint32_t acc = 0;
#pragma unroll
		for (int ww = 0; ww < kRxWarps; ww++) {
			woff[ww][d] = acc;
			acc += cnt[ww][d];
		}
	}
	__syncthreads();
#pragma unroll
	for (int j = 0; j < kRxIPT; j++) {
		uint64_t i = wbase + (uint64_t)j * 32 + l;
		if (i < n) {
			uint32_t d = (uint32_t)((k[j] >> shift) & 255);
			uint64_t pos = hoff[(uint64_t)d * ntiles + blockIdx.x] + woff[w][d] + rank[j];
			out[pos] = k[j];
		}
	}
}
}  // namespace

size_t radix_hist_words(uint64_t n) { return (size_t)256 * (size_t)((n + kRxTile - 1) / kRxTile + 1); }

void radix_sort_u64(unsigned long long *keys, unsigned long long *tmp, uint64_t n, int bit_lo, int bit_hi,
                    uint32_t *hist, unsigned long long *hoff, uint64_t *status, uint32_t *ticket, uint32_t *err,
                    cudaStream_t s) {
	if (n <= 1 || bit_hi <= bit_lo) return;
	const uint32_t ntiles = (uint32_t)((n + kRxTile - 1) / kRxTile);
	unsigned long long *src = keys, *dst = tmp;
	for (int sh = bit_lo; sh < bit_hi; sh += 8) {
		k_radix_hist<<<ntiles, kRxNT, 0, s>>>(src, n, sh, ntiles, hist);
		scan_impl(hist, (uint64_t)256 * ntiles, hoff, status, ticket, err, s, (const unsigned long long *)nullptr,
		          (unsigned long long *)nullptr, false, (uint32_t *)nullptr);
		k_radix_scatter<<<ntiles, kRxNT, 0, s>>>(src, n, sh, ntiles, hoff, dst);
		unsigned long long *t = src; src = dst; dst = t;
	}
	if (src != keys) cudaMemcpyAsync(keys, src, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
}

}  // namespace cc
