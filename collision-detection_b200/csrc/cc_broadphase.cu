// Uniform-grid broadphase (the reference's Broadphase::detectPossibleCollisions,
// src/broadphase/Broadphase.cu:344-545) as sm_100a kernels.
//
// Pair path (always):
//   k_bounds        scene bounds + extent sums + validation     (Broadphase.cu:368-376)
//   k_count         in-place shift by fabs(min) (:379-386) + per-cell counts on
//                   the search grid
//   scan            cell offsets (decoupled look-back)
//   k_scatter       cell-ordered (AABB, body) entries
//   k_pair_test     closed AABB overlap (:237) of every entry with the later
//                   entries of its cell; a pair is emitted only from its home
//                   cell (the cell holding the larger of the two min corners on
//                   every axis, a point of both boxes and so of both cell
//                   ranges), so each overlapping pair appears exactly once and no
//                   unique pass is needed (replaces :484-533)
//   scan            per-owner offsets (owner = smaller index)
//   k_owner_scatter bucket pairs by owner; k_segsort sorts each bucket
//                   -> the sorted, duplicate-free int64 list of :522-535
//
// Two overlapping boxes always share a cell of ANY grid built from a monotone
// cell map (float subtraction, multiplication and truncation are monotone), and
// the reference re-tests every candidate on the shifted boxes, so its pair list
// is exactly {(a,b): a<b, closed overlap of the shifted boxes}: the search grid
// here is chosen for speed, independent of the caller's bins per axis.
//
// Bin-list path (on request): the reference's own sorted (bin, body) list on
// the caller's grid, with its HashMin truncation and unclamped linear index
// (:125-200, :428-480), for parity checks.
//
// Compiled with -fmad=false (the shift and the bin scale must round exactly as
// the reference's host build does).
#include <algorithm>
#include <climits>
#include <cstdlib>

#include "cc_common.cuh"
#include "cc_internal.h"
#include "cc_math.cuh"
#include "cc_stats.cuh"

namespace cc {

namespace {
constexpr int kNT = 256;

__device__ __forceinline__ float3 ld3p(const float *p, uint64_t i) { return f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// A block's kNT boxes, staged through shared memory with 16-byte loads: the
// min corners of boxes [i0, i0+kNT) are 3*kNT contiguous floats at aabb+3*i0
// and the max corners the same at aabb+3*(n+i0). stage[0..3kNT) = mins,
// stage[3kNT..6kNT) = maxs. Vector accesses are used when both runs are
// 16-byte aligned and complete; otherwise scalar ones.
__device__ __forceinline__ bool tile_vec_ok(const float *aabb, uint64_t n, uint64_t i0) {
	return i0 + kNT <= n && ((reinterpret_cast<uintptr_t>(aabb + 3 * i0) & 15) == 0) &&
	       ((reinterpret_cast<uintptr_t>(aabb + 3 * (n + i0)) & 15) == 0);
}
// The same for 32-byte vector accesses.
__device__ __forceinline__ bool tile_vec_ok32(const float *aabb, uint64_t n, uint64_t i0) {
	return i0 + kNT <= n && ((reinterpret_cast<uintptr_t>(aabb + 3 * i0) & 31) == 0) &&
	       ((reinterpret_cast<uintptr_t>(aabb + 3 * (n + i0)) & 31) == 0);
}
__device__ __forceinline__ void load_tile_aabb(const float *__restrict__ aabb, uint64_t n, uint64_t i0, float *stage) {
	if (tile_vec_ok(aabb, n, i0)) {
		const float4 *lo = reinterpret_cast<const float4 *>(aabb + 3 * i0);
		const float4 *hi = reinterpret_cast<const float4 *>(aabb + 3 * (n + i0));
		float4 *st = reinterpret_cast<float4 *>(stage);
		for (int k = threadIdx.x; k < 3 * kNT / 4; k += kNT) {
			st[k] = lo[k];
			st[3 * kNT / 4 + k] = hi[k];
		}
	} else {
		const uint64_t m = i0 < n ? min((uint64_t)kNT, n - i0) : 0;
		for (int k = threadIdx.x; k < 3 * (int)m; k += kNT) {
			stage[k] = aabb[3 * i0 + k];
			stage[3 * kNT + k] = aabb[3 * (n + i0) + k];
		}
	}
}
__device__ __forceinline__ void store_tile_aabb(float *__restrict__ aabb, uint64_t n, uint64_t i0, const float *stage) {
	if (tile_vec_ok(aabb, n, i0)) {
		float4 *lo = reinterpret_cast<float4 *>(aabb + 3 * i0);
		float4 *hi = reinterpret_cast<float4 *>(aabb + 3 * (n + i0));
		const float4 *st = reinterpret_cast<const float4 *>(stage);
		for (int k = threadIdx.x; k < 3 * kNT / 4; k += kNT) {
			lo[k] = st[k];
			hi[k] = st[3 * kNT / 4 + k];
		}
	} else {
		const uint64_t m = i0 < n ? min((uint64_t)kNT, n - i0) : 0;
		for (int k = threadIdx.x; k < 3 * (int)m; k += kNT) {
			aabb[3 * i0 + k] = stage[k];
			aabb[3 * (n + i0) + k] = stage[3 * kNT + k];
		}
	}
}

// Search-grid cell of a shifted coordinate: monotone in v.
__device__ __forceinline__ int cell_of(float v, float lo, float inv, int dim) {
	float t = (v - lo) * inv;
	int c = (int)fminf(fmaxf(t, 0.f), (float)(dim - 1));
	return c;
}
struct CellRange {
	int c0[3], c1[3];
};
__device__ __forceinline__ CellRange cell_range(const Plan &p, float3 mn, float3 mx) {
	CellRange r;
	r.c0[0] = cell_of(mn.x, p.lo[0], p.inv[0], p.dim[0]);
	r.c0[1] = cell_of(mn.y, p.lo[1], p.inv[1], p.dim[1]);
	r.c0[2] = cell_of(mn.z, p.lo[2], p.inv[2], p.dim[2]);
	r.c1[0] = cell_of(mx.x, p.lo[0], p.inv[0], p.dim[0]);
	r.c1[1] = cell_of(mx.y, p.lo[1], p.inv[1], p.dim[1]);
	r.c1[2] = cell_of(mx.z, p.lo[2], p.inv[2], p.dim[2]);
	return r;
}
__device__ __forceinline__ uint32_t pack_cell(int x, int y, int z) {
	return (uint32_t)x | ((uint32_t)y << 10) | ((uint32_t)z << 20);
}
// Home-cell test by per-entry codes. cell_of is monotone, so the cell of the
// larger min corner of two boxes is, per axis, the larger of the two min
// corners' cells; it equals the cell (cx, cy, cz) both entries were entered in
// exactly when one min corner's cell equals it and the other's does not
// exceed it. home_code: bits 0-2 = min-corner cell == the cell's coordinate
// on x/y/z, bits 3-5 = min-corner cell <= it; computed once per entry (the
// dense-cell kernel, where most tested boxes overlap).
__device__ __forceinline__ uint32_t home_code(const Plan &p, float4 lo, uint32_t packed_cell) {
	const int cx = packed_cell & 1023, cy = (packed_cell >> 10) & 1023, cz = (packed_cell >> 20) & 1023;
	const int x = cell_of(lo.x, p.lo[0], p.inv[0], p.dim[0]);
	const int y = cell_of(lo.y, p.lo[1], p.inv[1], p.dim[1]);
	const int z = cell_of(lo.z, p.lo[2], p.inv[2], p.dim[2]);
	return (uint32_t)(x == cx) | ((uint32_t)(y == cy) << 1) | ((uint32_t)(z == cz) << 2) | ((uint32_t)(x <= cx) << 3) |
	       ((uint32_t)(y <= cy) << 4) | ((uint32_t)(z <= cz) << 5);
}
// cell_of(max(a.min, b.min)) == cell on every axis
__device__ __forceinline__ bool home_pair(uint32_t a, uint32_t b) {
	return (((a & (b >> 3)) | (b & (a >> 3))) & 7u) == 7u;
}

__global__ void __launch_bounds__(kNT) k_bounds(uint64_t n, const float *__restrict__ aabb, DevStats *stats,
                                                 PlanArgs pa, ZeroList zero) {
	zero_ranges(zero);
	const uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	float3 mn = f3(0.f, 0.f, 0.f), mx = mn;
	const bool have = i < n;
	if (have) {
		mn = ld3p(aabb, i);
		mx = ld3p(aabb, i + n);
	}
	accumulate_stats_one<kNT>(mn, mx, have, stats, pa);
}

// The plan a shape is searched with: the block's staged plan (one scene) or
// its scene's plan (batch).
template <bool kBatch>
__device__ __forceinline__ const Plan &plan_of(const Plan &sp, const SceneMap &sm, uint64_t shape, uint32_t &base) {
	if constexpr (kBatch) {
		const uint32_t s = __ldg(sm.scene_of + shape);
		base = __ldg(sm.cell_base + s);
		return sm.plans[s];
	} else {
		base = 0;
		return sp;
	}
}
__device__ __forceinline__ uint32_t cell_index(const Plan &p, uint32_t base, int x, int y, int z) {
	return base + (uint32_t)x + (uint32_t)p.dim[0] * ((uint32_t)y + (uint32_t)p.dim[1] * z);
}

template <bool kBatch>
__global__ void __launch_bounds__(kNT) k_count(uint64_t n, float *__restrict__ aabb, const DevStats *stats,
                                                uint32_t *__restrict__ cell_count, uint32_t *__restrict__ owner_count,
                                                SceneMap sm, int oshift, uint32_t *__restrict__ owner_cursor) {
	pdl_begin();
	__shared__ Plan sp;
	__shared__ __align__(16) float stage[6 * kNT];  // read and written as float4
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	__syncthreads();
	if (!kBatch && !sp.valid) return;  // invalid input: nothing is modified
	const uint64_t i0 = (uint64_t)blockIdx.x * kNT;
	if (!kBatch && tile_vec_ok32(aabb, n, i0)) {
		// in-place shift by fabs(min) (:382-386) on 32-byte vectors, in
		// registers on the way to shared memory: thread k < 96 takes floats
		// [8k, 8k + 8) of the min-corner run, thread 96 + k those of the
		// max-corner run; float 8k + j is component (2k + j) mod 3
		const int t = threadIdx.x;
		if (t < 3 * kNT / 4) {
			const int k = t < 3 * kNT / 8 ? t : t - 3 * kNT / 8;
			float *run = t < 3 * kNT / 8 ? aabb + 3 * i0 : aabb + 3 * (n + i0);
			const int r = (2 * k) % 3;
			const float o0 = sp.origin[r], o1 = sp.origin[r == 2 ? 0 : r + 1], o2 = sp.origin[r == 0 ? 2 : r - 1];
			float4 a, b;
			ld_global_v8(run + 8 * k, a, b);
			a = make_float4(a.x + o0, a.y + o1, a.z + o2, a.w + o0);
			b = make_float4(b.x + o1, b.y + o2, b.z + o0, b.w + o1);
			st_global_v8(run + 8 * k, a, b);
			float4 *st = reinterpret_cast<float4 *>(stage) + (t < 3 * kNT / 8 ? 0 : 3 * kNT / 4);
			st[2 * k] = a;
			st[2 * k + 1] = b;
		}
		__syncthreads();
	} else {
		load_tile_aabb(aabb, n, i0, stage);
		__syncthreads();
		// in-place shift by fabs(min) (:382-386), element by element
		if constexpr (kBatch) {
			for (int k = threadIdx.x; k < 6 * kNT; k += kNT) {
				const uint64_t shape = i0 + (uint64_t)((k % (3 * kNT)) / 3);
				if (shape < n) {
					const Plan &p = sm.plans[__ldg(sm.scene_of + shape)];
					if (p.valid) stage[k] = stage[k] + p.origin[k % 3];
				}
			}
		} else {
			for (int k = threadIdx.x; k < 6 * kNT; k += kNT) stage[k] = stage[k] + sp.origin[k % 3];
		}
		__syncthreads();
		store_tile_aabb(aabb, n, i0, stage);
	}
	const uint64_t i = i0 + threadIdx.x;
	if (i >= n) return;
	const float3 mn = f3(stage[3 * threadIdx.x], stage[3 * threadIdx.x + 1], stage[3 * threadIdx.x + 2]);
	const float *hs = stage + 3 * kNT;
	const float3 mx = f3(hs[3 * threadIdx.x], hs[3 * threadIdx.x + 1], hs[3 * threadIdx.x + 2]);
	if ((i & ((1ull << oshift) - 1)) == 0) {  // the first body of its owner bucket
		owner_count[i >> oshift] = 0u;
		if (owner_cursor) owner_cursor[i >> oshift] = 0u;
	}
	uint32_t base;
	const Plan &p = plan_of<kBatch>(sp, sm, i, base);
	if (kBatch && !p.valid) return;
	const CellRange r = cell_range(p, mn, mx);
	for (int z = r.c0[2]; z <= r.c1[2]; z++)
		for (int y = r.c0[1]; y <= r.c1[1]; y++)
			for (int x = r.c0[0]; x <= r.c1[0]; x++) atomicAdd(&cell_count[cell_index(p, base, x, y, z)], 1u);
}

// Cell-ordered entries: one thread per body, a cursor atomic per covered cell.
template <bool kBatch>
__global__ void __launch_bounds__(kNT) k_scatter(uint64_t n, const float *__restrict__ aabb, const DevStats *stats,
                                                  const uint32_t *__restrict__ cell_start,
                                                  uint32_t *__restrict__ cursor, float4 *__restrict__ entries,
                                                  uint64_t cap, uint32_t *err, SceneMap sm,
                                                  unsigned long long *__restrict__ cs) {
	pdl_begin();
	__shared__ Plan sp;
	__shared__ __align__(16) float stage[6 * kNT];  // read and written as float4
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	const uint64_t i0 = (uint64_t)blockIdx.x * kNT;
	load_tile_aabb(aabb, n, i0, stage);
	__syncthreads();
	const uint64_t i = i0 + threadIdx.x;
	if ((!kBatch && !sp.valid) || i >= n) return;
	const float3 mn = f3(stage[3 * threadIdx.x], stage[3 * threadIdx.x + 1], stage[3 * threadIdx.x + 2]);
	const float *hs = stage + 3 * kNT;
	const float3 mx = f3(hs[3 * threadIdx.x], hs[3 * threadIdx.x + 1], hs[3 * threadIdx.x + 2]);
	uint32_t base;
	const Plan &p = plan_of<kBatch>(sp, sm, i, base);
	if (kBatch && !p.valid) return;
	const CellRange r = cell_range(p, mn, mx);
	bool over = false;
	const float4 elo = make_float4(mn.x, mn.y, mn.z, __uint_as_float((uint32_t)i));
	const auto put = [&](uint64_t slot, uint32_t packed) {
		if (slot < cap) {  // one 32-byte store (entries are 32-byte aligned)
			st_global_v8(reinterpret_cast<float *>(entries + 2 * slot), elo,
			             make_float4(mx.x, mx.y, mx.z, __uint_as_float(packed)));
		} else {
			over = true;
		}
	};
	// a slot in cell c: start + cursor, from one packed 64-bit atomic when the
	// scan wrote the packed words, else a start load and a cursor atomic
	const auto take = [&](uint32_t c) -> uint64_t {
		if (cs) {
			const unsigned long long w = atomicAdd(cs + c, 1ull);
			return (w >> 32) + (w & 0xffffffffull);
		}
		return (uint64_t)cell_start[c] + atomicAdd(&cursor[c], 1u);
	};
	const int nx = r.c1[0] - r.c0[0] + 1, ny = r.c1[1] - r.c0[1] + 1, nz = r.c1[2] - r.c0[2] + 1;
	if (nx <= 2 && ny <= 2 && nz <= 2) {
		// up to 2x2x2 cells (nearly every box): the offset loads and cursor
		// atomics of all its cells are issued before any result is used, so a
		// thread waits one memory round trip instead of one per cell
		uint32_t cell[8], packed[8], slot[8];
#pragma unroll
		for (int q = 0; q < 8; q++) {
			const int x = r.c0[0] + (q & 1), y = r.c0[1] + ((q >> 1) & 1), z = r.c0[2] + (q >> 2);
			cell[q] = cell_index(p, base, x, y, z);
			packed[q] = pack_cell(x, y, z);
		}
#pragma unroll
		for (int q = 0; q < 8; q++)
			if ((q & 1) < nx && ((q >> 1) & 1) < ny && (q >> 2) < nz)
				slot[q] = (uint32_t)take(cell[q]);
#pragma unroll
		for (int q = 0; q < 8; q++)
			if ((q & 1) < nx && ((q >> 1) & 1) < ny && (q >> 2) < nz) put(slot[q], packed[q]);
	} else {
		for (int z = r.c0[2]; z <= r.c1[2]; z++)
			for (int y = r.c0[1]; y <= r.c1[1]; y++)
				for (int x = r.c0[0]; x <= r.c1[0]; x++) {
					const uint32_t c = cell_index(p, base, x, y, z);
					put(take(c), pack_cell(x, y, z));
				}
	}
	if (over) atomicOr(err, (uint32_t)kErrCapacity);
}

// Each entry is tested against the later entries of its cell; a warp takes
// 32 entries and deals their tests out evenly over its lanes (so a warp's
// rounds follow the SUM of its entries' partner counts, not 32 x the largest). A warp's 32 entries and the kWin - 32 that follow them are
// staged in shared memory with coalesced 16-byte loads (cells hold a handful
// of entries, so the inner loop almost never leaves the window); loops are
// warp-uniform so the emission can be warp-aggregated: found pairs collect in
// a per-warp shared buffer that is flushed with one counter atomic per
// kOutBuf - 31 pairs or more (dense scenes emit billions of pairs).
constexpr int kWinDefault = 96;  // window (entries per warp staged in shared memory); tunable: 64, 96, 128
constexpr int kOutBuf = 128;

__device__ __forceinline__ void flush_pairs(unsigned long long *buf, uint32_t cnt, uint32_t lane,
                                            unsigned long long *pair_counter, unsigned long long *pairs,
                                            uint64_t pair_cap) {
	unsigned long long start = 0;
	if (lane == 0) start = atomicAdd(pair_counter, (unsigned long long)cnt);
	start = __shfl_sync(0xffffffffu, start, 0);
	for (uint32_t k = lane; k < cnt; k += 32) {
		const unsigned long long pos = start + k;
		if (pos < pair_cap) pairs[pos] = buf[k];
	}
	__syncwarp();
}

template <bool kBatch, int kWin>
__global__ void __launch_bounds__(kNT, 5) k_pair_test(const DevStats *stats, const uint32_t *__restrict__ cell_start,
                                                    const float4 *__restrict__ entries,
                                                    uint64_t entry_cap, uint32_t *__restrict__ owner_count,
                                                    unsigned long long *__restrict__ pairs, uint64_t pair_cap,
                                                    unsigned long long *pair_counter, SceneMap sm, uint2 *dense,
                                                    uint64_t dense_cap, unsigned long long *dense_count,
                                                    uint32_t *err, uint32_t dense_cell, int oshift) {
	pdl_begin();
	__shared__ Plan sp;
	__shared__ float4 win_all[kNT / 32][2 * kWin];
	__shared__ unsigned long long out_all[kNT / 32][kOutBuf];
	__shared__ uint32_t owned_s[kNT];  // pairs owned by each lane's entry in the current window
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	__syncthreads();
	if (!kBatch && !sp.valid) return;
	float4 *win = win_all[threadIdx.x >> 5];
	unsigned long long *obuf = out_all[threadIdx.x >> 5];
	uint32_t ocnt = 0;  // pairs in obuf (warp-uniform)
	const uint64_t E = min((uint64_t)stats->entries, entry_cap);
	const uint32_t lane = threadIdx.x & 31;
	const uint32_t lt = (1u << lane) - 1u;
	const uint64_t warps = (uint64_t)gridDim.x * (kNT / 32);
	for (uint64_t base = ((uint64_t)blockIdx.x * (kNT / 32) + (threadIdx.x >> 5)) * 32; base < E; base += warps * 32) {
		// stage entries [base, base + kWin) of this warp
		const uint32_t nwin = (uint32_t)min((uint64_t)kWin, E - base);
		__syncwarp();
		// asynchronous 16-byte copies straight into shared memory: all of the
		// window's loads are in flight at once and hold no registers
		for (uint32_t k = lane; k < 2 * nwin; k += 32) cp_async16(win + k, entries + 2 * base + k);
		cp_async_wait_all();
		__syncwarp();
		const uint64_t e = base + lane;
		const bool valid = e < E;
		float4 alo = make_float4(0.f, 0.f, 0.f, 0.f), ahi = alo;
		int my_n = 0;
		int cx = 0, cy = 0, cz = 0;
		const uint32_t ida = valid ? __float_as_uint(win[2 * lane].w) : 0u;
		uint32_t cbase;
		const Plan &pl = plan_of<kBatch>(sp, sm, ida, cbase);
		if (valid) {
			alo = win[2 * lane];
			ahi = win[2 * lane + 1];
			const uint32_t pc = __float_as_uint(ahi.w);
			cx = pc & 1023; cy = (pc >> 10) & 1023; cz = (pc >> 20) & 1023;
			const uint32_t c = cell_index(pl, cbase, cx, cy, cz);
			const uint64_t beg = cell_start[c];
			const uint64_t end = min((uint64_t)cell_start[c + 1], entry_cap);
			my_n = (int)(end > e + 1 ? end - e - 1 : 0);
			if (end - beg > dense_cell) {
				if (dense) {  // left to k_pair_test_dense
					my_n = 0;
					if (e == beg) {
						const uint32_t chunks = (uint32_t)((end - beg + kNT - 1) / kNT);
						const unsigned long long at = atomicAdd(dense_count, (unsigned long long)chunks);
						for (uint32_t q = 0; q < chunks; q++)
							if (at + q < dense_cap) dense[at + q] = make_uint2(c, q * kNT);
							else atomicOr(err, (uint32_t)kErrCapacity);
					}
				} else if (e == beg) {
					// no dense-cell kernel this call (the last found no dense
					// cell): tested here, and counted so the next call has one
					atomicAdd(dense_count, 1ull);
				}
			}
		}
		float lo0 = pl.lo[0], lo1 = pl.lo[1], lo2 = pl.lo[2];
		float iv0 = pl.inv[0], iv1 = pl.inv[1], iv2 = pl.inv[2];
		int d0 = pl.dim[0], d1 = pl.dim[1], d2 = pl.dim[2];

		// the warp's sum(my_n) tests, dealt out 32 per round: test k belongs to
		// the lane a with pre[a] <= k < pre[a] + my_n[a] (pre: exclusive scan)
		int pre = my_n;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int v = __shfl_up_sync(0xffffffffu, pre, o);
			if ((int)lane >= o) pre += v;
		}
		const int total = __shfl_sync(0xffffffffu, pre, 31);
		pre -= my_n;
		owned_s[threadIdx.x] = 0;
		__syncwarp();
		for (int k0 = 0; k0 < total; k0 += 32) {
			const int k = k0 + (int)lane;
			int a = 0;
#pragma unroll
			for (int step = 16; step > 0; step >>= 1) {
				const int v = __shfl_sync(0xffffffffu, pre, a + step);
				if (v <= k) a += step;
			}
			const int t = k - __shfl_sync(0xffffffffu, pre, a);
			if constexpr (kBatch) {  // entries of one warp may come from different scenes
				lo0 = __shfl_sync(0xffffffffu, pl.lo[0], a);
				lo1 = __shfl_sync(0xffffffffu, pl.lo[1], a);
				lo2 = __shfl_sync(0xffffffffu, pl.lo[2], a);
				iv0 = __shfl_sync(0xffffffffu, pl.inv[0], a);
				iv1 = __shfl_sync(0xffffffffu, pl.inv[1], a);
				iv2 = __shfl_sync(0xffffffffu, pl.inv[2], a);
				d0 = __shfl_sync(0xffffffffu, pl.dim[0], a);
				d1 = __shfl_sync(0xffffffffu, pl.dim[1], a);
				d2 = __shfl_sync(0xffffffffu, pl.dim[2], a);
			}
			bool emit = false;
			unsigned long long key = 0;
			uint32_t other_owner = 0xffffffffu;
			if (k < total) {
				const float4 plo = win[2 * a], phi = win[2 * a + 1];
				const uint32_t pc = __float_as_uint(phi.w);
				const int px = pc & 1023, py = (pc >> 10) & 1023, pz = (pc >> 20) & 1023;
				const uint32_t loc = (uint32_t)a + 1 + (uint32_t)t;  // partner's position in the window
				float4 blo, bhi;
				if (loc < nwin) {
					blo = win[2 * loc];
					bhi = win[2 * loc + 1];
				} else {
					const uint64_t q = base + loc;
					blo = entries[2 * q];
					bhi = entries[2 * q + 1];
				}
				if (plo.x <= bhi.x && blo.x <= phi.x && plo.y <= bhi.y && blo.y <= phi.y && plo.z <= bhi.z &&
				    blo.z <= phi.z) {
					// home cell: the cell holding the larger min corner on every
					// axis (a point of both boxes, so of both cell ranges); few
					// boxes overlap in sparse cells, so it is evaluated per pair
					const bool hx = cell_of(fmaxf(plo.x, blo.x), lo0, iv0, d0) == px;
					const bool hy = cell_of(fmaxf(plo.y, blo.y), lo1, iv1, d1) == py;
					const bool hz = cell_of(fmaxf(plo.z, blo.z), lo2, iv2, d2) == pz;
					if (hx && hy && hz) {
						const uint32_t ia = __float_as_uint(plo.w), idb = __float_as_uint(blo.w);
						const uint32_t lo = min(ia, idb), hi = max(ia, idb);
						key = ((unsigned long long)lo << 32) | hi;
						emit = true;
						if (lo == ia) atomicAdd(&owned_s[(threadIdx.x & ~31u) + a], 1u);
						else other_owner = lo;
					}
				}
			}
			const uint32_t b = __ballot_sync(0xffffffffu, emit);
			if (b) {
				const uint32_t nb = __popc(b);
				if (ocnt + nb > kOutBuf) {
					flush_pairs(obuf, ocnt, lane, pair_counter, pairs, pair_cap);
					ocnt = 0;
				}
				if (emit) {
					obuf[ocnt + __popc(b & lt)] = key;
					if (other_owner != 0xffffffffu) atomicAdd(&owner_count[other_owner >> oshift], 1u);
				}
				ocnt += nb;
				__syncwarp();
			}
		}
		__syncwarp();
		const uint32_t owned = owned_s[threadIdx.x];
		if (owned) atomicAdd(&owner_count[ida >> oshift], owned);
	}
	if (ocnt) flush_pairs(obuf, ocnt, lane, pair_counter, pairs, pair_cap);
}

// Dense cells: one block per (cell, chunk of 256 rows). Thread t takes row
// i = r0 + t and tests it against every later entry j > i of the cell, the
// columns staged 256 at a time in shared memory and read by all lanes at once
// (a broadcast), so one warp instruction carries 32 tests. Pairs owned by the
// row (smaller index) are counted in a register, pairs owned by the column in
// a shared counter per column; both reach owner_count once per tile.
constexpr int kDenseOut = 512;
template <bool kBatch>
__global__ void __launch_bounds__(kNT) k_pair_test_dense(const DevStats *stats, const uint32_t *__restrict__ cell_start,
                                                          const float4 *__restrict__ entries, uint64_t entry_cap,
                                                          uint32_t *__restrict__ owner_count,
                                                          unsigned long long *__restrict__ pairs, uint64_t pair_cap,
                                                          unsigned long long *pair_counter, SceneMap sm,
                                                          const uint2 *__restrict__ dense, uint64_t dense_cap,
                                                          int oshift) {
	pdl_begin();
	__shared__ Plan sp;
	__shared__ float4 tlo[kNT], thi[kNT];
	__shared__ uint32_t colown[kNT], tcode[kNT];
	__shared__ unsigned long long out_all[kNT / 32][kDenseOut];
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	__syncthreads();
	if (!kBatch && !sp.valid) return;
	const uint64_t items = min((uint64_t)stats->dense_items, dense_cap);
	unsigned long long *obuf = out_all[threadIdx.x >> 5];
	uint32_t ocnt = 0;
	const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
	for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
		const uint2 w = dense[it];
		const uint64_t s0 = cell_start[w.x];
		const uint64_t s1 = min((uint64_t)cell_start[w.x + 1], entry_cap);
		const uint32_t k = (uint32_t)(s1 - s0), r0 = w.y;
		const uint32_t i = r0 + threadIdx.x;
		const bool row = i < k;
		float4 alo = make_float4(0.f, 0.f, 0.f, 0.f), ahi = alo;
		if (row) {
			alo = entries[2 * (s0 + i)];
			ahi = entries[2 * (s0 + i) + 1];
		}
		const uint32_t ida = __float_as_uint(alo.w);
		const uint32_t pc = __float_as_uint(ahi.w);
		uint32_t cb;
		const Plan &pl = plan_of<kBatch>(sp, sm, row ? ida : __float_as_uint(entries[2 * s0].w), cb);
		const uint32_t rcode = home_code(pl, alo, pc);
		uint32_t owned = 0;
		for (uint32_t c0 = r0; c0 < k; c0 += kNT) {
			const uint32_t nt = min((uint32_t)kNT, k - c0);
			__syncthreads();  // the previous tile is no longer read
			if (threadIdx.x < nt) {
				const float4 l = entries[2 * (s0 + c0 + threadIdx.x)], h = entries[2 * (s0 + c0 + threadIdx.x) + 1];
				tlo[threadIdx.x] = l;
				thi[threadIdx.x] = h;
				tcode[threadIdx.x] = home_code(pl, l, __float_as_uint(h.w));  // the rows' cell
			}
			colown[threadIdx.x] = 0;
			__syncthreads();
			// only j > i is tested: on the diagonal tile (c0 == r0) that needs a
			// check per column, every later tile lies wholly past this block's rows
			const auto column = [&](uint32_t jj, bool test) {
				bool emit = false;
				unsigned long long key = 0;
				if (test) {
					const float4 blo = tlo[jj], bhi = thi[jj];
					if (alo.x <= bhi.x && blo.x <= ahi.x && alo.y <= bhi.y && blo.y <= ahi.y && alo.z <= bhi.z &&
					    blo.z <= ahi.z) {
						if (home_pair(rcode, tcode[jj])) {
							const uint32_t idb = __float_as_uint(blo.w);
							const uint32_t lo = min(ida, idb), hi = max(ida, idb);
							key = ((unsigned long long)lo << 32) | hi;
							emit = true;
							if (lo == ida) owned++;
							else atomicAdd(&colown[jj], 1u);
						}
					}
				}
				const uint32_t bal = __ballot_sync(0xffffffffu, emit);
				if (bal) {
					const uint32_t nb = __popc(bal);
					if (ocnt + nb > kDenseOut) {
						flush_pairs(obuf, ocnt, lane, pair_counter, pairs, pair_cap);
						ocnt = 0;
					}
					if (emit) obuf[ocnt + __popc(bal & lt)] = key;
					ocnt += nb;
					__syncwarp();
				}
			};
			if (c0 == r0) {
				for (uint32_t jj = 0; jj < nt; jj++) column(jj, row && c0 + jj > i);
			} else {
#pragma unroll 4
				for (uint32_t jj = 0; jj < nt; jj++) column(jj, row);
			}
			__syncthreads();  // column counts complete
			if (threadIdx.x < nt && colown[threadIdx.x])
				atomicAdd(&owner_count[__float_as_uint(tlo[threadIdx.x].w) >> oshift], colown[threadIdx.x]);
		}
		if (owned) atomicAdd(&owner_count[ida >> oshift], owned);
	}
	if (ocnt) flush_pairs(obuf, ocnt, lane, pair_counter, pairs, pair_cap);
}

// Bucket the unsorted pairs by owner bucket (the smaller index >> oshift). P
// comes from the device; if it exceeds the scratch or the output nothing is
// written.
__global__ void __launch_bounds__(kNT) k_owner_scatter(DevStats *stats, uint64_t pair_cap, uint64_t out_cap,
                                                        const unsigned long long *__restrict__ tmp,
                                                        const unsigned long long *__restrict__ owner_off,
                                                        uint32_t *__restrict__ owner_count,
                                                        unsigned long long *__restrict__ out, int oshift) {
	pdl_begin();
	const unsigned long long P = stats->pairs;
	const bool fits = P <= pair_cap && P <= out_cap;
	if (blockIdx.x == 0 && threadIdx.x == 0) stats->np_n = fits ? P : 0ull;
	if (!fits) return;
	// lanes of a warp whose pairs share an owner take their slots with one
	// atomic (pair lists of dense cells arrive grouped by owner)
	const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
	const uint64_t step = (uint64_t)gridDim.x * kNT;
	for (uint64_t t0 = (uint64_t)blockIdx.x * kNT + (threadIdx.x & ~31u); t0 < P; t0 += step) {
		const uint64_t t = t0 + lane;
		const bool valid = t < P;
		const unsigned long long key = valid ? tmp[t] : 0ull;
		const uint32_t a = valid ? (uint32_t)(key >> 32) >> oshift : 0xffffffffu;
		const uint32_t peers = __match_any_sync(0xffffffffu, a);
		const int leader = __ffs(peers) - 1;
		uint32_t base = 0;
		if (valid && (int)lane == leader) base = atomicSub(&owner_count[a], (uint32_t)__popc(peers));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (valid) out[owner_off[a] + base - 1u - __popc(peers & lt)] = key;
	}
}

// Sort keys inside an owner bucket: 32-bit packings of the 64-bit pair keys
// that order like them (the bucket fixes the high bits of the owner).
struct KeyPack {
	int shift, kb;  // BpBuffers::owner_shift, key_bits
};
// kPack false: one owner per bucket (shift 0), the key is the partner half.
// The choice is a template parameter, resolved per kernel launch: a runtime
// test inside the register sorts' unrolled load and store loops made the
// warp-tier kernel almost twice as slow on the 16.7M clustered scene.
template <bool kPack>
__device__ __forceinline__ uint32_t pack_key(unsigned long long key, KeyPack kp) {
	const uint32_t b = (uint32_t)key;
	if constexpr (!kPack) {
		return b;
	} else {
		const uint32_t alo = (uint32_t)(key >> 32) & ((1u << kp.shift) - 1u);
		return (alo << kp.kb) | b;
	}
}
template <bool kPack>
__device__ __forceinline__ unsigned long long unpack_key(uint32_t v, uint32_t bucket, KeyPack kp) {
	if constexpr (!kPack) {
		return ((unsigned long long)bucket << 32) | v;
	} else {
		const uint32_t a = (bucket << kp.shift) | (v >> kp.kb);
		return ((unsigned long long)a << 32) | (v & ((1u << kp.kb) - 1u));
	}
}

constexpr int kTinySeg = 8;    // buckets sorted by one thread with a bubble network in registers
constexpr int kSmallSeg = 32;  // buckets sorted by one thread with a bitonic network in registers

// Compare-exchange of two 64-bit keys held in registers (ascending).
__device__ __forceinline__ void cx64(unsigned long long &x, unsigned long long &y) {
	const unsigned long long a = x, b = y;
	x = a < b ? a : b;
	y = a < b ? b : a;
}
constexpr int kMidSeg = 1024;
constexpr int kBigSeg = 16384;

// One bucket of at most kSmallSeg 64-bit keys sorted by one thread in
// registers: a bubble network up to kTinySeg keys, a bitonic network padded
// to kSmallSeg above (one load and one store round trip either way).
__device__ __forceinline__ void sort_thread_bucket(unsigned long long *__restrict__ out, uint64_t beg, uint64_t len) {
	if (len > 1 && len <= kTinySeg) {
		unsigned long long v[kTinySeg];
#pragma unroll
		for (int q = 0; q < kTinySeg; q++) v[q] = (uint64_t)q < len ? out[beg + q] : ~0ull;
#pragma unroll
		for (int r = 0; r < kTinySeg - 1; r++)
#pragma unroll
			for (int q = 0; q < kTinySeg - 1 - r; q++) cx64(v[q], v[q + 1]);
#pragma unroll
		for (int q = 0; q < kTinySeg; q++)
			if ((uint64_t)q < len) out[beg + q] = v[q];
	} else if (len > kTinySeg && len <= kSmallSeg) {
		unsigned long long v[kSmallSeg];
#pragma unroll
		for (int q = 0; q < kSmallSeg; q++) v[q] = (uint64_t)q < len ? out[beg + q] : ~0ull;
#pragma unroll
		for (int k = 2; k <= kSmallSeg; k <<= 1)
#pragma unroll
			for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
				for (int i = 0; i < kSmallSeg; i++) {
					const int l = i ^ j;
					if (l > i) {
						if ((i & k) == 0) cx64(v[i], v[l]);
						else cx64(v[l], v[i]);
					}
				}
#pragma unroll
		for (int q = 0; q < kSmallSeg; q++)
			if ((uint64_t)q < len) out[beg + q] = v[q];
	}
}

// Sorts each owner bucket (all keys share the bucket's owners, n here is the
// bucket count): <= 32 keys by one thread, loaded into registers at once and
// sorted there by a static network on the 64-bit keys (a bubble network up to
// 8 keys, a bitonic network padded to 32 above); longer buckets are listed for
// k_segsort_mid (<= 1024 keys, from the front of big_list) or k_segsort_big
// (<= 16384, from the back), which sort the packed 32-bit keys (pack_key).
__global__ void __launch_bounds__(kNT) k_segsort(uint64_t n, const unsigned long long *__restrict__ owner_off,
                                                  unsigned long long *__restrict__ out, uint32_t *big_list,
                                                  uint64_t big_cap, DevStats *stats) {
	pdl_begin();
	if (stats->np_n != stats->pairs) return;  // the pairs were not emitted (uniform over the grid)
	const uint64_t a = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	uint64_t len = 0;
	if (a < n) {
		const uint64_t beg = owner_off[a], end = owner_off[a + 1];
		len = end - beg;
		sort_thread_bucket(out, beg, len);
	}
	const bool longer = len > kSmallSeg;
	const uint32_t wmax = __reduce_max_sync(0xffffffffu, longer ? (uint32_t)min(len, (uint64_t)0xffffffffu) : 0u);
	if ((threadIdx.x & 31) == 0 && wmax) atomicMax(&stats->max_segment, (unsigned long long)wmax);
	if (len > kBigSeg) atomicOr(&stats->err, (uint32_t)kErrSegmentTooLong);
	// list the longer buckets, one counter atomic per warp and tier
	const bool mid = longer && len <= kMidSeg, big = len > kMidSeg && len <= kBigSeg;
	const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
#pragma unroll
	for (int tier = 0; tier < 2; tier++) {
		const bool want = tier == 0 ? mid : big;
		const uint32_t m = __ballot_sync(0xffffffffu, want);
		if (!m) continue;
		unsigned long long base = 0;
		if (lane == (uint32_t)(__ffs(m) - 1)) base = atomicAdd(tier == 0 ? &stats->big_segments : &stats->seg_big,
		                                                       (unsigned long long)__popc(m));
		base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
		if (want) {
			const unsigned long long slot = base + __popc(m & lt);
			if (slot < big_cap) big_list[tier == 0 ? slot : big_cap - 1 - slot] = (uint32_t)a;
			else atomicOr(&stats->err, (uint32_t)kErrSegmentTooLong);
		}
	}
}

// In-place bitonic sort of m (a power of two) 32-bit keys in shared memory by
// `nt` cooperating threads (thread t of them); sync() separates the steps.
template <class Sync>
__device__ __forceinline__ void bitonic_u32(uint32_t *s, int m, int t, int nt, Sync sync) {
	for (int k = 2; k <= m; k <<= 1) {
		for (int j = k >> 1; j > 0; j >>= 1) {
			// compare-exchange q pairs (i, i + j), i with bit j clear: every thread busy
			for (int q = t; q < (m >> 1); q += nt) {
				const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));
				const int p = i + j;
				const bool up = (i & k) == 0;
				const uint32_t x = s[i], y = s[p];
				if ((x > y) == up) {
					s[i] = y;
					s[p] = x;
				}
			}
			sync();
		}
	}
}

// Register bitonic sort of 32*K keys held by one warp, striped: key e = 32*r
// + lane sits in v[r] of that lane. Steps whose partner distance j is below 32
// exchange across lanes (shuffle), the others pair registers of the same lane
// (register distance j/32, resolved at compile time through a switch so that
// v stays in registers).
// el = the key index held in v[0] by this lane (the warp's first key +
// lane); the network sorts key e ascending where (e & k) == 0 in merge size k.
template <int K, int JR>
__device__ __forceinline__ void bitonic_reg_step(uint32_t (&v)[K], int el, int k) {
	if constexpr (JR < K) {
#pragma unroll
		for (int r = 0; r < K; r++)
			if ((r & JR) == 0) {
				const bool up = ((el + 32 * r) & k) == 0;
				const uint32_t x = v[r], y = v[r | JR];
				v[r] = up ? min(x, y) : max(x, y);
				v[r | JR] = up ? max(x, y) : min(x, y);
			}
	}
}
// One step of partner distance j < 32 * K (inside the warp's keys).
template <int K>
__device__ __forceinline__ void bitonic_warp_step(uint32_t (&v)[K], int el, int j, int k) {
	if (j < 32) {
		const bool lower = (el & j) == 0;
#pragma unroll
		for (int r = 0; r < K; r++) {
			const uint32_t o = __shfl_xor_sync(0xffffffffu, v[r], j);
			const bool up = ((el + 32 * r) & k) == 0;
			v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
		}
	} else {
		switch (j >> 5) {
		case 1: bitonic_reg_step<K, 1>(v, el, k); break;
		case 2: bitonic_reg_step<K, 2>(v, el, k); break;
		case 4: bitonic_reg_step<K, 4>(v, el, k); break;
		case 8: bitonic_reg_step<K, 8>(v, el, k); break;
		case 16: bitonic_reg_step<K, 16>(v, el, k); break;
		}
	}
}
template <int K>
__device__ __forceinline__ void bitonic_reg(uint32_t (&v)[K], int lane) {
	for (int k = 2; k <= 32 * K; k <<= 1)
		for (int j = k >> 1; j > 0; j >>= 1) bitonic_warp_step<K>(v, lane, j, k);
}
// One bucket of len <= 32*K keys: partner halves into registers (padding
// sorts last), sorted, written back with the owner in the high half.
template <int K, bool kPack>
__device__ __forceinline__ void sort_bucket_reg(unsigned long long *__restrict__ out, uint64_t beg, uint64_t len,
                                                uint32_t a, int lane, KeyPack kp) {
	uint32_t v[K];
#pragma unroll
	for (int r = 0; r < K; r++) {
		const uint64_t e = 32u * r + lane;
		v[r] = e < len ? pack_key<kPack>(out[beg + e], kp) : 0xffffffffu;
	}
	bitonic_reg<K>(v, lane);
#pragma unroll
	for (int r = 0; r < K; r++) {
		const uint64_t e = 32u * r + lane;
		if (e < len) out[beg + e] = unpack_key<kPack>(v[r], a, kp);
	}
}

// A bucket of 1025..2048 keys on a pair of warps (half = 0, 1), 1024 keys
// each, 32 per lane; the one step of partner distance 1024 exchanges through
// the pair's 8 KB of shared memory x, the pair synchronizing on its own
// named barrier `bar` (both warps run the same steps).
constexpr int kPairSeg = 2048;
__device__ __forceinline__ void pair_sync(int bar) { asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory"); }
template <bool kPack>
__device__ __forceinline__ void sort_bucket_pair(unsigned long long *__restrict__ out, uint64_t beg, uint64_t len,
                                                 uint32_t a, int half, int lane, uint32_t *x, int bar, KeyPack kp) {
	const int el = half * 1024 + lane;
	uint32_t v[32];
#pragma unroll
	for (int r = 0; r < 32; r++) {
		const uint64_t e = (uint64_t)el + 32u * r;
		v[r] = e < len ? pack_key<kPack>(out[beg + e], kp) : 0xffffffffu;
	}
	for (int k = 2; k <= kPairSeg; k <<= 1)
		for (int j = k >> 1; j > 0; j >>= 1) {
			if (j == 1024) {
#pragma unroll
				for (int r = 0; r < 32; r++) x[el + 32 * r] = v[r];
				pair_sync(bar);
				const bool lower = half == 0;
#pragma unroll
				for (int r = 0; r < 32; r++) {
					const uint32_t o = x[(el + 32 * r) ^ 1024];
					const bool up = ((el + 32 * r) & k) == 0;
					v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
				}
				pair_sync(bar);  // x is free again
			} else {
				bitonic_warp_step<32>(v, el, j, k);
			}
		}
#pragma unroll
	for (int r = 0; r < 32; r++) {
		const uint64_t e = (uint64_t)el + 32u * r;
		if (e < len) out[beg + e] = unpack_key<kPack>(v[r], a, kp);
	}
}

// Buckets of 33..1024 keys: one warp per bucket, sorted in registers
// (2..32 keys per lane by bucket size); then buckets of 1025..2048 keys
// (listed for k_segsort_big, which leaves them) on pairs of warps.
constexpr int kMidNT = 256;
template <bool kPack>
__global__ void __launch_bounds__(kMidNT, 2) k_segsort_mid(const DevStats *stats, uint64_t big_cap,
                                                         const uint32_t *__restrict__ big_list,
                                                         const unsigned long long *__restrict__ owner_off,
                                                         unsigned long long *__restrict__ out, KeyPack kp) {
	pdl_begin();
	if (stats->np_n != stats->pairs) return;
	const uint64_t nmid = min((uint64_t)stats->big_segments, big_cap);
	const int lane = threadIdx.x & 31;
	const uint64_t warps = (uint64_t)gridDim.x * (kMidNT / 32);
	for (uint64_t g = (uint64_t)blockIdx.x * (kMidNT / 32) + (threadIdx.x >> 5); g < nmid; g += warps) {
		const uint32_t a = big_list[g];
		const uint64_t beg = owner_off[a], len = owner_off[a + 1] - beg;  // 33..1024, listed by k_segsort
		if (len <= 64) sort_bucket_reg<2, kPack>(out, beg, len, a, lane, kp);
		else if (len <= 128) sort_bucket_reg<4, kPack>(out, beg, len, a, lane, kp);
		else if (len <= 256) sort_bucket_reg<8, kPack>(out, beg, len, a, lane, kp);
		else if (len <= 512) sort_bucket_reg<16, kPack>(out, beg, len, a, lane, kp);
		else sort_bucket_reg<32, kPack>(out, beg, len, a, lane, kp);
	}
	__shared__ uint32_t xch[kMidNT / 64][kPairSeg];
	const uint64_t nbig = min((uint64_t)stats->seg_big, big_cap);
	const int pair = threadIdx.x >> 6, half = (threadIdx.x >> 5) & 1;
	const uint64_t npairs = (uint64_t)gridDim.x * (kMidNT / 64);
	for (uint64_t g = (uint64_t)blockIdx.x * (kMidNT / 64) + pair; g < nbig; g += npairs) {
		const uint32_t a = big_list[big_cap - 1 - g];
		const uint64_t beg = owner_off[a], len = owner_off[a + 1] - beg;
		if (len > kPairSeg) continue;  // the block tier's (uniform over the pair)
		sort_bucket_pair<kPack>(out, beg, len, a, half, lane, xch[pair], 1 + pair, kp);
	}
}

// Buckets of 2049..16384 keys: one block per bucket (grid-stride over the
// device-side count), bitonic sort of the partner halves in 64 KB of
// dynamic shared memory.
template <bool kPack>
__global__ void __launch_bounds__(512) k_segsort_big(const DevStats *stats, uint64_t big_cap,
                                                      const uint32_t *__restrict__ big_list,
                                                      const unsigned long long *__restrict__ owner_off,
                                                      unsigned long long *__restrict__ out, KeyPack kp) {
	pdl_begin();
	extern __shared__ uint32_t s[];
	if (stats->np_n != stats->pairs) return;
	const uint64_t nbig = min((uint64_t)stats->seg_big, big_cap);
	for (uint64_t g = blockIdx.x; g < nbig; g += gridDim.x) {
		const uint32_t a = big_list[big_cap - 1 - g];
		const uint64_t beg = owner_off[a], len = owner_off[a + 1] - beg;
		if (len <= kPairSeg) continue;  // sorted by warp pairs in k_segsort_mid (uniform over the block)
		int m = 1;
		while ((uint64_t)m < len) m <<= 1;
		for (int i = threadIdx.x; i < m; i += blockDim.x) s[i] = (uint64_t)i < len ? pack_key<kPack>(out[beg + i], kp) : 0xffffffffu;
		__syncthreads();
		bitonic_u32(s, m, threadIdx.x, blockDim.x, [] { __syncthreads(); });
		for (int i = threadIdx.x; (uint64_t)i < len; i += blockDim.x) out[beg + i] = unpack_key<kPack>(s[i], a, kp);
		__syncthreads();
	}
}

// ---------------------------------------------------------------- fused owner sort
// Pair lists far shorter than the body count (the owner shift then keeps about
// eight pairs per bucket, so there are few buckets): the owner scan, the
// bucketing and every bucket sort of the path above run as ONE cooperative
// kernel. Each block scans all bucket counts itself into shared memory (a few
// KB read from L2 per block; no scan launch), buckets its share of the pairs
// through per-bucket cursors (zeroed by k_count, so the counts stay intact
// while other blocks still scan them), waits at one grid barrier, and sorts
// the buckets: <= 32 keys per thread, 33..1024 per warp in registers,
// 1025..kFusedSeg per block in shared memory. A longer bucket sets
// kErrSegmentTooLong (the caller then sorts the whole list).
constexpr int kFusedNT = 256;
constexpr int kFusedSeg = 4096;
constexpr uint32_t kFusedBuckets = 8191;  // offsets + block-tier keys fit the default 48 KB of shared memory

template <bool kPack>
__global__ void __launch_bounds__(kFusedNT) k_owner_sort_fused(DevStats *stats, uint64_t pair_cap, uint64_t out_cap,
                                                             const unsigned long long *__restrict__ tmp,
                                                             const uint32_t *__restrict__ owner_count,
                                                             uint32_t *__restrict__ cursor, uint32_t nbk,
                                                             unsigned long long *__restrict__ out, int oshift,
                                                             KeyPack kp) {
	extern __shared__ uint32_t fsm[];  // off[nbk + 1], then kFusedSeg keys of the block tier
	__shared__ unsigned long long scan_sm[40];
	uint32_t *off = fsm, *keys = fsm + nbk + 1;
	const unsigned long long P = stats->pairs;
	const bool fits = P <= pair_cap && P <= out_cap && P < 0xffffffffull;
	if (blockIdx.x == 0 && threadIdx.x == 0) stats->np_n = fits ? P : 0ull;
	if (!fits) return;  // uniform over the grid: no block reaches the barrier
	// 1. exclusive scan of the bucket counts: coalesced loads into shared
	// memory (all in flight at once), then one contiguous run per thread
	copy_words_to_shared<kFusedNT>(off, owner_count, nbk);
	__syncthreads();
	const uint32_t per = (nbk + kFusedNT - 1) / kFusedNT;
	const uint32_t b0 = min(nbk, threadIdx.x * per), b1 = min(nbk, b0 + per);
	unsigned long long run = 0;
	for (uint32_t b = b0; b < b1; b++) run += off[b];
	unsigned long long total;
	unsigned long long excl = block_excl_scan<unsigned long long, kFusedNT>(run, scan_sm, &total);
	for (uint32_t b = b0; b < b1; b++) {
		const uint32_t c = off[b];
		off[b] = (uint32_t)excl;
		excl += c;
	}
	if (threadIdx.x == 0) off[nbk] = (uint32_t)total;
	__syncthreads();
	// 2. bucket the pairs (lanes of a warp with one bucket share one atomic)
	const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
	const uint64_t step = (uint64_t)gridDim.x * kFusedNT;
	for (uint64_t t0 = (uint64_t)blockIdx.x * kFusedNT + (threadIdx.x & ~31u); t0 < P; t0 += step) {
		const uint64_t t = t0 + lane;
		const bool valid = t < P;
		const unsigned long long key = valid ? tmp[t] : 0ull;
		const uint32_t a = valid ? (uint32_t)(key >> 32) >> oshift : 0xffffffffu;
		const uint32_t peers = __match_any_sync(0xffffffffu, a);
		const int leader = __ffs(peers) - 1;
		uint32_t base = 0;
		if (valid && (int)lane == leader) base = atomicAdd(&cursor[a], (uint32_t)__popc(peers));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (valid) out[(uint64_t)off[a] + base + __popc(peers & lt)] = key;
	}
	grid_barrier(reinterpret_cast<GridBarrier *>(stats->bar_emit), &stats->err);
	// 3. sort the buckets, three tiers
	const uint64_t gt = (uint64_t)blockIdx.x * kFusedNT + threadIdx.x;
	uint32_t longest = 0;
	for (uint64_t b = gt; b < nbk; b += step) {
		const uint32_t beg = off[b], len = off[b + 1] - beg;
		sort_thread_bucket(out, beg, len);
		longest = max(longest, len);
	}
	longest = __reduce_max_sync(0xffffffffu, longest);
	if (lane == 0 && longest > kSmallSeg) atomicMax(&stats->max_segment, (unsigned long long)longest);
	if (lane == 0 && longest > kFusedSeg) atomicOr(&stats->err, (uint32_t)kErrSegmentTooLong);
	const uint64_t warps = step / 32;
	for (uint64_t b = gt / 32; b < nbk; b += warps) {
		const uint32_t beg = off[b], len = off[b + 1] - beg;  // uniform over the warp
		if (len <= kSmallSeg || len > kMidSeg) continue;
		if (len <= 64) sort_bucket_reg<2, kPack>(out, beg, len, (uint32_t)b, lane, kp);
		else if (len <= 128) sort_bucket_reg<4, kPack>(out, beg, len, (uint32_t)b, lane, kp);
		else if (len <= 256) sort_bucket_reg<8, kPack>(out, beg, len, (uint32_t)b, lane, kp);
		else if (len <= 512) sort_bucket_reg<16, kPack>(out, beg, len, (uint32_t)b, lane, kp);
		else sort_bucket_reg<32, kPack>(out, beg, len, (uint32_t)b, lane, kp);
	}
	for (uint64_t b = blockIdx.x; b < nbk; b += gridDim.x) {
		const uint32_t beg = off[b], len = off[b + 1] - beg;  // uniform over the block
		if (len <= kMidSeg || len > kFusedSeg) continue;
		int m = 1;
		while ((uint32_t)m < len) m <<= 1;
		for (int i = threadIdx.x; i < m; i += kFusedNT) keys[i] = (uint32_t)i < len ? pack_key<kPack>(out[beg + i], kp) : 0xffffffffu;
		__syncthreads();
		bitonic_u32(keys, m, threadIdx.x, kFusedNT, [] { __syncthreads(); });
		for (int i = threadIdx.x; (uint32_t)i < len; i += kFusedNT) out[beg + i] = unpack_key<kPack>(keys[i], (uint32_t)b, kp);
		__syncthreads();
	}
}

// ---------------------------------------------------------------- bin list
// float -> int as the reference's host build converts (x86 cvttss2si: NaN and
// out-of-range values give INT_MIN), HashMin Broadphase.cu:125-133.
__device__ __forceinline__ int32_t trunc_x86(float v) {
	if (!(v >= -2147483648.0f && v < 2147483648.0f)) return INT_MIN;
	return __float2int_rz(v);
}
struct RefRange {
	int32_t g0[3], g1[3];
};
__device__ __forceinline__ RefRange ref_range(const Plan &p, float3 mn, float3 mx) {
	RefRange r;
	r.g0[0] = trunc_x86(mn.x * p.invbin[0]);
	r.g0[1] = trunc_x86(mn.y * p.invbin[1]);
	r.g0[2] = trunc_x86(mn.z * p.invbin[2]);
	r.g1[0] = trunc_x86(mx.x * p.invbin[0]);
	r.g1[1] = trunc_x86(mx.y * p.invbin[1]);
	r.g1[2] = trunc_x86(mx.z * p.invbin[2]);
	return r;
}

// function_Count_AABB_BIN_Intersection (:150-154) on the shifted boxes.
__global__ void __launch_bounds__(kNT) k_ref_count(uint64_t n, const float *__restrict__ aabb, const DevStats *stats,
                                                    uint32_t *__restrict__ cnt) {
	__shared__ Plan sp;
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	__syncthreads();
	const uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	if (i >= n) return;
	const RefRange r = ref_range(sp, ld3p(aabb, i), ld3p(aabb, i + n));
	const uint32_t c = (uint32_t)(r.g1[0] - r.g0[0] + 1) * (uint32_t)(r.g1[1] - r.g0[1] + 1) *
	                   (uint32_t)(r.g1[2] - r.g0[2] + 1);
	cnt[i] = c;
}

// function_Store_AABB_BIN_Intersection (:172-195): x outer, z inner, bin id
// z*gy*gx + y*gx + x in uint arithmetic (Hash_Index :140-147); the key is
// (bin << 32) | body so a stable sort on the upper half gives :428-432.
__global__ void __launch_bounds__(kNT) k_ref_emit(uint64_t n, const float *__restrict__ aabb, DevStats *stats,
                                                   const unsigned long long *__restrict__ off,
                                                   unsigned long long *__restrict__ keys, uint64_t cap) {
	__shared__ Plan sp;
	if (threadIdx.x < sizeof(Plan) / 4)
		reinterpret_cast<uint32_t *>(&sp)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&stats->plan)[threadIdx.x];
	__syncthreads();
	const uint64_t i = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	if (i >= n) return;
	const RefRange r = ref_range(sp, ld3p(aabb, i), ld3p(aabb, i + n));
	const uint32_t gx = (uint32_t)sp.grid[0], gy = (uint32_t)sp.grid[1];
	uint64_t w = off[i];
	const uint64_t wend = off[i + 1];
	uint32_t mb = 0;
	for (uint32_t x = (uint32_t)r.g0[0]; x <= (uint32_t)r.g1[0]; x++)
		for (uint32_t y = (uint32_t)r.g0[1]; y <= (uint32_t)r.g1[1]; y++)
			for (uint32_t z = (uint32_t)r.g0[2]; z <= (uint32_t)r.g1[2] && w < wend; z++) {
				const uint32_t bin = z * gy * gx + y * gx + x;
				mb = max(mb, bin);
				if (w < cap) keys[w] = ((unsigned long long)bin << 32) | (uint32_t)i;
				w++;
			}
	atomicMax(&stats->max_bin, mb);
	if (w != wend) atomicOr(&stats->err, (uint32_t)kErrBinCount);
}

__global__ void __launch_bounds__(kNT) k_ref_flags(const unsigned long long *__restrict__ keys, uint64_t E,
                                                    uint32_t *__restrict__ flags) {
	const uint64_t e = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	if (e >= E) return;
	flags[e] = (e == 0 || (keys[e] >> 32) != (keys[e - 1] >> 32)) ? 1u : 0u;
}

// reduce_by_key (:439-443) + inclusive scan of the run lengths (:476-480).
__global__ void __launch_bounds__(kNT) k_ref_split(const unsigned long long *__restrict__ keys, uint64_t E,
                                                    const uint32_t *__restrict__ run_pos, uint32_t *bin_number,
                                                    uint32_t *body_number, uint32_t *active_bins, uint32_t *bin_end,
                                                    uint64_t cap_a) {
	const uint64_t e = (uint64_t)blockIdx.x * kNT + threadIdx.x;
	if (e >= E) return;
	const unsigned long long k = keys[e];
	const uint32_t bin = (uint32_t)(k >> 32);
	if (bin_number) bin_number[e] = bin;
	if (body_number) body_number[e] = (uint32_t)k;
	const uint32_t r = run_pos[e + 1] - 1u;  // run index of this entry
	if (r < cap_a) {
		if (active_bins && run_pos[e] == r) active_bins[r] = bin;  // first entry of the run
		if (bin_end && (e + 1 == E || run_pos[e + 2] != run_pos[e + 1])) bin_end[r] = (uint32_t)(e + 1);
	}
}

inline unsigned blocks_for(uint64_t n) { return (unsigned)((n + kNT - 1) / kNT); }
}  // namespace

void launch_bounds(uint64_t n, const float *aabb, DevStats *stats, const GridParams &gp, const int grid[3],
                   cudaStream_t s, const ZeroList &zero) {
	PlanArgs pa;
	pa.gp = gp;
	pa.gx = grid[0];
	pa.gy = grid[1];
	pa.gz = grid[2];
	pa.n = n;
	if (n) k_bounds<<<blocks_for(n), kNT, 0, s>>>(n, aabb, stats, pa, zero);
}

void launch_count(uint64_t n, float *aabb, const BpBuffers &b, cudaStream_t s) {
	if (!n) return;
	if (b.sm.plans)
		launch_pdl(k_count<true>, dim3(blocks_for(n)), dim3(kNT), 0, s, n, aabb, b.stats, b.cell_count, b.owner_count, b.sm, 0,
		           (uint32_t *)nullptr);
	else
		launch_pdl(k_count<false>, dim3(blocks_for(n)), dim3(kNT), 0, s, n, aabb, b.stats, b.cell_count, b.owner_count, b.sm,
		           b.owner_shift, b.owner_cursor);
}

// ---------------------------------------------------------------- cell offsets
// The cell offsets as one cooperative launch (reduce, one grid barrier, scan):
// each block sums its contiguous chunk of the counts, waits at the barrier,
// adds up the sums of the blocks before it (at most kScanCoopBlocks words)
// and scans its chunk on top, zeroing the counts behind it for the scatter's
// cursors. The single-pass look-back scan spent 13 us of a 1M-body step here
// almost entirely waiting (1 % SM throughput): its tiles wait on one another
// at L2 latency, the barrier is one round trip for the whole grid.
constexpr int kCsNT = 256, kCsIPT = 4, kCsTile = kCsNT * kCsIPT;
__global__ void __launch_bounds__(kCsNT) k_scan_cells_coop(DevStats *stats, uint32_t g_max, uint32_t *__restrict__ counts,
                                                         uint32_t *__restrict__ start,
                                                         unsigned long long *__restrict__ bsum,
                                                         unsigned long long *__restrict__ cs) {
	__shared__ unsigned long long sm[40];
	const uint64_t n = min((uint64_t)g_max, (uint64_t)stats->cells);
	const uint64_t per = ((n + gridDim.x - 1) / gridDim.x + kCsTile - 1) / kCsTile * kCsTile;
	const uint64_t lo = min(n, (uint64_t)blockIdx.x * per), hi = min(n, lo + per);
	unsigned long long part = 0;
	for (uint64_t i0 = lo + threadIdx.x; i0 < hi; i0 += 8 * kCsNT) {  // 8 loads in flight
		uint32_t v[8];
#pragma unroll
		for (int q = 0; q < 8; q++) v[q] = i0 + q * kCsNT < hi ? counts[i0 + q * kCsNT] : 0u;
#pragma unroll
		for (int q = 0; q < 8; q++) part += v[q];
	}
	unsigned long long total;
	(void)block_excl_scan<unsigned long long, kCsNT>(part, sm, &total);
	if (threadIdx.x == 0) bsum[blockIdx.x] = total;
	grid_barrier(reinterpret_cast<GridBarrier *>(stats->bar_scan), &stats->err);
	unsigned long long before = 0;
	for (uint32_t j = threadIdx.x; j < blockIdx.x; j += kCsNT) before += __ldcg(bsum + j);
	unsigned long long run_total;
	(void)block_excl_scan<unsigned long long, kCsNT>(before, sm, &run_total);
	for (uint64_t t0 = lo; t0 < hi; t0 += kCsTile) {
		const uint64_t i = t0 + (uint64_t)threadIdx.x * kCsIPT;
		uint32_t v[kCsIPT] = {0u, 0u, 0u, 0u};
		const bool full = i + kCsIPT <= hi;
		if (full) {
			const uint4 q = *reinterpret_cast<const uint4 *>(counts + i);
			v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
			*reinterpret_cast<uint4 *>(counts + i) = make_uint4(0u, 0u, 0u, 0u);
		} else {
#pragma unroll
			for (int j = 0; j < kCsIPT; j++)
				if (i + j < hi) {
					v[j] = counts[i + j];
					counts[i + j] = 0u;
				}
		}
		unsigned long long tile_total;
		const unsigned long long excl =
		    block_excl_scan<unsigned long long, kCsNT>((unsigned long long)v[0] + v[1] + v[2] + v[3], sm, &tile_total);
		uint32_t o[kCsIPT];
		unsigned long long r = run_total + excl;
#pragma unroll
		for (int j = 0; j < kCsIPT; j++) {
			o[j] = (uint32_t)r;
			r += v[j];
		}
		if (full) {
			*reinterpret_cast<uint4 *>(start + i) = make_uint4(o[0], o[1], o[2], o[3]);
		} else {
#pragma unroll
			for (int j = 0; j < kCsIPT; j++)
				if (i + j < hi) start[i + j] = o[j];
		}
		if (cs) {
#pragma unroll
			for (int j = 0; j < kCsIPT; j++)
				if (i + j < hi) cs[i + j] = (unsigned long long)o[j] << 32;
		}
		run_total += tile_total;
	}
	// the block whose chunk ends the counts (block 0 when there are none)
	// writes the end offset and the entry total
	if (threadIdx.x == 0 && hi == n && (lo < hi || (n == 0 && blockIdx.x == 0))) {
		start[n] = (uint32_t)run_total;
		stats->entries = run_total;
	}
}

void launch_scan_cells(const BpBuffers &b, uint32_t g_max, cudaStream_t s) {
	// the scan leaves the counts zeroed: they are the scatter's cursors
	if (b.scan_bsum) {
		static const int per_sm = [] {
			int v = 0;
			if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_scan_cells_coop, kCsNT, 0) != cudaSuccess || v < 1) v = 1;
			return v;
		}();
		const unsigned grid = (unsigned)std::max<uint64_t>(
		    1, std::min<uint64_t>((uint64_t)g_max / (8 * kCsTile), std::min<uint64_t>((uint64_t)per_sm * kNumSMs,
		                                                                               kScanCoopBlocks)));
		DevStats *st = b.stats;
		uint32_t gm = g_max, *cnt = b.cell_count, *start = b.cell_start;
		unsigned long long *bs = b.scan_bsum, *cs = b.cell_cs;
		void *args[] = {&st, &gm, &cnt, &start, &bs, &cs};
		cudaLaunchCooperativeKernel((const void *)k_scan_cells_coop, dim3(grid), dim3(kCsNT), args, 0, s);
		return;
	}
	launch_scan_u32_to_u32(b.cell_count, g_max, b.cell_start, b.status, b.ticket, &b.stats->err, s, &b.stats->cells,
	                       &b.stats->entries, b.pre_zeroed, b.cell_count);
}

void launch_scatter(uint64_t n, const float *aabb, const BpBuffers &b, cudaStream_t s, bool packed) {
	if (!n) return;
	unsigned long long *cs = packed ? b.cell_cs : nullptr;
	if (b.sm.plans)
		launch_pdl(k_scatter<true>, dim3(blocks_for(n)), dim3(kNT), 0, s, n, aabb, b.stats, b.cell_start, b.cell_count,
		           b.entries, b.entry_cap, &b.stats->err, b.sm, cs);
	else
		launch_pdl(k_scatter<false>, dim3(blocks_for(n)), dim3(kNT), 0, s, n, aabb, b.stats, b.cell_start, b.cell_count,
		           b.entries, b.entry_cap, &b.stats->err, b.sm, cs);
}

template <bool kBatch, int kWin>
void pair_test_as(const BpBuffers &b, unsigned grid, cudaStream_t s) {
	launch_pdl((k_pair_test<kBatch, kWin>), dim3(grid), dim3(kNT), 0, s, b.stats, b.cell_start, b.entries, b.entry_cap, b.owner_count,
	                                               b.pairs_tmp, b.pair_cap, &b.stats->pairs, b.sm, b.dense,
	                                               b.dense_cap, &b.stats->dense_items, &b.stats->err, b.dense_cell,
	                                               b.owner_shift);
}
template <bool kBatch>
void pair_test_window(const BpBuffers &b, unsigned grid, cudaStream_t s) {
	switch (b.pair_window) {
	case 64: pair_test_as<kBatch, 64>(b, grid, s); break;
	case 128: pair_test_as<kBatch, 128>(b, grid, s); break;
	default: pair_test_as<kBatch, kWinDefault>(b, grid, s); break;
	}
}

void launch_pair_test(uint64_t n, const BpBuffers &b, uint64_t entries_hint, cudaStream_t s) {
	(void)n;
	uint64_t want = (entries_hint + kNT - 1) / kNT;
	const uint64_t per_sm = b.pair_blocks_per_sm > 0 ? (uint64_t)b.pair_blocks_per_sm : 8;
	unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(want, 1), (uint64_t)kNumSMs * per_sm);
	if (b.sm.plans)
		pair_test_window<true>(b, grid, s);
	else
		pair_test_window<false>(b, grid, s);
	launch_pair_test_dense(b, s);
}


void launch_pair_test_dense(const BpBuffers &b, cudaStream_t s) {
	if (!b.dense || !b.dense_cap) return;
	// persistent blocks over the device-side item count (41 KB of shared memory each)
	const unsigned grid = kNumSMs * 4;
	if (b.sm.plans)
		launch_pdl(k_pair_test_dense<true>, dim3(grid), dim3(kNT), 0, s, b.stats, b.cell_start, b.entries, b.entry_cap, b.owner_count,
		                                             b.pairs_tmp, b.pair_cap, &b.stats->pairs, b.sm, b.dense,
		                                             b.dense_cap, b.owner_shift);
	else
		launch_pdl(k_pair_test_dense<false>, dim3(grid), dim3(kNT), 0, s, b.stats, b.cell_start, b.entries, b.entry_cap, b.owner_count,
		                                              b.pairs_tmp, b.pair_cap, &b.stats->pairs, b.sm, b.dense,
		                                              b.dense_cap, b.owner_shift);
}

void launch_scan_owner(uint64_t n, const BpBuffers &b, cudaStream_t s) {
	launch_scan_u32_to_u64(b.owner_count, owner_buckets(n, b.owner_shift), b.owner_off, b.status2 ? b.status2 : b.status,
	                       b.ticket2 ? b.ticket2 : b.ticket, &b.stats->err, s, nullptr, nullptr, b.pre_zeroed);
}

void launch_owner_scatter(uint64_t out_cap, unsigned long long *out, const BpBuffers &b, cudaStream_t s) {
	const uint64_t bound = std::min<uint64_t>(b.pair_cap, out_cap);
	const unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(blocks_for(bound), 1), (uint64_t)kNumSMs * 8);
	launch_pdl(k_owner_scatter, dim3(grid), dim3(kNT), 0, s, b.stats, b.pair_cap, out_cap, b.pairs_tmp, b.owner_off, b.owner_count, out,
	                                     b.owner_shift);
}

void launch_segsort(uint64_t n, unsigned long long *out, const BpBuffers &b, cudaStream_t s) {
	const uint64_t nbk = owner_buckets(n, b.owner_shift);
	launch_pdl(k_segsort, dim3(blocks_for(nbk)), dim3(kNT), 0, s, nbk, b.owner_off, out, b.big_list, b.big_cap, b.stats);
}

void launch_segsort_mid(unsigned long long *out, const BpBuffers &b, cudaStream_t s) {
	const KeyPack kp{b.owner_shift, b.key_bits};
	if (kp.shift)
		launch_pdl(k_segsort_mid<true>, dim3(kNumSMs * 6), dim3(kMidNT), 0, s, b.stats, b.big_cap, b.big_list, b.owner_off,
		           out, kp);
	else
		launch_pdl(k_segsort_mid<false>, dim3(kNumSMs * 6), dim3(kMidNT), 0, s, b.stats, b.big_cap, b.big_list, b.owner_off,
		           out, kp);
}
void launch_segsort_big(unsigned long long *out, const BpBuffers &b, cudaStream_t s) {
	static const bool attr = [] {
		return cudaFuncSetAttribute(k_segsort_big<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                            kBigSeg * (int)sizeof(uint32_t)) == cudaSuccess &&
		       cudaFuncSetAttribute(k_segsort_big<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                            kBigSeg * (int)sizeof(uint32_t)) == cudaSuccess;
	}();
	(void)attr;
	// 64 KB of shared memory a block: three blocks fit on an SM
	const KeyPack kp{b.owner_shift, b.key_bits};
	if (kp.shift)
		launch_pdl(k_segsort_big<true>, dim3(kNumSMs * 3), dim3(512), kBigSeg * sizeof(uint32_t), s, b.stats, b.big_cap,
		           b.big_list, b.owner_off, out, kp);
	else
		launch_pdl(k_segsort_big<false>, dim3(kNumSMs * 3), dim3(512), kBigSeg * sizeof(uint32_t), s, b.stats, b.big_cap,
		           b.big_list, b.owner_off, out, kp);
}

bool fused_sort_fits(uint64_t buckets) { return buckets >= 1 && buckets <= kFusedBuckets; }
bool fused_sort_enabled() {
	static const bool on = [] {
		const char *v = getenv("CC_FUSED_SORT");
		return !(v && v[0] == '0');
	}();
	return on;
}

void launch_owner_sort_fused(uint64_t n, uint64_t out_cap, unsigned long long *out, uint64_t P_hint, const BpBuffers &b,
                             cudaStream_t s) {
	const uint32_t nbk = (uint32_t)owner_buckets(n, b.owner_shift);
	const size_t smem = sizeof(uint32_t) * ((size_t)nbk + 1 + kFusedSeg);
	static const int per_sm = [] {
		int v = 0;
		const int most = (int)(sizeof(uint32_t) * ((size_t)kFusedBuckets + 1 + kFusedSeg));
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_owner_sort_fused<true>, kFusedNT, most) != cudaSuccess || v < 1)
			v = 1;
		return v;
	}();
	const uint64_t want = (std::max<uint64_t>(P_hint, nbk) + kFusedNT - 1) / kFusedNT;
	unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)per_sm * kNumSMs));
	uint64_t pair_cap = b.pair_cap;
	const unsigned long long *tmp = b.pairs_tmp;
	const uint32_t *cnt = b.owner_count;
	uint32_t *cur = b.owner_cursor;
	int oshift = b.owner_shift;
	KeyPack kp{b.owner_shift, b.key_bits};
	DevStats *st = b.stats;
	void *args[] = {&st, &pair_cap, &out_cap, &tmp, &cnt, &cur, (void *)&nbk, &out, &oshift, &kp};
	const void *k = kp.shift ? (const void *)k_owner_sort_fused<true> : (const void *)k_owner_sort_fused<false>;
	cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kFusedNT), args, smem, s);
}

void launch_ref_count(uint64_t n, const float *aabb_shifted, const DevStats *stats, uint32_t *cnt, cudaStream_t s) {
	if (n) k_ref_count<<<blocks_for(n), kNT, 0, s>>>(n, aabb_shifted, stats, cnt);
}
void launch_ref_emit(uint64_t n, const float *aabb_shifted, DevStats *stats, const unsigned long long *off,
                     unsigned long long *keys, uint64_t cap, cudaStream_t s) {
	if (n) k_ref_emit<<<blocks_for(n), kNT, 0, s>>>(n, aabb_shifted, stats, off, keys, cap);
}
void launch_ref_flags(const unsigned long long *keys, uint64_t E, uint32_t *flags, cudaStream_t s) {
	if (E) k_ref_flags<<<blocks_for(E), kNT, 0, s>>>(keys, E, flags);
}
void launch_ref_split(const unsigned long long *keys, uint64_t E, const uint32_t *run_pos, uint32_t *bin_number,
                      uint32_t *body_number, uint32_t *active_bins, uint32_t *bin_end, uint64_t cap_a,
                      cudaStream_t s) {
	if (E)
		k_ref_split<<<blocks_for(E), kNT, 0, s>>>(keys, E, run_pos, bin_number, body_number, active_bins, bin_end,
		                                          cap_a);
}

}  // namespace cc
