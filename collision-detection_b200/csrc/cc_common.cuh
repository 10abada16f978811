// Shared device utilities for the collision kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cstdlib>
#include <utility>
#include <cuda_runtime.h>

namespace cc {

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs; grids are sized in multiples of it

// Device-side error bits, OR-ed into Workspace::err (read by the host after a
// call). A set bit makes the C ABI return an error status; it never traps.
enum DeviceError : uint32_t {
	kErrNonFinite = 1u << 0,     // NaN/Inf in an AABB corner
	kErrInverted = 1u << 1,      // min > max on some axis
	kErrSpinLimit = 1u << 2,     // a bounded wait gave up (look-back scan)
	kErrCapacity = 1u << 3,      // an output buffer was too small (sizes still reported)
	kErrSegmentTooLong = 1u << 4,  // a pair segment exceeded the block sort size (host falls back)
	kErrBinCount = 1u << 5,      // a body covers a negative / overflowing number of reference bins
	kErrBadIndex = 1u << 6,      // a body id >= nb or a pair index >= n (the access is skipped)
	kErrHashFull = 1u << 7,      // the overlapped narrowphase's contact hash overflowed (host redoes it in order)
};

// Order-preserving map float -> uint32 (for atomicMin/atomicMax reductions).
__device__ __forceinline__ uint32_t f2ord(float f) {
	uint32_t u = __float_as_uint(f);
	return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t k) {
	uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
	return __uint_as_float(u);
}
__host__ __device__ inline float ord2f_host(uint32_t k) {
	uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
	float f;
	memcpy(&f, &u, 4);
	return f;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// 16-byte global -> shared copy that bypasses the registers (cp.async, L2
// only); both addresses 16-byte aligned. cp_async_wait_all waits for this
// thread's copies; a __syncwarp/__syncthreads after it publishes them.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// n words global -> shared, every thread keeping 8 loads in flight (a plain
// strided loop waits for each load before issuing the next).
template <int NT>
__device__ __forceinline__ void copy_words_to_shared(uint32_t *dst, const uint32_t *__restrict__ src, uint32_t n) {
	for (uint32_t b0 = threadIdx.x; b0 < n; b0 += 8 * NT) {
		uint32_t v[8];
#pragma unroll
		for (int q = 0; q < 8; q++) {
			const uint32_t b = b0 + q * NT;
			v[q] = b < n ? src[b] : 0u;
		}
#pragma unroll
		for (int q = 0; q < 8; q++) {
			const uint32_t b = b0 + q * NT;
			if (b < n) dst[b] = v[q];
		}
	}
}

// 32-byte global accesses (sm_100 256-bit vector ld/st): one L2 request where
// two 16-byte accesses make two. The address must be 32-byte aligned.
__device__ __forceinline__ void st_global_v8(float *p, float4 a, float4 b) {
	asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x), "f"(a.y), "f"(a.z),
	             "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
	             : "memory");
}
__device__ __forceinline__ void ld_global_v8(const float *p, float4 &a, float4 &b) {
	asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
	             : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
	             : "l"(p)
	             : "memory");
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v) {
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		T t = __shfl_up_sync(0xffffffffu, v, o);
		if ((int)lane_id() >= o) v += t;
	}
	return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Block-wide exclusive scan of one value per thread. `sm` holds >= 32 T.
// Returns the exclusive prefix; *total receives the block sum.
template <class T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T *sm, T *total) {
	constexpr int NW = NT / 32;
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	T inc = warp_incl_scan(v);
	if (l == 31) sm[w] = inc;
	__syncthreads();
	if (w == 0) {
		T s = (l < NW) ? sm[l] : T(0);
		T si = warp_incl_scan(s);
		if (l < NW) sm[l] = si - s;
		if (l == NW - 1) sm[NW] = si;
	}
	__syncthreads();
	T r = sm[w] + inc - v;
	*total = sm[NW];
	__syncthreads();
	return r;
}

// ---------------------------------------------------------------------------
// Decoupled look-back (single pass) for 64-bit sums.
//
// Tile status word: bits 63..62 = state (0 empty, 1 aggregate, 2 prefix),
// bits 61..0 = value. The status array must be zeroed before the launch.
// Tiles take indices from an atomic ticket, so every predecessor a tile waits
// on has already started; each wait is still bounded and sets kErrSpinLimit
// (treating the missing value as 0) instead of spinning forever.
// ---------------------------------------------------------------------------
constexpr uint64_t kStAgg = 1ull << 62, kStPre = 2ull << 62, kStMask = (1ull << 62) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ void st_publish(uint64_t *status, uint32_t tile, uint64_t state, uint64_t v) {
	__stcg((unsigned long long *)(status + tile), (unsigned long long)(state | (v & kStMask)));
}

// Called by warp 0 of a tile with the tile aggregate; returns the exclusive
// prefix of the tile (valid in all lanes of warp 0).
__device__ __forceinline__ uint64_t lookback_prefix(uint64_t *status, uint32_t tile, uint64_t agg, uint32_t *err) {
	const int l = lane_id();
	if (tile == 0) {
		if (l == 0) st_publish(status, 0, kStPre, agg);
		return 0;
	}
	if (l == 0) st_publish(status, tile, kStAgg, agg);
	uint64_t excl = 0;
	int64_t base = (int64_t)tile - 1;
	int spins = 0;
	while (true) {
		int64_t idx = base - l;
		uint64_t s = 0;
		if (idx >= 0) {
			s = __ldcg((const unsigned long long *)(status + idx));
		} else {
			s = kStPre;  // virtual tile before 0 has prefix 0
		}
		uint32_t pre = __ballot_sync(0xffffffffu, (s >> 62) == 2);
		uint32_t empty = __ballot_sync(0xffffffffu, (s >> 62) == 0);
		// lanes up to and including the first prefix lane contribute
		int stop = pre ? (__ffs(pre) - 1) : 31;
		uint32_t need = (stop == 31) ? 0xffffffffu : ((1u << (stop + 1)) - 1u);
		if (empty & need) {
			if (++spins > kSpinLimit) {
				if (l == 0) atomicOr(err, (uint32_t)kErrSpinLimit);
				break;
			}
			__nanosleep(32);
			continue;
		}
		uint64_t v = (l <= stop) ? (s & kStMask) : 0;
		excl += warp_sum(v);
		if (pre) break;
		base -= 32;
	}
	if (l == 0) st_publish(status, tile, kStPre, excl + agg);
	return excl;
}

// ---------------------------------------------------------------------------
// Grid-wide barrier of a cooperative launch (cudaLaunchCooperativeKernel: every
// block is resident at once). `arrived` counts the blocks at the barrier; the
// last one resets it and bumps `gen`, which the others poll. Both words start
// at zero (they live in per-call state that is zeroed before the pass) and
// `arrived` is zero again after every completed barrier. The wait is bounded:
// after kSpinLimit polls it sets kErrSpinLimit and lets the block go on, so a
// broken launch returns an error status instead of hanging.
// ---------------------------------------------------------------------------
struct GridBarrier {
	unsigned int arrived;
	unsigned int gen;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
	unsigned int v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

__device__ __forceinline__ void grid_barrier(GridBarrier *b, uint32_t *err) {
	__syncthreads();
	if (threadIdx.x == 0) {
		const unsigned int g = ld_acquire_u32(&b->gen);  // before arriving: the gen this barrier bumps
		__threadfence();                                 // the block's writes before its arrival
		if (atomicAdd(&b->arrived, 1u) == gridDim.x - 1) {
			atomicExch(&b->arrived, 0u);
			__threadfence();
			atomicAdd(&b->gen, 1u);
		} else {
			int spins = 0;
			while (ld_acquire_u32(&b->gen) == g) {
				if (++spins > kSpinLimit) {
					atomicOr(err, (uint32_t)kErrSpinLimit);
					break;
				}
				__nanosleep(64);
			}
		}
		__threadfence();
	}
	__syncthreads();
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch. The pipeline's kernels are launched with
// programmatic stream serialization (launch_pdl): a kernel's blocks may be
// scheduled while the previous kernel of the stream is still finishing, so
// the launch and ramp-up of each stage overlap the tail of the one before.
// Every kernel launched this way calls pdl_begin() first: griddepcontrol.wait
// blocks until the preceding grid has completed and its writes are visible
// (a no-op when the launch had no programmatic dependency), and
// griddepcontrol.launch_dependents then lets the next kernel start launching
// once all of this grid's blocks have started. It pays where kernels are
// short (1M bodies: about 9 us a step) and cost time where they are long (the
// 16.7M clustered broadphase: 311 -> 330 ms), so a call enqueues with it only
// below kPdlMaxBodies bodies a pass (PdlScope). Environment CC_PDL=0 turns the
// attribute off everywhere (plain stream order), CC_PDL=2 on for every size.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_begin() {
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

inline int pdl_mode() {
	static const int m = [] {
		const char *v = getenv("CC_PDL");
		return v && v[0] == '0' ? 0 : (v && v[0] == '2' ? 2 : 1);
	}();
	return m;
}
constexpr uint64_t kPdlMaxBodies = (uint64_t)1 << 22;
// Whether this host thread's current call enqueues with the attribute (set by
// PdlScope at the start of a call, from its body count).
inline thread_local bool t_pdl_call = true;
struct PdlScope {
	bool was;
	explicit PdlScope(uint64_t bodies) : was(t_pdl_call) {
		t_pdl_call = pdl_mode() == 2 || (pdl_mode() == 1 && bodies < kPdlMaxBodies);
	}
	~PdlScope() { t_pdl_call = was; }
};
inline bool pdl_enabled() { return t_pdl_call && pdl_mode() != 0; }

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args) {
	if (!pdl_enabled()) {
		kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
		return;
	}
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Grid-stride zeroing of the ranges of a ZeroList (called by every thread of
// a pass's first kernel).
template <class ZL>
__device__ __forceinline__ void zero_ranges(const ZL &z) {
	const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, step = (uint64_t)gridDim.x * blockDim.x;
#pragma unroll
	for (int r = 0; r < 5; r++)
		for (uint64_t i = t; i < z.words[r]; i += step) z.p[r][i] = 0u;
}

}  // namespace cc
