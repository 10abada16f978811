// The narrowphase's exact variant: the MPR state machine of cc_mpr.cuh with
// the reference's arithmetic in double (world coordinates, every direction
// normalized as v / sqrt(v.v), the reference's operation order). This
// translation unit is compiled with -fmad=false, so every product and sum
// rounds separately, as in the reference's host build with real = double:
// contacts equal the FP64 oracle's, rounded to float on output.
#include "cc_mpr.cuh"

namespace cc {

namespace {
constexpr int kNT = 64;

__global__ void __launch_bounds__(kNT) k_mpr_exact(uint64_t P_cap, const unsigned long long *P_dev, uint64_t n,
                                                    const int32_t *__restrict__ T, const float *__restrict__ A,
                                                    const float *__restrict__ B, const float *__restrict__ C,
                                                    const float *__restrict__ R, const uint32_t *__restrict__ ID,
                                                    uint64_t nb, const uint8_t *__restrict__ active,
                                                    const float *__restrict__ pos, const float *__restrict__ rot,
                                                    float envelope, const long long *__restrict__ pairs,
                                                    NpScratch sc) {
	pdl_begin();
	mpr::run<double, true, kNT>(P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc,
	                            sc.classes + 2 * kNpClasses);
}
}  // namespace

int mpr_exact_resident_blocks() {
	static const int b = [] {
		int v = 0;
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_mpr_exact, kNT, 0) != cudaSuccess || v < 1) v = 1;
		return v;
	}();
	return b;
}

void launch_mpr_exact(unsigned grid, uint64_t P_cap, const unsigned long long *P_dev, uint64_t n, const int32_t *T,
                      const float *A, const float *B, const float *C, const float *R, const uint32_t *ID, uint64_t nb,
                      const uint8_t *active, const float *pos, const float *rot, float envelope,
                      const long long *pairs, const NpScratch &sc, cudaStream_t s) {
	launch_pdl(k_mpr_exact, dim3(grid), dim3(kNT), 0, s, P_cap, P_dev, n, T, A, B, C, R, ID, nb, active, pos, rot, envelope, pairs, sc);
}

}  // namespace cc
