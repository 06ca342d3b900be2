// migrate_dispatch.cuh -- picks the kernel instantiation for one traveltime
// kind; each migrate_tt*.cu includes this with its own kind so that the four
// kinds compile in parallel.
#pragma once
#include "migrate.cuh"

namespace pstm {

struct TileShape {
    int R;     // output times per lane
    int PBG;   // pillars per warp group (a CTA has kWarpsP groups)
};

template <int TT, int AMP, bool VEL3D, bool AA, bool EXACT, int R, int PBG>
static cudaError_t launch_one(const KParams &P, const KParams *Pg, dim3 grid, size_t smem, cudaStream_t st) {
    auto kern = migrate_staged_kernel<TT, AMP, VEL3D, AA, EXACT, R, PBG>;
    static size_t configured = 0;   // dynamic shared memory opt-in, once per instantiation and size
    if (smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    kern<<<grid, kThreads, smem, st>>>(P, Pg);
    return cudaGetLastError();
}

template <int TT, int AMP, bool VEL3D, bool AA, bool EXACT>
static cudaError_t launch_shape(const KParams &P, const KParams *Pg, const TileShape &sh, dim3 grid, size_t smem,
                                cudaStream_t st) {
    if (sh.R == 2 && sh.PBG == 4) return launch_one<TT, AMP, VEL3D, AA, EXACT, 2, 4>(P, Pg, grid, smem, st);
    if (sh.R == 2 && sh.PBG == 8) return launch_one<TT, AMP, VEL3D, AA, EXACT, 2, 8>(P, Pg, grid, smem, st);
    return cudaErrorInvalidConfiguration;
}

template <int TT, bool EXACT>
static cudaError_t launch_prec(const KParams &P, const KParams *Pg, int amp, bool vel3d, bool aa,
                               const TileShape &sh, dim3 grid, size_t smem, cudaStream_t st) {
#define PSTM_CASE(A_, V_, AA_) \
    if (amp == A_ && vel3d == V_ && aa == AA_) return launch_shape<TT, A_, V_, AA_, EXACT>(P, Pg, sh, grid, smem, st);
    PSTM_CASE(AMP_F32, false, false) PSTM_CASE(AMP_F32, false, true)
    PSTM_CASE(AMP_F32, true, false)  PSTM_CASE(AMP_F32, true, true)
    PSTM_CASE(AMP_BF16, false, false) PSTM_CASE(AMP_BF16, false, true)
    PSTM_CASE(AMP_BF16, true, false)  PSTM_CASE(AMP_BF16, true, true)
    PSTM_CASE(AMP_F16, false, false) PSTM_CASE(AMP_F16, false, true)
    PSTM_CASE(AMP_F16, true, false)  PSTM_CASE(AMP_F16, true, true)
#undef PSTM_CASE
    return cudaErrorInvalidValue;
}

// exact: FP64 sample index (straight rays only); otherwise FP32 traveltime.
template <int TT>
cudaError_t launch_migrate_tt(const KParams &P, const KParams *Pg, int amp, bool vel3d, bool aa, bool exact,
                              const TileShape &sh, dim3 grid, size_t smem, cudaStream_t st) {
    if constexpr (TT == TT_STRAIGHT) {
        if (exact) return launch_prec<TT, true>(P, Pg, amp, vel3d, aa, sh, grid, smem, st);
    }
    return launch_prec<TT, false>(P, Pg, amp, vel3d, aa, sh, grid, smem, st);
}

}  // namespace pstm
