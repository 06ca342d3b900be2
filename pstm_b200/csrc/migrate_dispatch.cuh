// migrate_dispatch.cuh -- picks the kernel instantiation for one traveltime
// kind; each migrate_tt*.cu includes this with its own PSTM_TT so that the
// four kinds compile in parallel.
#pragma once
#include "migrate.cuh"

namespace pstm {

struct TileShape {
    int R;    // output times per lane
    int PB;   // pillars per CTA
    int C;    // traces per chunk
};

template <int TT, int AMP, bool VEL3D, bool AA>
static cudaError_t launch_shape(const KParams &P, const TileShape &sh, dim3 grid, cudaStream_t st) {
#define PSTM_LAUNCH(R_, PB_, C_)                                                              \
    if (sh.R == R_ && sh.PB == PB_ && sh.C == C_) {                                            \
        migrate_gather_kernel<TT, AMP, VEL3D, AA, R_, PB_, C_><<<grid, kThreads, 0, st>>>(P); \
        return cudaGetLastError();                                                             \
    }
    PSTM_LAUNCH(2, 8, 64)
    PSTM_LAUNCH(2, 4, 64)
#undef PSTM_LAUNCH
    return cudaErrorInvalidConfiguration;
}

template <int TT>
cudaError_t launch_migrate_tt(const KParams &P, int amp, bool vel3d, bool aa, const TileShape &sh,
                              dim3 grid, cudaStream_t st) {
#define PSTM_CASE(A_, V_, AA_) \
    if (amp == A_ && vel3d == V_ && aa == AA_) return launch_shape<TT, A_, V_, AA_>(P, sh, grid, st);
    PSTM_CASE(AMP_F32, false, false) PSTM_CASE(AMP_F32, false, true)
    PSTM_CASE(AMP_F32, true, false)  PSTM_CASE(AMP_F32, true, true)
    PSTM_CASE(AMP_BF16, false, false) PSTM_CASE(AMP_BF16, false, true)
    PSTM_CASE(AMP_BF16, true, false)  PSTM_CASE(AMP_BF16, true, true)
    PSTM_CASE(AMP_F16, false, false) PSTM_CASE(AMP_F16, false, true)
    PSTM_CASE(AMP_F16, true, false)  PSTM_CASE(AMP_F16, true, true)
#undef PSTM_CASE
    return cudaErrorInvalidValue;
}

}  // namespace pstm
