// migrate_dispatch.cuh -- picks the kernel instantiation.  Every traveltime
// kind is instantiated in its own translation unit (migrate_k<kind>.cu) so
// that they compile in parallel.
#pragma once
#include "migrate.cuh"

namespace pstm {

template <int TT, int AMP, bool VEL3D, bool EXACT, bool W2>
static cudaError_t launch_w(const KParams &P, const KParams *Pg, dim3 grid, size_t smem, cudaStream_t st) {
    auto kern = migrate_kernel<TT, AMP, VEL3D, EXACT, W2>;
    static size_t configured = 0;   // dynamic shared memory opt-in, per instantiation
    if (smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    kern<<<grid, kThreads, smem, st>>>(P, Pg);
    return cudaGetLastError();
}

template <int TT, int AMP, bool VEL3D, bool EXACT>
static cudaError_t launch_one(const KParams &P, const KParams *Pg, dim3 grid, size_t smem, cudaStream_t st) {
    if (P.spreading && P.obliquity) return launch_w<TT, AMP, VEL3D, EXACT, true>(P, Pg, grid, smem, st);
    return launch_w<TT, AMP, VEL3D, EXACT, false>(P, Pg, grid, smem, st);
}

template <int TT, bool EXACT>
static cudaError_t launch_prec(const KParams &P, const KParams *Pg, int amp, bool vel3d, dim3 grid, size_t smem,
                               cudaStream_t st) {
#define PSTM_CASE(A_, V_) \
    if (amp == A_ && vel3d == V_) return launch_one<TT, A_, V_, EXACT>(P, Pg, grid, smem, st);
    PSTM_CASE(AMP_F32, false) PSTM_CASE(AMP_F32, true)
    PSTM_CASE(AMP_BF16, false) PSTM_CASE(AMP_BF16, true)
    PSTM_CASE(AMP_F16, false) PSTM_CASE(AMP_F16, true)
#undef PSTM_CASE
    return cudaErrorInvalidValue;
}

// exact: FP64 sample index (straight rays only); otherwise FP32 traveltime.
template <int TT>
cudaError_t launch_migrate(const KParams &P, const KParams *Pg, int amp, bool vel3d, bool exact, dim3 grid,
                           size_t smem, cudaStream_t st) {
    if constexpr (TT == TT_STRAIGHT) {
        if (exact) return launch_prec<TT, true>(P, Pg, amp, vel3d, grid, smem, st);
    }
    return launch_prec<TT, false>(P, Pg, amp, vel3d, grid, smem, st);
}

}  // namespace pstm
