// migrate_dispatch.cuh -- picks the kernel instantiation.  Every traveltime
// kind is instantiated in its own translation unit (migrate_k<kind>.cu) so
// that they compile in parallel.
#pragma once
#include <mutex>

#include "launch.h"
#include "migrate.cuh"

namespace pstm {

// Dynamic shared-memory opt-in of one kernel.  cudaFuncSetAttribute applies to
// the calling thread's current device only, so the size set so far is kept per
// device; the mutex orders host threads that launch concurrently.
struct SmemOptIn {
    static constexpr int kMaxDevices = 64;
    std::mutex mu;
    size_t configured[kMaxDevices] = {};
};

template <typename Kernel>
static cudaError_t opt_in_smem(SmemOptIn &state, Kernel kern, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;   // within the default limit
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= SmemOptIn::kMaxDevices)
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    std::lock_guard<std::mutex> lock(state.mu);
    if (smem <= state.configured[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) state.configured[dev] = smem;
    return e;
}

template <int TT, int AMP, bool VEL3D, bool EXACT, bool W2, bool GUARD>
static cudaError_t launch_w(const KParams &P, const KParams *Pg, const Launch &L) {
    if (!L.bins && !L.scatter.boxes) {
        auto kern = migrate_kernel<TT, AMP, VEL3D, EXACT, W2, GUARD>;
        static SmemOptIn opt_in;   // per instantiation
        cudaError_t e = opt_in_smem(opt_in, kern, L.smem);
        if (e != cudaSuccess) return e;
        kern<<<L.grid, kThreads, L.smem, L.stream>>>(P, Pg);
        return cudaGetLastError();
    }
    auto kern = migrate_persistent_kernel<TT, AMP, VEL3D, EXACT, W2, GUARD>;
    static SmemOptIn opt_in;
    {
        cudaError_t e = opt_in_smem(opt_in, kern, L.smem);
        if (e != cudaSuccess) return e;
    }
    unsigned ctas = L.grid.x;
    if (ctas == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, L.smem);
        if (e != cudaSuccess) return e;
        ctas = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    }
    if (L.configure_only) {
        if (L.ctas_out) *L.ctas_out = ctas;
        return cudaSuccess;
    }
    kern<<<ctas, kThreads, L.smem, L.stream>>>(P, Pg, L.bins, L.n_bins, L.counter, L.scatter);
    return cudaGetLastError();
}

template <int TT, int AMP, bool VEL3D, bool EXACT, bool GUARD>
static cudaError_t launch_one(const KParams &P, const KParams *Pg, const Launch &L) {
    if (P.spreading && P.obliquity) return launch_w<TT, AMP, VEL3D, EXACT, true, GUARD>(P, Pg, L);
    return launch_w<TT, AMP, VEL3D, EXACT, false, GUARD>(P, Pg, L);
}

template <int TT, bool EXACT, bool GUARD>
static cudaError_t launch_prec(const KParams &P, const KParams *Pg, int amp, bool vel3d, const Launch &L) {
#define PSTM_CASE(A_, V_) \
    if (amp == A_ && vel3d == V_) return launch_one<TT, A_, V_, EXACT, GUARD>(P, Pg, L);
    PSTM_CASE(AMP_F32, false) PSTM_CASE(AMP_F32, true)
    PSTM_CASE(AMP_BF16, false) PSTM_CASE(AMP_BF16, true)
    PSTM_CASE(AMP_F16, false) PSTM_CASE(AMP_F16, true)
#undef PSTM_CASE
    return cudaErrorInvalidValue;
}

// prec: PSTM_PREC_EXACT the FP64 sample index; PSTM_PREC_FAST FP32 traveltime with
// FP64 re-decisions of the trace-end tests in a guard band; PSTM_PREC_FP32 FP32
// traveltime, sample index and trace-end tests (no guard band).
template <int TT>
cudaError_t launch_migrate(const KParams &P, const KParams *Pg, int amp, bool vel3d, int prec, const Launch &L) {
    if (prec == PSTM_PREC_EXACT) return launch_prec<TT, true, true>(P, Pg, amp, vel3d, L);
    if (prec == PSTM_PREC_FAST) return launch_prec<TT, false, true>(P, Pg, amp, vel3d, L);
    return launch_prec<TT, false, false>(P, Pg, amp, vel3d, L);
}

}  // namespace pstm
