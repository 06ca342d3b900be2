// launch.h -- host-side launch descriptor of the gather kernels.  The kernel
// templates are instantiated only in migrate_k<kind>.cu; host files include
// this header, not the kernel source.
#pragma once
#include <cuda_runtime.h>

#include "pstm_cuda.h"
#include "kparams.h"

namespace pstm {

// One launch: the per-tile grid form (bins and items null: grid is (pillar
// blocks, time blocks)), the persistent form over `n_bins` outputs, or the
// persistent form over the segments of the scatter schedule (grid.x CTAs; grid.x == 0 asks
// for one CTA per SM times the occupancy).
struct Launch {
    dim3 grid = dim3(0, 1, 1);   // dim3's own default is (1, 1, 1)
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    const BinWork *bins = nullptr;
    int n_bins = 0;
    unsigned long long *counter = nullptr;
    // the scatter schedule instead of bins (persistent form; item count read on the device)
    ScatterWork scatter = {nullptr, nullptr, 0, 0};
    bool configure_only = false;   // persistent form: set the shared-memory opt-in,
    unsigned *ctas_out = nullptr;  // report the CTA count and launch nothing
};

template <int TT>
cudaError_t launch_migrate(const KParams &P, const KParams *Pg, int amp, bool vel3d, int prec, const Launch &L);
// each kind is instantiated in its own migrate_k<kind>.cu, nowhere else
extern template cudaError_t launch_migrate<TT_STRAIGHT>(const KParams &, const KParams *, int, bool, int,
                                                        const Launch &);
extern template cudaError_t launch_migrate<TT_CURVED>(const KParams &, const KParams *, int, bool, int,
                                                      const Launch &);
extern template cudaError_t launch_migrate<TT_VTI>(const KParams &, const KParams *, int, bool, int, const Launch &);
extern template cudaError_t launch_migrate<TT_CURVED_VTI>(const KParams &, const KParams *, int, bool, int,
                                                          const Launch &);

// prec (pstm_precision) selects the FP64 sample-index path, FP32 traveltime
// with FP64 trace-end re-decisions, or FP32 throughout.
inline cudaError_t launch_kind(int traveltime, const KParams &P, const KParams *Pg, int amp, bool vel3d, int prec,
                               const Launch &L) {
    switch (traveltime) {
    case PSTM_TT_STRAIGHT: return launch_migrate<TT_STRAIGHT>(P, Pg, amp, vel3d, prec, L);
    case PSTM_TT_CURVED: return launch_migrate<TT_CURVED>(P, Pg, amp, vel3d, prec, L);
    case PSTM_TT_VTI: return launch_migrate<TT_VTI>(P, Pg, amp, vel3d, prec, L);
    default: return launch_migrate<TT_CURVED_VTI>(P, Pg, amp, vel3d, prec, L);
    }
}

__global__ void pack_geometry(const KParams P, double *geo);
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab, double *btab, float4 *ttime,
                                double *ttimeA, double *ttimeV);
__global__ void store_params(const KParams P, KParams *dst);

// Work descriptors carried by value into store_bins (kernel parameters are
// limited to 4 KB).
constexpr int kBinsPerStore = 64;
struct BinStore {
    int32_t first, count;
    BinWork w[kBinsPerStore];
};
__global__ void store_bins(const BinStore b, BinWork *dst);

}  // namespace pstm
