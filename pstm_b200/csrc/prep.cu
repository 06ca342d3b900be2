// prep.cu -- per-(pillar|0, time) tables for the gather kernel.
#include "launch.h"
#include "migrate.cuh"

namespace pstm {

// Per-(pillar or 0, output time): {1/v^2, aperture, 1/v, eta} and 1/(v dt)^2;
// per output time: {t0h2, Kt, tg, tguard}, {vz, vz2, 1/vz, t0 == 0},
// (t0/(2 dt))^2 and (curved kinds, when ttimeV is given) v(z) in FP64.
// Evaluated in FP64 as numba_cpu_optimized.py:378-399 does; the float4s are
// rounded once to FP32.
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab, double *btab, float4 *ttime,
                                double *ttimeA, double *ttimeV) {
    const int64_t n = n_p * P.nt;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / P.nt;
        const int t = (int)(i - p * P.nt);
        const double v = P.vel3d ? P.vrms[p * P.nt + t] : P.vrms[t];
        const double t0 = P.ta[t] / 1000.0;
        double ap = v * t0 * 0.5 * P.tan_dip;
        if (ap < P.min_ap) ap = P.min_ap;
        else if (ap > P.max_ap) ap = P.max_ap;
        double eta = P.eta_const;
        if (P.eta) eta = P.eta3d ? P.eta[p * P.nt + t] : P.eta[t];
        tab[i] = make_float4((float)(1.0 / (v * v)), (float)ap, (float)(1.0 / v), (float)eta);
        btab[i] = 1.0 / (v * v * P.dt_s * P.dt_s);
        if (p == 0) {
            const double tu = P.exact_units ? P.dt_s : 1.0;
            const double tguard = 0.001 / tu;
            // straight rays and VTI have T >= t0, so only t0 < 1.1 ms can give T <= 1 ms;
            // the curved-ray leg of the reference tends to 0 at large offsets
            const bool small_t = P.curved_kind || t0 < 0.0011;
            float vz = 0.f, vz2 = 0.f, ivwc = 0.f;
            if (P.curved_kind) {
                const double z = P.cr_k_zero ? P.cr_v0 * (t0 * 0.5)
                                             : (P.cr_v0 / P.cr_k) * (exp(P.cr_k * (t0 * 0.5)) - 1.0);
                const double vzd = P.cr_v0 + P.cr_k * z;
                vz = (float)vzd;
                vz2 = (float)(vzd * vzd);
                ivwc = (float)(1.0 / vzd);
                if (ttimeV) ttimeV[t] = vzd;
            }
            ttime[2 * t] = make_float4((float)((t0 * 0.5) * (t0 * 0.5)), P.obliquity ? (float)(t0 / tu) : 1.f,
                                       small_t ? (float)tguard : -1.f, (float)tguard);
            // w: 0 for t0 > 0; 1 for t0 = 0; 2 (3) for t0 = 0 where every T is exactly 0 and
            // the FP64 sample index of T = 0 lies inside (outside) the trace
            float w = 0.f;
            if (!(t0 > 0.0)) {
                const double s0 = (0.0 - P.tstart_s) / P.dt_s;
                w = P.t0_zero_exact ? ((s0 >= 0.0 && s0 < (double)(P.ns - 1)) ? 2.f : 3.f) : 1.f;
            }
            ttime[2 * t + 1] = make_float4(vz, vz2, ivwc, w);
            const double th = t0 * 0.5 / P.dt_s;
            ttimeA[t] = fmax(th * th, 1e-20);   // keeps the FP64 legs > 0 at t0 = 0
        }
    }
}

// Packed FP64 trace geometry for the bulk copies: kGeoDoubles per trace,
// sx sy rx ry mx my w 0 (w = 1 when the caller gives no weights).
__global__ void pack_geometry(const KParams P, double *geo) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P.n_traces;
         i += (int64_t)gridDim.x * blockDim.x) {
        double *g = geo + i * kGeoDoubles;
        g[0] = P.sx[i];
        g[1] = P.sy[i];
        g[2] = P.rx[i];
        g[3] = P.ry[i];
        g[4] = P.mx[i];
        g[5] = P.my[i];
        g[6] = P.w ? P.w[i] : 1.0;
        g[7] = 0.0;
    }
}

// Writes the launch parameters to device memory (the kernels' rare FP64 paths
// read them there).  A kernel rather than a copy from host memory, so that it
// can be captured in a CUDA graph and needs no staging buffer.
__global__ void store_params(const KParams P, KParams *dst) {
    const unsigned *src = reinterpret_cast<const unsigned *>(&P);
    unsigned *d = reinterpret_cast<unsigned *>(dst);
    for (unsigned i = threadIdx.x; i < sizeof(KParams) / 4; i += blockDim.x) d[i] = src[i];
}

// Writes up to kBinsPerStore work descriptors of the persistent form to
// device memory; their values travel as kernel parameters (graph-capturable).
__global__ void store_bins(const BinStore b, BinWork *dst) {
    for (int i = threadIdx.x; i < b.count; i += blockDim.x) dst[b.first + i] = b.w[i];
}

}  // namespace pstm
