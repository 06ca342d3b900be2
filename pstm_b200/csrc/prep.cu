// prep.cu -- per-(pillar|0, time) tables for the gather kernel.
#include "migrate.cuh"

namespace pstm {

// {1/v^2, aperture, 1/v, eta} and 1/(v dt)^2 per (pillar or 0, output time),
// evaluated in FP64 as numba_cpu_optimized.py:378-399 does; the float4 is
// rounded once to FP32.
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab, double *btab) {
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
    }
}

}  // namespace pstm
