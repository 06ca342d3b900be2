// interp.cu -- migration with a higher-order trace interpolator.
//
// The reference's NumbaKernel takes KernelConfig.interpolation_method and
// interpolates every sample with interpolate_sample (pstm/kernels/
// numba_cpu.py:341, pstm/kernels/interpolation.py:254-301): nearest,
// Catmull-Rom cubic, Hanning-windowed sinc of 4/8/16 points and Lanczos 3/5,
// the wide ones falling back to linear within their half-width of a trace end
// and normalising by the sum of their weights.  Linear interpolation stays on
// the tiled gather kernel; the other methods run here, in FP64 (traveltime,
// sample index, interpolation weights and accumulation), with one CTA of 128
// threads per (pillar, block of 128 output times) and the traces read from
// the packed geometry and the caller's panel.  Aperture, taper, weights, AA
// and fold are those of the gather kernel.
#include <cuda_runtime.h>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "migrate.cuh"
#include "ctx.h"

using namespace pstm;
using namespace pstm::ctx;

namespace {

template <int AMP>
__device__ inline double sample_at(const unsigned char *row, int64_t i) {
    return (double)amp_at<AMP>(row, (int)i);
}

__device__ inline double sinc_pi(double x) { return fabs(x) < 1e-10 ? 1.0 : sinpi(x) / (M_PI * x); }

// One interpolated sample at fractional index t (0 <= t < ns - 1 is checked by the caller).
template <int AMP>
__device__ double interpolate(const unsigned char *row, int ns, double t, int method) {
    if (method == PSTM_INTERP_NEAREST) {
        const int64_t i = (int64_t)(t + 0.5);
        return (i < 0 || i >= ns) ? 0.0 : sample_at<AMP>(row, i);
    }
    const int hw = method == PSTM_INTERP_SINC4 ? 2 : method == PSTM_INTERP_SINC8 ? 4
                 : method == PSTM_INTERP_SINC16 ? 8 : method == PSTM_INTERP_LANCZOS3 ? 3
                 : method == PSTM_INTERP_LANCZOS5 ? 5 : 0;
    const bool cubic_edge = method == PSTM_INTERP_CUBIC && (t < 1.0 || t >= (double)(ns - 2));
    const bool wide_edge = hw > 0 && (t < (double)hw || t >= (double)(ns - hw));
    if (method == PSTM_INTERP_LINEAR || cubic_edge || wide_edge || (method != PSTM_INTERP_CUBIC && hw == 0)) {
        const int64_t i0 = (int64_t)t;
        const double f = t - (double)i0;
        return sample_at<AMP>(row, i0) * (1.0 - f) + sample_at<AMP>(row, i0 + 1) * f;
    }
    if (method == PSTM_INTERP_CUBIC) {   // Catmull-Rom
        const int64_t i = (int64_t)t;
        const double u = t - (double)i;
        const double p0 = sample_at<AMP>(row, i - 1), p1 = sample_at<AMP>(row, i);
        const double p2 = sample_at<AMP>(row, i + 1), p3 = sample_at<AMP>(row, i + 2);
        const double c3 = -0.5 * p0 + 1.5 * p1 - 1.5 * p2 + 0.5 * p3;
        const double c2 = p0 - 2.5 * p1 + 2.0 * p2 - 0.5 * p3;
        const double c1 = -0.5 * p0 + 0.5 * p2;
        return ((c3 * u + c2) * u + c1) * u + p1;
    }
    const bool lanczos = method == PSTM_INTERP_LANCZOS3 || method == PSTM_INTERP_LANCZOS5;
    const int64_t ic = lanczos ? (int64_t)t : (int64_t)(t + 0.5);
    const double frac = t - (double)ic;
    double acc = 0.0, norm = 0.0;
    for (int k = -hw + 1; k <= hw; ++k) {
        const int64_t i = ic + k;
        if (i < 0 || i >= ns) continue;   // (sinc rounds to the nearest sample: ic + hw can reach ns)
        const double x = frac - (double)k;
        double w;
        if (lanczos) w = fabs(x) < 1e-10 ? 1.0 : (fabs(x) >= hw ? 0.0 : sinc_pi(x) * sinc_pi(x / hw));
        else w = sinc_pi(x) * (fabs(x) >= hw ? 0.0 : 0.5 * (1.0 + cospi(x / hw)));
        acc += sample_at<AMP>(row, i) * w;
        norm += w;
    }
    return norm > 1e-10 ? acc / norm : 0.0;
}

template <int TT>
__device__ inline double tt_of(double t0, double ds2, double dr2, double v, double eta, double v0, double k) {
    return traveltime_fp64<TT>(t0, ds2, dr2, v, eta, v0, k);
}

template <int AMP>
__global__ void __launch_bounds__(128) migrate_interp_kernel(const KParams P, int tt, int method) {
    const int p = blockIdx.x;
    const int ix = p / P.ny, iy = p - ix * P.ny;
    const double ox = P.xg ? P.xg[p] : P.xa[ix], oy = P.yg ? P.yg[p] : P.ya[iy];
    const int t = blockIdx.y * blockDim.x + threadIdx.x;
    const bool tv = t < P.nt;
    const int tc = tv ? t : P.nt - 1;
    const double t0 = P.ta[tc] / 1000.0;
    const double v = P.vel3d ? P.vrms[(int64_t)p * P.nt + tc] : P.vrms[tc];
    double eta = P.eta_const;
    if (P.eta) eta = P.eta3d ? P.eta[(int64_t)p * P.nt + tc] : P.eta[tc];
    double ap = v * t0 * 0.5 * P.tan_dip;
    ap = ap < P.min_ap ? P.min_ap : (ap > P.max_ap ? P.max_ap : ap);
    double vw = v;   // weights use v_rms, or v(z) at the image depth for curved rays
    if (P.curved_kind) {
        const double z = P.cr_k_zero ? P.cr_v0 * (t0 * 0.5) : (P.cr_v0 / P.cr_k) * (exp(P.cr_k * (t0 * 0.5)) - 1.0);
        vw = P.cr_v0 + P.cr_k * z;
    }
    const double gmax = P.aa_gmax, fdom = P.aa_fdom;
    const double taper_start = ap * (1.0 - P.taper);
    double acc = 0.0;
    int cnt = 0;
    for (int64_t tr = 0; tr < P.n_traces; ++tr) {
        const double *g = P.geo + tr * kGeoDoubles;
        const double dxm = ox - g[4], dym = oy - g[5];
        const double d2 = dxm * dxm + dym * dym;
        cnt += d2 <= P.fold_d2_max;
        const double d = sqrt(d2);
        const bool act = tv && !(d > ap);
        if (!__any_sync(0xffffffffu, act)) continue;
        if (!act) continue;
        const double dxs = ox - g[0], dys = oy - g[1], dxr = ox - g[2], dyr = oy - g[3];
        const double ds2 = dxs * dxs + dys * dys, dr2 = dxr * dxr + dyr * dyr;
        double T;
        switch (tt) {
        case TT_CURVED: T = tt_of<TT_CURVED>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
        case TT_VTI: T = tt_of<TT_VTI>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
        case TT_CURVED_VTI: T = tt_of<TT_CURVED_VTI>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
        default: T = tt_of<TT_STRAIGHT>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
        }
        const double s = (T - P.tstart_s) / P.dt_s;
        if (!(s >= 0.0 && s < (double)(P.ns - 1))) continue;
        const unsigned char *row =
            reinterpret_cast<const unsigned char *>(P.amps) + (tr * P.amp_stride) * (int64_t)P.elem;
        const double amp = interpolate<AMP>(row, P.ns, s, method);
        double w = g[6];
        if (d > taper_start) w *= 0.5 * (1.0 + cospi((d - taper_start) / (ap - taper_start)));
        if (P.aa && T >= 0.001) {
            const double st = fmin(fmax(fabs(dxm), fabs(dym)) / (vw * T), 1.0);
            if (st >= 0.01) {
                const double fmx = fmin(vw / (4.0 * gmax * st), 500.0);
                w *= fmax(0.0, 1.0 - fdom / fmx);
            }
        }
        if (P.spreading && T > 0.001) w *= 1.0 / (vw * T);
        if (P.obliquity && T > 0.001) w *= t0 / T;
        acc += amp * w;
    }
    if (tv) {
        const int64_t idx = (int64_t)p * P.nt + t;
        if (P.image_f32) reinterpret_cast<float *>(P.image)[idx] += (float)acc;
        else reinterpret_cast<double *>(P.image)[idx] += acc;
        if (P.fold && P.fold3d) P.fold[idx] += cnt;
    }
    if (P.fold && !P.fold3d && blockIdx.y == 0 && threadIdx.x == 0) P.fold[p] += cnt;
}

}  // namespace

namespace pstm {
namespace ctx {
// Launch of the higher-order-interpolation kernel on a prepared tile.
int32_t launch_interp(Ctx *c, const TilePlan &tp, int method, const pstm_output_desc *out) {
    const dim3 grid((unsigned)((int64_t)out->nx * out->ny), (unsigned)((out->nt + 127) / 128));
    switch (tp.amp) {
    case PSTM_AMP_F32: migrate_interp_kernel<AMP_F32><<<grid, 128, 0, tp.L.stream>>>(tp.P, tp.tt, method); break;
    case PSTM_AMP_BF16: migrate_interp_kernel<AMP_BF16><<<grid, 128, 0, tp.L.stream>>>(tp.P, tp.tt, method); break;
    default: migrate_interp_kernel<AMP_F16><<<grid, 128, 0, tp.L.stream>>>(tp.P, tp.tt, method); break;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSTM_OK : cuda_fail(c, e, "interpolation migrate kernel launch");
}
}  // namespace ctx
}  // namespace pstm
