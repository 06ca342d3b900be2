// interp.cu -- migration with a higher-order trace interpolator.
//
// The reference's NumbaKernel takes KernelConfig.interpolation_method and
// interpolates every sample with interpolate_sample (pstm/kernels/
// numba_cpu.py:341, pstm/kernels/interpolation.py:254-301): nearest,
// Catmull-Rom cubic, Hanning-windowed sinc of 4/8/16 points and Lanczos 3/5,
// the wide ones falling back to linear within their half-width of a trace end
// and normalising by the sum of their weights.  Linear interpolation stays on
// the tiled gather kernel; the other methods run here -- in FP64 (traveltime,
// sample index, interpolation weights and accumulation) on the exact path, with
// FP32 taps, interpolation and weights after the FP64 sample index on the fast
// path -- with one CTA of 128
// threads per (pillar, block of 128 output times) and the traces read from
// the packed geometry and the caller's panel.  Each warp stages the traces 32
// at a time in a shared-memory slice of its own: each lane takes one trace's
// pillar distances, counts it for the fold and keeps it if it lies inside the
// largest aperture of the warp's times; the kept traces, in trace order, go to
// the slice and every lane then runs them against its own output time.  Warps
// synchronise only with themselves, so none waits for a warp whose times
// keep more traces.  Aperture, taper, weights, AA and
// fold are those of the gather kernel.
#include <cuda_runtime.h>

#include <cstdint>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "migrate.cuh"
#include "ctx.h"

using namespace pstm;
using namespace pstm::ctx;

namespace {

constexpr int kInterpThreads = 128;
// CTAs per SM the register budget is sized for: the kernel is bound by
// dependent FP64 latency, so more resident warps beat the few values that
// spill to L1 at this budget.
#ifndef PSTM_INTERP_MIN_CTAS
#define PSTM_INTERP_MIN_CTAS 8
#endif

template <int AMP, typename R = double>
__device__ inline R sample_at(const unsigned char *row, int64_t i) {
    return (R)amp_at<AMP>(row, (int)i);
}

// sincospi in the interpolation arithmetic: FP64, or FP32 on the fast path.
__device__ inline void sincospi_r(double x, double *s, double *c) { sincospi(x, s, c); }
__device__ inline void sincospi_r(float x, float *s, float *c) { sincospif(x, s, c); }
// 1/x in the interpolation arithmetic: the hardware approximation refined by
// one Newton step in FP64 (~1 ulp), the approximation itself in FP32.
__device__ inline double rcp_r(double x) { return rcp_newton(x); }
__device__ inline float rcp_r(float x) { return rcp_approx(x); }

// Nearest, Catmull-Rom cubic and linear interpolation at fractional index t
// (0 <= t < ns - 1 is checked by the caller); linear also serves the wide
// methods within their half-width of a trace end.
// R is the arithmetic of the weights and taps: double (exact path) or float
// (fast path); the sample index t is FP64 in both.
template <int AMP, typename R>
__device__ R interpolate_narrow(const unsigned char *row, int ns, double t, int method) {
    if (method == PSTM_INTERP_NEAREST) {
        const int64_t i = (int64_t)(t + 0.5);
        return (i < 0 || i >= ns) ? R(0) : sample_at<AMP, R>(row, i);
    }
    if (method == PSTM_INTERP_CUBIC && t >= 1.0 && t < (double)(ns - 2)) {   // Catmull-Rom
        const int64_t i = (int64_t)t;
        const R u = (R)(t - (double)i);
        const R p0 = sample_at<AMP, R>(row, i - 1), p1 = sample_at<AMP, R>(row, i);
        const R p2 = sample_at<AMP, R>(row, i + 1), p3 = sample_at<AMP, R>(row, i + 2);
        const R c3 = R(-0.5) * p0 + R(1.5) * p1 - R(1.5) * p2 + R(0.5) * p3;
        const R c2 = p0 - R(2.5) * p1 + R(2.0) * p2 - R(0.5) * p3;
        const R c1 = R(-0.5) * p0 + R(0.5) * p2;
        return ((c3 * u + c2) * u + c1) * u + p1;
    }
    const int64_t i0 = (int64_t)t;
    const R f = (R)(t - (double)i0);
    return sample_at<AMP, R>(row, i0) * (R(1) - f) + sample_at<AMP, R>(row, i0 + 1) * f;
}

// Windowed sinc (LANCZOS false) or Lanczos (true) of half-width HW at
// fractional index t, normalised by the sum of the weights; linear within HW
// samples of a trace end.
//
// The taps need sin(pi x) and the sine or cosine of pi x / HW at x = frac - k,
// k = -HW+1 .. HW.  Since sin(pi (frac - k)) = (-1)^k sin(pi frac) and the
// window angle pi (frac - k) / HW moves by pi / HW from one tap to the next,
// a chain of window angles carried by rotations through (cos_d, sin_d) =
// (cos, sin)(pi / HW) gives every weight, and the factor sin(pi frac) common
// to all taps cancels in the normalisation.  A rotation
// adds about one rounding of a unit-sized value per tap (absolute 1e-15 after
// 16 taps), harmless where the window enters as 0.5 (1 + cos).  Lanczos
// divides sin(pi x / HW) by x, so it needs that sine accurate relative to its
// size near x = 0: it runs two chains, each started by its own sincospi at a
// tap beside x = 0 (k = 0 and k = 1) and carried outward.  The weights are
// otherwise those of the direct formulas: sinc(x) = sin(pi x) / (pi x) with 1
// for |x| < 1e-10, a Hann window 0.5 (1 + cos(pi x / HW)) that is 0 for
// |x| >= HW, Lanczos sinc(x) sinc(x / HW).
template <int AMP, int HW, bool LANCZOS, typename R>
__device__ R interpolate_wide(const unsigned char *row, int ns, double t, R cos_d, R sin_d) {
    if (t < (double)HW || t >= (double)(ns - HW)) {
        const int64_t i0 = (int64_t)t;
        const R f = (R)(t - (double)i0);
        return sample_at<AMP, R>(row, i0) * (R(1) - f) + sample_at<AMP, R>(row, i0 + 1) * f;
    }
    const int64_t ic = LANCZOS ? (int64_t)t : (int64_t)(t + 0.5);
    const R frac = (R)(t - (double)ic);
    // On a sample (|x| < 1e-10 at a tap: the tap's weight is 1 and the others'
    // sin(pi x) factors vanish) the interpolant is that sample.
    if (fabs(frac) < R(1e-10)) return sample_at<AMP, R>(row, ic);
    if (LANCZOS && fabs(frac - R(1)) < R(1e-10)) return sample_at<AMP, R>(row, ic + 1);
    // The factors common to every tap cancel in the normalisation, so they are
    // left out: sinc weights sin(pi x_k) / (pi x_k) * 0.5 (1 + cos w_k) with
    // sin(pi x_k) = (-1)^k sin(pi frac) become (-1)^k (1 + cos w_k) / x_k, and
    // Lanczos weights sin(pi x_k) sin(pi x_k / HW) HW / (pi^2 x_k^2) become
    // (-1)^k sin(pi x_k / HW) / x_k^2; one reciprocal per tap, no division.
    R acc = R(0), norm = R(0);
    auto tap = [&](int k, R sg, R s_w, R c_w) {
        const int64_t i = ic + k;
        if (i < 0 || i >= ns) return;   // (sinc rounds to the nearest sample: ic + HW can reach ns)
        const R x = frac - (R)k;
        const R rx = rcp_r(x);
        R w;
        if (LANCZOS) w = fabs(x) >= R(HW) ? R(0) : sg * s_w * rx * rx;
        else w = fabs(x) >= R(HW) ? R(0) : sg * (R(1) + c_w) * rx;
        acc += sample_at<AMP, R>(row, i) * w;
        norm += w;
    };
    if (!LANCZOS) {   // one chain, k = -HW+1 .. HW, window angle dropping by pi / HW per tap
        R s_w, c_w;
        sincospi_r((frac + (R)(HW - 1)) * (R(1) / (R)HW), &s_w, &c_w);
        R sg = ((HW - 1) & 1) ? R(-1) : R(1);
#pragma unroll
        for (int k = -HW + 1; k <= HW; ++k) {
            tap(k, sg, s_w, c_w);
            const R c_n = c_w * cos_d + s_w * sin_d;
            s_w = s_w * cos_d - c_w * sin_d;
            c_w = c_n;
            sg = -sg;
        }
    } else {          // k = 0, -1, .., -HW+1 (angle growing), then k = 1, .., HW (angle dropping)
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const R sin_a = side ? -sin_d : sin_d;
            R s_w, c_w;
            sincospi_r((frac - (R)side) * (R(1) / (R)HW), &s_w, &c_w);
            R sg = side ? R(-1) : R(1);
#pragma unroll
            for (int n = 0; n < HW; ++n) {
                tap(side ? 1 + n : -n, sg, s_w, c_w);
                const R c_n = c_w * cos_d - s_w * sin_a;
                s_w = s_w * cos_d + c_w * sin_a;
                c_w = c_n;
                sg = -sg;
            }
        }
    }
    return norm != R(0) ? acc * rcp_r(norm) : R(0);
}

template <int TT>
__device__ inline double tt_of(double t0, double ds2, double dr2, double v, double eta, double v0, double k) {
    return traveltime_fp64<TT>(t0, ds2, dr2, v, eta, v0, k);
}

// Per-trace values a warp stages in shared memory for the CTA's pillar.
struct Staged {
    double ds2[32], dr2[32], d[32], w[32], m[32];
    int tr[32];
};

// R: double on the exact path (FP64 end to end); float on the fast path,
// where only the traveltime, the sample index and the accumulation stay FP64
// and the taps, the interpolation and the weights are FP32.
template <int AMP, int HW, bool LANCZOS, typename R>
__global__ void __launch_bounds__(kInterpThreads, PSTM_INTERP_MIN_CTAS) migrate_interp_kernel(const KParams P, int tt, int method) {
    __shared__ Staged S_all[kInterpThreads / 32];
    const int p = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ix = p / P.ny, iy = p - ix * P.ny;
    const double ox = P.xg ? P.xg[p] : P.xa[ix], oy = P.yg ? P.yg[p] : P.ya[iy];
    const int t = blockIdx.y * kInterpThreads + threadIdx.x;
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
    const double inv_vw = 1.0 / vw;
    const double taper_start = ap * (1.0 - P.taper);
    const double inv_taper_w = ap > taper_start ? 1.0 / (ap - taper_start) : 0.0;
    const double iv2 = 1.0 / (v * v), t0h2 = (t0 * 0.5) * (t0 * 0.5), inv_dt = 1.0 / P.dt_s;
    R sin_d = R(0), cos_d = R(1);
    if (HW > 0) sincospi_r(R(1) / (R)HW, &sin_d, &cos_d);

    Staged &S = S_all[warp];
    // Largest aperture over the warp's output times: a trace farther than it
    // from the pillar adds nothing at any of them.
    double ap_w = tv ? ap : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ap_w = fmax(ap_w, __shfl_xor_sync(0xffffffffu, ap_w, o));

    double acc = 0.0;
    int cnt = 0;   // traces within the fold radius; the same in every lane
    for (int64_t c0 = 0; c0 < P.n_traces; c0 += 32) {
        const int64_t tr = c0 + lane;
        bool keep = false, in_fold = false;
        double dxm = 0.0, dym = 0.0, d = 0.0;
        const double *g = P.geo + tr * kGeoDoubles;
        if (tr < P.n_traces) {
            dxm = ox - g[4];
            dym = oy - g[5];
            const double d2 = dxm * dxm + dym * dym;
            in_fold = d2 <= P.fold_d2_max;
            d = sqrt(d2);
            keep = !(d > ap_w);
        }
        const unsigned kb = __ballot_sync(0xffffffffu, keep);
        cnt += __popc(__ballot_sync(0xffffffffu, in_fold));
        const int n_kept = __popc(kb);
        if (keep) {
            const int j = __popc(kb & ((1u << lane) - 1u));
            const double dxs = ox - g[0], dys = oy - g[1], dxr = ox - g[2], dyr = oy - g[3];
            S.ds2[j] = dxs * dxs + dys * dys;
            S.dr2[j] = dxr * dxr + dyr * dyr;
            S.d[j] = d;
            S.w[j] = g[6];
            S.m[j] = fmax(fabs(dxm), fabs(dym));
            S.tr[j] = (int)tr;
        }
        __syncwarp();
        for (int j = 0; j < n_kept; ++j) {
            const double dj = S.d[j];
            if (!tv || dj > ap) continue;
            const double ds2 = S.ds2[j], dr2 = S.dr2[j];
            double T;
            switch (tt) {
            case TT_CURVED: T = tt_of<TT_CURVED>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
            case TT_VTI: T = tt_of<TT_VTI>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
            case TT_CURVED_VTI: T = tt_of<TT_CURVED_VTI>(t0, ds2, dr2, v, eta, P.cr_v0, P.cr_k); break;
            default:   // the straight legs with this thread's 1/v^2 and the Newton-refined sqrt
                T = sqrt_newton(fma(ds2, iv2, t0h2)) + sqrt_newton(fma(dr2, iv2, t0h2));
                break;
            }
            const double s = (T - P.tstart_s) * inv_dt;
            if (!(s >= 0.0 && s < (double)(P.ns - 1))) continue;
            const unsigned char *row =
                reinterpret_cast<const unsigned char *>(P.amps) + ((int64_t)S.tr[j] * P.amp_stride) * (int64_t)P.elem;
            R amp;
            if (HW > 0) amp = interpolate_wide<AMP, HW, LANCZOS, R>(row, P.ns, s, cos_d, sin_d);
            else amp = interpolate_narrow<AMP, R>(row, P.ns, s, method);
            R w = (R)S.w[j];
            if (dj > taper_start) {
                const R x = (R)((dj - taper_start) * inv_taper_w);
                R cw;
                if constexpr (sizeof(R) == 8) cw = cospi(x);
                else cw = cospif(x);
                w *= R(0.5) * (R(1) + cw);
            }
            // One reciprocal of T per pair and 1/v per thread serve the AA,
            // spreading and obliquity terms: sin = m / (v T), f_max = min(v /
            // (4 gmax sin), 500 Hz) so f_dom / f_max = f_dom max(4 gmax sin / v,
            // 1 / 500), spreading 1 / (v T), obliquity t0 / T.
            const R Tr = (R)T, inv_T = rcp_r(Tr), ivw = (R)inv_vw;
            if (P.aa && T >= 0.001) {
                const R st = fmin((R)S.m[j] * inv_T * ivw, R(1));
                if (st >= R(0.01))
                    w *= fmax(R(0), R(1) - (R)fdom * fmax(R(4) * (R)gmax * st * ivw, R(1) / R(500)));
            }
            if (P.spreading && T > 0.001) w *= inv_T * ivw;
            if (P.obliquity && T > 0.001) w *= (R)t0 * inv_T;
            acc += (double)(amp * w);
        }
        __syncwarp();   // the next batch overwrites the staged values
    }
    if (tv) {
        const int64_t idx = (int64_t)p * P.nt + t;
        if (P.image_f32) reinterpret_cast<float *>(P.image)[idx] += (float)acc;
        else reinterpret_cast<double *>(P.image)[idx] += acc;
        if (P.fold && P.fold3d) P.fold[idx] += cnt;
    }
    if (P.fold && !P.fold3d && blockIdx.y == 0 && threadIdx.x == 0) P.fold[p] += cnt;
}

template <int AMP, int HW, bool LANCZOS>
void launch_one(const TilePlan &tp, dim3 grid, int method) {
    if (tp.exact)
        migrate_interp_kernel<AMP, HW, LANCZOS, double><<<grid, kInterpThreads, 0, tp.L.stream>>>(tp.P, tp.tt, method);
    else
        migrate_interp_kernel<AMP, HW, LANCZOS, float><<<grid, kInterpThreads, 0, tp.L.stream>>>(tp.P, tp.tt, method);
}

template <int AMP>
void launch_method(const TilePlan &tp, dim3 grid, int method) {
    switch (method) {
    case PSTM_INTERP_SINC4: launch_one<AMP, 2, false>(tp, grid, method); break;
    case PSTM_INTERP_SINC8: launch_one<AMP, 4, false>(tp, grid, method); break;
    case PSTM_INTERP_SINC16: launch_one<AMP, 8, false>(tp, grid, method); break;
    case PSTM_INTERP_LANCZOS3: launch_one<AMP, 3, true>(tp, grid, method); break;
    case PSTM_INTERP_LANCZOS5: launch_one<AMP, 5, true>(tp, grid, method); break;
    default: launch_one<AMP, 0, false>(tp, grid, method); break;   // nearest, cubic, linear
    }
}

}  // namespace

namespace pstm {
namespace ctx {
// Launch of the higher-order-interpolation kernel on a prepared tile.
int32_t launch_interp(Ctx *c, const TilePlan &tp, int method, const pstm_output_desc *out) {
    if (tp.P.n_traces > INT32_MAX) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "interpolation kernel takes at most 2^31 - 1 traces");
    const dim3 grid((unsigned)((int64_t)out->nx * out->ny), (unsigned)((out->nt + kInterpThreads - 1) / kInterpThreads));
    switch (tp.amp) {
    case PSTM_AMP_F32: launch_method<AMP_F32>(tp, grid, method); break;
    case PSTM_AMP_BF16: launch_method<AMP_BF16>(tp, grid, method); break;
    default: launch_method<AMP_F16>(tp, grid, method); break;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSTM_OK : cuda_fail(c, e, "interpolation migrate kernel launch");
}
}  // namespace ctx
}  // namespace pstm
