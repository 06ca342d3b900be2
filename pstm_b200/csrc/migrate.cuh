// migrate.cuh -- gather-form Kirchhoff PSTM kernel for sm_100a.
//
// One CTA (16 warps, 512 lanes) owns PB output pillars and, for each of them,
// a block of 512*R output times; lane `tid` owns the R times
// t = t_block + tid + 512*r, so every warp holds shallow and deep times alike
// and the work per warp is balanced.  A lane keeps the PB x R partial sums in
// registers.  Traces are streamed in chunks of C:
//   staging  the chunk's amplitude rows and packed FP64 geometry are copied
//            into shared memory by TMA bulk copies (cp.async.bulk + mbarrier),
//            double-buffered, so chunk k+1 lands while chunk k is processed;
//   records  every (pillar, trace) pair of the next chunk gets a record in
//            shared memory (FP64 geometry rounded once to FP32); the fold
//            predicate is evaluated in FP64 and counted with warp match /
//            ballot + popc;
//   pairs    every lane walks the records of the current chunk (warp-uniform
//            broadcast reads) and, for each of its R times, evaluates
//            traveltime, sample index, linear interpolation (from shared
//            memory) and weights, with warp-uniform skips instead of
//            divergent branches.
// Chunk partials are added into FP32 partial sums in shared memory (with
// their TwoSum rounding errors kept apart when compensated accumulation is
// on), which are added into the caller's image (+=) every 16 chunks and at
// the end; the fold is added in the epilogue.
//
// Reference semantics (paths relative to the reference project):
//   loop structure, fold, aperture, taper, weights  numba_cpu_optimized.py:147-231
//   per-time terms                                   numba_cpu_optimized.py:358-401
//   triangle AA weight                               pstm_migration.metal:95-132
//   curved-ray leg                                   pstm_curved_ray.metal:50-96
//   VTI leg                                          pstm_anisotropic_vti.metal:103-148
//
// Precision.  EXACT (straight rays): the sample index is formed in FP64 (DSR
// with a Newton-refined sqrt) and split into integer and fraction with bit
// operations, so the interpolation position carries ~2^-21 samples of error
// and the trace-end test is an FP64 decision.  Otherwise traveltime is FP32
// and the trace-end decision is re-taken in FP64 inside a guard band.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <type_traits>
#include "kparams.h"

namespace pstm {

constexpr int kThreads = 512;        // lanes per CTA = output times per r
constexpr int kMaxChunk = 32;        // traces per chunk, upper bound
constexpr int kGeoDoubles = 8;       // packed geometry per trace: sx sy rx ry mx my w 0
constexpr int kWaitIters = 1 << 20;  // default bound of every mbarrier wait loop (KParams::wait_iters)

// Unroll factors of the pair loops (records without / with a lane in the taper band).
#ifndef PSTM_UNROLL_PLAIN
#define PSTM_UNROLL_PLAIN 4
#endif
#ifndef PSTM_UNROLL_TAPER
#define PSTM_UNROLL_TAPER 2
#endif
// 1: the plain pair loop takes two records per step and does their weight
// arithmetic with packed FP32 pairs (add/mul/fma.f32x2, sm_100)
#ifndef PSTM_PACKED_PAIRS
#define PSTM_PACKED_PAIRS 1
#endif
// Unroll factor of the packed loop (steps of two records).
#ifndef PSTM_UNROLL_PACKED
#define PSTM_UNROLL_PACKED 2
#endif
#define PSTM_PRAGMA_STR(x) #x
#define PSTM_UNROLL(n) _Pragma(PSTM_PRAGMA_STR(unroll n))

// ---------------------------------------------------------------- math helpers
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// sqrt for q > 0: the hardware's approximate reciprocal square root
// (rsqrt.approx.f64) refined by one Newton step, accurate to ~2^-44.
__device__ __forceinline__ double sqrt_newton(double q) {
    double h;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(h) : "d"(q));
    const double u = q * h;
    const double c = fma(-u, u, q);
    return fma(c, 0.5 * h, u);
}
// 1/x for x > 0: the hardware's approximate reciprocal refined by one Newton step.
__device__ __forceinline__ double rcp_newton(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return fma(r, fma(-x, r, 1.0), r);
}
// Positive double in the float normal range -> float, truncating the
// mantissa (|error| < 1 float ulp), with integer ops only.
__device__ __forceinline__ float double_to_float_trunc(double x) {
    const unsigned hi = (unsigned)__double2hiint(x), lo = (unsigned)__double2loint(x);
    return __uint_as_float(__funnelshift_l(lo, hi, 3) - (896u << 23));
}

template <int AMP>
__device__ __forceinline__ float amp_at(const unsigned char *row, int i) {
    if constexpr (AMP == AMP_F32) {
        return reinterpret_cast<const float *>(row)[i];
    } else if constexpr (AMP == AMP_BF16) {
        return __uint_as_float(((unsigned)reinterpret_cast<const unsigned short *>(row)[i]) << 16);
    } else {
        return __half2float(reinterpret_cast<const __half *>(row)[i]);
    }
}

// ---------------------------------------------------------------- TMA bulk copies
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
// Bounded wait for the mbarrier phase with the given parity: at most `iters`
// polls (each a potentially blocking try_wait); false = gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int iters) {
    for (int i = 0; i < iters; ++i) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// ---------------------------------------------------------------- per-time state
// Quantities that depend on the output time only: one table entry per time
// (prep_time_table), loaded per (pillar, r) just before the record loop.
struct TimeState {
    float t0h2;
    float Kt;              // obliquity numerator t0 (in the weight's time unit) or 1
    float tg;              // weights apply only when T > tg ("T > 1 ms"); -1 when always
    float tguard;          // 1 ms in the unit of T
    float vz, vz2, ivwc;   // curved: velocity at image depth, 1/vz
    bool tzero;
    bool tz, tz_in;        // t0 = 0 with T = 0 exactly for every pair; its sample index inside the trace
    double A;              // EXACT: (t0 / (2 dt))^2 (at least 1e-20)
    double vz64, vz2_64;   // EXACT, curved kinds: v(z) of the image depth and its square
};

// Quantities that depend on (pillar, time).
struct PtState {
    float iv2, ap, itw, tsn;
    float K;               // weight numerator
    float ivw_t;           // 1/v_w per unit of T (AA sin theta)
    float aaA;             // 4 max(dx,dy) f_dom / v_w (AA)
    float aa_k, aa_thr;    // aaA / v_w per unit of T; minf / T above which sin(theta) >= 0.01
    float t02v2, c1, e2;   // VTI: (t0/2)^2 v^2, 1+2eta, 2 eta / v^2
    float iv2r;            // 1/v_rms^2 (the curved+VTI ratio's hyperbolic leg; iv2 may be 1/v0^2)
    double B;              // EXACT: 1/(v dt)^2
    double c1B, e2B2;      // EXACT, VTI kinds: (1+2eta) / (v dt)^2, 2 eta / (v dt)^4
};

template <int TT, bool EXACT>
__device__ __forceinline__ void load_states(const KParams &P, int p, int t, TimeState &ts, PtState &s) {
    const bool valid = t < P.nt;
    const int tc = valid ? t : P.nt - 1;
    const float4 a = P.ttime[2 * tc], b = P.ttime[2 * tc + 1];
    ts.t0h2 = a.x;
    ts.Kt = a.y;
    ts.tg = a.z;
    ts.tguard = a.w;
    ts.vz = b.x;
    ts.vz2 = b.y;
    ts.ivwc = b.z;
    ts.tzero = b.w != 0.f;
    ts.tz = b.w >= 2.f;
    ts.tz_in = b.w == 2.f;
    ts.A = EXACT ? P.ttimeA[tc] : 0.0;
    ts.vz64 = ts.vz2_64 = 0.0;
    if constexpr (EXACT && (TT == TT_CURVED || TT == TT_CURVED_VTI)) {
        ts.vz64 = P.ttimeV[tc];
        ts.vz2_64 = ts.vz64 * ts.vz64;
    }
    const int64_t ti = (P.vel3d || P.eta3d) ? (int64_t)p * P.nt + tc : tc;
    const float4 tab = P.ttab[ti];
    s.iv2 = tab.x;
    s.iv2r = tab.x;
    s.ap = valid ? tab.y : -1.f;   // a time past the tile end is never inside the aperture
    const float width = tab.y * P.taper_f;
    if (width > 0.f) {
        s.itw = rcp_approx(width);
        s.tsn = -(tab.y * (1.f - P.taper_f)) * s.itw;
    } else {
        s.itw = 0.f;
        s.tsn = -1.f;
    }
    float ivw = tab.z;
    if constexpr (TT == TT_CURVED || TT == TT_CURVED_VTI) {
        ivw = ts.ivwc;
        // |k| ~ 0: straight rays in the constant velocity v0 (curved_ray.py:35-38)
        if (P.cr_k_zero) s.iv2 = ts.ivwc * ts.ivwc;
    }
    // T is in seconds, or in samples on the EXACT path: 1/(v T_sec) = (1/(v dt)) / T_samples
    s.ivw_t = EXACT ? ivw * P.inv_dt_f : ivw;
    s.aaA = P.aa_cA * ivw;
    s.aa_k = s.aaA * s.ivw_t;
    s.aa_thr = 0.01f * rcp_approx(s.ivw_t);
    s.K = P.spreading ? ts.Kt * s.ivw_t : ts.Kt;
    s.t02v2 = 0.f;
    s.c1 = 1.f;
    s.e2 = 0.f;
    if constexpr (TT == TT_VTI || TT == TT_CURVED_VTI) {
        s.t02v2 = ts.t0h2 * rcp_approx(tab.x);   // (t0/2)^2 v^2
        s.c1 = 1.f + 2.f * tab.w;
        s.e2 = 2.f * tab.w * tab.x;
    }
    s.B = EXACT ? P.btab[ti] : 0.0;
    s.c1B = s.e2B2 = 0.0;
    if constexpr (EXACT && (TT == TT_VTI || TT == TT_CURVED_VTI)) {
        double eta = P.eta_const;
        if (P.eta) eta = P.eta3d ? P.eta[(int64_t)p * P.nt + tc] : P.eta[tc];
        s.c1B = (1.0 + 2.0 * eta) * s.B;
        s.e2B2 = 2.0 * eta * s.B * s.B;
    }
}

// FP64 traveltime in samples (the EXACT path of the curved and VTI kinds) of
// one pair from its record: B = {ds2, dr2}, C = curved {1/(bs br), 0} or
// curved+VTI {1/bs, 1/br}, bs = v0 + sqrt(v0^2 + k^2 ds2).  The formulas of
// traveltime_fp64 with every time divided by dt: A = (t0/2)^2/dt^2,
// h^2/(v dt)^2 = h^2 B, and the VTI correction 2 eta h^4 / (v^2 (t0h^2 v^2 +
// (1+2eta) h^2)) / dt^2 = e2B2 h^4 / (A + c1B h^2).
template <int TT>
__device__ __forceinline__ double exact_time_samples(const KParams &P, const TimeState &ts, const PtState &s,
                                                     const double2 &B, const double2 &C) {
    if constexpr (TT == TT_VTI) {
        if (ts.tz) return 0.0;   // the reference's VTI leg is 0 at t0 = 0
        const double Ds = fma(B.x, s.c1B, ts.A), Dr = fma(B.y, s.c1B, ts.A);
        const double rr = rcp_newton(Ds * Dr);
        const double qs = fma(-(s.e2B2 * B.x * B.x), Dr * rr, fma(B.x, s.B, ts.A));
        const double qr = fma(-(s.e2B2 * B.y * B.y), Ds * rr, fma(B.y, s.B, ts.A));
        return sqrt_newton(fmax(qs, 1e-300)) + sqrt_newton(fmax(qr, 1e-300));
    } else if constexpr (TT == TT_CURVED) {   // |k| ~ 0: straight rays in v0 (curved_ray.py:35-38)
        if (P.cr_k_zero) return sqrt_newton(fma(B.x, P.cr_B0, ts.A)) + sqrt_newton(fma(B.y, P.cr_B0, ts.A));
        if (ts.tz) return 0.0;   // depth 0: both legs are log(1) = 0
        const double as = ts.vz64 + sqrt_newton(fma(P.cr_k2, B.x, ts.vz2_64));
        const double ar = ts.vz64 + sqrt_newton(fma(P.cr_k2, B.y, ts.vz2_64));
        return log(as * ar * C.x) * P.cr_inv_k_dt;
    } else {
        double tcs, tcr;
        if (P.cr_k_zero) {
            tcs = sqrt_newton(fma(B.x, P.cr_B0, ts.A));
            tcr = sqrt_newton(fma(B.y, P.cr_B0, ts.A));
        } else {
            if (ts.tz) return 0.0;
            tcs = log((ts.vz64 + sqrt_newton(fma(P.cr_k2, B.x, ts.vz2_64))) * C.x) * P.cr_inv_k_dt;
            tcr = log((ts.vz64 + sqrt_newton(fma(P.cr_k2, B.y, ts.vz2_64))) * C.y) * P.cr_inv_k_dt;
        }
        if (ts.tzero) return tcs + tcr;   // t0 = 0: the curved legs alone
        // leg = t_curved sqrt(1 - corr / (A + h^2 B)), corr = e2B2 h^4 / (A + c1B h^2)
        const double Hs = fma(B.x, s.B, ts.A), Hr = fma(B.y, s.B, ts.A);
        const double Ds = fma(B.x, s.c1B, ts.A), Dr = fma(B.y, s.c1B, ts.A);
        const double ps = Ds * Hs, pr = Dr * Hr;
        const double rr = rcp_newton(ps * pr);
        const double xs = s.e2B2 * B.x * B.x * (pr * rr), xr = s.e2B2 * B.y * B.y * (ps * rr);
        return tcs * sqrt_newton(fmax(1.0 - xs, 1e-300)) + tcr * sqrt_newton(fmax(1.0 - xr, 1e-300));
    }
}

// 0.5 (1 + cos(pi x)) = cos^2(pi x / 2) for x in [0, 1]: Taylor series of cos
// about 0 through y^12 (|error| < 7e-9 on y in [0, pi/2]), then squared.
__device__ __forceinline__ float taper_weight(float x) {
    const float y = 1.57079632679489662f * x;
    const float u = y * y;
    float c = 2.08767569878681e-9f;                 //  1/12!
    c = fmaf(c, u, -2.75573192239859e-7f);          // -1/10!
    c = fmaf(c, u, 2.48015873015873e-5f);           //  1/8!
    c = fmaf(c, u, -1.38888888888889e-3f);          // -1/6!
    c = fmaf(c, u, 4.16666666666667e-2f);           //  1/4!
    c = fmaf(c, u, -0.5f);                          // -1/2!
    c = fmaf(c, u, 1.0f);
    return c * c;
}

// ---------------------------------------------------------------- FP64 exact decisions
// (rare paths: they read the launch parameters from a global copy, so the
// kernel's own parameter block never has its address taken)
// FP64 traveltime of one pair from its raw quantities: output time t0 (s),
// squared horizontal source and receiver distances, v_rms, eta and the
// curved-ray (v0, k).  The oracle's formulas; also the surrogate's target.
template <int TT>
__host__ __device__ inline double traveltime_fp64(double t0, double ds2, double dr2, double v, double eta, double v0,
                                                  double k) {
    const double t0h = t0 * 0.5;
    auto vti_corr = [&](double h2) {
        const double v2 = v * v;
        const double den = v2 * (t0h * t0h * v2 + (1.0 + 2.0 * eta) * h2);
        return fabs(den) > 1e-20 ? (2.0 * eta * h2 * h2) / den : 0.0;
    };
    auto curved_leg = [&](double h2) {
        if (fabs(k) < 1e-10) {
            const double z = v0 * t0h;
            const double r = sqrt(h2 + z * z);
            return r > 0.0 ? r / v0 : 0.0;
        }
        const double z = (v0 / k) * (exp(k * t0h) - 1.0);
        const double vz = v0 + k * z;
        const double kx2 = k * k * h2;
        const double a = vz + sqrt(vz * vz + kx2), b = v0 + sqrt(v0 * v0 + kx2);
        return b <= 0.0 ? 0.0 : (1.0 / k) * log(a / b);
    };
    if constexpr (TT == TT_STRAIGHT) {
        const double iv2 = 1.0 / (v * v);
        return sqrt(t0h * t0h + ds2 * iv2) + sqrt(t0h * t0h + dr2 * iv2);
    } else if constexpr (TT == TT_CURVED) {
        return curved_leg(ds2) + curved_leg(dr2);
    } else if constexpr (TT == TT_VTI) {
        if (v <= 0.0 || t0h <= 0.0) return 2.0 * t0h;
        auto leg = [&](double h2) {
            const double q = t0h * t0h + h2 / (v * v) - vti_corr(h2);
            return sqrt(q > 0.0 ? q : 0.0);
        };
        return leg(ds2) + leg(dr2);
    } else {
        auto leg = [&](double h2) {
            const double tc = curved_leg(h2);
            if (v <= 0.0 || t0h <= 0.0) return tc;
            const double r = 1.0 - vti_corr(h2) / (t0h * t0h + h2 / (v * v));
            return tc * sqrt(r > 0.0 ? r : 0.0);
        };
        return leg(ds2) + leg(dr2);
    }
}

template <int TT>
__device__ double exact_traveltime(const KParams *P, int64_t tr, int p, int t, double ox, double oy) {
    const double t0 = P->ta[t] / 1000.0;
    const double v = P->vel3d ? P->vrms[(int64_t)p * P->nt + t] : P->vrms[t];
    const double dxs = ox - P->sx[tr], dys = oy - P->sy[tr];
    const double dxr = ox - P->rx[tr], dyr = oy - P->ry[tr];
    double eta = P->eta_const;
    if (P->eta) eta = P->eta3d ? P->eta[(int64_t)p * P->nt + t] : P->eta[t];
    return traveltime_fp64<TT>(t0, dxs * dxs + dys * dys, dxr * dxr + dyr * dyr, v, eta, P->cr_v0, P->cr_k);
}

// Is the FP64 sample index of this pair inside [0, ns-1)?
template <int TT>
__device__ __noinline__ bool exact_sample_ok(const KParams *P, int64_t tr, int p, int t, double ox, double oy) {
    const double T = exact_traveltime<TT>(P, tr, p, t, ox, oy);
    const double s = (T - P->tstart_s) / P->dt_s;
    return s >= 0.0 && s < (double)(P->ns - 1);
}

// Is the midpoint outside the time-varying aperture, decided in FP64?
static __device__ __noinline__ bool exact_outside_aperture(const KParams *P, int64_t tr, int p, int t, double ox,
                                                           double oy) {
    const double dx = ox - P->mx[tr], dy = oy - P->my[tr];
    const double d = sqrt(dx * dx + dy * dy);
    const double v = P->vel3d ? P->vrms[(int64_t)p * P->nt + t] : P->vrms[t];
    double ap = v * (P->ta[t] / 1000.0) * 0.5 * P->tan_dip;
    if (ap < P->min_ap) ap = P->min_ap;
    else if (ap > P->max_ap) ap = P->max_ap;
    return d > ap;
}

// ---------------------------------------------------------------- traveltime (FP32)
// Records: A = {d, wt, minf, byte offset of the trace's staged row}; B = {ds2, dr2, k^2 ds2 | ds2^2, k^2 dr2 | dr2^2};
// C (curved kinds) = {1/(bs br) | 1/bs, 1/br, ds2^2, dr2^2}.  Result in seconds.
template <int TT>
__device__ __forceinline__ float traveltime(const KParams &P, const TimeState &ts, const PtState &s,
                                            const float4 &B, const float4 &Cc) {
    if constexpr (TT == TT_STRAIGHT) {
        return sqrt_approx(fmaf(B.x, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(B.y, s.iv2, ts.t0h2));
    } else if constexpr (TT == TT_CURVED) {
        if (P.cr_k_zero) {
            return sqrt_approx(fmaf(B.x, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(B.y, s.iv2, ts.t0h2));
        }
        const float a = ts.vz + sqrt_approx(ts.vz2 + B.z);
        const float b = ts.vz + sqrt_approx(ts.vz2 + B.w);
        return P.cr_inv_k_ln2 * lg2_approx(a * b * Cc.x);
    } else if constexpr (TT == TT_VTI) {
        if (ts.tzero) return 0.f;
        const float Ds = fmaf(s.c1, B.x, s.t02v2);
        const float Dr = fmaf(s.c1, B.y, s.t02v2);
        const float rr = rcp_approx(Ds * Dr);
        const float qs = fmaf(-(s.e2 * B.z), Dr * rr, fmaf(B.x, s.iv2, ts.t0h2));
        const float qr = fmaf(-(s.e2 * B.w), Ds * rr, fmaf(B.y, s.iv2, ts.t0h2));
        return sqrt_approx(fmaxf(qs, 0.f)) + sqrt_approx(fmaxf(qr, 0.f));
    } else {
        float tcs, tcr;
        if (P.cr_k_zero) {
            tcs = sqrt_approx(fmaf(B.x, s.iv2, ts.t0h2));
            tcr = sqrt_approx(fmaf(B.y, s.iv2, ts.t0h2));
        } else {
            const float a = ts.vz + sqrt_approx(ts.vz2 + B.z);
            const float b = ts.vz + sqrt_approx(ts.vz2 + B.w);
            tcs = P.cr_inv_k_ln2 * lg2_approx(a * Cc.x);
            tcr = P.cr_inv_k_ln2 * lg2_approx(b * Cc.y);
        }
        if (ts.tzero) return tcs + tcr;
        // leg = t_curved * sqrt(1 - corr / (t0h^2 + h^2/v^2)), corr = e2 h^4 / D, v = v_rms
        const float Hs = fmaf(B.x, s.iv2r, ts.t0h2), Hr = fmaf(B.y, s.iv2r, ts.t0h2);
        const float Ds = fmaf(s.c1, B.x, s.t02v2), Dr = fmaf(s.c1, B.y, s.t02v2);
        const float ps_ = Ds * Hs, pr_ = Dr * Hr;
        const float rr = rcp_approx(ps_ * pr_);
        const float xs = s.e2 * Cc.z * (pr_ * rr), xr = s.e2 * Cc.w * (ps_ * rr);
        return tcs * sqrt_approx(fmaxf(1.f - xs, 0.f)) + tcr * sqrt_approx(fmaxf(1.f - xr, 0.f));
    }
}

template <int TT>
struct RecLayout {
    static constexpr bool kHasC = (TT == TT_CURVED || TT == TT_CURVED_VTI);
};

constexpr int kMaxPB = 16;   // pillars per CTA, upper bound (one warp per pillar builds records)

// Bytes of one record buffer (the kernel keeps two): A, B and (curved kinds) C.
__host__ __device__ constexpr int record_buffer_bytes(int PB, bool has_c) {
    return PB * kMaxChunk * 16 * (has_c ? 3 : 2);
}
__host__ __device__ constexpr int geo_buffer_bytes() { return kMaxChunk * kGeoDoubles * 8; }
// FP32 partial sums of a CTA (PB x R x kThreads floats), and with compensated
// accumulation their TwoSum error terms, kept in BF16: an error term needs
// only a few significant bits (it corrects the partial's last bits), and half
// the bytes leave more of shared memory to the staged traces.
__host__ __device__ constexpr int partial_bytes(int PB, int R, bool compensated = false) {
    return PB * R * kThreads * (compensated ? 6 : 4);
}
__device__ __forceinline__ float bf16_to_f32(unsigned short h) { return __uint_as_float((unsigned)h << 16); }
__device__ __forceinline__ unsigned short f32_to_bf16(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// ---------------------------------------------------------------- the kernel
// What one work item migrates: PB pillars x one block of 512*R output times of
// one output image, against one contiguous range of traces.
struct Item {
    const unsigned char *amps;   // first amplitude row of the range
    const double *geo;           // first packed trace of the range
    int64_t trace0;              // global index of the first trace (FP64 re-decisions)
    int64_t n_traces;
    void *image;
    int32_t *fold;
    int pbx, pby, tblock;
};

// Shared-memory state of a CTA besides the dynamic buffers.
struct CtaShared {
    double ox[kMaxPB], oy[kMaxPB];
    int pid[kMaxPB];
    int fold[kMaxPB];
    int rank[kMaxPB][kMaxChunk];
    unsigned long long bar[2];
    long long item;
};

// Migrates one item.  `chunk_base` counts the chunks this CTA staged before
// (it selects the buffer and the mbarrier phase of every chunk).  Returns
// false when a bounded wait gave up.
// W2: spreading and obliquity both on (the common case), else the weight
// exponent is chosen at run time.  GUARD (FP32-traveltime path only): trace-end
// tests within 0.01 samples of a trace end are re-taken in FP64; without it
// (PSTM_PREC_FP32) they are FP32 like the rest of the sample index.
template <int TT, int AMP, bool VEL3D, bool EXACT, bool W2, bool GUARD>
__device__ __forceinline__ bool migrate_item(const KParams &P, const KParams *__restrict__ Pg, const Item &it,
                                             unsigned char *smem, CtaShared &sh, int64_t &chunk_base) {
    constexpr bool HAS_C = RecLayout<TT>::kHasC;
    double *const s_ox = sh.ox;
    double *const s_oy = sh.oy;
    int *const s_pid = sh.pid;
    int *const s_fold = sh.fold;
    auto &s_rank = sh.rank;

    const int PB = P.pb, R = P.r_per_lane;
    const int RECS = PB * kMaxChunk;
    const int REC_BYTES = record_buffer_bytes(PB, HAS_C);
    const int C = P.chunk;
    const int row_bytes = P.pitch * P.elem;
    const int amp_bytes = C * row_bytes;   // multiple of 16
    unsigned char *const amp_base = smem;
    unsigned char *const geo_base = smem + 2 * amp_bytes;
    unsigned char *const rec_base = geo_base + 2 * geo_buffer_bytes();
    float *const s_acc = reinterpret_cast<float *>(rec_base + 2 * REC_BYTES);   // [PB][R][kThreads]
    const bool comp = P.compensated != 0;
    unsigned short *const s_err =   // [PB][R][kThreads] BF16 error terms when comp
        reinterpret_cast<unsigned short *>(s_acc + PB * R * kThreads);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pbx = it.pbx, pby = it.pby;
    __syncthreads();   // the previous item is done with the shared state
    if (tid < PB) {
        const int ix = pbx * P.px + tid / P.py, iy = pby * P.py + tid % P.py;
        const bool ok = (tid < P.px * P.py) && ix < P.nx && iy < P.ny;
        const int p = ok ? ix * P.ny + iy : -1;
        s_pid[tid] = p;
        s_fold[tid] = 0;
        s_ox[tid] = ok ? (P.xg ? P.xg[p] : P.xa[ix]) : 0.0;
        s_oy[tid] = ok ? (P.yg ? P.yg[p] : P.ya[iy]) : 0.0;
    }
    const uint32_t bar0 = smem_u32(&sh.bar[0]), bar1 = smem_u32(&sh.bar[1]);
    const int t_lane = it.tblock * (kThreads * R) + tid;   // this thread's times: t_lane + r * kThreads

    // hot-loop constants in registers
    const float s_scale = P.s_scale, s_offset = P.s_offset;
    // guard bands around the trace ends, as distances from the middle of the trace:
    // |s - mid| <= g_in is inside by more than the band, g_in < |s - mid| <= g_out is in a band
    const float g_mid = 0.5f * (P.s_guard_lo + P.s_guard_hi);
    const float g_in = P.s_guard_hi - g_mid, g_out = P.s_rej_hi - g_mid;
    const float s_clamp = P.s_max_clamp;
    const unsigned ns_m1 = (unsigned)(P.ns - 1);
    const double magic = P.s_magic;
    const bool w_one = P.spreading + P.obliquity == 1, w_two = P.spreading + P.obliquity == 2;
    const float aa_cB = P.aa_cB;
    const bool aa_on = P.aa != 0;
    const bool hard_cut = !(P.taper_f > 0.f);
    const float one_m_taper = 1.f - P.taper_f;
    const int64_t n_chunks = (it.n_traces + C - 1) / C;
    const int flush_every = P.flush_every;

    // partials and (comp) the error terms behind them: PB R kThreads (3/2) floats
    for (int i = tid; i < PB * R * kThreads * (comp ? 3 : 2) / 2; i += kThreads) s_acc[i] = 0.f;

    // one thread: TMA bulk copies of chunk k (packed geometry, and the amplitude
    // rows when they are 16-byte aligned) into buffer b
    auto issue_chunk = [&](int64_t k, int b) {
        const int64_t c0 = k * C;
        const int rows = (int)min((int64_t)C, it.n_traces - c0);
        const uint32_t bar = b ? bar1 : bar0;
        const uint32_t geo_bytes = (uint32_t)(rows * kGeoDoubles * 8);
        mbar_expect_tx(bar, geo_bytes + (P.bulk ? (uint32_t)(rows * row_bytes) : 0u));
        bulk_g2s(smem_u32(geo_base + b * geo_buffer_bytes()), it.geo + c0 * kGeoDoubles, geo_bytes, bar);
        if (P.bulk) {
            const unsigned char *src = it.amps + c0 * P.amp_stride * P.elem;
            const uint32_t dst = smem_u32(amp_base + b * amp_bytes);
            for (int i = 0; i < rows; ++i)
                bulk_g2s(dst + i * row_bytes, src + (int64_t)i * P.amp_stride * P.elem, (uint32_t)row_bytes, bar);
        }
    };

    // Records of chunk k from the staged geometry in buffer b: warp q builds
    // pillar q's 32 records, counts its fold and sorts them by midpoint
    // distance (bitonic, in registers) so that, for any aperture, the records
    // inside it form a prefix.
    auto pillar_records = [&](int64_t k, int b, int q) {   // one warp: pillar q's records of chunk k
        const int64_t c0 = k * C;
        const int cmax = (int)min((int64_t)C, it.n_traces - c0);
        {
            const int c = lane;
            const double *geo = reinterpret_cast<const double *>(geo_base + b * geo_buffer_bytes());
            float4 *recA = reinterpret_cast<float4 *>(rec_base + b * REC_BYTES);
            const int p = s_pid[q];
            bool in = false;
            const float inf = __int_as_float(0x7f800000);
            float4 A = make_float4(inf, 0.f, 0.f, __int_as_float(c * row_bytes));
            float4 Bf = make_float4(0.f, 0.f, 0.f, 0.f), Cc = Bf;
            double2 B64 = make_double2(0.0, 0.0);
            if (p >= 0 && c < cmax) {
                const double *g = geo + c * kGeoDoubles;   // sx sy rx ry mx my w
                const double ox = s_ox[q], oy = s_oy[q];
                const double dxm = ox - g[4], dym = oy - g[5];
                const double d2 = dxm * dxm + dym * dym;
                in = d2 <= P.fold_d2_max;
                if (in) {
                    const double dxs = ox - g[0], dys = oy - g[1];
                    const double dxr = ox - g[2], dyr = oy - g[3];
                    const double ds2 = dxs * dxs + dys * dys, dr2 = dxr * dxr + dyr * dyr;
                    // the FP64 sqrt is needed only where the aperture cut is hard
                    const float d = hard_cut ? (float)sqrt(d2) : sqrt_approx((float)d2);
                    A = make_float4(d, (float)g[6], (float)fmax(fabs(dxm), fabs(dym)), __int_as_float(c * row_bytes));
                    B64 = make_double2(ds2, dr2);
                    Bf = make_float4((float)ds2, (float)dr2, 0.f, 0.f);
                    if constexpr (TT == TT_CURVED || TT == TT_CURVED_VTI) {
                        const double k2 = P.cr_k * P.cr_k, v0 = P.cr_v0;
                        const double bs = v0 + sqrt(v0 * v0 + k2 * ds2);
                        const double br = v0 + sqrt(v0 * v0 + k2 * dr2);
                        Bf.z = (float)(k2 * ds2);
                        Bf.w = (float)(k2 * dr2);
                        if constexpr (EXACT) {   // the C slot holds FP64 {1/(bs br), 0} or {1/bs, 1/br}
                            const double2 c64 = TT == TT_CURVED ? make_double2(1.0 / (bs * br), 0.0)
                                                                : make_double2(1.0 / bs, 1.0 / br);
                            Cc = make_float4(__int_as_float(__double2loint(c64.x)),
                                             __int_as_float(__double2hiint(c64.x)),
                                             __int_as_float(__double2loint(c64.y)),
                                             __int_as_float(__double2hiint(c64.y)));
                        } else if constexpr (TT == TT_CURVED) {
                            Cc = make_float4((float)(1.0 / (bs * br)), 0.f, 0.f, 0.f);
                        } else {
                            Cc = make_float4((float)(1.0 / bs), (float)(1.0 / br), (float)(ds2 * ds2),
                                             (float)(dr2 * dr2));
                        }
                    } else if constexpr (TT == TT_VTI) {
                        Bf.z = (float)(ds2 * ds2);
                        Bf.w = (float)(dr2 * dr2);
                    }
                }
            }
            const unsigned ballot = __ballot_sync(0xffffffffu, in);
            if (lane == 0) s_fold[q] += __popc(ballot);
            // bitonic sort of (d, lane) ascending across the warp
            float key = A.x;
            int idx = lane;
#pragma unroll
            for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
                for (int j = kk >> 1; j > 0; j >>= 1) {
                    const float ok_ = __shfl_xor_sync(0xffffffffu, key, j);
                    const int oi = __shfl_xor_sync(0xffffffffu, idx, j);
                    const bool up = (lane & kk) == 0, lower = (lane & j) == 0;
                    const bool other_less = ok_ < key || (ok_ == key && oi < idx);
                    const bool take = (lower == up) ? other_less : !other_less;
                    key = take ? ok_ : key;
                    idx = take ? oi : idx;
                }
            }
            s_rank[q][idx] = lane;   // lane L holds the L-th smallest: idx goes to slot L
            __syncwarp();
            const int ri = q * kMaxChunk + s_rank[q][lane];
            recA[ri] = A;
            if constexpr (EXACT) reinterpret_cast<double2 *>(recA + RECS)[ri] = B64;
            else reinterpret_cast<float4 *>(recA + RECS)[ri] = Bf;
            if constexpr (HAS_C) reinterpret_cast<float4 *>(recA + 2 * RECS)[ri] = Cc;
        }
    };
    // amplitude rows not 16-byte aligned (no TMA bulk copy): plain cooperative copy by all threads
    auto copy_rows = [&](int64_t k, int b) {
        const int64_t c0 = k * C;
        const int cmax = (int)min((int64_t)C, it.n_traces - c0);
        {
            unsigned char *dst = amp_base + b * amp_bytes;
            const unsigned char *src = it.amps;
            for (int e = tid; e < cmax * P.ns; e += kThreads) {
                const int rr = e / P.ns, ii = e - rr * P.ns;
                const int64_t gi = (c0 + rr) * P.amp_stride + ii;
                if (P.elem == 4)
                    reinterpret_cast<float *>(dst + rr * row_bytes)[ii] = reinterpret_cast<const float *>(src)[gi];
                else
                    reinterpret_cast<unsigned short *>(dst + rr * row_bytes)[ii] =
                        reinterpret_cast<const unsigned short *>(src)[gi];
            }
        }
    };
    auto build_records = [&](int64_t k, int b) {   // every pillar (warp q < PB) and the row copy
        if (warp < PB) pillar_records(k, b, warp);
        if (!P.bulk) copy_rows(k, b);
    };

    // add this lane's FP32 partial sums into the FP64 (or FP32) image and clear them
    auto flush = [&]() {
#pragma unroll 1
        for (int q = 0; q < PB; ++q) {
            const int p = s_pid[q];
#pragma unroll 1
            for (int r = 0; r < R; ++r) {
                const int t = t_lane + r * kThreads;
                float &sa = s_acc[(q * R + r) * kThreads + tid];
                float a = sa;
                if (comp) {   // the partial and its rounding error, summed in FP32 once more
                    unsigned short &se = s_err[(q * R + r) * kThreads + tid];
                    a += bf16_to_f32(se);
                    se = 0;
                }
                if (p >= 0 && t < P.nt && a != 0.f) {
                    const int64_t idx = (int64_t)p * P.nt + t;
                    if (P.atomic_flush) {   // items of several trace segments share the outputs
                        if (P.image_f32) atomicAdd(reinterpret_cast<float *>(it.image) + idx, a);
                        else atomicAdd(reinterpret_cast<double *>(it.image) + idx, (double)a);
                    } else if (P.image_f32) {
                        reinterpret_cast<float *>(it.image)[idx] += a;
                    } else {
                        reinterpret_cast<double *>(it.image)[idx] += (double)a;
                    }
                }
                sa = 0.f;
            }
        }
    };

    __syncthreads();   // pillars known
    // chunk k of this item is the CTA's chunk g = chunk_base + k: buffer g & 1,
    // mbarrier phase parity (g >> 1) & 1
    const int b0 = (int)(chunk_base & 1);
    const int wait_iters = P.wait_iters;
    // (fault injection: with inject_stall the first copies are never issued, so
    // nothing completes their phase and the bounded wait below runs out)
    if (tid == 0 && !P.inject_stall) {
        if (chunk_base > 0) fence_proxy_async();   // the previous item's reads of the buffers
        if (n_chunks > 0) issue_chunk(0, b0);
        if (n_chunks > 1) issue_chunk(1, b0 ^ 1);
    }
    bool aborted = false;
    if (n_chunks > 0) {
        const bool ok = mbar_wait(b0 ? bar1 : bar0, (uint32_t)((chunk_base >> 1) & 1), wait_iters);
        if (__syncthreads_or(!ok)) aborted = true;
        else build_records(0, b0);
    }
    __syncthreads();

    for (int64_t k = 0; k < n_chunks && !aborted; ++k) {
        const int64_t c0 = k * C;
        const int64_t g = chunk_base + k;
        const int buf = (int)(g & 1);
        const float4 *recA = reinterpret_cast<const float4 *>(rec_base + buf * REC_BYTES);
        const unsigned char *ampb = amp_base + buf * amp_bytes;

        // ---------------- pairs of chunk k
#pragma unroll 1
        for (int q = 0; q < PB; ++q) {
            const int p = s_pid[q];
            if (p < 0) continue;
            const float4 *A_q = recA + q * kMaxChunk;
            const float dl = A_q[lane].x;   // this lane's slot of the sorted distances
            const int vt = tid;             // the partial sums of this thread's times
#pragma unroll 1
            for (int r = 0; r < R; ++r) {
                const int t = t_lane + r * kThreads;
                TimeState ts;
                PtState s;
                load_states<TT, EXACT>(P, p, t, ts, s);
                // records inside the aperture of some lane: a prefix of length n;
                // records with no lane in its taper band: a prefix of length n0
                const float apw = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(s.ap)));
                // lanes past the tile end (ap < 0) take no part; a zero aperture gives 0
                const float tsl = s.ap >= 0.f ? s.ap * one_m_taper : __int_as_float(0x7f800000);
                const float tmin = __int_as_float(__reduce_min_sync(0xffffffffu, __float_as_int(tsl)));
                const int n = __popc(__ballot_sync(0xffffffffu, dl <= apw));
                const int n0 = min(n, __popc(__ballot_sync(0xffffffffu, dl <= tmin)));
                unsigned pmask = 0u;   // FP32 path: records with a pair in a trace-end guard band

                // contribution of record c (slot in the sorted order) to this lane's time
                // CHK: some lane of the warp may have T <= 1 ms (t0 < 1.1 ms, or curved rays),
                // so the "T > 1 ms" conditions of the weights are evaluated; otherwise every
                // T of the warp exceeds t0 >= 1.1 ms and they are known to hold
                // ALLIN: the record is inside every valid lane's aperture (c < n0), so the
                // aperture test is known to pass
                auto pair = [&](int c, auto taper_c, auto slow_c, auto hard_c, auto chk_c, auto allin_c) -> float {
                    constexpr bool TAPER = decltype(taper_c)::value;
                    constexpr bool SLOW = decltype(slow_c)::value;
                    constexpr bool HARD = decltype(hard_c)::value;
                    constexpr bool CHK = decltype(chk_c)::value;
                    constexpr bool ALLIN = decltype(allin_c)::value;
                    const int ri = q * kMaxChunk + c;
                    const float4 A = recA[ri];
                    bool act = ALLIN ? true : (A.x <= s.ap);
                    const int roff = __float_as_int(A.w);   // row offset; the trace is roff / row_bytes
                    if (HARD && (EXACT || GUARD) && A.x == s.ap)   // FP32 tie of distance and aperture: decide in FP64
                        act = !exact_outside_aperture(Pg, it.trace0 + c0 + roff / row_bytes, p, t, s_ox[q], s_oy[q]);
                    float T, f;
                    int i0;
                    bool ok;
                    if constexpr (EXACT) {
                        const double2 B = reinterpret_cast<const double2 *>(recA + RECS)[ri];
                        double T2;
                        if constexpr (TT == TT_STRAIGHT) {
                            T2 = sqrt_newton(fma(B.x, s.B, ts.A)) + sqrt_newton(fma(B.y, s.B, ts.A));
                        } else {
                            double2 C = make_double2(0.0, 0.0);
                            if constexpr (HAS_C) C = reinterpret_cast<const double2 *>(recA + 2 * RECS)[ri];
                            T2 = exact_time_samples<TT>(P, ts, s, B, C);
                        }
                        // s + 2^31 keeps s in the mantissa with 21 fraction bits
                        const double v = T2 + magic;
                        const unsigned vh = (unsigned)__double2hiint(v), vl = (unsigned)__double2loint(v);
                        const unsigned iu = __funnelshift_r(vl, vh, 21);
                        ok = act && iu < ns_m1;   // also rejects s < 0 and NaN
                        i0 = ok ? (int)iu : 0;
                        f = __uint_as_float(0x3F800000u | ((vl & 0x1FFFFFu) << 2)) - 1.0f;
                        // straight: T2 >= 2e-10 (A >= 1e-20); the other kinds can give T2 = 0
                        T = TT == TT_STRAIGHT ? double_to_float_trunc(T2) : (float)T2;
                    } else {
                        const float4 B = reinterpret_cast<const float4 *>(recA + RECS)[ri];
                        float4 Cc = make_float4(0.f, 0.f, 0.f, 0.f);
                        if constexpr (HAS_C) Cc = reinterpret_cast<const float4 *>(recA + 2 * RECS)[ri];
                        T = traveltime<TT>(P, ts, s, B, Cc);
                        if constexpr (TT != TT_STRAIGHT) T = ts.tz ? 0.f : T;
                        float sidx = fmaf(T, s_scale, s_offset);
                        if constexpr (GUARD) {
                            // T = 0 exactly: the FP64 decision is known per time, no guard band
                            const float x = fabsf(sidx - g_mid);
                            const bool fast_ok = ts.tz ? ts.tz_in : (x <= g_in);
                            const bool band = act && !fast_ok && !ts.tz && x <= g_out;
                            if constexpr (TT != TT_STRAIGHT) sidx = ts.tz ? fminf(fmaxf(sidx, 0.f), s_clamp) : sidx;
                            if constexpr (SLOW) {   // re-decide the guard band in FP64
                                ok = band && exact_sample_ok<TT>(Pg, it.trace0 + c0 + roff / row_bytes, p, t, s_ox[q],
                                                                 s_oy[q]);
                                sidx = fminf(fmaxf(sidx, 0.f), s_clamp);
                            } else {
                                ok = act && fast_ok;
                                pmask |= band ? (1u << c) : 0u;
                            }
                            sidx = ok ? sidx : 0.f;
                        } else {   // FP32 trace-end test: the index is inside iff clamping leaves it unchanged
                            const float sc = fminf(fmaxf(sidx, 0.f), s_clamp);   // (NaN -> 0, outside)
                            bool in = sc == sidx;
                            if constexpr (TT != TT_STRAIGHT) in = ts.tz ? ts.tz_in : in;
                            ok = act && in;
                            sidx = sc;
                        }
                        const float fl = __fadd_rd(sidx, 8388608.f);
                        i0 = __float_as_int(fl) - 0x4B000000;
                        f = sidx - (fl - 8388608.f);
                    }
                    const unsigned char *row = ampb + roff;
                    const float a0 = amp_at<AMP>(row, i0);
                    const float a1 = amp_at<AMP>(row, i0 + 1);
                    const float amp = fmaf(f, a1 - a0, a0);
                    float w = ok ? A.y : 0.f;
                    if constexpr (TAPER) {
                        const float x = fmaf(A.x, s.itw, s.tsn);
                        w *= x > 0.f ? taper_weight(x) : 1.f;
                    }
                    const float rT = rcp_approx(T);
                    float gw;
                    if constexpr (W2) gw = s.K * rT * rT;
                    else gw = w_two ? s.K * rT * rT : (w_one ? s.K * rT : 1.f);
                    if constexpr (CHK) gw = T > ts.tg ? gw : 1.f;   // the reference applies them only for T > 1 ms
                    if (aa_on) {
                        // sin(theta) = min(minf / (v_w T), 1); aaA sin(theta) = min(u aaA / v_w, aaA)
                        const float u = A.z * rT;
                        const float aa = fmaxf(0.f, 1.f - fmaxf(fminf(u * s.aa_k, s.aaA), aa_cB));
                        gw = (u >= s.aa_thr && (!CHK || T >= ts.tguard)) ? gw * aa : gw;
                    }
                    return amp * (w * gw);
                };
                // The plain case (records inside every lane's aperture, no taper band,
                // every T of the warp above 1 ms) two records at a time: the traveltime,
                // sample index and amplitude reads per record, then the interpolation
                // and the weights of both in packed FP32 pairs.  Same operations as
                // `pair`; the AA weight is clamp(1 - u aa_k, L, H) with L = max(0,
                // 1 - aaA), H = max(0, 1 - f_dom/500), the same function as
                // max(0, 1 - max(min(u aa_k, aaA), f_dom/500)).
                const float aa_lo = fmaxf(0.f, 1.f - s.aaA), aa_hi = fmaxf(0.f, 1.f - aa_cB);
                auto front = [&](int c, float &a0, float &a1, float &f, float &T, float &w, float &mz) {
                    const int ri = q * kMaxChunk + c;
                    const float4 A = recA[ri];
                    const int roff = __float_as_int(A.w);
                    int i0;
                    bool ok;
                    if constexpr (EXACT) {
                        const double2 B = reinterpret_cast<const double2 *>(recA + RECS)[ri];
                        double T2;
                        if constexpr (TT == TT_STRAIGHT) {
                            T2 = sqrt_newton(fma(B.x, s.B, ts.A)) + sqrt_newton(fma(B.y, s.B, ts.A));
                        } else {
                            double2 C = make_double2(0.0, 0.0);
                            if constexpr (HAS_C) C = reinterpret_cast<const double2 *>(recA + 2 * RECS)[ri];
                            T2 = exact_time_samples<TT>(P, ts, s, B, C);
                        }
                        const double v = T2 + magic;
                        const unsigned vh = (unsigned)__double2hiint(v), vl = (unsigned)__double2loint(v);
                        const unsigned iu = __funnelshift_r(vl, vh, 21);
                        ok = iu < ns_m1;
                        i0 = ok ? (int)iu : 0;
                        f = __uint_as_float(0x3F800000u | ((vl & 0x1FFFFFu) << 2));   // 1 + fraction
                        T = TT == TT_STRAIGHT ? double_to_float_trunc(T2) : (float)T2;
                    } else {
                        const float4 B = reinterpret_cast<const float4 *>(recA + RECS)[ri];
                        float4 Cc = make_float4(0.f, 0.f, 0.f, 0.f);
                        if constexpr (HAS_C) Cc = reinterpret_cast<const float4 *>(recA + 2 * RECS)[ri];
                        T = traveltime<TT>(P, ts, s, B, Cc);
                        if constexpr (TT != TT_STRAIGHT) T = ts.tz ? 0.f : T;
                        float sidx = fmaf(T, s_scale, s_offset);
                        if constexpr (GUARD) {
                            const float x = fabsf(sidx - g_mid);
                            const bool fast_ok = ts.tz ? ts.tz_in : (x <= g_in);
                            const bool band = !fast_ok && !ts.tz && x <= g_out;
                            if constexpr (TT != TT_STRAIGHT) sidx = ts.tz ? fminf(fmaxf(sidx, 0.f), s_clamp) : sidx;
                            ok = fast_ok;
                            pmask |= band ? (1u << c) : 0u;
                            sidx = ok ? sidx : 0.f;
                        } else {   // FP32 trace-end test, as in `pair`
                            const float sc = fminf(fmaxf(sidx, 0.f), s_clamp);
                            bool in = sc == sidx;
                            if constexpr (TT != TT_STRAIGHT) in = ts.tz ? ts.tz_in : in;
                            ok = in;
                            sidx = sc;
                        }
                        const float fl = __fadd_rd(sidx, 8388608.f);
                        i0 = __float_as_int(fl) - 0x4B000000;
                        f = sidx - (fl - 8388608.f);
                    }
                    const unsigned char *row = ampb + roff;
                    a0 = amp_at<AMP>(row, i0);
                    a1 = amp_at<AMP>(row, i0 + 1);
                    w = ok ? A.y : 0.f;
                    mz = A.z;
                };
                auto plain2 = [&](int c, float2 &acc) {
                    float2 a0, a1, f, T, w, mz;
                    front(c, a0.x, a1.x, f.x, T.x, w.x, mz.x);
                    front(c + 1, a0.y, a1.y, f.y, T.y, w.y, mz.y);
                    const float2 m1 = make_float2(-1.f, -1.f);
                    if constexpr (EXACT) f = __fadd2_rn(f, m1);   // the fraction, exactly
                    const float2 amp = __ffma2_rn(f, __ffma2_rn(a0, m1, a1), a0);
                    const float2 rT = make_float2(rcp_approx(T.x), rcp_approx(T.y));
                    const float2 K2 = make_float2(s.K, s.K);
                    float2 g;
                    if (W2 || w_two) g = __fmul2_rn(__fmul2_rn(K2, rT), rT);
                    else if (w_one) g = __fmul2_rn(K2, rT);
                    else g = make_float2(1.f, 1.f);
                    if (aa_on) {
                        const float2 u = __fmul2_rn(mz, rT);
                        float2 y = __ffma2_rn(u, make_float2(-s.aa_k, -s.aa_k), make_float2(1.f, 1.f));
                        y.x = u.x >= s.aa_thr ? fminf(fmaxf(y.x, aa_lo), aa_hi) : 1.f;
                        y.y = u.y >= s.aa_thr ? fminf(fmaxf(y.y, aa_lo), aa_hi) : 1.f;
                        g = __fmul2_rn(g, y);
                    }
                    acc = __ffma2_rn(amp, __fmul2_rn(w, g), acc);
                };
                using F = std::false_type;
                using Tr = std::true_type;
                float a = 0.f;
                const bool small_t = __any_sync(0xffffffffu, ts.tg >= 0.f);
                if (!hard_cut) {
                    if (small_t) {
                        PSTM_UNROLL(PSTM_UNROLL_TAPER)
                        for (int c = 0; c < n0; ++c) a += pair(c, F{}, F{}, F{}, Tr{}, Tr{});
                    } else if (PSTM_PACKED_PAIRS) {
                        float2 acc = make_float2(0.f, 0.f);
                        int c = 0;
                        PSTM_UNROLL(PSTM_UNROLL_PACKED)
                        for (; c + 1 < n0; c += 2) plain2(c, acc);
                        if (c < n0) a += pair(c, F{}, F{}, F{}, F{}, Tr{});
                        a += acc.x + acc.y;
                    } else {
                        PSTM_UNROLL(PSTM_UNROLL_PLAIN)
                        for (int c = 0; c < n0; ++c) a += pair(c, F{}, F{}, F{}, F{}, Tr{});
                    }
                    if (small_t) {
                        PSTM_UNROLL(PSTM_UNROLL_TAPER)
                        for (int c = n0; c < n; ++c) a += pair(c, Tr{}, F{}, F{}, Tr{}, F{});
                    } else {
                        PSTM_UNROLL(PSTM_UNROLL_TAPER)
                        for (int c = n0; c < n; ++c) a += pair(c, Tr{}, F{}, F{}, F{}, F{});
                    }
                } else {   // no taper: the aperture edge is a hard cut, ties are decided in FP64
                    PSTM_UNROLL(PSTM_UNROLL_TAPER)
                    for (int c = 0; c < n; ++c) a += pair(c, F{}, F{}, Tr{}, Tr{}, F{});
                }
                if constexpr (!EXACT && GUARD) {   // second pass over the flagged records only
                    unsigned m = __reduce_or_sync(0xffffffffu, pmask);
                    while (m) {
                        const int c = __ffs(m) - 1;
                        m &= m - 1u;
                        a += pair(c, Tr{}, Tr{}, Tr{}, Tr{}, F{});
                    }
                }
                float &sa = s_acc[(q * R + r) * kThreads + vt];
                if (comp) {   // TwoSum: sa + a = t + e exactly; the errors are kept apart
                    const float s0 = sa, t = s0 + a, bp = t - s0;
                    unsigned short &se = s_err[(q * R + r) * kThreads + vt];
                    se = f32_to_bf16(bf16_to_f32(se) + ((s0 - (t - bp)) + (a - bp)));
                    sa = t;
                } else {
                    sa += a;
                }
            }
        }

        // ---------------- records of chunk k+1 (its copy was issued a chunk ago)
        bool timeout = false;
        if (k + 1 < n_chunks) {
            const int nb = buf ^ 1;
            timeout = !mbar_wait(nb ? bar1 : bar0, (uint32_t)(((g + 1) >> 1) & 1), wait_iters);
            if (!timeout) build_records(k + 1, nb);
        }
        if ((k + 1) % flush_every == 0) flush();
        if (__syncthreads_or(timeout)) {   // also: buffer `buf` is free again
            aborted = true;
            break;
        }
        if (tid == 0 && k + 2 < n_chunks) {
            fence_proxy_async();
            issue_chunk(k + 2, buf);
        }
    }

    chunk_base += n_chunks;
    if (aborted) {
        // a copy never completed: report, drain what may still be in flight, leave
        if (tid == 0) {
            atomicOr(P.err, (int)KERR_WAIT_TIMEOUT);
            mbar_wait(bar0, 0, wait_iters);
            mbar_wait(bar0, 1, wait_iters);
            mbar_wait(bar1, 0, wait_iters);
            mbar_wait(bar1, 1, wait_iters);
        }
        __syncthreads();
        return false;
    }

    // ---------------- epilogue: image += the last partials; fold += count
    flush();
    if (it.fold && P.fold3d) {
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const int p = s_pid[q];
            if (p < 0) continue;
            const int cnt = s_fold[q];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int t = t_lane + r * kThreads;
                if (t < P.nt) {
                    int32_t *f = it.fold + (int64_t)p * P.nt + t;
                    if (P.atomic_flush) atomicAdd(f, cnt);
                    else *f += cnt;
                }
            }
        }
    }
    if (it.fold && !P.fold3d && it.tblock == 0 && tid < PB) {
        const int p = s_pid[tid];
        if (p >= 0) {
            if (P.atomic_flush) atomicAdd(it.fold + p, s_fold[tid]);
            else it.fold[p] += s_fold[tid];
        }
    }
    return true;
}

// Initialises the two staging mbarriers of a CTA.
__device__ __forceinline__ void init_barriers(CtaShared &sh) {
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&sh.bar[0]), 1);
        mbar_init(smem_u32(&sh.bar[1]), 1);
        fence_barrier_init();
    }
}

// One CTA per (pillar block, time block) of one tile.
template <int TT, int AMP, bool VEL3D, bool EXACT, bool W2, bool GUARD>
__global__ void __launch_bounds__(kThreads, 1)
migrate_kernel(const KParams P, const KParams *__restrict__ Pg) {
    static_assert(kMaxPB <= kThreads / 32, "one warp per pillar builds the records");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ CtaShared sh;
    init_barriers(sh);
    Item it;
    it.amps = reinterpret_cast<const unsigned char *>(P.amps);
    it.geo = P.geo;
    it.trace0 = 0;
    it.n_traces = P.n_traces;
    it.image = P.image;
    it.fold = P.fold;
    it.pbx = blockIdx.x / P.n_pblk_y;
    it.pby = blockIdx.x - it.pbx * P.n_pblk_y;
    it.tblock = blockIdx.y;
    int64_t chunk_base = 0;
    migrate_item<TT, AMP, VEL3D, EXACT, W2, GUARD>(P, Pg, it, smem, sh, chunk_base);
}

// Persistent form for many outputs (offset bins): one CTA per SM fetches
// items from a work counter; items of the bins with the most traces come
// first (the host orders `bins`), so uneven bins balance.  With a scatter
// schedule (sw.boxes non-null) the items are (segment, pillar block, time
// block) of P.image / P.fold, numbered segment by segment; an item finds its
// segment by binary search in the segments' inclusive prefix counts.
template <int TT, int AMP, bool VEL3D, bool EXACT, bool W2, bool GUARD>
__global__ void __launch_bounds__(kThreads, 1)
migrate_persistent_kernel(const KParams P, const KParams *__restrict__ Pg, const BinWork *__restrict__ bins,
                          int n_bins, unsigned long long *work_counter, const ScatterWork sw) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ CtaShared sh;
    init_barriers(sh);
    const int n_pblk_x = (P.nx + P.px - 1) / P.px;
    const long long per_bin = (long long)n_pblk_x * P.n_pblk_y * P.n_tblk;
    const long long n_items = sw.boxes ? (sw.n_seg > 0 ? sw.ends[sw.n_seg - 1] : 0) : per_bin * n_bins;
    int64_t chunk_base = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sh.item = (long long)atomicAdd(work_counter, 1ull);
        __syncthreads();
        const long long item = sh.item;
        if (item >= n_items) break;
        if (sw.boxes) {
            __shared__ int64_t s_seg;
            if (threadIdx.x == 0) {   // the first segment whose inclusive count exceeds the item
                int64_t lo = 0, hi = sw.n_seg - 1;
                while (lo < hi) {
                    const int64_t mid = (lo + hi) >> 1;
                    if (sw.ends[mid] > item) hi = mid;
                    else lo = mid + 1;
                }
                s_seg = lo;
            }
            __syncthreads();
            const int64_t seg = s_seg;
            const SegmentBox bx = sw.boxes[seg];
            long long k = item - (seg > 0 ? sw.ends[seg - 1] : 0);
            const int nby = bx.pby1 - bx.pby0 + 1;
            Item it;
            it.tblock = (int)(k % P.n_tblk);
            k /= P.n_tblk;
            it.pby = bx.pby0 + (int)(k % nby);
            it.pbx = bx.pbx0 + (int)(k / nby);
            it.trace0 = seg * sw.seg_traces;
            it.n_traces = min(sw.seg_traces, P.n_traces - it.trace0);
            it.amps = reinterpret_cast<const unsigned char *>(P.amps) + it.trace0 * P.amp_stride * P.elem;
            it.geo = P.geo + it.trace0 * kGeoDoubles;
            it.image = P.image;
            it.fold = P.fold;
            if (!migrate_item<TT, AMP, VEL3D, EXACT, W2, GUARD>(P, Pg, it, smem, sh, chunk_base)) break;
            continue;
        }
        const BinWork &bw = bins[item / per_bin];
        long long rem = item - (item / per_bin) * per_bin;
        Item it;
        it.tblock = (int)(rem % P.n_tblk);
        rem /= P.n_tblk;
        it.pbx = (int)(rem / P.n_pblk_y);
        it.pby = (int)(rem - (long long)it.pbx * P.n_pblk_y);
        it.trace0 = bw.trace0;
        it.n_traces = bw.n_traces;
        it.amps = reinterpret_cast<const unsigned char *>(P.amps) + bw.trace0 * P.amp_stride * P.elem;
        it.geo = P.geo + bw.trace0 * kGeoDoubles;
        it.image = bw.image;
        it.fold = bw.fold;
        if (!migrate_item<TT, AMP, VEL3D, EXACT, W2, GUARD>(P, Pg, it, smem, sh, chunk_base)) break;
    }
}

// Per-time tables: 2 x float4 {t0h2, Kt, tg, tguard}, {vz, vz2, 1/vz, t0==0}
// and double A, per output time; per-(pillar|0, time) tables {1/v^2,
// aperture, 1/v, eta} and 1/(v dt)^2; all evaluated in FP64 as
// numba_cpu_optimized.py:378-399 does, the float4s rounded once to FP32.
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab, double *btab, float4 *ttime,
                                double *ttimeA);

// Packed FP64 trace geometry, kGeoDoubles per trace: sx sy rx ry mx my w 0.
__global__ void pack_geometry(const KParams P, double *geo);

}  // namespace pstm
