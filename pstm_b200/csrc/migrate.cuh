// migrate.cuh -- gather-form Kirchhoff PSTM kernel for sm_100a.
//
// One CTA (16 warps) owns a patch of PB output pillars and a block of
// kWarpsT * 32 * R consecutive output times.  The warps form kWarpsP pillar
// groups x kWarpsT time groups; a lane owns R output times (t = base + r*32 +
// lane) for the PBG = PB / kWarpsP pillars of its group and keeps their sums in
// registers.  Traces are streamed in chunks of C:
//   staging  the chunk's amplitude rows are copied into shared memory by TMA
//            bulk copies (cp.async.bulk + mbarrier), double-buffered, so the
//            copy of chunk k+1 overlaps the arithmetic of chunk k;
//   phase A  every (pillar, trace) pair of the chunk gets a record in shared
//            memory (FP64 geometry rounded once to FP32); the fold predicate
//            is evaluated in FP64 and counted with warp match/ballot + popc;
//   phase B  every lane walks the records (warp-uniform broadcast reads) and,
//            for each of its R times, evaluates traveltime, the sample index,
//            the linear interpolation (from shared memory) and the weights.
// Chunk partials are folded into compensated (TwoSum) FP32 sums and the
// epilogue adds them once into the caller's image (+=) and fold.
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
// and decisions that are discontinuous in the inputs (aperture cut, trace-end
// bounds) are re-taken in FP64 inside a guard band.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include "kparams.h"

namespace pstm {

constexpr int kWarpsT = 8;                         // warps along time
constexpr int kWarpsP = 2;                         // warp groups along pillars
constexpr int kThreads = 32 * kWarpsT * kWarpsP;   // 512
constexpr int kMaxChunk = 32;                      // traces per chunk, upper bound
constexpr int kWaitIters = 1 << 20;                // bound of every mbarrier wait loop

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
// Bounded wait for the mbarrier phase with the given parity; false = gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kWaitIters; ++i) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// ---------------------------------------------------------------- per-time state
// Quantities that depend on the output time only (one copy per lane and r).
struct TimeState {
    float t0, t0h2;
    float Kt;              // obliquity numerator t0 (in the weight's time unit) or 1
    float tguard;          // T <= tguard means "T <= 1 ms" (in the unit of T)
    float vz, vz2, ivwc;   // curved: velocity at image depth, 1/vz
    double A;              // EXACT: (t0 / (2 dt))^2
    bool valid, guard, tzero;
};

// Quantities that depend on (pillar, time): from the per-pillar tables.
struct PtState {
    float iv2, ap, itw, tsn;
    float K;               // weight numerator
    float ivw_t;           // 1/v_w in the weight's time unit (AA sin theta)
    float ivw;             // 1/v_w in s/m (AA f_max)
    float t02v2, c1, e2;   // VTI: (t0/2)^2 v^2, 1+2eta, 2 eta / v^2
    double B;              // EXACT: 1/(v dt)^2
};

template <int TT, bool EXACT>
__device__ __forceinline__ void make_time_state(const KParams &P, int t, TimeState &s) {
    s.valid = t < P.nt;
    const int tc = s.valid ? t : (P.nt - 1);
    const double t0 = P.ta[tc] / 1000.0;
    const double tu = EXACT ? P.dt_s : 1.0;   // weights' time unit: seconds, or samples
    s.t0 = (float)t0;
    s.t0h2 = (float)((t0 * 0.5) * (t0 * 0.5));
    s.Kt = P.obliquity ? (float)(t0 / tu) : 1.f;
    s.tguard = (float)(0.001 / tu);
    s.vz = 0.f;
    s.vz2 = 0.f;
    s.ivwc = 0.f;
    if constexpr (TT == TT_CURVED || TT == TT_CURVED_VTI) {
        const double z = P.cr_k_zero ? P.cr_v0 * (t0 * 0.5) : (P.cr_v0 / P.cr_k) * (exp(P.cr_k * (t0 * 0.5)) - 1.0);
        const double vz = P.cr_v0 + P.cr_k * z;
        s.vz = (float)vz;
        s.vz2 = (float)(vz * vz);
        s.ivwc = (float)(1.0 / vz);
    }
    const double th = t0 * 0.5 / P.dt_s;
    s.A = EXACT ? th * th : 0.0;
    s.guard = t0 < 0.0011;
    s.tzero = !(t0 > 0.0);
}

template <int TT, bool EXACT>
__device__ __forceinline__ void make_pt_state(const KParams &P, const TimeState &ts, float4 tab, double b,
                                              PtState &s) {
    s.iv2 = tab.x;
    s.ap = tab.y;
    const float width = s.ap * P.taper_f;
    if (width > 0.f) {
        s.itw = rcp_approx(width);
        s.tsn = -(s.ap * (1.f - P.taper_f)) * s.itw;
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
    const float inv_tu = EXACT ? (float)(1.0 / P.dt_s) : 1.f;
    s.ivw = ivw;
    s.ivw_t = ivw * inv_tu;
    s.K = P.spreading ? ts.Kt * s.ivw_t : ts.Kt;
    s.t02v2 = 0.f;
    s.c1 = 1.f;
    s.e2 = 0.f;
    if constexpr (TT == TT_VTI || TT == TT_CURVED_VTI) {
        s.t02v2 = ts.t0h2 * rcp_approx(tab.x);   // (t0/2)^2 v^2
        s.c1 = 1.f + 2.f * tab.w;
        s.e2 = 2.f * tab.w * tab.x;
    }
    s.B = b;
}

// ---------------------------------------------------------------- FP64 exact decisions
// (rare paths: they read the launch parameters from a global copy, so the
// kernel's own parameter block never has its address taken)
template <int TT>
__device__ double exact_traveltime(const KParams *P, int64_t tr, int p, int t, double ox, double oy) {
    const double t0 = P->ta[t] / 1000.0;
    const double v = P->vel3d ? P->vrms[(int64_t)p * P->nt + t] : P->vrms[t];
    const double dxs = ox - P->sx[tr], dys = oy - P->sy[tr];
    const double dxr = ox - P->rx[tr], dyr = oy - P->ry[tr];
    const double ds2 = dxs * dxs + dys * dys, dr2 = dxr * dxr + dyr * dyr;
    const double t0h = t0 * 0.5;
    double eta = P->eta_const;
    if (P->eta) eta = P->eta3d ? P->eta[(int64_t)p * P->nt + t] : P->eta[t];
    auto vti_corr = [&](double h2) {
        const double v2 = v * v;
        const double den = v2 * (t0h * t0h * v2 + (1.0 + 2.0 * eta) * h2);
        return fabs(den) > 1e-20 ? (2.0 * eta * h2 * h2) / den : 0.0;
    };
    auto curved_leg = [&](double h2) {
        const double k = P->cr_k, v0 = P->cr_v0;
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
// rec0 = {ds2, dr2, d, wt}; rec1/rec2 kind-specific (see phase A).  Seconds.
template <int TT>
__device__ __forceinline__ float traveltime(const KParams &P, const TimeState &ts, const PtState &s,
                                            const float4 &r0, const float4 &r1, const float4 &r2) {
    if constexpr (TT == TT_STRAIGHT) {
        return sqrt_approx(fmaf(r0.x, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(r0.y, s.iv2, ts.t0h2));
    } else if constexpr (TT == TT_CURVED) {
        if (P.cr_k_zero) {
            return sqrt_approx(fmaf(r0.x, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(r0.y, s.iv2, ts.t0h2));
        }
        const float a = ts.vz + sqrt_approx(ts.vz2 + r1.y);
        const float b = ts.vz + sqrt_approx(ts.vz2 + r1.z);
        return P.cr_inv_k_ln2 * lg2_approx(a * b * r1.w);
    } else if constexpr (TT == TT_VTI) {
        if (ts.tzero) return 0.f;
        const float Ds = fmaf(s.c1, r0.x, s.t02v2);
        const float Dr = fmaf(s.c1, r0.y, s.t02v2);
        const float rr = rcp_approx(Ds * Dr);
        const float qs = fmaf(-(s.e2 * r1.y), Dr * rr, fmaf(r0.x, s.iv2, ts.t0h2));
        const float qr = fmaf(-(s.e2 * r1.z), Ds * rr, fmaf(r0.y, s.iv2, ts.t0h2));
        return sqrt_approx(fmaxf(qs, 0.f)) + sqrt_approx(fmaxf(qr, 0.f));
    } else {
        float tcs, tcr;
        if (P.cr_k_zero) {
            tcs = sqrt_approx(fmaf(r0.x, s.iv2, ts.t0h2));
            tcr = sqrt_approx(fmaf(r0.y, s.iv2, ts.t0h2));
        } else {
            const float a = ts.vz + sqrt_approx(ts.vz2 + r1.y);
            const float b = ts.vz + sqrt_approx(ts.vz2 + r1.z);
            tcs = P.cr_inv_k_ln2 * lg2_approx(a * r1.w);
            tcr = P.cr_inv_k_ln2 * lg2_approx(b * r2.x);
        }
        if (ts.tzero) return tcs + tcr;
        // leg = t_curved * sqrt(1 - corr / (t0h^2 + h^2/v^2)), corr = e2 h^4 / D
        const float Hs = fmaf(r0.x, s.iv2, ts.t0h2), Hr = fmaf(r0.y, s.iv2, ts.t0h2);
        const float Ds = fmaf(s.c1, r0.x, s.t02v2), Dr = fmaf(s.c1, r0.y, s.t02v2);
        const float ps_ = Ds * Hs, pr_ = Dr * Hr;
        const float rr = rcp_approx(ps_ * pr_);
        const float xs = s.e2 * r2.y * (pr_ * rr), xr = s.e2 * r2.z * (ps_ * rr);
        return tcs * sqrt_approx(fmaxf(1.f - xs, 0.f)) + tcr * sqrt_approx(fmaxf(1.f - xr, 0.f));
    }
}

template <int TT, bool AA>
struct RecCount {
    static constexpr int value = (TT == TT_CURVED_VTI) ? 3 : ((TT == TT_STRAIGHT && !AA) ? 1 : 2);
};

// Record area of the dynamic shared memory (after the two staging buffers).
__host__ __device__ constexpr int records_bytes(int PB, int nrec, bool exact) {
    return PB * kMaxChunk * (16 * nrec + (exact ? 16 : 0));
}

// ---------------------------------------------------------------- the kernel
template <int TT, int AMP, bool VEL3D, bool AA, bool EXACT, int R, int PBG>
__global__ void __launch_bounds__(kThreads, 1)
migrate_staged_kernel(const KParams P, const KParams *__restrict__ Pg) {
    static_assert(!EXACT || TT == TT_STRAIGHT, "the FP64 sample-index path is straight-ray only");
    constexpr int PB = PBG * kWarpsP;
    constexpr int NREC = RecCount<TT, AA>::value;
    constexpr int RECS = PB * kMaxChunk;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_ox[PB], s_oy[PB];
    __shared__ int s_pid[PB];
    __shared__ int s_fold[PB];
    __shared__ __align__(8) unsigned long long s_bar[2];

    const int C = P.chunk;
    const int buf_bytes = C * P.pitch * P.elem;
    float4 *s_rec = reinterpret_cast<float4 *>(smem + 2 * buf_bytes);     // [NREC][RECS]
    double2 *s_rec64 = reinterpret_cast<double2 *>(s_rec + NREC * RECS);  // [RECS] (EXACT)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wp = warp / kWarpsT, wt = warp - wp * kWarpsT;
    const int pbx = blockIdx.x / P.n_pblk_y, pby = blockIdx.x - pbx * P.n_pblk_y;
    if (tid < PB) {
        const int ix = pbx * P.px + tid / P.py, iy = pby * P.py + tid % P.py;
        const bool ok = (tid < P.px * P.py) && ix < P.nx && iy < P.ny;
        const int p = ok ? ix * P.ny + iy : -1;
        s_pid[tid] = p;
        s_fold[tid] = 0;
        s_ox[tid] = ok ? (P.xg ? P.xg[p] : P.xa[ix]) : 0.0;
        s_oy[tid] = ok ? (P.yg ? P.yg[p] : P.ya[iy]) : 0.0;
    }
    const uint32_t bar0 = smem_u32(&s_bar[0]), bar1 = smem_u32(&s_bar[1]);
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        fence_barrier_init();
    }
    const int t_base = blockIdx.y * (kWarpsT * 32 * R) + wt * (32 * R) + lane;

    // hot-loop constants in registers
    const float s_scale = P.s_scale, s_offset = P.s_offset;
    const float sg_lo = P.s_guard_lo, sg_hi = P.s_guard_hi, sr_lo = P.s_rej_lo, sr_hi = P.s_rej_hi;
    const float s_clamp = P.s_max_clamp;
    const unsigned ns_m1 = (unsigned)(P.ns - 1);
    const double magic = P.s_magic;
    const float ap_max_f = P.ap_max_f;
    const int nw = P.spreading + P.obliquity;
    const float aa_cA = P.aa_cA, aa_cB = P.aa_cB;
    const int row_bytes = P.pitch * P.elem;
    const int64_t n_chunks = (P.n_traces + C - 1) / C;

    TimeState ts[R];
    PtState ps[R];
#pragma unroll
    for (int r = 0; r < R; ++r) make_time_state<TT, EXACT>(P, t_base + r * 32, ts[r]);
    if constexpr (!VEL3D) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = min(t_base + r * 32, P.nt - 1);
            make_pt_state<TT, EXACT>(P, ts[r], P.ttab[t], EXACT ? P.btab[t] : 0.0, ps[r]);
        }
    }

    float acc[PBG][R], hi[PBG][R], lo[PBG][R];
#pragma unroll
    for (int g = 0; g < PBG; ++g)
#pragma unroll
        for (int r = 0; r < R; ++r) { acc[g][r] = 0.f; hi[g][r] = 0.f; lo[g][r] = 0.f; }

    // copy the amplitude rows of chunk k into buffer b (one thread, TMA bulk)
    auto issue_chunk = [&](int64_t k, int b) {
        const int64_t c0 = k * C;
        const int rows = (int)min((int64_t)C, P.n_traces - c0);
        const uint32_t bar = b ? bar1 : bar0;
        mbar_expect_tx(bar, (uint32_t)(rows * row_bytes));
        const unsigned char *src = reinterpret_cast<const unsigned char *>(P.amps) + c0 * P.amp_stride * P.elem;
        const uint32_t dst = smem_u32(smem + b * buf_bytes);
        for (int i = 0; i < rows; ++i)
            bulk_g2s(dst + i * row_bytes, src + (int64_t)i * P.amp_stride * P.elem, (uint32_t)row_bytes, bar);
    };

    __syncthreads();
    if (P.bulk && tid == 0) {
        issue_chunk(0, 0);
        if (n_chunks > 1) issue_chunk(1, 1);
    }

    bool aborted = false;
    for (int64_t k = 0; k < n_chunks; ++k) {
        const int64_t c0 = k * C;
        const int buf = (int)(k & 1);
        const int cmax = (int)min((int64_t)C, P.n_traces - c0);
        // ---------------- phase A: (pillar, trace) records, FP64 geometry
        const int nrec = PB * C;
        for (int j = tid; j < ((nrec + 31) & ~31); j += kThreads) {
            const bool live = j < nrec;
            const int q = live ? j / C : PB - 1;
            const int c = live ? j - q * C : 0;
            const int64_t tr = c0 + c;
            const int p = s_pid[q];
            bool in = false;
            float4 r0 = make_float4(0.f, 0.f, __int_as_float(0x7f800000), 0.f);
            float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f), r2 = r1;
            double2 r64 = make_double2(0.0, 0.0);
            if (live && p >= 0 && c < cmax) {
                const double ox = s_ox[q], oy = s_oy[q];
                const double dxm = ox - P.mx[tr], dym = oy - P.my[tr];
                const double d2 = dxm * dxm + dym * dym;
                in = d2 <= P.fold_d2_max;
                if (in) {
                    const double dxs = ox - P.sx[tr], dys = oy - P.sy[tr];
                    const double dxr = ox - P.rx[tr], dyr = oy - P.ry[tr];
                    const double ds2 = dxs * dxs + dys * dys, dr2 = dxr * dxr + dyr * dyr;
                    const float wt = P.w ? (float)P.w[tr] : 1.f;
                    r0 = make_float4((float)ds2, (float)dr2, (float)sqrt(d2), wt);
                    r64 = make_double2(ds2, dr2);
                    const float minf = (float)fmax(fabs(dxm), fabs(dym));
                    if constexpr (TT == TT_CURVED || TT == TT_CURVED_VTI) {
                        const double k2 = P.cr_k * P.cr_k, v0 = P.cr_v0;
                        const double bs = v0 + sqrt(v0 * v0 + k2 * ds2);
                        const double br = v0 + sqrt(v0 * v0 + k2 * dr2);
                        if constexpr (TT == TT_CURVED) {
                            r1 = make_float4(minf, (float)(k2 * ds2), (float)(k2 * dr2), (float)(1.0 / (bs * br)));
                        } else {
                            r1 = make_float4(minf, (float)(k2 * ds2), (float)(k2 * dr2), (float)(1.0 / bs));
                            r2 = make_float4((float)(1.0 / br), (float)(ds2 * ds2), (float)(dr2 * dr2), 0.f);
                        }
                    } else if constexpr (TT == TT_VTI) {
                        r1 = make_float4(minf, (float)(ds2 * ds2), (float)(dr2 * dr2), 0.f);
                    } else {
                        r1 = make_float4(minf, 0.f, 0.f, 0.f);
                    }
                }
            }
            // fold: lanes with the same pillar share one shared-memory add
            const unsigned peers = __match_any_sync(0xffffffffu, q);
            const unsigned ballot = __ballot_sync(0xffffffffu, in);
            if (lane == __ffs(peers) - 1) {
                const int cnt = __popc(ballot & peers);
                if (cnt) atomicAdd(&s_fold[q], cnt);
            }
            if (live) {
                const int ri = q * kMaxChunk + c;
                s_rec[ri] = r0;
                if constexpr (NREC > 1) s_rec[RECS + ri] = r1;
                if constexpr (NREC > 2) s_rec[2 * RECS + ri] = r2;
                if constexpr (EXACT) s_rec64[ri] = r64;
            }
        }
        if (!P.bulk) {   // rows not 16-byte aligned: plain cooperative copy
            unsigned char *dst = smem + buf * buf_bytes;
            const unsigned char *src = reinterpret_cast<const unsigned char *>(P.amps);
            const int per_row = P.ns;
            for (int e = tid; e < cmax * per_row; e += kThreads) {
                const int rr = e / per_row, ii = e - rr * per_row;
                const int64_t gi = (c0 + rr) * P.amp_stride + ii;
                if (P.elem == 4)
                    reinterpret_cast<float *>(dst + rr * row_bytes)[ii] = reinterpret_cast<const float *>(src)[gi];
                else
                    reinterpret_cast<unsigned short *>(dst + rr * row_bytes)[ii] =
                        reinterpret_cast<const unsigned short *>(src)[gi];
            }
        }
        __syncthreads();
        if (P.bulk) {
            const bool ok = mbar_wait(buf ? bar1 : bar0, (uint32_t)((k >> 1) & 1));
            if (__syncthreads_or(!ok)) {
                aborted = true;
                break;
            }
        }

        // ---------------- phase B: pairs
        const unsigned char *bufp = smem + buf * buf_bytes;
#pragma unroll
        for (int g = 0; g < PBG; ++g) {
            const int q = wp * PBG + g;
            const int p = s_pid[q];
            if (p < 0) continue;
            if constexpr (VEL3D) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int64_t ti = (int64_t)p * P.nt + min(t_base + r * 32, P.nt - 1);
                    make_pt_state<TT, EXACT>(P, ts[r], P.ttab[ti], EXACT ? P.btab[ti] : 0.0, ps[r]);
                }
            }
#pragma unroll 2
            for (int c = 0; c < cmax; ++c) {
                const int ri = q * kMaxChunk + c;
                const float4 r0 = s_rec[ri];
                if (!(r0.z <= ap_max_f)) continue;
                float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f), r2 = r1;
                if constexpr (NREC > 1) r1 = s_rec[RECS + ri];
                if constexpr (NREC > 2) r2 = s_rec[2 * RECS + ri];
                double2 r64 = make_double2(0.0, 0.0);
                if constexpr (EXACT) r64 = s_rec64[ri];
                const unsigned char *row = bufp + c * row_bytes;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const TimeState &t_ = ts[r];
                    const PtState &s = ps[r];
                    if (!t_.valid) continue;
                    if (r0.z >= s.ap) {
                        if (r0.z > s.ap) continue;
                        if (exact_outside_aperture(Pg, c0 + c, p, t_base + r * 32, s_ox[q], s_oy[q])) continue;
                    }
                    float T, f;
                    int i0;
                    if constexpr (EXACT) {
                        const double qs = fma(r64.x, s.B, t_.A);
                        const double qr = fma(r64.y, s.B, t_.A);
                        double T2;
                        if (!t_.guard) {
                            T2 = sqrt_newton(qs) + sqrt_newton(qr);
                        } else {
                            T2 = (qs > 0.0 ? sqrt_newton(qs) : 0.0) + (qr > 0.0 ? sqrt_newton(qr) : 0.0);
                        }
                        // s + 2^31 keeps s in the mantissa with 21 fraction bits
                        const double v = T2 + magic;
                        const unsigned vh = (unsigned)__double2hiint(v), vl = (unsigned)__double2loint(v);
                        const unsigned iu = __funnelshift_r(vl, vh, 21);
                        if (iu >= ns_m1) continue;   // also rejects s < 0 and NaN
                        i0 = (int)iu;
                        f = __uint_as_float(0x3F800000u | ((vl & 0x1FFFFFu) << 2)) - 1.0f;
                        T = t_.guard ? (float)T2 : double_to_float_trunc(T2);
                    } else {
                        T = traveltime<TT>(P, t_, s, r0, r1, r2);
                        float sidx = fmaf(T, s_scale, s_offset);
                        if (!(sidx >= sg_lo && sidx <= sg_hi)) {
                            if (!(sidx >= sr_lo && sidx <= sr_hi)) continue;
                            if (!exact_sample_ok<TT>(Pg, c0 + c, p, t_base + r * 32, s_ox[q], s_oy[q])) continue;
                            sidx = fminf(fmaxf(sidx, 0.f), s_clamp);
                        }
                        const float fl = __fadd_rd(sidx, 8388608.f);
                        i0 = __float_as_int(fl) - 0x4B000000;
                        f = sidx - (fl - 8388608.f);
                    }
                    const float a0 = amp_at<AMP>(row, i0);
                    const float a1 = amp_at<AMP>(row, i0 + 1);
                    const float amp = fmaf(f, a1 - a0, a0);
                    float w = r0.w;
                    const float x = fmaf(r0.z, s.itw, s.tsn);
                    if (x > 0.f) w *= 0.5f + 0.5f * __cosf(3.14159265358979f * x);
                    const float rT = rcp_approx(T);
                    float gw = 1.f;
                    if (nw) {
                        gw = s.K * rT;
                        if (nw == 2) gw *= rT;
                    }
                    constexpr bool kSmallT = (TT == TT_CURVED || TT == TT_CURVED_VTI);
                    if ((kSmallT || t_.guard) && !(T > t_.tguard)) gw = 1.f;
                    if constexpr (AA) {
                        if (T >= t_.tguard) {
                            const float sth = fminf(r1.x * s.ivw_t * rT, 1.f);
                            if (sth >= 0.01f) gw *= fmaxf(0.f, 1.f - fmaxf(aa_cA * sth * s.ivw, aa_cB));
                        }
                    }
                    acc[g][r] = fmaf(amp, w * gw, acc[g][r]);
                }
            }
        }
        // fold chunk partials into the compensated sums
#pragma unroll
        for (int g = 0; g < PBG; ++g)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float y = acc[g][r];
                if (P.compensated) {
                    const float sum = hi[g][r] + y;
                    const float bp = sum - hi[g][r];
                    lo[g][r] += (hi[g][r] - (sum - bp)) + (y - bp);
                    hi[g][r] = sum;
                } else {
                    hi[g][r] += y;
                }
                acc[g][r] = 0.f;
            }
        __syncthreads();   // buffer `buf` and the records are free again
        if (P.bulk && tid == 0 && k + 2 < n_chunks) {
            fence_proxy_async();
            issue_chunk(k + 2, buf);
        }
    }

    if (aborted) {
        // a copy never completed: report, drain what is still in flight, and leave
        if (tid == 0) {
            atomicOr(P.err, (int)KERR_WAIT_TIMEOUT);
            mbar_wait(bar0, 0);
            mbar_wait(bar0, 1);
            mbar_wait(bar1, 0);
            mbar_wait(bar1, 1);
        }
        __syncthreads();
        return;
    }

    // ---------------- epilogue: image += sum; fold += count
#pragma unroll
    for (int g = 0; g < PBG; ++g) {
        const int q = wp * PBG + g;
        const int p = s_pid[q];
        if (p < 0) continue;
        const int cnt = s_fold[q];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = t_base + r * 32;
            if (t >= P.nt) continue;
            const int64_t idx = (int64_t)p * P.nt + t;
            if (P.image_f32) {
                float *img = reinterpret_cast<float *>(P.image);
                img[idx] += hi[g][r] + lo[g][r];
            } else {
                double *img = reinterpret_cast<double *>(P.image);
                img[idx] += (double)hi[g][r] + (double)lo[g][r];
            }
            if (P.fold && P.fold3d) P.fold[idx] += cnt;
        }
    }
    if (P.fold && !P.fold3d && blockIdx.y == 0 && tid < PB) {
        const int p = s_pid[tid];
        if (p >= 0) P.fold[p] += s_fold[tid];
    }
}

// Per-(pillar|0, time) tables: {1/v^2, aperture, 1/v, eta} and 1/(v dt)^2,
// evaluated in FP64 as numba_cpu_optimized.py:378-399 does, the first rounded
// once to FP32.
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab, double *btab);

}  // namespace pstm
