// migrate.cuh -- gather-form Kirchhoff PSTM kernel for sm_100a.
//
// One CTA owns a patch of PB output pillars (px x py) and a block of
// 8 warps * 32 lanes * R consecutive output times; every lane owns R output
// times (t = base + r*32 + lane) for all PB pillars and keeps their partial
// sums in registers.  Traces are streamed in chunks of C:
//   phase A  every (pillar, trace) pair of the chunk gets a record in shared
//            memory (FP64 geometry rounded once to FP32), the fold predicate is
//            evaluated in FP64 and counted with a warp ballot + popc;
//   phase B  every lane walks the records (warp-uniform broadcast reads) and,
//            for each of its R times, evaluates traveltime, the sample index,
//            the linear interpolation and the weights, and accumulates.
// Chunk partials are folded into compensated (TwoSum) FP32 sums, and the
// epilogue adds them once into the caller's image (+=) and fold.
//
// Reference semantics (paths relative to the reference project):
//   loop structure, fold, aperture, taper, weights  numba_cpu_optimized.py:147-231
//   per-time terms                                   numba_cpu_optimized.py:358-401
//   triangle AA weight                               pstm_migration.metal:95-132
//   curved-ray leg                                   pstm_curved_ray.metal:50-96
//   VTI leg                                          pstm_anisotropic_vti.metal:103-148
//
// Decisions that are discontinuous in the inputs (aperture cut, trace-end
// bounds) are taken in FP32 with a guard band and re-decided in FP64 inside
// the band, so that they agree with the FP64 reference.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include "kparams.h"

namespace pstm {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

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

template <int AMP>
__device__ __forceinline__ float load_amp(const void *base, int64_t idx) {
    if constexpr (AMP == AMP_F32) {
        return __ldg(reinterpret_cast<const float *>(base) + idx);
    } else if constexpr (AMP == AMP_BF16) {
        unsigned short u = __ldg(reinterpret_cast<const unsigned short *>(base) + idx);
        return __uint_as_float(((unsigned int)u) << 16);
    } else {
        return __half2float(__ldg(reinterpret_cast<const __half *>(base) + idx));
    }
}

// ---------------------------------------------------------------- per-time state
struct TState {
    float t0, t0h2, iv2, ap;
    float itw, tsn;        // taper: x = d*itw + tsn, taper when x > 0
    float K, ivw;          // weight numerator, 1/v_w (AA)
    float vz, vz2;         // curved: velocity at image depth
    float t02v2, c1, e2;   // VTI: t0h^2 v^2, 1+2eta, 2 eta / v^2
    bool valid, guard, tzero;
};

template <int TT>
__device__ __forceinline__ void make_tstate(const KParams &P, int t, float4 tab, TState &s) {
    s.valid = t < P.nt;
    const int tc = s.valid ? t : (P.nt - 1);
    const double t0 = P.ta[tc] / 1000.0;
    s.t0 = (float)t0;
    s.t0h2 = (float)((t0 * 0.5) * (t0 * 0.5));
    s.iv2 = tab.x;
    s.ap = tab.y;
    const float width = s.ap * P.taper_f;
    if (width > 0.f) {
        s.itw = 1.f / width;
        s.tsn = -(s.ap * (1.f - P.taper_f)) * s.itw;
    } else {
        s.itw = 0.f;
        s.tsn = -1.f;
    }
    float ivw = tab.w;
    s.vz = 0.f;
    s.vz2 = 0.f;
    if constexpr (TT == TT_CURVED || TT == TT_CURVED_VTI) {
        double z = P.cr_k_zero ? P.cr_v0 * (t0 * 0.5) : (P.cr_v0 / P.cr_k) * (exp(P.cr_k * (t0 * 0.5)) - 1.0);
        double vz = P.cr_v0 + P.cr_k * z;
        s.vz = (float)vz;
        s.vz2 = (float)(vz * vz);
        ivw = (float)(1.0 / vz);
        // |k| ~ 0: straight rays in the constant velocity v0 (curved_ray.py:35-38)
        if (P.cr_k_zero) s.iv2 = (float)(1.0 / (P.cr_v0 * P.cr_v0));
    }
    s.ivw = ivw;
    float K = 1.f;
    if (P.spreading) K *= ivw;
    if (P.obliquity) K *= s.t0;
    s.K = K;
    s.t02v2 = 0.f;
    s.c1 = 1.f;
    s.e2 = 0.f;
    if constexpr (TT == TT_VTI || TT == TT_CURVED_VTI) {
        const float v = 1.f / tab.w;   // tab.w = 1/v
        s.t02v2 = s.t0h2 * v * v;
        s.c1 = 1.f + 2.f * tab.z;
        s.e2 = 2.f * tab.z * s.iv2;
    }
    s.guard = t0 < 0.0011;
    s.tzero = !(t0 > 0.0);
}

// ---------------------------------------------------------------- FP64 exact decisions
template <int TT>
__device__ double exact_traveltime(const KParams &P, int64_t tr, int p, int t, double ox, double oy) {
    const double t0 = P.ta[t] / 1000.0;
    const double v = P.vel3d ? P.vrms[(int64_t)p * P.nt + t] : P.vrms[t];
    const double dxs = ox - P.sx[tr], dys = oy - P.sy[tr];
    const double dxr = ox - P.rx[tr], dyr = oy - P.ry[tr];
    const double ds2 = dxs * dxs + dys * dys, dr2 = dxr * dxr + dyr * dyr;
    const double t0h = t0 * 0.5;
    double eta = P.eta_const;
    if (P.eta) eta = P.eta3d ? P.eta[(int64_t)p * P.nt + t] : P.eta[t];
    auto vti_corr = [&](double h2) {
        const double v2 = v * v;
        const double den = v2 * (t0h * t0h * v2 + (1.0 + 2.0 * eta) * h2);
        return fabs(den) > 1e-20 ? (2.0 * eta * h2 * h2) / den : 0.0;
    };
    auto curved_leg = [&](double h2) {
        const double k = P.cr_k, v0 = P.cr_v0;
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
            const double q = tc * tc - vti_corr(h2);
            return sqrt(q > 0.0 ? q : 0.0);
        };
        return leg(ds2) + leg(dr2);
    }
}

// Is the FP64 sample index of this pair inside [0, ns-1)?
template <int TT>
__device__ __noinline__ bool exact_sample_ok(const KParams &P, int64_t tr, int p, int t, double ox, double oy) {
    const double T = exact_traveltime<TT>(P, tr, p, t, ox, oy);
    const double s = (T - P.tstart_s) / P.dt_s;
    return s >= 0.0 && s < (double)(P.ns - 1);
}

// Is the midpoint outside the time-varying aperture, decided in FP64?
static __device__ __noinline__ bool exact_outside_aperture(const KParams &P, int64_t tr, int p, int t, double ox, double oy) {
    const double dx = ox - P.mx[tr], dy = oy - P.my[tr];
    const double d = sqrt(dx * dx + dy * dy);
    const double v = P.vel3d ? P.vrms[(int64_t)p * P.nt + t] : P.vrms[t];
    double ap = v * (P.ta[t] / 1000.0) * 0.5 * P.tan_dip;
    if (ap < P.min_ap) ap = P.min_ap;
    else if (ap > P.max_ap) ap = P.max_ap;
    return d > ap;
}

// ---------------------------------------------------------------- traveltime (FP32)
// rec0 = {ds2, dr2, d, wt}; rec1/rec2 kind-specific (see phase A).
template <int TT>
__device__ __forceinline__ float traveltime(const KParams &P, const TState &s, const float4 &r0,
                                            const float4 &r1, const float4 &r2) {
    if constexpr (TT == TT_STRAIGHT) {
        return sqrt_approx(fmaf(r0.x, s.iv2, s.t0h2)) + sqrt_approx(fmaf(r0.y, s.iv2, s.t0h2));
    } else if constexpr (TT == TT_CURVED) {
        if (P.cr_k_zero) {
            return sqrt_approx(fmaf(r0.x, s.iv2, s.t0h2)) + sqrt_approx(fmaf(r0.y, s.iv2, s.t0h2));
        }
        const float a = s.vz + sqrt_approx(s.vz2 + r1.y);
        const float b = s.vz + sqrt_approx(s.vz2 + r1.z);
        return P.cr_inv_k_ln2 * lg2_approx(a * b * r1.w);
    } else if constexpr (TT == TT_VTI) {
        if (s.tzero) return 0.f;
        const float Ds = fmaf(s.c1, r0.x, s.t02v2);
        const float Dr = fmaf(s.c1, r0.y, s.t02v2);
        const float rr = rcp_approx(Ds * Dr);
        const float qs = fmaf(-(s.e2 * r1.y), Dr * rr, fmaf(r0.x, s.iv2, s.t0h2));
        const float qr = fmaf(-(s.e2 * r1.z), Ds * rr, fmaf(r0.y, s.iv2, s.t0h2));
        return sqrt_approx(fmaxf(qs, 0.f)) + sqrt_approx(fmaxf(qr, 0.f));
    } else {
        float tcs, tcr;
        if (P.cr_k_zero) {
            tcs = sqrt_approx(fmaf(r0.x, s.iv2, s.t0h2));
            tcr = sqrt_approx(fmaf(r0.y, s.iv2, s.t0h2));
        } else {
            const float a = s.vz + sqrt_approx(s.vz2 + r1.y);
            const float b = s.vz + sqrt_approx(s.vz2 + r1.z);
            tcs = P.cr_inv_k_ln2 * lg2_approx(a * r1.w);
            tcr = P.cr_inv_k_ln2 * lg2_approx(b * r2.x);
        }
        if (s.tzero) return tcs + tcr;
        const float Ds = fmaf(s.c1, r0.x, s.t02v2);
        const float Dr = fmaf(s.c1, r0.y, s.t02v2);
        const float rr = rcp_approx(Ds * Dr);
        const float qs = fmaf(-(s.e2 * r2.y), Dr * rr, tcs * tcs);
        const float qr = fmaf(-(s.e2 * r2.z), Ds * rr, tcr * tcr);
        return sqrt_approx(fmaxf(qs, 0.f)) + sqrt_approx(fmaxf(qr, 0.f));
    }
}

template <int TT, bool AA>
struct RecCount {
    static constexpr int value = (TT == TT_CURVED_VTI) ? 3 : ((TT == TT_STRAIGHT && !AA) ? 1 : 2);
};

// ---------------------------------------------------------------- the kernel
template <int TT, int AMP, bool VEL3D, bool AA, int R, int PB, int C>
__global__ void __launch_bounds__(kThreads, 2) migrate_gather_kernel(const KParams P) {
    constexpr int NREC = RecCount<TT, AA>::value;
    static_assert(C % 32 == 0, "chunk must be a multiple of the warp width");
    __shared__ float4 s_rec[NREC][PB * C];
    __shared__ double s_ox[PB], s_oy[PB];
    __shared__ int s_pid[PB];
    __shared__ int s_fold[PB];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pbx = blockIdx.x / P.n_pblk_y, pby = blockIdx.x - pbx * P.n_pblk_y;
    if (tid < PB) {
        const int ix = pbx * P.px + tid / P.py, iy = pby * P.py + tid % P.py;
        const bool ok = (tid < P.px * P.py) && ix < P.nx && iy < P.ny;
        const int p = ok ? ix * P.ny + iy : -1;
        s_pid[tid] = p;
        s_fold[tid] = 0;
        if (ok) {
            s_ox[tid] = P.xg ? P.xg[p] : P.xa[ix];
            s_oy[tid] = P.yg ? P.yg[p] : P.ya[iy];
        } else {
            s_ox[tid] = 0.0;
            s_oy[tid] = 0.0;
        }
    }
    const int t_base = blockIdx.y * (kThreads * R) + warp * (32 * R) + lane;

    TState st[R];
    if constexpr (!VEL3D) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = t_base + r * 32;
            const float4 tab = P.ttab[t < P.nt ? t : P.nt - 1];
            make_tstate<TT>(P, t, tab, st[r]);
        }
    }

    float acc[PB][R], hi[PB][R], lo[PB][R];
#pragma unroll
    for (int q = 0; q < PB; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) { acc[q][r] = 0.f; hi[q][r] = 0.f; lo[q][r] = 0.f; }

    const float sg_lo = P.s_guard_lo, sg_hi = P.s_guard_hi;
    __syncthreads();

    for (int64_t c0 = 0; c0 < P.n_traces; c0 += C) {
        // ---------------- phase A: (pillar, trace) records, FP64 geometry
        for (int j = tid; j < PB * C; j += kThreads) {
            const int q = j / C, c = j - q * C;
            const int64_t tr = c0 + c;
            const int p = s_pid[q];
            bool in = false;
            float4 r0 = make_float4(0.f, 0.f, __int_as_float(0x7f800000), 0.f);
            float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f), r2 = r1;
            if (p >= 0 && tr < P.n_traces) {
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
            const unsigned ballot = __ballot_sync(0xffffffffu, in);
            if (lane == 0 && ballot) atomicAdd(&s_fold[q], __popc(ballot));
            s_rec[0][j] = r0;
            if constexpr (NREC > 1) s_rec[1][j] = r1;
            if constexpr (NREC > 2) s_rec[2][j] = r2;
        }
        __syncthreads();

        // ---------------- phase B: pairs
        const int cmax = (P.n_traces - c0) < C ? (int)(P.n_traces - c0) : C;
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const int p = s_pid[q];
            if (p < 0) continue;
            if constexpr (VEL3D) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int t = t_base + r * 32;
                    const float4 tab = P.ttab[(int64_t)p * P.nt + (t < P.nt ? t : P.nt - 1)];
                    make_tstate<TT>(P, t, tab, st[r]);
                }
            }
            for (int c = 0; c < cmax; ++c) {
                const float4 r0 = s_rec[0][q * C + c];
                if (!(r0.z <= P.ap_max_f)) continue;
                float4 r1 = make_float4(0.f, 0.f, 0.f, 0.f), r2 = r1;
                if constexpr (NREC > 1) r1 = s_rec[1][q * C + c];
                if constexpr (NREC > 2) r2 = s_rec[2][q * C + c];
                const int64_t tr = c0 + c;
                const int64_t row = tr * P.amp_stride;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const TState &s = st[r];
                    if (!s.valid) continue;
                    if (r0.z >= s.ap) {
                        if (r0.z > s.ap) continue;
                        if (exact_outside_aperture(P, tr, p, t_base + r * 32, s_ox[q], s_oy[q])) continue;
                    }
                    const float T = traveltime<TT>(P, s, r0, r1, r2);
                    float sidx = fmaf(T, P.s_scale, P.s_offset);
                    if (!(sidx >= sg_lo && sidx <= sg_hi)) {
                        if (!(sidx >= P.s_rej_lo && sidx <= P.s_rej_hi)) continue;
                        if (!exact_sample_ok<TT>(P, tr, p, t_base + r * 32, s_ox[q], s_oy[q])) continue;
                        sidx = fminf(fmaxf(sidx, 0.f), P.s_max_clamp);
                    }
                    const float fl = __fadd_rd(sidx, 8388608.f);
                    const int i0 = __float_as_int(fl) - 0x4B000000;
                    const float f = sidx - (fl - 8388608.f);
                    const float a0 = load_amp<AMP>(P.amps, row + i0);
                    const float a1 = load_amp<AMP>(P.amps, row + i0 + 1);
                    const float amp = fmaf(f, a1 - a0, a0);
                    float w = r0.w;
                    const float x = fmaf(r0.z, s.itw, s.tsn);
                    if (x > 0.f) w *= 0.5f + 0.5f * __cosf(3.14159265358979f * x);
                    const float rT = rcp_approx(T);
                    float g = 1.f;
                    if (P.spreading | P.obliquity) {
                        g = s.K * rT;
                        if (P.spreading & P.obliquity) g *= rT;
                    }
                    if (s.guard && !(T > 0.001f)) g = 1.f;
                    if constexpr (AA) {
                        if (T >= 0.001f) {
                            const float sth = fminf(r1.x * s.ivw * rT, 1.f);
                            if (sth >= 0.01f) g *= fmaxf(0.f, 1.f - fmaxf(P.aa_cA * sth * s.ivw, P.aa_cB));
                        }
                    }
                    acc[q][r] = fmaf(amp, w * g, acc[q][r]);
                }
            }
        }
        // fold chunk partials into the compensated sums
#pragma unroll
        for (int q = 0; q < PB; ++q)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float y = acc[q][r];
                if (P.compensated) {
                    const float sum = hi[q][r] + y;
                    const float bp = sum - hi[q][r];
                    lo[q][r] += (hi[q][r] - (sum - bp)) + (y - bp);
                    hi[q][r] = sum;
                } else {
                    hi[q][r] += y;
                }
                acc[q][r] = 0.f;
            }
        __syncthreads();
    }

    // ---------------- epilogue: image += sum; fold += count
#pragma unroll
    for (int q = 0; q < PB; ++q) {
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
                img[idx] += hi[q][r] + lo[q][r];
            } else {
                double *img = reinterpret_cast<double *>(P.image);
                img[idx] += (double)hi[q][r] + (double)lo[q][r];
            }
            if (P.fold && P.fold3d) P.fold[idx] += cnt;
        }
    }
    if (P.fold && !P.fold3d && blockIdx.y == 0 && tid < PB) {
        const int p = s_pid[tid];
        if (p >= 0) P.fold[p] += s_fold[tid];
    }
}

// Per-(pillar|0, time) table: {1/v^2, aperture, eta, 1/v}, evaluated in FP64
// and rounded once (numba_cpu_optimized.py:378-399).
__global__ void prep_time_table(const KParams P, int64_t n_p, float4 *tab);

}  // namespace pstm
