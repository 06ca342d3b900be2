/*
 * pstm_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Double-precision CPU restatement of the reference `pstm` package's
 * per-output-point Kirchhoff summation (`migrate_tile`).  It is the checker
 * for the CUDA backend: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs load it.  Nothing in the product path calls it.
 *
 * Semantics restated (paths relative to the reference project):
 *   base loop, fold, time-varying aperture, taper, spreading, obliquity,
 *   linear interpolation, trace weights, image "+=":
 *       pstm/kernels/numba_cpu_optimized.py:93-233   (_migrate_tile_kernel_optimized)
 *       pstm/kernels/numba_cpu_optimized.py:358-401  (_precompute_time_terms)
 *       pstm/kernels/numba_cpu.py:108-211            (weights, taper, aperture)
 *   triangle anti-aliasing weight:
 *       pstm/metal/shaders/pstm_migration.metal:95-132, applied :253-262
 *   3-D velocity (per pillar v_rms(t)):
 *       pstm/metal/shaders/pstm_migration.metal:187-197
 *   curved-ray traveltime V(z)=v0+k z:
 *       pstm/algorithm/curved_ray.py:19-52, :239-262, :287-316
 *       pstm/metal/shaders/pstm_curved_ray.metal:50-96, :196-279
 *   VTI (eta) traveltime per leg:
 *       pstm/algorithm/anisotropy_vti.py:148-220
 *       pstm/metal/shaders/pstm_anisotropic_vti.metal:103-148, :252-333
 *   curved-ray + VTI: the reference has no combined formula; this build
 *       defines each leg as the curved-ray leg time scaled by the VTI /
 *       hyperbolic ratio of the same leg in the NMO velocity v_rms(t):
 *       t = t_curved * sqrt(1 - corr / (t0h^2 + h^2/v^2)), which is t_curved
 *       at eta = 0 and never cancels (corr < h^2/v^2).
 *
 * Fold follows the Numba path for every traveltime kind: per pillar, the
 * number of traces whose midpoint lies within max_aperture, added to every
 * output sample of that pillar (numba_cpu_optimized.py:168-175, :231).
 *
 * Build: see oracle/Makefile (plain gcc, -O2, no fast-math; OpenMP over
 * pillars).
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_TT_STRAIGHT   0
#define ORACLE_TT_CURVED     1
#define ORACLE_TT_VTI        2
#define ORACLE_TT_CURVED_VTI 3

typedef struct {
    /* traces */
    int64_t n_traces;
    int32_t n_samples;
    int32_t amp_is_f64;          /* 0: float32 amplitudes, 1: float64 */
    const void *amplitudes;      /* (n_traces, n_samples) row-major */
    const double *source_x, *source_y, *receiver_x, *receiver_y;
    const double *midpoint_x, *midpoint_y;
    const double *weights;       /* nullable -> 1.0 */
    double sample_rate_ms, start_time_ms;
    /* output tile */
    int32_t nx, ny, nt;
    const double *x_axis, *y_axis;   /* (nx), (ny) */
    const double *x_grid, *y_grid;   /* nullable, (nx*ny) rotated grid */
    const double *t_axis_ms;         /* (nt) */
    double *image;                   /* (nx, ny, nt) accumulated with += */
    int32_t *fold;                   /* (nx, ny, nt) or (nx, ny); nullable */
    int32_t fold_is_3d;
    /* velocity */
    const double *vrms;              /* (nt) or (nx, ny, nt) */
    int32_t vel_is_3d;
    /* parameters */
    double max_aperture_m, min_aperture_m, max_dip_degrees, taper_fraction;
    int32_t apply_spreading, apply_obliquity;
    int32_t aa_enabled;
    double aa_dominant_freq, grid_dx, grid_dy;
    int32_t traveltime_kind;
    double curved_v0, curved_k;
    const double *eta;               /* nullable; (nt) or (nx, ny, nt) */
    int32_t eta_is_3d;
    double eta_constant;
    /* pillar subset [pillar_begin, pillar_end) in flattened ix*ny+iy order;
       pillar_end <= 0 means all pillars */
    int64_t pillar_begin, pillar_end;
    int32_t n_threads;               /* <= 0: OpenMP default */
    int32_t interp_method;           /* ORACLE_INTERP_* (0: linear) */
} oracle_args;

/* Trace interpolators of pstm/kernels/interpolation.py:59-285 (codes here put
 * linear first; the reference numbers nearest 0 and linear 1). */
#define ORACLE_INTERP_LINEAR   0
#define ORACLE_INTERP_NEAREST  1
#define ORACLE_INTERP_CUBIC    2
#define ORACLE_INTERP_SINC4    3
#define ORACLE_INTERP_SINC8    4
#define ORACLE_INTERP_SINC16   5
#define ORACLE_INTERP_LANCZOS3 6
#define ORACLE_INTERP_LANCZOS5 7

/* straight-ray one-way leg, numba_cpu_optimized.py:192-194 */
static double leg_straight(double t0h2, double h2, double inv_v2)
{
    return sqrt(t0h2 + h2 * inv_v2);
}

/* curved_ray.py:239-262 (time_to_depth_curved) */
static double curved_depth(double t_one_way, double v0, double k)
{
    if (fabs(k) < 1e-10) return v0 * t_one_way;
    return (v0 / k) * (exp(k * t_one_way) - 1.0);
}

/* curved_ray.py:19-52 (curved_ray_traveltime) */
static double leg_curved(double h, double z, double v0, double k)
{
    if (fabs(k) < 1e-10) {
        double r = sqrt(h * h + z * z);
        return r > 0.0 ? r / v0 : 0.0;
    }
    double vz = v0 + k * z;
    double kx = k * h;
    double term1 = vz + sqrt(vz * vz + kx * kx);
    double term2 = v0 + sqrt(v0 * v0 + kx * kx);
    if (term2 <= 0.0) return 0.0;
    return (1.0 / k) * log(term1 / term2);
}

/* quartic eta correction, anisotropy_vti.py:181-220 / pstm_anisotropic_vti.metal:103-127 */
static double vti_correction(double t0h, double h, double v, double eta)
{
    double h2 = h * h, v2 = v * v, t02 = t0h * t0h;
    double denom = v2 * (t02 * v2 + (1.0 + 2.0 * eta) * h2);
    if (fabs(denom) > 1e-20) return (2.0 * eta * h2 * h2) / denom;
    return 0.0;
}

/* vti_one_way_time, pstm_anisotropic_vti.metal:103-127 */
static double leg_vti(double t0h, double h, double v, double eta)
{
    if (v <= 0.0 || t0h <= 0.0) return t0h;
    double t2 = t0h * t0h + (h * h) / (v * v) - vti_correction(t0h, h, v, eta);
    return sqrt(t2 > 0.0 ? t2 : 0.0);
}

/* build-defined curved + VTI leg (see header) */
static double leg_curved_vti(double t0h, double h, double z, double v0, double k,
                             double v, double eta)
{
    double tc = leg_curved(h, z, v0, k);
    if (v <= 0.0 || t0h <= 0.0) return tc;
    double hyp = t0h * t0h + (h * h) / (v * v);
    double r = 1.0 - vti_correction(t0h, h, v, eta) / hyp;
    return tc * sqrt(r > 0.0 ? r : 0.0);
}

/* compute_aa_weight, pstm_migration.metal:95-132 */
static double aa_weight(double ox, double oy, double mx, double my, double v,
                        double t_travel, double dx, double dy, double fdom)
{
    if (t_travel < 0.001) return 1.0;
    double denom = v * v * t_travel * 0.5;
    double dip_x = (mx - ox) / denom;
    double dip_y = (my - oy) / denom;
    double stx = fabs(dip_x) * v * 0.5; if (stx > 1.0) stx = 1.0;
    double sty = fabs(dip_y) * v * 0.5; if (sty > 1.0) sty = 1.0;
    double st = stx > sty ? stx : sty;
    if (st < 0.01) return 1.0;
    double g = dx > dy ? dx : dy;
    double fmax = v / (4.0 * g * st);
    if (fmax > 500.0) fmax = 500.0;
    double w = 1.0 - fdom / fmax;
    return w > 0.0 ? w : 0.0;
}

typedef struct {
    const oracle_args *a;
    int64_t tr;
} trace_ref;
static double interp_sample(double (*get)(const void *, int64_t), const void *ctx, int32_t n, double t, int32_t m);

static inline double amp_at(const oracle_args *a, int64_t tr, int64_t i)
{
    if (a->amp_is_f64) return ((const double *)a->amplitudes)[tr * a->n_samples + i];
    return (double)((const float *)a->amplitudes)[tr * a->n_samples + i];
}

static double trace_get(const void *p, int64_t i)
{
    const trace_ref *r = (const trace_ref *)p;
    return amp_at(r->a, r->tr, i);
}

/*
 * Migrate the pillar subset.  Returns 0 on success, nonzero on bad arguments.
 */
int pstm_oracle_migrate(const oracle_args *a)
{
    if (!a || a->nx <= 0 || a->ny <= 0 || a->nt <= 0 || a->n_samples < 2 || !a->image)
        return 1;
    if (a->n_traces < 0) return 1;
    const int64_t n_pillars = (int64_t)a->nx * a->ny;
    int64_t pb = a->pillar_begin < 0 ? 0 : a->pillar_begin;
    int64_t pe = a->pillar_end <= 0 ? n_pillars : a->pillar_end;
    if (pe > n_pillars) pe = n_pillars;
    const int nt = a->nt;
    const int ns = a->n_samples;
    const double dt_s = a->sample_rate_ms / 1000.0;
    const double tstart_s = a->start_time_ms / 1000.0;
    const double tan_dip = tan(a->max_dip_degrees * M_PI / 180.0);
    const double tap = a->taper_fraction;

#ifdef _OPENMP
    if (a->n_threads > 0) omp_set_num_threads(a->n_threads);
#pragma omp parallel
#endif
    {
        double *t0s = (double *)__builtin_alloca(sizeof(double) * 8 * (size_t)nt);
        double *t0h2 = t0s + nt, *iv2 = t0h2 + nt, *ap = iv2 + nt, *vv = ap + nt,
               *zc = vv + nt, *vz = zc + nt, *et = vz + nt;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
        for (int64_t p = pb; p < pe; ++p) {
            const int ix = (int)(p / a->ny), iy = (int)(p % a->ny);
            const double ox = a->x_grid ? a->x_grid[p] : a->x_axis[ix];
            const double oy = a->y_grid ? a->y_grid[p] : a->y_axis[iy];
            /* per-time terms: numba_cpu_optimized.py:378-399 */
            for (int it = 0; it < nt; ++it) {
                double v = a->vel_is_3d ? a->vrms[p * nt + it] : a->vrms[it];
                double t = a->t_axis_ms[it] / 1000.0;
                t0s[it] = t;
                t0h2[it] = (t * 0.5) * (t * 0.5);
                iv2[it] = 1.0 / (v * v);
                vv[it] = v;
                double apv = v * t * 0.5 * tan_dip;
                if (apv < a->min_aperture_m) apv = a->min_aperture_m;
                else if (apv > a->max_aperture_m) apv = a->max_aperture_m;
                ap[it] = apv;
                zc[it] = curved_depth(t * 0.5, a->curved_v0, a->curved_k);
                vz[it] = a->curved_v0 + a->curved_k * zc[it];
                if (a->eta) et[it] = a->eta_is_3d ? a->eta[p * nt + it] : a->eta[it];
                else et[it] = a->eta_constant;
            }
            int32_t local_fold = 0;
            double *img = a->image + p * nt;
            for (int64_t tr = 0; tr < a->n_traces; ++tr) {
                const double mx = a->midpoint_x[tr], my = a->midpoint_y[tr];
                const double dmid = sqrt((ox - mx) * (ox - mx) + (oy - my) * (oy - my));
                if (dmid > a->max_aperture_m) continue;
                local_fold += 1;
                const double sx = a->source_x[tr], sy = a->source_y[tr];
                const double rx = a->receiver_x[tr], ry = a->receiver_y[tr];
                const double ds2 = (ox - sx) * (ox - sx) + (oy - sy) * (oy - sy);
                const double dr2 = (ox - rx) * (ox - rx) + (oy - ry) * (oy - ry);
                const double hs = sqrt(ds2), hr = sqrt(dr2);
                const double wtr = a->weights ? a->weights[tr] : 1.0;
                for (int it = 0; it < nt; ++it) {
                    const double apt = ap[it];
                    if (dmid > apt) continue;
                    double T, vw;
                    switch (a->traveltime_kind) {
                    case ORACLE_TT_CURVED:
                        T = leg_curved(hs, zc[it], a->curved_v0, a->curved_k) +
                            leg_curved(hr, zc[it], a->curved_v0, a->curved_k);
                        vw = vz[it];
                        break;
                    case ORACLE_TT_VTI:
                        T = leg_vti(t0s[it] * 0.5, hs, vv[it], et[it]) +
                            leg_vti(t0s[it] * 0.5, hr, vv[it], et[it]);
                        vw = vv[it];
                        break;
                    case ORACLE_TT_CURVED_VTI:
                        T = leg_curved_vti(t0s[it] * 0.5, hs, zc[it], a->curved_v0, a->curved_k, vv[it], et[it]) +
                            leg_curved_vti(t0s[it] * 0.5, hr, zc[it], a->curved_v0, a->curved_k, vv[it], et[it]);
                        vw = vz[it];
                        break;
                    default:
                        T = leg_straight(t0h2[it], ds2, iv2[it]) + leg_straight(t0h2[it], dr2, iv2[it]);
                        vw = vv[it];
                        break;
                    }
                    const double s = (T - tstart_s) / dt_s;
                    if (s < 0.0 || s >= (double)(ns - 1)) continue;
                    double amp;
                    if (a->interp_method == ORACLE_INTERP_LINEAR) {
                        const int64_t i0 = (int64_t)s;
                        const double f = s - (double)i0;
                        amp = amp_at(a, tr, i0) * (1.0 - f) + amp_at(a, tr, i0 + 1) * f;
                    } else {
                        const trace_ref r = {a, tr};
                        amp = interp_sample(trace_get, &r, ns, s, a->interp_method);
                    }
                    double w = wtr;
                    const double ts = apt * (1.0 - tap);
                    if (dmid > ts) {
                        const double x = (dmid - ts) / (apt - ts);
                        w *= 0.5 * (1.0 + cos(M_PI * x));
                    }
                    if (a->aa_enabled)
                        w *= aa_weight(ox, oy, mx, my, vw, T, a->grid_dx, a->grid_dy, a->aa_dominant_freq);
                    if (a->apply_spreading && T > 0.001) w *= 1.0 / (vw * T);
                    if (a->apply_obliquity && T > 0.001) w *= t0s[it] / T;
                    img[it] += amp * w;
                }
            }
            if (a->fold) {
                if (a->fold_is_3d) {
                    int32_t *f = a->fold + p * nt;
                    for (int it = 0; it < nt; ++it) f[it] += local_fold;
                } else {
                    a->fold[p] += local_fold;
                }
            }
        }
    }
    return 0;
}

/*
 * Exact traveltime (seconds) for a batch of (t0, dx_s, dy_s, dx_r, dy_r, v, eta)
 * rows -- the surrogate network's training target and yardstick.  kind as above;
 * curved-ray parameters shared.  out[i] = T.
 */
void pstm_oracle_traveltime(int32_t kind, int64_t n, const double *feat7,
                            double curved_v0, double curved_k, double *out)
{
    for (int64_t i = 0; i < n; ++i) {
        const double *f = feat7 + 7 * i;
        const double t0 = f[0], v = f[5], eta = f[6];
        const double hs = sqrt(f[1] * f[1] + f[2] * f[2]);
        const double hr = sqrt(f[3] * f[3] + f[4] * f[4]);
        const double z = curved_depth(t0 * 0.5, curved_v0, curved_k);
        double T;
        switch (kind) {
        case ORACLE_TT_CURVED:
            T = leg_curved(hs, z, curved_v0, curved_k) + leg_curved(hr, z, curved_v0, curved_k);
            break;
        case ORACLE_TT_VTI:
            T = leg_vti(t0 * 0.5, hs, v, eta) + leg_vti(t0 * 0.5, hr, v, eta);
            break;
        case ORACLE_TT_CURVED_VTI:
            T = leg_curved_vti(t0 * 0.5, hs, z, curved_v0, curved_k, v, eta) +
                leg_curved_vti(t0 * 0.5, hr, z, curved_v0, curved_k, v, eta);
            break;
        default:
            T = leg_straight(t0 * t0 * 0.25, hs * hs, 1.0 / (v * v)) +
                leg_straight(t0 * t0 * 0.25, hr * hr, 1.0 / (v * v));
        }
        out[i] = T;
    }
}

/* sin(pi x)/(pi x), 1 at x ~ 0 (interpolation.py:139-144) */
static double sinc_pi(double x)
{
    if (fabs(x) < 1e-10) return 1.0;
    return sin(M_PI * x) / (M_PI * x);
}

/* One sample of `trace` (n samples, read through get(i)) at fractional index t:
 * nearest (:59-66), linear (:68-92), Catmull-Rom cubic (:95-135), Hanning-
 * windowed sinc of half-width 2/4/8 (:147-189), Lanczos 3/5 (:208-249); the
 * higher-order methods fall back to linear within their half-width of an end
 * and normalise by the sum of their weights. */
static double interp_sample(double (*get)(const void *, int64_t), const void *ctx, int32_t n, double t, int32_t m)
{
    if (m == ORACLE_INTERP_NEAREST) {
        const int64_t i = (int64_t)(t + 0.5);
        return (i < 0 || i >= n) ? 0.0 : get(ctx, i);
    }
    const int hw = m == ORACLE_INTERP_SINC4 ? 2 : m == ORACLE_INTERP_SINC8 ? 4 : m == ORACLE_INTERP_SINC16 ? 8
                 : m == ORACLE_INTERP_LANCZOS3 ? 3 : m == ORACLE_INTERP_LANCZOS5 ? 5 : 0;
    const int cubic_edge = m == ORACLE_INTERP_CUBIC && (t < 1.0 || t >= (double)(n - 2));
    const int wide_edge = hw > 0 && (t < (double)hw || t >= (double)(n - hw));
    if (m == ORACLE_INTERP_LINEAR || cubic_edge || wide_edge) {
        if (t < 0.0 || t >= (double)(n - 1)) return 0.0;
        const int64_t i0 = (int64_t)t;
        const double f = t - (double)i0;
        return get(ctx, i0) * (1.0 - f) + get(ctx, i0 + 1) * f;
    }
    if (m == ORACLE_INTERP_CUBIC) {
        const int64_t i = (int64_t)t;
        const double u = t - (double)i;
        const double p0 = get(ctx, i - 1), p1 = get(ctx, i), p2 = get(ctx, i + 1), p3 = get(ctx, i + 2);
        const double c3 = -0.5 * p0 + 1.5 * p1 - 1.5 * p2 + 0.5 * p3;
        const double c2 = p0 - 2.5 * p1 + 2.0 * p2 - 0.5 * p3;
        const double c1 = -0.5 * p0 + 0.5 * p2;
        return ((c3 * u + c2) * u + c1) * u + p1;
    }
    const int lanczos = m == ORACLE_INTERP_LANCZOS3 || m == ORACLE_INTERP_LANCZOS5;
    const int64_t ic = lanczos ? (int64_t)t : (int64_t)(t + 0.5);
    const double frac = t - (double)ic;
    double acc = 0.0, norm = 0.0;
    for (int k = -hw + 1; k <= hw; ++k) {
        const int64_t i = ic + k;
        if (i < 0 || i >= n) continue;
        const double x = frac - (double)k;
        double w;
        if (lanczos) w = fabs(x) < 1e-10 ? 1.0 : (fabs(x) >= hw ? 0.0 : sinc_pi(x) * sinc_pi(x / hw));
        else w = sinc_pi(x) * (fabs(x) >= hw ? 0.0 : 0.5 * (1.0 + cos(M_PI * x / hw)));
        acc += get(ctx, i) * w;
        norm += w;
    }
    return norm > 1e-10 ? acc / norm : 0.0;
}

static double get_f64(const void *p, int64_t i) { return ((const double *)p)[i]; }

double pstm_oracle_interp(const double *trace, int32_t n, double t_sample, int32_t method)
{
    return interp_sample(get_f64, trace, n, t_sample, method);
}

/* The reference's linear interpolator, pstm/kernels/interpolation.py:68-92. */
double pstm_oracle_linear_interp(const double *trace, int32_t n, double t_sample)
{
    if (t_sample < 0.0 || t_sample >= (double)(n - 1)) return 0.0;
    int32_t i0 = (int32_t)t_sample;
    double f = t_sample - (double)i0;
    return trace[i0] * (1.0 - f) + trace[i0 + 1] * f;
}

int32_t pstm_oracle_abi_version(void) { return 1; }
