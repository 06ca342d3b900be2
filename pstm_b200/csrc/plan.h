// plan.h -- host-side launch planning shared by the entry points: argument
// checks, launch parameters, and the split of shared memory between staged
// trace rows, records and partial sums.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "pstm_cuda.h"
#include "kparams.h"
#include "migrate.cuh"

namespace pstm {
namespace plan {

inline size_t amp_elem_bytes(int32_t dt) { return dt == PSTM_AMP_F32 ? 4 : 2; }

// Largest double B such that the correctly rounded sqrt(B) <= a, i.e. the
// FP64 predicate "sqrt(d2) > a" used by the reference equals "d2 > B".
inline double sqrt_threshold(double a) {
    double b = a * a;
    while (std::sqrt(b) > a) b = std::nextafter(b, 0.0);
    while (std::sqrt(std::nextafter(b, INFINITY)) <= a) b = std::nextafter(b, INFINITY);
    return b;
}

// Argument checks shared by every entry point; on failure `msg` says why.
inline int32_t check_args(const pstm_traces_desc *tr, const pstm_output_desc *out,
                          const pstm_velocity_desc *vel, const pstm_params *prm, const char *&msg) {
    auto fail = [&](int32_t code, const char *m) { msg = m; return code; };
    if (!tr || !out || !vel || !prm) return fail(PSTM_ERR_INVALID_ARGUMENT, "null descriptor");
    if (tr->n_traces < 0) return fail(PSTM_ERR_INVALID_ARGUMENT, "n_traces < 0");
    if (tr->n_samples < 2) return fail(PSTM_ERR_INVALID_ARGUMENT, "n_samples must be >= 2");
    if (tr->amp_dtype < PSTM_AMP_F32 || tr->amp_dtype > PSTM_AMP_F16)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "unknown amplitude dtype");
    if (tr->amp_row_stride < tr->n_samples)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "amp_row_stride < n_samples");
    if (tr->n_traces > 0 && (!tr->amplitudes || !tr->source_x || !tr->source_y || !tr->receiver_x ||
                             !tr->receiver_y || !tr->midpoint_x || !tr->midpoint_y))
        return fail(PSTM_ERR_INVALID_ARGUMENT, "null trace array");
    if (!(tr->sample_rate_ms > 0.0)) return fail(PSTM_ERR_INVALID_ARGUMENT, "sample_rate_ms must be > 0");
    if (out->nx <= 0 || out->ny <= 0 || out->nt <= 0)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "empty output tile");
    if (!out->image) return fail(PSTM_ERR_INVALID_ARGUMENT, "null image");
    if (out->image_dtype != PSTM_IMAGE_F64 && out->image_dtype != PSTM_IMAGE_F32)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "unknown image dtype");
    if (!out->t_axis_ms) return fail(PSTM_ERR_INVALID_ARGUMENT, "null t axis");
    if ((!out->x_grid || !out->y_grid) && (!out->x_axis || !out->y_axis))
        return fail(PSTM_ERR_INVALID_ARGUMENT, "need x/y axes or x/y grids");
    if ((out->x_grid == nullptr) != (out->y_grid == nullptr))
        return fail(PSTM_ERR_INVALID_ARGUMENT, "x_grid and y_grid must be given together");
    if (!vel->vrms) return fail(PSTM_ERR_INVALID_ARGUMENT, "null velocity");
    if (prm->traveltime < PSTM_TT_STRAIGHT || prm->traveltime > PSTM_TT_CURVED_VTI)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "unknown traveltime kind");
    if (prm->precision != PSTM_PREC_EXACT && prm->precision != PSTM_PREC_FAST && prm->precision != PSTM_PREC_FP32)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "unknown precision");
    if (prm->interpolation < PSTM_INTERP_LINEAR || prm->interpolation > PSTM_INTERP_LANCZOS5)
        return fail(PSTM_ERR_INVALID_ARGUMENT, "unknown interpolation method");
    if (!(prm->max_aperture_m >= 0.0) || !(prm->taper_fraction >= 0.0) || !(prm->taper_fraction <= 1.0))
        return fail(PSTM_ERR_INVALID_ARGUMENT, "bad aperture/taper parameters");
    if ((prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI) && !(prm->curved_v0 > 0.0))
        return fail(PSTM_ERR_INVALID_ARGUMENT, "curved_v0 must be > 0");
    return PSTM_OK;
}

inline KParams make_params(const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_velocity_desc *vel,
                    const pstm_params *prm, int PB) {
    KParams P;
    std::memset(&P, 0, sizeof(P));
    P.amps = tr->amplitudes;
    P.amp_stride = tr->amp_row_stride;
    P.n_traces = tr->n_traces;
    P.ns = tr->n_samples;
    P.elem = (int32_t)amp_elem_bytes(tr->amp_dtype);
    P.sx = tr->source_x; P.sy = tr->source_y;
    P.rx = tr->receiver_x; P.ry = tr->receiver_y;
    P.mx = tr->midpoint_x; P.my = tr->midpoint_y;
    P.w = tr->weights;
    P.dt_s = tr->sample_rate_ms / 1000.0;
    P.tstart_s = tr->start_time_ms / 1000.0;
    P.s_scale = (float)(1.0 / P.dt_s);
    P.s_offset = (float)(-P.tstart_s / P.dt_s);
    const float g = 1e-2f;   // guard band in samples around the FP64 decision boundaries
    const float smax = (float)(tr->n_samples - 1);
    P.s_guard_lo = g;
    P.s_guard_hi = smax - g;
    P.s_rej_lo = -g;
    P.s_rej_hi = smax + g;
    P.s_max_clamp = std::nextafter(smax, 0.0f);
    P.s_magic = 2147483648.0 - P.tstart_s / P.dt_s;
    P.inv_dt_f = (float)(1.0 / P.dt_s);

    P.image = out->image;
    P.fold = out->fold;
    P.image_f32 = out->image_dtype == PSTM_IMAGE_F32;
    P.fold3d = out->fold_is_3d;
    P.nx = out->nx; P.ny = out->ny; P.nt = out->nt;
    P.xa = out->x_axis; P.ya = out->y_axis;
    P.xg = out->x_grid; P.yg = out->y_grid;
    P.ta = out->t_axis_ms;

    P.vrms = vel->vrms;
    P.vel3d = vel->is_3d;
    P.eta = prm->eta;
    P.eta3d = prm->eta ? prm->eta_is_3d : 0;
    P.eta_const = prm->eta_constant;

    P.max_ap = prm->max_aperture_m;
    P.min_ap = prm->min_aperture_m;
    P.tan_dip = std::tan(prm->max_dip_degrees * M_PI / 180.0);
    P.taper = prm->taper_fraction;
    P.fold_d2_max = sqrt_threshold(prm->max_aperture_m);
    P.ap_max_f = (float)prm->max_aperture_m;
    P.taper_f = (float)prm->taper_fraction;
    P.spreading = prm->apply_spreading ? 1 : 0;
    P.obliquity = prm->apply_obliquity ? 1 : 0;
    P.aa = prm->aa_enabled ? 1 : 0;
    const double gmax = prm->grid_dx > prm->grid_dy ? prm->grid_dx : prm->grid_dy;
    P.aa_cA = (float)(4.0 * gmax * prm->aa_dominant_freq);
    P.aa_cB = (float)(prm->aa_dominant_freq / 500.0);
    P.aa_gmax = gmax;
    P.aa_fdom = prm->aa_dominant_freq;
    P.cr_v0 = prm->curved_v0;
    P.cr_k = prm->curved_k;
    P.cr_v0f = (float)prm->curved_v0;
    P.cr_kf = (float)prm->curved_k;
    P.cr_k_zero = std::fabs(prm->curved_k) < 1e-10 ? 1 : 0;
    P.cr_inv_k_ln2 = P.cr_k_zero ? 0.f : (float)(M_LN2 / prm->curved_k);
    // VTI returns 2 t0/2 = 0 at t0 = 0; the curved leg of depth 0 is log(1) = 0 for k != 0
    P.t0_zero_exact = (prm->traveltime == PSTM_TT_VTI ||
                       ((prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI) &&
                        !P.cr_k_zero)) ? 1 : 0;
    P.compensated = prm->compensated ? 1 : 0;
    P.cr_B0 = 1.0 / (prm->curved_v0 * prm->curved_v0 * P.dt_s * P.dt_s);
    P.cr_k2 = prm->curved_k * prm->curved_k;
    P.cr_inv_k_dt = P.cr_k_zero ? 0.0 : 1.0 / (prm->curved_k * P.dt_s);
    P.wait_iters = kWaitIters;
    // Fault injection for the tests of the bounded waits: PSTM_CUDA_INJECT_FAULT=wait
    // leaves the first trace chunks' copies unissued, so the kernel's bounded
    // wait for them runs out after a few polls and it reports KERR_WAIT_TIMEOUT.
    // Read when a launch is prepared (a captured batch keeps what it saw).
    if (const char *inj = std::getenv("PSTM_CUDA_INJECT_FAULT")) {
        if (std::strcmp(inj, "wait") == 0) {
            P.inject_stall = 1;
            P.wait_iters = 256;
        }
    }

    // pillar patch: PB pillars as px x py, favouring y (the fastest image axis)
    int py = PB, px = 1;
    while (py > 1 && py > out->ny) { py /= 2; px *= 2; }
    if (py == PB && PB >= 4) { py = PB / 2; px = 2; }
    P.px = px;
    P.py = py;
    P.n_pblk_y = (out->ny + py - 1) / py;
    return P;
}


// Output times per lane (R) and pillars per CTA (PB) for a tile; force_* > 0
// override them (tuning).  amp_dtype: 16-bit rows stage twice the traces per
// byte, and there 8 pillars per CTA amortise a chunk's staging, records and
// barrier over twice the pairs (measured on the case-2 tile, 262,144 traces:
// FP16 5 % faster with 8 than with 4 pillars, FP32 6 % slower).
inline void choose_shape(int nt, int force_r, int force_pb, int &R, int &PB, int amp_dtype = PSTM_AMP_F32) {
    R = (nt + kThreads - 1) / kThreads;   // the whole output trace in one CTA where it fits
    if (R > 8) R = 8;
    if (force_r >= 1 && force_r <= 8) R = force_r;
    PB = (R <= 1 || amp_dtype != PSTM_AMP_F32) ? 8 : 4;
    if (force_pb >= 1 && force_pb <= kMaxPB) PB = force_pb;
}

// Staging plan: row pitch, TMA eligibility, traces per chunk and the dynamic
// shared memory of one CTA.  Returns false when a row does not fit.
inline bool plan_staging(KParams &P, const pstm_traces_desc *tr, const pstm_params *prm, int PB, int R,
                         int smem_optin, size_t &smem, int force_chunk = 0) {
    const int eb = P.elem;
    const int per16 = 16 / eb;
    const int pitch = (tr->n_samples + per16 - 1) / per16 * per16;
    const bool aligned = ((uintptr_t)tr->amplitudes % 16 == 0) && ((tr->amp_row_stride * eb) % 16 == 0);
    P.pitch = pitch;
    P.bulk = (aligned && tr->amp_row_stride >= pitch) ? 1 : 0;
    const bool has_c = prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI;
    const size_t fixed = 2 * (size_t)geo_buffer_bytes() + 2 * (size_t)record_buffer_bytes(PB, has_c) +
                         (size_t)partial_bytes(PB, R, prm->compensated != 0);
    const size_t static_bytes = 3072;   // s_ox/s_oy/s_pid/s_fold/s_rank/barriers, rounded up
    const size_t budget = (size_t)smem_optin > fixed + static_bytes ? smem_optin - fixed - static_bytes : 0;
    int chunk = (int)(budget / (2 * (size_t)pitch * eb));
    if (chunk > kMaxChunk) chunk = kMaxChunk;
    if (force_chunk >= 1 && force_chunk < chunk) chunk = force_chunk;   // tuning: a shallower panel
    if (chunk < 1) return false;
    P.chunk = chunk;
    P.pb = PB;
    P.r_per_lane = R;
    P.flush_every = 16;
    P.n_tblk = (P.nt + kThreads * R - 1) / (kThreads * R);
    smem = 2 * (size_t)chunk * pitch * eb + fixed;
    return true;
}

}  // namespace plan
}  // namespace pstm
