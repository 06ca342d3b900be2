// kparams.h -- launch parameters shared by the host side (capi.cu) and the
// migration kernels.  Plain C++ struct passed by value to every launch.
#pragma once
#include <stdint.h>
#include <vector_types.h>

namespace pstm {

enum AmpKind { AMP_F32 = 0, AMP_BF16 = 1, AMP_F16 = 2 };
enum TTKind { TT_STRAIGHT = 0, TT_CURVED = 1, TT_VTI = 2, TT_CURVED_VTI = 3 };

// error bits a kernel can raise in *err
enum KernelError { KERR_WAIT_TIMEOUT = 1, KERR_UNSORTED_AXIS = 2 };

// One output of the persistent form: its traces and its image/fold.
struct BinWork {
    int64_t trace0;              // first trace in the concatenated panel
    int64_t n_traces;
    void *image;
    int32_t *fold;
};

// The scatter schedule of the persistent form: the panel cut into segments
// of seg_traces traces; segment s reaches the pillar blocks
// [pbx0, pbx1] x [pby0, pby1] (empty when pbx0 > pbx1) and contributes
// (pbx1 - pbx0 + 1) (pby1 - pby0 + 1) n_tblk work items; ends[s] is the
// inclusive prefix sum of those counts.
struct SegmentBox {
    int32_t pbx0, pbx1, pby0, pby1;
};
struct ScatterWork {
    const SegmentBox *boxes;
    const long long *ends;
    int64_t n_seg;
    int64_t seg_traces;
};

struct KParams {
    // ---- traces ----
    const void *amps;
    int64_t amp_stride;          // elements between rows
    int64_t n_traces;
    int32_t ns;                  // samples per trace
    int32_t elem;                // bytes per amplitude
    const double *sx, *sy, *rx, *ry, *mx, *my, *w;   // w nullable
    const double *geo;           // packed per trace: sx sy rx ry mx my w 0 (scratch)
    double dt_s, tstart_s;       // input sampling (seconds)
    float s_scale, s_offset;     // sample index s = T * s_scale + s_offset
    float s_guard_lo, s_guard_hi;  // fast-path accept window for s
    float s_rej_lo, s_rej_hi;    // outside [s_rej_lo, s_rej_hi] the pair is rejected
    float s_max_clamp;           // largest s allowed for the interpolation read
    int32_t pad1;
    double s_magic;              // 2^31 - tstart/dt: FP64 sample index + 2^31 (EXACT path)

    // ---- staging of trace rows in shared memory ----
    int32_t chunk;               // traces per chunk (<= kMaxChunk)
    int32_t n_tblk;              // time blocks per output (persistent form)
    int32_t atomic_flush;        // outputs shared by concurrent items: atomic image/fold adds
    int32_t pb;                  // pillars per CTA (<= kMaxPB)
    int32_t r_per_lane;          // output times per lane (R)
    int32_t pitch;               // staged row pitch, elements (multiple of 16 bytes)
    int32_t bulk;                // 1: rows are copied by TMA bulk copies
    int32_t pad2;

    // ---- output ----
    void *image;
    int32_t *fold;
    int32_t image_f32;           // 0: f64 image, 1: f32 image
    int32_t fold3d;
    int32_t nx, ny, nt;
    int32_t px, py;              // pillar patch of one CTA (px * py pillars)
    int32_t n_pblk_y;            // number of patches along y
    const double *xa, *ya, *xg, *yg, *ta;   // xg/yg nullable

    // ---- velocity / per-time tables ----
    const double *vrms;          // (nt) or (nx*ny*nt), FP64 (exact paths)
    int32_t vel3d;
    int32_t eta3d;
    const float4 *ttab;          // per (pillar|0, t): {1/v^2, aperture, 1/v, eta}
    const double *btab;          // per (pillar|0, t): 1/(v dt)^2 (EXACT path)
    const float4 *ttime;         // per t: {t0h2, Kt, tg, tguard}, {vz, vz2, 1/vz, t0 == 0}
    const double *ttimeA;        // per t: (t0 / (2 dt))^2 (EXACT path)
    float inv_dt_f;              // 1 / dt (s)
    int32_t flush_every;         // chunks between flushes of the FP32 partials
    int32_t exact_units;         // weights' time unit: 1 = samples (EXACT), 0 = seconds
    int32_t curved_kind;         // curved-ray traveltime (its T can be ~0 at t0 > 0)
    int32_t t0_zero_exact;       // at t0 = 0 every pair has T = 0 exactly in FP64 (VTI; curved, k != 0)
    const double *eta;           // nullable (FP64, exact paths)
    double eta_const;

    // ---- parameters ----
    double max_ap, min_ap, tan_dip, taper;
    double fold_d2_max;          // largest d^2 with RN(sqrt(d^2)) <= max_ap
    float ap_max_f;              // (float)max_ap
    float taper_f;               // taper fraction
    int32_t spreading, obliquity;
    int32_t aa;
    float aa_cA, aa_cB;          // 4*max(dx,dy)*f_dom, f_dom/500
    double aa_gmax, aa_fdom;     // max(dx, dy), f_dom (FP64 paths)
    double cr_v0, cr_k;
    float cr_v0f, cr_kf, cr_inv_k_ln2;   // inv_k * ln2 (log2 based)
    int32_t cr_k_zero;           // |k| < 1e-10: straight-ray fallback with v0
    int32_t compensated;
    int32_t *err;                // device error word (KernelError bits)
    // FP64 sample-index path of the curved kinds (samples as the time unit)
    const double *ttimeV;        // per t: v(z) of the image depth, FP64 (curved kinds)
    double cr_B0;                // 1 / (v0 dt)^2: |k| ~ 0 straight rays in v0
    double cr_k2;                // k^2
    double cr_inv_k_dt;          // 1 / (k dt)
    int32_t wait_iters;          // polls of one bounded mbarrier wait before it gives up
    int32_t inject_stall;        // fault injection: the first chunks' copies are never issued, so the
                                 // bounded waits for them run out (host-selected, tests only)
};

}  // namespace pstm
