// metal_ref.cpp -- the reference's Metal compute shaders compiled as C++ on
// the CPU.  Test infrastructure only: it checks the oracle against the
// shaders' own code, it is never the thing measured or shipped.
//
// oracle/Makefile's `ref` target builds it from the shader files where they
// lie in the reference tree (their paths arrive as the PSTM_METAL_* macros)
// into oracle/_ref/, with the Metal standard-library subset of
// metal_compat/metal_stdlib.  Each shader is included in a namespace of its
// own (they define helpers of the same names), and a migration runs the
// shader's kernel function once per (ix, iy, it) grid position, as a Metal
// dispatch of nx x ny x nt threads would:
//   pstm_migration.metal       pstm_migrate_3d[_simd]         (straight rays, AA, 1-D or 3-D velocity)
//   pstm_curved_ray.metal      pstm_migrate_curved_ray[_simd] (V(z) = v0 + k z)
//   pstm_anisotropic_vti.metal pstm_migrate_vti[_simd]        (eta moveout)
// (`simd` picks the _simd variant, the Metal backend's default, which reads
// the geometry of four traces at a time as float4.)
//   pstm_migration.metal       pstm_migrate_time_variant (straight rays at the
//                              sample times of time-variant windows)
// The helpers (AA weight, DSR, curved and VTI traveltimes) are exported too.
#include <metal_stdlib>

#include <cstdint>

namespace ref_straight {
#include PSTM_METAL_STRAIGHT
}
namespace ref_curved {
#include PSTM_METAL_CURVED
}
namespace ref_vti {
#include PSTM_METAL_VTI
}

#undef kernel
#undef device
#undef constant
#undef thread
#undef threadgroup

using metal::atomic_int;
using metal::uint3;

extern "C" {

// One migration call: FP32 inputs in the shaders' layouts; image (nx, ny, nt)
// is assigned, fold is (nx, ny, nt) for the straight kernel (contributing
// traces per sample) and (nx, ny) for curved/VTI (contributing traces at it = 0).
typedef struct {
    const float *amps;                          // (n_traces, n_samples)
    const float *sx, *sy, *rx, *ry, *mx, *my;   // (n_traces)
    const float *x_coords, *y_coords;           // (nx * ny)
    const float *t0_s, *t0_half_sq, *apertures, *eta;   // (nt)
    const float *inv_v_sq;                      // (nt), or (nx, ny, nt) with use_3d_velocity
    float *image;
    int32_t *fold;
    int32_t n_traces, n_samples, nx, ny, nt;
    int32_t spreading, obliquity, aa, use_3d_velocity, eta_is_1d;
    float dx, dy, dt_ms, t_start_ms, max_aperture, min_aperture, taper_fraction, max_dip_deg;
    float aa_dominant_freq, v0, k, eta_constant;
} pstm_ref_call;

float pstm_ref_aa_weight(float ox, float oy, float mx, float my, float v, float t, float dx, float dy, float fdom) {
    return ref_straight::compute_aa_weight(ox, oy, mx, my, v, t, dx, dy, fdom);
}
float pstm_ref_dsr(float ds2, float dr2, float t0_half_sq, float inv_v_sq) {
    return ref_straight::compute_dsr_traveltime(ds2, dr2, t0_half_sq, inv_v_sq);
}
float pstm_ref_time_to_depth(float t_s, float v0, float k) { return ref_curved::time_to_depth(t_s, v0, k); }
float pstm_ref_curved_dsr(float h_s, float h_r, float z, float v0, float k) {
    return ref_curved::curved_ray_dsr_traveltime(h_s, h_r, z, v0, k);
}
float pstm_ref_vti_dsr(float t0_s, float h_s, float h_r, float v, float eta) {
    return ref_vti::vti_dsr_traveltime(t0_s, h_s, h_r, v, eta);
}

void pstm_ref_migrate_straight(const pstm_ref_call *c, int32_t simd) {
    ref_straight::MigrationParams p{};
    p.dx = c->dx;
    p.dy = c->dy;
    p.dt_ms = c->dt_ms;
    p.t_start_ms = c->t_start_ms;
    p.max_aperture = c->max_aperture;
    p.min_aperture = c->min_aperture;
    p.taper_fraction = c->taper_fraction;
    p.max_dip_deg = c->max_dip_deg;
    p.apply_spreading = c->spreading;
    p.apply_obliquity = c->obliquity;
    p.apply_aa = c->aa;
    p.aa_dominant_freq = c->aa_dominant_freq;
    p.n_traces = c->n_traces;
    p.n_samples = c->n_samples;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nt = c->nt;
    p.use_3d_velocity = c->use_3d_velocity;
#pragma omp parallel for schedule(dynamic, 1)
    for (int ix = 0; ix < c->nx; ++ix)
        for (int iy = 0; iy < c->ny; ++iy)
            for (int it = 0; it < c->nt; ++it)
                (simd ? ref_straight::pstm_migrate_3d_simd : ref_straight::pstm_migrate_3d)(
                    c->amps, c->sx, c->sy, c->rx, c->ry, c->mx, c->my, c->image, c->fold, c->x_coords, c->y_coords,
                    c->t0_half_sq, c->inv_v_sq, c->t0_s, c->apertures, p,
                    uint3{(unsigned)ix, (unsigned)iy, (unsigned)it});
}

void pstm_ref_migrate_curved(const pstm_ref_call *c, int32_t simd) {
    ref_curved::CurvedRayParams p{};
    p.dx = c->dx;
    p.dy = c->dy;
    p.dt_ms = c->dt_ms;
    p.t_start_ms = c->t_start_ms;
    p.v0 = c->v0;
    p.k = c->k;
    p.max_aperture = c->max_aperture;
    p.min_aperture = c->min_aperture;
    p.taper_fraction = c->taper_fraction;
    p.max_dip_deg = c->max_dip_deg;
    p.apply_spreading = c->spreading;
    p.apply_obliquity = c->obliquity;
    p.apply_aa = c->aa;
    p.aa_dominant_freq = c->aa_dominant_freq;
    p.n_traces = c->n_traces;
    p.n_samples = c->n_samples;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nt = c->nt;
    atomic_int *fold = reinterpret_cast<atomic_int *>(c->fold);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ix = 0; ix < c->nx; ++ix)   // fold[ix, iy] is written by the it = 0 thread only
        for (int iy = 0; iy < c->ny; ++iy)
            for (int it = 0; it < c->nt; ++it)
                (simd ? ref_curved::pstm_migrate_curved_ray_simd : ref_curved::pstm_migrate_curved_ray)(
                    c->amps, c->sx, c->sy, c->rx, c->ry, c->mx, c->my, c->image, fold, c->x_coords, c->y_coords,
                    c->t0_s, c->apertures, p, uint3{(unsigned)ix, (unsigned)iy, (unsigned)it});
}

void pstm_ref_migrate_vti(const pstm_ref_call *c, int32_t simd) {
    ref_vti::VTIParams p{};
    p.dx = c->dx;
    p.dy = c->dy;
    p.dt_ms = c->dt_ms;
    p.t_start_ms = c->t_start_ms;
    p.max_aperture = c->max_aperture;
    p.min_aperture = c->min_aperture;
    p.taper_fraction = c->taper_fraction;
    p.max_dip_deg = c->max_dip_deg;
    p.apply_spreading = c->spreading;
    p.apply_obliquity = c->obliquity;
    p.apply_aa = c->aa;
    p.aa_dominant_freq = c->aa_dominant_freq;
    p.eta_constant = c->eta_constant;
    p.eta_is_1d = c->eta_is_1d;
    p.n_traces = c->n_traces;
    p.n_samples = c->n_samples;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nt = c->nt;
    atomic_int *fold = reinterpret_cast<atomic_int *>(c->fold);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ix = 0; ix < c->nx; ++ix)
        for (int iy = 0; iy < c->ny; ++iy)
            for (int it = 0; it < c->nt; ++it)
                (simd ? ref_vti::pstm_migrate_vti_simd : ref_vti::pstm_migrate_vti)(
                    c->amps, c->sx, c->sy, c->rx, c->ry, c->mx, c->my, c->image, fold, c->x_coords, c->y_coords,
                    c->t0_s, c->inv_v_sq, c->apertures, c->eta, p, uint3{(unsigned)ix, (unsigned)iy, (unsigned)it});
}

// Time-variant form: windows as the shader's TimeWindow records (t_start_ms,
// t_end_ms, dt_effective_ms as float; downsample_factor, sample_offset,
// n_samples as int32), velocity at the base sampling c->dt_ms (nt_base values,
// or nx * ny * nt_base with use_3d_velocity); image and fold are (nx, ny,
// total samples of the windows).  c->t0_s, t0_half_sq, apertures, eta and
// inv_v_sq are not used.
void pstm_ref_migrate_time_variant(const pstm_ref_call *c, const float *vrms_base, int32_t nt_base,
                                   const ref_straight::TimeWindow *windows, int32_t n_windows) {
    ref_straight::TimeVariantParams p{};
    p.dx = c->dx;
    p.dy = c->dy;
    p.dt_base_ms = c->dt_ms;
    p.t_start_ms = c->t_start_ms;
    p.max_aperture = c->max_aperture;
    p.min_aperture = c->min_aperture;
    p.taper_fraction = c->taper_fraction;
    p.max_dip_deg = c->max_dip_deg;
    p.apply_spreading = c->spreading;
    p.apply_obliquity = c->obliquity;
    p.apply_aa = c->aa;
    p.aa_dominant_freq = c->aa_dominant_freq;
    p.n_traces = c->n_traces;
    p.n_samples = c->n_samples;
    p.nx = c->nx;
    p.ny = c->ny;
    p.n_windows = n_windows;
    p.total_output_samples = c->nt;
    p.use_3d_velocity = c->use_3d_velocity;
    p.nt_base = nt_base;
#pragma omp parallel for schedule(dynamic, 1)
    for (int ix = 0; ix < c->nx; ++ix)
        for (int iy = 0; iy < c->ny; ++iy)
            for (int it = 0; it < c->nt; ++it)
                ref_straight::pstm_migrate_time_variant(c->amps, c->sx, c->sy, c->rx, c->ry, c->mx, c->my, c->image,
                                                        c->fold, c->x_coords, c->y_coords, vrms_base, windows, p,
                                                        uint3{(unsigned)ix, (unsigned)iy, (unsigned)it});
}

}  // extern "C"
