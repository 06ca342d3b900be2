/*
 * pstm_cuda.h -- C ABI of the B200 (sm_100a) Kirchhoff PSTM backend.
 *
 * This library is the CUDA counterpart of the reference `pstm` package's
 * kernel backends (Numba CPU, Metal).  Each entry point below names the
 * reference interface it replaces (paths relative to the reference project).
 * All descriptors carry plain pointers and sizes; no C++ or framework types
 * cross this boundary.  Every function returns a pstm_status; 0 is success and
 * a nonzero status leaves a message in pstm_cuda_last_error().
 *
 * Pointer spaces: the *_dev entry points take DEVICE pointers (cudaMalloc'd or
 * any device-accessible memory) and run asynchronously on the given stream;
 * the *_host entry points take HOST pointers, stage them through buffers the
 * context owns and return after the result has been copied back.
 *
 * Accumulation semantics follow the reference Numba backend
 * (pstm/kernels/numba_cpu_optimized.py:147-231): image is accumulated with
 * "+=", and fold receives, for every pillar, the number of traces whose
 * midpoint lies within max_aperture_m, added to every output sample of that
 * pillar when fold is 3-D (nx, ny, nt) or once when it is 2-D (nx, ny).
 */
#ifndef PSTM_CUDA_H
#define PSTM_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSTM_CUDA_ABI_VERSION 5

typedef enum {
    PSTM_OK = 0,
    PSTM_ERR_INVALID_ARGUMENT = 1,  /* reference: ValueError */
    PSTM_ERR_CUDA = 2,              /* reference: RuntimeError from the device */
    PSTM_ERR_OUT_OF_MEMORY = 3,
    PSTM_ERR_NOT_INITIALIZED = 4,   /* reference: RuntimeError("Kernel not initialized") */
    PSTM_ERR_UNSUPPORTED = 5,
    PSTM_ERR_TIMEOUT = 6,           /* a bounded device-side wait gave up */
    PSTM_ERR_INJECTED = 7           /* host-side fault injection (PSTM_CUDA_INJECT_FAULT) */
} pstm_status;

typedef enum { PSTM_AMP_F32 = 0, PSTM_AMP_BF16 = 1, PSTM_AMP_F16 = 2 } pstm_amp_dtype;

/* Traveltime arithmetic of the gather kernels (every traveltime kind).  EXACT
 * forms the fractional sample index in FP64 (the reference Numba path's
 * precision for the interpolation position and the trace-end test).  FAST
 * uses FP32 traveltime and re-takes in FP64 the trace-end tests that fall
 * within 0.01 samples of a trace end.  FP32 is FP32 throughout: traveltime,
 * sample index and trace-end tests, with FP64 only in the coordinate
 * differences of the (pillar, trace) records and the fold test (the
 * precision form's arithmetic).  Weights and accumulation are FP32 in all. */
typedef enum { PSTM_PREC_EXACT = 0, PSTM_PREC_FAST = 1, PSTM_PREC_FP32 = 2 } pstm_precision;
typedef enum { PSTM_IMAGE_F64 = 0, PSTM_IMAGE_F32 = 1 } pstm_image_dtype;

/* Trace interpolators of pstm/kernels/interpolation.py:26-301 (linear is 0
 * here, so a zeroed pstm_params interpolates linearly; the reference numbers
 * nearest 0 and linear 1).  Non-linear methods run a separate FP64 kernel on
 * the per-tile entry points. */
typedef enum {
    PSTM_INTERP_LINEAR = 0, PSTM_INTERP_NEAREST = 1, PSTM_INTERP_CUBIC = 2, PSTM_INTERP_SINC4 = 3,
    PSTM_INTERP_SINC8 = 4, PSTM_INTERP_SINC16 = 5, PSTM_INTERP_LANCZOS3 = 6, PSTM_INTERP_LANCZOS5 = 7
} pstm_interp;

/* Traveltime kinds.  Reference: executor dispatch pstm/pipeline/executor.py:1691-1745
 * (migrate_tile / migrate_tile_curved_ray / migrate_tile_vti). */
typedef enum {
    PSTM_TT_STRAIGHT = 0,    /* DSR, numba_cpu_optimized.py:192-194 */
    PSTM_TT_CURVED = 1,      /* V(z)=v0+kz, pstm_curved_ray.metal:50-96 */
    PSTM_TT_VTI = 2,         /* eta moveout, pstm_anisotropic_vti.metal:103-148 */
    PSTM_TT_CURVED_VTI = 3   /* curved leg x VTI/hyperbolic leg ratio (no reference formula) */
} pstm_traveltime;

/* Trace panel + geometry.  Reference carrier: TraceBlock, pstm/kernels/base.py:27-116. */
typedef struct {
    const void *amplitudes;       /* (n_traces, amp_row_stride) of amp_dtype */
    int32_t amp_dtype;            /* pstm_amp_dtype */
    int32_t n_samples;            /* samples per trace (>= 2) */
    int64_t n_traces;
    int64_t amp_row_stride;       /* elements between trace rows (>= n_samples) */
    const double *source_x, *source_y;
    const double *receiver_x, *receiver_y;
    const double *midpoint_x, *midpoint_y;
    const double *weights;        /* nullable: all ones */
    double sample_rate_ms;
    double start_time_ms;
} pstm_traces_desc;

/* Output tile.  Reference carrier: OutputTile, pstm/kernels/base.py:119-177. */
typedef struct {
    void *image;                  /* (nx, ny, nt), accumulated with += */
    int32_t image_dtype;          /* pstm_image_dtype */
    int32_t fold_is_3d;           /* 1: fold is (nx, ny, nt); 0: (nx, ny) */
    int32_t *fold;                /* nullable */
    int32_t nx, ny, nt;
    const double *x_axis;         /* (nx) */
    const double *y_axis;         /* (ny) */
    const double *x_grid;         /* nullable (nx*ny): rotated-grid coordinates */
    const double *y_grid;         /* nullable (nx*ny) */
    const double *t_axis_ms;      /* (nt) output times */
} pstm_output_desc;

/* RMS velocity.  Reference carrier: VelocitySlice, pstm/kernels/base.py:180-194. */
typedef struct {
    const double *vrms;           /* (nt) or (nx, ny, nt) */
    int32_t is_3d;
    int32_t reserved;
} pstm_velocity_desc;

/* Kernel parameters.  Reference carrier: KernelConfig, pstm/kernels/base.py:197-265. */
typedef struct {
    double max_aperture_m;
    double min_aperture_m;
    double max_dip_degrees;
    double taper_fraction;
    int32_t apply_spreading;
    int32_t apply_obliquity;
    int32_t aa_enabled;           /* triangle AA weight, pstm_migration.metal:95-132 */
    int32_t traveltime;           /* pstm_traveltime */
    double aa_dominant_freq;      /* Hz; reference default 30 (metal_compiled.py:706) */
    double grid_dx, grid_dy;      /* bin spacing used by the AA weight */
    double curved_v0, curved_k;   /* V(z) = v0 + k z */
    const double *eta;            /* nullable: eta_constant; else (nt) or (nx, ny, nt) */
    int32_t eta_is_3d;
    int32_t compensated;          /* 1: compensated (TwoSum) FP32 accumulation */
    double eta_constant;
    int32_t precision;            /* pstm_precision */
    int32_t interpolation;        /* pstm_interp; KernelConfig.interpolation_method, base.py:213 */
} pstm_params;

/* Library / ABI version (no reference counterpart: a binding sanity check). */
int32_t pstm_cuda_abi_version(void);

/* Create a context on a CUDA device.  Replaces the backend constructor +
 * initialize(): MigrationKernel.initialize, pstm/kernels/base.py:302;
 * OptimizedNumbaKernel.initialize, numba_cpu_optimized.py:498-543. */
int32_t pstm_cuda_create(int32_t device, void **ctx_out);

/* Release a context and every buffer it owns.  Replaces
 * MigrationKernel.cleanup, pstm/kernels/base.py:317. */
void pstm_cuda_destroy(void *ctx);

/* Migrate one tile, device pointers, asynchronous on `stream` (a
 * cudaStream_t; NULL = the context's stream; pass cudaStreamLegacy, 0x1, for
 * the legacy default stream).  Calls on one context must not overlap on the
 * device: the context's per-launch tables are reused by the next call.  Replaces
 * MigrationKernel.migrate_tile, base.py:305-313;
 * OptimizedNumbaKernel.migrate_tile, numba_cpu_optimized.py:545-626;
 * CompiledMetalKernel.migrate_tile[_curved_ray/_vti], metal_compiled.py:567,1275,1456. */
int32_t pstm_cuda_migrate_tile_dev(void *ctx, const pstm_traces_desc *traces,
                                   const pstm_output_desc *output,
                                   const pstm_velocity_desc *velocity,
                                   const pstm_params *params, void *stream);

/* Migrate one tile against the traces of `n_runs` ranges of a resident panel:
 * runs[2i] .. runs[2i+1] - 1, ascending and disjoint, inside [0, n_traces).
 * The result is that of pstm_cuda_migrate_tile_dev on the concatenation of the
 * ranges, up to the order of floating-point additions, without copying the
 * ranges together: geometry is packed for the span of the runs and one
 * persistent launch takes (run segment, pillar block, time block) items that
 * add into the image and fold atomically (non-linear interpolation: one
 * migration per run).  A panel sorted by midpoint (pstm_b200.spatial) gives
 * each output tile's traces as a few such runs.  Device pointers;
 * asynchronous on `stream` as pstm_cuda_migrate_tile_dev.  Replaces the
 * executor's per-tile trace query and gather, SpatialIndex.query_traces_for_tile
 * (pstm/data/spatial_index.py:423-460) followed by the trace load of
 * _process_tile (pstm/pipeline/executor.py:1397-1858). */
int32_t pstm_cuda_migrate_tile_runs_dev(void *ctx, const pstm_traces_desc *traces, const int64_t *runs,
                                        int32_t n_runs, const pstm_output_desc *output,
                                        const pstm_velocity_desc *velocity, const pstm_params *params,
                                        void *stream);

/* The trace-centric (scatter) schedule of a migration: instead of every tile
 * reading every trace of its selection box, every trace is read for the whole
 * output grid once.  The panel is cut into segments of segment_traces traces
 * (0: 64 staged chunks; midpoint order, pstm_b200.spatial, keeps segments
 * compact); on the device, each segment's midpoint box grown by the maximum
 * aperture is mapped to pillar blocks by binary search in the ascending grid
 * axes, the item counts are prefix-summed, and one persistent launch
 * migrates (segment, pillar block, time block) items with FP32 partial sums
 * per chunk and one atomic add per output sample per item.  Same result as
 * pstm_cuda_migrate_tile_dev up to the order of floating-point additions;
 * regular grids (x_axis, y_axis) and linear interpolation only.  Device
 * pointers; asynchronous on `stream`, except that a non-null n_items_out
 * synchronises it to report the number of items.  Replaces the reference's
 * trace-centric kernel, pstm/metal/shaders/pstm_trace_centric.metal:112-236
 * (one thread per trace, one atomic add per pair, a per-sample fold: here the
 * fold is the Numba count of traces within the maximum aperture). */
int32_t pstm_cuda_migrate_scatter_dev(void *ctx, const pstm_traces_desc *traces, int64_t segment_traces,
                                      const pstm_output_desc *output, const pstm_velocity_desc *velocity,
                                      const pstm_params *params, int64_t *n_items_out, void *stream);

/* Same, host pointers: inputs are copied to the device, the tile is migrated
 * and image/fold are copied back and accumulated (+=) into the host arrays.
 * Synchronous, like the reference backends.  Native precedent: the pybind11
 * migrate_tile binding, pstm/metal/src/bindings.cpp:48-62. */
int32_t pstm_cuda_migrate_tile_host(void *ctx, const pstm_traces_desc *traces,
                                    const pstm_output_desc *output,
                                    const pstm_velocity_desc *velocity,
                                    const pstm_params *params);

/* Allocation-free variant of pstm_cuda_migrate_tile_dev; it has no
 * counterpart in the reference.  It is for callers that cannot allocate
 * device memory while they run -- an application whose memory manager owns
 * the whole GPU, or a job that must not stall the device (cudaMalloc
 * synchronises it) or fail on an allocation after start-up.  It needs no
 * context and allocates nothing: its scratch (tables, packed geometry, launch
 * parameters) is a fixed 16 MiB array in this library's device memory, held
 * by every device that loads the library until the process exits.  Limits of
 * one call: n_traces <= 131072, nt <= 8192, and (nx*ny if the velocity or eta
 * is 3-D, else 1) * nt <= 262144; larger inputs are rejected with
 * PSTM_ERR_INVALID_ARGUMENT (split the traces over several calls: image and
 * fold accumulate).  Inputs and outputs are device pointers; work is queued
 * on `stream` (NULL = the legacy default stream) of the calling thread's
 * current device.  The first call on a device looks up the array's address;
 * make that first call before any stream capture.  All calls share the array,
 * so calls that overlap on the GPU race: serialise them.  The call is
 * asynchronous: its return status covers argument checks and launches, and
 * device-side failures are read afterwards with pstm_cuda_noalloc_status.
 * Messages are reported by pstm_cuda_last_error(NULL). */
int32_t pstm_cuda_migrate_tile_noalloc(const pstm_traces_desc *traces, const pstm_output_desc *output,
                                       const pstm_velocity_desc *velocity, const pstm_params *params,
                                       void *stream);

/* Device-side status of the last pstm_cuda_migrate_tile_noalloc call on the
 * current device (no reference counterpart; the allocation-free form has
 * none).  Waits for `stream` (NULL = the legacy default stream), then reads the
 * kernel's error word from the fixed scratch array without allocating:
 * PSTM_OK, or PSTM_ERR_TIMEOUT when a bounded device-side wait gave up -- the
 * image and fold of that call may then hold partial sums and must be
 * discarded.  Each allocation-free call clears the word when it starts. */
int32_t pstm_cuda_noalloc_status(void *stream);

/* The precision form's trace format (no reference counterpart: the reference
 * keeps FP32 traces, TraceBlock.amplitudes, pstm/kernels/base.py:27-116).
 * Converts n_traces FP32 rows (src, src_stride elements apart) to FP16 rows
 * (dst, dst_stride elements apart) with one power-of-two scale per trace --
 * the trace times 2^e, its largest |amplitude| in [2^13, 2^14) -- and writes
 * weights_out[i] = (weights ? weights[i] : 1) * 2^-e, so that migrating the
 * FP16 panel with weights_out gives the FP32 panel's image up to the FP16
 * rounding of the amplitudes.  Device pointers; asynchronous on `stream`
 * (NULL = the context's stream). */
int32_t pstm_cuda_traces_to_f16(void *ctx, const float *src, int64_t n_traces, int32_t n_samples,
                                int64_t src_stride, void *dst, int64_t dst_stride, const double *weights,
                                double *weights_out, void *stream);

/* One output of the batched form: a contiguous range of the batch's traces and
 * its own image and fold.  Reference: one bin of the gather-bin loop,
 * pstm/pipeline/executor.py:960-975, which migrates every offset/OVT bin into
 * its own volume (_migrate_single_bin, executor.py:977). */
typedef struct {
    int64_t trace_begin;          /* first trace of the bin in the traces descriptor */
    int64_t n_traces;             /* traces of the bin, contiguous */
    void *image;                  /* device, (nx, ny, nt) of output->image_dtype, += */
    int32_t *fold;                /* device, nullable; shaped as output->fold_is_3d says */
} pstm_bin_desc;

/* Launch shape chosen by pstm_cuda_autotune_bins. */
typedef struct {
    int32_t pillars_per_cta;      /* output traces one CTA migrates together */
    int32_t times_per_lane;       /* output times per thread (512 * this per CTA) */
    int32_t traces_per_chunk;     /* depth of the staged trace panel */
    int32_t n_candidates;         /* shapes timed */
    float best_ms;                /* time of the chosen shape on the tuning sample */
    float default_ms;             /* time of the untuned default shape on the same sample */
} pstm_tune_result;

/* Migrate many bins that share one output tile geometry, velocity and
 * parameters in ONE persistent launch: one CTA per SM takes (bin, pillar
 * block, time block) items from a work counter, the bins with the most traces
 * first, so bins of very different sizes keep every SM busy.  The whole
 * sequence (table preparation, geometry packing, the launch) is captured in a
 * CUDA graph that the context keeps and replays while the arguments repeat;
 * new arguments re-capture it.  `output` gives the tile geometry (its image
 * and fold pointers are ignored; each bin has its own, and they must not
 * overlap).  Device pointers; asynchronous on `stream` as
 * pstm_cuda_migrate_tile_dev; at most 4096 bins.  Uses the shape that
 * pstm_cuda_autotune_bins chose for this class of workload, if it ran.
 * Replaces the per-bin sequence of migrate_tile calls of the executor
 * (executor.py:960-975 -> :1730). */
int32_t pstm_cuda_migrate_bins_dev(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                   const pstm_velocity_desc *velocity, const pstm_params *params,
                                   const pstm_bin_desc *bins, int32_t n_bins, void *stream);

/* Autotuner of the batched form (no reference counterpart; the reference
 * picks its threadgroup shape by a fixed rule, compute_optimal_threadgroup,
 * pstm/kernels/metal_compiled.py:292-335, used at :742-743).  Times
 * candidate launch shapes (pillars per CTA, output times per lane, traces per
 * chunk) on a sample of the batch -- the largest bins, clipped so that one
 * candidate migrates about `pairs_per_candidate` sample-trace pairs (0: 2^36)
 * into scratch outputs of the context -- keeps the fastest for this class of
 * workload (traveltime kind, trace dtype, 3-D velocity, precision, nt, ns) and
 * reports it.  Synchronous; the bins' images and folds are not touched. */
int32_t pstm_cuda_autotune_bins(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                const pstm_velocity_desc *velocity, const pstm_params *params,
                                const pstm_bin_desc *bins, int32_t n_bins, int64_t pairs_per_candidate,
                                pstm_tune_result *result);

/* ---------------------------------------------------------------- learned form
 * A 7 -> 64 -> 64 -> 64 -> 1 SiLU network (BF16 weights on the tensor cores,
 * FP32 accumulation) approximates the VTI or curved+VTI traveltime as the
 * straight-ray DSR time plus a learned residual:
 *   T = T_DSR(t0, h_s, h_r, v_rms) + out_scale * net((x - shift) * scale),
 *   x = (t0 [s], dx_s, dy_s, dx_r, dy_r [m, output point minus source /
 *   receiver], v_rms [m/s], eta).
 * No reference counterpart: the reference evaluates the formulas only
 * (pstm_anisotropic_vti.metal:103-148, pstm_curved_ray.metal:50-96). */
typedef struct {
    int32_t traveltime;           /* PSTM_TT_VTI or PSTM_TT_CURVED_VTI */
    int32_t reserved;
    double curved_v0, curved_k;   /* curved+VTI: V(z) = v0 + k z */
    double t0_max_s;              /* t0 uniform in [0, t0_max_s] */
    double h_max_m;               /* dx_s, dy_s, dx_r, dy_r uniform in [-h_max_m, h_max_m] */
    double v_a, v_b, v_rel;       /* v_rms = (v_a + v_b t0) (1 + v_rel u), u uniform in [-1, 1] */
    double eta_slope, eta_jitter, eta_max;   /* eta = clip(eta_slope t0 + eta_jitter u', 0, eta_max) */
} pstm_surrogate_domain;

typedef struct {
    float shift[8], scale[8];     /* input normalisation (entries 7 unused) */
    float out_scale;              /* seconds per unit of network output */
    int32_t traveltime;           /* the kind the network was trained on */
    const float *params;          /* device: pstm_cuda_surrogate_param_count() FP32 parameters */
} pstm_surrogate;

typedef struct {
    float probe_max_ms;           /* largest |T_surrogate - T_exact| over the in-aperture probes */
    float probe_rms_ms;
    int32_t n_probe_used;         /* probes that fell inside their pair's aperture */
    int32_t used_surrogate;       /* 1: the tile was migrated with the surrogate; 0: exact fallback */
} pstm_learned_report;

/* Number of FP32 parameters of the network (layout W1[64][7] b1 W2[64][64] b2 W3 b3 w4[64] b4). */
int32_t pstm_cuda_surrogate_param_count(void);

/* Seeded training/evaluation samples with exact FP64 targets: for sample
 * first+j (j < n), raw[8 j .. 8 j + 6] = x (FP32) and residual[j] =
 * T_exact - T_DSR (s); t_exact (nullable) gets T_exact.  Device pointers. */
int32_t pstm_cuda_surrogate_samples(void *ctx, const pstm_surrogate_domain *domain, uint64_t seed, int64_t first,
                                    int32_t n, float *raw, float *residual, double *t_exact, void *stream);

/* Forward and backward pass over n samples: grads += d(mean squared error of
 * the normalised residual)/d(params), loss_sum += the sum of squared errors. */
int32_t pstm_cuda_surrogate_gradients(void *ctx, const pstm_surrogate *net, const float *raw, const float *residual,
                                      int32_t n, float *grads, float *loss_sum, void *stream);

/* One Adam step (beta 0.9 / 0.999, bias-corrected) on params; clears grads. */
int32_t pstm_cuda_surrogate_adam(void *ctx, float *params, float *grads, float *m, float *v, int32_t step, float lr,
                                 void *stream);

/* Network residual (s) of n samples (raw as written by pstm_cuda_surrogate_samples). */
int32_t pstm_cuda_surrogate_eval(void *ctx, const pstm_surrogate *net, const float *raw, int32_t n, float *residual,
                                 void *stream);

/* The learned form of pstm_cuda_migrate_tile_dev: n_probe random in-aperture
 * (pillar, trace, time) pairs of the tile compare the surrogate with the exact
 * FP64 traveltime; if the largest residual is at most max_residual_ms (0: the
 * default 0.1 ms; negative: always use the surrogate) the tile is migrated
 * with the surrogate traveltime, else with the exact kernel.  params->traveltime
 * must be the network's kind.  Synchronises the stream once (the probe). */
int32_t pstm_cuda_migrate_tile_learned_dev(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                           const pstm_velocity_desc *velocity, const pstm_params *params,
                                           const pstm_surrogate *net, float max_residual_ms, int32_t n_probe,
                                           pstm_learned_report *report, void *stream);

/* Linear interpolation of n_rows rows of n_src samples (dtype: PSTM_IMAGE_F64
 * or PSTM_IMAGE_F32) from the ascending times src_times onto dst_times, the
 * edge value outside (np.interp's rule); all device pointers.  Replaces the
 * per-trace np.interp of resample_to_uniform,
 * pstm/algorithm/time_variant.py:354-397, for device images. */
int32_t pstm_cuda_interp_rows(void *ctx, int32_t dtype, const void *src, int64_t n_rows, int32_t n_src,
                              const double *src_times, int32_t n_dst, const double *dst_times, void *dst,
                              void *stream);

/* Measured MUFU (special-function unit) throughput of `device`, in operations
 * per second: a full-occupancy grid of independent sqrt.approx / rcp.approx
 * chains, timed with CUDA events (best of three after a warm-up).  No
 * reference counterpart: the denominator of the gather kernel's roofline, whose
 * per-pair work is counted in MUFU operations.  Synchronous; allocates a
 * small sink buffer. */
int32_t pstm_cuda_measure_sfu_peak(int32_t device, double *ops_per_second);

/* Wait for all work queued on the context's stream.  Replaces
 * MigrationKernel.synchronize, pstm/kernels/base.py:315. */
int32_t pstm_cuda_synchronize(void *ctx);

/* Message of the last failing call on this context (or, when ctx is NULL, of
 * the calling thread's last failing pstm_cuda_create or
 * pstm_cuda_migrate_tile_noalloc).  Reference: the RuntimeError text the
 * Metal backend raises, metal_compiled.py:763-764. */
const char *pstm_cuda_last_error(void *ctx);

#ifdef __cplusplus
}
#endif
#endif /* PSTM_CUDA_H */
