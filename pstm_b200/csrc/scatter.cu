// scatter.cu -- the trace-centric (scatter) schedule of the migration.
//
// The reference's trace-centric Metal kernel (pstm_trace_centric.metal:112-236)
// gives every trace one thread that walks the output points inside its
// maximum aperture and adds one atomic per (point, sample); each trace is then
// read once for the whole grid instead of once per tile whose selection box it
// falls in.  Here the same decomposition runs on the gather machinery:
//
//   * the panel (any order; midpoint order keeps the segments compact) is cut
//     into segments of S traces;
//   * segment_boxes (one warp per segment) reduces the segment's midpoint
//     bounding box, grows it by the maximum aperture and finds the pillar
//     index ranges it covers by binary search in the grid axes, then the
//     pillar blocks and the number of (pillar block, time block) items;
//   * scan_counts turns the counts into inclusive prefix sums, on the device,
//     so nothing is read back before the launch;
//   * one persistent launch takes items from a work counter; an item finds its
//     segment by binary search in the prefix sums and migrates the segment's
//     traces against one pillar block and one time block, with the partial
//     sums of the gather kernel (FP32 per chunk in shared memory) and one
//     atomic add per output sample per item -- not one per pair.
//
// Pillars outside a segment's box are farther than the maximum aperture from
// every midpoint of the segment, so they receive nothing from it: image and
// fold (the reference Numba semantics, a count of traces within the maximum
// aperture) equal the gather form's up to the order of the additions.
#include <cuda_runtime.h>
#include <cmath>
#include <string>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "plan.h"
#include "ctx.h"

using namespace pstm;
using namespace pstm::ctx;

namespace {

constexpr int kScanThreads = 1024;

// First index i in [0, n) with a[i] >= x (n when none); a ascending.
__device__ int lower_bound_d(const double *a, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// First index i in [0, n) with a[i] > x (n when none); a ascending.
__device__ int upper_bound_d(const double *a, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One warp per segment: midpoint bounding box grown by `reach`, pillar index
// ranges by binary search in the axes, pillar blocks and item count.
__global__ void segment_boxes(const double *__restrict__ mx, const double *__restrict__ my, int64_t n,
                              int64_t seg_traces, int64_t n_seg, const double *__restrict__ xa, int nx,
                              const double *__restrict__ ya, int ny, double reach, int px, int py, int n_tblk,
                              SegmentBox *__restrict__ boxes, long long *__restrict__ counts,
                              int32_t *__restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int64_t seg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (seg >= n_seg) return;
    if (seg == 0 && lane == 0) {   // the binary searches need ascending axes
        bool ok = true;
        for (int i = 0; i + 1 < nx; ++i) ok = ok && xa[i] <= xa[i + 1];
        for (int i = 0; i + 1 < ny; ++i) ok = ok && ya[i] <= ya[i + 1];
        if (!ok) atomicOr(err, (int)KERR_UNSORTED_AXIS);
    }
    const int64_t b = seg * seg_traces, e = min(n, b + seg_traces);
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (int64_t i = b + lane; i < e; i += 32) {
        const double x = mx[i], y = my[i];
        x0 = fmin(x0, x);
        x1 = fmax(x1, x);
        y0 = fmin(y0, y);
        y1 = fmax(y1, y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane != 0) return;
    const int ix0 = lower_bound_d(xa, nx, x0 - reach), ix1 = upper_bound_d(xa, nx, x1 + reach) - 1;
    const int iy0 = lower_bound_d(ya, ny, y0 - reach), iy1 = upper_bound_d(ya, ny, y1 + reach) - 1;
    SegmentBox bx;
    long long cnt = 0;
    if (e > b && ix0 <= ix1 && iy0 <= iy1) {
        bx = {ix0 / px, ix1 / px, iy0 / py, iy1 / py};
        cnt = (long long)(bx.pbx1 - bx.pbx0 + 1) * (bx.pby1 - bx.pby0 + 1) * n_tblk;
    } else {
        bx = {1, 0, 1, 0};
    }
    boxes[seg] = bx;
    counts[seg] = cnt;
}

// Inclusive prefix sums of counts[0, n) in place, one CTA: every thread sums a
// contiguous slice, the slice sums are scanned in shared memory, then every
// thread rewrites its slice.
__global__ void __launch_bounds__(kScanThreads) scan_counts(long long *counts, int64_t n) {
    __shared__ long long part[kScanThreads];
    const int t = threadIdx.x;
    const int64_t per = (n + kScanThreads - 1) / kScanThreads;
    const int64_t b = t * per, e = min(n, b + per);
    long long s = 0;
    for (int64_t i = b; i < e; ++i) s += counts[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {   // Hillis-Steele inclusive scan of the slice sums
        const long long v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = t > 0 ? part[t - 1] : 0;
    for (int64_t i = b; i < e; ++i) {
        run += counts[i];
        counts[i] = run;
    }
}

}  // namespace

extern "C" int32_t pstm_cuda_migrate_scatter_dev(void *ctx, const pstm_traces_desc *traces, int64_t segment_traces,
                                                 const pstm_output_desc *output, const pstm_velocity_desc *velocity,
                                                 const pstm_params *params, int64_t *n_items_out, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (output && (output->x_grid || output->y_grid))
        return fail(c, PSTM_ERR_UNSUPPORTED, "the scatter schedule needs a regular grid (x_axis, y_axis)");
    if (params && params->interpolation != PSTM_INTERP_LINEAR)
        return fail(c, PSTM_ERR_UNSUPPORTED, "the scatter schedule interpolates linearly");
    if (segment_traces < 0) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "segment_traces must be >= 0");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    if (n_items_out) *n_items_out = 0;
    TilePlan tp;
    int32_t rc = prepare_tile(c, traces, output, velocity, params, st, tp);
    if (rc || tp.empty) return rc;
    const KParams &P = tp.P;
    // segments: a multiple of the staged chunk depth; default 64 chunks
    int64_t S = segment_traces > 0 ? segment_traces : 64 * (int64_t)P.chunk;
    S = (S + P.chunk - 1) / P.chunk * P.chunk;
    const int64_t n_seg = (P.n_traces + S - 1) / S;
    cudaError_t e;
    if ((e = ensure(c->seg_bins, (size_t)n_seg * sizeof(SegmentBox))) != cudaSuccess ||
        (e = ensure(c->scatter_ends, (size_t)n_seg * sizeof(long long))) != cudaSuccess ||
        (e = ensure(c->seg_counter, sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the scatter schedule");
    SegmentBox *boxes = reinterpret_cast<SegmentBox *>(c->seg_bins.ptr);
    long long *ends = reinterpret_cast<long long *>(c->scatter_ends.ptr);
    // a pillar farther than max_aperture (1 + 1e-9) + 1 um from every midpoint
    // of the segment is beyond the FP64 fold and aperture tests of them all
    const double reach = params->max_aperture_m * (1.0 + 1e-9) + 1e-6;
    {
        const int64_t threads = n_seg * 32;
        const int64_t blocks = (threads + 255) / 256;
        if (blocks > 0x7fffffff) return fail(c, PSTM_ERR_UNSUPPORTED, "too many segments");
        segment_boxes<<<(unsigned)blocks, 256, 0, st>>>(traces->midpoint_x, traces->midpoint_y, P.n_traces, S,
                                                        n_seg, output->x_axis, output->nx, output->y_axis,
                                                        output->ny, reach, P.px, P.py, P.n_tblk, boxes, ends, P.err);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "segment_boxes launch");
        scan_counts<<<1, kScanThreads, 0, st>>>(ends, n_seg);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "scan_counts launch");
    }
    if ((e = cudaMemsetAsync(c->seg_counter.ptr, 0, sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(c, e, "clearing the work counter");
    KParams Pa = P;
    Pa.atomic_flush = 1;
    Launch L;
    L.smem = tp.L.smem;
    L.stream = st;
    L.counter = reinterpret_cast<unsigned long long *>(c->seg_counter.ptr);
    L.scatter = ScatterWork{boxes, ends, n_seg, S};
    e = launch_kind(tp.tt, Pa, tp.Pg, tp.amp, tp.per_pillar, tp.prec, L);
    if (e != cudaSuccess) return cuda_fail(c, e, "scatter migrate launch");
    if (n_items_out) {   // diagnostics: the schedule's item count (synchronises the stream)
        long long total = 0;
        if ((e = cudaMemcpyAsync(&total, ends + (n_seg - 1), sizeof(total), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(c, e, "reading the item count");
        *n_items_out = total;
    }
    return PSTM_OK;
}
