// capi.cu -- the C ABI declared in include/pstm_cuda.h: contexts, argument
// validation, launch-parameter derivation and the host-pointer staging path.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "plan.h"
#include "ctx.h"

using namespace pstm;

namespace {
thread_local std::string g_create_err;
}

namespace pstm {
// Message of the last failing call that has no context (create, noalloc).
void set_context_free_error(const std::string &msg) { g_create_err = msg; }

namespace ctx {

int32_t fail(Ctx *c, int32_t code, const std::string &msg) {
    if (c) c->err = msg;
    else g_create_err = msg;
    return code;
}

int32_t cuda_fail(Ctx *c, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(c, e == cudaErrorMemoryAllocation ? PSTM_ERR_OUT_OF_MEMORY : PSTM_ERR_CUDA, m);
}

bool injected(const char *site) {
    const char *v = std::getenv("PSTM_CUDA_INJECT_FAULT");
    if (!v || !*v) return false;
    return std::strcmp(v, site) == 0 || std::strcmp(v, "all") == 0;
}

cudaError_t ensure(DevBuf &b, size_t bytes) {
    if (bytes <= b.bytes && b.ptr) return cudaSuccess;
    if (b.ptr) {
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e == cudaSuccess) b.bytes = want;
    return e;
}

void release(DevBuf &b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

}  // namespace ctx
}  // namespace pstm

namespace {

using namespace pstm::ctx;

using plan::amp_elem_bytes;
using plan::make_params;

int32_t validate(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out,
                 const pstm_velocity_desc *vel, const pstm_params *prm) {
    const char *msg = "";
    const int32_t rc = plan::check_args(tr, out, vel, prm, msg);
    return rc ? fail(c, rc, msg) : PSTM_OK;
}

}  // namespace

namespace pstm {
namespace ctx {

int32_t prepare_tile(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_velocity_desc *vel,
                     const pstm_params *prm, cudaStream_t st, TilePlan &tp) {
    tp.empty = true;
    int32_t rc = validate(c, tr, out, vel, prm);
    if (rc) return rc;
    if (injected("migrate")) return fail(c, PSTM_ERR_INJECTED, "injected fault: migrate");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    int R, PB;
    plan::choose_shape(out->nt, c->force_r, c->force_pb, R, PB, tr->amp_dtype);
    KParams &P = tp.P;
    P = make_params(tr, out, vel, prm, PB);
    if (tr->n_traces == 0) return PSTM_OK;   // nothing to add: image += 0, fold += 0

    const bool per_pillar = vel->is_3d || (prm->eta && prm->eta_is_3d);
    const int64_t n_p = per_pillar ? (int64_t)out->nx * out->ny : 1;
    const size_t n_tab = (size_t)n_p * out->nt;
    if ((e = ensure(c->ttab, n_tab * sizeof(float4))) != cudaSuccess ||
        (e = ensure(c->btab, n_tab * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->ttime, (size_t)out->nt * 2 * sizeof(float4))) != cudaSuccess ||
        (e = ensure(c->ttimeA, (size_t)out->nt * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->ttimeV, (size_t)out->nt * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->errword, sizeof(int32_t))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the per-time tables");
    float4 *tab = reinterpret_cast<float4 *>(c->ttab.ptr);
    double *btab = reinterpret_cast<double *>(c->btab.ptr);
    const bool exact = prm->precision == PSTM_PREC_EXACT;
    P.exact_units = exact ? 1 : 0;
    P.curved_kind = (prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI) ? 1 : 0;
    {
        int blocks = (int)(((int64_t)n_tab + 255) / 256);
        if (blocks > 148 * 32) blocks = 148 * 32;
        prep_time_table<<<blocks, 256, 0, st>>>(P, n_p, tab, btab, reinterpret_cast<float4 *>(c->ttime.ptr),
                                                reinterpret_cast<double *>(c->ttimeA.ptr),
                                                reinterpret_cast<double *>(c->ttimeV.ptr));
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "prep_time_table launch");
    }
    P.ttime = reinterpret_cast<const float4 *>(c->ttime.ptr);
    P.ttimeA = reinterpret_cast<const double *>(c->ttimeA.ptr);
    P.ttimeV = reinterpret_cast<const double *>(c->ttimeV.ptr);
    P.ttab = tab;
    P.btab = btab;
    P.err = reinterpret_cast<int32_t *>(c->errword.ptr);
    if ((e = cudaMemsetAsync(P.err, 0, sizeof(int32_t), st)) != cudaSuccess)
        return cuda_fail(c, e, "clearing the error word");

    // packed FP64 geometry, staged per chunk by TMA bulk copies
    if ((e = ensure(c->packed_geo, (size_t)tr->n_traces * kGeoDoubles * sizeof(double))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the packed geometry");
    {
        int blocks = (int)((tr->n_traces + 255) / 256);
        if (blocks > 148 * 32) blocks = 148 * 32;
        pack_geometry<<<blocks, 256, 0, st>>>(P, reinterpret_cast<double *>(c->packed_geo.ptr));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "pack_geometry launch");
    }
    P.geo = reinterpret_cast<const double *>(c->packed_geo.ptr);

    // shared-memory staging of trace rows: pitch rounded up to 16 bytes; TMA
    // bulk copies when the rows are 16-byte aligned and the padded row is
    // inside the caller's stride, else a plain cooperative copy
    size_t smem = 0;
    if (!plan::plan_staging(P, tr, prm, PB, R, c->smem_optin, smem))
        return fail(c, PSTM_ERR_UNSUPPORTED, "trace rows too long to stage in shared memory");

    // a device copy of the launch parameters for the kernel's rare FP64 paths
    e = ensure(c->kparams, sizeof(KParams));
    if (e != cudaSuccess) return cuda_fail(c, e, "allocating the parameter block");
    e = cudaMemcpyAsync(c->kparams.ptr, &P, sizeof(KParams), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "copying the parameter block");
    const KParams *Pg = reinterpret_cast<const KParams *>(c->kparams.ptr);

    const int n_pblk_x = (out->nx + P.px - 1) / P.px;
    const int64_t nblk_p = (int64_t)n_pblk_x * P.n_pblk_y;
    const int tb = kThreads * R;
    const int nblk_t = (out->nt + tb - 1) / tb;
    if (nblk_p > 0x7fffffff || nblk_t > 65535) return fail(c, PSTM_ERR_UNSUPPORTED, "tile too large for one launch");
    tp.Pg = Pg;
    tp.L = Launch();
    tp.L.grid = dim3((unsigned)nblk_p, (unsigned)nblk_t);
    tp.L.smem = smem;
    tp.L.stream = st;
    tp.tt = prm->traveltime;
    tp.amp = tr->amp_dtype;
    tp.per_pillar = per_pillar;
    tp.exact = exact;
    tp.prec = prm->precision;
    tp.n_p = n_p;
    tp.empty = false;
    return PSTM_OK;
}

// Trace-segment length of the segment-major schedule for this tile (0: the
// context never splits).
int64_t segment_traces(const Ctx *c, const KParams &P) {
    if (c->segment_bytes <= 0) return 0;
    const int64_t row_bytes = (int64_t)P.pitch * P.elem;
    const int64_t S = c->segment_bytes / row_bytes;
    return S < 16 * (int64_t)P.chunk ? 16 * (int64_t)P.chunk : S / P.chunk * P.chunk;
}

// Items for traces [b0, b0 + n) of the prepared panel, S traces at most each
// (S <= 0: one item).
void append_segments(std::vector<BinWork> &w, int64_t b0, int64_t n, int64_t S, void *image, int32_t *fold) {
    if (S <= 0) S = n;
    for (int64_t b = 0; b < n; b += S) w.push_back({b0 + b, (n - b) < S ? (n - b) : S, image, fold});
}

// One persistent launch over a list of trace items of the prepared tile, all
// adding into its image and fold atomically.
int32_t launch_items(Ctx *c, const TilePlan &tp, const std::vector<BinWork> &w) {
    if (w.size() > (size_t)0x7fffffff) return fail(c, PSTM_ERR_UNSUPPORTED, "too many trace items for one launch");
    cudaError_t e;
    if ((e = ensure(c->seg_bins, w.size() * sizeof(BinWork))) != cudaSuccess ||
        (e = ensure(c->seg_counter, sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the segment list");
    if ((e = cudaMemcpyAsync(c->seg_bins.ptr, w.data(), w.size() * sizeof(BinWork), cudaMemcpyHostToDevice,
                             tp.L.stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->seg_counter.ptr, 0, sizeof(unsigned long long), tp.L.stream)) != cudaSuccess)
        return cuda_fail(c, e, "writing the segment list");
    KParams P = tp.P;
    P.atomic_flush = 1;
    Launch L;
    L.smem = tp.L.smem;
    L.stream = tp.L.stream;
    L.bins = reinterpret_cast<const BinWork *>(c->seg_bins.ptr);
    L.n_bins = (int)w.size();
    L.counter = reinterpret_cast<unsigned long long *>(c->seg_counter.ptr);
    e = launch_kind(tp.tt, P, tp.Pg, tp.amp, tp.per_pillar, tp.prec, L);
    return e == cudaSuccess ? PSTM_OK : cuda_fail(c, e, "segmented migrate kernel launch");
}

// A panel much larger than L2 is migrated segment by segment: the persistent
// kernel takes items (trace segment, pillar block, time block) in segment
// order, so every resident CTA streams the same L2-sized segment at a time
// and the panel is read from DRAM about once instead of once per CTA; the
// items of a pillar block in different segments add into the image and fold
// atomically.
int32_t launch_tile(Ctx *c, const TilePlan &tp) {
    const KParams &P0 = tp.P;
    const int64_t row_bytes = (int64_t)P0.pitch * P0.elem;
    if (c->segment_bytes > 0 && P0.n_traces * row_bytes > 2 * c->segment_bytes) {
        std::vector<BinWork> w;
        append_segments(w, 0, P0.n_traces, segment_traces(c, P0), P0.image, P0.fold);
        return launch_items(c, tp, w);
    }
    const cudaError_t e = launch_kind(tp.tt, tp.P, tp.Pg, tp.amp, tp.per_pillar, tp.prec, tp.L);
    return e == cudaSuccess ? PSTM_OK : cuda_fail(c, e, "migrate kernel launch");
}

}  // namespace ctx
}  // namespace pstm

namespace {

int32_t run_dev(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out,
                const pstm_velocity_desc *vel, const pstm_params *prm, cudaStream_t st) {
    TilePlan tp;
    const int32_t rc = prepare_tile(c, tr, out, vel, prm, st, tp);
    if (rc || tp.empty) return rc;
    if (prm->interpolation != PSTM_INTERP_LINEAR) return launch_interp(c, tp, prm->interpolation, out);
    return launch_tile(c, tp);
}

}  // namespace

// Read back the kernels' error word (after the stream has drained).
int32_t pstm::ctx::check_error_word(Ctx *c) {
    if (!c->errword.ptr) return PSTM_OK;
    int32_t w = 0;
    cudaError_t e = cudaMemcpy(&w, c->errword.ptr, sizeof(w), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(c, e, "reading the error word");
    if (w & KERR_UNSORTED_AXIS)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT,
                    "the scatter schedule needs ascending x and y axes; the image and fold were not computed "
                    "correctly and must be discarded");
    if (w & KERR_WAIT_TIMEOUT)
        return fail(c, PSTM_ERR_TIMEOUT,
                    "a bounded wait for a trace-row copy gave up; the image and fold may hold partial sums "
                    "of this call and must be discarded");
    return PSTM_OK;
}

namespace {

template <typename T>
cudaError_t stage(DevBuf &b, const T *src, size_t count, cudaStream_t st, const T **dst) {
    if (!src) {
        *dst = nullptr;
        return cudaSuccess;
    }
    cudaError_t e = ensure(b, count * sizeof(T));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(b.ptr, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
    *dst = reinterpret_cast<const T *>(b.ptr);
    return e;
}

}  // namespace

extern "C" {

int32_t pstm_cuda_abi_version(void) { return PSTM_CUDA_ABI_VERSION; }

int32_t pstm_cuda_create(int32_t device, void **ctx_out) {
    if (!ctx_out) return fail(nullptr, PSTM_ERR_INVALID_ARGUMENT, "ctx_out is null");
    *ctx_out = nullptr;
    if (injected("create")) return fail(nullptr, PSTM_ERR_INJECTED, "injected fault: create");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(nullptr, PSTM_ERR_INVALID_ARGUMENT, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    Ctx *c = new Ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(nullptr, e, "cudaStreamCreate");
    }
    e = cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return cuda_fail(nullptr, e, "cudaDeviceGetAttribute");
    }
    const char *rr = std::getenv("PSTM_CUDA_R");   // output times per lane override (1..4)
    if (rr) c->force_r = std::atoi(rr);
    const char *pb = std::getenv("PSTM_CUDA_PB");   // pillars per CTA override (1..16)
    if (pb) c->force_pb = std::atoi(pb);
    const char *seg = std::getenv("PSTM_CUDA_SEGMENT_MB");   // trace-segment size; 0: never split a panel
    if (seg) c->segment_bytes = (int64_t)std::atoll(seg) << 20;
    *ctx_out = c;
    return PSTM_OK;
}

void pstm_cuda_destroy(void *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release(c->ttab);
    release(c->btab);
    release(c->ttime);
    release(c->ttimeA);
    release(c->ttimeV);
    release(c->kparams);
    release(c->errword);
    release(c->packed_geo);
    release(c->amps);
    for (auto &g : c->geo) release(g);
    release(c->xa); release(c->ya); release(c->xg); release(c->yg); release(c->ta);
    release(c->vel); release(c->eta); release(c->image); release(c->fold);
    release(c->scatter_ends);
    release_batch(c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int32_t pstm_cuda_migrate_tile_dev(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                   const pstm_velocity_desc *velocity, const pstm_params *params, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    return run_dev(c, traces, output, velocity, params, st);
}

namespace {

// The traces [a, a + n) of a panel as a panel of their own (no copy).
pstm_traces_desc sub_panel(const pstm_traces_desc &t, int64_t a, int64_t n) {
    pstm_traces_desc s = t;
    s.amplitudes = static_cast<const unsigned char *>(t.amplitudes) +
                   a * t.amp_row_stride * (int64_t)amp_elem_bytes(t.amp_dtype);
    s.source_x = t.source_x + a;
    s.source_y = t.source_y + a;
    s.receiver_x = t.receiver_x + a;
    s.receiver_y = t.receiver_y + a;
    s.midpoint_x = t.midpoint_x + a;
    s.midpoint_y = t.midpoint_y + a;
    if (t.weights) s.weights = t.weights + a;
    s.n_traces = n;
    return s;
}

}  // namespace

int32_t pstm_cuda_migrate_tile_runs_dev(void *ctx, const pstm_traces_desc *traces, const int64_t *runs,
                                        int32_t n_runs, const pstm_output_desc *output,
                                        const pstm_velocity_desc *velocity, const pstm_params *params,
                                        void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (!traces || n_runs < 0 || (n_runs > 0 && !runs))
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "runs: n_runs >= 0 [begin, end) pairs required");
    int32_t rc = validate(c, traces, output, velocity, params);
    if (rc) return rc;
    std::vector<std::pair<int64_t, int64_t>> rv;
    int64_t prev = 0;
    for (int32_t i = 0; i < n_runs; ++i) {
        const int64_t a = runs[2 * i], b = runs[2 * i + 1];
        if (a < prev || b < a || b > traces->n_traces)
            return fail(c, PSTM_ERR_INVALID_ARGUMENT,
                        "runs must be ascending, disjoint [begin, end) trace ranges inside the panel");
        prev = b;
        if (b > a) rv.emplace_back(a, b);
    }
    if (rv.empty()) return PSTM_OK;   // no traces: image += 0, fold += 0
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    if (params->interpolation != PSTM_INTERP_LINEAR || rv.size() == 1) {
        for (const auto &r : rv) {
            const pstm_traces_desc sub = sub_panel(*traces, r.first, r.second - r.first);
            if ((rc = run_dev(c, &sub, output, velocity, params, st)) != PSTM_OK) return rc;
        }
        return PSTM_OK;
    }
    // One tile preparation over the span of the runs (geometry packed for the
    // span) and one persistent launch over the runs' segments.
    const int64_t a0 = rv.front().first;
    const pstm_traces_desc span = sub_panel(*traces, a0, rv.back().second - a0);
    TilePlan tp;
    if ((rc = prepare_tile(c, &span, output, velocity, params, st, tp)) != PSTM_OK || tp.empty) return rc;
    const int64_t S = segment_traces(c, tp.P);
    std::vector<BinWork> w;
    for (const auto &r : rv) append_segments(w, r.first - a0, r.second - r.first, S, tp.P.image, tp.P.fold);
    return launch_items(c, tp, w);
}

static int32_t migrate_host_impl(Ctx *c, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                 const pstm_velocity_desc *velocity, const pstm_params *params);

int32_t pstm_cuda_migrate_tile_host(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                    const pstm_velocity_desc *velocity, const pstm_params *params) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    int32_t rc = migrate_host_impl(c, traces, output, velocity, params);
    // On failure, drain the stream so no queued copy outlives the caller's buffers.
    if (rc != PSTM_OK && c->stream) cudaStreamSynchronize(c->stream);
    return rc;
}

static int32_t migrate_host_impl(Ctx *c, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                 const pstm_velocity_desc *velocity, const pstm_params *params) {
    int32_t rc = validate(c, traces, output, velocity, params);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = c->stream;
    const int64_t N = traces->n_traces;
    const int nx = output->nx, ny = output->ny, nt = output->nt;
    const size_t npix = (size_t)nx * ny * nt;

    pstm_traces_desc dt = *traces;
    pstm_output_desc dout = *output;
    pstm_velocity_desc dv = *velocity;
    pstm_params dp = *params;
    const size_t eb = amp_elem_bytes(traces->amp_dtype);
    // amplitudes: packed to n_samples per row on the device
    if (N > 0) {
        // rows padded to a 16-byte pitch so the kernel can stage them with TMA bulk copies
        const size_t per16 = 16 / eb;
        const size_t pitch = ((size_t)traces->n_samples + per16 - 1) / per16 * per16;
        e = ensure(c->amps, (size_t)N * pitch * eb);
        if (e != cudaSuccess) return cuda_fail(c, e, "staging amplitudes");
        e = cudaMemcpy2DAsync(c->amps.ptr, pitch * eb, traces->amplitudes,
                              traces->amp_row_stride * eb, traces->n_samples * eb, (size_t)N,
                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(c, e, "copying amplitudes");
        dt.amplitudes = c->amps.ptr;
        dt.amp_row_stride = (int64_t)pitch;
    }
    const double *src_geo[7] = {traces->source_x, traces->source_y, traces->receiver_x, traces->receiver_y,
                                traces->midpoint_x, traces->midpoint_y, traces->weights};
    const double *dst_geo[7];
    for (int i = 0; i < 7; ++i) {
        e = stage(c->geo[i], N > 0 ? src_geo[i] : nullptr, (size_t)N, st, &dst_geo[i]);
        if (e != cudaSuccess) return cuda_fail(c, e, "copying geometry");
    }
    dt.source_x = dst_geo[0]; dt.source_y = dst_geo[1];
    dt.receiver_x = dst_geo[2]; dt.receiver_y = dst_geo[3];
    dt.midpoint_x = dst_geo[4]; dt.midpoint_y = dst_geo[5];
    dt.weights = dst_geo[6];

    if ((e = stage(c->xa, output->x_axis, (size_t)nx, st, &dout.x_axis)) != cudaSuccess ||
        (e = stage(c->ya, output->y_axis, (size_t)ny, st, &dout.y_axis)) != cudaSuccess ||
        (e = stage(c->xg, output->x_grid, (size_t)nx * ny, st, &dout.x_grid)) != cudaSuccess ||
        (e = stage(c->yg, output->y_grid, (size_t)nx * ny, st, &dout.y_grid)) != cudaSuccess ||
        (e = stage(c->ta, output->t_axis_ms, (size_t)nt, st, &dout.t_axis_ms)) != cudaSuccess)
        return cuda_fail(c, e, "copying output axes");
    const size_t nvel = velocity->is_3d ? npix : (size_t)nt;
    if ((e = stage(c->vel, velocity->vrms, nvel, st, &dv.vrms)) != cudaSuccess)
        return cuda_fail(c, e, "copying velocity");
    if (params->eta) {
        const size_t neta = params->eta_is_3d ? npix : (size_t)nt;
        if ((e = stage(c->eta, params->eta, neta, st, &dp.eta)) != cudaSuccess)
            return cuda_fail(c, e, "copying eta");
    }
    const size_t img_bytes = npix * (output->image_dtype == PSTM_IMAGE_F32 ? 4 : 8);
    if ((e = ensure(c->image, img_bytes)) != cudaSuccess) return cuda_fail(c, e, "staging image");
    if ((e = cudaMemcpyAsync(c->image.ptr, output->image, img_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(c, e, "copying image");
    dout.image = c->image.ptr;
    const size_t fold_bytes = (output->fold_is_3d ? npix : (size_t)nx * ny) * sizeof(int32_t);
    if (output->fold) {
        if ((e = ensure(c->fold, fold_bytes)) != cudaSuccess) return cuda_fail(c, e, "staging fold");
        if ((e = cudaMemcpyAsync(c->fold.ptr, output->fold, fold_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cuda_fail(c, e, "copying fold");
        dout.fold = reinterpret_cast<int32_t *>(c->fold.ptr);
    }
    rc = run_dev(c, &dt, &dout, &dv, &dp, st);
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(output->image, c->image.ptr, img_bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(c, e, "reading image back");
    if (output->fold &&
        (e = cudaMemcpyAsync(output->fold, c->fold.ptr, fold_bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(c, e, "reading fold back");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(c, e, "migrate_tile");
    return check_error_word(c);
}

int32_t pstm_cuda_synchronize(void *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (injected("sync")) return fail(c, PSTM_ERR_INJECTED, "injected fault: sync");
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "synchronize");
    return check_error_word(c);
}

const char *pstm_cuda_last_error(void *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    return c ? c->err.c_str() : g_create_err.c_str();
}

}  // extern "C"
