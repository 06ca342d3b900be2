// batch.cu -- the batched form: many bins (offset or OVT gathers) that share
// one output tile geometry, migrated by ONE persistent launch that is
// captured in a CUDA graph, plus the autotuner of its launch shape.
//
// The reference migrates its gather bins one after another, each bin a
// sequence of per-tile kernel calls (pstm/pipeline/executor.py:960-975).
// Here the bins of a tile are one launch: one CTA per SM takes items (bin,
// pillar block, time block) from a work counter; the bins are ordered by
// decreasing trace count, so the long items start first and bins of very
// different sizes still end together.
#include <cuda_runtime.h>
#include <algorithm>
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
using namespace pstm::ctx;

namespace {

constexpr int kMaxBins = 4096;

struct BatchPlan {
    KParams P;
    Launch L;
    int tt = 0, amp = 0;
    bool per_pillar = false, exact = false;
    int prec = PSTM_PREC_EXACT;   // pstm_precision
    int64_t n_p = 0;
    std::vector<BinWork> work;   // non-empty bins, most traces first
};

// Workload class of the tuned shapes.
std::string class_key(const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_velocity_desc *vel,
                      const pstm_params *prm) {
    char buf[192];
    const int per_pillar = (vel->is_3d || (prm->eta && prm->eta_is_3d)) ? 1 : 0;
    std::snprintf(buf, sizeof(buf), "tt%d amp%d pp%d prec%d nt%d ns%d aa%d sp%d ob%d img%d", prm->traveltime,
                  tr->amp_dtype, per_pillar, prm->precision, out->nt, tr->n_samples, prm->aa_enabled,
                  prm->apply_spreading, prm->apply_obliquity, out->image_dtype);
    return buf;
}

int32_t check_bins(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_bin_desc *bins,
                   int32_t n_bins) {
    char buf[160];
    if (n_bins < 0 || n_bins > kMaxBins) {
        std::snprintf(buf, sizeof(buf), "n_bins %d outside [0, %d]", n_bins, kMaxBins);
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, buf);
    }
    if (n_bins > 0 && !bins) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null bins");
    if (out->nx <= 0 || out->ny <= 0 || out->nt <= 0) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "empty output tile");
    const uint64_t npix = (uint64_t)out->nx * out->ny * out->nt;
    const uint64_t img_bytes = npix * (out->image_dtype == PSTM_IMAGE_F32 ? 4 : 8);
    const uint64_t fold_bytes = (out->fold_is_3d ? npix : (uint64_t)out->nx * out->ny) * 4;
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    for (int i = 0; i < n_bins; ++i) {
        const pstm_bin_desc &b = bins[i];
        if (b.trace_begin < 0 || b.n_traces < 0 || b.trace_begin > tr->n_traces - b.n_traces) {
            std::snprintf(buf, sizeof(buf), "bin %d: traces [%lld, +%lld) outside the %lld traces of the batch", i,
                          (long long)b.trace_begin, (long long)b.n_traces, (long long)tr->n_traces);
            return fail(c, PSTM_ERR_INVALID_ARGUMENT, buf);
        }
        if (!b.image) {
            std::snprintf(buf, sizeof(buf), "bin %d: null image", i);
            return fail(c, PSTM_ERR_INVALID_ARGUMENT, buf);
        }
        ranges.emplace_back((uint64_t)(uintptr_t)b.image, (uint64_t)(uintptr_t)b.image + img_bytes);
        if (b.fold) ranges.emplace_back((uint64_t)(uintptr_t)b.fold, (uint64_t)(uintptr_t)b.fold + fold_bytes);
    }
    std::sort(ranges.begin(), ranges.end());
    for (size_t i = 1; i < ranges.size(); ++i)
        if (ranges[i].first < ranges[i - 1].second)
            return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bins' images and folds must not overlap");
    return PSTM_OK;
}

// Validates the arguments, picks the launch shape (forced, tuned or default),
// makes sure every buffer exists and fills the plan.  Allocates; enqueues
// nothing.  bp.work is empty when there is nothing to migrate.
int32_t plan_batch(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_velocity_desc *vel,
                   const pstm_params *prm, const pstm_bin_desc *bins, int32_t n_bins, const Shape *force,
                   BatchPlan &bp) {
    int32_t rc = check_bins(c, tr, out, bins, n_bins);
    if (rc) return rc;
    bp.work.clear();
    if (n_bins == 0) return PSTM_OK;
    pstm_output_desc o = *out;
    o.image = bins[0].image;
    o.fold = nullptr;
    const char *msg = "";
    if ((rc = plan::check_args(tr, &o, vel, prm, msg)) != PSTM_OK) return fail(c, rc, msg);
    if (prm->interpolation != PSTM_INTERP_LINEAR)
        return fail(c, PSTM_ERR_UNSUPPORTED, "the batched form interpolates linearly");
    for (int i = 0; i < n_bins; ++i)
        if (bins[i].n_traces > 0)
            bp.work.push_back({bins[i].trace_begin, bins[i].n_traces, bins[i].image, bins[i].fold});
    if (bp.work.empty()) return PSTM_OK;
    std::stable_sort(bp.work.begin(), bp.work.end(),
                     [](const BinWork &a, const BinWork &b) { return a.n_traces > b.n_traces; });

    int R, PB, chunk = 0;
    if (force) {
        R = force->r;
        PB = force->pb;
        chunk = force->chunk;
    } else {
        plan::choose_shape(out->nt, c->force_r, c->force_pb, R, PB, tr->amp_dtype);
        auto it = c->tuned.find(class_key(tr, out, vel, prm));
        if (it != c->tuned.end() && !c->force_r && !c->force_pb) {
            R = it->second.r;
            PB = it->second.pb;
            chunk = it->second.chunk;
        }
    }
    if (R < 1 || R > 8 || PB < 1 || PB > kMaxPB) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "launch shape out of range");

    KParams &P = bp.P;
    P = plan::make_params(tr, &o, vel, prm, PB);
    bp.tt = prm->traveltime;
    bp.amp = tr->amp_dtype;
    bp.per_pillar = vel->is_3d || (prm->eta && prm->eta_is_3d);
    bp.exact = prm->precision == PSTM_PREC_EXACT;
    bp.prec = prm->precision;
    P.exact_units = bp.exact ? 1 : 0;
    P.curved_kind = (prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI) ? 1 : 0;
    bp.n_p = bp.per_pillar ? (int64_t)out->nx * out->ny : 1;
    const size_t n_tab = (size_t)bp.n_p * out->nt;
    cudaError_t e;
    if ((e = ensure(c->ttab, n_tab * sizeof(float4))) != cudaSuccess ||
        (e = ensure(c->btab, n_tab * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->ttime, (size_t)out->nt * 2 * sizeof(float4))) != cudaSuccess ||
        (e = ensure(c->ttimeA, (size_t)out->nt * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->ttimeV, (size_t)out->nt * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->errword, sizeof(int32_t))) != cudaSuccess ||
        (e = ensure(c->kparams, sizeof(KParams))) != cudaSuccess ||
        (e = ensure(c->packed_geo, (size_t)tr->n_traces * kGeoDoubles * sizeof(double))) != cudaSuccess ||
        (e = ensure(c->bins, bp.work.size() * sizeof(BinWork))) != cudaSuccess ||
        (e = ensure(c->counter, sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the batch buffers");
    P.ttab = reinterpret_cast<const float4 *>(c->ttab.ptr);
    P.btab = reinterpret_cast<const double *>(c->btab.ptr);
    P.ttime = reinterpret_cast<const float4 *>(c->ttime.ptr);
    P.ttimeA = reinterpret_cast<const double *>(c->ttimeA.ptr);
    P.ttimeV = reinterpret_cast<const double *>(c->ttimeV.ptr);
    P.geo = reinterpret_cast<const double *>(c->packed_geo.ptr);
    P.err = reinterpret_cast<int32_t *>(c->errword.ptr);
    size_t smem = 0;
    if (!plan::plan_staging(P, tr, prm, PB, R, c->smem_optin, smem, chunk))
        return fail(c, PSTM_ERR_UNSUPPORTED, "trace rows too long to stage in shared memory");

    // bins much larger than L2 are split into trace segments (consecutive in the
    // work list, so the resident CTAs share each segment in L2); split bins add
    // into their outputs atomically
    const int64_t row_bytes = (int64_t)P.pitch * P.elem;
    if (c->segment_bytes > 0) {
        int64_t S = c->segment_bytes / row_bytes;
        S = S < 16 * (int64_t)P.chunk ? 16 * (int64_t)P.chunk : S / P.chunk * P.chunk;
        std::vector<BinWork> split;
        for (const BinWork &w : bp.work) {
            if (w.n_traces * row_bytes <= 2 * c->segment_bytes) {
                split.push_back(w);
                continue;
            }
            for (int64_t b = 0; b < w.n_traces; b += S)
                split.push_back({w.trace0 + b, (w.n_traces - b) < S ? (w.n_traces - b) : S, w.image, w.fold});
            P.atomic_flush = 1;
        }
        if (split.size() > (size_t)(64 * kMaxBins))
            return fail(c, PSTM_ERR_UNSUPPORTED, "too many trace segments in one batch");
        bp.work.swap(split);
        if ((e = ensure(c->bins, bp.work.size() * sizeof(BinWork))) != cudaSuccess)
            return cuda_fail(c, e, "allocating the batch work list");
    }

    bp.L = Launch();
    bp.L.smem = smem;
    bp.L.bins = reinterpret_cast<const BinWork *>(c->bins.ptr);
    bp.L.n_bins = (int)bp.work.size();
    bp.L.counter = reinterpret_cast<unsigned long long *>(c->counter.ptr);
    // resolve the CTA count and the shared-memory opt-in now: nothing but
    // stream work may happen while the launch sequence is captured
    unsigned ctas = 0;
    bp.L.configure_only = true;
    bp.L.ctas_out = &ctas;
    e = launch_kind(bp.tt, P, reinterpret_cast<const KParams *>(c->kparams.ptr), bp.amp, bp.per_pillar, bp.prec,
                    bp.L);
    if (e != cudaSuccess) return cuda_fail(c, e, "configuring the persistent kernel");
    bp.L.configure_only = false;
    bp.L.ctas_out = nullptr;
    bp.L.grid = dim3(ctas);
    return PSTM_OK;
}

// Enqueues the whole batch on `st`: error word and work counter cleared,
// tables, packed geometry, parameter block, work list, the persistent launch.
// Allocates nothing, so it can be captured.
int32_t enqueue_batch(Ctx *c, BatchPlan &bp, cudaStream_t st) {
    KParams &P = bp.P;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->errword.ptr, 0, sizeof(int32_t), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->counter.ptr, 0, sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(c, e, "clearing the error word and work counter");
    const int64_t n_tab = bp.n_p * P.nt;
    int blocks = (int)std::min<int64_t>((n_tab + 255) / 256, 148 * 32);
    prep_time_table<<<blocks, 256, 0, st>>>(P, bp.n_p, reinterpret_cast<float4 *>(c->ttab.ptr),
                                            reinterpret_cast<double *>(c->btab.ptr),
                                            reinterpret_cast<float4 *>(c->ttime.ptr),
                                            reinterpret_cast<double *>(c->ttimeA.ptr),
                                            reinterpret_cast<double *>(c->ttimeV.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "prep_time_table launch");
    blocks = (int)std::min<int64_t>((P.n_traces + 255) / 256, 148 * 32);
    if (blocks > 0) {
        pack_geometry<<<blocks, 256, 0, st>>>(P, reinterpret_cast<double *>(c->packed_geo.ptr));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "pack_geometry launch");
    }
    store_params<<<1, 32, 0, st>>>(P, reinterpret_cast<KParams *>(c->kparams.ptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "store_params launch");
    for (size_t i = 0; i < bp.work.size(); i += kBinsPerStore) {
        BinStore b;
        std::memset(&b, 0, sizeof(b));
        b.first = (int32_t)i;
        b.count = (int32_t)std::min<size_t>(kBinsPerStore, bp.work.size() - i);
        std::copy(bp.work.begin() + i, bp.work.begin() + i + b.count, b.w);
        store_bins<<<1, kBinsPerStore, 0, st>>>(b, reinterpret_cast<BinWork *>(c->bins.ptr));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "store_bins launch");
    }
    bp.L.stream = st;
    e = launch_kind(bp.tt, P, reinterpret_cast<const KParams *>(c->kparams.ptr), bp.amp, bp.per_pillar, bp.prec,
                    bp.L);
    if (e != cudaSuccess) return cuda_fail(c, e, "persistent migrate kernel launch");
    return PSTM_OK;
}

// The arguments a captured graph depends on: every launch parameter, the work
// list and the launch shape (the buffers of the context are inside P).
std::vector<unsigned char> graph_key(const BatchPlan &bp) {
    std::vector<unsigned char> k;
    auto put = [&](const void *p, size_t n) {
        const unsigned char *b = static_cast<const unsigned char *>(p);
        k.insert(k.end(), b, b + n);
    };
    put(&bp.P, sizeof(KParams));
    if (!bp.work.empty()) put(bp.work.data(), bp.work.size() * sizeof(BinWork));
    const int64_t extra[8] = {bp.tt, bp.amp, bp.per_pillar, bp.prec, (int64_t)bp.L.grid.x, (int64_t)bp.L.smem,
                              (int64_t)(uintptr_t)bp.L.bins, (int64_t)(uintptr_t)bp.L.counter};
    put(extra, sizeof(extra));
    return k;
}

bool graphs_enabled() {
    const char *v = std::getenv("PSTM_CUDA_GRAPH");   // "0": enqueue the batch directly
    return !(v && std::strcmp(v, "0") == 0);
}

int32_t run_graph(Ctx *c, BatchPlan &bp, cudaStream_t st) {
    std::vector<unsigned char> key = graph_key(bp);
    cudaError_t e;
    if (!(c->graph && key == c->graph_key)) {
        c->graph_key.clear();
        if ((e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(c, e, "cudaStreamBeginCapture");
        const int32_t rc = enqueue_batch(c, bp, c->stream);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(c->stream, &g);
        if (rc != PSTM_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        if (c->graph) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(c->graph, g, &info) != cudaSuccess) {
                (void)cudaGetLastError();
                cudaGraphExecDestroy(c->graph);
                c->graph = nullptr;
            }
        }
        if (!c->graph && (e = cudaGraphInstantiate(&c->graph, g, 0)) != cudaSuccess) {
            c->graph = nullptr;
            cudaGraphDestroy(g);
            return cuda_fail(c, e, "cudaGraphInstantiate");
        }
        cudaGraphDestroy(g);
        c->graph_key = std::move(key);
    }
    if ((e = cudaGraphLaunch(c->graph, st)) != cudaSuccess) return cuda_fail(c, e, "cudaGraphLaunch");
    return PSTM_OK;
}

}  // namespace

namespace pstm {
namespace ctx {
void release_batch(Ctx *c) {
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_key.clear();
    release(c->bins);
    release(c->counter);
    release(c->tune_image);
    release(c->tune_fold);
    release(c->probe);
    release(c->seg_bins);
    release(c->seg_counter);
}
}  // namespace ctx
}  // namespace pstm

extern "C" {

int32_t pstm_cuda_migrate_bins_dev(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                   const pstm_velocity_desc *velocity, const pstm_params *params,
                                   const pstm_bin_desc *bins, int32_t n_bins, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (!traces || !output || !velocity || !params) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null descriptor");
    if (injected("migrate")) return fail(c, PSTM_ERR_INJECTED, "injected fault: migrate");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    BatchPlan bp;
    int32_t rc = plan_batch(c, traces, output, velocity, params, bins, n_bins, nullptr, bp);
    if (rc || bp.work.empty()) return rc;
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    return graphs_enabled() ? run_graph(c, bp, st) : enqueue_batch(c, bp, st);
}

int32_t pstm_cuda_autotune_bins(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                const pstm_velocity_desc *velocity, const pstm_params *params,
                                const pstm_bin_desc *bins, int32_t n_bins, int64_t pairs_per_candidate,
                                pstm_tune_result *result) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (!traces || !output || !velocity || !params || !result)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null descriptor");
    std::memset(result, 0, sizeof(*result));
    int32_t rc = check_bins(c, traces, output, bins, n_bins);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    if (pairs_per_candidate <= 0) pairs_per_candidate = int64_t(1) << 36;

    // the sample: the largest bins (at most 8), a band of whole output rows of
    // about 1024 pillars, each bin clipped to its first traces
    std::vector<pstm_bin_desc> big;
    for (int i = 0; i < n_bins; ++i)
        if (bins[i].n_traces > 0) big.push_back(bins[i]);
    if (big.empty()) return PSTM_OK;
    std::stable_sort(big.begin(), big.end(),
                     [](const pstm_bin_desc &a, const pstm_bin_desc &b) { return a.n_traces > b.n_traces; });
    if (big.size() > 8) big.resize(8);
    pstm_output_desc o = *output;
    o.nx = std::max(1, std::min(output->nx, (1024 + output->ny - 1) / output->ny));
    const int64_t pillars = (int64_t)o.nx * o.ny;
    const int64_t cap = std::max<int64_t>(1024, pairs_per_candidate / (pillars * o.nt * (int64_t)big.size()));
    const size_t npix = (size_t)pillars * o.nt;
    const size_t img_bytes = (npix * (o.image_dtype == PSTM_IMAGE_F32 ? 4 : 8) + 255) / 256 * 256;
    const size_t fold_bytes = ((o.fold_is_3d ? npix : (size_t)pillars) * 4 + 255) / 256 * 256;
    if ((e = ensure(c->tune_image, big.size() * img_bytes)) != cudaSuccess ||
        (e = ensure(c->tune_fold, big.size() * fold_bytes)) != cudaSuccess)
        return cuda_fail(c, e, "allocating the tuning outputs");
    if ((e = cudaMemsetAsync(c->tune_image.ptr, 0, big.size() * img_bytes, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->tune_fold.ptr, 0, big.size() * fold_bytes, c->stream)) != cudaSuccess)
        return cuda_fail(c, e, "clearing the tuning outputs");
    for (size_t i = 0; i < big.size(); ++i) {
        big[i].n_traces = std::min(big[i].n_traces, cap);
        big[i].image = static_cast<unsigned char *>(c->tune_image.ptr) + i * img_bytes;
        big[i].fold = reinterpret_cast<int32_t *>(static_cast<unsigned char *>(c->tune_fold.ptr) + i * fold_bytes);
    }

    // candidates: the default shape first, then pillars per CTA x times per
    // lane x panel depth
    Shape def;
    plan::choose_shape(o.nt, 0, 0, def.r, def.pb, traces->amp_dtype);
    std::vector<Shape> cand{def};
    std::vector<int> rs{def.r};
    if (def.r > 1) rs.push_back((def.r + 1) / 2);
    for (int r : rs)
        for (int pb : {2, 4, 8})
            for (int ch : {0, 16, 8}) {
                Shape s{pb, r, ch};
                if (!(s.pb == def.pb && s.r == def.r && s.chunk == 0)) cand.push_back(s);
            }

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if ((e = cudaEventCreate(&ev0)) != cudaSuccess || (e = cudaEventCreate(&ev1)) != cudaSuccess) {
        if (ev0) cudaEventDestroy(ev0);
        return cuda_fail(c, e, "cudaEventCreate");
    }
    Shape best = def;
    float best_ms = -1.f, default_ms = -1.f;
    int timed = 0;
    for (const Shape &s : cand) {
        BatchPlan bp;
        rc = plan_batch(c, traces, &o, velocity, params, big.data(), (int32_t)big.size(), &s, bp);
        if (rc == PSTM_ERR_UNSUPPORTED) {   // does not fit in shared memory
            rc = PSTM_OK;
            continue;
        }
        if (rc) break;
        if (s.chunk && bp.P.chunk != s.chunk) continue;   // deeper than fits: the same as chunk 0
        float ms = 1e30f;
        for (int rep = 0; rep < 2 && rc == PSTM_OK; ++rep) {   // the first run warms up
            if ((e = cudaEventRecord(ev0, c->stream)) != cudaSuccess) {
                rc = cuda_fail(c, e, "cudaEventRecord");
                break;
            }
            if ((rc = enqueue_batch(c, bp, c->stream)) != PSTM_OK) break;
            if ((e = cudaEventRecord(ev1, c->stream)) != cudaSuccess ||
                (e = cudaEventSynchronize(ev1)) != cudaSuccess) {
                rc = cuda_fail(c, e, "timing a candidate");
                break;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, ev0, ev1);
            if (rep > 0) ms = t;
        }
        if (rc) break;
        int32_t w = 0;
        if ((e = cudaMemcpy(&w, c->errword.ptr, sizeof(w), cudaMemcpyDeviceToHost)) != cudaSuccess) {
            rc = cuda_fail(c, e, "reading the error word");
            break;
        }
        if (w & KERR_WAIT_TIMEOUT) {
            rc = fail(c, PSTM_ERR_TIMEOUT, "a bounded wait gave up while tuning");
            break;
        }
        ++timed;
        const Shape eff{s.pb, s.r, s.chunk ? bp.P.chunk : 0};
        if (timed == 1) default_ms = ms;
        if (best_ms < 0.f || ms < best_ms) {
            best_ms = ms;
            best = eff;
        }
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (rc) return rc;
    c->tuned[class_key(traces, output, velocity, params)] = best;
    result->pillars_per_cta = best.pb;
    result->times_per_lane = best.r;
    result->traces_per_chunk = best.chunk;
    result->n_candidates = timed;
    result->best_ms = best_ms;
    result->default_ms = default_ms;
    return PSTM_OK;
}

}  // extern "C"
