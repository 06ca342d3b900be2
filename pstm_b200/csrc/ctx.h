// ctx.h -- the context behind a pstm_cuda handle: its stream, the device
// buffers it reuses from call to call, and the state of the batched form
// (cached CUDA graph, tuned launch shapes).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "pstm_cuda.h"
#include "launch.h"

namespace pstm {
namespace ctx {

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

// Launch shape of the gather kernels: pillars per CTA, output times per lane,
// traces per staged chunk (0: as many as shared memory holds).
struct Shape {
    int pb = 0, r = 0, chunk = 0;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    DevBuf ttab, btab, ttime, ttimeA, ttimeV, kparams, errword, packed_geo;
    // staging for the host-pointer path
    DevBuf amps, geo[7], xa, ya, xg, yg, ta, vel, eta, image, fold;
    int force_r = 0;      // PSTM_CUDA_R override of the output times per lane
    int force_pb = 0;     // PSTM_CUDA_PB override of the pillars per CTA
    int smem_optin = 0;   // max dynamic shared memory per block
    // batched form
    DevBuf bins, counter, tune_image, tune_fold;
    DevBuf probe;                           // learned form: per-probe residuals
    DevBuf seg_bins, seg_counter;           // per-tile launches split into trace segments
    DevBuf scatter_ends;                    // scatter schedule: prefix counts of the segments' items
    int64_t segment_bytes = 24ll << 20;     // trace-panel bytes per segment (0: never split)
    std::vector<unsigned char> graph_key;   // arguments the cached graph was captured with
    cudaGraphExec_t graph = nullptr;
    std::map<std::string, Shape> tuned;     // autotuned shapes by workload class
};

// A per-tile launch prepared by prepare_tile: tables, packed geometry and the
// device parameter block are enqueued; the migration launch is not.
struct TilePlan {
    KParams P;
    const KParams *Pg = nullptr;
    Launch L;
    int tt = 0, amp = 0;
    bool per_pillar = false, exact = false;
    int prec = PSTM_PREC_EXACT;   // pstm_precision of the launch
    int64_t n_p = 0;
    bool empty = true;   // no traces: nothing to launch
};

int32_t prepare_tile(Ctx *c, const pstm_traces_desc *tr, const pstm_output_desc *out, const pstm_velocity_desc *vel,
                     const pstm_params *prm, cudaStream_t st, TilePlan &tp);
int32_t launch_tile(Ctx *c, const TilePlan &tp);
int32_t launch_interp(Ctx *c, const TilePlan &tp, int method, const pstm_output_desc *out);   // interp.cu
int32_t check_error_word(Ctx *c);   // after the stream has drained

int32_t fail(Ctx *c, int32_t code, const std::string &msg);
int32_t cuda_fail(Ctx *c, cudaError_t e, const char *what);
bool injected(const char *site);
cudaError_t ensure(DevBuf &b, size_t bytes);
void release(DevBuf &b);
void release_batch(Ctx *c);   // batch.cu

}  // namespace ctx
}  // namespace pstm
