// noalloc.cu -- pstm_cuda_migrate_tile_noalloc: the migration of one tile
// without any device-memory allocation.
//
// Some callers cannot allocate device memory while they run: a host
// application whose memory manager reserves the whole GPU up front and owns
// every byte of it, or a long-running job that must not fail on an allocation
// (or stall the device: cudaMalloc synchronizes it) once it has started
// processing tiles.  For them this entry point keeps every scratch buffer the
// kernel needs -- the per-time tables, the packed trace geometry, the launch
// parameters and the error word -- in one fixed array of this module's device
// memory.  The caller passes its inputs and outputs as device pointers, as to
// pstm_cuda_migrate_tile_dev.
//
// The array is 16 MiB and every device that loads this library holds it until
// the process exits.  Its size bounds one call (see the limits below); larger
// trace sets can be split over several calls, since the image and fold are
// accumulated with "+=".  All calls share the array and it keeps the last
// call's contents, so calls whose work overlaps on the GPU (different streams,
// different host threads) race and must be serialised by the caller.
//
// The kernel reports device-side failures (a bounded wait for a trace-row copy
// that gave up) in an error word inside the array; pstm_cuda_noalloc_status
// reads it back once the caller's stream has drained.
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include <string>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "plan.h"

namespace pstm {
void set_context_free_error(const std::string &msg);
}  // namespace pstm

using namespace pstm;

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;   // the whole array
constexpr int64_t kMaxTraces = 131072;               // packed geometry, 64 B per trace
constexpr int64_t kMaxTable = 262144;                // (pillar | 0, time) entries, 24 B each
constexpr int kMaxTimes = 8192;                      // output times, 40 B each

constexpr size_t kOffParams = 0;                                  // KParams
constexpr size_t kOffErr = 2048;                                  // error word
constexpr size_t kOffTime = 4096;                                 // 2 x float4 per time
constexpr size_t kOffTimeA = kOffTime + size_t(kMaxTimes) * 32;   // double per time
constexpr size_t kOffTab = kOffTimeA + size_t(kMaxTimes) * 8;     // float4 per entry
constexpr size_t kOffBtab = kOffTab + size_t(kMaxTable) * 16;     // double per entry
constexpr size_t kOffGeo = kOffBtab + size_t(kMaxTable) * 8;      // 8 doubles per trace
constexpr size_t kOffTimeV = kOffGeo + size_t(kMaxTraces) * kGeoDoubles * 8;   // double per time
static_assert(sizeof(KParams) <= kOffErr && sizeof(KParams) % 4 == 0, "launch parameters overlap the error word");
static_assert(kOffTimeV + size_t(kMaxTimes) * 8 <= kScratchBytes, "scratch layout overflows");
static_assert(kOffTab % 256 == 0 && kOffGeo % 256 == 0 && kOffTimeV % 256 == 0,
              "scratch regions must stay 256-byte aligned");

// The scratch array.  Host code must not use the symbol as a pointer: it is a
// host-side stand-in.  Its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_dev[kMaxDevices] = {};   // device address of g_scratch, per device
int g_smem_optin[kMaxDevices] = {};

int32_t fail(int32_t code, const std::string &msg) {
    set_context_free_error(msg);
    return code;
}

int32_t cuda_fail(cudaError_t e, const char *what) {
    return fail(e == cudaErrorMemoryAllocation ? PSTM_ERR_OUT_OF_MEMORY : PSTM_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Once per device, with that device current: the scratch array's device
// address and the shared-memory limit.
int32_t setup(int dev, unsigned char **scratch, int *optin) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_dev[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        int smem = 0;
        e = cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        g_smem_optin[dev] = smem;
        g_scratch_dev[dev] = static_cast<unsigned char *>(ptr);
    }
    *scratch = g_scratch_dev[dev];
    *optin = g_smem_optin[dev];
    return PSTM_OK;
}

}  // namespace

extern "C" int32_t pstm_cuda_migrate_tile_noalloc(const pstm_traces_desc *tr, const pstm_output_desc *out,
                                                  const pstm_velocity_desc *vel, const pstm_params *prm,
                                                  void *stream) {
    const char *msg = "";
    int32_t rc = plan::check_args(tr, out, vel, prm, msg);
    if (rc) return fail(rc, msg);
    if (prm->interpolation != PSTM_INTERP_LINEAR)
        return fail(PSTM_ERR_UNSUPPORTED, "the allocation-free entry point interpolates linearly");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(PSTM_ERR_UNSUPPORTED, "device index beyond the supported range");

    // size limits of the fixed scratch array
    const bool per_pillar = vel->is_3d || (prm->eta && prm->eta_is_3d);
    const int64_t n_p = per_pillar ? (int64_t)out->nx * out->ny : 1;
    char buf[256];
    if (tr->n_traces > kMaxTraces) {
        std::snprintf(buf, sizeof(buf),
                      "n_traces %lld exceeds the %lld traces one allocation-free call holds; split the traces "
                      "over several calls (image and fold accumulate) or use pstm_cuda_migrate_tile_dev",
                      (long long)tr->n_traces, (long long)kMaxTraces);
        return fail(PSTM_ERR_INVALID_ARGUMENT, buf);
    }
    if (out->nt > kMaxTimes || n_p * out->nt > kMaxTable) {
        std::snprintf(buf, sizeof(buf),
                      "tile tables of %lld entries (nt %d) exceed the allocation-free limits (%lld entries, "
                      "nt <= %d); use smaller tiles or pstm_cuda_migrate_tile_dev",
                      (long long)(n_p * out->nt), out->nt, (long long)kMaxTable, kMaxTimes);
        return fail(PSTM_ERR_INVALID_ARGUMENT, buf);
    }

    unsigned char *scratch = nullptr;
    int optin = 0;
    if ((rc = setup(dev, &scratch, &optin)) != PSTM_OK) return rc;
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : cudaStreamLegacy;

    int R, PB;
    plan::choose_shape(out->nt, 0, 0, R, PB, tr->amp_dtype);
    KParams P = plan::make_params(tr, out, vel, prm, PB);
    if (tr->n_traces == 0) return PSTM_OK;   // image += 0, fold += 0
    const bool exact = prm->precision == PSTM_PREC_EXACT;
    P.exact_units = exact ? 1 : 0;
    P.curved_kind = (prm->traveltime == PSTM_TT_CURVED || prm->traveltime == PSTM_TT_CURVED_VTI) ? 1 : 0;
    P.ttime = reinterpret_cast<const float4 *>(scratch + kOffTime);
    P.ttimeA = reinterpret_cast<const double *>(scratch + kOffTimeA);
    P.ttimeV = reinterpret_cast<const double *>(scratch + kOffTimeV);
    P.ttab = reinterpret_cast<const float4 *>(scratch + kOffTab);
    P.btab = reinterpret_cast<const double *>(scratch + kOffBtab);
    P.geo = reinterpret_cast<const double *>(scratch + kOffGeo);
    P.err = reinterpret_cast<int32_t *>(scratch + kOffErr);
    size_t smem = 0;
    if (!plan::plan_staging(P, tr, prm, PB, R, optin, smem))
        return fail(PSTM_ERR_UNSUPPORTED, "trace rows too long to stage in shared memory");

    // the error word is the only scratch that must start at zero; the tables,
    // the packed geometry and the parameter block are rewritten below
    if ((e = cudaMemsetAsync(P.err, 0, sizeof(int32_t), st)) != cudaSuccess)
        return cuda_fail(e, "clearing the error word");
    const int64_t n_tab = n_p * out->nt;
    int blocks = (int)((n_tab + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    prep_time_table<<<blocks, 256, 0, st>>>(P, n_p, reinterpret_cast<float4 *>(scratch + kOffTab),
                                            reinterpret_cast<double *>(scratch + kOffBtab),
                                            reinterpret_cast<float4 *>(scratch + kOffTime),
                                            reinterpret_cast<double *>(scratch + kOffTimeA),
                                            reinterpret_cast<double *>(scratch + kOffTimeV));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "prep_time_table launch");
    blocks = (int)((tr->n_traces + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    pack_geometry<<<blocks, 256, 0, st>>>(P, reinterpret_cast<double *>(scratch + kOffGeo));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "pack_geometry launch");
    // the launch parameters for the kernel's rare FP64 paths: written by a
    // kernel rather than copied from host memory
    store_params<<<1, 32, 0, st>>>(P, reinterpret_cast<KParams *>(scratch + kOffParams));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "store_params launch");
    const KParams *Pg = reinterpret_cast<const KParams *>(scratch + kOffParams);

    const int n_pblk_x = (out->nx + P.px - 1) / P.px;
    const int64_t nblk_p = (int64_t)n_pblk_x * P.n_pblk_y;
    const int tb = kThreads * R;
    const int nblk_t = (out->nt + tb - 1) / tb;
    if (nblk_p > 0x7fffffff || nblk_t > 65535) return fail(PSTM_ERR_UNSUPPORTED, "tile too large for one launch");
    Launch L;
    L.grid = dim3((unsigned)nblk_p, (unsigned)nblk_t);
    L.smem = smem;
    L.stream = st;
    e = launch_kind(prm->traveltime, P, Pg, tr->amp_dtype, per_pillar, prm->precision, L);
    if (e != cudaSuccess) return cuda_fail(e, "migrate kernel launch");
    return PSTM_OK;
}

// Status of the last allocation-free call on the current device: waits for
// `stream`, then reads the kernel's error word from the scratch array (a copy
// from the array's symbol into a host int: nothing is allocated).
extern "C" int32_t pstm_cuda_noalloc_status(void *stream) {
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "waiting for the allocation-free call");
    int32_t w = 0;
    e = cudaMemcpyFromSymbol(&w, g_scratch, sizeof(w), kOffErr, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "reading the allocation-free error word");
    if (w & KERR_WAIT_TIMEOUT)
        return fail(PSTM_ERR_TIMEOUT,
                    "a bounded wait for a trace-row copy gave up in the last allocation-free call; its image "
                    "and fold may hold partial sums and must be discarded");
    return PSTM_OK;
}
