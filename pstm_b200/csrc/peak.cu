// peak.cu -- measured issue ceiling of the special-function unit (MUFU).
//
// The gather kernel's roofline is stated in MUFU operations per sample-trace
// pair (two square roots of the DSR legs, the reciprocal of T, the AA
// reciprocal).  Its denominator is measured here on the device the kernel runs
// on rather than derived from a nominal per-SM rate: every thread of a
// full-occupancy grid runs kChains independent dependency chains of
// alternating sqrt.approx.ftz.f32 and rcp.approx.ftz.f32 (one MUFU operation
// each), so the MUFU pipe, not latency, bounds the kernel.
#include <cuda_runtime.h>
#include <string>

#include "pstm_cuda.h"

namespace pstm {
void set_context_free_error(const std::string &msg);
}  // namespace pstm

namespace {

constexpr int kChains = 8;
constexpr int kThreadsPerCta = 512;

__global__ void __launch_bounds__(kThreadsPerCta) mufu_chains(int iters, float seed, float *sink) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = seed + 0.001f * (float)(c + (threadIdx.x & 7));
    for (int i = 0; i < iters; ++i) {
        float y[kChains];   // all chains' square roots, then all reciprocals: independent neighbours
#pragma unroll
        for (int c = 0; c < kChains; ++c) asm volatile("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y[c]) : "f"(x[c]));
#pragma unroll
        for (int c = 0; c < kChains; ++c) asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(x[c]) : "f"(y[c]));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.f) sink[threadIdx.x] = s;   // keeps the chains alive; never true for these seeds
}

int32_t fail(int32_t code, const std::string &m) {
    pstm::set_context_free_error(m);
    return code;
}

}  // namespace

extern "C" int32_t pstm_cuda_measure_sfu_peak(int32_t device, double *ops_per_second) {
    if (!ops_per_second) return fail(PSTM_ERR_INVALID_ARGUMENT, "ops_per_second is null");
    *ops_per_second = 0.0;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(PSTM_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    int sms = 0, per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mufu_chains, kThreadsPerCta, 0)) != cudaSuccess)
        return fail(PSTM_ERR_CUDA, std::string("occupancy query: ") + cudaGetErrorString(e));
    if (per_sm < 1) per_sm = 1;
    const int blocks = sms * per_sm;
    const int iters = 8192;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float *sink = nullptr;
    float best = 1e30f;
    int32_t rc = PSTM_OK;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ev0)) != cudaSuccess || (e = cudaEventCreate(&ev1)) != cudaSuccess ||
        (e = cudaMalloc(&sink, kThreadsPerCta * sizeof(float))) != cudaSuccess) {
        rc = fail(PSTM_ERR_CUDA, std::string("setting up the SFU measurement: ") + cudaGetErrorString(e));
    }
    for (int rep = 0; rep < 4 && rc == PSTM_OK; ++rep) {   // the first run warms up
        cudaEventRecord(ev0, st);
        mufu_chains<<<blocks, kThreadsPerCta, 0, st>>>(iters, 1.5f + 0.25f * rep, sink);
        cudaEventRecord(ev1, st);
        if ((e = cudaEventSynchronize(ev1)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) {
            rc = fail(PSTM_ERR_CUDA, std::string("SFU measurement kernel: ") + cudaGetErrorString(e));
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        if (rep > 0 && ms < best) best = ms;
    }
    if (rc == PSTM_OK) {
        const double ops = (double)blocks * kThreadsPerCta * (double)iters * kChains * 2.0;
        *ops_per_second = ops / (best * 1e-3);
    }
    if (sink) cudaFree(sink);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
    return rc;
}
