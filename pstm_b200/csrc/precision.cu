// precision.cu -- the precision form's trace format: FP32 traces stored as
// FP16 with one power-of-two scale per trace.
//
// FP16 keeps 11 significant bits (BF16 keeps 8), so a noise-dominated panel
// stored in FP16 stays within the 1e-3 image error of the FP32 panel where
// BF16 does not; its narrow exponent range (normal numbers from 2^-14 to
// 65504) is what the per-trace scale is for.  Each trace is multiplied by
// 2^e, e chosen so that its largest |amplitude| lands in [2^13, 2^14) -- exact
// in FP32, and with headroom to FP16's largest finite value -- and its weight
// is multiplied by 2^-e, also exact.  The migration kernel already multiplies
// every contribution by the trace weight, so the scale costs nothing per pair:
// amplitude * weight is the FP32 trace's, up to the FP16 rounding.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cmath>
#include <string>

#include "pstm_cuda.h"
#include "ctx.h"

using namespace pstm;
using namespace pstm::ctx;

namespace {

constexpr int kWarpsPerCta = 8;

// One warp per trace: the largest |amplitude|, then the scaled FP16 row and
// the trace weight divided by the scale.
__global__ void __launch_bounds__(32 * kWarpsPerCta)
traces_to_f16_kernel(const float *__restrict__ src, int64_t n, int ns, int64_t src_stride, __half *__restrict__ dst,
                     int64_t dst_stride, const double *__restrict__ w_in, double *__restrict__ w_out) {
    const int lane = threadIdx.x & 31;
    const int64_t tr = (int64_t)blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (tr >= n) return;
    const float *row = src + tr * src_stride;
    float m = 0.f;
    for (int i = lane; i < ns; i += 32) m = fmaxf(m, fabsf(row[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    if (m > 0.f && isfinite(m)) {
        int ex;
        frexpf(m, &ex);   // m = f 2^ex, f in [0.5, 1)
        e = 14 - ex;      // m 2^e in [2^13, 2^14)
    }
    const float scale = ldexpf(1.f, e);
    __half *out = dst + tr * dst_stride;
    for (int i = lane; i < ns; i += 32) out[i] = __float2half_rn(row[i] * scale);
    if (lane == 0) w_out[tr] = (w_in ? w_in[tr] : 1.0) * ldexp(1.0, -e);
}

}  // namespace

extern "C" int32_t pstm_cuda_traces_to_f16(void *ctx, const float *src, int64_t n_traces, int32_t n_samples,
                                           int64_t src_stride, void *dst, int64_t dst_stride,
                                           const double *weights, double *weights_out, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (n_traces < 0 || n_samples < 1 || src_stride < n_samples || dst_stride < n_samples)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "traces_to_f16: bad sizes or strides");
    if (n_traces == 0) return PSTM_OK;
    if (!src || !dst || !weights_out) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "traces_to_f16: null pointer");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    const int64_t blocks = (n_traces + kWarpsPerCta - 1) / kWarpsPerCta;
    if (blocks > 0x7fffffff) return fail(c, PSTM_ERR_UNSUPPORTED, "traces_to_f16: too many traces for one launch");
    traces_to_f16_kernel<<<(unsigned)blocks, 32 * kWarpsPerCta, 0, st>>>(
        src, n_traces, n_samples, src_stride, reinterpret_cast<__half *>(dst), dst_stride, weights, weights_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "traces_to_f16 launch");
    return PSTM_OK;
}
