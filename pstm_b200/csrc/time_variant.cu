// time_variant.cu -- linear interpolation of image rows from one time axis to
// another, with np.interp's end rule (the edge value outside the source
// axis).  The time-variant form uses it to bring an image computed at the
// windows' sample times back to the uniform axis (the reference's
// resample_to_uniform, pstm/algorithm/time_variant.py:354-397) and to put
// velocity and eta onto the window times.
#include <cuda_runtime.h>

#include "pstm_cuda.h"
#include "ctx.h"

using namespace pstm::ctx;

namespace {

// Largest k with xs[k] <= x (xs ascending, n >= 1; x inside [xs[0], xs[n-1]]).
__device__ inline int bracket(const double *xs, int n, double x) {
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xs[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <typename T>
__global__ void interp_rows_kernel(const T *__restrict__ src, int64_t n_rows, int n_src, const double *__restrict__ xs,
                                   int n_dst, const double *__restrict__ xd, T *__restrict__ dst) {
    const int64_t total = n_rows * (int64_t)n_dst;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / n_dst;
        const int j = (int)(i - r * n_dst);
        const T *row = src + r * n_src;
        const double x = xd[j];
        double v;
        if (x <= xs[0]) v = (double)row[0];
        else if (x >= xs[n_src - 1]) v = (double)row[n_src - 1];
        else {
            const int k = bracket(xs, n_src, x);
            const double f = (x - xs[k]) / (xs[k + 1] - xs[k]);
            v = (double)row[k] + f * ((double)row[k + 1] - (double)row[k]);
        }
        dst[i] = (T)v;
    }
}

}  // namespace

extern "C" int32_t pstm_cuda_interp_rows(void *ctx, int32_t dtype, const void *src, int64_t n_rows, int32_t n_src,
                                         const double *src_times, int32_t n_dst, const double *dst_times, void *dst,
                                         void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (n_rows < 0 || n_src < 1 || n_dst < 0 || (dtype != PSTM_IMAGE_F64 && dtype != PSTM_IMAGE_F32))
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bad interpolation sizes or dtype");
    if (n_rows == 0 || n_dst == 0) return PSTM_OK;
    if (!src || !src_times || !dst_times || !dst) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null interpolation array");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    int64_t blocks = (n_rows * (int64_t)n_dst + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (dtype == PSTM_IMAGE_F64)
        interp_rows_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const double *>(src), n_rows, n_src,
                                                                     src_times, n_dst, dst_times,
                                                                     static_cast<double *>(dst));
    else
        interp_rows_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(static_cast<const float *>(src), n_rows, n_src,
                                                                    src_times, n_dst, dst_times,
                                                                    static_cast<float *>(dst));
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "interpolation launch");
    return PSTM_OK;
}
