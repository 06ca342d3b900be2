// mlp.cuh -- the traveltime surrogate network and its warp-level evaluation.
//
// Network: 7 inputs -> 64 -> 64 -> 64 -> 1, SiLU after the three hidden
// layers.  Weights are kept in FP32 (the optimiser's master copy) and staged
// as BF16 in shared memory; every matrix product runs on the tensor cores as
// mma.sync m16n8k16 (BF16 x BF16 -> FP32), the output layer (64 -> 1) is an
// FP32 dot product.  Inputs are normalised, x_n = (x - shift) * scale.
//
// A warp evaluates 16 samples per m-tile.  Fragment layout of
// mma.m16n8k16 (gid = lane / 4, q = lane % 4):
//   A (16 x 16, rows = samples):  a0 = (gid, 2q..2q+1)   a1 = (gid+8, 2q..2q+1)
//                                 a2 = (gid, 2q+8..+9)   a3 = (gid+8, 2q+8..+9)
//   B (16 x 8, k x n):            b0 = (2q..2q+1, gid)   b1 = (2q+8..+9, gid)
//   C (16 x 8):                   c0,c1 = (gid, 2q..2q+1)  c2,c3 = (gid+8, 2q..2q+1)
// so the C tiles of one layer (n-tiles 2kt, 2kt+1) are the A fragment of
// k-tile kt of the next layer without any data movement.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace pstm {
namespace mlp {

constexpr int kIn = 7;
constexpr int kH = 64;
// flat FP32 parameter vector: W1[64][7] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kIn;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH * kH;
constexpr int kOffW4 = kOffB3 + kH;
constexpr int kOffB4 = kOffW4 + kH;
constexpr int kParams = kOffB4 + 1;   // 8897

constexpr int kS1 = 24;   // row stride (bf16) of the 64 x 16 first layer: conflict-free fragment loads
constexpr int kS = 72;    // row stride (bf16) of the 64 x 64 layers

// Shared-memory copy of the network for evaluation (and, with the
// transposes, for the backward pass).
struct Weights {
    __nv_bfloat16 w1[kH * kS1];    // [out][in], in padded to 16 with zeros
    __nv_bfloat16 w2[kH * kS];     // [out][in]
    __nv_bfloat16 w3[kH * kS];
    float b1[kH], b2[kH], b3[kH], w4[kH];
    float b4;
};
struct WeightsT {                  // transposes [in][out] of W2 and W3 for dX = dZ W
    __nv_bfloat16 w2t[kH * kS];
    __nv_bfloat16 w3t[kH * kS];
};

// Input normalisation and output scale of a trained network.
struct Norm {
    float shift[8];
    float scale[8];
    float out_scale;               // network output x out_scale = residual in seconds
};

// Cooperative load of the FP32 parameter vector into `w` (BF16 matrices).
__device__ inline void stage_weights(const float *__restrict__ prm, Weights &w, WeightsT *wt) {
    for (int i = threadIdx.x; i < kH * kS1; i += blockDim.x) {
        const int o = i / kS1, k = i - o * kS1;
        w.w1[i] = __float2bfloat16_rn(k < kIn ? prm[kOffW1 + o * kIn + k] : 0.f);
    }
    for (int i = threadIdx.x; i < kH * kS; i += blockDim.x) {
        const int o = i / kS, k = i - o * kS;
        const bool in = k < kH;
        w.w2[i] = __float2bfloat16_rn(in ? prm[kOffW2 + o * kH + k] : 0.f);
        w.w3[i] = __float2bfloat16_rn(in ? prm[kOffW3 + o * kH + k] : 0.f);
        if (wt) {   // row o of the transpose holds column o of W
            wt->w2t[i] = __float2bfloat16_rn(in ? prm[kOffW2 + k * kH + o] : 0.f);
            wt->w3t[i] = __float2bfloat16_rn(in ? prm[kOffW3 + k * kH + o] : 0.f);
        }
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        w.b1[i] = prm[kOffB1 + i];
        w.b2[i] = prm[kOffB2 + i];
        w.b3[i] = prm[kOffB3 + i];
        w.w4[i] = prm[kOffW4 + i];
    }
    if (threadIdx.x == 0) w.b4 = prm[kOffB4];
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x (low half) = lo
    return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint32_t *>(p);
}
__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU and its derivative, with the hardware tanh: sigma(z) = (1 + tanh(z/2)) / 2.
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigmoid(z);
    return s * fmaf(z, 1.f - s, 1.f);
}

// z = A W^T + b for one m-tile: A given as KT k-tiles of fragments, W [64][S]
// (rows = output features) in shared memory; z as 8 n-tiles of C fragments.
template <int KT, int S>
__device__ __forceinline__ void layer(const uint32_t (&a)[KT][4], const __nv_bfloat16 *W, const float *b,
                                      float (&z)[8][4]) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, q = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float b0 = b ? b[8 * j + 2 * q] : 0.f, b1 = b ? b[8 * j + 2 * q + 1] : 0.f;
        z[j][0] = b0;
        z[j][1] = b1;
        z[j][2] = b0;
        z[j][3] = b1;
        const __nv_bfloat16 *row = W + (8 * j + gid) * S + 2 * q;
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) mma(z[j], a[kt], ld32(row + 16 * kt), ld32(row + 16 * kt + 8));
    }
}

// C fragments (8 n-tiles) -> A fragments (4 k-tiles) of the next layer.
__device__ __forceinline__ void to_a(const float (&h)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        a[kt][0] = pack_bf16(h[2 * kt][0], h[2 * kt][1]);
        a[kt][1] = pack_bf16(h[2 * kt][2], h[2 * kt][3]);
        a[kt][2] = pack_bf16(h[2 * kt + 1][0], h[2 * kt + 1][1]);
        a[kt][3] = pack_bf16(h[2 * kt + 1][2], h[2 * kt + 1][3]);
    }
}

// First-layer A fragment from the normalised inputs of rows gid and gid+8:
// this lane supplies features 2q and 2q+1 of both rows (feature 7 and the
// k-columns 8..15 are zero padding).
__device__ __forceinline__ void input_fragment(float r0f0, float r0f1, float r1f0, float r1f1,
                                               uint32_t (&a)[1][4]) {
    a[0][0] = pack_bf16(r0f0, r0f1);
    a[0][1] = pack_bf16(r1f0, r1f1);
    a[0][2] = 0u;
    a[0][3] = 0u;
}

// Output layer of one m-tile: y for rows gid (first) and gid+8 (second), the
// same in the 4 lanes of a quad.
__device__ __forceinline__ float2 output(const float (&h)[8][4], const Weights &w) {
    const int q = threadIdx.x & 3;
    float p0 = 0.f, p1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float u0 = w.w4[8 * j + 2 * q], u1 = w.w4[8 * j + 2 * q + 1];
        p0 = fmaf(u0, h[j][0], fmaf(u1, h[j][1], p0));
        p1 = fmaf(u0, h[j][2], fmaf(u1, h[j][3], p1));
    }
    p0 += __shfl_xor_sync(0xffffffffu, p0, 1);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 1);
    p0 += __shfl_xor_sync(0xffffffffu, p0, 2);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 2);
    return make_float2(p0 + w.b4, p1 + w.b4);
}

// Forward pass of one m-tile (inference): returns y of rows gid, gid+8.
__device__ __forceinline__ float2 forward(const uint32_t (&a1)[1][4], const Weights &w) {
    float z[8][4];
    uint32_t a[4][4];
    layer<1, kS1>(a1, w.w1, w.b1, z);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) z[j][e] = silu(z[j][e]);
    to_a(z, a);
    layer<4, kS>(a, w.w2, w.b2, z);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) z[j][e] = silu(z[j][e]);
    to_a(z, a);
    layer<4, kS>(a, w.w3, w.b3, z);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) z[j][e] = silu(z[j][e]);
    return output(z, w);
}

}  // namespace mlp
}  // namespace pstm
