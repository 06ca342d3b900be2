// surrogate.cu -- the learned traveltime form.
//
// A 7 -> 64 -> 64 -> 64 -> 1 SiLU network (mlp.cuh) learns, for one
// traveltime kind (VTI or curved+VTI), the difference between the exact FP64
// traveltime and the straight-ray DSR time at v_rms:
//     T(t0, dx_s, dy_s, dx_r, dy_r, v_rms, eta) = T_DSR + out_scale * net(x_n).
// Everything is written here: the seeded sample generator (exact FP64
// targets), the forward/backward pass on the tensor cores, Adam, batched
// inference, the per-tile probe and the migration kernel that uses the
// network per pair.  The learned tile entry point probes the network against
// the exact formula on random in-aperture pairs of the tile and falls back
// to the exact kernel when the largest residual exceeds the threshold.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "pstm_cuda.h"
#include "kparams.h"
#include "launch.h"
#include "migrate.cuh"
#include "mlp.cuh"
#include "ctx.h"

using namespace pstm;
using namespace pstm::ctx;

namespace {

// ------------------------------------------------------------------ helpers
__host__ __device__ inline uint64_t mix64(uint64_t z) {   // splitmix64 finaliser
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ inline double uniform01(uint64_t seed, uint64_t i, int k) {
    return (double)(mix64(seed ^ mix64(i * 16 + (uint64_t)k)) >> 11) * (1.0 / 9007199254740992.0);
}

mlp::Norm to_norm(const pstm_surrogate *net) {
    mlp::Norm n;
    for (int i = 0; i < 8; ++i) {
        n.shift[i] = net->shift[i];
        n.scale[i] = net->scale[i];
    }
    n.out_scale = net->out_scale;
    return n;
}

// One network evaluation per lane of a warp (32 samples, two m-tiles): `f`
// holds this lane's 7 normalised inputs; returns this lane's output.
__device__ inline float warp_mlp32(const mlp::Weights &w, const float (&f)[7]) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, q = lane & 3;
    float out[4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        float r0[7], r1[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            r0[k] = __shfl_sync(0xffffffffu, f[k], 16 * m + gid);
            r1[k] = __shfl_sync(0xffffffffu, f[k], 16 * m + gid + 8);
        }
        // features 2q, 2q+1 of rows gid and gid+8 (feature 7 is zero)
        float a0, a1, c0, c1;
        if (q == 0) { a0 = r0[0]; a1 = r0[1]; c0 = r1[0]; c1 = r1[1]; }
        else if (q == 1) { a0 = r0[2]; a1 = r0[3]; c0 = r1[2]; c1 = r1[3]; }
        else if (q == 2) { a0 = r0[4]; a1 = r0[5]; c0 = r1[4]; c1 = r1[5]; }
        else { a0 = r0[6]; a1 = 0.f; c0 = r1[6]; c1 = 0.f; }
        uint32_t a[1][4];
        mlp::input_fragment(a0, a1, c0, c1, a);
        const float2 y = mlp::forward(a, w);
        out[2 * m] = y.x;
        out[2 * m + 1] = y.y;
    }
    // row `lane` sits in m-tile lane/16, local row lane%16, held by quad (lane%8)
    const int src = (lane & 7) << 2;
    const float y0 = __shfl_sync(0xffffffffu, out[0], src), y1 = __shfl_sync(0xffffffffu, out[1], src);
    const float y2 = __shfl_sync(0xffffffffu, out[2], src), y3 = __shfl_sync(0xffffffffu, out[3], src);
    return lane < 8 ? y0 : (lane < 16 ? y1 : (lane < 24 ? y2 : y3));
}

__device__ inline void normalise(const mlp::Norm &n, const float (&raw)[7], float (&f)[7]) {
#pragma unroll
    for (int k = 0; k < 7; ++k) f[k] = (raw[k] - n.shift[k]) * n.scale[k];
}

// ------------------------------------------------------------------ samples
struct Domain {
    int kind;
    double v0, k, t0_max, h_max, v_a, v_b, v_rel, eta_slope, eta_jitter, eta_max;
};

template <int TT>
__global__ void samples_kernel(Domain d, uint64_t seed, int64_t first, int n, float *raw, float *residual,
                               double *t_exact) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint64_t i = (uint64_t)(first + j);
        const double t0 = d.t0_max * uniform01(seed, i, 0);
        const double dxs = d.h_max * (2.0 * uniform01(seed, i, 1) - 1.0);
        const double dys = d.h_max * (2.0 * uniform01(seed, i, 2) - 1.0);
        const double dxr = d.h_max * (2.0 * uniform01(seed, i, 3) - 1.0);
        const double dyr = d.h_max * (2.0 * uniform01(seed, i, 4) - 1.0);
        const double v = (d.v_a + d.v_b * t0) * (1.0 + d.v_rel * (2.0 * uniform01(seed, i, 5) - 1.0));
        double eta = d.eta_slope * t0 + d.eta_jitter * (2.0 * uniform01(seed, i, 6) - 1.0);
        eta = eta < 0.0 ? 0.0 : (eta > d.eta_max ? d.eta_max : eta);
        // the values the network sees are the FP32-rounded inputs
        const float f[7] = {(float)t0, (float)dxs, (float)dys, (float)dxr, (float)dyr, (float)v, (float)eta};
        const double ds2 = (double)f[1] * f[1] + (double)f[2] * f[2], dr2 = (double)f[3] * f[3] + (double)f[4] * f[4];
        const double T = traveltime_fp64<TT>(f[0], ds2, dr2, f[5], f[6], d.v0, d.k);
        const double Td = traveltime_fp64<TT_STRAIGHT>(f[0], ds2, dr2, f[5], 0.0, d.v0, d.k);
        for (int k = 0; k < 7; ++k) raw[(int64_t)j * 8 + k] = f[k];
        raw[(int64_t)j * 8 + 7] = 0.f;
        residual[j] = (float)(T - Td);
        if (t_exact) t_exact[j] = T;
    }
}

// ------------------------------------------------------------------ training
constexpr int kTrainWarps = 8;
constexpr int kTrainRows = 16 * kTrainWarps;   // samples per CTA
constexpr int kST = kTrainRows + 8;            // row stride (bf16) of the transposed activations

struct TrainSmem {
    mlp::Weights w;
    mlp::WeightsT wt;
    __nv_bfloat16 hT0[16 * kST];                // [input feature][sample]
    __nv_bfloat16 hT1[64 * kST], hT2[64 * kST]; // [feature][sample]
    __nv_bfloat16 dzT1[64 * kST], dzT2[64 * kST], dzT3[64 * kST];
    float gsmall[3 * 64 + 64 + 1];              // b1 b2 b3 w4 b4 gradients of this CTA
    float loss;
};

// Sum over the 8 row groups (lanes with the same q) of per-lane column partials.
__device__ __forceinline__ float sum_rows(float x) {
    x += __shfl_xor_sync(0xffffffffu, x, 4);
    x += __shfl_xor_sync(0xffffffffu, x, 8);
    x += __shfl_xor_sync(0xffffffffu, x, 16);
    return x;
}

// Column sums over the 16 rows of an m-tile of C fragments, added into g[64].
__device__ __forceinline__ void add_col_sums(const float (&z)[8][4], float *g) {
    const int lane = threadIdx.x & 31, q = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float s0 = sum_rows(z[j][0] + z[j][2]);
        const float s1 = sum_rows(z[j][1] + z[j][3]);
        if (lane < 4) {
            atomicAdd(&g[8 * j + 2 * q], s0);
            atomicAdd(&g[8 * j + 2 * q + 1], s1);
        }
    }
}

// Transposed BF16 store of an m-tile (rows = samples row0, row0+8) into T[feature][sample].
__device__ __forceinline__ void store_t(const float (&h)[8][4], __nv_bfloat16 *T, int row0) {
    const int q = threadIdx.x & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * q;
        T[c * kST + row0] = __float2bfloat16_rn(h[j][0]);
        T[(c + 1) * kST + row0] = __float2bfloat16_rn(h[j][1]);
        T[c * kST + row0 + 8] = __float2bfloat16_rn(h[j][2]);
        T[(c + 1) * kST + row0 + 8] = __float2bfloat16_rn(h[j][3]);
    }
}

// Gradients of loss = mean over n of (net(x_n) - residual/out_scale)^2,
// accumulated (+=) into grads; loss_sum += the sum of squared errors.
__global__ void __launch_bounds__(32 * kTrainWarps)
train_grad_kernel(const float *__restrict__ prm, mlp::Norm nrm, const float *__restrict__ raw,
                  const float *__restrict__ residual, int n, float inv_n, float *grads, float *loss_sum) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
    mlp::stage_weights(prm, S.w, &S.wt);
    for (int i = threadIdx.x; i < 16 * kST; i += blockDim.x) S.hT0[i] = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < 3 * 64 + 64 + 1; i += blockDim.x) S.gsmall[i] = 0.f;
    if (threadIdx.x == 0) S.loss = 0.f;
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, q = lane & 3;
    const int row0 = 16 * warp + gid;                 // CTA-local rows of this lane
    const int64_t s0 = (int64_t)blockIdx.x * kTrainRows + row0, s1 = s0 + 8;
    const bool v0 = s0 < n, v1 = s1 < n;
    float x0[2] = {0.f, 0.f}, x1[2] = {0.f, 0.f};     // features 2q, 2q+1 of the two rows
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int k = 2 * q + e;
        if (k < 7) {
            if (v0) x0[e] = (raw[s0 * 8 + k] - nrm.shift[k]) * nrm.scale[k];
            if (v1) x1[e] = (raw[s1 * 8 + k] - nrm.shift[k]) * nrm.scale[k];
        }
        S.hT0[k * kST + row0] = __float2bfloat16_rn(x0[e]);
        S.hT0[k * kST + row0 + 8] = __float2bfloat16_rn(x1[e]);
    }
    uint32_t a1[1][4];
    mlp::input_fragment(x0[0], x0[1], x1[0], x1[1], a1);

    // forward, keeping the pre-activations
    float z1[8][4], z2[8][4], z3[8][4], h[8][4];
    uint32_t a[4][4];
    mlp::layer<1, mlp::kS1>(a1, S.w.w1, S.w.b1, z1);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) h[j][e] = mlp::silu(z1[j][e]);
    store_t(h, S.hT1, 16 * warp + gid);
    mlp::to_a(h, a);
    mlp::layer<4, mlp::kS>(a, S.w.w2, S.w.b2, z2);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) h[j][e] = mlp::silu(z2[j][e]);
    store_t(h, S.hT2, 16 * warp + gid);
    mlp::to_a(h, a);
    mlp::layer<4, mlp::kS>(a, S.w.w3, S.w.b3, z3);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) h[j][e] = mlp::silu(z3[j][e]);
    const float2 y = mlp::output(h, S.w);

    // loss and dL/dy (rows outside n contribute nothing)
    const float e0 = v0 ? y.x - residual[s0] / nrm.out_scale : 0.f;
    const float e1 = v1 ? y.y - residual[s1] / nrm.out_scale : 0.f;
    if (q == 0) atomicAdd(&S.loss, e0 * e0 + e1 * e1);
    const float dy0 = 2.f * e0 * inv_n, dy1 = 2.f * e1 * inv_n;
    if (q == 0) atomicAdd(&S.gsmall[4 * 64], dy0 + dy1);   // b4

    // output layer: dw4 = sum_rows dy h3; dh3 = dy w4; dz3 = dh3 silu'(z3)
    float g[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        g[j][0] = dy0 * h[j][0];
        g[j][1] = dy0 * h[j][1];
        g[j][2] = dy1 * h[j][2];
        g[j][3] = dy1 * h[j][3];
    }
    add_col_sums(g, &S.gsmall[3 * 64]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float u0 = S.w.w4[8 * j + 2 * q], u1 = S.w.w4[8 * j + 2 * q + 1];
        g[j][0] = dy0 * u0 * mlp::dsilu(z3[j][0]);
        g[j][1] = dy0 * u1 * mlp::dsilu(z3[j][1]);
        g[j][2] = dy1 * u0 * mlp::dsilu(z3[j][2]);
        g[j][3] = dy1 * u1 * mlp::dsilu(z3[j][3]);
    }
    add_col_sums(g, &S.gsmall[2 * 64]);   // b3
    store_t(g, S.dzT3, 16 * warp + gid);
    // dh2 = dz3 W3; dz2 = dh2 silu'(z2)
    mlp::to_a(g, a);
    mlp::layer<4, mlp::kS>(a, S.wt.w3t, nullptr, h);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) g[j][e] = h[j][e] * mlp::dsilu(z2[j][e]);
    add_col_sums(g, &S.gsmall[1 * 64]);   // b2
    store_t(g, S.dzT2, 16 * warp + gid);
    mlp::to_a(g, a);
    mlp::layer<4, mlp::kS>(a, S.wt.w2t, nullptr, h);
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) g[j][e] = h[j][e] * mlp::dsilu(z1[j][e]);
    add_col_sums(g, &S.gsmall[0]);        // b1
    store_t(g, S.dzT1, 16 * warp + gid);
    __syncthreads();

    // weight gradients dW[o][i] = sum_s dz[s][o] h[s][i]: mma with M = o, N = i,
    // K = the CTA's 128 samples; 32 + 32 + 8 output tiles over the 8 warps
    for (int tile = warp; tile < 72; tile += kTrainWarps) {
        const __nv_bfloat16 *A, *B;
        int mt, nt, off, nin;
        if (tile < 32) { A = S.dzT3; B = S.hT2; mt = tile >> 3; nt = tile & 7; off = mlp::kOffW3; nin = 64; }
        else if (tile < 64) { A = S.dzT2; B = S.hT1; mt = (tile - 32) >> 3; nt = (tile - 32) & 7; off = mlp::kOffW2; nin = 64; }
        else { A = S.dzT1; B = S.hT0; mt = (tile - 64) >> 1; nt = (tile - 64) & 1; off = mlp::kOffW1; nin = 7; }
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16 *ar0 = A + (16 * mt + gid) * kST + 2 * q, *ar1 = ar0 + 8 * kST;
        const __nv_bfloat16 *br = B + (8 * nt + gid) * kST + 2 * q;
#pragma unroll
        for (int kt = 0; kt < kTrainRows / 16; ++kt) {
            const uint32_t af[4] = {mlp::ld32(ar0 + 16 * kt), mlp::ld32(ar1 + 16 * kt), mlp::ld32(ar0 + 16 * kt + 8),
                                    mlp::ld32(ar1 + 16 * kt + 8)};
            mlp::mma(d, af, mlp::ld32(br + 16 * kt), mlp::ld32(br + 16 * kt + 8));
        }
        const int o0 = 16 * mt + gid, i0 = 8 * nt + 2 * q;
        if (i0 < nin) {
            atomicAdd(&grads[off + o0 * nin + i0], d[0]);
            atomicAdd(&grads[off + (o0 + 8) * nin + i0], d[2]);
        }
        if (i0 + 1 < nin) {
            atomicAdd(&grads[off + o0 * nin + i0 + 1], d[1]);
            atomicAdd(&grads[off + (o0 + 8) * nin + i0 + 1], d[3]);
        }
    }
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        atomicAdd(&grads[mlp::kOffB1 + i], S.gsmall[i]);
        atomicAdd(&grads[mlp::kOffB2 + i], S.gsmall[64 + i]);
        atomicAdd(&grads[mlp::kOffB3 + i], S.gsmall[128 + i]);
        atomicAdd(&grads[mlp::kOffW4 + i], S.gsmall[192 + i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grads[mlp::kOffB4], S.gsmall[256]);
        atomicAdd(loss_sum, S.loss);
    }
}

// Adam (bias-corrected) on the FP32 master parameters; clears the gradients.
__global__ void adam_kernel(float *prm, float *grads, float *m, float *v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = grads[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        prm[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        grads[i] = 0.f;
    }
}

// ------------------------------------------------------------------ inference
__global__ void __launch_bounds__(256) eval_kernel(const float *__restrict__ prm, mlp::Norm nrm,
                                                   const float *__restrict__ raw, int n, float *residual) {
    __shared__ mlp::Weights w;
    mlp::stage_weights(prm, w, nullptr);
    __syncthreads();
    const int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll;   // this warp's 32 samples
    for (int64_t b = base; b < n; b += (int64_t)gridDim.x * blockDim.x) {   // warp-uniform loop
        const int64_t i = b + (threadIdx.x & 31);
        float r[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, f[7];
        if (i < n)
            for (int k = 0; k < 7; ++k) r[k] = raw[i * 8 + k];
        normalise(nrm, r, f);
        const float y = warp_mlp32(w, f);
        if (i < n) residual[i] = y * nrm.out_scale;
    }
}

// ------------------------------------------------------------------ probe
// Random in-aperture (pillar, trace, time) pairs of the tile: |T_surrogate -
// T_exact| in ms, or -1 for a draw outside the pair's aperture.
template <int TT>
__global__ void __launch_bounds__(256) probe_kernel(const KParams P, const KParams *__restrict__ Pg,
                                                    const float *__restrict__ prm, mlp::Norm nrm, uint64_t seed,
                                                    int n_probe, float *err_ms) {
    __shared__ mlp::Weights w;
    mlp::stage_weights(prm, w, nullptr);
    __syncthreads();
    const int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll;
    const int64_t n_p = (int64_t)P.nx * P.ny;
    for (int64_t b = base; b < n_probe; b += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = b + (threadIdx.x & 31);
        const uint64_t h1 = mix64(seed ^ mix64((uint64_t)i * 3 + 0));
        const uint64_t h2 = mix64(seed ^ mix64((uint64_t)i * 3 + 1));
        const uint64_t h3 = mix64(seed ^ mix64((uint64_t)i * 3 + 2));
        const int p = (int)(h1 % (uint64_t)n_p);
        const int64_t tr = (int64_t)(h2 % (uint64_t)P.n_traces);
        const int t = (int)(h3 % (uint64_t)P.nt);
        const int ix = p / P.ny, iy = p - ix * P.ny;
        const double ox = P.xg ? P.xg[p] : P.xa[ix], oy = P.yg ? P.yg[p] : P.ya[iy];
        TimeState ts;
        PtState s;
        load_states<TT_STRAIGHT, false>(P, p, t, ts, s);
        const double dxm = ox - P.mx[tr], dym = oy - P.my[tr];
        const bool act = (float)sqrt(dxm * dxm + dym * dym) <= s.ap;
        const float4 tab = P.ttab[(P.vel3d || P.eta3d) ? (int64_t)p * P.nt + t : t];
        const float dxs = (float)(ox - P.sx[tr]), dys = (float)(oy - P.sy[tr]);
        const float dxr = (float)(ox - P.rx[tr]), dyr = (float)(oy - P.ry[tr]);
        const float r[7] = {(float)(P.ta[t] / 1000.0), dxs, dys, dxr, dyr, 1.f / tab.z, tab.w};
        float f[7];
        normalise(nrm, r, f);
        const float y = warp_mlp32(w, f);
        const float ds2 = fmaf(dxs, dxs, dys * dys), dr2 = fmaf(dxr, dxr, dyr * dyr);
        const float Td = sqrt_approx(fmaf(ds2, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(dr2, s.iv2, ts.t0h2));
        const double Te = exact_traveltime<TT>(Pg, tr, p, t, ox, oy);
        const float Ts = ts.tz ? 0.f : Td + y * nrm.out_scale;   // t0 = 0: T = 0 exactly, as the exact kernel
        if (i < n_probe) err_ms[i] = act ? (float)(fabs((double)Ts - Te) * 1000.0) : -1.f;
    }
}

// ------------------------------------------------------------------ learned migration
// One CTA of 4 warps = one pillar x 128 output times; every warp walks all
// traces and evaluates the network for its 32 times of each in-aperture
// trace.  Weights, interpolation and accumulation follow the exact kernel.
template <int AMP>
__global__ void __launch_bounds__(128) migrate_learned_kernel(const KParams P, const float *__restrict__ prm,
                                                              mlp::Norm nrm) {
    __shared__ mlp::Weights w;
    mlp::stage_weights(prm, w, nullptr);
    __syncthreads();
    const int p = blockIdx.x;
    const int ix = p / P.ny, iy = p - ix * P.ny;
    const double ox = P.xg ? P.xg[p] : P.xa[ix], oy = P.yg ? P.yg[p] : P.ya[iy];
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.y * blockDim.x + threadIdx.x;
    const bool tv = t < P.nt;
    const int tc = tv ? t : P.nt - 1;
    TimeState ts;
    PtState s;
    // the weight tables are in samples when the tile was prepared for the FP64
    // sample-index kernel (its exact fallback), else in seconds; T is in seconds
    const bool samples = P.exact_units != 0;
    if (samples) load_states<TT_STRAIGHT, true>(P, p, t, ts, s);   // s.ap < 0 past the tile end
    else load_states<TT_STRAIGHT, false>(P, p, t, ts, s);
    const float tw = samples ? P.inv_dt_f : 1.f;   // T in the weights' unit
    const float4 tab = P.ttab[(P.vel3d || P.eta3d) ? (int64_t)p * P.nt + tc : tc];
    const float t0 = (float)(P.ta[tc] / 1000.0), v = 1.f / tab.z, eta = tab.w;
    const bool w_one = P.spreading + P.obliquity == 1, w_two = P.spreading + P.obliquity == 2;
    const float smax = (float)(P.ns - 1);
    float acc = 0.f;
    int cnt = 0;
    for (int64_t tr = 0; tr < P.n_traces; ++tr) {
        const double *g = P.geo + tr * kGeoDoubles;
        const double dxm = ox - g[4], dym = oy - g[5];
        const double d2 = dxm * dxm + dym * dym;
        cnt += d2 <= P.fold_d2_max;
        const float d = (float)sqrt(d2);
        const bool act = tv && d <= s.ap;
        if (__any_sync(0xffffffffu, act)) {
            const float dxs = (float)(ox - g[0]), dys = (float)(oy - g[1]);
            const float dxr = (float)(ox - g[2]), dyr = (float)(oy - g[3]);
            const float r[7] = {t0, dxs, dys, dxr, dyr, v, eta};
            float f[7];
            normalise(nrm, r, f);
            const float y = warp_mlp32(w, f);
            const float ds2 = fmaf(dxs, dxs, dys * dys), dr2 = fmaf(dxr, dxr, dyr * dyr);
            float T = sqrt_approx(fmaf(ds2, s.iv2, ts.t0h2)) + sqrt_approx(fmaf(dr2, s.iv2, ts.t0h2)) +
                      y * nrm.out_scale;
            T = ts.tz ? 0.f : T;   // t0 = 0: every pair has T = 0 exactly (VTI; curved with k != 0)
            float sidx = fmaf(T, P.s_scale, P.s_offset);
            const bool ok = act && sidx >= 0.f && sidx < smax;
            sidx = ok ? sidx : 0.f;
            const int i0 = (int)sidx;
            const float fr = sidx - (float)i0;
            const unsigned char *row =
                reinterpret_cast<const unsigned char *>(P.amps) + (tr * P.amp_stride) * (int64_t)P.elem;
            const float a0 = amp_at<AMP>(row, i0), a1 = amp_at<AMP>(row, ok ? i0 + 1 : 0);
            const float amp = fmaf(fr, a1 - a0, a0);
            float wt = ok ? (float)g[6] : 0.f;
            const float x = fmaf(d, s.itw, s.tsn);
            wt *= x > 0.f ? taper_weight(x) : 1.f;
            const float Tw = T * tw;
            const float rT = rcp_approx(Tw);
            float gw = w_two ? s.K * rT * rT : (w_one ? s.K * rT : 1.f);
            gw = Tw > ts.tg ? gw : 1.f;
            if (P.aa) {
                const float sth = fminf((float)fmax(fabs(dxm), fabs(dym)) * s.ivw_t * rT, 1.f);
                const float aa = fmaxf(0.f, 1.f - fmaxf(s.aaA * sth, P.aa_cB));
                gw = (sth >= 0.01f && Tw >= ts.tguard) ? gw * aa : gw;
            }
            acc = fmaf(amp, wt * gw, acc);
        }
        if ((tr & 511) == 511 && tv) {   // FP32 partials into the image every 512 traces
            const int64_t idx = (int64_t)p * P.nt + t;
            if (P.image_f32) reinterpret_cast<float *>(P.image)[idx] += acc;
            else reinterpret_cast<double *>(P.image)[idx] += (double)acc;
            acc = 0.f;
        }
    }
    if (tv) {
        const int64_t idx = (int64_t)p * P.nt + t;
        if (P.image_f32) reinterpret_cast<float *>(P.image)[idx] += acc;
        else reinterpret_cast<double *>(P.image)[idx] += (double)acc;
        if (P.fold && P.fold3d) P.fold[idx] += cnt;
    }
    if (P.fold && !P.fold3d && blockIdx.y == 0 && threadIdx.x == 0) P.fold[p] += cnt;
    (void)warp;
}

int32_t check_net(Ctx *c, const pstm_surrogate *net) {
    if (!net || !net->params) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null surrogate or parameters");
    if (!(net->out_scale > 0.f)) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "surrogate out_scale must be > 0");
    if (net->traveltime != PSTM_TT_VTI && net->traveltime != PSTM_TT_CURVED_VTI)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "the surrogate approximates VTI or curved+VTI traveltime");
    return PSTM_OK;
}

int grid_for(int64_t n, int per_block) {
    int64_t b = (n + per_block - 1) / per_block;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b > 0 ? b : 1);
}

}  // namespace

extern "C" {

int32_t pstm_cuda_surrogate_param_count(void) { return mlp::kParams; }

int32_t pstm_cuda_surrogate_samples(void *ctx, const pstm_surrogate_domain *dom, uint64_t seed, int64_t first,
                                    int32_t n, float *raw, float *residual, double *t_exact, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (!dom || n < 0 || (n > 0 && (!raw || !residual))) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bad sample arguments");
    if (dom->traveltime != PSTM_TT_VTI && dom->traveltime != PSTM_TT_CURVED_VTI)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "the surrogate approximates VTI or curved+VTI traveltime");
    if (n == 0) return PSTM_OK;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    Domain d{dom->traveltime, dom->curved_v0, dom->curved_k, dom->t0_max_s, dom->h_max_m, dom->v_a, dom->v_b,
             dom->v_rel, dom->eta_slope, dom->eta_jitter, dom->eta_max};
    if (dom->traveltime == PSTM_TT_VTI)
        samples_kernel<TT_VTI><<<grid_for(n, 256), 256, 0, st>>>(d, seed, first, n, raw, residual, t_exact);
    else
        samples_kernel<TT_CURVED_VTI><<<grid_for(n, 256), 256, 0, st>>>(d, seed, first, n, raw, residual, t_exact);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "samples launch");
    return PSTM_OK;
}

int32_t pstm_cuda_surrogate_gradients(void *ctx, const pstm_surrogate *net, const float *raw, const float *residual,
                                      int32_t n, float *grads, float *loss_sum, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    int32_t rc = check_net(c, net);
    if (rc) return rc;
    if (n <= 0 || !raw || !residual || !grads || !loss_sum)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bad gradient arguments");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    // set on every call: the attribute belongs to the current device, and a
    // context may live on any device
    e = cudaFuncSetAttribute(train_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
    if (e != cudaSuccess) return cuda_fail(c, e, "configuring the training kernel");
    const int blocks = (n + kTrainRows - 1) / kTrainRows;
    train_grad_kernel<<<blocks, 32 * kTrainWarps, sizeof(TrainSmem), st>>>(net->params, to_norm(net), raw, residual,
                                                                         n, 1.f / (float)n, grads, loss_sum);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "training kernel launch");
    return PSTM_OK;
}

int32_t pstm_cuda_surrogate_adam(void *ctx, float *params, float *grads, float *m, float *v, int32_t step, float lr,
                                 void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    if (!params || !grads || !m || !v || step < 1) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bad Adam arguments");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, step)));
    adam_kernel<<<grid_for(mlp::kParams, 256), 256, 0, st>>>(params, grads, m, v, mlp::kParams, lr, b1, b2, 1e-8f,
                                                             c1, c2);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "Adam launch");
    return PSTM_OK;
}

int32_t pstm_cuda_surrogate_eval(void *ctx, const pstm_surrogate *net, const float *raw, int32_t n, float *residual,
                                 void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    int32_t rc = check_net(c, net);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!raw || !residual))) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "bad evaluation arguments");
    if (n == 0) return PSTM_OK;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    eval_kernel<<<grid_for(n, 256), 256, 0, st>>>(net->params, to_norm(net), raw, n, residual);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "evaluation launch");
    return PSTM_OK;
}

int32_t pstm_cuda_migrate_tile_learned_dev(void *ctx, const pstm_traces_desc *traces, const pstm_output_desc *output,
                                           const pstm_velocity_desc *velocity, const pstm_params *params,
                                           const pstm_surrogate *net, float max_residual_ms, int32_t n_probe,
                                           pstm_learned_report *report, void *stream) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return fail(nullptr, PSTM_ERR_NOT_INITIALIZED, "Kernel not initialized");
    int32_t rc = check_net(c, net);
    if (rc) return rc;
    if (!params || !report) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "null descriptor");
    std::memset(report, 0, sizeof(*report));
    if (params->interpolation != PSTM_INTERP_LINEAR)
        return fail(c, PSTM_ERR_UNSUPPORTED, "the learned form interpolates linearly");
    if (params->traveltime != net->traveltime)
        return fail(c, PSTM_ERR_INVALID_ARGUMENT, "the surrogate was trained for another traveltime kind");
    if (n_probe < 32) n_probe = 32;
    if (n_probe > (1 << 22)) return fail(c, PSTM_ERR_INVALID_ARGUMENT, "n_probe above 4M");
    cudaStream_t st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    TilePlan tp;
    if ((rc = prepare_tile(c, traces, output, velocity, params, st, tp)) != PSTM_OK || tp.empty) return rc;

    // probe: |T_surrogate - T_exact| on random in-aperture pairs of this tile
    cudaError_t e;
    if ((e = ensure(c->probe, (size_t)n_probe * sizeof(float))) != cudaSuccess)
        return cuda_fail(c, e, "allocating the probe buffer");
    float *err = reinterpret_cast<float *>(c->probe.ptr);
    const mlp::Norm nrm = to_norm(net);
    const uint64_t seed = 0x5EED5EEDull ^ (uint64_t)tp.P.n_traces;
    if (tp.tt == PSTM_TT_VTI)
        probe_kernel<TT_VTI><<<grid_for(n_probe, 256), 256, 0, st>>>(tp.P, tp.Pg, net->params, nrm, seed, n_probe, err);
    else
        probe_kernel<TT_CURVED_VTI><<<grid_for(n_probe, 256), 256, 0, st>>>(tp.P, tp.Pg, net->params, nrm, seed,
                                                                            n_probe, err);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "probe launch");
    std::string host(n_probe * sizeof(float), '\0');
    if ((e = cudaMemcpyAsync(&host[0], err, n_probe * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(c, e, "reading the probe");
    const float *h = reinterpret_cast<const float *>(host.data());
    double mx = 0.0, ss = 0.0;
    int used = 0;
    for (int i = 0; i < n_probe; ++i)
        if (h[i] >= 0.f) {
            mx = h[i] > mx ? h[i] : mx;
            ss += (double)h[i] * h[i];
            ++used;
        }
    report->probe_max_ms = (float)mx;
    report->probe_rms_ms = used ? (float)std::sqrt(ss / used) : 0.f;
    report->n_probe_used = used;
    const float thr = max_residual_ms == 0.f ? 0.1f : max_residual_ms;
    const bool learned = used > 0 && (thr < 0.f || mx <= thr);
    report->used_surrogate = learned ? 1 : 0;
    if (!learned) return launch_tile(c, tp);   // exact fallback

    const dim3 grid((unsigned)((int64_t)output->nx * output->ny), (unsigned)((output->nt + 127) / 128));
    switch (traces->amp_dtype) {
    case PSTM_AMP_F32: migrate_learned_kernel<AMP_F32><<<grid, 128, 0, st>>>(tp.P, net->params, nrm); break;
    case PSTM_AMP_BF16: migrate_learned_kernel<AMP_BF16><<<grid, 128, 0, st>>>(tp.P, net->params, nrm); break;
    default: migrate_learned_kernel<AMP_F16><<<grid, 128, 0, st>>>(tp.P, net->params, nrm); break;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(c, e, "learned migrate kernel launch");
    return PSTM_OK;
}

}  // extern "C"
