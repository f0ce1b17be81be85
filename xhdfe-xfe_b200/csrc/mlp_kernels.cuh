// The learned warm start's network: a 3-hidden-layer, 64-wide MLP with BF16
// weights and activations and FP32 accumulation (no counterpart in the
// reference; its FP64 CPU restatement, the oracle of these kernels, is
// oracle/mlp_oracle.py):
//
//     h1 = bf16(relu(W1 x + b1)), h2 = bf16(relu(W2 h1 + b2)),
//     h3 = bf16(relu(W3 h2 + b3)), y = W4 h3 + b4        (8 -> 64 -> 64 -> 64 -> 2)
//
// Master parameters are FP32 (flat layout: W1 64x8, b1, W2 64x64, b2, W3 64x64,
// b3, W4 2x64, b4; 9026 values).  mlp_pack_kernel rounds the weights to BF16
// into the padded layout the forward kernel stages in shared memory.
//
// * mlp_forward_kernel (inference): tensor cores, mma.sync m16n8k16 BF16 with
//   FP32 accumulators; a warp runs 16 samples through all four layers, each
//   layer's accumulator fragments repacked in registers as the next layer's A
//   fragments (the m16n8 accumulator of two adjacent n-tiles is exactly one
//   m16k16 A fragment).
// * mlp_grad_kernel (training): the loss gradient of a batch, per CTA over
//   blocks of 64 samples staged in shared memory, FP32 arithmetic on the same
//   BF16-rounded weights and activations; per-CTA partial gradients summed in
//   CTA order in FP64 by mlp_reduce_kernel (deterministic), then
//   mlp_adam_kernel updates the FP32 master parameters.

#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace b200fe {

constexpr int kMlpIn = 8, kMlpHid = 64, kMlpOut = 2;
constexpr int kMlpParams = kMlpHid * kMlpIn + kMlpHid + 2 * (kMlpHid * kMlpHid + kMlpHid) +
                           kMlpOut * kMlpHid + kMlpOut;  // 9026
// offsets of the flat FP32 master layout
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpHid * kMlpIn, kOffW2 = kOffB1 + kMlpHid,
              kOffB2 = kOffW2 + kMlpHid * kMlpHid, kOffW3 = kOffB2 + kMlpHid,
              kOffB3 = kOffW3 + kMlpHid * kMlpHid, kOffW4 = kOffB3 + kMlpHid,
              kOffB4 = kOffW4 + kMlpOut * kMlpHid;

// Packed BF16 weights (rows padded so that the B-fragment loads of the eight
// row groups hit distinct shared-memory banks) and FP32 biases.
constexpr int kLd1 = 24;  // W1 row stride (16 used: 8 inputs + 8 zero)
constexpr int kLdH = 72;  // W2, W3, W4 row stride (64 used)
struct MlpPacked {
    __nv_bfloat16 w1[kMlpHid * kLd1];
    __nv_bfloat16 w2[kMlpHid * kLdH];
    __nv_bfloat16 w3[kMlpHid * kLdH];
    __nv_bfloat16 w4[8 * kLdH];  // rows 2..7 zero
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[8];
};

__global__ void mlp_pack_kernel(const float* __restrict__ p, MlpPacked* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpHid * kLdH; i += gridDim.x * blockDim.x) {
        const int r = i / kLdH, c = i % kLdH;
        if (i < kMlpHid * kLd1) {
            const int r1 = i / kLd1, c1 = i % kLd1;
            out->w1[i] = __float2bfloat16_rn(c1 < kMlpIn ? p[kOffW1 + r1 * kMlpIn + c1] : 0.0f);
        }
        out->w2[i] = __float2bfloat16_rn(c < kMlpHid ? p[kOffW2 + r * kMlpHid + c] : 0.0f);
        out->w3[i] = __float2bfloat16_rn(c < kMlpHid ? p[kOffW3 + r * kMlpHid + c] : 0.0f);
        if (i < 8 * kLdH)
            out->w4[i] = __float2bfloat16_rn((r < kMlpOut && c < kMlpHid) ? p[kOffW4 + r * kMlpHid + c] : 0.0f);
        if (i < kMlpHid) {
            out->b1[i] = p[kOffB1 + i];
            out->b2[i] = p[kOffB2 + i];
            out->b3[i] = p[kOffB3 + i];
        }
        if (i < 8) out->b4[i] = i < kMlpOut ? p[kOffB4 + i] : 0.0f;
    }
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A * B + D, A 16x16 BF16 (row), B 16x8 BF16 (col), D 16x8 FP32
__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One 64-wide layer on a 16-sample tile: acc[j] (n-tile j = units 8j..8j+7)
// = bias + sum over the four k-tiles of A[kk] x W^T; W rows padded to kLdH.
__device__ __forceinline__ void mlp_layer64(float (&acc)[8][4], const uint32_t (&a)[4][4],
                                            const __nv_bfloat16* w, const float* bias, int g, int t) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float b0 = bias[8 * j + 2 * t], b1 = bias[8 * j + 2 * t + 1];
        acc[j][0] = b0; acc[j][1] = b1; acc[j][2] = b0; acc[j][3] = b1;
        const __nv_bfloat16* wr = w + (8 * j + g) * kLdH + 2 * t;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const uint32_t b0r = *reinterpret_cast<const uint32_t*>(wr + 16 * kk);
            const uint32_t b1r = *reinterpret_cast<const uint32_t*>(wr + 16 * kk + 8);
            mma_16816(acc[j], a[kk], b0r, b1r);
        }
    }
}

// relu, BF16 rounding, and the repack of a 16x64 accumulator as A fragments
__device__ __forceinline__ void mlp_to_a(const float (&acc)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        a[kk][0] = pack_bf16x2(fmaxf(acc[2 * kk][0], 0.f), fmaxf(acc[2 * kk][1], 0.f));
        a[kk][1] = pack_bf16x2(fmaxf(acc[2 * kk][2], 0.f), fmaxf(acc[2 * kk][3], 0.f));
        a[kk][2] = pack_bf16x2(fmaxf(acc[2 * kk + 1][0], 0.f), fmaxf(acc[2 * kk + 1][1], 0.f));
        a[kk][3] = pack_bf16x2(fmaxf(acc[2 * kk + 1][2], 0.f), fmaxf(acc[2 * kk + 1][3], 0.f));
    }
}

// y[n][2] = MLP(x[n][8]); 16 samples per warp per step.
__global__ void __launch_bounds__(256)
mlp_forward_kernel(const MlpPacked* __restrict__ pk, const float* __restrict__ x, int64_t n,
                   float* __restrict__ y) {
    __shared__ MlpPacked s;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(pk);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
        for (int i = threadIdx.x; i < static_cast<int>(sizeof(MlpPacked) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int64_t ntiles = (n + 15) / 16;
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t tile = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
         tile < ntiles; tile += nwarps) {
        const int64_t r0 = tile * 16 + g, r1 = r0 + 8;
        // layer 1: K = 8 inputs (+ 8 zero columns)
        uint32_t a1[4];
        {
            float2 v0 = make_float2(0.f, 0.f), v1 = make_float2(0.f, 0.f);
            if (r0 < n) v0 = *reinterpret_cast<const float2*>(x + r0 * kMlpIn + 2 * t);
            if (r1 < n) v1 = *reinterpret_cast<const float2*>(x + r1 * kMlpIn + 2 * t);
            a1[0] = pack_bf16x2(v0.x, v0.y);
            a1[1] = pack_bf16x2(v1.x, v1.y);
            a1[2] = 0u;
            a1[3] = 0u;
        }
        float acc[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float b0 = s.b1[8 * j + 2 * t], b1 = s.b1[8 * j + 2 * t + 1];
            acc[j][0] = b0; acc[j][1] = b1; acc[j][2] = b0; acc[j][3] = b1;
            const uint32_t w0 = *reinterpret_cast<const uint32_t*>(s.w1 + (8 * j + g) * kLd1 + 2 * t);
            mma_16816(acc[j], a1, w0, 0u);
        }
        uint32_t a[4][4];
        mlp_to_a(acc, a);
        mlp_layer64(acc, a, s.w2, s.b2, g, t);
        mlp_to_a(acc, a);
        mlp_layer64(acc, a, s.w3, s.b3, g, t);
        mlp_to_a(acc, a);
        // output layer: one n-tile (outputs 0, 1 real)
        float o[4] = {s.b4[2 * t], s.b4[2 * t + 1], s.b4[2 * t], s.b4[2 * t + 1]};
        const __nv_bfloat16* wr = s.w4 + g * kLdH + 2 * t;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma_16816(o, a[kk], *reinterpret_cast<const uint32_t*>(wr + 16 * kk),
                      *reinterpret_cast<const uint32_t*>(wr + 16 * kk + 8));
        if (t == 0) {
            if (r0 < n) *reinterpret_cast<float2*>(y + r0 * kMlpOut) = make_float2(o[0], o[1]);
            if (r1 < n) *reinterpret_cast<float2*>(y + r1 * kMlpOut) = make_float2(o[2], o[3]);
        }
    }
}

// ---------------------------------------------------------------------------
// Training gradient.  Targets per sample: (t0, t1, w0, w1); loss
// L = (1/n_total) sum w_o (y_o - t_o)^2.  A CTA takes blocks of kMlpBlock
// samples (blocks b, b + gridDim, ...), runs forward and backward on them in
// shared memory and accumulates its own gradient entries in registers:
// thread t owns row j = t % 64 of W2 and W3 (columns 16 (t / 64) .. + 15), of W1
// (columns 2 (t / 64), + 1), entry t of W4 (t < 128) and the biases of unit t
// (t < 64).  The CTA's gradient and loss go to partial[blockIdx][0..kMlpParams].
// ---------------------------------------------------------------------------
constexpr int kMlpBlock = 64;     // samples staged per step
constexpr int kMlpGradThreads = 256;
constexpr int kLdW = 65;          // padded row stride of the FP32 weight copies

struct MlpGradSmem {
    float w1[kMlpHid * 9], w2[kMlpHid * kLdW], w3[kMlpHid * kLdW], w4[kMlpOut * kMlpHid];
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[kMlpOut];
    float x[kMlpBlock * kMlpIn];
    float h1[kMlpBlock * kMlpHid], h2[kMlpBlock * kMlpHid], h3[kMlpBlock * kMlpHid];
    float da[kMlpBlock * kMlpHid], db[kMlpBlock * kMlpHid];
    float dy[kMlpBlock * kMlpOut];
    float tg[kMlpBlock * 4];
    float red[kMlpGradThreads];
};

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__global__ void __launch_bounds__(kMlpGradThreads)
mlp_grad_kernel(const float* __restrict__ prm, const float* __restrict__ x, const float* __restrict__ tgt,
                int64_t n, float inv_n, float* __restrict__ partial) {
    extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
    MlpGradSmem& S = *reinterpret_cast<MlpGradSmem*>(mlp_smem_raw);
    const int t = threadIdx.x;
    // BF16-rounded weights (FP32 copies), FP32 biases
    for (int i = t; i < kMlpHid * kMlpIn; i += kMlpGradThreads)
        S.w1[(i / kMlpIn) * 9 + i % kMlpIn] = bf16r(prm[kOffW1 + i]);
    for (int i = t; i < kMlpHid * kMlpHid; i += kMlpGradThreads) {
        S.w2[(i / kMlpHid) * kLdW + i % kMlpHid] = bf16r(prm[kOffW2 + i]);
        S.w3[(i / kMlpHid) * kLdW + i % kMlpHid] = bf16r(prm[kOffW3 + i]);
    }
    if (t < kMlpOut * kMlpHid) S.w4[t] = bf16r(prm[kOffW4 + t]);
    if (t < kMlpHid) {
        S.b1[t] = prm[kOffB1 + t];
        S.b2[t] = prm[kOffB2 + t];
        S.b3[t] = prm[kOffB3 + t];
    }
    if (t < kMlpOut) S.b4[t] = prm[kOffB4 + t];
    const int jj = t % kMlpHid;        // unit of this thread's rows
    const int sb = t / kMlpHid;        // sample phase (0..3)
    const int ib = 16 * sb;            // column block of W2 / W3 gradients
    float g2[16], g3[16], g1[2] = {0.f, 0.f}, g4 = 0.f, gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gb4 = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) g2[k] = g3[k] = 0.f;
    float loss = 0.f;
    __syncthreads();
    const int64_t nblk = (n + kMlpBlock - 1) / kMlpBlock;
    for (int64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int64_t s0 = blk * kMlpBlock;
        const int nb = static_cast<int>(n - s0 < kMlpBlock ? n - s0 : kMlpBlock);
        for (int i = t; i < kMlpBlock * kMlpIn; i += kMlpGradThreads)
            S.x[i] = i / kMlpIn < nb ? bf16r(x[s0 * kMlpIn + i]) : 0.f;
        for (int i = t; i < kMlpBlock * 4; i += kMlpGradThreads)
            S.tg[i] = i / 4 < nb ? tgt[s0 * 4 + i] : 0.f;
        __syncthreads();
        // forward: thread (unit jj, samples sb, sb + 4, ...)
        for (int sI = sb; sI < kMlpBlock; sI += 4) {
            float z = S.b1[jj];
#pragma unroll
            for (int i = 0; i < kMlpIn; ++i) z = fmaf(S.w1[jj * 9 + i], S.x[sI * kMlpIn + i], z);
            S.h1[sI * kMlpHid + jj] = bf16r(fmaxf(z, 0.f));
        }
        __syncthreads();
        for (int sI = sb; sI < kMlpBlock; sI += 4) {
            float z = S.b2[jj];
            for (int i = 0; i < kMlpHid; ++i) z = fmaf(S.w2[jj * kLdW + i], S.h1[sI * kMlpHid + i], z);
            S.h2[sI * kMlpHid + jj] = bf16r(fmaxf(z, 0.f));
        }
        __syncthreads();
        for (int sI = sb; sI < kMlpBlock; sI += 4) {
            float z = S.b3[jj];
            for (int i = 0; i < kMlpHid; ++i) z = fmaf(S.w3[jj * kLdW + i], S.h2[sI * kMlpHid + i], z);
            S.h3[sI * kMlpHid + jj] = bf16r(fmaxf(z, 0.f));
        }
        __syncthreads();
        if (t < kMlpBlock * kMlpOut) {  // output, loss term and its gradient
            const int sI = t / kMlpOut, o = t % kMlpOut;
            float yv = S.b4[o];
            for (int i = 0; i < kMlpHid; ++i) yv = fmaf(S.w4[o * kMlpHid + i], S.h3[sI * kMlpHid + i], yv);
            const float d = yv - S.tg[sI * 4 + o], w = S.tg[sI * 4 + 2 + o];
            S.dy[t] = sI < nb ? 2.f * w * d * inv_n : 0.f;
            if (sI < nb) loss = fmaf(w * d, d, loss);
        }
        __syncthreads();
        // backward
        if (t < kMlpOut * kMlpHid) {
            const int o = t / kMlpHid, i = t % kMlpHid;
            for (int sI = 0; sI < kMlpBlock; ++sI) g4 = fmaf(S.dy[sI * kMlpOut + o], S.h3[sI * kMlpHid + i], g4);
        }
        if (t < kMlpOut)
            for (int sI = 0; sI < kMlpBlock; ++sI) gb4 += S.dy[sI * kMlpOut + t];
        for (int sI = sb; sI < kMlpBlock; sI += 4) {  // d3 = (W4' dy) . [h3 > 0]
            float d = 0.f;
#pragma unroll
            for (int o = 0; o < kMlpOut; ++o) d = fmaf(S.dy[sI * kMlpOut + o], S.w4[o * kMlpHid + jj], d);
            S.da[sI * kMlpHid + jj] = S.h3[sI * kMlpHid + jj] > 0.f ? d : 0.f;
        }
        __syncthreads();
        for (int sI = 0; sI < kMlpBlock; ++sI) {  // W3 rows: d3 h2'
            const float dv = S.da[sI * kMlpHid + jj];
#pragma unroll
            for (int k = 0; k < 16; ++k) g3[k] = fmaf(dv, S.h2[sI * kMlpHid + ib + k], g3[k]);
        }
        if (t < kMlpHid)
            for (int sI = 0; sI < kMlpBlock; ++sI) gb3 += S.da[sI * kMlpHid + t];
        for (int sI = sb; sI < kMlpBlock; sI += 4) {  // d2 = (W3' d3) . [h2 > 0]
            float d = 0.f;
            for (int j = 0; j < kMlpHid; ++j) d = fmaf(S.da[sI * kMlpHid + j], S.w3[j * kLdW + jj], d);
            S.db[sI * kMlpHid + jj] = S.h2[sI * kMlpHid + jj] > 0.f ? d : 0.f;
        }
        __syncthreads();
        for (int sI = 0; sI < kMlpBlock; ++sI) {  // W2 rows: d2 h1'
            const float dv = S.db[sI * kMlpHid + jj];
#pragma unroll
            for (int k = 0; k < 16; ++k) g2[k] = fmaf(dv, S.h1[sI * kMlpHid + ib + k], g2[k]);
        }
        if (t < kMlpHid)
            for (int sI = 0; sI < kMlpBlock; ++sI) gb2 += S.db[sI * kMlpHid + t];
        __syncthreads();  // d3 (da) is read above; d1 overwrites it
        for (int sI = sb; sI < kMlpBlock; sI += 4) {  // d1 = (W2' d2) . [h1 > 0]
            float d = 0.f;
            for (int j = 0; j < kMlpHid; ++j) d = fmaf(S.db[sI * kMlpHid + j], S.w2[j * kLdW + jj], d);
            S.da[sI * kMlpHid + jj] = S.h1[sI * kMlpHid + jj] > 0.f ? d : 0.f;
        }
        __syncthreads();
        for (int sI = 0; sI < kMlpBlock; ++sI) {  // W1 rows: d1 x'
            const float dv = S.da[sI * kMlpHid + jj];
            g1[0] = fmaf(dv, S.x[sI * kMlpIn + 2 * sb], g1[0]);
            g1[1] = fmaf(dv, S.x[sI * kMlpIn + 2 * sb + 1], g1[1]);
        }
        if (t < kMlpHid)
            for (int sI = 0; sI < kMlpBlock; ++sI) gb1 += S.da[sI * kMlpHid + t];
        __syncthreads();  // the next block overwrites x, h and the deltas
    }
    float* out = partial + static_cast<int64_t>(blockIdx.x) * (kMlpParams + 1);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        out[kOffW2 + jj * kMlpHid + ib + k] = g2[k];
        out[kOffW3 + jj * kMlpHid + ib + k] = g3[k];
    }
    out[kOffW1 + jj * kMlpIn + 2 * sb] = g1[0];
    out[kOffW1 + jj * kMlpIn + 2 * sb + 1] = g1[1];
    if (t < kMlpOut * kMlpHid) out[kOffW4 + t] = g4;
    if (t < kMlpHid) {
        out[kOffB1 + t] = gb1;
        out[kOffB2 + t] = gb2;
        out[kOffB3 + t] = gb3;
    }
    if (t < kMlpOut) out[kOffB4 + t] = gb4;
    // loss: fixed tree over the threads
    S.red[t] = loss;
    __syncthreads();
    for (int h = kMlpGradThreads / 2; h > 0; h >>= 1) {
        if (t < h) S.red[t] += S.red[t + h];
        __syncthreads();
    }
    if (t == 0) out[kMlpParams] = S.red[0] * inv_n;
}

// grad[i] = sum over CTAs (in CTA order, FP64) of partial[c][i]; i = kMlpParams: loss
__global__ void mlp_reduce_kernel(const float* __restrict__ partial, int nparts, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= kMlpParams; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < nparts; ++c) s += static_cast<double>(partial[static_cast<int64_t>(c) * (kMlpParams + 1) + i]);
        out[i] = s;
    }
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters, arithmetic in FP64.
__global__ void mlp_adam_kernel(float* __restrict__ prm, float* __restrict__ m, float* __restrict__ v,
                                const double* __restrict__ grad, int step, double lr, double beta1,
                                double beta2, double eps) {
    const double c1 = 1.0 - pow(beta1, static_cast<double>(step));
    const double c2 = 1.0 - pow(beta2, static_cast<double>(step));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
        const double g = grad[i];
        const double mi = beta1 * static_cast<double>(m[i]) + (1.0 - beta1) * g;
        const double vi = beta2 * static_cast<double>(v[i]) + (1.0 - beta2) * g * g;
        m[i] = static_cast<float>(mi);
        v[i] = static_cast<float>(vi);
        prm[i] = static_cast<float>(static_cast<double>(prm[i]) - lr * (mi / c1) / (sqrt(vi / c2) + eps));
    }
}

}  // namespace b200fe
