// Features, prediction and training targets of the learned warm start
// (mlp_kernels.cuh holds the network).
//
// For the Schur system S a = b of the non-primary FE rows (every column c on
// its own), the features of row g are those of the first Jacobi iterates
//
//     a1 = D^-1 b,  a2 = a1 + D^-1 (b - S a1),  a3 = a2 + D^-1 (b - S a2)
//
// (D the diagonal of S; a1 is the first sweep's group mean of the
// primary-demeaned residual), each scaled by the column's sigma_c = RMS of a1:
//
//     x = [u1, u2, u3, u2 - u1, u3 - u2, log1p(W_g) / 8, diag(S)_g / W_g, small]
//
// with W_g the level's weight, diag(S)_g / W_g the share of that weight that
// moves between primary groups (the level's mobility), and small = 1 for the
// levels of a small dim.  The network's outputs y = (y0, y1) give the warm
// start a0 = sigma_c (u3 + y0) and the row's Jacobi scaling
// exp(clamp(mean_c y1, +-kWsMaxLogScale)).  Training targets from a converged
// a*: y0* = a*/sigma - u3, y1* = log(a* / a1) where both have one sign.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200fe {

constexpr int kWsFeatures = 8;
constexpr double kWsMaxLogScale = 1.5;

// out = a + dinv (b - q), rows [GR][CP]
__global__ void ws_jacobi_kernel(int64_t GR, int CP, const double* __restrict__ a, const double* __restrict__ b,
                                 const double* __restrict__ q, const double* __restrict__ dinv,
                                 double* __restrict__ out) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < GR * CP;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double base = a ? a[i] : 0.0;
        out[i] = base + dinv[i / CP] * (b[i] - (q ? q[i] : 0.0));
    }
}

// sigma[c] = sqrt(sum_g a1[g][c]^2 / GR) from the column sums of squares
__global__ void ws_sigma_kernel(const double* __restrict__ sumsq, int64_t GR, int CP, double* __restrict__ sigma) {
    const int c = threadIdx.x;
    if (c < CP) sigma[c] = GR > 0 ? sqrt(sumsq[c] / static_cast<double>(GR)) : 0.0;
}

__device__ __forceinline__ double ws_div(double v, double s) { return s > 0.0 ? v / s : 0.0; }

// features of sample g * cols + c
__global__ void ws_features_kernel(int64_t GR, int CP, int cols, const double* __restrict__ a1,
                                   const double* __restrict__ a2, const double* __restrict__ a3,
                                   const double* __restrict__ sigma, const double* __restrict__ w_rows,
                                   const double* __restrict__ dinv, int64_t small_row0,
                                   float* __restrict__ feat) {
    for (int64_t sI = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; sI < GR * cols;
         sI += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = sI / cols;
        const int c = static_cast<int>(sI - g * cols);
        const int64_t i = g * CP + c;
        const double s = sigma[c];
        const double u1 = ws_div(a1[i], s), u2 = ws_div(a2[i], s), u3 = ws_div(a3[i], s);
        const double W = w_rows[g];
        const double d = dinv[g];
        float* f = feat + sI * kWsFeatures;
        f[0] = static_cast<float>(u1);
        f[1] = static_cast<float>(u2);
        f[2] = static_cast<float>(u3);
        f[3] = static_cast<float>(u2 - u1);
        f[4] = static_cast<float>(u3 - u2);
        f[5] = static_cast<float>(log1p(fmax(W, 0.0)) * 0.125);
        f[6] = static_cast<float>((d > 0.0 && W > 0.0) ? fmin(1.0 / (d * W), 1.0) : 0.0);
        f[7] = g >= small_row0 ? 1.0f : 0.0f;
    }
}

// a0[g][c] = sigma_c (u3 + y0) for c < cols, 0 in the padding columns
__global__ void ws_apply_kernel(int64_t GR, int CP, int cols, const double* __restrict__ a3,
                                const double* __restrict__ sigma, const float* __restrict__ y,
                                double* __restrict__ a0) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < GR * CP;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = i / CP;
        const int c = static_cast<int>(i - g * CP);
        double v = 0.0;
        if (c < cols && sigma[c] > 0.0) {
            const double yv = static_cast<double>(y[(g * cols + c) * 2]);
            v = a3[i] + sigma[c] * (isfinite(yv) ? yv : 0.0);
        }
        a0[i] = v;
    }
}

// per-row Jacobi scaling exp(clamp(mean_c y1)): scaled copies of dinv
__global__ void ws_scale_kernel(int64_t GR, int cols, const float* __restrict__ y,
                                const double* __restrict__ dinv, double* __restrict__ dinv64s,
                                float* __restrict__ dinv32s) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < GR;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double m = 0.0;
        for (int c = 0; c < cols; ++c) {
            const double v = static_cast<double>(y[(g * cols + c) * 2 + 1]);
            m += isfinite(v) ? v : 0.0;
        }
        m = fmin(fmax(m / cols, -kWsMaxLogScale), kWsMaxLogScale);
        const double d = dinv[g] * exp(m);
        dinv64s[g] = d;
        dinv32s[g] = static_cast<float>(d);
    }
}

// training targets (t0, t1, w0, w1) of sample g * cols + c from the converged a*
__global__ void ws_targets_kernel(int64_t GR, int CP, int cols, const double* __restrict__ astar,
                                  const double* __restrict__ a1, const double* __restrict__ a3,
                                  const double* __restrict__ sigma, float* __restrict__ targ) {
    for (int64_t sI = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; sI < GR * cols;
         sI += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = sI / cols;
        const int c = static_cast<int>(sI - g * cols);
        const int64_t i = g * CP + c;
        const double s = sigma[c];
        float* t = targ + sI * 4;
        if (!(s > 0.0)) {
            t[0] = t[1] = t[2] = t[3] = 0.0f;
            continue;
        }
        const double d0 = fmin(fmax(astar[i] / s - a3[i] / s, -20.0), 20.0);
        t[0] = static_cast<float>(d0);
        t[2] = 1.0f;
        const double ra = astar[i] / s, r1 = a1[i] / s;
        if (ra * r1 > 0.0 && fabs(r1) > 1e-3) {
            t[1] = static_cast<float>(fmin(fmax(log(ra / r1), -kWsMaxLogScale), kWsMaxLogScale));
            t[3] = static_cast<float>(fmin(fabs(r1), 1.0) * 0.25);
        } else {
            t[1] = 0.0f;
            t[3] = 0.0f;
        }
    }
}

}  // namespace b200fe
