// OLS on the within-transformed columns, on the device: the data-sized parts
// of the reference's run_ols (src/ols.cpp:1237-1520, compute_covariance
// :495-700).  What touches every observation runs here with fixed-order
// reductions (bitwise reproducible); the p x p algebra stays on the host.
//
//   moments_kernel  sum_i f_i a_i b_i over the pairs (a <= b) of P staged
//                   columns, f_i a per-row factor:
//                     Gram  [X y]' W [X y]      f = w,          columns X, y
//                     robust meat               f = (w e)^2 (analytic weights)
//                                                   or w e^2 (frequency weights)
//                   and, in the robust mode, sum_i w_i e_i^2 (the RSS);
//                   the RSS mode computes the RSS alone (no pair sums).
//   cluster_chunk_kernel  per chunk of one cluster (rows in cluster order):
//                   the score sums sum w e x_j and sum w e, e = y - x'b.
//
// A CTA owns a contiguous range of rows, stages kOlsTile rows of every
// column in shared memory (coalesced), and thread t owns pairs t, t + 256,
// ...; partials per CTA are summed in CTA order.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common_kernels.cuh"

namespace b200fe {

constexpr int kOlsMaxP = 32;      // regressors
constexpr int kOlsTile = 64;      // rows staged per step
constexpr int kOlsThreads = 256;
constexpr int kOlsChunk = 256;    // rows per cluster chunk
constexpr int kOlsSmallCluster = 32;  // clusters up to this many rows: one thread each

enum OlsMomentMode { kMomGram = 0, kMomRobust = 1, kMomPlain = 2, kMomRss = 3 };

struct MomentArgs {
    int64_t n;
    int P;                  // staged columns (p + 1 for the Gram with y)
    int p;                  // regressors (columns of X)
    const double* X;        // element (row, j) at X[j * cs + row * rs]
    int64_t cs, rs;
    const double* y;        // outcome (Gram: column P-1; robust: residuals); plain: column P-1
    const double* w;        // weights or null
    const int32_t* perm;    // row order or null
    int mode;
    int wfreq;              // frequency weights (robust meat uses w e^2)
    double beta[kOlsMaxP];  // robust mode: coefficients for the residuals
    double* partial;        // [grid][npairs]
    double* rss_partial;    // [grid] (robust mode)
};

__device__ __forceinline__ void pair_index(int t, int P, int& a, int& b) {
    // pairs ordered row by row of the upper triangle: (0,0) (0,1) .. (0,P-1) (1,1) ..
    a = 0;
    int rem = t;
    while (rem >= P - a) {
        rem -= P - a;
        ++a;
    }
    b = a + rem;
}

__global__ void __launch_bounds__(kOlsThreads)
moments_kernel(const MomentArgs m) {
    __shared__ double tile[kOlsMaxP + 1][kOlsTile + 1];  // padded: no bank conflicts across columns
    __shared__ double fac[kOlsTile];
    __shared__ double red[kOlsThreads];
    const int tid = threadIdx.x;
    const int npairs = m.P * (m.P + 1) / 2;
    // few pairs: R row slices of them (thread = slice x pair, slices combined
    // in order at the end); many pairs: up to three pairs per thread, all rows
    const int R = npairs <= kOlsThreads / 2 ? kOlsThreads / npairs : 1;
    const int slice = R > 1 ? tid / npairs : 0;
    const int pbase = R > 1 ? tid % npairs : tid;
    int pa[3], pb[3];
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        const int t = pbase + u * kOlsThreads;
        const bool mine = R > 1 ? (u == 0 && slice < R) : t < npairs;
        if (mine) pair_index(t, m.P, pa[u], pb[u]);
        else pa[u] = pb[u] = -1;
    }
    // row-major rows of P values (X then y at offset p, the score matrix)
    const bool row_major = m.mode == kMomPlain && m.cs == 1 && m.rs >= m.P && !m.perm;
    const int64_t per = (m.n + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t r1 = min(m.n, r0 + per);
    double rss = 0.0;
    for (int64_t base = r0; base < r1; base += kOlsTile) {
        const int nr = static_cast<int>(min(static_cast<int64_t>(kOlsTile), r1 - base));
        __syncthreads();
        // stage the tile's columns (and y) coalesced: column by column for
        // column-major data, row by row for row-major data (the cluster scores)
        if (row_major) {
            for (int i = tid; i < m.P * kOlsTile; i += kOlsThreads) {
                const int r = i / m.P, col = i - r * m.P;
                double v = 0.0;
                if (r < nr) {
                    const int64_t row = base + r;
                    v = col < m.p ? m.X[col + row * m.rs] : m.y[row * m.rs];
                }
                tile[col][r] = v;
            }
        } else {
            for (int i = tid; i < m.P * kOlsTile; i += kOlsThreads) {
                const int col = i / kOlsTile, r = i - col * kOlsTile;
                double v = 0.0;
                if (r < nr) {
                    const int64_t row = m.perm ? m.perm[base + r] : base + r;
                    v = col < m.p ? m.X[static_cast<int64_t>(col) * m.cs + row * m.rs]
                                  : m.y[row * (m.mode == kMomPlain ? m.rs : 1)];
                }
                tile[col][r] = v;
            }
        }
        if (m.mode == kMomRobust || m.mode == kMomRss) {
            for (int i = tid; i < kOlsTile; i += kOlsThreads) tile[m.p][i] = 0.0;
        }
        __syncthreads();
        // per-row factors (and residuals in the robust mode)
        if (tid < kOlsTile) {
            double f = 0.0;
            if (tid < nr) {
                const int64_t row = m.perm ? m.perm[base + tid] : base + tid;
                const double wr = m.w ? m.w[row] : 1.0;
                if (m.mode == kMomRobust || m.mode == kMomRss) {
                    double fit = 0.0;
                    for (int j = 0; j < m.p; ++j) fit = fma(tile[j][tid], m.beta[j], fit);
                    const double e = m.y[row] - fit;
                    rss = fma(wr * e, e, rss);
                    f = m.wfreq ? wr * e * e : (wr * e) * (wr * e);
                } else if (m.mode == kMomGram) {
                    f = wr;
                } else {
                    f = 1.0;
                }
            }
            fac[tid] = f;
        }
        __syncthreads();
        if (m.mode == kMomRss) continue;
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            if (pa[u] < 0) continue;
            const double* ca = tile[pa[u]];
            const double* cb = tile[pb[u]];
            double s = acc[u];
            for (int r = slice; r < nr; r += R) s = fma(fac[r] * ca[r], cb[r], s);
            acc[u] = s;
        }
    }
    if (R > 1) {
        __syncthreads();
        red[tid] = pa[0] >= 0 ? acc[0] : 0.0;
        __syncthreads();
        if (tid < npairs) {
            double t = 0.0;
            for (int sl = 0; sl < R; ++sl) t += red[sl * npairs + tid];
            m.partial[static_cast<int64_t>(blockIdx.x) * npairs + tid] = t;
        }
    } else {
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int t = tid + u * kOlsThreads;
            if (t < npairs) m.partial[static_cast<int64_t>(blockIdx.x) * npairs + t] = acc[u];
        }
    }
    if (m.rss_partial) {
        __syncthreads();
        red[tid] = rss;
        __syncthreads();
        if (tid == 0) {
            double sacc = 0.0;
            for (int i = 0; i < kOlsTile; ++i) sacc += red[i];
            m.rss_partial[blockIdx.x] = sacc;
        }
    }
}

// sum of CTA partials in CTA order, one thread per entry
__global__ void partial_sum_kernel(const double* __restrict__ partial, int nparts, int width,
                                   double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < width; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nparts; ++b) s += partial[static_cast<int64_t>(b) * width + i];
        out[i] = s;
    }
}

struct ClusterArgs {
    int64_t nchunks;
    const int32_t* chunk_grp;   // cluster of each chunk
    const int32_t* chunk_beg;   // [nchunks] positions in cluster order
    const int32_t* chunk_end;
    const uint8_t* chunk_whole; // the cluster's only chunk
    const int32_t* perm;        // cluster order -> row (null: identity)
    int p;
    const double* X;
    int64_t ld;
    const double* y;
    const double* w;
    double beta[kOlsMaxP];
    double* scores;             // [G][p + 1]: sum w e x_j, then sum w e
    double* chunk_part;         // [nchunks][p + 1]
    int32_t small_max;          // whole-cluster chunks this short go to cluster_small_kernel
};

// One warp per chunk: lane l takes rows l, l + 32, ... of the chunk, then the
// lanes' sums are combined by a fixed shuffle tree.
__global__ void __launch_bounds__(kOlsThreads)
cluster_chunk_kernel(const ClusterArgs c) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (kOlsThreads / 32);
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * (kOlsThreads / 32) + (threadIdx.x >> 5);
         k < c.nchunks; k += nwarps) {
        if (c.chunk_whole[k] && c.chunk_end[k] - c.chunk_beg[k] <= c.small_max) continue;
        double s[kOlsMaxP + 1];
#pragma unroll
        for (int j = 0; j <= kOlsMaxP; ++j) s[j] = 0.0;
        for (int32_t r = c.chunk_beg[k] + lane; r < c.chunk_end[k]; r += 32) {
            const int64_t row = c.perm ? c.perm[r] : r;
            double fit = 0.0;
            for (int j = 0; j < c.p; ++j) fit = fma(c.X[static_cast<int64_t>(j) * c.ld + row], c.beta[j], fit);
            const double wr = c.w ? c.w[row] : 1.0;
            const double we = wr * (c.y[row] - fit);
#pragma unroll
            for (int j = 0; j < kOlsMaxP; ++j)
                if (j < c.p) s[j] = fma(we, c.X[static_cast<int64_t>(j) * c.ld + row], s[j]);
            s[kOlsMaxP] += we;
        }
#pragma unroll
        for (int j = 0; j <= kOlsMaxP; ++j) {
            if (j < c.p || j == kOlsMaxP) {
                double v = s[j];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                s[j] = v;
            }
        }
        if (lane == 0) {
            double* dst = c.chunk_whole[k] ? c.scores + static_cast<int64_t>(c.chunk_grp[k]) * (c.p + 1)
                                           : c.chunk_part + k * (c.p + 1);
#pragma unroll
            for (int j = 0; j < kOlsMaxP; ++j)
                if (j < c.p) dst[j] = s[j];
            dst[c.p] = s[kOlsMaxP];
        }
    }
}

// Clusters of at most small_max rows (and empty ones): one thread per cluster
// walks its rows in cluster order; an empty cluster gets zero scores.
__global__ void __launch_bounds__(kOlsThreads)
cluster_small_kernel(const ClusterArgs c, const int32_t* __restrict__ off, int32_t G) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = off[g], e = off[g + 1];
        if (e - b > c.small_max) continue;
        double s[kOlsMaxP + 1];
#pragma unroll
        for (int j = 0; j <= kOlsMaxP; ++j) s[j] = 0.0;
        for (int32_t r = b; r < e; ++r) {
            const int64_t row = c.perm ? c.perm[r] : r;
            double fit = 0.0;
            for (int j = 0; j < c.p; ++j) fit = fma(c.X[static_cast<int64_t>(j) * c.ld + row], c.beta[j], fit);
            const double wr = c.w ? c.w[row] : 1.0;
            const double we = wr * (c.y[row] - fit);
#pragma unroll
            for (int j = 0; j < kOlsMaxP; ++j)
                if (j < c.p) s[j] = fma(we, c.X[static_cast<int64_t>(j) * c.ld + row], s[j]);
            s[kOlsMaxP] += we;
        }
        double* dst = c.scores + g * (c.p + 1);
#pragma unroll
        for (int j = 0; j < kOlsMaxP; ++j)
            if (j < c.p) dst[j] = s[j];
        dst[c.p] = s[kOlsMaxP];
    }
}

// clusters the per-thread kernel takes get no chunks
__global__ void drop_small_chunks_kernel(const int32_t* __restrict__ off, int32_t G,
                                         int32_t small_max, int32_t* __restrict__ nch) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (off[g + 1] - off[g] <= small_max) nch[g] = 0;
}

// clusters of several chunks: chunk sums in chunk order
__global__ void cluster_combine_kernel(int64_t nmulti, const int32_t* __restrict__ multi_grp,
                                       const int32_t* __restrict__ multi_c0,
                                       const int32_t* __restrict__ multi_c1,
                                       const double* __restrict__ chunk_part, int width,
                                       double* __restrict__ scores) {
    const int64_t total = nmulti * width;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t r = i / width;
        const int j = static_cast<int>(i - r * width);
        double s = 0.0;
        for (int32_t k = multi_c0[r]; k < multi_c1[r]; ++k) s += chunk_part[static_cast<int64_t>(k) * width + j];
        scores[static_cast<int64_t>(multi_grp[r]) * width + j] = s;
    }
}

}  // namespace b200fe
