// Absorption with heterogeneous slopes: the FE space of a dimension d is
// spanned per group g by the intercept 1_g, the slope z_d 1_g, or both
// (the reference's HeterogeneousSlopeTerm, include/fe_absorption.hpp:49-53;
// GpuFeInput.is_slope / slope_has_intercept / slope_values,
// include/fe_absorption_cuda.hpp:12-22).  The within transform is the
// W-orthogonal residual of every column on the sum of those spaces.
//
// Solver: CG on the normal equations in residual form (CGLS), all columns in
// lock step, preconditioned by the exact per-group block inverse of every
// dimension (block Jacobi = additive Schwarz over the FE blocks).  A group's
// 2x2 block [W Z; Z ZZ] (W = sum w, Z = sum w z, ZZ = sum w z^2) is inverted
// with the reference's determinant rule (compute_slope_coefficients_kernel,
// src/fe_absorption_cuda.cu:586-650): det > 1e-12 max(1, W ZZ), otherwise the
// group keeps its intercept only; a slope without intercept needs
// ZZ > 1e-12 max(1, ZZ).  FP64 throughout.
//
// Layout (observations in the order of the primary dimension, the one with
// the most groups):
//   R, Q      [n][C] row-major FP64: residual and the search image D p
//   ids_d     [n]   group of every observation in dimension d
//   z_d       [n]   slope values (slope dims)
//   perm_d    [n]   positions sorted by ids_d (stable); null for the primary
//   chunks    per dim: ranges of <= ceil(len / nch) positions of one group,
//             nch <= 4096 per group; a group of more than 32 chunks has its
//             chunk sums pre-reduced by one warp (slope_big_reduce_kernel)
//   coefficients per dim [G][nb][C]: block 0 the intercept (if any), then the
//             slope (if any)
// Every sum is taken in a fixed order (chunk, then lane slots, then chunks in
// group order, then CTAs in order), so results are bitwise reproducible.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200fe {

constexpr int kSlopeThreads = 256;
constexpr int kSlopeChunkRows = 64;   // minimum rows per chunk
constexpr int kSlopeMaxChunks = 4096; // chunks per group at most
constexpr int kSlopeMaxCols = 256;
constexpr double kSlopeDetTol = 1e-12;
constexpr int kSlopeMaxDims = 9;  // 8 FE dimensions + the individual dimension
constexpr int kFinSerialChunks = 32;  // more chunk partials: a warp sums them first

struct SlopeDim {
    const int32_t* ids;     // [n] group per observation (primary order)
    const double* z;        // [n] slope values or null
    const int32_t* perm;    // [n] sorted positions or null (identity)
    const int32_t* ch_beg;  // [nch] chunk ranges in sorted positions
    const int32_t* ch_end;
    const int32_t* grp_ch;  // [G + 1] first chunk of every group
    const double* minv;     // [G][3] block inverse (m00, m01, m11)
    double* part;           // [nch][nb][C] chunk sums
    double* zv;             // [G][nb][C] preconditioned gradient
    double* p;              // [G][nb][C] search direction
    double* big;            // [G][nb][C] chunk sums of groups with many chunks, or null
    int32_t G;
    int32_t nch;
    int has_a, has_b, nb;
};

// ---------------------------------------------------------------------------
// Setup: chunk ranges and per-group moments
// ---------------------------------------------------------------------------

// number of chunks of every group (0 for an empty group)
__global__ void slope_chunk_count_kernel(const int32_t* __restrict__ off, int32_t G,
                                         int32_t* __restrict__ nch) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g <= G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (g == G) {
            nch[g] = 0;
            continue;
        }
        const int32_t len = off[g + 1] - off[g];
        int32_t c = (len + kSlopeChunkRows - 1) / kSlopeChunkRows;
        nch[g] = min(c, kSlopeMaxChunks);
    }
}

__global__ void slope_chunk_fill_kernel(const int32_t* __restrict__ off, int32_t G,
                                        const int32_t* __restrict__ grp_ch,
                                        int32_t* __restrict__ ch_beg, int32_t* __restrict__ ch_end,
                                        int32_t* __restrict__ ch_grp) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = off[g], e = off[g + 1];
        const int32_t c0 = grp_ch[g], nc = grp_ch[g + 1] - c0;
        if (nc == 0) continue;
        const int32_t L = (e - b + nc - 1) / nc;
        for (int32_t i = 0; i < nc; ++i) {
            ch_beg[c0 + i] = min(e, b + i * L);
            ch_end[c0 + i] = min(e, b + (i + 1) * L);
            if (ch_grp) ch_grp[c0 + i] = static_cast<int32_t>(g);
        }
    }
}

// Per chunk: sum w, sum w z, sum w z^2, sum w^2, sum w^2 z^2 over its rows,
// one warp per chunk (lanes stride the rows, fixed shuffle tree).
__global__ void __launch_bounds__(kSlopeThreads)
slope_moments_kernel(const SlopeDim d, const double* __restrict__ w, double* __restrict__ cm) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = static_cast<int64_t>(gridDim.x) * (kSlopeThreads / 32);
    for (int64_t j = static_cast<int64_t>(blockIdx.x) * (kSlopeThreads / 32) + (threadIdx.x >> 5);
         j < d.nch; j += nw) {
        double m[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int32_t pos = d.ch_beg[j] + lane; pos < d.ch_end[j]; pos += 32) {
            const int32_t k = d.perm ? d.perm[pos] : pos;
            const double wk = w ? w[k] : 1.0;
            const double zk = d.z ? d.z[k] : 0.0;
            m[0] += wk;
            m[1] = fma(wk, zk, m[1]);
            m[2] = fma(wk * zk, zk, m[2]);
            m[3] = fma(wk, wk, m[3]);
            m[4] = fma(wk * zk, wk * zk, m[4]);
        }
#pragma unroll
        for (int u = 0; u < 5; ++u) {
            double v = m[u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            m[u] = v;
        }
        if (lane == 0) {
#pragma unroll
            for (int u = 0; u < 5; ++u) cm[j * 5 + u] = m[u];
        }
    }
}

// Per group: combine the chunk moments in chunk order, form the block inverse
// and the group's share of ||D'W||_F^2 (sum of the squared multipliers w and
// w z of its basis columns); CTA partials of the latter in part_op[block].
__global__ void __launch_bounds__(kSlopeThreads)
slope_block_inverse_kernel(const SlopeDim d, const double* __restrict__ cm,
                           double* __restrict__ minv, double* __restrict__ part_op) {
    __shared__ double red[kSlopeThreads];
    double op = 0.0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < d.G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double m[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int32_t j = d.grp_ch[g]; j < d.grp_ch[g + 1]; ++j)
#pragma unroll
            for (int u = 0; u < 5; ++u) m[u] += cm[static_cast<int64_t>(j) * 5 + u];
        const double W = m[0], Z = m[1], ZZ = m[2];
        double m00 = 0.0, m01 = 0.0, m11 = 0.0;
        if (d.has_a && d.has_b) {
            if (W > 0.0) {
                const double det = W * ZZ - Z * Z;
                const double scale = fmax(1.0, W * ZZ);
                if (det > kSlopeDetTol * scale) {
                    m00 = ZZ / det;
                    m01 = -Z / det;
                    m11 = W / det;
                } else {
                    m00 = 1.0 / W;
                }
            }
        } else if (d.has_a) {
            if (W > 0.0) m00 = 1.0 / W;
        } else {
            const double scale = fmax(1.0, ZZ);
            if (ZZ > kSlopeDetTol * scale) m11 = 1.0 / ZZ;
        }
        minv[g * 3 + 0] = m00;
        minv[g * 3 + 1] = m01;
        minv[g * 3 + 2] = m11;
        op += (d.has_a ? m[3] : 0.0) + (d.has_b ? m[4] : 0.0);
    }
    red[threadIdx.x] = op;
    __syncthreads();
    for (int s = kSlopeThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part_op[blockIdx.x] = red[0];
}

// R[k][c] = v[c * n + pord[k]] (row-major in primary order)
__global__ void slope_load_kernel(const double* __restrict__ v, const int32_t* __restrict__ pord,
                                  int64_t n, int C, double* __restrict__ R) {
    const int64_t total = n * C;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = e / C;
        const int c = static_cast<int>(e - k * C);
        const int64_t src = pord ? pord[k] : k;
        R[e] = v[static_cast<int64_t>(c) * n + src];
    }
}

// out[c * n + pord[k]] = R[k][c]
__global__ void slope_store_kernel(const double* __restrict__ R, const int32_t* __restrict__ pord,
                                   int64_t n, int C, double* __restrict__ out) {
    const int64_t total = n * C;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = e / C;
        const int c = static_cast<int>(e - k * C);
        const int64_t dst = pord ? pord[k] : k;
        out[static_cast<int64_t>(c) * n + dst] = R[e];
    }
}

// flags[3] |= 1 when a slope value is not finite
__global__ void finite_values_kernel(const double* __restrict__ z, int64_t n, int* flags) {
    int bad = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        bad |= !(fabs(z[i]) <= 1.7976931348623157e308);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags + 3, 1);
}

// ---------------------------------------------------------------------------
// Column-wise CTA reduction for element kernels whose block holds RB rows of
// C columns (thread t owns column t % C for the whole grid-stride loop).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void column_reduce(double* red, double v, int C, int RB, double* out) {
    red[threadIdx.x] = v;
    __syncthreads();
    if (static_cast<int>(threadIdx.x) < C) {
        double s = 0.0;
        for (int r = 0; r < RB; ++r) s += red[r * C + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// per column, CTA partials of sum w r^2 and sum r^2 (the norms of the input)
__global__ void __launch_bounds__(kSlopeThreads)
slope_norms_kernel(const double* __restrict__ R, const double* __restrict__ w, int64_t n, int C,
                   int RB, double* __restrict__ part_w, double* __restrict__ part_u) {
    __shared__ double red[kSlopeThreads];
    const int col = threadIdx.x % C, rr = threadIdx.x / C;
    double aw = 0.0, au = 0.0;
    if (rr < RB) {
        for (int64_t k = static_cast<int64_t>(blockIdx.x) * RB + rr; k < n;
             k += static_cast<int64_t>(gridDim.x) * RB) {
            const double r = R[k * C + col];
            const double wk = w ? w[k] : 1.0;
            aw = fma(wk * r, r, aw);
            au = fma(r, r, au);
        }
    }
    column_reduce(red, aw, C, RB, part_w + static_cast<int64_t>(blockIdx.x) * C);
    column_reduce(red, au, C, RB, part_u + static_cast<int64_t>(blockIdx.x) * C);
}

// The individual dimension of a group/individual design (the reference's
// GroupIndividualStructure, include/fe_absorption.hpp:13-21): observation k
// (a group) holds the individuals ind[beg[k] .. end[k]), and the basis column
// of individual i is scale_k at every group k that holds i.
struct GiRows {
    const int32_t* beg;   // [n] first edge of every row (primary order)
    const int32_t* end;   // [n]
    const int32_t* ind;   // [E] individual of every edge (group-major)
    const double* scale;  // [n] group scale (primary order)
    const double* p;      // [I][C] search direction of the individual dim
};

struct SlopeGatherArgs {
    int nd;
    SlopeDim dim[8];
    int has_gi;
    GiRows gi;
    int64_t n;
    int C, RB;
    const double* w;
    double* Q;
    double* part;  // [grid][C] sums of w q^2
};

// Q = D p, with CTA partials of q' W q per column.  ND > 0 unrolls the
// dimension loop (descriptors load once), ND == 0 loops over a.nd.
template <int ND>
__global__ void __launch_bounds__(kSlopeThreads)
slope_gather_kernel(const SlopeGatherArgs a) {
    __shared__ double red[kSlopeThreads];
    const int C = a.C;
    const int col = threadIdx.x % C, rr = threadIdx.x / C;
    double acc = 0.0;
    if (rr < a.RB) {
        for (int64_t k = static_cast<int64_t>(blockIdx.x) * a.RB + rr; k < a.n;
             k += static_cast<int64_t>(gridDim.x) * a.RB) {
            double q = 0.0;
#pragma unroll
            for (int d = 0; d < (ND > 0 ? ND : 8); ++d) {
                if (ND == 0 && d >= a.nd) break;
                const SlopeDim& D = a.dim[d];
                const int64_t base = (static_cast<int64_t>(D.ids[k]) * D.nb) * C + col;
                if (D.has_a) q += D.p[base];
                if (D.has_b) q = fma(D.z[k], D.p[base + (D.has_a ? C : 0)], q);
            }
            if (a.has_gi) {
                double t = 0.0;
                for (int32_t e = a.gi.beg[k]; e < a.gi.end[k]; ++e)
                    t += a.gi.p[static_cast<int64_t>(a.gi.ind[e]) * C + col];
                q = fma(a.gi.scale[k], t, q);
            }
            a.Q[k * C + col] = q;
            const double wk = a.w ? a.w[k] : 1.0;
            acc = fma(wk * q, q, acc);
        }
    }
    column_reduce(red, acc, C, a.RB, a.part + static_cast<int64_t>(blockIdx.x) * C);
}

// alpha_c = gamma_c / (q' W q)_c for the columns still iterating; the dots
// come as CTA partials of one or two kernels, summed in order
__global__ void slope_alpha_kernel(const double* __restrict__ part, int nparts,
                                   const double* __restrict__ part2, int nparts2, int C,
                                   const double* __restrict__ gamma, const int* __restrict__ active,
                                   double* __restrict__ alpha) {
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        double dl = 0.0;
        for (int b = 0; b < nparts; ++b) dl += part[static_cast<int64_t>(b) * C + c];
        for (int b = 0; b < nparts2; ++b) dl += part2[static_cast<int64_t>(b) * C + c];
        alpha[c] = (active[c] && dl > 0.0) ? gamma[c] / dl : 0.0;
    }
}

struct SlopeSegArgs {
    SlopeDim d;
    int C;
    int slots;           // rows a warp takes per step (32 / C for C <= 32, else 1)
    double* R;
    const double* Q;     // null: no update (the first gradient)
    const double* alpha; // [C]
    const double* w;
    int write;           // store the updated residual (the primary dim only)
};

// Chunk sums of w r and w z r per column, r = R - alpha Q (stored back by the
// writer).  One warp per chunk.  For C <= 32 the lanes form `slots` row slots
// of C columns; for C > 32 lane l owns columns l, l + 32, ... (CW of them).
template <int CW>
__global__ void __launch_bounds__(kSlopeThreads)
slope_segment_kernel(const SlopeSegArgs a) {
    __shared__ double sred[kSlopeThreads / 32][2][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int C = a.C;
    const SlopeDim& D = a.d;
    const int S = a.slots;
    const int slot = CW == 1 ? lane / C : 0;
    const int col0 = CW == 1 ? lane - slot * C : lane;
    const bool live = CW == 1 ? slot < S : true;
    double al[CW];
#pragma unroll
    for (int u = 0; u < CW; ++u) {
        const int c = col0 + 32 * u;
        al[u] = (a.Q && live && c < C) ? a.alpha[c] : 0.0;
    }
    const int64_t nw = static_cast<int64_t>(gridDim.x) * (kSlopeThreads / 32);
    for (int64_t j = static_cast<int64_t>(blockIdx.x) * (kSlopeThreads / 32) + wid; j < D.nch;
         j += nw) {
        double sa[CW], sb[CW];
#pragma unroll
        for (int u = 0; u < CW; ++u) sa[u] = sb[u] = 0.0;
        if (live) {
            const int32_t e = D.ch_end[j];
            for (int32_t pos = D.ch_beg[j] + slot; pos < e; pos += S) {
                const int64_t k = D.perm ? D.perm[pos] : pos;
                const double wk = a.w ? a.w[k] : 1.0;
                const double zk = D.has_b ? D.z[k] : 0.0;
#pragma unroll
                for (int u = 0; u < CW; ++u) {
                    const int c = col0 + 32 * u;
                    if (c < C) {
                        double r = a.R[k * C + c];
                        if (a.Q) r = fma(-al[u], a.Q[k * C + c], r);
                        if (a.write) a.R[k * C + c] = r;
                        const double wr = wk * r;
                        sa[u] += wr;
                        sb[u] = fma(wr, zk, sb[u]);
                    }
                }
            }
        }
        double* out = D.part + (j * D.nb) * C;
        if (CW == 1) {
            // combine the row slots in slot order
            sred[wid][0][lane] = sa[0];
            sred[wid][1][lane] = sb[0];
            __syncwarp();
            if (lane < C) {
                double ta = 0.0, tb = 0.0;
                for (int s = 0; s < S; ++s) {
                    ta += sred[wid][0][s * C + lane];
                    tb += sred[wid][1][s * C + lane];
                }
                if (D.has_a) out[lane] = ta;
                if (D.has_b) out[(D.has_a ? C : 0) + lane] = tb;
            }
            __syncwarp();
        } else {
#pragma unroll
            for (int u = 0; u < CW; ++u) {
                const int c = col0 + 32 * u;
                if (c < C) {
                    if (D.has_a) out[c] = sa[u];
                    if (D.has_b) out[(D.has_a ? C : 0) + c] = sb[u];
                }
            }
        }
    }
}

// Per group and column: the gradient s (chunk sums in chunk order), the
// preconditioned gradient zv = M^-1 s, and CTA partials of s'zv (gamma) and
// s's (the certificate's ||D'W r||^2).
__global__ void __launch_bounds__(kSlopeThreads)
slope_finalize_kernel(SlopeDim d, int C, int RB, double* __restrict__ part_g,
                      double* __restrict__ part_n) {
    __shared__ double red[kSlopeThreads];
    const int col = threadIdx.x % C, rr = threadIdx.x / C;
    double ag = 0.0, an = 0.0;
    if (rr < RB) {
        for (int64_t g = static_cast<int64_t>(blockIdx.x) * RB + rr; g < d.G;
             g += static_cast<int64_t>(gridDim.x) * RB) {
            double sa = 0.0, sb = 0.0;
            if (d.big && d.grp_ch[g + 1] - d.grp_ch[g] > kFinSerialChunks) {
                // summed by slope_big_reduce_kernel
                const double* bj = d.big + (g * d.nb) * C + col;
                if (d.has_a) sa = bj[0];
                if (d.has_b) sb = bj[d.has_a ? C : 0];
            } else {
                for (int32_t j = d.grp_ch[g]; j < d.grp_ch[g + 1]; ++j) {
                    const double* pj = d.part + (static_cast<int64_t>(j) * d.nb) * C + col;
                    if (d.has_a) sa += pj[0];
                    if (d.has_b) sb += pj[d.has_a ? C : 0];
                }
            }
            const double m00 = d.minv[g * 3 + 0], m01 = d.minv[g * 3 + 1], m11 = d.minv[g * 3 + 2];
            double* zg = d.zv + (g * d.nb) * C + col;
            if (d.has_a && d.has_b) {
                const double za = fma(m00, sa, m01 * sb);
                const double zb = fma(m01, sa, m11 * sb);
                zg[0] = za;
                zg[C] = zb;
                ag = fma(sa, za, fma(sb, zb, ag));
            } else if (d.has_a) {
                const double za = m00 * sa;
                zg[0] = za;
                ag = fma(sa, za, ag);
            } else {
                const double zb = m11 * sb;
                zg[0] = zb;
                ag = fma(sb, zb, ag);
            }
            an = fma(sa, sa, fma(sb, sb, an));
        }
    }
    column_reduce(red, ag, C, RB, part_g + static_cast<int64_t>(blockIdx.x) * C);
    column_reduce(red, an, C, RB, part_n + static_cast<int64_t>(blockIdx.x) * C);
}

struct SlopeBetaArgs {
    int nd, C;
    int grid[kSlopeMaxDims]; // finalize CTAs per dim
    int64_t stride;          // partial slots per dim
    const double* part_g;    // [nd][stride][C]
    const double* part_n;
    const double* thr;       // [C] stop threshold on gamma
    double* gamma;           // [C]
    double* beta;            // [C]
    double* nu;              // [C] ||D'W r||^2 at the last gradient
    int* active;             // [C]
    int* done;               // all columns stopped
    int init;
};

// One CTA: gamma_new = sum over dims and CTAs (fixed order), beta, stop test.
__global__ void slope_beta_kernel(const SlopeBetaArgs a) {
    int any = 0;
    for (int c = threadIdx.x; c < a.C; c += blockDim.x) {
        double g = 0.0, nu = 0.0;
        for (int d = 0; d < a.nd; ++d)
            for (int b = 0; b < a.grid[d]; ++b) {
                const int64_t o = (d * a.stride + b) * a.C + c;
                g += a.part_g[o];
                nu += a.part_n[o];
            }
        a.nu[c] = nu;
        if (a.init) {
            a.gamma[c] = g;
            a.beta[c] = 0.0;
            a.active[c] = g > a.thr[c] ? 1 : 0;
        } else if (a.active[c]) {
            a.beta[c] = a.gamma[c] > 0.0 ? g / a.gamma[c] : 0.0;
            a.gamma[c] = g;
            if (!(g > a.thr[c])) a.active[c] = 0;
        } else {
            a.beta[c] = 0.0;
        }
        any |= a.active[c];
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) *a.done = any ? 0 : 1;
}

// R -= alpha Q (designs without an FE dimension that covers every row once)
__global__ void slope_update_kernel(double* __restrict__ R, const double* __restrict__ Q,
                                    const double* __restrict__ alpha, int64_t n, int C) {
    const int64_t total = n * C;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        R[e] = fma(-alpha[e % C], Q[e], R[e]);
}

// inv[ord[k]] = k
__global__ void inverse_perm_kernel(const int32_t* __restrict__ ord, int64_t n,
                                    int32_t* __restrict__ inv) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        inv[ord[k]] = static_cast<int32_t>(k);
}

// edge -> row position in primary order (map null: identity)
__global__ void map_rows_kernel(const int32_t* __restrict__ rows, int64_t E,
                                const int32_t* __restrict__ map, int32_t* __restrict__ out) {
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < E;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[e] = map ? map[rows[e]] : rows[e];
}

// per row in primary order: its edge range in the group-major edge list
__global__ void row_edges_kernel(const int32_t* __restrict__ gptr, const int32_t* __restrict__ pord,
                                 int64_t n, int32_t* __restrict__ beg, int32_t* __restrict__ end) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = pord ? pord[k] : k;
        beg[k] = gptr[g];
        end[k] = gptr[g + 1];
    }
}

// ---------------------------------------------------------------------------
// Schur form (the primary dimension eliminated exactly).  The CGLS runs on
// min || (I - P_p)(v - D_r a) ||_W over the other dimensions' coefficients a,
// P_p the W-projection on the primary groups' bases (segment sums in primary
// order times the groups' block inverses).  Its block-Jacobi preconditioner is the exact block diagonal of the
// Schur complement D_r' W (I - P_p) D_r: for group g of dimension d,
//   S_g = B_g - sum over primary groups j meeting g of C_jg' M_j^-1 C_jg,
// C_jg the sums over the rows in (j, g) of w times the primary basis (1, and
// the primary's slope t when it has one) times g's basis (1, z), and M_j^-1
// the primary group's block inverse (1 / W_j for a primary without slope).
// In dimension d's stable sorted order the rows of g are in primary order, so
// every pair (j, g) is one contiguous run there.
// ---------------------------------------------------------------------------
constexpr double kSchurRel = 1e-11;  // null-space test of a Schur block, relative to B

// A primary with intercept and slope is eliminated in the centred basis
// (1, t - tbar_g), tbar_g = sum w t / W_g: the same span, but a block close to
// diag(W, SS) instead of [W Z; Z ZZ], so projecting a constant off a group
// leaves rounding of order eps instead of eps * cond(M_g) -- which the CGLS,
// whose search directions reach the constants shared by the primary and the
// other dimensions' intercepts, would otherwise pump up.
__global__ void slope_group_center_kernel(const SlopeDim d, const double* __restrict__ cm,
                                          double* __restrict__ tbar) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < d.G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double W = 0.0, Z = 0.0;
        for (int32_t j = d.grp_ch[g]; j < d.grp_ch[g + 1]; ++j) {
            W += cm[static_cast<int64_t>(j) * 5];
            Z += cm[static_cast<int64_t>(j) * 5 + 1];
        }
        tbar[g] = W > 0.0 ? Z / W : 0.0;
    }
}

// zc[k] = t[k] - tbar[ids[k]] (primary order)
__global__ void slope_center_rows_kernel(const int32_t* __restrict__ ids, const double* __restrict__ t,
                                         const double* __restrict__ tbar, int64_t n,
                                         double* __restrict__ zc) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        zc[k] = t[k] - tbar[ids[k]];
}

// Block inverse in the centred basis from the centred chunk moments; the
// slope stays in a group's basis where the reference's rule kept it on the
// uncentred block (minv_u[g][2] != 0).
__global__ void slope_centred_inverse_kernel(const SlopeDim d, const double* __restrict__ cm,
                                             const double* __restrict__ minv_u,
                                             double* __restrict__ minv) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < d.G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double W = 0.0, Z = 0.0, SS = 0.0;
        for (int32_t j = d.grp_ch[g]; j < d.grp_ch[g + 1]; ++j) {
            W += cm[static_cast<int64_t>(j) * 5];
            Z += cm[static_cast<int64_t>(j) * 5 + 1];
            SS += cm[static_cast<int64_t>(j) * 5 + 2];
        }
        double m00 = W > 0.0 ? 1.0 / W : 0.0, m01 = 0.0, m11 = 0.0;
        const double det = W * SS - Z * Z;
        if (minv_u[g * 3 + 2] != 0.0 && W > 0.0 && det > 0.0) {
            m00 = SS / det;
            m01 = -Z / det;
            m11 = W / det;
        }
        minv[g * 3 + 0] = m00;
        minv[g * 3 + 1] = m01;
        minv[g * 3 + 2] = m11;
    }
}

// flag[pos] = 1 where a (primary group, group of d) pair starts in d's order
__global__ void pair_flags_kernel(const int32_t* __restrict__ perm, const int32_t* __restrict__ ids_d,
                                  const int32_t* __restrict__ ids_p, int64_t n,
                                  int32_t* __restrict__ flag) {
    for (int64_t pos = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; pos < n;
         pos += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int32_t f = 1;
        if (pos > 0) {
            const int32_t k = perm[pos], kp = perm[pos - 1];
            f = (ids_d[k] != ids_d[kp] || ids_p[k] != ids_p[kp]) ? 1 : 0;
        }
        flag[pos] = f;
    }
}

// start[pid[pos] - 1] = pos at every pair start; start[npairs] = n
__global__ void pair_start_kernel(const int32_t* __restrict__ flag, const int32_t* __restrict__ pid,
                                  int64_t n, int32_t* __restrict__ start) {
    for (int64_t pos = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; pos <= n;
         pos += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (pos == n) start[pid[n - 1]] = static_cast<int32_t>(n);
        else if (flag[pos]) start[pid[pos] - 1] = static_cast<int32_t>(pos);
    }
}

// per pair (j, g): the entries (aa, ab, bb) of C' M_j^-1 C, C[m][f] the sum over
// the pair's rows of w times the primary basis function m (1, the primary's
// slope t) times g's basis function f (1, z), M_j the primary group's block --
// (c_a^2, c_a c_b, c_b^2) / W_j for a primary without slope (three planes of
// npairs values)
__global__ void pair_contrib_kernel(const SlopeDim d, const SlopeDim P,
                                    const double* __restrict__ w,
                                    const int32_t* __restrict__ start, int64_t npairs,
                                    double* __restrict__ contrib) {
    for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < npairs;
         q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double ca = 0.0, cb = 0.0, ta = 0.0, tb = 0.0;  // rows 1 and t of C
        const int32_t b = start[q], e = start[q + 1];
        for (int32_t pos = b; pos < e; ++pos) {
            const int32_t k = d.perm[pos];
            const double wk = w ? w[k] : 1.0;
            const double wz = d.has_b ? wk * d.z[k] : 0.0;
            ca += wk;
            cb += wz;
            if (P.has_b) {
                ta = fma(wk, P.z[k], ta);
                tb = fma(wz, P.z[k], tb);
            }
        }
        const double* mj = P.minv + static_cast<int64_t>(P.ids[d.perm[b]]) * 3;
        if (!P.has_b) {
            contrib[q] = ca * ca * mj[0];
            contrib[npairs + q] = ca * cb * mj[0];
            contrib[2 * npairs + q] = cb * cb * mj[0];
        } else {
            // u' M v for the columns u, v of C
            auto qf = [&](double u0, double u1, double v0, double v1) {
                return mj[0] * u0 * v0 + mj[1] * (u0 * v1 + u1 * v0) + mj[2] * u1 * v1;
            };
            contrib[q] = qf(ca, ta, ca, ta);
            contrib[npairs + q] = qf(ca, ta, cb, tb);
            contrib[2 * npairs + q] = qf(cb, tb, cb, tb);
        }
    }
}

// first pair of every group of d (groups own contiguous pair ranges; an empty
// group gets the next group's first pair)
__global__ void pair_offsets_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ pid,
                                    int32_t G, int64_t n, int32_t npairs,
                                    int32_t* __restrict__ pair_off) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g <= G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)
        pair_off[g] = off[g] < n ? pid[off[g]] - 1 : npairs;
}

// Block inverse of the Schur block of every group (pseudo-inverse on the
// null space: a block whose projected intercept or slope vanishes against its
// unprojected size keeps the other direction; a slope the reference's rule
// drops from the basis stays dropped), and the group's share of ||D'W||_F^2.
__global__ void __launch_bounds__(kSlopeThreads)
schur_block_inverse_kernel(const SlopeDim d, const double* __restrict__ cm,
                           const double* __restrict__ csum, double* __restrict__ minv,
                           double* __restrict__ part_op) {
    __shared__ double red[kSlopeThreads];
    double op = 0.0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < d.G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double m[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int32_t j = d.grp_ch[g]; j < d.grp_ch[g + 1]; ++j)
#pragma unroll
            for (int u = 0; u < 5; ++u) m[u] += cm[static_cast<int64_t>(j) * 5 + u];
        const double W = m[0], Z = m[1], ZZ = m[2];
        // csum: per group the sums of the three pair planes (segmented reduce)
        const double s11 = W - csum[g], s12 = Z - csum[d.G + g], s22 = ZZ - csum[2 * static_cast<int64_t>(d.G) + g];
        bool slope_in = false;  // the reference's basis rule on the unprojected block
        if (d.has_a && d.has_b)
            slope_in = W > 0.0 && W * ZZ - Z * Z > kSlopeDetTol * fmax(1.0, W * ZZ);
        else if (d.has_b)
            slope_in = ZZ > kSlopeDetTol * fmax(1.0, ZZ);
        const bool a_ok = d.has_a && W > 0.0 && s11 > kSchurRel * W;
        const bool b_ok = slope_in && s22 > kSchurRel * ZZ;
        double m00 = 0.0, m01 = 0.0, m11 = 0.0;
        const double det = s11 * s22 - s12 * s12;
        if (a_ok && b_ok && det > kSchurRel * W * ZZ) {
            m00 = s22 / det;
            m01 = -s12 / det;
            m11 = s11 / det;
        } else if (a_ok) {
            m00 = 1.0 / s11;
        } else if (b_ok) {
            m11 = 1.0 / s22;
        }
        minv[g * 3 + 0] = m00;
        minv[g * 3 + 1] = m01;
        minv[g * 3 + 2] = m11;
        op += (d.has_a ? m[3] : 0.0) + (d.has_b ? m[4] : 0.0);
    }
    red[threadIdx.x] = op;
    __syncthreads();
    for (int st = kSlopeThreads / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) part_op[blockIdx.x] = red[0];
}

// X[k][c] -= the fit of row k on its primary group's basis (the group's
// weighted mean, or intercept + slope t_k; P.zv[g] holds M_g^-1 B_g' W x), with
// CTA partials of sum w x^2 per column when part is not null.
__global__ void __launch_bounds__(kSlopeThreads)
slope_project_kernel(double* __restrict__ X, const SlopeDim P, const double* __restrict__ w,
                     int64_t n, int C, int RB, double* __restrict__ part) {
    __shared__ double red[kSlopeThreads];
    const int col = threadIdx.x % C, rr = threadIdx.x / C;
    double acc = 0.0;
    if (rr < RB) {
        for (int64_t k = static_cast<int64_t>(blockIdx.x) * RB + rr; k < n;
             k += static_cast<int64_t>(gridDim.x) * RB) {
            const double* zg = P.zv + (static_cast<int64_t>(P.ids[k]) * P.nb) * C + col;
            double fit = P.has_a ? zg[0] : 0.0;
            if (P.has_b) fit = fma(P.z[k], zg[P.has_a ? C : 0], fit);
            const double x = X[k * C + col] - fit;
            X[k * C + col] = x;
            const double wk = w ? w[k] : 1.0;
            acc = fma(wk * x, x, acc);
        }
    }
    if (part) column_reduce(red, acc, C, RB, part + static_cast<int64_t>(blockIdx.x) * C);
}

// ---------------------------------------------------------------------------
// Schur-form image Q = (I - P_p) D_r p in one pass for the primary groups held
// by a single chunk (every primary group of at most 64 rows): a warp forms the
// rows of D_r p, sums w q per column over the group, and forms the rows again
// (the same loads, the same order, so the same values) to store q - mean and
// accumulate q' W q.  Rows of groups spread over several chunks are stored
// raw with their chunk sums, and schur_fix_mean_kernel /
// schur_fix_apply_kernel finish them.
// ---------------------------------------------------------------------------
struct SchurGatherArgs {
    int nd;
    SlopeDim dim[8];          // the CG dimensions (all but the primary)
    const int32_t* ch_beg;    // primary chunks
    const int32_t* ch_end;
    const int32_t* ch_grp;    // primary chunk -> group
    const int32_t* grp_ch;    // primary group -> first chunk
    const double* minv_p;     // [Gp][3] block inverse of the primary groups
    const double* z_p;        // [n] the primary's slope values, or null
    int p_has_a, p_has_b, p_nb;
    int32_t nch;
    double* part_p;           // [nch][p_nb][C] sums of w q (and w t q) of multi-chunk groups' chunks
    int64_t n;
    int C, slots;
    const double* w;
    double* Q;
    double* dpart;            // [grid][C] sums of w q'^2 of the single-chunk groups
};

// (D_r p)_k for column c; ND > 0 unrolls the dimension loop (the
// descriptors then load once per kernel), ND == 0 loops over a.nd
template <int ND>
__device__ __forceinline__ double schur_q(const SchurGatherArgs& a, int64_t k, int c) {
    double q = 0.0;
#pragma unroll
    for (int d = 0; d < (ND > 0 ? ND : 8); ++d) {
        if (ND == 0 && d >= a.nd) break;
        const SlopeDim& D = a.dim[d];
        const int64_t base = (static_cast<int64_t>(D.ids[k]) * D.nb) * a.C + c;
        if (D.has_a) q += D.p[base];
        if (D.has_b) q = fma(D.z[k], D.p[base + (D.has_a ? a.C : 0)], q);
    }
    return q;
}

template <int CW, int ND>
__global__ void __launch_bounds__(kSlopeThreads)
schur_gather_kernel(const SchurGatherArgs a) {
    constexpr int kSchurRows = CW == 1 ? 8 : (CW == 2 ? 4 : (CW == 4 ? 2 : 1));
    __shared__ double sred[kSlopeThreads / 32][32];
    __shared__ double tred[kSlopeThreads / 32][32];
    __shared__ double dred[kSlopeThreads / 32][32 * CW];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int C = a.C;
    const int S = a.slots;
    const int slot = CW == 1 ? lane / C : 0;
    const int col0 = CW == 1 ? lane - slot * C : lane;
    const bool live = CW == 1 ? slot < S : true;
    double dacc[CW];
#pragma unroll
    for (int u = 0; u < CW; ++u) dacc[u] = 0.0;
    const int64_t nw = static_cast<int64_t>(gridDim.x) * (kSlopeThreads / 32);
    for (int64_t j = static_cast<int64_t>(blockIdx.x) * (kSlopeThreads / 32) + wid; j < a.nch;
         j += nw) {
        const int32_t b = a.ch_beg[j], e = a.ch_end[j], g = a.ch_grp[j];
        const bool single = a.grp_ch[g + 1] - a.grp_ch[g] == 1;
        double sw[CW], st[CW];  // sums of w q and of w t q (t: the primary's slope values)
#pragma unroll
        for (int u = 0; u < CW; ++u) sw[u] = st[u] = 0.0;
        // the lane's first kSchurRows rows: formed together (their loads in
        // flight at once) and kept in registers for the second phase
        double qc[kSchurRows][CW];
        if (live) {
#pragma unroll
            for (int t = 0; t < kSchurRows; ++t) {
                const int32_t pos = b + slot + t * S;
#pragma unroll
                for (int u = 0; u < CW; ++u) {
                    const int c = col0 + 32 * u;
                    qc[t][u] = (pos < e && c < C) ? schur_q<ND>(a, pos, c) : 0.0;
                }
            }
#pragma unroll
            for (int t = 0; t < kSchurRows; ++t) {
                const int32_t pos = b + slot + t * S;
                if (pos < e) {
                    const double wk = a.w ? a.w[pos] : 1.0;
                    const double tk = a.p_has_b ? a.z_p[pos] : 0.0;
#pragma unroll
                    for (int u = 0; u < CW; ++u) {
                        const int c = col0 + 32 * u;
                        if (c < C) {
                            sw[u] = fma(wk, qc[t][u], sw[u]);
                            if (a.p_has_b) st[u] = fma(wk * tk, qc[t][u], st[u]);
                            if (!single) a.Q[static_cast<int64_t>(pos) * C + c] = qc[t][u];
                        }
                    }
                }
            }
            for (int32_t pos = b + slot + kSchurRows * S; pos < e; pos += S) {
                const double wk = a.w ? a.w[pos] : 1.0;
                const double tk = a.p_has_b ? a.z_p[pos] : 0.0;
#pragma unroll
                for (int u = 0; u < CW; ++u) {
                    const int c = col0 + 32 * u;
                    if (c < C) {
                        const double q = schur_q<ND>(a, pos, c);
                        sw[u] = fma(wk, q, sw[u]);
                        if (a.p_has_b) st[u] = fma(wk * tk, q, st[u]);
                        if (!single) a.Q[static_cast<int64_t>(pos) * C + c] = q;
                    }
                }
            }
        }
        // column totals over the row slots, in slot order, seen by every lane
        double tot[CW], tot_t[CW];
        if (CW == 1) {
            sred[wid][lane] = sw[0];
            tred[wid][lane] = st[0];
            __syncwarp();
            double t0 = 0.0, t1 = 0.0;
            if (live && col0 < C)
                for (int sl = 0; sl < S; ++sl) {
                    t0 += sred[wid][sl * C + col0];
                    t1 += tred[wid][sl * C + col0];
                }
            tot[0] = t0;
            tot_t[0] = t1;
            __syncwarp();
        } else {
#pragma unroll
            for (int u = 0; u < CW; ++u) {
                tot[u] = sw[u];
                tot_t[u] = st[u];
            }
        }
        if (single) {
            // the group's fit al + be t, (al, be) = M_g^-1 (sum w q, sum w t q)
            const double* mg = a.minv_p + static_cast<int64_t>(g) * 3;
            double al[CW], be[CW];
#pragma unroll
            for (int u = 0; u < CW; ++u) {
                const double sa = a.p_has_a ? tot[u] : 0.0;
                const double sb = a.p_has_b ? tot_t[u] : 0.0;
                al[u] = a.p_has_b ? fma(mg[0], sa, mg[1] * sb) : sa * mg[0];
                be[u] = a.p_has_b ? fma(mg[1], sa, mg[2] * sb) : 0.0;
            }
            if (live) {
                for (int32_t t = 0, pos = b + slot; pos < e; ++t, pos += S) {
                    const double wk = a.w ? a.w[pos] : 1.0;
                    const double tk = a.p_has_b ? a.z_p[pos] : 0.0;
#pragma unroll
                    for (int u = 0; u < CW; ++u) {
                        const int c = col0 + 32 * u;
                        if (c < C) {
                            double q = 0.0;
                            if (t < kSchurRows) {
#pragma unroll
                                for (int tt = 0; tt < kSchurRows; ++tt)
                                    if (tt == t) q = qc[tt][u];
                            } else {
                                q = schur_q<ND>(a, pos, c);
                            }
                            const double x = q - (a.p_has_b ? fma(be[u], tk, al[u]) : al[u]);
                            a.Q[static_cast<int64_t>(pos) * C + c] = x;
                            dacc[u] = fma(wk * x, x, dacc[u]);
                        }
                    }
                }
            }
        } else if (slot == 0) {
#pragma unroll
            for (int u = 0; u < CW; ++u) {
                const int c = col0 + 32 * u;
                if (c < C) {
                    double* pj = a.part_p + (j * a.p_nb) * C + c;
                    if (a.p_has_a) pj[0] = tot[u];
                    if (a.p_has_b) pj[a.p_has_a ? C : 0] = tot_t[u];
                }
            }
        }
    }
    // CTA partials of q' W q per column: warps, then row slots, in order
#pragma unroll
    for (int u = 0; u < CW; ++u) dred[wid][lane + 32 * u] = dacc[u];
    __syncthreads();
    if (static_cast<int>(threadIdx.x) < C) {
        const int c = threadIdx.x;
        double t = 0.0;
        for (int w8 = 0; w8 < kSlopeThreads / 32; ++w8) {
            if (CW == 1) {
                for (int sl = 0; sl < S; ++sl) t += dred[w8][sl * C + c];
            } else {
                t += dred[w8][c];
            }
        }
        a.dpart[static_cast<int64_t>(blockIdx.x) * C + c] = t;
    }
}

// the fit of the listed multi-chunk primary groups: their chunk sums, in chunk
// order, times the group's block inverse, into P.zv[g][nb][C]
__global__ void schur_fix_mean_kernel(const int32_t* __restrict__ groups, int32_t ngroups,
                                      const SlopeDim P, int C) {
    const int64_t total = static_cast<int64_t>(ngroups) * C;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = e / C;
        const int c = static_cast<int>(e - i * C);
        const int32_t g = groups[i];
        const int ob = P.has_a ? C : 0;
        double sa = 0.0, sb = 0.0;
        for (int32_t j = P.grp_ch[g]; j < P.grp_ch[g + 1]; ++j) {
            const double* pj = P.part + (static_cast<int64_t>(j) * P.nb) * C + c;
            if (P.has_a) sa += pj[0];
            if (P.has_b) sb += pj[ob];
        }
        const double* mg = P.minv + static_cast<int64_t>(g) * 3;
        double* zg = P.zv + (static_cast<int64_t>(g) * P.nb) * C + c;
        if (P.has_b) {
            if (P.has_a) zg[0] = fma(mg[0], sa, mg[1] * sb);
            zg[ob] = fma(mg[1], sa, mg[2] * sb);
        } else {
            zg[0] = sa * mg[0];
        }
    }
}

// Q -= the group's fit over the rows of the listed chunks (multi-chunk
// groups), with CTA partials of q' W q; one warp per chunk, row slots as in
// the gather
template <int CW>
__global__ void __launch_bounds__(kSlopeThreads)
schur_fix_apply_kernel(const int32_t* __restrict__ chunks, int32_t nchunks,
                       const int32_t* __restrict__ ch_grp, const SlopeDim P,
                       const double* __restrict__ w, double* __restrict__ Q, int C, int S,
                       double* __restrict__ dpart) {
    __shared__ double dred[kSlopeThreads / 32][32 * CW];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int slot = CW == 1 ? lane / C : 0;
    const int col0 = CW == 1 ? lane - slot * C : lane;
    const bool live = CW == 1 ? slot < S : true;
    double dacc[CW];
#pragma unroll
    for (int u = 0; u < CW; ++u) dacc[u] = 0.0;
    const int64_t nw = static_cast<int64_t>(gridDim.x) * (kSlopeThreads / 32);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * (kSlopeThreads / 32) + wid; i < nchunks;
         i += nw) {
        if (!live) continue;
        const int32_t j = chunks[i];
        const int32_t g = ch_grp[j];
        const double* zg = P.zv + (static_cast<int64_t>(g) * P.nb) * C;
        for (int32_t pos = P.ch_beg[j] + slot; pos < P.ch_end[j]; pos += S) {
            const double wk = w ? w[pos] : 1.0;
            const double tk = P.has_b ? P.z[pos] : 0.0;
#pragma unroll
            for (int u = 0; u < CW; ++u) {
                const int c = col0 + 32 * u;
                if (c < C) {
                    const int64_t o = static_cast<int64_t>(pos) * C + c;
                    double fit = P.has_a ? zg[c] : 0.0;
                    if (P.has_b) fit = fma(tk, zg[c + (P.has_a ? C : 0)], fit);
                    const double x = Q[o] - fit;
                    Q[o] = x;
                    dacc[u] = fma(wk * x, x, dacc[u]);
                }
            }
        }
    }
#pragma unroll
    for (int u = 0; u < CW; ++u) dred[wid][lane + 32 * u] = dacc[u];
    __syncthreads();
    if (static_cast<int>(threadIdx.x) < C) {
        const int c = threadIdx.x;
        double t = 0.0;
        for (int w8 = 0; w8 < kSlopeThreads / 32; ++w8) {
            if (CW == 1) {
                for (int sl = 0; sl < S; ++sl) t += dred[w8][sl * C + c];
            } else {
                t += dred[w8][c];
            }
        }
        dpart[static_cast<int64_t>(blockIdx.x) * C + c] = t;
    }
}

// flag[i] = 1 where a group holds more than `above` chunks (groups) or a chunk
// belongs to such a group (chunks, ch_grp given)
__global__ void multi_chunk_flags_kernel(const int32_t* __restrict__ grp_ch,
                                         const int32_t* __restrict__ ch_grp, int64_t m,
                                         int32_t* __restrict__ flag, int32_t above = 1) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = ch_grp ? ch_grp[i] : i;
        flag[i] = grp_ch[g + 1] - grp_ch[g] > above ? 1 : 0;
    }
}

// list[idx[i]] = i where flag[i] (idx: exclusive scan of the flags)
__global__ void compact_kernel(const int32_t* __restrict__ flag, const int32_t* __restrict__ idx,
                               int64_t m, int32_t* __restrict__ list) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (flag[i]) list[idx[i]] = static_cast<int32_t>(i);
}

// Groups with more than kFinSerialChunks chunks: one warp per (listed group,
// column, block); lane l sums partials l, l + 32, ... in order, then a fixed
// shuffle tree combines the lanes.  Result in d.big[g][b][c].
__global__ void __launch_bounds__(kSlopeThreads)
slope_big_reduce_kernel(const SlopeDim d, const int32_t* __restrict__ groups, int32_t ngroups,
                        int C) {
    const int lane = threadIdx.x & 31;
    const int64_t total = static_cast<int64_t>(ngroups) * d.nb * C;
    const int64_t nw = static_cast<int64_t>(gridDim.x) * (kSlopeThreads / 32);
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * (kSlopeThreads / 32) + (threadIdx.x >> 5);
         t < total; t += nw) {
        const int64_t i = t / (static_cast<int64_t>(d.nb) * C);
        const int rem = static_cast<int>(t - i * d.nb * C);
        const int b = rem / C, c = rem - b * C;
        const int32_t g = groups[i];
        double v = 0.0;
        for (int32_t j = d.grp_ch[g] + lane; j < d.grp_ch[g + 1]; j += 32)
            v += d.part[(static_cast<int64_t>(j) * d.nb + b) * C + c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) d.big[(static_cast<int64_t>(g) * d.nb + b) * C + c] = v;
    }
}

// p = zv + beta p (p = zv where beta is 0, so p needs no initial value)
__global__ void slope_direction_kernel(SlopeDim d, int C, const double* __restrict__ beta) {
    const int64_t total = static_cast<int64_t>(d.G) * d.nb * C;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double b = beta[e % C];
        d.p[e] = b == 0.0 ? d.zv[e] : fma(b, d.p[e], d.zv[e]);
    }
}

}  // namespace b200fe
