// The Schur block of the one large non-primary dimension, built explicitly.
//
// With the primary dim p eliminated and one large dim f (firms) left, the
// firm block of the Schur complement is
//
//     S_ff = D_f' W (I - P_p) D_f = sum_s ( diag(C_s) - C_s C_s' / W_s )
//
// where s runs over primary segments (workers), C_s[g] is the weight of
// segment s's observations in group g and W_s the segment's weight.  A
// segment whose observations all sit in one group adds C = W_s on the
// diagonal and C^2 / W_s = W_s off it: nothing.  So only segments with two or
// more distinct groups (movers) contribute, each u^2 entries for u distinct
// groups:
//
//     S[g_i][g_i] += C_i (sum_{j != i} C_j) / W_s      (no cancellation)
//     S[g_i][g_j] -= C_i C_j / W_s                      (i != j)
//
// On a 50M-observation AKM panel (5M workers, 490k firms) that is about 19M
// contributions merging into 6M nonzeros, against 9.4M runs whose 16-column
// rows the run-level matvec writes and reads back every iteration.  The CG
// matvec becomes one sparse gather per row chunk (sparse_gather_kernel), with
// the dense small-dim coupling and the finalize step unchanged.
//
// Determinism: contributions are emitted in segment order, sorted by a stable
// radix sort on (row, column), and each nonzero sums its contributions in
// that order (a fixed-order block reduction for very long ones); every row of
// the gather sums its nonzeros in column order.  No floating-point atomics.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace b200fe {

constexpr int kSparseMaxRuns = 64;     // runs per segment the pair build handles
constexpr int kSparseChunk = 64;       // nonzeros per gather chunk
constexpr int kSparseMergeSerial = 512;  // contributions one thread merges serially

// Per segment: the number of contributions it emits (u^2 for u >= 2 distinct
// groups among its runs, else 0).  flag |= 1 when a segment has more runs than
// kSparseMaxRuns (the caller then keeps the run-level matvec).
__global__ void sparse_pair_count_kernel(int32_t Gp, const int32_t* __restrict__ run_base,
                                         const int32_t* __restrict__ run_grp,
                                         int32_t* __restrict__ count, int32_t* __restrict__ flag,
                                         unsigned long long* __restrict__ total) {
    unsigned long long mine = 0;
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < Gp;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = run_base[s], e = run_base[s + 1];
        int32_t u = 0;
        if (e - b > kSparseMaxRuns) {
            atomicOr(flag, 1);
        } else if (e - b >= 2) {
            for (int32_t a = b; a < e; ++a) {
                const int32_t g = run_grp[a];
                bool seen = false;
                for (int32_t c = b; c < a && !seen; ++c) seen = run_grp[c] == g;
                u += seen ? 0 : 1;
            }
        }
        const int32_t cnt = u >= 2 ? u * u : 0;
        count[s] = cnt;
        mine += static_cast<unsigned long long>(cnt);
    }
    // integer atomics: the total does not depend on their order
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(total, mine);
}

// Per contributing segment: its distinct groups in order of first appearance,
// their weights C_i (runs of one group summed in run order), and the u^2
// contributions at off[s] .. off[s] + u^2, row-major in that order.
__global__ void sparse_pair_fill_kernel(int32_t Gp, const int32_t* __restrict__ run_base,
                                        const int32_t* __restrict__ run_grp,
                                        const double* __restrict__ run_w,
                                        const double* __restrict__ inv_wp,
                                        const int32_t* __restrict__ count,
                                        const int32_t* __restrict__ off, int32_t G,
                                        unsigned long long* __restrict__ keys,
                                        double* __restrict__ vals) {
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < Gp;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (count[s] == 0) continue;
        const int32_t b = run_base[s], e = run_base[s + 1];
        int32_t grp[kSparseMaxRuns];
        double cw[kSparseMaxRuns];
        int u = 0;
        for (int32_t a = b; a < e; ++a) {
            const int32_t g = run_grp[a];
            const double c = run_w[a];
            int i = 0;
            while (i < u && grp[i] != g) ++i;
            if (i == u) {
                grp[u] = g;
                cw[u] = c;
                ++u;
            } else {
                cw[i] += c;
            }
        }
        const double iw = inv_wp[s];
        int64_t o = off[s];
        for (int i = 0; i < u; ++i) {
            double others = 0.0;
            for (int j = 0; j < u; ++j)
                if (j != i) others += cw[j];
            const unsigned long long row = static_cast<unsigned long long>(grp[i]) *
                                           static_cast<unsigned long long>(G);
            for (int j = 0; j < u; ++j) {
                keys[o] = row + static_cast<unsigned long long>(grp[j]);
                vals[o] = (j == i) ? cw[i] * others * iw : -(cw[i] * cw[j]) * iw;
                ++o;
            }
        }
    }
}

// flags[i] = 1 where sorted key i starts a new nonzero
__global__ void sparse_key_flags_kernel(const unsigned long long* __restrict__ keys, int64_t n,
                                        int32_t* __restrict__ flags) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// For nonzero u (uid = inclusive scan of the flags): first contribution,
// row and column.  ustart[nnz] = n is written by the thread of the last key.
__global__ void sparse_unique_fill_kernel(const unsigned long long* __restrict__ keys, int64_t n,
                                          const int32_t* __restrict__ flags,
                                          const int32_t* __restrict__ uid, int32_t G,
                                          int32_t* __restrict__ ustart, int32_t* __restrict__ urow,
                                          int32_t* __restrict__ ucol) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (flags[i]) {
            const int32_t u = uid[i] - 1;
            const unsigned long long k = keys[i];
            ustart[u] = static_cast<int32_t>(i);
            urow[u] = static_cast<int32_t>(k / static_cast<unsigned long long>(G));
            ucol[u] = static_cast<int32_t>(k % static_cast<unsigned long long>(G));
        }
        if (i == n - 1) ustart[uid[i]] = static_cast<int32_t>(n);
    }
}

// Nonzeros with at most kSparseMergeSerial contributions: summed in order by
// one thread; longer ones are appended to long_list (an integer counter: the
// list's order varies, each listed value is still summed in a fixed order).
__global__ void sparse_merge_kernel(int64_t nnz, const int32_t* __restrict__ ustart,
                                    const double* __restrict__ vals, double* __restrict__ val64,
                                    int32_t* __restrict__ long_list, int32_t* __restrict__ long_count) {
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < nnz;
         u += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = ustart[u], e = ustart[u + 1];
        if (e - b > kSparseMergeSerial) {
            long_list[atomicAdd(long_count, 1)] = static_cast<int32_t>(u);
            continue;
        }
        double s = 0.0;
        for (int32_t i = b; i < e; ++i) s += vals[i];
        val64[u] = s;
    }
}

// One CTA per listed nonzero: thread t sums contributions t, t+B, t+2B, ... in
// order, then a fixed tree (the result does not depend on scheduling).
__global__ void __launch_bounds__(256)
sparse_merge_long_kernel(const int32_t* __restrict__ long_list, const int32_t* __restrict__ long_count,
                         const int32_t* __restrict__ ustart, const double* __restrict__ vals,
                         double* __restrict__ val64) {
    __shared__ double red[256];
    const int32_t nl = *long_count;
    for (int32_t li = blockIdx.x; li < nl; li += gridDim.x) {
        const int32_t u = long_list[li];
        const int32_t b = ustart[u], e = ustart[u + 1];
        double s = 0.0;
        for (int32_t i = b + threadIdx.x; i < e; i += 256) s += vals[i];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) val64[u] = red[0];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// q_f = S_ff x_f (+ C_fy x_small) over row chunks of the explicit block.
// A lane group of CQ lanes (4 columns each) owns a chunk and sums its
// nonzeros in column order, four gathers in flight; whole-row chunks store
// the row (and add to the CTA's dot with dotv), others leave a partial that
// finalize_kernel adds up in chunk order.  Same outputs and partial layout as
// run_gather_kernel.
// ---------------------------------------------------------------------------
template <typename T>
struct SparseGatherArgs {
    int CP;
    int64_t nchunks;
    const int32_t* chunk_grp;   // [nchunks] row of the chunk
    const int32_t* chunk_beg;   // [nchunks] first nonzero
    const int32_t* chunk_end;   // [nchunks]
    const uint8_t* chunk_whole; // [nchunks] 1 if the chunk is its row's only chunk
    const int32_t* col;         // [nnz]
    const T* val;               // [nnz]
    const T* x;                 // rows of this dim in the matvec input (offset)
    T* out;                     // rows of this dim (offset)
    double* partial;            // [nchunks][CP] for multi-chunk rows
    double* dot_partial;        // [gridDim][CP] or null
    const T* cfy;               // [G][SGP] dense coupling to the small dim, or null
    const T* xs;                // small-dim rows of the matvec input [SG][CP]
    int SG, SGP;
};

template <typename T, int CQ>
__global__ void __launch_bounds__(kRowThreads)
sparse_gather_kernel(const SparseGatherArgs<T> a) {
    __shared__ double red[kRowThreads][4];
    extern __shared__ __align__(16) unsigned char sgsmem_raw[];
    T* xs_s = reinterpret_cast<T*>(sgsmem_raw);  // [SGP][CP] small rows of x
    const int q = threadIdx.x % CQ;
    if (a.cfy) {
        for (int i = threadIdx.x; i < a.SGP * a.CP; i += kRowThreads)
            xs_s[i] = i < a.SG * a.CP ? a.xs[i] : T(0);
        __syncthreads();
    }
    const int64_t grp0 = (static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x) / CQ;
    const int64_t ngroups = static_cast<int64_t>(gridDim.x) * kRowThreads / CQ;
    double dot[4] = {0.0, 0.0, 0.0, 0.0};
    constexpr int U = 4;
    for (int64_t c = grp0; c < a.nchunks; c += ngroups) {
        const int32_t g = a.chunk_grp[c];
        const int32_t b = a.chunk_beg[c];
        const int32_t e = a.chunk_end[c];
        Acc4 acc;  // terms in the solve's precision, sums in FP64
        acc_zero(acc);
        int32_t j = b;
        for (; j + U <= e; j += U) {
            int32_t cj[U];
            T vj[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                cj[u] = __ldg(a.col + j + u);
                vj[u] = __ldg(a.val + j + u);
            }
            V4<T> xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) v4_load(a.x + static_cast<int64_t>(cj[u]) * a.CP + 4 * q, xv[u]);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    acc.v[i] = fma(static_cast<double>(vj[u]), static_cast<double>(xv[u].v[i]), acc.v[i]);
        }
        for (; j < e; ++j) {
            const int32_t cj = __ldg(a.col + j);
            const T vj = __ldg(a.val + j);
            V4<T> xv;
            v4_load(a.x + static_cast<int64_t>(cj) * a.CP + 4 * q, xv);
#pragma unroll
            for (int i = 0; i < 4; ++i)
                acc.v[i] = fma(static_cast<double>(vj), static_cast<double>(xv.v[i]), acc.v[i]);
        }
        if (a.chunk_whole[c]) {
            if (a.cfy) {  // + C_fy[g] x_small, four levels per load
                const T* crow = a.cfy + static_cast<int64_t>(g) * a.SGP;
                for (int h0 = 0; h0 < a.SGP; h0 += 4) {
                    T c4[4];
                    load4<T>(crow + h0, c4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T* xr = xs_s + (h0 + u) * a.CP + 4 * q;
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            acc.v[i] = fma(static_cast<double>(c4[u]), static_cast<double>(xr[i]), acc.v[i]);
                    }
                }
            }
            T* dst = a.out + static_cast<int64_t>(g) * a.CP + 4 * q;
            store_quad(dst, acc);
            if (a.dot_partial) {
                V4<T> pv;
                v4_load(a.x + static_cast<int64_t>(g) * a.CP + 4 * q, pv);
#pragma unroll
                for (int i = 0; i < 4; ++i)  // dot with the stored (rounded) value
                    dot[i] = fma(static_cast<double>(pv.v[i]),
                                 static_cast<double>(static_cast<T>(acc.v[i])), dot[i]);
            }
        } else {
            double* dst = a.partial + c * a.CP + 4 * q;
#pragma unroll
            for (int i = 0; i < 4; ++i) dst[i] = acc.v[i];
        }
    }
    if (a.dot_partial) {
        for (int i = 0; i < 4; ++i) red[threadIdx.x][i] = dot[i];
        __syncthreads();
        if (threadIdx.x < CQ) {
            double s4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = threadIdx.x; t < kRowThreads; t += CQ)
                for (int i = 0; i < 4; ++i) s4[i] += red[t][i];
            for (int i = 0; i < 4; ++i)
                a.dot_partial[static_cast<int64_t>(blockIdx.x) * a.CP + 4 * threadIdx.x + i] = s4[i];
        }
    }
}

}  // namespace b200fe
