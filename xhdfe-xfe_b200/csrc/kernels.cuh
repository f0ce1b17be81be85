// Device kernels of the B200 fixed-effects absorber.
//
// Problem: for every column v of [y X], v~ = v - D a with D'W D a = D'W v.
// The largest FE dimension p ("primary", e.g. worker) is eliminated exactly:
// its block of D'W D is diagonal, so with r = the remaining dims,
//
//     S a_r = b,   S = D_r' W (I - P_p) D_r,   b = D_r' W (I - P_p) v,
//     v~ = (I - P_p)(v - D_r a_r),
//
// where P_p is the weighted projection on the primary group means.  S is
// solved by preconditioned CG with the exact diagonal of S (Jacobi).  This is
// the Schur-complement form of the alternating projections the reference runs
// in observation space (src/fe_absorption_cuda.cu:3070 run_demean,
// :3598-3998 Irons-Tuck loop, :4004-4408 block CG): the iterate lives in the
// small alpha space, so a CG iteration reads only the FE structure, never the
// n x C data columns.
//
// Layout in HBM (all device resident for the whole solve):
//   * observations in primary order (sorted by primary id; identity when the
//     input already is), primary segments given by seg_off;
//   * per large non-primary dim l: rid_l[k] (group id of obs k);
//     a "run" is a maximal block of consecutive obs of one primary segment
//     with the same rid_l; run m's sums go to row run_dest_l[m] of R_l, which
//     is ordered by group, so a group's runs are contiguous (grp chunks);
//   * small non-primary dims (<= 64 levels): 8-bit ids packed in sid[k];
//     their sums are privatised per warp in shared memory;
//   * alpha-space vectors: rows [GR][CP] (CP = 4*CQ columns, padded), large
//     dims first then small dims, at row offsets base[j].
//
// Every reduction has a fixed order (no floating-point atomics), so results
// are bitwise reproducible run to run.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200fe {

constexpr int kMaxDims = 8;
constexpr int kMaxLarge = 2;
constexpr int kMaxSmall = 4;
constexpr int kSmallLevels = 64;
constexpr int kPassThreads = 128;  // primary pass CTA size (4 warps)
constexpr int kRowThreads = 256;   // alpha-space row kernels

// ---------------------------------------------------------------------------
// 4-wide column quads.  A lane owns columns 4q..4q+3 of an alpha row.
// ---------------------------------------------------------------------------
struct Acc4 {
    double v[4];
};

__device__ __forceinline__ void acc_zero(Acc4& a) {
#pragma unroll
    for (int j = 0; j < 4; ++j) a.v[j] = 0.0;
}

__device__ __forceinline__ void load_quad(const float* p, Acc4& out) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    out.v[0] = t.x; out.v[1] = t.y; out.v[2] = t.z; out.v[3] = t.w;
}
__device__ __forceinline__ void load_quad(const double* p, Acc4& out) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    out.v[0] = a.x; out.v[1] = a.y; out.v[2] = b.x; out.v[3] = b.y;
}
__device__ __forceinline__ void add_quad(const float* p, Acc4& acc) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    acc.v[0] += t.x; acc.v[1] += t.y; acc.v[2] += t.z; acc.v[3] += t.w;
}
__device__ __forceinline__ void add_quad(const double* p, Acc4& acc) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    acc.v[0] += a.x; acc.v[1] += a.y; acc.v[2] += b.x; acc.v[3] += b.y;
}
// Streaming (read-once) variants: keep the alpha gathers resident in L2.
__device__ __forceinline__ void add_quad_stream(const float* p, Acc4& acc) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    acc.v[0] += t.x; acc.v[1] += t.y; acc.v[2] += t.z; acc.v[3] += t.w;
}
__device__ __forceinline__ void add_quad_stream(const double* p, Acc4& acc) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    acc.v[0] += a.x; acc.v[1] += a.y; acc.v[2] += b.x; acc.v[3] += b.y;
}
__device__ __forceinline__ void store_quad(float* p, const Acc4& a) {
    *reinterpret_cast<float4*>(p) =
        make_float4(static_cast<float>(a.v[0]), static_cast<float>(a.v[1]),
                    static_cast<float>(a.v[2]), static_cast<float>(a.v[3]));
}
__device__ __forceinline__ void store_quad(double* p, const Acc4& a) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a.v[0], a.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(a.v[2], a.v[3]);
}
__device__ __forceinline__ void store_quad_stream(float* p, const Acc4& a) {
    __stcs(reinterpret_cast<float4*>(p),
           make_float4(static_cast<float>(a.v[0]), static_cast<float>(a.v[1]),
                       static_cast<float>(a.v[2]), static_cast<float>(a.v[3])));
}
__device__ __forceinline__ void store_quad_stream(double* p, const Acc4& a) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(a.v[0], a.v[1]));
    __stcs(reinterpret_cast<double2*>(p) + 1, make_double2(a.v[2], a.v[3]));
}

// ---------------------------------------------------------------------------
// Primary-segment pass.
//
// One group of CQ lanes owns one primary segment s at a time.  For each obs
// k in s it forms a value val_k (per mode), then
//     mean_s = sum_k w_k val_k / W_s                          (loop 1)
//     z_k    = w_k (val_k - mean_s)                           (loop 2)
// and scatters z_k into the runs of every large dim and the per-warp bins of
// every small dim.  Modes:
//   kMatvec : val_k = (D_r x)_k           -> runs/bins give S x
//   kRhs    : val_k = v_k (data columns)  -> runs/bins give b = D_r'W(I-P_p)v
//   kFinal  : val_k = v_k - (D_r a)_k     -> writes v~_k = val_k - mean_s, and
//             (certify) runs/bins of z_k give D_r' W v~ for the certificate
// ---------------------------------------------------------------------------
enum PassMode { kMatvec = 0, kRhs = 1, kFinal = 2 };

template <typename T>
struct PassArgs {
    int64_t n;
    int32_t Gp;
    int cols;  // data columns C (y + X)
    int CP;    // padded columns of alpha rows
    int nL, nS;
    const int32_t* seg_off;   // [Gp+1]
    const double* inv_wp;     // [Gp] 1/W_s (0 for empty segments)
    const T* wp;              // [n] weights in primary order, or null (unit)
    const int32_t* pord;      // [n] primary order -> input row, or null (identity)
    const int32_t* rid[kMaxLarge];
    const int32_t* run_base[kMaxLarge];
    const int32_t* run_dest[kMaxLarge];
    int64_t lbase[kMaxLarge];  // alpha row offset of each large dim
    const uint32_t* sid;       // [n] packed small-dim ids (8 bits each) or null
    int64_t sbase[kMaxSmall];  // alpha row offset of each small dim
    const T* x;                // alpha-space input [GR][CP] (kMatvec, kFinal)
    const double* v;           // data, column-major n x cols (kRhs, kFinal)
    double* out;               // output, column-major n x cols (kFinal)
    T* R[kMaxLarge];           // run rows [nruns][CP]
    double* bins_partial;      // [gridDim][nS][64][CP]
    double* colsq_partial;     // [gridDim][CP]: kRhs sum v^2; kFinal sum_s (sum_k z_k)^2
    int scatter;               // kFinal: 1 to scatter z for the certificate
};

template <typename T, int MODE>
__device__ __forceinline__ void pass_value(const PassArgs<T>& a, int64_t k, int q,
                                           Acc4& val) {
    acc_zero(val);
    if (MODE == kRhs || MODE == kFinal) {
        const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = 4 * q + j;
            if (c < a.cols) val.v[j] = __ldg(a.v + static_cast<int64_t>(c) * a.n + o);
        }
    }
    if (MODE == kMatvec || MODE == kFinal) {
        Acc4 u;
        acc_zero(u);
#pragma unroll
        for (int l = 0; l < kMaxLarge; ++l) {
            if (l < a.nL) {
                const int32_t g = __ldg(a.rid[l] + k);
                add_quad(a.x + (a.lbase[l] + g) * a.CP + 4 * q, u);
            }
        }
        if (a.nS > 0) {
            const uint32_t packed = __ldg(a.sid + k);
            for (int s = 0; s < a.nS; ++s) {
                const uint32_t h = (packed >> (8 * s)) & 0xffu;
                add_quad(a.x + (a.sbase[s] + h) * a.CP + 4 * q, u);
            }
        }
        if (MODE == kMatvec) {
            val = u;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) val.v[j] -= u.v[j];
        }
    }
}

template <typename T, int CQ, int MODE>
__global__ void __launch_bounds__(kPassThreads)
primary_pass_kernel(const PassArgs<T> a) {
    extern __shared__ double smem_bins[];  // [warps][nS][64][CP]
    constexpr int GPW = 32 / CQ;           // segment groups per warp
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gw = lane / CQ;              // group within warp
    const int q = lane % CQ;
    const int warps_per_block = kPassThreads / 32;
    const int bin_stride = a.nS * kSmallLevels * a.CP;  // doubles per warp
    double* my_bins = smem_bins + warp * bin_stride;
    const bool scatter = (MODE != kFinal) || a.scatter;

    for (int i = threadIdx.x; i < warps_per_block * bin_stride; i += kPassThreads)
        smem_bins[i] = 0.0;
    __syncthreads();

    double colsq[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t total_warps = static_cast<int64_t>(gridDim.x) * warps_per_block;
    const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * warps_per_block + warp;

    for (int64_t s0 = warp_id * GPW; s0 < a.Gp; s0 += total_warps * GPW) {
        const int64_t s = s0 + gw;
        const bool valid = s < a.Gp;
        int64_t beg = 0, len = 0;
        double inv_w = 0.0;
        if (valid) {
            beg = a.seg_off[s];
            len = a.seg_off[s + 1] - beg;
            inv_w = a.inv_wp[s];
        }
        // loop 1: weighted segment mean of the value
        Acc4 acc;
        acc_zero(acc);
        for (int64_t t = 0; t < len; ++t) {
            const int64_t k = beg + t;
            Acc4 val;
            pass_value<T, MODE>(a, k, q, val);
            const double w = a.wp ? static_cast<double>(a.wp[k]) : 1.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) acc.v[j] = fma(w, val.v[j], acc.v[j]);
            if (MODE == kRhs) {
#pragma unroll
                for (int j = 0; j < 4; ++j) colsq[j] = fma(val.v[j], val.v[j], colsq[j]);
            }
        }
        Acc4 mean;
#pragma unroll
        for (int j = 0; j < 4; ++j) mean.v[j] = acc.v[j] * inv_w;

        // loop 2: z_k = w_k (val_k - mean); outputs, runs and bins
        int64_t steps = len;
        if (a.nS > 0 && scatter) {
            int64_t m = len;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
            steps = m;
        }
        int32_t cur[kMaxLarge];
        int32_t prev[kMaxLarge];
        Acc4 racc[kMaxLarge];
#pragma unroll
        for (int l = 0; l < kMaxLarge; ++l) {
            cur[l] = (l < a.nL && valid && len > 0) ? a.run_base[l][s] : 0;
            prev[l] = -1;
            acc_zero(racc[l]);
        }
        Acc4 zsum;
        acc_zero(zsum);
        for (int64_t t = 0; t < steps; ++t) {
            const bool active = t < len;
            const int64_t k = beg + t;
            Acc4 z;
            acc_zero(z);
            uint32_t packed = 0;
            if (active) {
                Acc4 val;
                pass_value<T, MODE>(a, k, q, val);
                const double w = a.wp ? static_cast<double>(a.wp[k]) : 1.0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double d = val.v[j] - mean.v[j];
                    z.v[j] = w * d;
                    if (MODE == kFinal) val.v[j] = d;
                }
                if (MODE == kFinal) {
                    const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int c = 4 * q + j;
                        if (c < a.cols) __stcs(a.out + static_cast<int64_t>(c) * a.n + o, val.v[j]);
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) zsum.v[j] += z.v[j];
                }
                if (scatter) {
#pragma unroll
                    for (int l = 0; l < kMaxLarge; ++l) {
                        if (l >= a.nL) continue;
                        const int32_t g = __ldg(a.rid[l] + k);
                        if (t > 0 && g != prev[l]) {
                            store_quad_stream(a.R[l] + static_cast<int64_t>(a.run_dest[l][cur[l]]) * a.CP + 4 * q,
                                              racc[l]);
                            ++cur[l];
                            acc_zero(racc[l]);
                        }
                        prev[l] = g;
#pragma unroll
                        for (int j = 0; j < 4; ++j) racc[l].v[j] += z.v[j];
                    }
                    if (a.nS > 0) packed = __ldg(a.sid + k);
                }
            }
            if (a.nS > 0 && scatter) {
                // fixed-order, race-free bin update: one segment group at a time
                for (int j = 0; j < GPW; ++j) {
                    __syncwarp();
                    if (gw == j && active) {
                        for (int s2 = 0; s2 < a.nS; ++s2) {
                            const uint32_t h = (packed >> (8 * s2)) & 0xffu;
                            double* b = my_bins + (s2 * kSmallLevels + h) * a.CP + 4 * q;
#pragma unroll
                            for (int c = 0; c < 4; ++c) b[c] += z.v[c];
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (scatter && valid && len > 0) {
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l)
                if (l < a.nL) store_quad_stream(a.R[l] + static_cast<int64_t>(a.run_dest[l][cur[l]]) * a.CP + 4 * q,
                                  racc[l]);
        }
        if (MODE == kFinal && valid) {
#pragma unroll
            for (int j = 0; j < 4; ++j) colsq[j] = fma(zsum.v[j], zsum.v[j], colsq[j]);
        }
    }

    // per-CTA bins: warps summed in fixed order
    __syncthreads();
    if (a.nS > 0 && scatter) {
        double* dst = a.bins_partial + static_cast<int64_t>(blockIdx.x) * bin_stride;
        for (int i = threadIdx.x; i < bin_stride; i += kPassThreads) {
            double s = 0.0;
            for (int w = 0; w < warps_per_block; ++w) s += smem_bins[w * bin_stride + i];
            dst[i] = s;
        }
    }
    if (MODE == kRhs || MODE == kFinal) {
        // per-CTA column sums of colsq: lanes with the same q hold the same columns
        __syncthreads();
        double* red = smem_bins;  // reuse: [kPassThreads][4]
        // make sure there is room: bins area may be empty (nS == 0) -> caller
        // sizes dynamic smem to at least kPassThreads*4 doubles.
        for (int j = 0; j < 4; ++j) red[threadIdx.x * 4 + j] = colsq[j];
        __syncthreads();
        if (threadIdx.x < CQ) {
            double s4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = threadIdx.x; t < kPassThreads; t += CQ)
                for (int j = 0; j < 4; ++j) s4[j] += red[t * 4 + j];
            for (int j = 0; j < 4; ++j)
                a.colsq_partial[static_cast<int64_t>(blockIdx.x) * a.CP + 4 * threadIdx.x + j] = s4[j];
        }
    }
}

// ---------------------------------------------------------------------------
// Run gather-sum (large dims): out row of group g = sum of its runs' rows.
// Chunks (group, begin, end) with end-begin <= chunk size; groups with one
// chunk are written directly, multi-chunk groups leave a partial per chunk.
// Also accumulates, per CTA, the dot of the written rows with `dotv`.
// ---------------------------------------------------------------------------
template <typename T>
struct GatherArgs {
    int CP;
    int64_t nchunks;
    const int32_t* chunk_grp;   // [nchunks]
    const int32_t* chunk_beg;   // [nchunks]
    const int32_t* chunk_end;   // [nchunks]
    const uint8_t* chunk_whole; // [nchunks] 1 if the chunk is its group's only chunk
    const T* R;                 // [nruns][CP]
    T* out;                     // alpha rows of this dim (already offset by base)
    double* partial;            // [nchunks][CP] for multi-chunk groups
    const T* dotv;              // alpha rows of this dim (offset) or null
    double* dot_partial;        // [gridDim][CP] or null
};

template <typename T, int CQ>
__global__ void __launch_bounds__(kRowThreads)
run_gather_kernel(const GatherArgs<T> a) {
    __shared__ double red[kRowThreads][4];
    const int q = threadIdx.x % CQ;
    const int64_t grp0 = (static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x) / CQ;
    const int64_t ngroups = static_cast<int64_t>(gridDim.x) * kRowThreads / CQ;
    double dot[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t c = grp0; c < a.nchunks; c += ngroups) {
        const int32_t g = a.chunk_grp[c];
        const int32_t b = a.chunk_beg[c];
        const int32_t e = a.chunk_end[c];
        Acc4 acc;
        acc_zero(acc);
        for (int32_t j = b; j < e; ++j)
            add_quad_stream(a.R + static_cast<int64_t>(j) * a.CP + 4 * q, acc);
        if (a.chunk_whole[c]) {
            T* dst = a.out + static_cast<int64_t>(g) * a.CP + 4 * q;
            store_quad(dst, acc);
            if (a.dotv) {
                Acc4 pv;
                load_quad(a.dotv + static_cast<int64_t>(g) * a.CP + 4 * q, pv);
#pragma unroll
                for (int j = 0; j < 4; ++j)  // dot with the stored (rounded) value
                    dot[j] = fma(pv.v[j], static_cast<double>(static_cast<T>(acc.v[j])), dot[j]);
            }
        } else {
            double* dst = a.partial + c * a.CP + 4 * q;
#pragma unroll
            for (int j = 0; j < 4; ++j) dst[j] = acc.v[j];
        }
    }
    if (a.dot_partial) {
        for (int j = 0; j < 4; ++j) red[threadIdx.x][j] = dot[j];
        __syncthreads();
        if (threadIdx.x < CQ) {
            double s4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = threadIdx.x; t < kRowThreads; t += CQ)
                for (int j = 0; j < 4; ++j) s4[j] += red[t][j];
            for (int j = 0; j < 4; ++j)
                a.dot_partial[static_cast<int64_t>(blockIdx.x) * a.CP + 4 * threadIdx.x + j] = s4[j];
        }
    }
}

// ---------------------------------------------------------------------------
// Finalize: multi-chunk large groups and small-dim bins; then the last CTA
// reduces every dot partial (run_gather CTAs and this kernel's) in a fixed
// order into dot_out[CP].
// ---------------------------------------------------------------------------
template <typename T>
struct FinalizeArgs {
    int CP;
    int nL, nS;
    // multi-chunk groups of each large dim
    int64_t nmulti[kMaxLarge];
    const int32_t* multi_grp[kMaxLarge];
    const int32_t* multi_c0[kMaxLarge];
    const int32_t* multi_c1[kMaxLarge];
    const double* partial[kMaxLarge];
    int64_t lbase[kMaxLarge];
    // small dims
    int32_t sG[kMaxSmall];
    int64_t sbase[kMaxSmall];
    const double* bins_partial;  // [nbins_ctas][nS][64][CP]
    int nbins_ctas;
    T* out;                      // alpha rows [GR][CP]
    const T* dotv;               // or null
    // dot reduction
    double* dot_partial;         // this kernel's [gridDim][CP]
    const double* gather_dot_partial[kMaxLarge];  // run_gather's partials
    int gather_ctas[kMaxLarge];
    double* dot_out;             // [CP]
    unsigned int* ticket;
};

template <typename T>
__global__ void __launch_bounds__(kRowThreads)
finalize_kernel(const FinalizeArgs<T> a) {
    __shared__ double red[kRowThreads];
    __shared__ bool last;
    // item space: (multi groups of each large dim) then (small bins), per column
    double dot = 0.0;
    int mycol = -1;
    int64_t items = 0;
    for (int l = 0; l < a.nL; ++l) items += a.nmulti[l] * a.CP;
    for (int s = 0; s < a.nS; ++s) items += static_cast<int64_t>(a.sG[s]) * a.CP;
    // stride is a multiple of CP so each thread keeps one column
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kRowThreads;
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x;
    for (int64_t it = start; it < items; it += stride) {
        int64_t r = it;
        const int c = static_cast<int>(r % a.CP);
        int64_t rowi = r / a.CP;
        mycol = c;
        double sum = 0.0;
        int64_t orow = -1;
        bool done = false;
        for (int l = 0; l < a.nL && !done; ++l) {
            if (rowi < a.nmulti[l]) {
                const int32_t g = a.multi_grp[l][rowi];
                for (int32_t ch = a.multi_c0[l][rowi]; ch < a.multi_c1[l][rowi]; ++ch)
                    sum += a.partial[l][static_cast<int64_t>(ch) * a.CP + c];
                orow = a.lbase[l] + g;
                done = true;
            } else {
                rowi -= a.nmulti[l];
            }
        }
        for (int s = 0; s < a.nS && !done; ++s) {
            if (rowi < a.sG[s]) {
                const int64_t off = (static_cast<int64_t>(s) * kSmallLevels + rowi) * a.CP + c;
                const int64_t stride_cta = static_cast<int64_t>(a.nS) * kSmallLevels * a.CP;
                for (int b = 0; b < a.nbins_ctas; ++b) sum += a.bins_partial[b * stride_cta + off];
                orow = a.sbase[s] + rowi;
                done = true;
            } else {
                rowi -= a.sG[s];
            }
        }
        const T stored = static_cast<T>(sum);
        a.out[orow * a.CP + c] = stored;
        if (a.dotv) dot = fma(static_cast<double>(a.dotv[orow * a.CP + c]),
                              static_cast<double>(stored), dot);
    }
    if (!a.dot_out) return;
    // per-CTA per-column partials: thread t always handles column (start % CP)
    // because stride % CP == 0 is guaranteed by the launcher.
    red[threadIdx.x] = dot;
    (void)mycol;
    __syncthreads();
    if (threadIdx.x < a.CP) {
        double s = 0.0;
        for (int t = threadIdx.x; t < kRowThreads; t += a.CP) s += red[t];
        a.dot_partial[static_cast<int64_t>(blockIdx.x) * a.CP + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(a.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < a.CP) {
        const int c = threadIdx.x;
        double s = 0.0;
        for (int l = 0; l < a.nL; ++l)
            for (int b = 0; b < a.gather_ctas[l]; ++b)
                s += __ldcg(a.gather_dot_partial[l] + static_cast<int64_t>(b) * a.CP + c);
        for (int b = 0; b < static_cast<int>(gridDim.x); ++b)
            s += __ldcg(a.dot_partial + static_cast<int64_t>(b) * a.CP + c);
        a.dot_out[c] = s;
    }
    if (threadIdx.x == 0) *a.ticket = 0u;
}

// ---------------------------------------------------------------------------
// PCG vector kernels over the alpha rows (GR x CP), per-column scalars.
// ---------------------------------------------------------------------------
struct CgScalars {
    // per column (CP entries each)
    double* rz;      // r'z
    double* pq;      // p'Sp
    double* rr;      // r'r
    double* bb;      // b'b (fixed per solve)
    double* beta;
    double* alpha;
    int* active;     // 1 while the column iterates
    int* iters;      // iterations taken per column
    double* partial; // [grid][2*CP]
    unsigned int* ticket;
    int* n_active;   // number of active columns
};

// alpha = rz/pq; x += alpha p; r -= alpha q; z = dinv r; partial r'z, r'r.
// The last CTA finalises beta, rz, the convergence flags.
template <typename T>
__global__ void __launch_bounds__(kRowThreads)
cg_update_kernel(int64_t GR, int CP, T* __restrict__ x, T* __restrict__ r,
                 T* __restrict__ z, const T* __restrict__ p, const T* __restrict__ qv,
                 const T* __restrict__ dinv, CgScalars sc, double tol2, int iter) {
    __shared__ double red[kRowThreads][2];
    __shared__ bool last;
    const int64_t total = GR * CP;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kRowThreads;  // multiple of CP
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x;
    const int c = static_cast<int>(start % CP);
    const bool act = sc.active[c] != 0;
    const double pqc = sc.pq[c];
    const double al = (act && pqc > 0.0) ? sc.rz[c] / pqc : 0.0;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = start; i < total; i += stride) {
        const int64_t row = i / CP;
        double ri = static_cast<double>(r[i]);
        if (al != 0.0) {
            x[i] = static_cast<T>(static_cast<double>(x[i]) + al * static_cast<double>(p[i]));
            ri -= al * static_cast<double>(qv[i]);
            r[i] = static_cast<T>(ri);
            ri = static_cast<double>(r[i]);
        }
        const double zi = static_cast<double>(dinv[row]) * ri;
        z[i] = static_cast<T>(zi);
        rz = fma(ri, static_cast<double>(static_cast<T>(zi)), rz);
        rr = fma(ri, ri, rr);
    }
    red[threadIdx.x][0] = rz;
    red[threadIdx.x][1] = rr;
    __syncthreads();
    if (threadIdx.x < CP) {
        double s0 = 0.0, s1 = 0.0;
        for (int t = threadIdx.x; t < kRowThreads; t += CP) {
            s0 += red[t][0];
            s1 += red[t][1];
        }
        sc.partial[static_cast<int64_t>(blockIdx.x) * 2 * CP + threadIdx.x] = s0;
        sc.partial[static_cast<int64_t>(blockIdx.x) * 2 * CP + CP + threadIdx.x] = s1;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(sc.ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < CP) {
        const int cc = threadIdx.x;
        double s0 = 0.0, s1 = 0.0;
        for (int b = 0; b < static_cast<int>(gridDim.x); ++b) {
            s0 += __ldcg(sc.partial + static_cast<int64_t>(b) * 2 * CP + cc);
            s1 += __ldcg(sc.partial + static_cast<int64_t>(b) * 2 * CP + CP + cc);
        }
        const int was_active = sc.active[cc];
        if (was_active) {
            const double old = sc.rz[cc];
            sc.beta[cc] = old > 0.0 ? s0 / old : 0.0;
            sc.rz[cc] = s0;
            sc.rr[cc] = s1;
            if (iter >= 0) sc.iters[cc] = iter + 1;
            if (!(s1 > tol2 * sc.bb[cc]) || !(s0 > 0.0)) sc.active[cc] = 0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int na = 0;
        for (int cc = 0; cc < CP; ++cc) na += sc.active[cc];
        *sc.n_active = na;
        *sc.ticket = 0u;
    }
}

// p = z + beta p for active columns (first iteration: p = z).
template <typename T>
__global__ void __launch_bounds__(kRowThreads)
cg_direction_kernel(int64_t GR, int CP, T* __restrict__ p, const T* __restrict__ z,
                    CgScalars sc, int first) {
    const int64_t total = GR * CP;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kRowThreads;
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x;
    const int c = static_cast<int>(start % CP);
    const bool act = sc.active[c] != 0;
    const double be = first ? 0.0 : sc.beta[c];
    if (!act && !first) return;
    for (int64_t i = start; i < total; i += stride)
        p[i] = static_cast<T>(static_cast<double>(z[i]) + be * static_cast<double>(p[i]));
}

}  // namespace b200fe
