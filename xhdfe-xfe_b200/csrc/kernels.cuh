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

#include "limits.cuh"

namespace b200fe {


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
// Primary-segment passes.
//
// For every primary segment s (one value of the eliminated dim) and every
// observation k in s, with a per-mode value val_k:
//     mean_s = sum_k w_k val_k / W_s
//     z_k    = w_k (val_k - mean_s)
// z_k is scattered into the runs of every large dim and the bins of every
// small dim.  Modes:
//   kMatvec : val_k = (D_r x)_k           -> runs/bins give S x
//   kRhs    : val_k = v_k (data columns)  -> runs/bins give b = D_r'W(I-P_p)v
//   kFinal  : val_k = v_k - (D_r a)_k     -> writes v~_k = val_k - mean_s, and
//             (certify) runs/bins of z_k give D_r' W v~ for the certificate
//
// tile_pass_kernel handles tiles of whole segments (<= kTileObs obs): all
// loads of a tile are issued at once into shared memory, then segment means,
// runs and bins are reduced from shared memory.  Segments longer than
// kLongSeg form their own tiles and go through segment_pass_kernel.
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
    const int32_t* run_base[kMaxLarge];   // [Gp+1] first run of each segment
    const int32_t* run_start[kMaxLarge];  // [nruns+1] first obs of each run
    const int32_t* run_dest[kMaxLarge];   // [nruns] row of each run in R (group order)
    int64_t lbase[kMaxLarge];  // alpha row offset of each large dim
    const uint32_t* sid;       // [n] packed small-dim ids (8 bits each) or null
    int64_t sbase[kMaxSmall];  // alpha row offset of each small dim
    int sgoff[kMaxSmall];      // bin row offset of each small dim
    int SG;                    // bin rows (levels over all small dims)
    const T* x;                // alpha-space input [GR][CP] (kMatvec, kFinal)
    const double* v;           // data, column-major n x cols (kRhs, kFinal)
    double* out;               // output, column-major n x cols (kFinal)
    T* R[kMaxLarge];           // run rows [nruns][CP]
    double* bins_partial;      // [ctas][SG][CP]; this launch writes from bins_cta0
    double* colsq_partial;     // [ctas][CP]: kRhs sum v^2; kFinal sum_s (sum_k z_k)^2
    int bins_cta0;             // first CTA slot of this launch in the partial arrays
    int scatter;               // kFinal: 1 to scatter z for the certificate
    double* mean_out;          // kFinal: [Gp][CP] primary segment means of v - D_r a, or null
    int bins_no_diag;          // kMatvec: bins get z_k - w_k x_s[h_k] (finalize adds W_h x_s[h])
    // tiles
    const int32_t* tile_seg;   // [ntiles+1] first segment of each tile
    const uint8_t* tile_long;  // [ntiles] 1 for a single long segment
    int64_t ntiles;
    // long segments (segment_pass_kernel)
    const int32_t* long_segs;
    int64_t nlong;
};

// (D_r x)_k for the 4 columns of lane quad q
template <typename T>
__device__ __forceinline__ void gather_u(const PassArgs<T>& a, int64_t k, int q, Acc4& u) {
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
}

template <typename T>
__device__ __forceinline__ void smem_load4(const T* p, Acc4& o);
template <>
__device__ __forceinline__ void smem_load4<float>(const float* p, Acc4& o) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o.v[0] = t.x; o.v[1] = t.y; o.v[2] = t.z; o.v[3] = t.w;
}
template <>
__device__ __forceinline__ void smem_load4<double>(const double* p, Acc4& o) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    o.v[0] = a.x; o.v[1] = a.y; o.v[2] = b.x; o.v[3] = b.y;
}
template <typename T>
__device__ __forceinline__ void smem_store4(T* p, const Acc4& o);
template <>
__device__ __forceinline__ void smem_store4<float>(float* p, const Acc4& o) {
    *reinterpret_cast<float4*>(p) = make_float4(static_cast<float>(o.v[0]), static_cast<float>(o.v[1]),
                                                static_cast<float>(o.v[2]), static_cast<float>(o.v[3]));
}
template <>
__device__ __forceinline__ void smem_store4<double>(double* p, const Acc4& o) {
    reinterpret_cast<double2*>(p)[0] = make_double2(o.v[0], o.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(o.v[2], o.v[3]);
}

// Dynamic shared memory of tile_pass_kernel, in bytes.
template <typename T>
__host__ __device__ constexpr size_t tile_smem_bytes(int CP, int SG) {
    return static_cast<size_t>(kTileObs + 1) * CP * sizeof(T)  // staged values
           + static_cast<size_t>(kTileObs) * sizeof(T)         // weights
           + static_cast<size_t>(kTileThreads / 32) * SG * (CP + 1) * sizeof(double)  // bins
           + static_cast<size_t>(kTileThreads) * 4 * sizeof(double);                 // colsq red
}

// Staged tile values: kMatvec keeps rows [kl][CP] (16-byte quads, gathered
// per observation); the data modes keep columns [c][kTileObs + 1] so the
// coalesced column loads and stores are free of bank conflicts.
template <typename T, int CP, int MODE>
struct Stage {
    static constexpr int LD = kTileObs + 1;
    __device__ static __forceinline__ void load4(const T* u, int kl, int q, Acc4& o) {
        if (MODE == kMatvec) {
            smem_load4<T>(u + kl * CP + 4 * q, o);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) o.v[j] = static_cast<double>(u[(4 * q + j) * LD + kl]);
        }
    }
    __device__ static __forceinline__ void store4(T* u, int kl, int q, const Acc4& o) {
        if (MODE == kMatvec) {
            smem_store4<T>(u + kl * CP + 4 * q, o);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) u[(4 * q + j) * LD + kl] = static_cast<T>(o.v[j]);
        }
    }
    __device__ static __forceinline__ T& at(T* u, int kl, int c) {
        return MODE == kMatvec ? u[kl * CP + c] : u[c * LD + kl];
    }
};

template <typename T, int CQ, int MODE>
__global__ void __launch_bounds__(kTileThreads)
tile_pass_kernel(const PassArgs<T> a) {
    constexpr int CP = 4 * CQ;
    using St = Stage<T, CP, MODE>;
    constexpr int GPB = kTileThreads / CQ;  // lane groups per block
    constexpr int BROW = CP + 1;            // padded bin row (doubles)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ubuf = reinterpret_cast<T*>(smem_raw);
    T* wbuf = ubuf + (kTileObs + 1) * CP;
    double* bins = reinterpret_cast<double*>(wbuf + kTileObs);
    double* red = bins + (kTileThreads / 32) * a.SG * BROW;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = tid / CQ;  // lane group
    const int q = tid % CQ;
    const bool scatter = (MODE != kFinal) || a.scatter;
    double* my_bins = bins + warp * a.SG * BROW;
    for (int i = tid; i < (kTileThreads / 32) * a.SG * BROW; i += kTileThreads) bins[i] = 0.0;
    double colsq[4] = {0.0, 0.0, 0.0, 0.0};

    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        if (a.tile_long[t]) continue;
        const int32_t s0 = a.tile_seg[t], s1 = a.tile_seg[t + 1];
        const int64_t k0 = a.seg_off[s0];
        const int nk = static_cast<int>(a.seg_off[s1] - k0);
        __syncthreads();  // previous tile fully consumed
        // ---- phase A: stage values and weights --------------------------
        if (MODE == kMatvec) {
            for (int kl = g; kl < nk; kl += GPB) {
                Acc4 u;
                gather_u(a, k0 + kl, q, u);
                St::store4(ubuf, kl, q, u);
            }
        } else {
            const int total = CP * nk;
            for (int idx = tid; idx < total; idx += kTileThreads) {
                const int c = idx / nk;
                const int kl = idx - c * nk;
                double val = 0.0;
                if (c < a.cols) {
                    const int64_t k = k0 + kl;
                    const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
                    val = __ldcs(a.v + static_cast<int64_t>(c) * a.n + o);
                }
                St::at(ubuf, kl, c) = static_cast<T>(val);
            }
        }
        for (int kl = tid; kl < nk; kl += kTileThreads)
            wbuf[kl] = a.wp ? a.wp[k0 + kl] : static_cast<T>(1);
        if (MODE == kFinal) {
            __syncthreads();
            for (int kl = g; kl < nk; kl += GPB) {
                Acc4 u, val;
                gather_u(a, k0 + kl, q, u);
                St::load4(ubuf, kl, q, val);
#pragma unroll
                for (int j = 0; j < 4; ++j) val.v[j] -= u.v[j];
                St::store4(ubuf, kl, q, val);
            }
        }
        __syncthreads();
        // ---- phase B: segment means; ubuf <- z (kMatvec/kRhs) or d (kFinal)
        for (int32_t s = s0 + g; s < s1; s += GPB) {
            const int b = static_cast<int>(a.seg_off[s] - k0);
            const int e = static_cast<int>(a.seg_off[s + 1] - k0);
            Acc4 acc;
            acc_zero(acc);
            for (int kl = b; kl < e; ++kl) {
                Acc4 val;
                St::load4(ubuf, kl, q, val);
                const double w = static_cast<double>(wbuf[kl]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc.v[j] = fma(w, val.v[j], acc.v[j]);
                    if (MODE == kRhs) colsq[j] = fma(val.v[j], val.v[j], colsq[j]);
                }
            }
            const double iw = a.inv_wp[s];
            Acc4 zs;
            acc_zero(zs);
            for (int kl = b; kl < e; ++kl) {
                Acc4 val;
                St::load4(ubuf, kl, q, val);
                const double w = static_cast<double>(wbuf[kl]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double d = val.v[j] - acc.v[j] * iw;
                    val.v[j] = (MODE == kFinal) ? d : w * d;
                    if (MODE == kFinal) zs.v[j] = fma(w, d, zs.v[j]);
                }
                St::store4(ubuf, kl, q, val);
            }
            if (MODE == kFinal) {
#pragma unroll
                for (int j = 0; j < 4; ++j) colsq[j] = fma(zs.v[j], zs.v[j], colsq[j]);
            }
        }
        __syncthreads();
        // ---- phase C: runs of the large dims -----------------------------
        if (scatter) {
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l) {
                if (l >= a.nL) continue;
                const int32_t rb = a.run_base[l][s0], re = a.run_base[l][s1];
                for (int32_t m = rb + g; m < re; m += GPB) {
                    const int b = static_cast<int>(a.run_start[l][m] - k0);
                    const int e = static_cast<int>(a.run_start[l][m + 1] - k0);
                    Acc4 acc;
                    acc_zero(acc);
                    for (int kl = b; kl < e; ++kl) {
                        Acc4 z;
                        St::load4(ubuf, kl, q, z);
                        const double w = (MODE == kFinal) ? static_cast<double>(wbuf[kl]) : 1.0;
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc.v[j] = fma(w, z.v[j], acc.v[j]);
                    }
                    store_quad_stream(a.R[l] + static_cast<int64_t>(a.run_dest[l][m]) * CP + 4 * q,
                                      acc);
                }
            }
            // ---- phase C': small-dim bins, warp-private, fixed order ------
            // A warp step covers 32/CP consecutive observations, one per
            // group of CP lanes (lane = column).  Groups with the same level
            // are summed in group order by the first of them, which then
            // updates the warp's bin row once.
            if (a.nS > 0) {
                constexpr int G = 32 / CP;
                const int gi = lane / CP;
                const int c = lane % CP;
                const int per_warp = (nk + (kTileThreads / 32) - 1) / (kTileThreads / 32);
                const int wb = warp * per_warp;
                const int we = min(nk, wb + per_warp);
                for (int base = wb; base < we; base += G) {
                    const int kl = base + gi;
                    const bool valid = kl < we;
                    const uint32_t packed = valid ? __ldg(a.sid + k0 + kl) : 0u;
                    for (int s = 0; s < a.nS; ++s) {
                        const uint32_t key = valid ? ((packed >> (8 * s)) & 0xffu) : 0x100u + gi;
                        const unsigned int match = __match_any_sync(0xffffffffu, key);
                        if (valid && (__ffs(match) - 1) / CP == gi) {
                            double acc = 0.0;
#pragma unroll
                            for (int g2 = 0; g2 < G; ++g2) {
                                if (match & (1u << (g2 * CP))) {
                                    const int kj = base + g2;
                                    const double w =
                                        (MODE == kFinal) ? static_cast<double>(wbuf[kj]) : 1.0;
                                    acc = fma(w, static_cast<double>(St::at(ubuf, kj, c)), acc);
                                }
                            }
                            my_bins[(a.sgoff[s] + static_cast<int>(key)) * BROW + c] += acc;
                        }
                        __syncwarp();
                    }
                }
            }
        }
        // ---- phase D: write the within transform -------------------------
        if (MODE == kFinal) {
            const int total = a.cols * nk;
            for (int idx = tid; idx < total; idx += kTileThreads) {
                const int c = idx / nk;
                const int kl = idx - c * nk;
                const int64_t k = k0 + kl;
                const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
                __stcs(a.out + static_cast<int64_t>(c) * a.n + o,
                       static_cast<double>(St::at(ubuf, kl, c)));
            }
        }
    }
    __syncthreads();
    const int cta = a.bins_cta0 + blockIdx.x;
    if (a.nS > 0 && scatter) {
        double* dst = a.bins_partial + static_cast<int64_t>(cta) * a.SG * CP;
        for (int i = tid; i < a.SG * CP; i += kTileThreads) {
            const int r = i / CP, c = i - r * CP;
            double s = 0.0;
            for (int w = 0; w < kTileThreads / 32; ++w) s += bins[(w * a.SG + r) * BROW + c];
            dst[i] = s;
        }
    }
    if (MODE == kRhs || MODE == kFinal) {
        for (int j = 0; j < 4; ++j) red[tid * 4 + j] = colsq[j];
        __syncthreads();
        if (tid < CQ) {
            double s4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = tid; t < kTileThreads; t += CQ)
                for (int j = 0; j < 4; ++j) s4[j] += red[t * 4 + j];
            for (int j = 0; j < 4; ++j)
                a.colsq_partial[static_cast<int64_t>(cta) * CP + 4 * tid + j] = s4[j];
        }
    }
}

// ---------------------------------------------------------------------------
// Block-level matvec (at most one large and one small non-primary dim).
//
// A run is a maximal block of obs of one primary segment s with the same
// large-dim group f; a run is cut into blocks of obs whose small-dim levels
// are consecutive (h0, h0+1, ..., h0+len-1) and whose weights are equal (w_b).
// With P the prefix sums of the small-dim rows of x (P[h] = sum_{h'<h} x_y[h']):
//     U_m  = c_m x_f[f_m] + sum_{b in m} w_b (P[h0_b + len_b] - P[h0_b])
//     t_s  = sum_{m in s} U_m / W_s
//     R_m  = U_m - c_m t_s                               (run row of S x)
// and each block adds w_b (x_f[f_m] - t_s) to the small-dim bins of levels
// h0_b .. h0_b + len_b - 1 (a difference-array update at two points); the
// diagonal part W_h x_y[h] of the small rows is added by finalize.  Work is
// per run and per block, not per observation.  A matched panel observed in
// consecutive years has about one block per run.
// ---------------------------------------------------------------------------
constexpr int kBlockThreads = 128;

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

template <typename T>
struct BlockArgs {
    int32_t Gp;
    int CP;
    int has_large;          // one large dim: runs carry x_f and write R rows
    int has_small;          // one small dim
    int SG;                 // its levels
    const int2* seg_meta;   // [Gp+1] {first obs, first run}
    const double* inv_wp;   // [Gp]
    const int4* run_meta;   // [nruns] {group, dest row, first block, end block}
    const T* run_w;         // [nruns] run weights c_m
    const int2* block_meta; // [nblocks] {first small level, length}
    const T* block_w;       // [nblocks] or null (unit weights)
    int64_t lbase;          // alpha row of the large dim
    int64_t sbase;          // alpha row of small level 0
    const T* x;             // alpha [GR][CP]
    T* R;                   // [nruns][CP]
    double* bins_partial;   // [ctas][SG][CP]
    int bins_cta0;
    int all_segs;           // 1: long segments too (no segment kernel follows)
};

template <typename T>
__host__ __device__ size_t block_smem_bytes(int CP, int SG) {
    return align16(static_cast<size_t>(SG + 1) * CP * sizeof(T)) +
           static_cast<size_t>(kBlockThreads / 32) * (SG + 1) * CP * sizeof(double);
}

// 4-wide vector in the solve's own precision (float math for the FP32 inner
// solve, double for the FP64 refinement).
template <typename T>
struct V4 {
    T v[4];
};
template <typename T>
__device__ __forceinline__ void v4_zero(V4<T>& a) {
#pragma unroll
    for (int j = 0; j < 4; ++j) a.v[j] = static_cast<T>(0);
}
__device__ __forceinline__ void v4_load(const float* p, V4<float>& o) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    o.v[0] = t.x; o.v[1] = t.y; o.v[2] = t.z; o.v[3] = t.w;
}
__device__ __forceinline__ void v4_load(const double* p, V4<double>& o) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o.v[0] = a.x; o.v[1] = a.y; o.v[2] = b.x; o.v[3] = b.y;
}
__device__ __forceinline__ void v4_lds(const float* p, V4<float>& o) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o.v[0] = t.x; o.v[1] = t.y; o.v[2] = t.z; o.v[3] = t.w;
}
__device__ __forceinline__ void v4_lds(const double* p, V4<double>& o) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    o.v[0] = a.x; o.v[1] = a.y; o.v[2] = b.x; o.v[3] = b.y;
}
__device__ __forceinline__ void v4_store_stream(float* p, const V4<float>& a) {
    __stcs(reinterpret_cast<float4*>(p), make_float4(a.v[0], a.v[1], a.v[2], a.v[3]));
}
__device__ __forceinline__ void v4_store_stream(double* p, const V4<double>& a) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(a.v[0], a.v[1]));
    __stcs(reinterpret_cast<double2*>(p) + 1, make_double2(a.v[2], a.v[3]));
}

// Adds +delta (side 0) or -delta (side 1) to row `key` of the warp's
// difference array.  Groups with distinct keys update in parallel; groups
// sharing a key update one after another in group order (deterministic).
template <typename T, int CQ>
__device__ __forceinline__ void diff_update(double* wD, int CP, int key, bool active, int gw,
                                            int lane, int q, const V4<T>& delta, bool negate) {
    const uint32_t k = active ? static_cast<uint32_t>(key) : 0x10000u + gw;
    const unsigned int match = __match_any_sync(0xffffffffu, k);
    double* row = wD + key * CP + 4 * q;
    if (__all_sync(0xffffffffu, __popc(match) == CQ)) {
        if (active) {
#pragma unroll
            for (int i = 0; i < 4; ++i) row[i] += negate ? -static_cast<double>(delta.v[i])
                                                         : static_cast<double>(delta.v[i]);
        }
        return;
    }
    const int rank = __popc(match & ((1u << lane) - 1u)) / CQ;
    const int msize = static_cast<int>(
        __reduce_max_sync(0xffffffffu, static_cast<unsigned>(__popc(match) / CQ)));
    for (int r = 0; r < msize; ++r) {
        if (active && rank == r) {
#pragma unroll
            for (int i = 0; i < 4; ++i) row[i] += negate ? -static_cast<double>(delta.v[i])
                                                         : static_cast<double>(delta.v[i]);
        }
        __syncwarp();
    }
}

template <typename T, int CQ>
__global__ void __launch_bounds__(kBlockThreads)
block_pass_kernel(const BlockArgs<T> a) {
    constexpr int CP = 4 * CQ;
    constexpr int GPW = 32 / CQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int SG1 = a.SG + 1;
    T* P = reinterpret_cast<T*>(smem_raw);
    double* D = reinterpret_cast<double*>(smem_raw + align16(static_cast<size_t>(SG1) * CP * sizeof(T)));
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int gw = lane / CQ;
    const int q = lane % CQ;
    if (a.has_small) {
        // prefix sums of the small-dim rows of x, one column per thread
        for (int c = tid; c < CP; c += kBlockThreads) {
            double acc = 0.0;
            P[c] = static_cast<T>(0);
            for (int h = 0; h < a.SG; ++h) {
                acc += static_cast<double>(a.x[(a.sbase + h) * CP + c]);
                P[(h + 1) * CP + c] = static_cast<T>(acc);
            }
        }
        for (int i = tid; i < (kBlockThreads / 32) * SG1 * CP; i += kBlockThreads) D[i] = 0.0;
    }
    __syncthreads();
    double* wD = D + warp * SG1 * CP;
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (kBlockThreads / 32);
    const int64_t wid = static_cast<int64_t>(blockIdx.x) * (kBlockThreads / 32) + warp;

    for (int64_t s0 = wid * GPW; s0 < a.Gp; s0 += nwarps * GPW) {
        const int64_t s = s0 + gw;
        int rb = 0, re = 0;
        T iw = static_cast<T>(0);
        if (s < a.Gp) {
            const int2 m0 = a.seg_meta[s], m1 = a.seg_meta[s + 1];
            if (a.all_segs || m1.x - m0.x <= kLongSeg) {  // else the long path
                rb = m0.y;
                re = m1.y;
            }
            iw = static_cast<T>(a.inv_wp[s]);
        }
        // pass 1 (per group): t = sum_m U_m / W_s
        V4<T> tsum;
        v4_zero(tsum);
        int bfirst = 0, bend = 0;
        if (re > rb) {
            bfirst = a.run_meta[rb].z;
            bend = a.run_meta[re - 1].w;
        }
        if (a.has_large) {
            for (int m = rb; m < re; ++m) {
                const int f = a.run_meta[m].x;
                const T cm = a.run_w[m];
                V4<T> xf;
                v4_load(a.x + (a.lbase + f) * CP + 4 * q, xf);
#pragma unroll
                for (int i = 0; i < 4; ++i) tsum.v[i] = fma(cm, xf.v[i], tsum.v[i]);
            }
        }
        if (a.has_small) {
            for (int b = bfirst; b < bend; ++b) {
                const int2 bm = a.block_meta[b];
                const T wb = a.block_w ? a.block_w[b] : static_cast<T>(1);
                V4<T> p0, p1;
                v4_lds(P + bm.x * CP + 4 * q, p0);
                v4_lds(P + (bm.x + bm.y) * CP + 4 * q, p1);
#pragma unroll
                for (int i = 0; i < 4; ++i) tsum.v[i] = fma(wb, p1.v[i] - p0.v[i], tsum.v[i]);
            }
        }
        V4<T> t;
#pragma unroll
        for (int i = 0; i < 4; ++i) t.v[i] = tsum.v[i] * iw;

        if (!a.has_small) {
            // no small dim: one R row per run, R_m = c_m (x_f - t)
            for (int m = rb; m < re && a.has_large; ++m) {
                const int4 rm = a.run_meta[m];
                const T cm = a.run_w[m];
                V4<T> xf, r;
                v4_load(a.x + (a.lbase + rm.x) * CP + 4 * q, xf);
#pragma unroll
                for (int i = 0; i < 4; ++i) r.v[i] = cm * (xf.v[i] - t.v[i]);
                v4_store_stream(a.R + static_cast<int64_t>(rm.y) * CP + 4 * q, r);
            }
            continue;
        }
        // pass 2: warp-synchronous over this segment's blocks
        const int nb = bend - bfirst;
        const int steps = static_cast<int>(__reduce_max_sync(0xffffffffu, static_cast<unsigned>(nb)));
        int m = rb;
        int run_bend = 0, rdest = 0;
        T cm = static_cast<T>(0);
        V4<T> xf, U;
        v4_zero(xf);
        v4_zero(U);
        if (nb > 0) {
            const int4 rm = a.run_meta[m];
            run_bend = rm.w;
            rdest = rm.y;
            if (a.has_large) {
                cm = a.run_w[m];
                v4_load(a.x + (a.lbase + rm.x) * CP + 4 * q, xf);
            }
        }
        for (int step = 0; step < steps; ++step) {
            const bool active = step < nb;
            const int b = bfirst + step;
            int h0 = 0, h1 = 0;
            V4<T> delta;
            v4_zero(delta);
            if (active) {
                if (b == run_bend) {  // the current run is complete
                    if (a.has_large) {
                        V4<T> r;
#pragma unroll
                        for (int i = 0; i < 4; ++i) r.v[i] = fma(cm, xf.v[i] - t.v[i], U.v[i]);
                        v4_store_stream(a.R + static_cast<int64_t>(rdest) * CP + 4 * q, r);
                    }
                    ++m;
                    const int4 rm = a.run_meta[m];
                    run_bend = rm.w;
                    rdest = rm.y;
                    if (a.has_large) {
                        cm = a.run_w[m];
                        v4_load(a.x + (a.lbase + rm.x) * CP + 4 * q, xf);
                    }
                    v4_zero(U);
                }
                const int2 bm = a.block_meta[b];
                const T wb = a.block_w ? a.block_w[b] : static_cast<T>(1);
                h0 = bm.x;
                h1 = bm.x + bm.y;
                V4<T> p0, p1;
                v4_lds(P + h0 * CP + 4 * q, p0);
                v4_lds(P + h1 * CP + 4 * q, p1);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    U.v[i] = fma(wb, p1.v[i] - p0.v[i], U.v[i]);
                    delta.v[i] = wb * (xf.v[i] - t.v[i]);
                }
            }
            diff_update<T, CQ>(wD, CP, h0, active, gw, lane, q, delta, false);
            diff_update<T, CQ>(wD, CP, h1, active, gw, lane, q, delta, true);
        }
        if (nb > 0 && a.has_large) {
            V4<T> r;
#pragma unroll
            for (int i = 0; i < 4; ++i) r.v[i] = fma(cm, xf.v[i] - t.v[i], U.v[i]);
            v4_store_stream(a.R + static_cast<int64_t>(rdest) * CP + 4 * q, r);
        }
    }
    __syncthreads();
    if (a.has_small) {
        // bins = prefix sums of the difference arrays, warps summed in order
        double* dst = a.bins_partial + static_cast<int64_t>(a.bins_cta0 + blockIdx.x) * a.SG * CP;
        for (int c = tid; c < CP; c += kBlockThreads) {
            double run = 0.0;
            for (int h = 0; h < a.SG; ++h) {
                double d = 0.0;
                for (int w = 0; w < kBlockThreads / 32; ++w) d += D[(w * SG1 + h) * CP + c];
                run += d;
                dst[h * CP + c] = run;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Run-level matvec for one large dim and no small dim in the pass (two-way
// panels, and the coupled matvec, where the small dim enters through its
// dense coupling rows):  t_s = sum_{m in s} c_m x_f[f_m] / W_s,
// R_m = c_m (x_f[f_m] - t_s).  A group of CQ lanes owns one primary segment;
// runs are fetched NB at a time (independent loads in flight) and the first
// NB are kept in registers for the second pass.
// ---------------------------------------------------------------------------
template <typename T, int CQ, int NB>
__global__ void __launch_bounds__(kBlockThreads)
run_pass_kernel(const BlockArgs<T> a) {
    constexpr int CP = 4 * CQ;
    constexpr int GPW = 32 / CQ;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gw = lane / CQ;
    const int q = lane % CQ;
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (kBlockThreads / 32);
    const int64_t wid = static_cast<int64_t>(blockIdx.x) * (kBlockThreads / 32) + warp;
    for (int64_t s0 = wid * GPW; s0 < a.Gp; s0 += nwarps * GPW) {
        const int64_t s = s0 + gw;
        if (s >= a.Gp) continue;
        const int2 m0 = a.seg_meta[s], m1 = a.seg_meta[s + 1];
        if (!a.all_segs && m1.x - m0.x > kLongSeg) continue;  // the long path takes it
        const int rb = m0.y, re = m1.y;
        const T iw = static_cast<T>(a.inv_wp[s]);
        V4<T> xc[NB];
        T cc[NB];
        int dc[NB];
        V4<T> tsum;
        v4_zero(tsum);
        for (int m = rb; m < re; m += NB) {
            int4 rm[NB];
            T cm[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                if (m + u < re) {
                    rm[u] = a.run_meta[m + u];
                    cm[u] = a.run_w[m + u];
                } else {
                    rm[u] = make_int4(0, 0, 0, 0);
                    cm[u] = static_cast<T>(0);
                }
            }
            V4<T> xv[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                if (m + u < re) v4_load(a.x + (a.lbase + rm[u].x) * CP + 4 * q, xv[u]);
                else v4_zero(xv[u]);
            }
#pragma unroll
            for (int u = 0; u < NB; ++u)
#pragma unroll
                for (int i = 0; i < 4; ++i) tsum.v[i] = fma(cm[u], xv[u].v[i], tsum.v[i]);
            if (m == rb) {
#pragma unroll
                for (int u = 0; u < NB; ++u) {
                    xc[u] = xv[u];
                    cc[u] = cm[u];
                    dc[u] = rm[u].y;
                }
            }
        }
        V4<T> t;
#pragma unroll
        for (int i = 0; i < 4; ++i) t.v[i] = tsum.v[i] * iw;
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            if (rb + u < re) {
                V4<T> r;
#pragma unroll
                for (int i = 0; i < 4; ++i) r.v[i] = cc[u] * (xc[u].v[i] - t.v[i]);
                v4_store_stream(a.R + static_cast<int64_t>(dc[u]) * CP + 4 * q, r);
            }
        }
        for (int m = rb + NB; m < re; ++m) {  // runs beyond the first NB
            const int4 rm = a.run_meta[m];
            const T cm = a.run_w[m];
            V4<T> xf, r;
            v4_load(a.x + (a.lbase + rm.x) * CP + 4 * q, xf);
#pragma unroll
            for (int i = 0; i < 4; ++i) r.v[i] = cm * (xf.v[i] - t.v[i]);
            v4_store_stream(a.R + static_cast<int64_t>(rm.y) * CP + 4 * q, r);
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 data passes (kRhs, kFinal) over tiles of whole segments, lane = column.
//
// A group of CP lanes (one per column) owns one segment, run or observation at
// a time; the tile's columns are staged column-major in shared memory, so the
// coalesced column loads/stores and the per-column reductions are free of
// bank conflicts.  Everything a later phase indexes by observation or run
// (large-dim ids, packed small-dim ids, run offsets and destination rows) is
// staged in the same coalesced first phase, so the serial per-group loops
// after it touch only shared memory and the gathered alpha rows (L2), and no
// global load waits on another.  Same outputs as tile_pass_kernel in these
// modes.
// ---------------------------------------------------------------------------
constexpr int kDataThreads = 256;

__host__ __device__ constexpr size_t data_smem_bytes(int CP, int SG, int nL) {
    return static_cast<size_t>(CP) * (kTileObs + 1) * sizeof(double)     // staged columns
           + static_cast<size_t>(kTileObs) * sizeof(double)              // weights
           + static_cast<size_t>(kDataThreads / 32) * SG * CP * sizeof(double)  // bins
           + static_cast<size_t>(kTileObs) * sizeof(uint32_t)            // packed small ids
           + static_cast<size_t>(nL) * kTileObs * sizeof(int32_t)        // large-dim ids
           + static_cast<size_t>(nL) * kTileObs * sizeof(int32_t)        // run rows in R
           + static_cast<size_t>(nL) * (kTileObs + 2) * sizeof(uint16_t);  // run offsets
}

template <int CP, int MODE>
__global__ void __launch_bounds__(kDataThreads, 2)
data_pass_kernel(const PassArgs<double> a) {
    constexpr int LD = kTileObs + 1;
    constexpr int GPB = kDataThreads / CP;  // lane groups per block
    constexpr int G = 32 / CP;              // lane groups per warp
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* ubuf = reinterpret_cast<double*>(smem_raw);
    double* wbuf = ubuf + CP * LD;
    double* bins = wbuf + kTileObs;
    uint32_t* sidbuf = reinterpret_cast<uint32_t*>(bins + (kDataThreads / 32) * a.SG * CP);
    int32_t* ridbuf = reinterpret_cast<int32_t*>(sidbuf + kTileObs);  // [nL][kTileObs]
    int32_t* dstbuf = ridbuf + a.nL * kTileObs;                        // [nL][kTileObs]
    uint16_t* offbuf = reinterpret_cast<uint16_t*>(dstbuf + a.nL * kTileObs);  // [nL][kTileObs+2]
    double* red = ubuf;  // colsq reduction, after the tile loop
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = tid / CP;   // group in block
    const int gi = lane / CP; // group in warp
    const int c = tid % CP;   // column of this lane
    const bool scatter = (MODE != kFinal) || a.scatter;
    double* my_bins = bins + warp * a.SG * CP;
    for (int i = tid; i < (kDataThreads / 32) * a.SG * CP; i += kDataThreads) bins[i] = 0.0;
    double colsq = 0.0;

    // Tile pipeline: the next regular tile's bounds are read at the top of an
    // iteration, and (RHS pass) its columns, weights, ids and run tables are
    // loaded into registers right after the current tile is committed to
    // shared memory, so those loads are in flight while the current tile is
    // worked on.  Thread tid holds observations tid and tid + kDataThreads of
    // a tile and run table entries tid + u * kDataThreads, u < 3.
    static_assert(kTileObs <= 2 * kDataThreads, "at most two observations per thread");
    struct Meta {
        int32_t s0, s1;
        int64_t k0;
        int nk;
        int32_t rb[kMaxLarge], nr[kMaxLarge];
    };
    auto next_tile = [&](int64_t t) {
        while (t < a.ntiles && a.tile_long[t]) t += gridDim.x;
        return t;
    };
    auto load_meta = [&](int64_t t, Meta& m) {
        m.s0 = a.tile_seg[t];
        m.s1 = a.tile_seg[t + 1];
        m.k0 = a.seg_off[m.s0];
        m.nk = static_cast<int>(a.seg_off[m.s1] - m.k0);
#pragma unroll
        for (int l = 0; l < kMaxLarge; ++l) {
            m.rb[l] = (l < a.nL && scatter) ? a.run_base[l][m.s0] : 0;
            m.nr[l] = (l < a.nL && scatter) ? a.run_base[l][m.s1] - m.rb[l] : 0;
        }
    };
    double pv[2][CP];
    double pw[2];
    uint32_t ps[2];
    int32_t po[3][kMaxLarge], pd[3][kMaxLarge];
    auto prefetch = [&](const Meta& m) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int kl = tid + u * kDataThreads;
            if (kl < m.nk) {
                const int64_t k = m.k0 + kl;
                const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
#pragma unroll
                for (int cc = 0; cc < CP; ++cc)
                    pv[u][cc] = cc < a.cols ? __ldcs(a.v + static_cast<int64_t>(cc) * a.n + o) : 0.0;
                pw[u] = a.wp ? a.wp[k] : 1.0;
                ps[u] = a.nS > 0 ? __ldg(a.sid + k) : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int j = tid + u * kDataThreads;
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l) {
                if (l < a.nL && scatter && j <= m.nr[l]) {
                    po[u][l] = __ldg(a.run_start[l] + m.rb[l] + j) - static_cast<int32_t>(m.k0);
                    pd[u][l] = j < m.nr[l] ? __ldg(a.run_dest[l] + m.rb[l] + j) : 0;
                }
            }
        }
    };
    auto commit = [&](const Meta& m) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int kl = tid + u * kDataThreads;
            if (kl < m.nk) {
#pragma unroll
                for (int cc = 0; cc < CP; ++cc) ubuf[cc * LD + kl] = pv[u][cc];
                wbuf[kl] = pw[u];
                sidbuf[kl] = ps[u];
            }
        }
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int j = tid + u * kDataThreads;
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l) {
                if (l < a.nL && scatter && j <= m.nr[l]) {
                    offbuf[l * (kTileObs + 2) + j] = static_cast<uint16_t>(po[u][l]);
                    if (j < m.nr[l]) dstbuf[l * kTileObs + j] = pd[u][l];
                }
            }
        }
    };
    // direct staging (final pass): each value goes to shared memory as loaded
    auto stage_direct = [&](const Meta& m) {
        for (int kl = tid; kl < m.nk; kl += kDataThreads) {
            const int64_t k = m.k0 + kl;
            const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
#pragma unroll
            for (int cc = 0; cc < CP; ++cc)
                ubuf[cc * LD + kl] = cc < a.cols ? __ldcs(a.v + static_cast<int64_t>(cc) * a.n + o) : 0.0;
            wbuf[kl] = a.wp ? a.wp[k] : 1.0;
            if (a.nS > 0) sidbuf[kl] = __ldg(a.sid + k);
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l)
                if (l < a.nL) ridbuf[l * kTileObs + kl] = __ldg(a.rid[l] + k);
        }
#pragma unroll
        for (int l = 0; l < kMaxLarge; ++l) {
            if (l >= a.nL || !scatter) continue;
            for (int j = tid; j <= m.nr[l]; j += kDataThreads) {
                offbuf[l * (kTileObs + 2) + j] =
                    static_cast<uint16_t>(__ldg(a.run_start[l] + m.rb[l] + j) - m.k0);
                if (j < m.nr[l]) dstbuf[l * kTileObs + j] = __ldg(a.run_dest[l] + m.rb[l] + j);
            }
        }
    };

    // The register pipeline pays in the RHS pass; the final pass (more
    // registers for the gather) stages its tile after the barrier instead and
    // keeps only the one-tile-ahead bounds.
    constexpr bool kPipe = MODE == kRhs;
    Meta cur{}, nxt{};
    int64_t t = next_tile(blockIdx.x);
    if (t < a.ntiles) {
        load_meta(t, cur);
        if (kPipe) prefetch(cur);
    }
    while (t < a.ntiles) {
        const int64_t tn = next_tile(t + gridDim.x);
        if (tn < a.ntiles) load_meta(tn, nxt);
        __syncthreads();  // the previous tile is done with shared memory
        if constexpr (kPipe) {
            commit(cur);
            if (tn < a.ntiles) prefetch(nxt);
        } else {
            stage_direct(cur);
        }
        const int32_t s0 = cur.s0, s1 = cur.s1;
        const int64_t k0 = cur.k0;
        const int nk = cur.nk;
        int32_t nr[kMaxLarge];
#pragma unroll
        for (int l = 0; l < kMaxLarge; ++l) nr[l] = cur.nr[l];
        if (MODE == kFinal) {
            __syncthreads();
            // v - D_r a: one alpha row per lane group; the ids come from shared
            // memory, so the unrolled loads of several observations overlap
#pragma unroll 4
            for (int kl = g; kl < nk; kl += GPB) {
                double u = 0.0;
#pragma unroll
                for (int l = 0; l < kMaxLarge; ++l)
                    if (l < a.nL) u += __ldg(a.x + (a.lbase[l] + ridbuf[l * kTileObs + kl]) * CP + c);
                if (a.nS > 0) {
                    const uint32_t packed = sidbuf[kl];
                    for (int s = 0; s < a.nS; ++s)
                        u += __ldg(a.x + (a.sbase[s] + ((packed >> (8 * s)) & 0xffu)) * CP + c);
                }
                ubuf[c * LD + kl] -= u;
            }
        }
        __syncthreads();
        // ---- segment means; ubuf <- z (kRhs) or d (kFinal) -----------------
        for (int32_t s = s0 + g; s < s1; s += GPB) {
            const int b = static_cast<int>(a.seg_off[s] - k0);
            const int e = static_cast<int>(a.seg_off[s + 1] - k0);
            double acc = 0.0;
            for (int kl = b; kl < e; ++kl) {
                const double val = ubuf[c * LD + kl];
                acc = fma(wbuf[kl], val, acc);
                if (MODE == kRhs) colsq = fma(val, val, colsq);
            }
            const double mean = acc * a.inv_wp[s];
            if (MODE == kFinal && a.mean_out) a.mean_out[static_cast<int64_t>(s) * CP + c] = mean;
            double zs = 0.0;
            for (int kl = b; kl < e; ++kl) {
                const double d = ubuf[c * LD + kl] - mean;
                const double w = wbuf[kl];
                ubuf[c * LD + kl] = (MODE == kFinal) ? d : w * d;
                if (MODE == kFinal) zs = fma(w, d, zs);
            }
            if (MODE == kFinal) colsq = fma(zs, zs, colsq);
        }
        __syncthreads();
        if (scatter) {
            // ---- runs of the large dims ---------------------------------------
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l) {
                if (l >= a.nL) continue;
                const uint16_t* off = offbuf + l * (kTileObs + 2);
                const int32_t* dst = dstbuf + l * kTileObs;
                for (int j = g; j < nr[l]; j += GPB) {
                    const int b = off[j], e = off[j + 1];
                    double acc = 0.0;
                    for (int kl = b; kl < e; ++kl)
                        acc = fma((MODE == kFinal) ? wbuf[kl] : 1.0, ubuf[c * LD + kl], acc);
                    __stcs(a.R[l] + static_cast<int64_t>(dst[j]) * CP + c, acc);
                }
            }
            // ---- small-dim bins (warp-private, groups with equal levels summed
            //      in group order by the first of them) ---------------------------
            if (a.nS > 0) {
                const int per_warp = (nk + (kDataThreads / 32) - 1) / (kDataThreads / 32);
                const int wb = warp * per_warp;
                const int we = min(nk, wb + per_warp);
                for (int base = wb; base < we; base += G) {
                    const int kl = base + gi;
                    const bool valid = kl < we;
                    const uint32_t packed = valid ? sidbuf[kl] : 0u;
                    for (int s = 0; s < a.nS; ++s) {
                        const uint32_t key = valid ? ((packed >> (8 * s)) & 0xffu) : 0x100u + gi;
                        const unsigned int match = __match_any_sync(0xffffffffu, key);
                        if (valid && (__ffs(match) - 1) / CP == gi) {
                            double acc = 0.0;
#pragma unroll
                            for (int g2 = 0; g2 < G; ++g2) {
                                if (match & (1u << (g2 * CP))) {
                                    const int kj = base + g2;
                                    acc = fma((MODE == kFinal) ? wbuf[kj] : 1.0, ubuf[c * LD + kj], acc);
                                }
                            }
                            my_bins[(a.sgoff[s] + static_cast<int>(key)) * CP + c] += acc;
                        }
                        __syncwarp();
                    }
                }
            }
        }
        // ---- write the within transform (coalesced) ---------------------------
        if (MODE == kFinal) {
            for (int kl = tid; kl < nk; kl += kDataThreads) {
                const int64_t k = k0 + kl;
                const int64_t o = a.pord ? static_cast<int64_t>(a.pord[k]) : k;
#pragma unroll
                for (int cc = 0; cc < CP; ++cc)
                    if (cc < a.cols) __stcs(a.out + static_cast<int64_t>(cc) * a.n + o, ubuf[cc * LD + kl]);
            }
        }
        cur = nxt;
        t = tn;
    }
    __syncthreads();
    const int cta = a.bins_cta0 + blockIdx.x;
    if (a.nS > 0 && scatter) {
        double* dst = a.bins_partial + static_cast<int64_t>(cta) * a.SG * CP;
        for (int i = tid; i < a.SG * CP; i += kDataThreads) {
            double sum = 0.0;
            for (int w = 0; w < kDataThreads / 32; ++w) sum += bins[w * a.SG * CP + i];
            dst[i] = sum;
        }
    }
    red[tid] = colsq;
    __syncthreads();
    if (tid < CP) {
        double sum = 0.0;
        for (int j = 0; j < GPB; ++j) sum += red[j * CP + tid];
        a.colsq_partial[static_cast<int64_t>(cta) * CP + tid] = sum;
    }
}

// Long segments: one group of CQ lanes walks one listed segment serially.
// Correct for any length; used only for the few segments longer than
// kLongSeg, which do not fit a tile.
template <typename T, int MODE>
__device__ __forceinline__ void seg_value(const PassArgs<T>& a, int64_t k, int q, Acc4& val) {
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
        gather_u(a, k, q, u);
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
segment_pass_kernel(const PassArgs<T> a) {
    extern __shared__ double smem_bins[];  // [warps][SG][CP], then colsq red
    constexpr int GPW = 32 / CQ;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gw = lane / CQ;
    const int q = lane % CQ;
    const int warps_per_block = kPassThreads / 32;
    const int bin_stride = a.SG * a.CP;
    double* my_bins = smem_bins + warp * bin_stride;
    const bool scatter = (MODE != kFinal) || a.scatter;
    for (int i = threadIdx.x; i < warps_per_block * bin_stride; i += kPassThreads)
        smem_bins[i] = 0.0;
    __syncthreads();
    double colsq[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t total_warps = static_cast<int64_t>(gridDim.x) * warps_per_block;
    const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * warps_per_block + warp;
    for (int64_t i0 = warp_id * GPW; i0 < a.nlong; i0 += total_warps * GPW) {
        const int64_t li = i0 + gw;
        const bool valid = li < a.nlong;
        const int32_t s = valid ? a.long_segs[li] : 0;
        int64_t beg = 0, len = 0;
        double inv_w = 0.0;
        if (valid) {
            beg = a.seg_off[s];
            len = a.seg_off[s + 1] - beg;
            inv_w = a.inv_wp[s];
        }
        Acc4 acc;
        acc_zero(acc);
        for (int64_t t = 0; t < len; ++t) {
            const int64_t k = beg + t;
            Acc4 val;
            seg_value<T, MODE>(a, k, q, val);
            const double w = a.wp ? static_cast<double>(a.wp[k]) : 1.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc.v[j] = fma(w, val.v[j], acc.v[j]);
                if (MODE == kRhs) colsq[j] = fma(val.v[j], val.v[j], colsq[j]);
            }
        }
        Acc4 mean;
#pragma unroll
        for (int j = 0; j < 4; ++j) mean.v[j] = acc.v[j] * inv_w;
        if (MODE == kFinal && a.mean_out && valid) {
#pragma unroll
            for (int j = 0; j < 4; ++j) a.mean_out[static_cast<int64_t>(s) * a.CP + 4 * q + j] = mean.v[j];
        }
        int64_t steps = len;
        if (a.nS > 0 && scatter) {
            int64_t m = len;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
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
                seg_value<T, MODE>(a, k, q, val);
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
                        const int32_t gid = __ldg(a.rid[l] + k);
                        if (t > 0 && gid != prev[l]) {
                            store_quad_stream(a.R[l] + static_cast<int64_t>(a.run_dest[l][cur[l]]) * a.CP + 4 * q,
                                              racc[l]);
                            ++cur[l];
                            acc_zero(racc[l]);
                        }
                        prev[l] = gid;
#pragma unroll
                        for (int j = 0; j < 4; ++j) racc[l].v[j] += z.v[j];
                    }
                    if (a.nS > 0) packed = __ldg(a.sid + k);
                }
            }
            if (a.nS > 0 && scatter) {
                for (int j = 0; j < GPW; ++j) {
                    __syncwarp();
                    if (gw == j && active) {
                        for (int s2 = 0; s2 < a.nS; ++s2) {
                            const uint32_t h = (packed >> (8 * s2)) & 0xffu;
                            double* b = my_bins + (a.sgoff[s2] + h) * a.CP + 4 * q;
                            Acc4 zb = z;
                            if (MODE == kMatvec && a.bins_no_diag) {
                                Acc4 xh;
                                load_quad(a.x + (a.sbase[s2] + h) * a.CP + 4 * q, xh);
                                const double w = a.wp ? static_cast<double>(a.wp[k]) : 1.0;
#pragma unroll
                                for (int c = 0; c < 4; ++c) zb.v[c] -= w * xh.v[c];
                            }
#pragma unroll
                            for (int c = 0; c < 4; ++c) b[c] += zb.v[c];
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (scatter && valid && len > 0) {
#pragma unroll
            for (int l = 0; l < kMaxLarge; ++l)
                if (l < a.nL)
                    store_quad_stream(a.R[l] + static_cast<int64_t>(a.run_dest[l][cur[l]]) * a.CP + 4 * q,
                                      racc[l]);
        }
        if (MODE == kFinal && valid) {
#pragma unroll
            for (int j = 0; j < 4; ++j) colsq[j] = fma(zsum.v[j], zsum.v[j], colsq[j]);
        }
    }
    __syncthreads();
    const int cta = a.bins_cta0 + blockIdx.x;
    if (a.nS > 0 && scatter) {
        double* dst = a.bins_partial + static_cast<int64_t>(cta) * bin_stride;
        for (int i = threadIdx.x; i < bin_stride; i += kPassThreads) {
            double s = 0.0;
            for (int w = 0; w < warps_per_block; ++w) s += smem_bins[w * bin_stride + i];
            dst[i] = s;
        }
    }
    if (MODE == kRhs || MODE == kFinal) {
        __syncthreads();
        double* red = smem_bins;
        for (int j = 0; j < 4; ++j) red[threadIdx.x * 4 + j] = colsq[j];
        __syncthreads();
        if (threadIdx.x < CQ) {
            double s4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = threadIdx.x; t < kPassThreads; t += CQ)
                for (int j = 0; j < 4; ++j) s4[j] += red[t * 4 + j];
            for (int j = 0; j < 4; ++j)
                a.colsq_partial[static_cast<int64_t>(cta) * a.CP + 4 * threadIdx.x + j] = s4[j];
        }
    }
}

// ---------------------------------------------------------------------------
// Deterministic block reduction of per-column partials: out[c] = sum over
// parts p in [0, nparts) of part[p * stride + c], c < CP.  Thread t sums the
// parts p == t / CP (mod blockDim / CP) in order; a fixed tree finishes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_column_sum(const double* part, int64_t nparts,
                                                   int64_t stride, int CP, double* red) {
    const int t = threadIdx.x;
    const int J = blockDim.x / CP;
    const int c = t % CP;
    const int j = t / CP;
    double s = 0.0;
    if (j < J) {
        // eight independent accumulators keep eight loads in flight; their
        // fixed combination order keeps the sum deterministic
        double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int64_t p = j;
        for (; p + 7 * J < nparts; p += 8 * J) {
#pragma unroll
            for (int u = 0; u < 8; ++u) acc[u] += __ldcg(part + (p + u * J) * stride + c);
        }
        for (; p < nparts; p += J) acc[0] += __ldcg(part + p * stride + c);
        s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    }
    red[t] = s;
    __syncthreads();
    for (int h = J / 2; h > 0; h >>= 1) {
        if (j < h) red[t] += red[t + h * CP];
        __syncthreads();
    }
    return red[c];  // valid for every thread after the tree
}

// ---------------------------------------------------------------------------
// Run gather-sum (large dims): row of group g = sum of its runs' rows.
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
    const T* cfy;               // [G][SGP] dense coupling to the small dim, or null
    const T* xs;                // small-dim rows of the matvec input [SG][CP]
    int SG, SGP;                // levels of the small dim; row stride of cfy (SG rounded up to 4)
};

template <typename T>
__device__ __forceinline__ void load4(const T* p, T (&v)[4]);
template <>
__device__ __forceinline__ void load4<float>(const float* p, float (&v)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
template <>
__device__ __forceinline__ void load4<double>(const double* p, double (&v)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <typename T, int CQ>
__global__ void __launch_bounds__(kRowThreads)
run_gather_kernel(const GatherArgs<T> a) {
    __shared__ double red[kRowThreads][4];
    extern __shared__ __align__(16) unsigned char gsmem_raw[];
    T* xs_s = reinterpret_cast<T*>(gsmem_raw);  // [SGP][CP] small rows of x (coupled matvec)
    const int q = threadIdx.x % CQ;
    if (a.cfy) {
        for (int i = threadIdx.x; i < a.SGP * a.CP; i += kRowThreads)
            xs_s[i] = i < a.SG * a.CP ? a.xs[i] : T(0);
        __syncthreads();
    }
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
            if (a.cfy) {  // + C_fy[g] x_small, four levels per load
                const T* crow = a.cfy + static_cast<int64_t>(g) * a.SGP;
                for (int h0 = 0; h0 < a.SGP; h0 += 4) {
                    T c4[4];
                    load4<T>(crow + h0, c4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const T* xr = xs_s + (h0 + u) * a.CP + 4 * q;
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            acc.v[j] = fma(static_cast<double>(c4[u]), static_cast<double>(xr[j]), acc.v[j]);
                    }
                }
            }
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
// Finalize: one CTA per output row that needs a second reduction level
// (multi-chunk large groups, then small-dim levels); each sums its partials
// with block_column_sum.  The last CTA then reduces every dot partial
// (run_gather CTAs, then this kernel's rows) into dot_out[CP].
// ---------------------------------------------------------------------------
template <typename T>
struct FinalizeArgs {
    int CP;
    int nL, nS;
    int64_t nmulti[kMaxLarge];
    const int32_t* multi_grp[kMaxLarge];
    const int32_t* multi_c0[kMaxLarge];
    const int32_t* multi_c1[kMaxLarge];
    const double* partial[kMaxLarge];
    const int32_t* multi_s0[kMaxLarge];     // super-chunk range of each multi row (or null)
    const int32_t* multi_s1[kMaxLarge];
    const double* super_partial[kMaxLarge]; // [nsup][CP]
    int64_t lbase[kMaxLarge];
    int SG;                      // small-dim levels (bin rows)
    int64_t sgbase;              // alpha row of bin row 0 (small dims are contiguous)
    const double* bins_partial;  // [nbins_ctas][SG][CP]
    int nbins_ctas;
    const double* small_diag;    // [SG] level weights W_h to add W_h x[h] (block pass), or null
    const double* small_dense;   // [SG][SG] C_yy to add C_yy x_small (coupled matvec), or null
    const T* cfy;                // [G_0][SGP] C_fy to add C_fy x_small to large dim 0's rows, or null
    int SGP;                     // row stride of cfy
    const T* x;                  // the matvec input (for small_diag / small_dense / cfy)
    int64_t nrows;               // sum nmulti + SG
    T* out;                      // alpha rows [GR][CP]
    const T* dotv;               // or null
    double* dot_partial;         // this kernel's [gridDim][CP]
    const double* gather_dot_partial[kMaxLarge];
    int gather_ctas[kMaxLarge];
    double* dot_out;             // [CP] or null
    unsigned int* ticket;
};

constexpr int kFinFewParts = 16;  // rows with at most this many partials take one lane group
constexpr int kSuperParts = 64;   // chunk partials per super-chunk

// Super-chunks: one lane group (CP lanes) sums kSuperParts chunk partials of
// a large group with four interleaved accumulators combined in a fixed order.
__global__ void __launch_bounds__(kRowThreads)
multi_super_kernel(int64_t nsup, const int32_t* __restrict__ sup_c0, const int32_t* __restrict__ sup_c1,
                   const double* __restrict__ partial, int CP, double* __restrict__ out) {
    const int NG = kRowThreads / CP;
    const int gid = threadIdx.x / CP, c = threadIdx.x % CP;
    for (int64_t sI = static_cast<int64_t>(blockIdx.x) * NG + gid; sI < nsup;
         sI += static_cast<int64_t>(gridDim.x) * NG) {
        const int32_t b = sup_c0[sI], e = sup_c1[sI];
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int32_t j = b;
        for (; j + 4 <= e; j += 4) {
            a0 += __ldcg(partial + static_cast<int64_t>(j) * CP + c);
            a1 += __ldcg(partial + static_cast<int64_t>(j + 1) * CP + c);
            a2 += __ldcg(partial + static_cast<int64_t>(j + 2) * CP + c);
            a3 += __ldcg(partial + static_cast<int64_t>(j + 3) * CP + c);
        }
        for (; j < e; ++j) a0 += __ldcg(partial + static_cast<int64_t>(j) * CP + c);
        out[sI * CP + c] = (a0 + a1) + (a2 + a3);
    }
}

// A finalize row: its partial slots, output row and extra terms.
struct FinRow {
    const double* part;
    int64_t np, stride, orow, cgrp, small;  // small: small-dim level, or -1
};

template <typename T>
__device__ __forceinline__ FinRow fin_row(const FinalizeArgs<T>& a, int64_t r) {
    FinRow f{nullptr, 0, a.CP, -1, -1, -1};
    int64_t ri = r;
    for (int l = 0; l < a.nL && f.orow < 0; ++l) {
        if (ri < a.nmulti[l]) {
            const int32_t c0 = a.multi_c0[l][ri], c1 = a.multi_c1[l][ri];
            const int32_t s0 = a.multi_s0[l] ? a.multi_s0[l][ri] : 0;
            const int32_t s1 = a.multi_s0[l] ? a.multi_s1[l][ri] : 0;
            if (s1 > s0) {  // summed in super-chunk slices
                f.part = a.super_partial[l] + static_cast<int64_t>(s0) * a.CP;
                f.np = s1 - s0;
            } else {
                f.part = a.partial[l] + static_cast<int64_t>(c0) * a.CP;
                f.np = c1 - c0;
            }
            f.orow = a.lbase[l] + a.multi_grp[l][ri];
            if (l == 0) f.cgrp = a.multi_grp[l][ri];
        } else {
            ri -= a.nmulti[l];
        }
    }
    if (f.orow < 0) {  // small-dim level ri
        f.part = a.bins_partial + ri * a.CP;
        f.np = a.nbins_ctas;
        f.stride = static_cast<int64_t>(a.SG) * a.CP;
        f.orow = a.sgbase + ri;
        f.small = ri;
    }
    return f;
}

// The terms a row adds to its partial sum (column c), then the store and the
// dot with dotv.
template <typename T>
__device__ __forceinline__ void fin_store(const FinalizeArgs<T>& a, const FinRow& f, int c, double sum,
                                          double& dotc) {
    const int CP = a.CP;
    if (a.small_dense && f.small >= 0) {
        const double* crow = a.small_dense + f.small * a.SG;
#pragma unroll 4
        for (int h = 0; h < a.SG; ++h)
            sum = fma(crow[h], static_cast<double>(a.x[(a.sgbase + h) * CP + c]), sum);
    } else if (a.small_diag && f.small >= 0) {
        sum = fma(a.small_diag[f.small], static_cast<double>(a.x[f.orow * CP + c]), sum);
    }
    if (a.cfy && f.cgrp >= 0) {
        const T* crow = a.cfy + f.cgrp * a.SGP;
#pragma unroll 4
        for (int h = 0; h < a.SG; ++h)
            sum = fma(static_cast<double>(crow[h]), static_cast<double>(a.x[(a.sgbase + h) * CP + c]), sum);
    }
    const T stored = static_cast<T>(sum);
    a.out[f.orow * CP + c] = stored;
    if (a.dotv) dotc = fma(static_cast<double>(a.dotv[f.orow * CP + c]), static_cast<double>(stored), dotc);
}


template <typename T>
__global__ void __launch_bounds__(kRowThreads)
finalize_kernel(const FinalizeArgs<T> a) {
    __shared__ double red[kRowThreads];
    __shared__ bool last;
    const int CP = a.CP;
    const int NG = kRowThreads / CP;  // lane groups per CTA
    const int gid = threadIdx.x / CP, c = threadIdx.x % CP;
    double dotc = 0.0;  // this thread's dot contribution of column c
    // rows with few partials (most multi-chunk groups): one lane group each,
    // lane c sums column c serially in slot order
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * NG + gid; r < a.nrows;
         r += static_cast<int64_t>(gridDim.x) * NG) {
        const FinRow f = fin_row(a, r);
        if (f.np > kFinFewParts) continue;
        double sum = 0.0;
        for (int64_t p = 0; p < f.np; ++p) sum += __ldcg(f.part + p * f.stride + c);
        fin_store(a, f, c, sum, dotc);
    }
    // rows with many partials (small-dim bins, very large groups): the whole CTA
    for (int64_t r = blockIdx.x; r < a.nrows; r += gridDim.x) {
        const FinRow f = fin_row(a, r);
        if (f.np <= kFinFewParts) continue;
        const double sum = block_column_sum(f.part, f.np, f.stride, CP, red);
        if (threadIdx.x < CP) fin_store(a, f, threadIdx.x, sum, dotc);
        __syncthreads();
    }
    // this CTA's dot per column: threads of column c summed in group order
    red[threadIdx.x] = dotc;
    __syncthreads();
    if (threadIdx.x < CP) {
        double d = 0.0;
        for (int g = 0; g < NG; ++g) d += red[g * CP + threadIdx.x];
        dotc = d;
    }
    __syncthreads();
    if (!a.dot_out) return;
    if (threadIdx.x < CP) a.dot_partial[static_cast<int64_t>(blockIdx.x) * CP + threadIdx.x] = dotc;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(a.ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    double total = 0.0;
    for (int l = 0; l < a.nL; ++l) {
        total += block_column_sum(a.gather_dot_partial[l], a.gather_ctas[l], CP, CP, red);
        __syncthreads();
    }
    total += block_column_sum(a.dot_partial, gridDim.x, CP, CP, red);
    if (threadIdx.x < CP) a.dot_out[threadIdx.x] = total;
    if (threadIdx.x == 0) *a.ticket = 0u;
}

// ---------------------------------------------------------------------------
// PCG vector kernels over the alpha rows (GR x CP), per-column scalars.
// ---------------------------------------------------------------------------
struct CgScalars {
    double* rz;      // r'z
    double* pq;      // p'Sp
    double* rr;      // r'r
    double* bb;      // per-column stop threshold on r'r
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
    __shared__ double red1[kRowThreads];
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
    const double s0 = block_column_sum(sc.partial, gridDim.x, 2 * CP, CP, red1);
    __syncthreads();
    const double s1 = block_column_sum(sc.partial + CP, gridDim.x, 2 * CP, CP, red1);
    if (threadIdx.x < CP) {
        const int cc = threadIdx.x;
        const int was_active = sc.active[cc];
        if (was_active) {
            const double old = sc.rz[cc];
            sc.beta[cc] = old > 0.0 ? s0 / old : 0.0;
            sc.rz[cc] = s0;
            sc.rr[cc] = s1;
            if (iter >= 0) sc.iters[cc] += 1;  // iterations while active
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
    if (first) {  // p is not read: its memory is uninitialised before the first step
        for (int64_t i = start; i < total; i += stride) p[i] = z[i];
        return;
    }
    for (int64_t i = start; i < total; i += stride)
        p[i] = static_cast<T>(static_cast<double>(z[i]) + be * static_cast<double>(p[i]));
}

// ---------------------------------------------------------------------------
// C_fy' x_f for the coupled matvec: per CTA a contiguous range of groups of
// the large dim; thread (h, q) accumulates C_fy[g][h] x_f[g][4q..4q+3] in the
// solve precision and writes the CTA's [SG][CP] partial (summed in CTA order
// by finalize_kernel, with C_yy x_small, into the small-dim rows).
// ---------------------------------------------------------------------------
constexpr int kCoupleXfUnroll = 8;  // groups whose loads are in flight per step

template <typename T, int CQ>
__global__ void __launch_bounds__(256)
coupling_xf_kernel(int64_t G, int SG, int SGP, const T* __restrict__ cfy, const T* __restrict__ xf,
                   double* __restrict__ partial) {
    constexpr int CP = 4 * CQ;
    const int h = threadIdx.x / CQ, q = threadIdx.x % CQ;
    const int64_t per = (G + gridDim.x - 1) / gridDim.x;
    const int64_t g0 = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t g1 = min(G, g0 + per);
    if (h >= SG) return;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    int64_t g = g0;
    constexpr int U = kCoupleXfUnroll;
    for (; g + U <= g1; g += U) {  // U groups' loads in flight
        T cv[U];
        Acc4 xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            cv[u] = __ldg(cfy + (g + u) * SGP + h);
            load_quad(xf + (g + u) * CP + 4 * q, xv[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] = fma(cv[u], static_cast<T>(xv[u].v[j]), acc[j]);
    }
    for (; g < g1; ++g) {
        const T c = __ldg(cfy + g * SGP + h);
        Acc4 xv;
        load_quad(xf + g * CP + 4 * q, xv);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[j] = fma(c, static_cast<T>(xv.v[j]), acc[j]);
    }
    double* dst = partial + (static_cast<int64_t>(blockIdx.x) * SG + h) * CP + 4 * q;
#pragma unroll
    for (int j = 0; j < 4; ++j) dst[j] = static_cast<double>(acc[j]);
}


// ---------------------------------------------------------------------------
// Fixed-effect coefficients per dimension (saved FEs): column c of dimension
// d's [G_d][cols] column-major output from the alpha rows (non-primary dims)
// or the primary segment means, for the column block starting at c0.
// ---------------------------------------------------------------------------
struct FeLayoutArgs {
    int nd;
    int32_t G[kMaxDims];
    int64_t row0[kMaxDims];  // alpha row of level 0, or -1 for the primary dim
    double* out[kMaxDims];   // [G_d][cols_total] column-major
    int cols_total, c0, cb, CP;
    const double* a;         // alpha rows [GR][CP]
    const double* means;     // primary means [Gp][CP]
};

__global__ void fe_layout_kernel(const FeLayoutArgs f) {
    for (int d = 0; d < f.nd; ++d) {
        const int64_t total = static_cast<int64_t>(f.G[d]) * f.cb;
        for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
             i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
            const int c = static_cast<int>(i / f.G[d]);
            const int64_t g = i - static_cast<int64_t>(c) * f.G[d];
            const double v = f.row0[d] < 0 ? f.means[g * f.CP + c] : f.a[(f.row0[d] + g) * f.CP + c];
            f.out[d][static_cast<int64_t>(f.c0 + c) * f.G[d] + g] = v;
        }
    }
}

}  // namespace b200fe
