// Setup kernels: build the device-resident FE structure once per call (or
// once per structure when the caller reuses it).  They replace the host-side
// indexer work the reference does before every GPU absorption
// (build_indexer / compute_weight_sums, src/fe_absorption.cpp:845-942, and
// the CSR offsets of finalize_contiguous_groups, :547-590).

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common_kernels.cuh"
#include "kernels.cuh"

namespace b200fe {

// out[c] = bits of max over alpha rows g with W_g > 0 of |r[g][c]| / W_g (the
// largest group mean of the within transform, by dimension-row); the maximum
// of non-negative doubles is taken on their bit patterns (integer atomics:
// exact and order-free)
__global__ void row_linf_kernel(int64_t GR, int CP, int cols, const double* __restrict__ r,
                                const double* __restrict__ w_rows,
                                unsigned long long* __restrict__ out) {
    const int64_t total = GR * CP;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = e / CP;
        const int c = static_cast<int>(e - g * CP);
        const double W = w_rows[g];
        if (c < cols && W > 0.0) {
            const double v = fabs(r[e]) / W;
            if (v > 0.0) atomicMax(out + c, static_cast<unsigned long long>(__double_as_longlong(v)));
        }
    }
}

__global__ void to_float_kernel(const double* __restrict__ src, int64_t n, float* __restrict__ dst) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<float>(src[i]);
}

// Pack the small dims' ids (< 64 levels each) into 8-bit fields.
struct SmallPackArgs {
    int nS;
    const int32_t* ids[kMaxSmall];
};
__global__ void pack_small_kernel(SmallPackArgs a, const int32_t* __restrict__ ord, int64_t n,
                                  uint32_t* __restrict__ sid) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t o = ord ? ord[i] : i;
        uint32_t p = 0;
        for (int s = 0; s < a.nS; ++s) p |= (static_cast<uint32_t>(a.ids[s][o]) & 0xffu) << (8 * s);
        sid[i] = p;
    }
}

// Segment weight sums, serial in primary order per segment (deterministic).
// Unit weights: the count.  Writes 1/W (0 for empty or zero-weight segments).
__global__ void segment_inv_weight_kernel(const int32_t* __restrict__ seg_off, int32_t G,
                                          const double* __restrict__ wp,
                                          double* __restrict__ wsum,
                                          double* __restrict__ inv_w) {
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < G;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = seg_off[s], e = seg_off[s + 1];
        double W = 0.0;
        if (wp) {
            for (int32_t k = b; k < e; ++k) W += wp[k];
        } else {
            W = static_cast<double>(e - b);
        }
        if (wsum) wsum[s] = W;
        inv_w[s] = W > 0.0 ? 1.0 / W : 0.0;
    }
}

// Run-start flags of a large dim in primary order: obs k starts a run when it
// starts its primary segment or its id differs from obs k-1.
__global__ void run_flags_kernel(const int32_t* __restrict__ gp, const int32_t* __restrict__ rid,
                                 int64_t n, int32_t* __restrict__ flags) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flags[k] = (k == 0 || gp[k] != gp[k - 1] || rid[k] != rid[k - 1]) ? 1 : 0;
}

// For run starts: run_grp, run_start, run_seg.  run_id is the inclusive scan.
__global__ void run_fill_kernel(const int32_t* __restrict__ flags, const int32_t* __restrict__ run_id,
                                const int32_t* __restrict__ gp, const int32_t* __restrict__ rid,
                                int64_t n, int32_t* __restrict__ run_grp,
                                int32_t* __restrict__ run_start, int32_t* __restrict__ run_seg) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (flags[k]) {
            const int32_t m = run_id[k] - 1;
            run_grp[m] = rid[k];
            run_start[m] = static_cast<int32_t>(k);
            run_seg[m] = gp[k];
        }
    }
}

// run_base[s] = index of the first run at or after segment s's first obs
// (so run_base is non-decreasing and empty segments own no run);
// run_base[G] = nruns.
__global__ void run_base_kernel(const int32_t* __restrict__ seg_off, int32_t G,
                                const int32_t* __restrict__ run_id, int64_t n, int64_t nruns,
                                int32_t* __restrict__ run_base) {
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s <= G;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = seg_off[s];
        run_base[s] = (s < G && b < n) ? run_id[b] - 1 : static_cast<int32_t>(nruns);
    }
}

// Tiles of whole primary segments.  A tile starts at segment s when s is the
// first segment, s or s-1 is long (> kLongSeg obs), or s starts in a later
// window of kTileStride observations than s-1.  A regular tile then holds at
// most kTileStride + kLongSeg = kTileObs observations; a long segment is a
// tile of its own.
__global__ void tile_flag_kernel(const int32_t* __restrict__ seg_off, int32_t G,
                                 int32_t* __restrict__ tflag, int32_t* __restrict__ lflag) {
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s <= G;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (s == G) {
            tflag[s] = 0;
            lflag[s] = 0;
            continue;
        }
        const int32_t b = seg_off[s];
        const bool lng = seg_off[s + 1] - b > kLongSeg;
        bool start = (s == 0) || lng;
        if (!start) {
            const int32_t pb = seg_off[s - 1];
            start = (b - pb > kLongSeg) || (b / kTileStride != pb / kTileStride);
        }
        tflag[s] = start ? 1 : 0;
        lflag[s] = lng ? 1 : 0;
    }
}

__global__ void tile_fill_kernel(const int32_t* __restrict__ seg_off, int32_t G,
                                 const int32_t* __restrict__ tflag, const int32_t* __restrict__ tidx,
                                 const int32_t* __restrict__ lflag, const int32_t* __restrict__ lidx,
                                 int32_t* __restrict__ tile_seg, uint8_t* __restrict__ tile_long,
                                 int32_t* __restrict__ long_segs) {
    for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s <= G;
         s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (s == G) {
            tile_seg[tidx[G]] = G;  // sentinel
            continue;
        }
        if (tflag[s]) {
            tile_seg[tidx[s]] = static_cast<int32_t>(s);
            tile_long[tidx[s]] = lflag[s] ? 1 : 0;
        }
        if (lflag[s]) long_segs[lidx[s]] = static_cast<int32_t>(s);
    }
}

// Per run m, in run (primary) order: weight c_m (its observations' weights
// summed in order, or their count) and its diagonal term c_m^2 / W_seg.
__global__ void run_weights_kernel(int64_t nruns, const int32_t* __restrict__ run_start, int64_t n,
                                   const int32_t* __restrict__ run_seg, const double* __restrict__ wp,
                                   const double* __restrict__ inv_wp, double* __restrict__ cw_run,
                                   double* __restrict__ ce_run) {
    for (int64_t m = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; m < nruns;
         m += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = run_start[m];
        const int32_t e = (m + 1 < nruns) ? run_start[m + 1] : static_cast<int32_t>(n);
        double c = 0.0;
        if (wp) {
            for (int32_t k = b; k < e; ++k) c += wp[k];
        } else {
            c = static_cast<double>(e - b);
        }
        cw_run[m] = c;
        ce_run[m] = c * c * inv_wp[run_seg[m]];
    }
}

// The run weights at the runs' sorted positions, and run_dest (the inverse of
// the sorted order): one gather pair and one scatter per run.
__global__ void run_sorted_weights_kernel(const int32_t* __restrict__ sorted_runs, int64_t nruns,
                                          const double* __restrict__ cw_run,
                                          const double* __restrict__ ce_run, int32_t* __restrict__ run_dest,
                                          double* __restrict__ cw_sorted, double* __restrict__ ce_sorted) {
    for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < nruns;
         j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t m = sorted_runs[j];
        run_dest[m] = static_cast<int32_t>(j);
        cw_sorted[j] = cw_run[m];
        ce_sorted[j] = ce_run[m];
    }
}

// Blocks of the block-level pass, in primary order: obs k starts a block when
// it starts its primary segment or its large-dim run, when its small-dim
// level is not the previous obs's level + 1, or when its weight differs.
__global__ void block_flags_kernel(const int32_t* __restrict__ gp, const int32_t* __restrict__ rid,
                                   const uint32_t* __restrict__ sid, const double* __restrict__ wp,
                                   int64_t n, int32_t* __restrict__ flags) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        bool st = (k == 0) || gp[k] != gp[k - 1];
        if (!st && rid) st = rid[k] != rid[k - 1];
        if (!st && sid) st = (sid[k] & 0xffu) != (sid[k - 1] & 0xffu) + 1u;
        if (!st && wp) st = wp[k] != wp[k - 1];
        flags[k] = st ? 1 : 0;
    }
}

__global__ void block_start_kernel(const int32_t* __restrict__ flags, const int32_t* __restrict__ bid,
                                   int64_t n, int32_t* __restrict__ block_start) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (flags[k]) block_start[bid[k] - 1] = static_cast<int32_t>(k);
}

__global__ void block_meta_kernel(const int32_t* __restrict__ block_start, int64_t nblocks, int64_t n,
                                  const uint32_t* __restrict__ sid, const double* __restrict__ wp,
                                  int2* __restrict__ block_meta, double* __restrict__ bw64,
                                  float* __restrict__ bw32) {
    for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < nblocks;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t k = block_start[b];
        const int32_t e = (b + 1 < nblocks) ? block_start[b + 1] : static_cast<int32_t>(n);
        block_meta[b] = make_int2(sid ? static_cast<int>(sid[k] & 0xffu) : 0, e - k);
        if (wp) {
            bw64[b] = wp[k];
            bw32[b] = static_cast<float>(wp[k]);
        }
    }
}

// Packed metadata of the block-level pass.  With a large dim:
// seg_meta[s] = {first obs, first run}, run_meta[m] = {group, dest row, first
// block, end block}, run weights as float and double.  Without one, each
// segment is a pseudo-run: seg_meta[s] = {first obs, s} and run_meta[s] =
// {0, 0, first block, end block}.
__global__ void pack_meta_kernel(const int32_t* __restrict__ seg_off,
                                 const int32_t* __restrict__ run_base, int32_t G,
                                 const int32_t* __restrict__ run_grp,
                                 const int32_t* __restrict__ run_dest,
                                 const int32_t* __restrict__ run_start, int64_t nruns,
                                 const double* __restrict__ cw_run, const int32_t* __restrict__ bid,
                                 int64_t nblocks, int64_t n, int2* __restrict__ seg_meta,
                                 int4* __restrict__ run_meta, double* __restrict__ rw64,
                                 float* __restrict__ rw32) {
    const int64_t npr = run_base ? nruns : static_cast<int64_t>(G);  // (pseudo-)runs
    const int64_t total = max(static_cast<int64_t>(G) + 1, npr);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (i <= G) seg_meta[i] = make_int2(seg_off[i], run_base ? run_base[i] : static_cast<int>(i));
        if (i < npr) {
            const int64_t k0 = run_base ? run_start[i] : seg_off[i];
            const int64_t k1 = run_base ? run_start[i + 1] : seg_off[i + 1];
            const int32_t b0 = k0 < n ? bid[k0] - 1 : static_cast<int32_t>(nblocks);
            const int32_t b1 = k1 < n ? bid[k1] - 1 : static_cast<int32_t>(nblocks);
            run_meta[i] = make_int4(run_base ? run_grp[i] : 0, run_base ? run_dest[i] : 0, b0, b1);
            const double c = run_base ? cw_run[i] : 0.0;
            rw64[i] = c;
            rw32[i] = static_cast<float>(c);
        }
    }
}

// Chunk list of a large dim: group g owns runs [grp_off[g], grp_off[g+1]),
// split into ceil(len/CH) chunks (one chunk for an empty group).
__global__ void chunk_count_kernel(const int32_t* __restrict__ grp_off, int32_t G, int32_t CH,
                                   int32_t* __restrict__ nch) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t len = grp_off[g + 1] - grp_off[g];
        nch[g] = len <= CH ? 1 : (len + CH - 1) / CH;
    }
}

__global__ void chunk_fill_kernel(const int32_t* __restrict__ grp_off, int32_t G, int32_t CH,
                                  const int32_t* __restrict__ ch_off,
                                  int32_t* __restrict__ chunk_grp, int32_t* __restrict__ chunk_beg,
                                  int32_t* __restrict__ chunk_end, uint8_t* __restrict__ chunk_whole,
                                  const int32_t* __restrict__ multi_idx,
                                  int32_t* __restrict__ multi_grp, int32_t* __restrict__ multi_c0,
                                  int32_t* __restrict__ multi_c1) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = grp_off[g], e = grp_off[g + 1];
        const int32_t c0 = ch_off[g], c1 = ch_off[g + 1];
        const bool whole = (c1 - c0) == 1;
        for (int32_t c = c0; c < c1; ++c) {
            const int32_t cb = b + (c - c0) * CH;
            chunk_grp[c] = static_cast<int32_t>(g);
            chunk_beg[c] = cb;
            chunk_end[c] = min(e, cb + CH);
            chunk_whole[c] = whole ? 1 : 0;
        }
        if (c1 - c0 > 1) {  // several chunks (a group may also have none)
            const int32_t mi = multi_idx[g];
            multi_grp[mi] = static_cast<int32_t>(g);
            multi_c0[mi] = c0;
            multi_c1[mi] = c1;
        }
    }
}

__global__ void multi_flag_kernel(const int32_t* __restrict__ nch, int32_t G, int32_t* __restrict__ f) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)
        f[g] = nch[g] > 1 ? 1 : 0;
}

// Small dims: per-level weight sum and diagonal correction, deterministic:
// each warp owns a contiguous range, lanes update the warp's bins one at a
// time, CTA partials are summed in a fixed order by small_diag_reduce_kernel.
__global__ void __launch_bounds__(128)
small_diag_partial_kernel(const uint32_t* __restrict__ sid, int nS, int64_t n,
                          const int32_t* __restrict__ gp, const double* __restrict__ wp,
                          const double* __restrict__ inv_wp, double* __restrict__ partial) {
    __shared__ double bins[4][kMaxSmall * kSmallLevels * 2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 4 * kMaxSmall * kSmallLevels * 2; i += 128)
        (&bins[0][0])[i] = 0.0;
    __syncthreads();
    const int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = static_cast<int64_t>(blockIdx.x) * per_block;
    const int64_t b1 = min(n, b0 + per_block);
    const int64_t per_warp = (max(b1 - b0, int64_t(0)) + 3) / 4;
    const int64_t w0 = b0 + warp * per_warp, w1 = min(b1, w0 + per_warp);
    for (int64_t base = w0; base < w1; base += 32) {
        const int64_t k = base + lane;
        const bool valid = k < w1;
        uint32_t packed = 0;
        double w = 0.0, e = 0.0;
        if (valid) {
            packed = sid[k];
            w = wp ? wp[k] : 1.0;
            e = w * w * inv_wp[gp[k]];
        }
        for (int j = 0; j < 32; ++j) {
            __syncwarp();
            if (lane == j && valid) {
                for (int s = 0; s < nS; ++s) {
                    const uint32_t h = (packed >> (8 * s)) & 0xffu;
                    bins[warp][(s * kSmallLevels + h) * 2 + 0] += w;
                    bins[warp][(s * kSmallLevels + h) * 2 + 1] += e;
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nS * kSmallLevels * 2; i += 128)
        partial[static_cast<int64_t>(blockIdx.x) * kMaxSmall * kSmallLevels * 2 + i] =
            ((bins[0][i] + bins[1][i]) + bins[2][i]) + bins[3][i];
}

__global__ void small_diag_reduce_kernel(const double* __restrict__ partial, int nblocks, int nS,
                                         double* __restrict__ wsum_out, double* __restrict__ e_out) {
    const int i = threadIdx.x;  // over nS * 64
    if (i >= nS * kSmallLevels) return;
    double W = 0.0, E = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        W += partial[static_cast<int64_t>(b) * kMaxSmall * kSmallLevels * 2 + 2 * i];
        E += partial[static_cast<int64_t>(b) * kMaxSmall * kSmallLevels * 2 + 2 * i + 1];
    }
    wsum_out[i] = W;
    e_out[i] = E;
}

// dinv = 1/(W - E) for identified unknowns, 0 for levels without weight or in
// the null space of S (diagonal below 1e-11 of the level weight).
__global__ void dinv_kernel(const double* __restrict__ W, const double* __restrict__ E, int64_t G,
                            double* __restrict__ dinv64, float* __restrict__ dinv32) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double d = W[g] - E[g];
        const double v = (W[g] > 0.0 && d > 1e-11 * W[g]) ? 1.0 / d : 0.0;
        dinv64[g] = v;
        dinv32[g] = static_cast<float>(v);
    }
}

// Column-wise dot of two alpha-row arrays with a last-CTA fixed-order reduce.
template <typename A, typename B>
__global__ void __launch_bounds__(kRowThreads)
row_dot_kernel(int64_t GR, int CP, const A* __restrict__ a, const B* __restrict__ b,
               double* __restrict__ partial, unsigned int* ticket, double* __restrict__ out) {
    __shared__ double red[kRowThreads];
    __shared__ bool last;
    const int64_t total = GR * CP;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kRowThreads;
    double s = 0.0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * kRowThreads + threadIdx.x; i < total;
         i += stride)
        s = fma(static_cast<double>(a[i]), static_cast<double>(b[i]), s);
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < CP) {
        double t = 0.0;
        for (int k = threadIdx.x; k < kRowThreads; k += CP) t += red[k];
        partial[static_cast<int64_t>(blockIdx.x) * CP + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < CP) {
        double t = 0.0;
        for (int bb = 0; bb < static_cast<int>(gridDim.x); ++bb)
            t += __ldcg(partial + static_cast<int64_t>(bb) * CP + threadIdx.x);
        out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// Elementwise helpers over alpha rows.
// dst = src64 * inv_scale[c]   (per-column scaling of an inner right-hand side)
template <typename T>
__global__ void scale_rows_kernel(int64_t GR, int CP, const double* __restrict__ src,
                                  const double* __restrict__ inv_scale, T* __restrict__ dst) {
    const int64_t total = GR * CP;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<T>(src[i] * inv_scale[i % CP]);
}
// a64 += scale[c] * x
template <typename T>
__global__ void axpy_rows_kernel(int64_t GR, int CP, const T* __restrict__ x,
                                 const double* __restrict__ scale, double* __restrict__ a) {
    const int64_t total = GR * CP;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        a[i] += scale[i % CP] * static_cast<double>(x[i]);
}
// r = b - q
__global__ void sub_kernel(int64_t total, const double* __restrict__ b, const double* __restrict__ q,
                           double* __restrict__ r) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        r[i] = b[i] - q[i];
}

// Gauss-Seidel max-delta (FE recovery check): means of dim d over the
// residual, then subtract.  Deterministic per-group serial sums over a CSR.
__global__ void group_mean_csr_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ ord,
                                      int32_t G, const double* __restrict__ v,
                                      const double* __restrict__ w, double* __restrict__ mean,
                                      double* __restrict__ absmax_partial) {
    double mx = 0.0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double s = 0.0, W = 0.0;
        for (int32_t j = off[g]; j < off[g + 1]; ++j) {
            const int32_t i = ord[j];
            const double wi = w ? w[i] : 1.0;
            s += wi * v[i];
            W += wi;
        }
        const double m = W > 0.0 ? s / W : 0.0;
        mean[g] = m;
        mx = fmax(mx, fabs(m));
    }
    __shared__ double red[256];
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x == 0) absmax_partial[blockIdx.x] = red[0];
}

__global__ void subtract_mean_kernel(double* __restrict__ v, const int32_t* __restrict__ gid,
                                     const double* __restrict__ mean, int64_t n) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[i] -= mean[gid[i]];
}

// ---------------------------------------------------------------------------
// Dense small-dim coupling of the block-level structure (one large dim f, one
// small dim h with SG <= kCoupleMaxSG levels).  With y_m[h] the weight of run
// m's observations at level h and Y_s[h] that of primary segment s (both read
// off the blocks: consecutive levels h0 .. h0+len-1 of one weight w_b),
//     C_fy[f][h]  = sum_{runs m of f} ( y_m[h] - c_m Y_s(m)[h] / W_s(m) ),
//     C_yy[h][h'] = W_h [h = h'] - sum_s Y_s[h] Y_s[h'] / W_s,
// i.e. the blocks D_f' W (I - P_p) D_y and D_y' W (I - P_p) D_y of S.  Lane l
// of a warp owns the levels h = l and h = l + 32.  Sums have a fixed order.
// ---------------------------------------------------------------------------
constexpr int kCoupleMaxSG = 64;

__device__ __forceinline__ int lo_clear(int hmin, int SG) { return hmin < SG ? hmin : SG; }

// Adds w to row[h] for the levels of block bm (a lane's private row).
__device__ __forceinline__ void couple_row_add(double* row, const int2 bm, double w) {
    for (int h = bm.x; h < bm.x + bm.y; ++h) row[h] += w;
}

// Pitch of the per-lane shared-memory rows: odd in doubles, so that the 16
// lanes of a 64-bit shared access that touch level h of 16 different rows fall
// in 16 different bank pairs (an even pitch such as 36 puts lanes l and l + 4
// in the same banks: 8-way conflicts on every row access).
__host__ __device__ __forceinline__ int couple_pitch(int SG) { return SG | 1; }

// C_fy over ranges of kFyRangeRuns consecutive runs in firm order (sorted_runs),
// one warp per range, across firm boundaries (most firms own a few runs: one
// warp per firm would leave most lanes idle).  Lane i takes run j0 + i of each
// batch of 32: its metadata and blocks are read by the 32 lanes in parallel,
// and lane i writes y_m - c_m Y_s / W_s into its own shared-memory row (levels
// hmin .. hmax of its segment, cleared again after the batch); lane l then sums
// level l (and l + 32) over the batch's rows in order, and writes a firm's sum
// when the firm ends.  A firm inside the range writes its row of C_fy (stride
// SGP = SG rounded up to 4, padding zero); the piece of a firm that begins
// before the range goes to slot 0 of the range's partials, the piece of a firm
// that begins in the range and ends after it to slot 1, and
// coupling_fy_join_kernel adds the pieces of those firms in range order.  Firm
// ids with no runs (between two consecutive firms of the order, or before the
// first or after the last) get zero rows from the warp that passes them.
constexpr int kCoupleWarps = 8;
constexpr int kFyRangeRuns = 512;
constexpr int kFyPrefetch = 4;

__device__ __forceinline__ void couple_put_row(double* dst, double a0, double a1, int lane, int SG, int SGP) {
    if (lane < SGP) dst[lane] = lane < SG ? a0 : 0.0;
    if (lane + 32 < SGP) dst[lane + 32] = lane + 32 < SG ? a1 : 0.0;
}

__device__ __forceinline__ void couple_zero_rows(double* out_fy, int64_t g0, int64_t g1, int lane, int SGP) {
    for (int64_t g = g0; g < g1; ++g)
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (lane + 32 * k < SGP) out_fy[g * SGP + lane + 32 * k] = 0.0;
}

// Per run m, written at its sorted position j = run_dest[m]: the block range
// of its segment [x, y), its own block range [z, w) and c_m / W_s(m) - one
// coalesced record per lane of coupling_fy_range_kernel in place of a chain of
// dependent gathers (run -> segment -> the segment's first and last runs).
__global__ void fy_run_record_kernel(int64_t nruns, const int32_t* __restrict__ run_dest,
                                     const int32_t* __restrict__ run_seg, const int4* __restrict__ run_meta,
                                     const int2* __restrict__ seg_meta, const double* __restrict__ cw_run,
                                     const double* __restrict__ inv_wp, int4* __restrict__ rec,
                                     double* __restrict__ rec_cf) {
    for (int64_t m = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; m < nruns;
         m += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t sg = run_seg[m];
        const int4 rm = run_meta[m];
        const int32_t r0 = seg_meta[sg].y, r1 = seg_meta[sg + 1].y;
        const int32_t j = run_dest[m];
        rec[j] = make_int4(run_meta[r0].z, run_meta[r1 - 1].w, rm.z, rm.w);
        rec_cf[j] = cw_run[m] * inv_wp[sg];
    }
}

__global__ void __launch_bounds__(kCoupleWarps * 32)
coupling_fy_range_kernel(int64_t nruns, int64_t nranges, int32_t G, const int4* __restrict__ rec,
                         const double* __restrict__ rec_cf, const int32_t* __restrict__ sorted_grp,
                         const int32_t* __restrict__ grp_off, const int2* __restrict__ block_meta,
                         const double* __restrict__ block_w, int SG, int SGP, double* __restrict__ out_fy,
                         double* __restrict__ part) {
    extern __shared__ double cf_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int SGQ = couple_pitch(SG);
    double* rows = cf_smem + static_cast<int64_t>(warp) * 32 * SGQ;
    double* myrow = rows + lane * SGQ;
    for (int h = 0; h < SGQ; ++h) myrow[h] = 0.0;
    __syncwarp();
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kCoupleWarps;
    for (int64_t rg = static_cast<int64_t>(blockIdx.x) * kCoupleWarps + warp; rg < nranges; rg += nwarps) {
        const int64_t rb = rg * kFyRangeRuns, re = min(rb + kFyRangeRuns, nruns);
        int32_t cur = sorted_grp[rb];
        const int32_t prev = rb > 0 ? sorted_grp[rb - 1] : -1;
        if (cur != prev) couple_zero_rows(out_fy, prev + 1, cur, lane, SGP);
        // where the pieces of the current firm go
        auto flush = [&](int32_t f, double a0, double a1) {
            const int32_t fb = grp_off[f], fe = grp_off[f + 1];
            double* dst = (fb >= rb && fe <= re) ? out_fy + static_cast<int64_t>(f) * SGP
                          : (fb < rb)            ? part + (rg * 2 + 0) * SGP
                                                 : part + (rg * 2 + 1) * SGP;
            couple_put_row(dst, a0, a1, lane, SG, SGP);
        };
        double acc0 = 0.0, acc1 = 0.0;
        for (int64_t j0 = rb; j0 < re; j0 += 32) {
            int32_t g = -1;
            int hmin = SG, hmax = 0;
            if (j0 + lane < re) {
                const int4 rc = rec[j0 + lane];
                const double cf = rec_cf[j0 + lane];
                g = sorted_grp[j0 + lane];
                // the segment's first kFyPrefetch blocks are loaded together
                int2 bq[kFyPrefetch];
                double wq[kFyPrefetch];
#pragma unroll
                for (int q = 0; q < kFyPrefetch; ++q) {
                    const bool in = rc.x + q < rc.y;
                    bq[q] = in ? block_meta[rc.x + q] : make_int2(0, 0);
                    wq[q] = (in && block_w) ? block_w[rc.x + q] : 1.0;
                }
                auto block_at = [&](int bb, int2& bm, double& w) {
                    const int q = bb - rc.x;
                    if (q < kFyPrefetch) {
                        bm = bq[0];
                        w = wq[0];
#pragma unroll
                        for (int t = 1; t < kFyPrefetch; ++t)
                            if (q == t) {
                                bm = bq[t];
                                w = wq[t];
                            }
                    } else {
                        bm = block_meta[bb];
                        w = block_w ? block_w[bb] : 1.0;
                    }
                };
                for (int bb = rc.z; bb < rc.w; ++bb) {
                    int2 bm;
                    double w;
                    block_at(bb, bm, w);
                    couple_row_add(myrow, bm, w);
                }
                for (int bb = rc.x; bb < rc.y; ++bb) {
                    int2 bm;
                    double w;
                    block_at(bb, bm, w);
                    couple_row_add(myrow, bm, -cf * w);
                    hmin = min(hmin, bm.x);
                    hmax = max(hmax, bm.x + bm.y);
                }
            }
            __syncwarp();
            const int nj = static_cast<int>(min(static_cast<int64_t>(32), re - j0));
            for (int i = 0; i < nj; ++i) {
                const int32_t gi = __shfl_sync(0xffffffffu, g, i);
                if (gi != cur) {  // warp-uniform: the firm of run j0 + i starts here
                    flush(cur, acc0, acc1);
                    couple_zero_rows(out_fy, static_cast<int64_t>(cur) + 1, gi, lane, SGP);
                    acc0 = acc1 = 0.0;
                    cur = gi;
                }
                if (lane < SG) acc0 += rows[i * SGQ + lane];
                if (lane + 32 < SG) acc1 += rows[i * SGQ + lane + 32];
            }
            __syncwarp();
            for (int h = lo_clear(hmin, SG); h < max(hmax, 0); ++h) myrow[h] = 0.0;
            __syncwarp();
        }
        flush(cur, acc0, acc1);
        if (re == nruns) couple_zero_rows(out_fy, static_cast<int64_t>(cur) + 1, G, lane, SGP);
    }
}

// Rows of the firms split across ranges: the range holding a firm's first run
// sees it as its last firm, continuing past the range; its row is slot 1 of that
// range plus slot 0 of each following range up to the firm's last run, added in
// range order (warp w sums ranges r + 1 + w, r + 9 + w, ...; the eight warp sums
// are then added to slot 1 in warp order).  One CTA per range.
__global__ void __launch_bounds__(256)
coupling_fy_join_kernel(int64_t nruns, int64_t nranges, const int32_t* __restrict__ sorted_grp,
                        const int32_t* __restrict__ grp_off, const double* __restrict__ part, int SGP,
                        double* __restrict__ out_fy) {
    __shared__ double ws[8][kCoupleMaxSG];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t r = blockIdx.x; r < nranges; r += gridDim.x) {
        const int64_t rb = r * kFyRangeRuns, re = min(rb + kFyRangeRuns, nruns);
        const int32_t f = sorted_grp[re - 1];
        const int64_t fb = grp_off[f], fe = grp_off[f + 1];
        if (fb < rb || fe <= re) continue;  // uniform over the CTA
        const int64_t r1 = (fe - 1) / kFyRangeRuns;
        double acc[2] = {0.0, 0.0};
        for (int64_t q = r + 1 + warp; q <= r1; q += 8) {
#pragma unroll
            for (int k = 0; k < 2; ++k)
                if (lane + 32 * k < SGP) acc[k] += __ldcg(part + (q * 2 + 0) * SGP + lane + 32 * k);
        }
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (lane + 32 * k < SGP) ws[warp][lane + 32 * k] = acc[k];
        __syncthreads();
        if (threadIdx.x < SGP) {
            double v = __ldcg(part + (r * 2 + 1) * SGP + threadIdx.x);
            for (int w = 0; w < 8; ++w) v += ws[w][threadIdx.x];
            out_fy[static_cast<int64_t>(f) * SGP + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// sum_s Y_s Y_s' / W_s and the level weights W_h = sum_s Y_s[h].  Lane i of a
// warp builds Y_s of segment s0 + i in its own shared row (the 32 lanes read
// their blocks in parallel); then, segment by segment in lane order, lane l
// adds Y_s[h] Y_s[h'] / W_s to rows h = l and l + 32 of the warp's SG x SG
// accumulator, for h' in the segment's level range, and Y_s[h] to W_h.  Rows of
// Y and of the accumulator have the odd pitch couple_pitch(SG).  Per-CTA
// partials [SG*SG + SG], summed in CTA order by coupling_yy_reduce_kernel.
constexpr int kCoupleYyWarps = 2;

__host__ __device__ __forceinline__ int couple_yy_warp_words(int SG) {
    return SG * couple_pitch(SG) + SG + 32 * couple_pitch(SG);  // acc, W, 32 rows Y
}

__global__ void __launch_bounds__(kCoupleYyWarps * 32)
coupling_yy_kernel(int32_t Gp, const int2* __restrict__ seg_meta, const int4* __restrict__ run_meta,
                   const int2* __restrict__ block_meta, const double* __restrict__ block_w,
                   const double* __restrict__ inv_wp, int SG, double* __restrict__ partial) {
    extern __shared__ double cy_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int SS = SG * SG;
    const int SGQ = couple_pitch(SG);
    const int WS = couple_yy_warp_words(SG);
    double* acc = cy_smem + static_cast<int64_t>(warp) * WS;
    double* Wh = acc + SG * SGQ;
    double* Y = Wh + SG;
    double* myY = Y + lane * SGQ;
    for (int i = threadIdx.x; i < kCoupleYyWarps * WS; i += blockDim.x) cy_smem[i] = 0.0;
    __syncthreads();
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kCoupleYyWarps;
    const int64_t wid = static_cast<int64_t>(blockIdx.x) * kCoupleYyWarps + warp;
    for (int64_t s0 = wid * 32; s0 < Gp; s0 += nwarps * 32) {
        int hmin = SG, hmax = 0;
        double iw = 0.0;
        if (s0 + lane < Gp) {
            const int64_t sg = s0 + lane;
            const int32_t r0 = seg_meta[sg].y, r1 = seg_meta[sg + 1].y;
            if (r1 > r0) {
                const int sb0 = run_meta[r0].z, sb1 = run_meta[r1 - 1].w;
                for (int bb = sb0; bb < sb1; ++bb) {
                    const int2 bm = block_meta[bb];
                    couple_row_add(myY, bm, block_w ? block_w[bb] : 1.0);
                    hmin = min(hmin, bm.x);
                    hmax = max(hmax, bm.x + bm.y);
                }
            }
            iw = inv_wp[sg];
        }
        __syncwarp();
        const int ns = static_cast<int>(min(static_cast<int64_t>(32), Gp - s0));
        for (int i = 0; i < ns; ++i) {
            const int lo = __shfl_sync(0xffffffffu, hmin, i), hi = __shfl_sync(0xffffffffu, hmax, i);
            const double w_inv = __shfl_sync(0xffffffffu, iw, i);
            const double* Yi = Y + i * SGQ;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int h = lane + 32 * k;
                if (h >= lo && h < hi) {
                    const double yh = Yi[h];
                    Wh[h] += yh;
                    const double a = yh * w_inv;
                    if (a != 0.0)
                        for (int h2 = lo; h2 < hi; ++h2) acc[h * SGQ + h2] = fma(a, Yi[h2], acc[h * SGQ + h2]);
                }
            }
        }
        __syncwarp();
        for (int h = lo_clear(hmin, SG); h < max(hmax, 0); ++h) myY[h] = 0.0;
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SS + SG; i += blockDim.x) {
        const int src = i < SS ? (i / SG) * SGQ + (i - (i / SG) * SG) : SG * SGQ + (i - SS);
        double v = 0.0;
        for (int w = 0; w < kCoupleYyWarps; ++w) v += cy_smem[static_cast<int64_t>(w) * WS + src];
        partial[static_cast<int64_t>(blockIdx.x) * (SS + SG) + i] = v;
    }
}

// The same sums with the accumulator in registers, for SG <= 8 RT and SG <= 4 CT.
// Lane l owns the RT x CT tile of entries (h, h') with h in 8-lane row group
// l / 4 (rows RT (l / 4) ..) and h' in column group l % 4 (columns CT (l % 4) ..);
// the lanes with l % 4 == 0 also own W_h of their rows.  For each segment of
// the warp's batch of 32 (in lane order) every lane adds Y_s[h] / W_s * Y_s[h']
// to its whole tile: a level outside the segment's range has Y_s = 0 and adds
// an exact zero (all terms are >= 0), so each entry still sums its nonzero terms
// in segment order, as coupling_yy_kernel does, with independent FMAs in place
// of a chain of shared-memory updates.  Rows of Y have the odd pitch
// couple_tile_pitch(RT, CT), levels >= SG stay zero.  The warps' tiles are added
// into the CTA's partial in warp order.
constexpr int kCoupleTileWarps = 4;

__host__ __device__ constexpr int couple_tile_pitch(int RT, int CT) {
    return (8 * RT > 4 * CT ? 8 * RT : 4 * CT) | 1;
}

template <int RT, int CT>
__global__ void __launch_bounds__(kCoupleTileWarps * 32)
coupling_yy_tile_kernel(int32_t Gp, const int2* __restrict__ seg_meta, const int4* __restrict__ run_meta,
                        const int2* __restrict__ block_meta, const double* __restrict__ block_w,
                        const double* __restrict__ inv_wp, int SG, double* __restrict__ partial) {
    constexpr int P = couple_tile_pitch(RT, CT);
    extern __shared__ double ct_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int SS = SG * SG;
    double* red = ct_smem;                                   // SS + SG
    double* Y = ct_smem + SS + SG + static_cast<int64_t>(warp) * 32 * P;
    double* myY = Y + lane * P;
    for (int i = threadIdx.x; i < SS + SG + kCoupleTileWarps * 32 * P; i += blockDim.x) ct_smem[i] = 0.0;
    __syncthreads();
    const int R0 = RT * (lane >> 2), C0 = CT * (lane & 3);
    double acc[RT][CT], wacc[RT];
#pragma unroll
    for (int r = 0; r < RT; ++r) {
        wacc[r] = 0.0;
#pragma unroll
        for (int c = 0; c < CT; ++c) acc[r][c] = 0.0;
    }
    const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kCoupleTileWarps;
    const int64_t wid = static_cast<int64_t>(blockIdx.x) * kCoupleTileWarps + warp;
    for (int64_t s0 = wid * 32; s0 < Gp; s0 += nwarps * 32) {
        int hmin = SG, hmax = 0;
        double iw = 0.0;
        if (s0 + lane < Gp) {
            const int64_t sg = s0 + lane;
            const int32_t r0 = seg_meta[sg].y, r1 = seg_meta[sg + 1].y;
            if (r1 > r0) {
                const int sb0 = run_meta[r0].z, sb1 = run_meta[r1 - 1].w;
                for (int bb = sb0; bb < sb1; ++bb) {
                    const int2 bm = block_meta[bb];
                    couple_row_add(myY, bm, block_w ? block_w[bb] : 1.0);
                    hmin = min(hmin, bm.x);
                    hmax = max(hmax, bm.x + bm.y);
                }
            }
            iw = inv_wp[sg];
        }
        __syncwarp();
        const int ns = static_cast<int>(min(static_cast<int64_t>(32), Gp - s0));
        for (int i = 0; i < ns; ++i) {
            const double w_inv = __shfl_sync(0xffffffffu, iw, i);
            const double* Yi = Y + i * P;
            double a[RT], b[CT];
#pragma unroll
            for (int r = 0; r < RT; ++r) {
                const double yh = Yi[R0 + r];
                wacc[r] += yh;
                a[r] = yh * w_inv;
            }
#pragma unroll
            for (int c = 0; c < CT; ++c) b[c] = Yi[C0 + c];
#pragma unroll
            for (int r = 0; r < RT; ++r)
#pragma unroll
                for (int c = 0; c < CT; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncwarp();
        for (int h = lo_clear(hmin, SG); h < max(hmax, 0); ++h) myY[h] = 0.0;
        __syncwarp();
    }
    for (int w = 0; w < kCoupleTileWarps; ++w) {
        if (warp == w) {
#pragma unroll
            for (int r = 0; r < RT; ++r) {
                const int h = R0 + r;
                if (h < SG) {
#pragma unroll
                    for (int c = 0; c < CT; ++c)
                        if (C0 + c < SG) red[h * SG + C0 + c] += acc[r][c];
                    if ((lane & 3) == 0) red[SS + h] += wacc[r];
                }
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < SS + SG; i += blockDim.x)
        partial[static_cast<int64_t>(blockIdx.x) * (SS + SG) + i] = red[i];
}

// C_yy = diag(W) - sum_s Y_s Y_s' / W_s, CTA partials summed in CTA order; the
// level weights W_h and E_h = sum_s Y_s[h]^2 / W_s also go to the diagonal
// arrays of the Jacobi preconditioner (diag C_yy = W_h - E_h, exact).
__global__ void coupling_yy_reduce_kernel(const double* __restrict__ partial, int nparts, int SG,
                                          double* __restrict__ out_yy, double* __restrict__ W_out,
                                          double* __restrict__ E_out) {
    const int SS = SG * SG;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < SS; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nparts; ++b) acc += partial[static_cast<int64_t>(b) * (SS + SG) + i];
        const int h = i / SG, h2 = i - h * SG;
        if (h == h2) {
            double W = 0.0;
            for (int b = 0; b < nparts; ++b) W += partial[static_cast<int64_t>(b) * (SS + SG) + SS + h];
            W_out[h] = W;
            E_out[h] = acc;
            out_yy[i] = W - acc;
        } else {
            out_yy[i] = -acc;
        }
    }
}

// Diagonal terms of a large dim per group, W_g = sum c_m and
// E_g = sum c_m^2 / W_s(m) over its runs (in group order), over the chunk list:
// a chunk that is its group's only one writes the group's sums; the others
// write partials that multi_wsum_kernel adds in chunk order.
__global__ void chunk_wsum_kernel(int64_t nchunks, const int32_t* __restrict__ chunk_grp,
                                  const int32_t* __restrict__ chunk_beg,
                                  const int32_t* __restrict__ chunk_end,
                                  const uint8_t* __restrict__ chunk_whole,
                                  const double* __restrict__ cw_sorted,
                                  const double* __restrict__ ce_sorted, double* __restrict__ W,
                                  double* __restrict__ E, double* __restrict__ part2) {
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < nchunks;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double sw = 0.0, se = 0.0;
        for (int32_t j = chunk_beg[c]; j < chunk_end[c]; ++j) {
            sw += cw_sorted[j];
            se += ce_sorted[j];
        }
        if (chunk_whole[c]) {
            W[chunk_grp[c]] = sw;
            E[chunk_grp[c]] = se;
        } else {
            part2[2 * c] = sw;
            part2[2 * c + 1] = se;
        }
    }
}

// One CTA per multi-chunk group: thread t adds chunks c0 + t, c0 + t + 256,
// ..., then a fixed-order tree in shared memory.
__global__ void __launch_bounds__(256)
multi_wsum_kernel(int64_t nmulti, const int32_t* __restrict__ multi_grp,
                  const int32_t* __restrict__ multi_c0, const int32_t* __restrict__ multi_c1,
                  const double* __restrict__ part2, double* __restrict__ W, double* __restrict__ E) {
    __shared__ double rw[256], re[256];
    for (int64_t r = blockIdx.x; r < nmulti; r += gridDim.x) {
        double sw = 0.0, se = 0.0;
        for (int32_t c = multi_c0[r] + threadIdx.x; c < multi_c1[r]; c += 256) {
            sw += part2[2 * static_cast<int64_t>(c)];
            se += part2[2 * static_cast<int64_t>(c) + 1];
        }
        rw[threadIdx.x] = sw;
        re[threadIdx.x] = se;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h) {
                rw[threadIdx.x] += rw[threadIdx.x + h];
                re[threadIdx.x] += re[threadIdx.x + h];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            W[multi_grp[r]] = rw[0];
            E[multi_grp[r]] = re[0];
        }
        __syncthreads();
    }
}

}  // namespace b200fe
