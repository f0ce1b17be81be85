// Host-side preprocessing of the reference, on the device:
//   * dense group ids from raw ids, the rule of build_indexer
//     (src/fe_absorption.cpp:845-940): when the raw range is at most 50M and
//     at most 2n, ids are raw - min, compacted in raw order if fewer than 90%
//     of the range is present; otherwise the rank of the raw value among the
//     distinct values (sorted keys);
//   * the singleton cascade of compute_keep_mask_drop_singletons
//     (src/hdfe_regressor_v11.cpp:4056-4290): rounds that drop every kept row
//     sitting alone in a group of any dimension, until a round drops nothing.
// Counts use integer atomics (order-free, so exact and reproducible).

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200fe {

constexpr long long kDenseRangeCap = 50000000LL;

__global__ void minmax_kernel(const int32_t* __restrict__ raw, int64_t n, int* __restrict__ mm) {
    int lo = INT_MAX, hi = INT_MIN;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int v = raw[i];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

// seen[raw - lo] = 1 (idempotent stores); count of distinct values
__global__ void mark_seen_kernel(const int32_t* __restrict__ raw, int64_t n, int lo,
                                 int32_t* __restrict__ seen) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        seen[raw[i] - lo] = 1;
}

__global__ void count_ones_kernel(const int32_t* __restrict__ f, int64_t m, int* __restrict__ out) {
    int c = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        c += f[i] != 0;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// out[i] = remap[raw[i] - lo] (remap null: raw[i] - lo)
__global__ void map_ids_kernel(const int32_t* __restrict__ raw, int64_t n, int lo,
                               const int32_t* __restrict__ remap, int32_t* __restrict__ out) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t m = raw[i] - lo;
        out[i] = remap ? remap[m] : m;
    }
}

// signed -> order-preserving unsigned keys
__global__ void flip_sign_kernel(const int32_t* __restrict__ raw, int64_t n, uint32_t* __restrict__ key) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        key[i] = static_cast<uint32_t>(raw[i]) ^ 0x80000000u;
}

// flag[k] = 1 where the sorted key starts a new value
__global__ void new_key_flags_kernel(const uint32_t* __restrict__ skey, int64_t n, int32_t* __restrict__ flag) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flag[k] = (k == 0 || skey[k] != skey[k - 1]) ? 1 : 0;
}

// out[perm[k]] = rank[k] - 1 (rank = inclusive scan of the flags)
__global__ void scatter_rank_kernel(const int32_t* __restrict__ rank, const int32_t* __restrict__ perm,
                                    int64_t n, int32_t* __restrict__ out) {
    for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[perm[k]] = rank[k] - 1;
}

struct SingletonArgs {
    int nd;
    const int32_t* ids[8];
    int32_t* counts[8];
};

// counts of the kept rows per group of every dim; lanes of a warp that hit the
// same group add once (warp-aggregated), which matters for very large groups
__global__ void singleton_count_kernel(const SingletonArgs a, int64_t n, const uint8_t* __restrict__ keep) {
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < n;
         base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool live = i < n && keep[i];
        for (int d = 0; d < a.nd; ++d) {
            const int32_t g = live ? a.ids[d][i] : -1 - static_cast<int32_t>(threadIdx.x & 31);
            const unsigned int peers = __match_any_sync(0xffffffffu, g);
            const int leader = __ffs(peers) - 1;
            if (live && (threadIdx.x & 31) == leader) atomicAdd(a.counts[d] + g, __popc(peers));
        }
    }
}

// drop the kept rows that are alone in a group of some dim
__global__ void singleton_drop_kernel(const SingletonArgs a, int64_t n, uint8_t* __restrict__ keep,
                                      unsigned long long* __restrict__ dropped) {
    unsigned int local = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (!keep[i]) continue;
        bool single = false;
        for (int d = 0; d < a.nd && !single; ++d) single = a.counts[d][a.ids[d][i]] == 1;
        if (single) {
            keep[i] = 0;
            ++local;
        }
    }
    local = __reduce_add_sync(0xffffffffu, local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(dropped, static_cast<unsigned long long>(local));
}

}  // namespace b200fe
