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

// ---------------------------------------------------------------------------
// Connected components of the bipartite graph of two FE dimensions (nodes:
// the groups of both dims; edges: observations), the mobility groups of the
// reference's compute_first_pair_component_stats
// (src/hdfe_regressor_v11.cpp:7192-7270).  Min-label hooking: every edge
// points the larger of its two roots at the smaller (atomicMin), then pointer
// jumping flattens the trees; repeated until no edge joins two roots.  The
// final label of a node is the smallest node id of its component, whatever
// the order of the atomics.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t cc_root(const int32_t* parent, int32_t x) {
    int32_t p = parent[x];
    while (p != x) {
        x = p;
        p = parent[x];
    }
    return x;
}

__global__ void cc_hook_kernel(const int32_t* __restrict__ g1, const int32_t* __restrict__ g2,
                               int64_t n, int32_t G1, int32_t* parent, int* changed) {
    int local = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t ru = cc_root(parent, g1[i]);
        const int32_t rv = cc_root(parent, G1 + g2[i]);
        if (ru != rv) {
            atomicMin(parent + max(ru, rv), min(ru, rv));
            local = 1;
        }
    }
    if (__syncthreads_or(local) && threadIdx.x == 0) atomicOr(changed, 1);
}

__global__ void cc_compress_kernel(int32_t* parent, int32_t N) {
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < N;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x)
        parent[v] = cc_root(parent, static_cast<int32_t>(v));
}

// component label of every observation (trees already flat)
__global__ void cc_label_kernel(const int32_t* __restrict__ g1, int64_t n,
                                const int32_t* __restrict__ parent, int32_t* __restrict__ label) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        label[i] = parent[g1[i]];
}

// per-node observation counts from the offsets; the largest, and the number of
// non-empty components (integer atomics: order-free)
__global__ void cc_count_kernel(const int32_t* __restrict__ off, int32_t N, int* __restrict__ ncomp,
                                int* __restrict__ largest) {
    int c = 0, m = 0;
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < N;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int k = off[v + 1] - off[v];
        c += k > 0;
        m = max(m, k);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    m = static_cast<int>(__reduce_max_sync(0xffffffffu, static_cast<unsigned>(m)));
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(ncomp, c);
        atomicMax(largest, m);
    }
}

// flags[0] |= 1 when a weight is not finite and positive
__global__ void positive_weights_kernel(const double* __restrict__ w, int64_t n, int* flags) {
    int bad = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        bad |= !(w[i] > 0.0) || !(w[i] < 1e300);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags, 1);
}

}  // namespace b200fe
