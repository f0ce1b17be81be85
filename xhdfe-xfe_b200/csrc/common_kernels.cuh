// Small kernels shared by the translation units of the library (ids and
// weights validation, iota, segment offsets, gathers into primary order,
// non-empty group counts).  They have internal linkage, so every unit that
// includes this header gets its own copy.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200fe {

// flags[0] |= 1 if some id is out of [0, G); flags[1] |= 1 if ids are not
// non-decreasing (only checked when check_sorted).
static __global__ void validate_ids_kernel(const int32_t* __restrict__ g, int64_t n, int32_t G,
                                    int check_sorted, int* flags) {
    int bad = 0, unsorted = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t v = g[i];
        bad |= (v < 0 || v >= G);
        if (check_sorted && i > 0) unsorted |= (v < g[i - 1]);
    }
    bad = __syncthreads_or(bad);
    unsorted = __syncthreads_or(unsorted);
    if (threadIdx.x == 0) {
        if (bad) atomicOr(flags, 1);
        if (unsorted) atomicOr(flags + 1, 1);
    }
}

// flags[2] |= 1 if a weight is negative or not finite.
static __global__ void validate_weights_kernel(const double* __restrict__ w, int64_t n, int* flags) {
    int bad = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = w[i];
        bad |= !(v >= 0.0) || !(v <= 1.7976931348623157e308);
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0 && bad) atomicOr(flags + 2, 1);
}

static __global__ void iota_kernel(int32_t* __restrict__ out, int64_t n) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<int32_t>(i);
}

// Integer histogram (exact, order independent).
static __global__ void histogram_kernel(const int32_t* __restrict__ ids, int64_t n,
                                 int32_t* __restrict__ counts) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        atomicAdd(counts + ids[i], 1);
}

// off[g] = first position i with sorted[i] >= g, g = 0..G (ids sorted, in
// [0, G)): each position fills the offsets of the ids it starts, so empty
// groups get the next group's offset.  No atomics; one pass over the ids.
static __global__ void segment_offsets_kernel(const int32_t* __restrict__ sorted, int64_t n, int32_t G,
                                       int32_t* __restrict__ off) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t cur = i < n ? sorted[i] : G;
        const int32_t prev = i > 0 ? sorted[i - 1] : -1;
        for (int32_t g = prev + 1; g <= cur; ++g) off[g] = static_cast<int32_t>(i);
    }
}

// Gather a dense id array (or weights) into primary order.
template <typename V>
static __global__ void gather_kernel(const V* __restrict__ src, const int32_t* __restrict__ ord,
                              int64_t n, V* __restrict__ dst) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = ord ? src[ord[i]] : src[i];
}

// number of non-empty clusters
static __global__ void count_nonempty_kernel(const int32_t* __restrict__ off, int32_t G, int* __restrict__ out) {
    int c = 0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)
        c += off[g + 1] > off[g] ? 1 : 0;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);  // integer count: order-free
}

}  // namespace b200fe
