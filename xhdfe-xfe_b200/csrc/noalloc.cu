// One-way within transform that allocates no device memory.
//
// Some callers cannot allocate device memory while they call into this
// library: a host application that hands us the GPU inside its own
// fixed-size memory pool, a plugin whose process must not grow its CUDA
// footprint mid-session, or code running while another component forbids
// cudaMalloc (which synchronises the whole device).  For them this file offers
// b200fe_demean_sorted_noalloc: the caller passes every input and output
// buffer, and the only scratch the computation needs (the segment offsets of
// the group ids and a status word) lives in a fixed file-scope __device__
// array.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxGroups groups (the array holds their offsets); larger
//     calls are rejected with B200FE_INVALID_ARG before any GPU work;
//   * every GPU on which this part of the library is loaded keeps the array
//     (about 4 MiB) until the process exits.  CUDA loads a library's device
//     code lazily, per device: creating an absorber context on a device
//     (b200fe_context_create) loads it there and resolves the array's address,
//     so a caller that creates a context first has nothing placed on the GPU
//     by its no-alloc calls; without a context, the first no-alloc call on a
//     device loads it (the array plus this file's kernels), unless the process
//     runs with CUDA_MODULE_LOADING=EAGER, which loads it with the CUDA context;
//   * all calls on a device share the array and it keeps the last call's
//     contents, so calls whose GPU work overlaps (different streams or host
//     threads without ordering between them) race on it; order such calls;
//   * the array's device address is resolved once per device (with that
//     device current), at context creation or else by the first call; make
//     that first call before any stream capture;
//   * every call waits for its stream once (it reads back the status word of
//     the id check before the demeaning kernels are launched).
//
// The arithmetic is that of the absorber's segment means for a single FE
// dimension: per group and column a weighted mean by a fixed-order reduction,
// then v - mean.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "b200fe.h"

namespace {

constexpr int32_t kNoAllocMaxGroups = 1 << 20;
constexpr int kNoAllocStatus = kNoAllocMaxGroups + 1;  // index of the status word
constexpr int kMaxDevices = 64;

// offsets[0..G] of the group segments, then the status word
static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocMaxGroups + 1 + 63];

std::mutex g_setup_mutex;
int32_t* g_scratch_ptr[kMaxDevices] = {nullptr};

// status |= 1: an id outside [0, G); status |= 2: ids not non-decreasing
__global__ void noalloc_check_kernel(const int32_t* __restrict__ g, int64_t n, int32_t G,
                                     int32_t* __restrict__ status) {
    int bad = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t v = g[i];
        if (v < 0 || v >= G) bad |= 1;
        if (i > 0 && v < g[i - 1]) bad |= 2;
    }
    const int b1 = __syncthreads_or(bad & 1) ? 1 : 0;
    const int b2 = __syncthreads_or(bad & 2) ? 2 : 0;
    if (threadIdx.x == 0 && (b1 | b2)) atomicOr(status, b1 | b2);
}

// off[h] = first i with g[i] >= h, for h = 0..G (binary search, ids sorted)
__global__ void noalloc_offsets_kernel(const int32_t* __restrict__ g, int64_t n, int32_t G,
                                       int32_t* __restrict__ off) {
    for (int64_t h = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; h <= G;
         h += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (g[mid] < h) lo = mid + 1;
            else hi = mid;
        }
        off[h] = static_cast<int32_t>(lo);
    }
}

// One warp per (group, column): weighted mean by a fixed-order warp
// reduction (deterministic), then out = v - mean.
__global__ void noalloc_demean_kernel(const double* __restrict__ v, int64_t n, int cols,
                                      const int32_t* __restrict__ off, int32_t G,
                                      const double* __restrict__ w, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    const int64_t wid = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t items = static_cast<int64_t>(G) * cols;
    for (int64_t it = wid; it < items; it += warps) {
        const int64_t grp = it / cols;
        const int c = static_cast<int>(it - grp * cols);
        const int32_t b = off[grp], e = off[grp + 1];
        const double* col = v + static_cast<int64_t>(c) * n;
        double s = 0.0, W = 0.0;
        for (int32_t k = b + lane; k < e; k += 32) {
            const double wk = w ? w[k] : 1.0;
            s = fma(wk, col[k], s);
            W += wk;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            W += __shfl_xor_sync(0xffffffffu, W, o);
        }
        const double mean = W > 0.0 ? s / W : 0.0;
        double* oc = out + static_cast<int64_t>(c) * n;
        for (int32_t k = b + lane; k < e; k += 32) oc[k] = col[k] - mean;
    }
}

}  // namespace

namespace b200fe_host {

// Resolves the scratch array's device address once per device (that device
// current); the host-side name of the array is not a device address.  Called
// by b200fe_context_create, so a process that creates a context on a device
// loads this file's device code and places the array there before any
// no-alloc call, and by every no-alloc call (a lookup once resolved).
int noalloc_scratch_for_current_device(int32_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return B200FE_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = static_cast<int32_t*>(p);
    }
    if (out) *out = g_scratch_ptr[dev];
    return B200FE_OK;
}

}  // namespace b200fe_host

namespace {

int grid_cap(int64_t work, int threads, int cap) {
    const int64_t g = (work + threads - 1) / threads;
    return static_cast<int>(g < 1 ? 1 : (g < cap ? g : cap));
}

}  // namespace

extern "C" int b200fe_demean_sorted_noalloc(const double* d_v, int64_t n, int cols,
                                            const int32_t* d_group_ids, int32_t num_groups,
                                            const double* d_weights, double* d_out,
                                            void* stream) {
    if (!d_v || !d_out || !d_group_ids || n <= 0 || n >= (int64_t(1) << 31) - 1 || cols <= 0)
        return B200FE_INVALID_ARG;
    if (num_groups <= 0 || num_groups > kNoAllocMaxGroups) return B200FE_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    // an error left by the caller's earlier CUDA work is reported, not dropped
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return B200FE_CUDA_ERROR;
    }
    int32_t* scratch = nullptr;
    const int rc = b200fe_host::noalloc_scratch_for_current_device(&scratch);
    if (rc != B200FE_OK) return rc;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int32_t* status = scratch + kNoAllocStatus;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256;
    // the status word keeps the previous call's value: clear it first
    if (cudaMemsetAsync(status, 0, sizeof(int32_t), s) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_CUDA_ERROR;
    }
    noalloc_check_kernel<<<grid_cap(n, threads, sms * 8), threads, 0, s>>>(d_group_ids, n,
                                                                           num_groups, status);
    int32_t host_status = 0;
    if (cudaMemcpyAsync(&host_status, status, sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_CUDA_ERROR;
    }
    if (host_status != 0) return B200FE_INVALID_ARG;  // ids out of range or not sorted
    noalloc_offsets_kernel<<<grid_cap(static_cast<int64_t>(num_groups) + 1, threads, sms * 8),
                             threads, 0, s>>>(d_group_ids, n, num_groups, scratch);
    const int64_t warps = static_cast<int64_t>(num_groups) * cols;
    noalloc_demean_kernel<<<grid_cap(warps * 32, threads, sms * 16), threads, 0, s>>>(
        d_v, n, cols, scratch, num_groups, d_weights, d_out);
    if (cudaGetLastError() != cudaSuccess) return B200FE_CUDA_ERROR;
    return B200FE_OK;
}
