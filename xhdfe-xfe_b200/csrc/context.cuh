// Internal to the library (not installed): the context every entry point
// works on, its grow-only device workspace, the FE structure of the main
// solver, and the host helpers the translation units share (error macros,
// workspace buffers, grid sizing, CUB calls, event profiling).

#pragma once

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_segmented_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <string>
#include <unordered_map>
#include <vector>

#include "b200fe.h"
#include "limits.cuh"

namespace b200fe_host {

using namespace b200fe;

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct LargeDim {
    int dim = -1;
    int32_t G = 0;
    int64_t nruns = 0;
    int64_t nchunks = 0;
    int64_t nmulti = 0;
    int32_t *rid = nullptr, *run_base = nullptr, *run_dest = nullptr, *run_start = nullptr;
    int32_t* run_grp = nullptr;
    double* cw_run = nullptr;
    int32_t *chunk_grp = nullptr, *chunk_beg = nullptr, *chunk_end = nullptr;
    uint8_t* chunk_whole = nullptr;
    int32_t *multi_grp = nullptr, *multi_c0 = nullptr, *multi_c1 = nullptr;
    // second reduction level for groups of more than kFinFewParts chunks:
    // super-chunks of at most kSuperParts chunk partials
    int64_t nsup = 0;
    int32_t *multi_s0 = nullptr, *multi_s1 = nullptr;  // [nmulti] super range (empty: none)
    int32_t *sup_c0 = nullptr, *sup_c1 = nullptr;      // [nsup] chunk range of each super-chunk
};

struct Structure {
    bool valid = false;
    int64_t n = 0;
    int D = 0;
    int p = 0;
    int32_t G[B200FE_MAX_DIMS] = {0};
    int32_t present[B200FE_MAX_DIMS] = {0};
    int nL = 0, nS = 0;
    LargeDim L[kMaxLarge];
    int sdim[kMaxSmall] = {0};
    int32_t sG[kMaxSmall] = {0};
    int64_t lbase[kMaxLarge] = {0};
    int64_t sbase[kMaxSmall] = {0};
    int64_t GR = 0;
    bool weighted = false;
    double sum_w2 = 0.0;
    int32_t* pord = nullptr;
    int32_t* seg_off = nullptr;
    double* inv_wp = nullptr;
    double* wp64 = nullptr;
    float* wp32 = nullptr;
    uint32_t* sid = nullptr;
    double* dinv64 = nullptr;
    double* w_rows = nullptr;  // [GR] level weight of every alpha row
    float* dinv32 = nullptr;
    int32_t* gp = nullptr;  // primary ids in primary order (setup only)
    int SG = 0;             // bin rows over all small dims
    int sgoff[kMaxSmall] = {0};
    int32_t* tile_seg = nullptr;
    uint8_t* tile_long = nullptr;
    int64_t ntiles = 0;
    int32_t* long_segs = nullptr;
    int64_t nlong = 0;
    // block-level pass metadata (at most one large and one small dim)
    bool block_ok = false;
    int2* seg_meta = nullptr;
    int4* run_meta = nullptr;
    double* run_w64 = nullptr;
    float* run_w32 = nullptr;
    int2* block_meta = nullptr;
    double* block_w64 = nullptr;
    float* block_w32 = nullptr;
    int64_t nblocks = 0;
    double* small_w = nullptr;  // [SG] level weights of the small dim
    // dense coupling of the small dim (block level, one small dim): the CG
    // matvec then runs the block pass over the large dim only and adds
    // C_fy x_small, C_fy' x_f and C_yy x_small
    bool coupled = false;
    int SGP = 0;              // row stride of cfy: SG rounded up to 4 (padding zero)
    double* cfy64 = nullptr;  // [G_f][SGP]
    float* cfy32 = nullptr;
    double* cyy = nullptr;    // [SG][SG]
    // explicit Schur block of the one large dim (sparse_kernels.cuh): CSR rows
    // of S_ff over the large dim's levels; the CG matvec then gathers these
    // rows instead of passing over the runs
    bool sparse = false;
    int64_t sp_pairs = 0;              // contributions before merging
    int64_t sp_nnz = 0;
    int32_t* sp_row_off = nullptr;     // [G_f + 1]
    int32_t* sp_col = nullptr;         // [nnz] column (level of the large dim)
    double* sp_val64 = nullptr;        // [nnz]
    float* sp_val32 = nullptr;
    LargeDim sp;                       // chunk lists over the CSR rows (chunk fields only)
    // work lists of the persistent PCG over the same rows (pcg_kernels.cuh)
    int64_t pc_nshort = 0, pc_nlong = 0, pc_nlchunks = 0;
    int4* pc_short_meta = nullptr;     // {row, begin, end, 0} of the short rows
    int32_t *pc_long_rows = nullptr, *pc_long_c0 = nullptr, *pc_long_c1 = nullptr;
    int4* pc_lchunk_meta = nullptr;    // {row, begin, end, first} of the long-row chunks
    int64_t pc_nhuge = 0;
    int32_t* pc_huge_li = nullptr;
    // records of the regular tiles for the bulk-copy data passes
    // (stream_kernels.cuh); stream_ok when every one fits the staged sizes
    bool stream_ok = false;
    int64_t stream_nreg = 0;
    int4* stream_meta = nullptr;
    int32_t* stream_boff = nullptr;        // [nreg + 1] record offsets (16-byte units)
    unsigned char* stream_blob = nullptr;  // the records (stream_kernels.cuh: tile_blob_kernel)
    int stream_blob_max = 0;               // largest record (bytes)
    int stream_aux_stride = 0;
};

constexpr int32_t kChunkRuns = 64;

// The warm-start network (learned.cu): BF16 packing of FP32 master
// parameters into a named workspace buffer, and the forward pass y[n][2] of
// features x[n][8] on the context's stream.
int mlp_pack_device(b200fe_context* ctx, const float* d_params, const char* name, void** packed);
int mlp_forward_device(b200fe_context* ctx, const void* packed, const float* d_x, int64_t n, float* d_y);

// Device address of the no-alloc entry point's scratch array on the current
// device (noalloc.cu); resolving it loads that file's device code there.
int noalloc_scratch_for_current_device(int32_t** out);

}  // namespace b200fe_host

struct b200fe_context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    std::unordered_map<std::string, b200fe_host::Buf> bufs;
    b200fe_host::Structure st;
    long long launches = 0;
    long long lib_calls = 0;
    int* h_pinned = nullptr;     // small pinned scratch
    double* h_pinned_d = nullptr;
    // mapped pinned staging of the small transfers (small_d2h / small_h2d):
    // host pointer and the device's address of the same memory
    char* h_xout = nullptr;
    char* h_xout_dev = nullptr;
    char* h_xin = nullptr;
    char* h_xin_dev = nullptr;
    size_t xin_pos = 0;
    // opt-in event profiler (b200fe_options.profile)
    struct ProfRec {
        cudaEvent_t a, b;
        int cat;
        double bytes;
    };
    bool profiling = false;
    int pass_kernel = 0;
    bool sparse_schur = true;  // explicit Schur block of the large dim when it applies
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<ProfRec> prof;
    // saved FEs: device outputs per dim ([G_d][cols] column-major) while a
    // b200fe_absorb_fe call runs, and the first column of the current block
    double* fe_dev[B200FE_MAX_DIMS] = {nullptr};
    int fe_cols = 0;
    int fe_c0 = 0;
    // CUDA graphs of the PCG's check blocks (captured on cap_stream, launched
    // on the call's stream; one executable per kernel set, updated in place
    // for the next panel); off when B200FE_GRAPHS=0 at context creation
    bool graphs = true;
    // persistent PCG kernel over the explicit Schur block (one cooperative
    // launch per inner solve); off when B200FE_PERSISTENT=0 at context creation
    bool persistent = true;
    // host-array calls copy column groups in and out on their own streams,
    // overlapped with the solves of other groups; off when B200FE_PIPELINE=0
    bool pipeline = true;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    // FP64 data passes fed by bulk copies (stream_kernels.cuh); off when
    // B200FE_STREAM=0 at context creation.  stream_status is set by a pass
    // whose pipeline wait ran out; stream_smem_set marks the kernels whose
    // shared-memory limit was raised
    bool stream_pass = true;
    int* stream_status = nullptr;
    unsigned stream_smem_set = 0;
    // learned warm start (b200fe_warmstart_set): packed network and mode bits
    // (1: start the refinement from its prediction, 2: scale the Jacobi
    // diagonal by its per-row factor); training-sample collection
    // (b200fe_warmstart_samples) while ws_feat is set
    int ws_mode = 0;
    void* ws_packed = nullptr;
    float* ws_feat = nullptr;
    float* ws_targ = nullptr;
    int64_t ws_cap = 0, ws_count = 0;
    cudaStream_t cap_stream = nullptr;
    std::unordered_map<int, cudaGraphExec_t> graph_exec;
};

namespace b200fe_host {

using namespace b200fe;

#define B_TRY(expr)                                                              \
    do {                                                                         \
        cudaError_t e_ = (expr);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            ctx->err = std::string(#expr) + ": " + cudaGetErrorString(e_);       \
            return B200FE_CUDA_ERROR;                                            \
        }                                                                        \
    } while (0)

#define B_LAUNCHED()                                                             \
    do {                                                                         \
        ++ctx->launches;                                                         \
        cudaError_t e_ = cudaGetLastError();                                     \
        if (e_ != cudaSuccess) {                                                 \
            ctx->err = std::string("kernel launch: ") + cudaGetErrorString(e_);  \
            return B200FE_CUDA_ERROR;                                            \
        }                                                                        \
    } while (0)

#define B_CHECK(...)                                                             \
    do {                                                                         \
        int rc_ = (__VA_ARGS__);                                                        \
        if (rc_ != B200FE_OK) return rc_;                                        \
    } while (0)

// Debug aid: B200FE_POISON=<substring> fills newly allocated floating-point
// workspace whose name contains the substring ("*" for all) with NaN bytes,
// so a read before the first write shows up as a NaN.  Index arrays are never
// poisoned.
inline const char* poison_filter() {
    static const char* f = std::getenv("B200FE_POISON");
    return f;
}

template <typename T>
inline int get_buf(b200fe_context* ctx, const std::string& name, size_t count, T** out) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    bytes = (bytes + 255) & ~size_t(255);
    Buf& b = ctx->bufs[name];
    if (b.bytes < bytes) {
        if (b.p) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(b.p);
            b.p = nullptr;
            b.bytes = 0;
        }
        cudaError_t e = cudaMalloc(&b.p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ctx->err = "cudaMalloc(" + name + ", " + std::to_string(bytes) + " B): " +
                       cudaGetErrorString(e);
            return B200FE_CUDA_ERROR;
        }
        b.bytes = bytes;
        const char* pf = poison_filter();
        if (pf && (std::is_same<T, double>::value || std::is_same<T, float>::value) &&
            (std::strcmp(pf, "*") == 0 || name.find(pf) != std::string::npos)) {
            cudaMemsetAsync(b.p, 0xff, bytes, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
        }
    }
    *out = static_cast<T*>(b.p);
    return B200FE_OK;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit is process-wide per kernel and device, so it is only ever raised:
// contexts on other host threads that launch the same kernel with more shared
// memory are never undercut.
inline cudaError_t raise_smem_limit(const void* func, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    int& cur = limit[{dev, func}];
    if (cur >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

inline int grid_for(b200fe_context* ctx, int64_t work, int threads, int per_sm = 8) {
    int64_t g = (work + threads - 1) / threads;
    g = std::max<int64_t>(1, std::min<int64_t>(g, static_cast<int64_t>(ctx->num_sms) * per_sm));
    return static_cast<int>(g);
}

// Records a CUDA-event interval on the context stream around a scope when
// profiling is on; the bytes are the launches' algorithmic traffic.
struct ProfScope {
    b200fe_context* ctx;
    int cat;
    double bytes;
    cudaEvent_t a = nullptr;
    static cudaEvent_t event(b200fe_context* c) {
        if (c->ev_used < c->ev_pool.size()) return c->ev_pool[c->ev_used++];
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        c->ev_pool.push_back(e);
        ++c->ev_used;
        return e;
    }
    ProfScope(b200fe_context* c, int category, double b) : ctx(c), cat(category), bytes(b) {
        if (ctx->profiling) {
            a = event(ctx);
            if (a) cudaEventRecord(a, ctx->stream);
        }
    }
    ~ProfScope() {
        if (ctx->profiling && a) {
            cudaEvent_t b = event(ctx);
            if (b) {
                cudaEventRecord(b, ctx->stream);
                ctx->prof.push_back({a, b, cat, bytes});
            }
        }
    }
};

// ---------------------------------------------------------------------------
// CUB helpers (setup only)
// ---------------------------------------------------------------------------
inline int cub_exclusive_sum(b200fe_context* ctx, const int32_t* in, int32_t* out, int64_t n) {
    size_t tmp = 0;
    B_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, ctx->stream));
    void* t;
    B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
    B_TRY(cub::DeviceScan::ExclusiveSum(t, tmp, in, out, n, ctx->stream));
    ++ctx->lib_calls;
    return B200FE_OK;
}

inline int cub_inclusive_sum(b200fe_context* ctx, const int32_t* in, int32_t* out, int64_t n) {
    size_t tmp = 0;
    B_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp, in, out, n, ctx->stream));
    void* t;
    B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
    B_TRY(cub::DeviceScan::InclusiveSum(t, tmp, in, out, n, ctx->stream));
    ++ctx->lib_calls;
    return B200FE_OK;
}

inline int bits_for(int32_t G) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) < G) ++b;
    return b;
}

// Stable sort of (key, value) pairs by key.
inline int cub_sort_pairs(b200fe_context* ctx, const int32_t* keys_in, int32_t* keys_out,
                   const int32_t* vals_in, int32_t* vals_out, int64_t n, int32_t G) {
    size_t tmp = 0;
    const uint32_t* ki = reinterpret_cast<const uint32_t*>(keys_in);
    uint32_t* ko = reinterpret_cast<uint32_t*>(keys_out);
    const int eb = bits_for(G);
    B_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ki, ko, vals_in, vals_out, n, 0, eb,
                                          ctx->stream));
    void* t;
    B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
    B_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, ki, ko, vals_in, vals_out, n, 0, eb,
                                          ctx->stream));
    ++ctx->lib_calls;
    return B200FE_OK;
}

// Small transfers between host and device that bypass the copy engines: a
// kernel on the context's stream reads or writes the context's mapped pinned
// staging memory.  A copy-engine transfer queues behind every large copy
// already submitted in the same direction (on any stream), so a scalar read
// back by the solver would wait for a gigabyte copy overlapped with it on
// another stream; these do not.  Sizes are multiples of 4 bytes.
constexpr size_t kXferOutBytes = size_t(1) << 20;
constexpr size_t kXferInBytes = size_t(1) << 16;

static __global__ void xfer_words_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                         int64_t nwords) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nwords;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = src[i];
}

inline int launch_xfer(b200fe_context* ctx, const void* src, void* dst, size_t bytes) {
    const int64_t words = static_cast<int64_t>(bytes / 4);
    const int grid = static_cast<int>(std::min<int64_t>((words + 255) / 256, 64));
    xfer_words_kernel<<<std::max(grid, 1), 256, 0, ctx->stream>>>(static_cast<const uint32_t*>(src),
                                                                   static_cast<uint32_t*>(dst), words);
    ++ctx->launches;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->err = std::string("kernel launch: ") + cudaGetErrorString(e);
        return B200FE_CUDA_ERROR;
    }
    return B200FE_OK;
}

// device -> host, waits for the context's stream
inline int small_d2h(b200fe_context* ctx, const void* dptr, size_t bytes, void* host) {
    if (bytes == 0) return B200FE_OK;
    if (!ctx->h_xout || bytes > kXferOutBytes || (bytes & 3)) {
        B_TRY(cudaMemcpyAsync(host, dptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        B_TRY(cudaStreamSynchronize(ctx->stream));
        return B200FE_OK;
    }
    B_CHECK(launch_xfer(ctx, dptr, ctx->h_xout_dev, bytes));
    B_TRY(cudaStreamSynchronize(ctx->stream));
    std::memcpy(host, ctx->h_xout, bytes);
    return B200FE_OK;
}

// host -> device, stream-ordered; the host data is staged at once, so the
// caller may reuse its buffer on return
inline int small_h2d(b200fe_context* ctx, void* dptr, const void* host, size_t bytes) {
    if (bytes == 0) return B200FE_OK;
    if (!ctx->h_xin || bytes > kXferInBytes || (bytes & 3)) {
        B_TRY(cudaMemcpyAsync(dptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
        B_TRY(cudaStreamSynchronize(ctx->stream));
        return B200FE_OK;
    }
    const size_t slot = (bytes + 255) & ~size_t(255);
    if (ctx->xin_pos + slot > kXferInBytes) {  // earlier slots may still be read
        B_TRY(cudaStreamSynchronize(ctx->stream));
        ctx->xin_pos = 0;
    }
    std::memcpy(ctx->h_xin + ctx->xin_pos, host, bytes);
    B_CHECK(launch_xfer(ctx, ctx->h_xin_dev + ctx->xin_pos, dptr, bytes));
    ctx->xin_pos += slot;
    return B200FE_OK;
}

inline int sync_read_int(b200fe_context* ctx, const int32_t* dptr, int count, int* host) {
    return small_d2h(ctx, dptr, sizeof(int) * count, host);
}

inline int sync_read_double(b200fe_context* ctx, const double* dptr, int count, double* host) {
    return small_d2h(ctx, dptr, sizeof(double) * count, host);
}

inline int check_common(b200fe_context* ctx, int64_t n, int cols, int num_dims, const int32_t* G) {
    if (!ctx) return B200FE_INVALID_ARG;
    if (n <= 0 || n >= (int64_t(1) << 31) - 1) {
        ctx->err = "n must be in [1, 2^31-2]";
        return B200FE_INVALID_ARG;
    }
    if (cols <= 0) {
        ctx->err = "need at least one column";
        return B200FE_INVALID_ARG;
    }
    if (num_dims < 0 || num_dims > B200FE_MAX_DIMS) {
        ctx->err = "num_dims must be in [0, 8]";
        return B200FE_INVALID_ARG;
    }
    for (int d = 0; d < num_dims; ++d) {
        if (!G || G[d] <= 0) {
            ctx->err = "num_groups must be positive";
            return B200FE_INVALID_ARG;
        }
    }
    return B200FE_OK;
}
inline double tol_eff(const b200fe_options& o) {
    if (o.tol > 0.0 && o.tolerance_mode == 1) return std::min(o.tol, 1e-9);
    return o.tol;
}
inline float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return 0.0f;
    }
    return ms;
}
inline void clear_result(b200fe_result* r) {
    std::memset(r, 0, sizeof(*r));
    r->primary_dim = -1;
}

}  // namespace b200fe_host
