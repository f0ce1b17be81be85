// AKM/KSS two-way solver: batched grounded Jacobi-PCG on the firm system
//
//     S z = rhs,   S = Df - B' Dw^{-1} B   (J x J, ground firm J-1 pinned),
//
// with B the N x J worker-firm match matrix (entries m_c), Dw / Df its row and
// column sums.  This is the linear system behind every leverage, JLA draw and
// standard-error simulation of the reference's leave-out decomposition
// (src/akm_kss.cpp TwoWaySolver, :1000-1800); its CUDA backend is
// src/akm_kss_cuda.cu (akm_cuda_solve_S / akm_cuda_solve_S_multi).
//
// B200 layout and schedule (not the reference's):
//   * every solver vector is stored lane-interleaved, [rows][LW] with LW the
//     lane pitch (a power of two >= nb): the row of a firm or worker holds
//     all lanes contiguously, so each match gathers one coalesced row
//     (256 B at 32 lanes) instead of nb scattered doubles;
//   * S p is two passes over the matches: a worker pass t = Dw^{-1} B p (one
//     group of lanes per worker, matches in worker order) and a firm pass
//     Ap = Df p - B' t over the matches in firm order, cut into chunks of at
//     most kChunk matches so a firm with a large share of the matches (Zipf
//     firm sizes) is summed by many groups; chunk partials are combined per
//     firm in chunk order (fixed order, no atomics);
//   * the PCG scalars (alpha, beta, convergence, per-lane iteration counts and
//     retirement) are computed on the device by the last CTA of each
//     reduction, so a PCG step has no host round trip; the host reads one
//     counter of active lanes every kPollEvery steps.  A retired lane is
//     frozen exactly as in the reference, so per-lane iteration counts and
//     results follow the same stopping rule.
// Every reduction has a fixed order: results are bitwise reproducible.

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "b200fe.h"

namespace {

constexpr int kKssThreads = 256;
constexpr int kKssMaxLanes = 64;
constexpr int kChunk = 64;      // matches per firm chunk
constexpr int kPollEvery = 8;   // PCG steps between host reads of the active-lane count

// Per-lane PCG state on the device.
struct KssScalars {
    double alpha[kKssMaxLanes];
    double beta[kKssMaxLanes];
    double rz[kKssMaxLanes];
    double tol2[kKssMaxLanes];
    int its[kKssMaxLanes];
    int active[kKssMaxLanes];
    int ok[kKssMaxLanes];
    int nactive;
    int nb;
    int max_iter;
    double tol;
    unsigned int ticket;
};

enum KssAction { kActNorm = 0, kActRz = 1, kActAlpha = 2, kActConverge = 3 };

// ---------------------------------------------------------------------------
// Kernels.  LW = lane pitch; a group of TG = min(LW, 32) threads owns one row,
// VL = LW / TG lanes per thread.
// ---------------------------------------------------------------------------
template <int LW>
struct LaneGeom {
    static constexpr int TG = LW < 32 ? LW : 32;
    static constexpr int VL = LW / TG;
};

template <int VL>
__device__ __forceinline__ void row_load(const double* p, double (&v)[VL]) {
    if constexpr (VL == 2) {
        const double2 d = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = d.x;
        v[1] = d.y;
    } else {
        v[0] = __ldg(p);
    }
}

template <int VL>
__device__ __forceinline__ void row_store(double* p, const double (&v)[VL]) {
    if constexpr (VL == 2) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    } else {
        p[0] = v[0];
    }
}

// t[w] = Dw^{-1} sum_{matches a of w} c_a p[f_a]   (matches in worker order)
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_worker_kernel(int N, const int64_t* __restrict__ w_ptr, const int32_t* __restrict__ m_f,
                  const double* __restrict__ m_c, const double* __restrict__ inv_dw,
                  const double* __restrict__ p, double* __restrict__ t,
                  const KssScalars* __restrict__ sc) {
    if (sc->nactive == 0) return;
    constexpr int TG = LaneGeom<LW>::TG, VL = LaneGeom<LW>::VL;
    const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x) / TG;
    const int tg = threadIdx.x % TG;
    const int64_t ng = static_cast<int64_t>(gridDim.x) * (kKssThreads / TG);
    for (int64_t w = g0; w < N; w += ng) {
        double acc[VL];
#pragma unroll
        for (int v = 0; v < VL; ++v) acc[v] = 0.0;
        const int64_t a1 = __ldg(w_ptr + w + 1);
        for (int64_t a = __ldg(w_ptr + w); a < a1; ++a) {
            const int64_t f = __ldg(m_f + a);
            const double c = __ldg(m_c + a);
            double pv[VL];
            row_load<VL>(p + f * LW + tg * VL, pv);
#pragma unroll
            for (int v = 0; v < VL; ++v) acc[v] = fma(c, pv[v], acc[v]);
        }
        const double iw = __ldg(inv_dw + w);
#pragma unroll
        for (int v = 0; v < VL; ++v) acc[v] *= iw;
        row_store<VL>(t + w * LW + tg * VL, acc);
    }
}

// Firm chunks: acc = sum_{a in chunk} c_a t[w_a] (matches in firm order).  A
// firm of one chunk writes Ap[f] = Df[f] p[f] - acc (0 at the ground); a
// longer firm writes its chunk partials, combined by kss_firm_combine_kernel.
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_firm_kernel(int64_t nchunks, const int64_t* __restrict__ cbeg, const int32_t* __restrict__ cfirm,
                const int32_t* __restrict__ cslot, const int32_t* __restrict__ mw_f,
                const double* __restrict__ mc_f, const double* __restrict__ t,
                const double* __restrict__ Df, const double* __restrict__ p,
                double* __restrict__ Ap, double* __restrict__ part, int ground,
                const KssScalars* __restrict__ sc) {
    if (sc->nactive == 0) return;
    constexpr int TG = LaneGeom<LW>::TG, VL = LaneGeom<LW>::VL;
    const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x) / TG;
    const int tg = threadIdx.x % TG;
    const int64_t ng = static_cast<int64_t>(gridDim.x) * (kKssThreads / TG);
    for (int64_t k = g0; k < nchunks; k += ng) {
        double acc[VL];
#pragma unroll
        for (int v = 0; v < VL; ++v) acc[v] = 0.0;
        const int64_t a1 = __ldg(cbeg + k + 1);
        for (int64_t a = __ldg(cbeg + k); a < a1; ++a) {
            const int64_t w = __ldg(mw_f + a);
            const double c = __ldg(mc_f + a);
            double tv[VL];
            row_load<VL>(t + w * LW + tg * VL, tv);
#pragma unroll
            for (int v = 0; v < VL; ++v) acc[v] = fma(c, tv[v], acc[v]);
        }
        const int32_t slot = __ldg(cslot + k);
        if (slot >= 0) {
            row_store<VL>(part + static_cast<int64_t>(slot) * LW + tg * VL, acc);
        } else {
            const int64_t f = __ldg(cfirm + k);
            double pv[VL], out[VL];
            row_load<VL>(p + f * LW + tg * VL, pv);
            const double df = __ldg(Df + f);
#pragma unroll
            for (int v = 0; v < VL; ++v) out[v] = (f == ground) ? 0.0 : df * pv[v] - acc[v];
            row_store<VL>(Ap + f * LW + tg * VL, out);
        }
    }
}

template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_firm_combine_kernel(int64_t nmulti, const int32_t* __restrict__ mfirm,
                        const int32_t* __restrict__ mslot0, const int32_t* __restrict__ mnslot,
                        const double* __restrict__ part, const double* __restrict__ Df,
                        const double* __restrict__ p, double* __restrict__ Ap, int ground,
                        const KssScalars* __restrict__ sc) {
    if (sc->nactive == 0) return;
    constexpr int TG = LaneGeom<LW>::TG, VL = LaneGeom<LW>::VL;
    const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x) / TG;
    const int tg = threadIdx.x % TG;
    const int64_t ng = static_cast<int64_t>(gridDim.x) * (kKssThreads / TG);
    for (int64_t i = g0; i < nmulti; i += ng) {
        const int64_t f = __ldg(mfirm + i);
        const int64_t s0 = __ldg(mslot0 + i);
        const int ns = __ldg(mnslot + i);
        double acc[VL];
#pragma unroll
        for (int v = 0; v < VL; ++v) acc[v] = 0.0;
        for (int s = 0; s < ns; ++s) {
            double pv[VL];
            row_load<VL>(part + (s0 + s) * LW + tg * VL, pv);
#pragma unroll
            for (int v = 0; v < VL; ++v) acc[v] += pv[v];
        }
        double pv[VL], out[VL];
        row_load<VL>(p + f * LW + tg * VL, pv);
        const double df = __ldg(Df + f);
#pragma unroll
        for (int v = 0; v < VL; ++v) out[v] = (f == ground) ? 0.0 : df * pv[v] - acc[v];
        row_store<VL>(Ap + f * LW + tg * VL, out);
    }
}

// The per-lane scalar step run by the last CTA of a reduction (thread l owns
// lane l).  Mirrors the host logic of akm_cuda_solve_S_multi
// (src/akm_kss_cuda.cu:575-640).
__device__ void kss_action(KssScalars* sc, int action, int l, double d0, double d1) {
    const bool lane_used = l < sc->nb;
    switch (action) {
        case kActNorm:  // d0 = ||r||^2 of the grounded rhs
            sc->tol2[l] = sc->tol * sc->tol * d0;
            sc->its[l] = 0;
            sc->ok[l] = (lane_used && d0 == 0.0) ? 1 : 0;
            sc->active[l] = (lane_used && d0 != 0.0) ? 1 : 0;
            sc->alpha[l] = 0.0;
            sc->beta[l] = 0.0;
            break;
        case kActRz:
            sc->rz[l] = d0;
            break;
        case kActAlpha:  // d0 = p'Ap
            if (!sc->active[l]) {
                sc->alpha[l] = 0.0;
            } else if (!(d0 > 0.0) || !(d0 < 1e300)) {
                sc->active[l] = 0;  // breakdown: the lane fails
                sc->alpha[l] = 0.0;
            } else {
                sc->alpha[l] = sc->rz[l] / d0;
            }
            break;
        case kActConverge:  // d0 = ||r||^2, d1 = r'z after the update
            if (sc->active[l]) {
                ++sc->its[l];
                if (d0 <= sc->tol2[l]) {
                    sc->ok[l] = 1;
                    sc->active[l] = 0;
                } else if (sc->its[l] >= sc->max_iter) {
                    sc->active[l] = 0;
                }
            }
            if (sc->active[l]) {
                const double rz = sc->rz[l];
                sc->beta[l] = (rz != 0.0) ? d1 / rz : 0.0;
                sc->rz[l] = d1;
            } else {
                sc->beta[l] = 0.0;
            }
            break;
        default:
            break;
    }
}

// Block partials of one or two per-lane dots, then the last CTA sums the
// partials in block order and runs the scalar step.
template <int LW, int NDOT>
__device__ __forceinline__ void kss_reduce_tail(double s0, double s1, double* __restrict__ part,
                                                KssScalars* sc, int action) {
    __shared__ double red[NDOT][kKssThreads];
    __shared__ bool last;
    const int tid = threadIdx.x;
    red[0][tid] = s0;
    if (NDOT == 2) red[NDOT - 1][tid] = s1;
    __syncthreads();
    if (tid < LW) {
#pragma unroll
        for (int d = 0; d < NDOT; ++d) {
            double acc = 0.0;
            for (int j = tid; j < kKssThreads; j += LW) acc += red[d][j];
            part[(static_cast<int64_t>(blockIdx.x) * NDOT + d) * LW + tid] = acc;
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (tid < LW) {
        double d[2] = {0.0, 0.0};
        for (unsigned b = 0; b < gridDim.x; ++b)
#pragma unroll
            for (int k = 0; k < NDOT; ++k) d[k] += __ldcg(part + (static_cast<int64_t>(b) * NDOT + k) * LW + tid);
        kss_action(sc, action, tid, d[0], d[1]);
    }
    __syncthreads();
    if (tid == 0) {
        int na = 0;
        for (int l = 0; l < LW; ++l) na += sc->active[l];
        sc->nactive = na;
        sc->ticket = 0;
    }
}

// One per-lane dot a'b over rows x LW, then the scalar step.
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_dot_kernel(int64_t rows, const double* __restrict__ a, const double* __restrict__ b,
               double* __restrict__ part, KssScalars* sc, int action, int skip_if_done) {
    if (skip_if_done && sc->nactive == 0) return;
    const int64_t total = rows * LW;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kKssThreads;
    double s = 0.0;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x; e < total; e += stride)
        s = fma(__ldcg(a + e), __ldcg(b + e), s);
    kss_reduce_tail<LW, 1>(s, 0.0, part, sc, action);
}

// x += alpha p, r -= alpha Ap, z = inv_diag r for active lanes, with the
// dots r'r and r'z; then the convergence / beta step.
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_update_kernel(int64_t rows, const double* __restrict__ inv_diag, const double* __restrict__ p,
                  const double* __restrict__ Ap, double* __restrict__ x, double* __restrict__ r,
                  double* __restrict__ z, double* __restrict__ part, KssScalars* sc) {
    if (sc->nactive == 0) return;
    const int lane = threadIdx.x % LW;  // fixed per thread: the stride is a multiple of LW
    const bool act = sc->active[lane] != 0;
    const double al = sc->alpha[lane];
    const int64_t total = rows * LW;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kKssThreads;
    double rr = 0.0, rzs = 0.0;
    if (act) {
        for (int64_t e = static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x; e < total;
             e += stride) {
            const double pe = __ldcg(p + e);
            const double ape = __ldcg(Ap + e);
            x[e] = fma(al, pe, x[e]);
            const double re = fma(-al, ape, r[e]);
            r[e] = re;
            const double ze = __ldg(inv_diag + e / LW) * re;
            z[e] = ze;
            rr = fma(re, re, rr);
            rzs = fma(re, ze, rzs);
        }
    }
    kss_reduce_tail<LW, 2>(rr, rzs, part, sc, kActConverge);
}

// p = z + beta p for active lanes.
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_direction_kernel(int64_t rows, const double* __restrict__ z, double* __restrict__ p,
                     const KssScalars* __restrict__ sc) {
    if (sc->nactive == 0) return;
    const int lane = threadIdx.x % LW;
    if (!sc->active[lane]) return;
    const double be = sc->beta[lane];
    const int64_t total = rows * LW;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kKssThreads;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x; e < total; e += stride)
        p[e] = fma(be, p[e], __ldcg(z + e));
}

// z = inv_diag r (lanes that start active), p = z.
template <int LW>
__global__ void __launch_bounds__(kKssThreads)
kss_precond_init_kernel(int64_t rows, const double* __restrict__ inv_diag, const double* __restrict__ r,
                        double* __restrict__ z, double* __restrict__ p, const KssScalars* __restrict__ sc) {
    const int lane = threadIdx.x % LW;
    const bool act = sc->active[lane] != 0;
    const int64_t total = rows * LW;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kKssThreads;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * kKssThreads + threadIdx.x; e < total; e += stride) {
        const double ze = act ? __ldg(inv_diag + e / LW) * r[e] : 0.0;
        z[e] = ze;
        p[e] = ze;
    }
}

// lane-major [nb][J] -> interleaved [J][LW], ground row and padding lanes zero
__global__ void kss_pack_in_kernel(int64_t J, int LW, int nb, int ground,
                                   const double* __restrict__ src, double* __restrict__ dst) {
    const int64_t total = J * LW;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t row = e / LW;
        const int l = static_cast<int>(e - row * LW);
        dst[e] = (l < nb && row != ground) ? src[static_cast<int64_t>(l) * J + row] : 0.0;
    }
}

// interleaved x -> lane-major [nb][J]; ground entries and failed lanes zero
__global__ void kss_pack_out_kernel(int64_t J, int LW, int nb, int ground,
                                    const double* __restrict__ x, double* __restrict__ dst,
                                    const KssScalars* __restrict__ sc) {
    const int64_t total = J * nb;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int l = static_cast<int>(e / J);
        const int64_t row = e - static_cast<int64_t>(l) * J;
        dst[e] = (sc->ok[l] && row != ground) ? x[row * LW + l] : 0.0;
    }
}

__global__ void kss_iota_kernel(int64_t* out, int64_t n) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = i;
}

int lane_pitch(int nb) {
    int lw = 1;
    while (lw < nb) lw <<= 1;
    return lw;
}

}  // namespace

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct b200fe_kss {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    int N = 0, J = 0, ground = 0;
    int64_t M = 0;
    // structure (device)
    int64_t* w_ptr = nullptr;
    int32_t* m_f = nullptr;
    double* m_c = nullptr;
    double* inv_dw = nullptr;
    int32_t* mw_f = nullptr;  // worker of each match, firm order
    double* mc_f = nullptr;   // weight of each match, firm order
    int64_t* cbeg = nullptr;
    int32_t* cfirm = nullptr;
    int32_t* cslot = nullptr;
    int64_t nchunks = 0;
    int32_t* mfirm = nullptr;
    int32_t* mslot0 = nullptr;
    int32_t* mnslot = nullptr;
    int64_t nmulti = 0, nslots = 0;
    double* Df = nullptr;
    double* inv_diag = nullptr;
    // workspace for lw_cap lanes
    int lw_cap = 0;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *t = nullptr;
    double* slot_part = nullptr;
    double* dot_part = nullptr;
    double* stage = nullptr;
    int dot_grid = 0;
    KssScalars* sc = nullptr;
    KssScalars* h_sc = nullptr;  // pinned copy
    double* h_pack = nullptr;
    int pack_nb = 0;
    std::vector<void*> owned;

    ~b200fe_kss() {
        if (device >= 0) cudaSetDevice(device);
        for (void* q : owned) cudaFree(q);
        cudaFree(x); cudaFree(r); cudaFree(z); cudaFree(p); cudaFree(Ap); cudaFree(t);
        cudaFree(slot_part); cudaFree(stage);
        if (h_pack) cudaFreeHost(h_pack);
        if (h_sc) cudaFreeHost(h_sc);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

#define K_TRY(call)                                                        \
    do {                                                                   \
        const cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) {                                           \
            kss->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            cudaGetLastError();                                            \
            return B200FE_CUDA_ERROR;                                      \
        }                                                                  \
    } while (0)

template <typename T>
int upload(b200fe_kss* kss, T** dst, const T* src, size_t count) {
    K_TRY(cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(count, 1)));
    kss->owned.push_back(*dst);
    if (count) K_TRY(cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice));
    return B200FE_OK;
}

#define K_CHECK(expr)                      \
    do {                                   \
        const int rc_ = (expr);            \
        if (rc_ != B200FE_OK) return rc_;  \
    } while (0)

int ensure_lanes(b200fe_kss* kss, int lw) {
    if (kss->lw_cap >= lw) return B200FE_OK;
    cudaFree(kss->x); cudaFree(kss->r); cudaFree(kss->z); cudaFree(kss->p); cudaFree(kss->Ap);
    cudaFree(kss->t); cudaFree(kss->slot_part); cudaFree(kss->stage);
    kss->x = kss->r = kss->z = kss->p = kss->Ap = kss->t = kss->slot_part = kss->stage = nullptr;
    kss->lw_cap = 0;
    const size_t J = static_cast<size_t>(kss->J), N = static_cast<size_t>(kss->N);
    const size_t L = static_cast<size_t>(lw);
    K_TRY(cudaMalloc(&kss->x, sizeof(double) * J * L));
    K_TRY(cudaMalloc(&kss->r, sizeof(double) * J * L));
    K_TRY(cudaMalloc(&kss->z, sizeof(double) * J * L));
    K_TRY(cudaMalloc(&kss->p, sizeof(double) * J * L));
    K_TRY(cudaMalloc(&kss->Ap, sizeof(double) * J * L));
    K_TRY(cudaMalloc(&kss->t, sizeof(double) * std::max<size_t>(N, 1) * L));
    K_TRY(cudaMalloc(&kss->slot_part, sizeof(double) * std::max<int64_t>(kss->nslots, 1) * L));
    K_TRY(cudaMalloc(&kss->stage, sizeof(double) * J * L));
    kss->lw_cap = lw;
    return B200FE_OK;
}

int grid_for(const b200fe_kss* kss, int64_t threads, int per_sm) {
    const int64_t g = (threads + kKssThreads - 1) / kKssThreads;
    const int64_t cap = static_cast<int64_t>(kss->sms) * per_sm;
    return static_cast<int>(std::max<int64_t>(1, std::min(g, cap)));
}

template <int LW>
int run_solve(b200fe_kss* kss, int nb) {
    constexpr int TG = LaneGeom<LW>::TG;
    const cudaStream_t s = kss->stream;
    const int64_t J = kss->J;
    const int flat_grid = grid_for(kss, J * LW, 4);
    const int worker_grid = grid_for(kss, static_cast<int64_t>(kss->N) * TG, 8);
    const int firm_grid = grid_for(kss, kss->nchunks * TG, 8);
    const int multi_grid = grid_for(kss, kss->nmulti * TG, 8);
    // r = grounded rhs, x = 0; ||r||^2 -> tol2, active lanes
    kss_pack_in_kernel<<<flat_grid, kKssThreads, 0, s>>>(J, LW, nb, kss->ground, kss->stage, kss->r);
    K_TRY(cudaMemsetAsync(kss->x, 0, sizeof(double) * J * LW, s));
    K_TRY(cudaMemsetAsync(kss->Ap, 0, sizeof(double) * J * LW, s));
    kss_dot_kernel<LW><<<kss->dot_grid, kKssThreads, 0, s>>>(J, kss->r, kss->r, kss->dot_part, kss->sc,
                                                            kActNorm, 0);
    kss_precond_init_kernel<LW><<<flat_grid, kKssThreads, 0, s>>>(J, kss->inv_diag, kss->r, kss->z,
                                                                 kss->p, kss->sc);
    kss_dot_kernel<LW><<<kss->dot_grid, kKssThreads, 0, s>>>(J, kss->r, kss->z, kss->dot_part, kss->sc,
                                                            kActRz, 0);
    K_TRY(cudaGetLastError());
    for (;;) {
        for (int step = 0; step < kPollEvery; ++step) {
            kss_worker_kernel<LW><<<worker_grid, kKssThreads, 0, s>>>(
                kss->N, kss->w_ptr, kss->m_f, kss->m_c, kss->inv_dw, kss->p, kss->t, kss->sc);
            kss_firm_kernel<LW><<<firm_grid, kKssThreads, 0, s>>>(
                kss->nchunks, kss->cbeg, kss->cfirm, kss->cslot, kss->mw_f, kss->mc_f, kss->t, kss->Df,
                kss->p, kss->Ap, kss->slot_part, kss->ground, kss->sc);
            if (kss->nmulti > 0)
                kss_firm_combine_kernel<LW><<<multi_grid, kKssThreads, 0, s>>>(
                    kss->nmulti, kss->mfirm, kss->mslot0, kss->mnslot, kss->slot_part, kss->Df, kss->p,
                    kss->Ap, kss->ground, kss->sc);
            kss_dot_kernel<LW><<<kss->dot_grid, kKssThreads, 0, s>>>(J, kss->p, kss->Ap, kss->dot_part,
                                                                    kss->sc, kActAlpha, 1);
            kss_update_kernel<LW><<<kss->dot_grid, kKssThreads, 0, s>>>(
                J, kss->inv_diag, kss->p, kss->Ap, kss->x, kss->r, kss->z, kss->dot_part, kss->sc);
            kss_direction_kernel<LW><<<flat_grid, kKssThreads, 0, s>>>(J, kss->z, kss->p, kss->sc);
        }
        K_TRY(cudaGetLastError());
        K_TRY(cudaMemcpyAsync(&kss->h_sc->nactive, &kss->sc->nactive, sizeof(int), cudaMemcpyDeviceToHost, s));
        K_TRY(cudaStreamSynchronize(s));
        if (kss->h_sc->nactive == 0) break;
    }
    kss_pack_out_kernel<<<flat_grid, kKssThreads, 0, s>>>(J, LW, nb, kss->ground, kss->x, kss->stage,
                                                          kss->sc);
    K_TRY(cudaGetLastError());
    return B200FE_OK;
}

int solve_lanes(b200fe_kss* kss, const double* rhs_pack, double* z_pack, int nb, double tol,
                int max_iter, int* iters_out) {
    if (!kss || !rhs_pack || !z_pack || !iters_out || nb < 1 || nb > kKssMaxLanes || !(tol >= 0.0))
        return B200FE_INVALID_ARG;
    K_TRY(cudaSetDevice(kss->device));
    const int lw = lane_pitch(nb);
    K_CHECK(ensure_lanes(kss, lw));
    const cudaStream_t s = kss->stream;
    const size_t bytes = sizeof(double) * static_cast<size_t>(kss->J) * nb;
    // scalars: nb, tol, max_iter; nactive > 0 so the first reductions run
    KssScalars init;
    std::memset(&init, 0, sizeof(init));
    init.nb = nb;
    init.tol = tol;
    init.max_iter = max_iter;
    init.nactive = 1;
    *kss->h_sc = init;
    K_TRY(cudaMemcpyAsync(kss->sc, kss->h_sc, sizeof(KssScalars), cudaMemcpyHostToDevice, s));
    K_TRY(cudaMemcpyAsync(kss->stage, rhs_pack, bytes, cudaMemcpyHostToDevice, s));
    int rc = B200FE_OK;
    switch (lw) {
        case 1: rc = run_solve<1>(kss, nb); break;
        case 2: rc = run_solve<2>(kss, nb); break;
        case 4: rc = run_solve<4>(kss, nb); break;
        case 8: rc = run_solve<8>(kss, nb); break;
        case 16: rc = run_solve<16>(kss, nb); break;
        case 32: rc = run_solve<32>(kss, nb); break;
        default: rc = run_solve<64>(kss, nb); break;
    }
    if (rc != B200FE_OK) return rc;
    K_TRY(cudaMemcpyAsync(z_pack, kss->stage, bytes, cudaMemcpyDeviceToHost, s));
    K_TRY(cudaMemcpyAsync(kss->h_sc, kss->sc, sizeof(KssScalars), cudaMemcpyDeviceToHost, s));
    K_TRY(cudaStreamSynchronize(s));
    for (int l = 0; l < nb; ++l) iters_out[l] = kss->h_sc->ok[l] ? kss->h_sc->its[l] : -1;
    return B200FE_OK;
}

}  // namespace

extern "C" {

int b200fe_kss_create(int n_workers, int n_firms, const int32_t* m_w, const int32_t* m_f,
                      const double* m_c, int64_t n_matches, const int64_t* w_ptr,
                      const int64_t* f_ptr, const int64_t* f_matches, const double* Dw,
                      const double* Df, const double* inv_diagS, b200fe_kss** out) {
    if (!out) return B200FE_INVALID_ARG;
    *out = nullptr;
    if (n_workers < 0 || n_firms < 1 || n_matches < 0 || n_matches >= INT_MAX || !w_ptr || !f_ptr ||
        !Dw || !Df || !inv_diagS || (n_matches > 0 && (!m_w || !m_f || !m_c || !f_matches)))
        return B200FE_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    // host-side checks of the structure the kernels index by
    if (w_ptr[0] != 0 || w_ptr[n_workers] != n_matches || f_ptr[0] != 0 || f_ptr[n_firms] != n_matches)
        return B200FE_INVALID_ARG;
    for (int w = 0; w < n_workers; ++w)
        if (w_ptr[w + 1] < w_ptr[w]) return B200FE_INVALID_ARG;
    for (int f = 0; f < n_firms; ++f)
        if (f_ptr[f + 1] < f_ptr[f]) return B200FE_INVALID_ARG;
    for (int64_t m = 0; m < n_matches; ++m) {
        if (m_f[m] < 0 || m_f[m] >= n_firms || m_w[m] < 0 || m_w[m] >= n_workers) return B200FE_INVALID_ARG;
        if (f_matches[m] < 0 || f_matches[m] >= n_matches) return B200FE_INVALID_ARG;
    }
    b200fe_kss* kss = new (std::nothrow) b200fe_kss();
    if (!kss) return B200FE_CUDA_ERROR;
    auto fail = [&](int rc) {
        delete kss;
        return rc;
    };
    if (cudaGetDevice(&kss->device) != cudaSuccess) {
        cudaGetLastError();
        return fail(B200FE_UNAVAILABLE);
    }
    cudaDeviceGetAttribute(&kss->sms, cudaDevAttrMultiProcessorCount, kss->device);
    if (cudaStreamCreateWithFlags(&kss->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return fail(B200FE_CUDA_ERROR);
    }
    kss->N = n_workers;
    kss->J = n_firms;
    kss->ground = n_firms - 1;
    kss->M = n_matches;
    const size_t M = static_cast<size_t>(n_matches);
    std::vector<double> inv_dw(static_cast<size_t>(n_workers));
    for (int w = 0; w < n_workers; ++w) inv_dw[w] = 1.0 / Dw[w];
    // matches in firm order
    std::vector<int32_t> mw_f(M);
    std::vector<double> mc_f(M);
    for (size_t a = 0; a < M; ++a) {
        const int64_t m = f_matches[a];
        mw_f[a] = m_w[m];
        mc_f[a] = m_c[m];
    }
    // firm chunks of at most kChunk matches; longer firms get partial slots
    std::vector<int64_t> cbeg;
    std::vector<int32_t> cfirm, cslot, mfirm, mslot0, mnslot;
    int64_t slots = 0;
    for (int f = 0; f < n_firms; ++f) {
        const int64_t b = f_ptr[f], e = f_ptr[f + 1];
        if (e - b <= kChunk) {
            cbeg.push_back(b);
            cfirm.push_back(f);
            cslot.push_back(-1);
            continue;
        }
        const int64_t nc = (e - b + kChunk - 1) / kChunk;
        mfirm.push_back(f);
        mslot0.push_back(static_cast<int32_t>(slots));
        mnslot.push_back(static_cast<int32_t>(nc));
        for (int64_t k = 0; k < nc; ++k) {
            cbeg.push_back(b + k * kChunk);
            cfirm.push_back(f);
            cslot.push_back(static_cast<int32_t>(slots + k));
        }
        slots += nc;
    }
    cbeg.push_back(n_matches);
    kss->nchunks = static_cast<int64_t>(cfirm.size());
    kss->nmulti = static_cast<int64_t>(mfirm.size());
    kss->nslots = slots;
    kss->dot_grid = kss->sms * 2;
    int rc = B200FE_OK;
    if ((rc = upload(kss, &kss->w_ptr, w_ptr, static_cast<size_t>(n_workers) + 1)) ||
        (rc = upload(kss, &kss->m_f, m_f, M)) || (rc = upload(kss, &kss->m_c, m_c, M)) ||
        (rc = upload(kss, &kss->inv_dw, inv_dw.data(), inv_dw.size())) ||
        (rc = upload(kss, &kss->mw_f, mw_f.data(), M)) || (rc = upload(kss, &kss->mc_f, mc_f.data(), M)) ||
        (rc = upload(kss, &kss->cbeg, cbeg.data(), cbeg.size())) ||
        (rc = upload(kss, &kss->cfirm, cfirm.data(), cfirm.size())) ||
        (rc = upload(kss, &kss->cslot, cslot.data(), cslot.size())) ||
        (rc = upload(kss, &kss->mfirm, mfirm.data(), mfirm.size())) ||
        (rc = upload(kss, &kss->mslot0, mslot0.data(), mslot0.size())) ||
        (rc = upload(kss, &kss->mnslot, mnslot.data(), mnslot.size())) ||
        (rc = upload(kss, &kss->Df, Df, static_cast<size_t>(n_firms))) ||
        (rc = upload(kss, &kss->inv_diag, inv_diagS, static_cast<size_t>(n_firms))))
        return fail(rc);
    void* dp = nullptr;
    if (cudaMalloc(&dp, sizeof(double) * kss->dot_grid * 2 * kKssMaxLanes) != cudaSuccess) {
        cudaGetLastError();
        return fail(B200FE_CUDA_ERROR);
    }
    kss->owned.push_back(dp);
    kss->dot_part = static_cast<double*>(dp);
    void* sp = nullptr;
    if (cudaMalloc(&sp, sizeof(KssScalars)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&kss->h_sc), sizeof(KssScalars)) != cudaSuccess) {
        cudaGetLastError();
        if (sp) cudaFree(sp);
        return fail(B200FE_CUDA_ERROR);
    }
    kss->owned.push_back(sp);
    kss->sc = static_cast<KssScalars*>(sp);
    if (cudaMemset(kss->sc, 0, sizeof(KssScalars)) != cudaSuccess) {
        cudaGetLastError();
        return fail(B200FE_CUDA_ERROR);
    }
    *out = kss;
    return B200FE_OK;
}

void b200fe_kss_destroy(b200fe_kss* kss) { delete kss; }

const char* b200fe_kss_last_error(const b200fe_kss* kss) { return kss ? kss->err.c_str() : ""; }

int b200fe_kss_max_lanes(void) { return kKssMaxLanes; }

double* b200fe_kss_pack_buffer(b200fe_kss* kss, int nb) {
    if (!kss || nb < 1 || nb > kKssMaxLanes) return nullptr;
    if (kss->pack_nb >= nb) return kss->h_pack;
    if (cudaSetDevice(kss->device) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (kss->h_pack) cudaFreeHost(kss->h_pack);
    kss->h_pack = nullptr;
    kss->pack_nb = 0;
    if (cudaMallocHost(reinterpret_cast<void**>(&kss->h_pack),
                       sizeof(double) * static_cast<size_t>(kss->J) * nb) != cudaSuccess) {
        cudaGetLastError();
        kss->h_pack = nullptr;
        return nullptr;
    }
    kss->pack_nb = nb;
    return kss->h_pack;
}

int b200fe_kss_solve_multi(b200fe_kss* kss, const double* rhs_pack, double* z_pack, int nb,
                           double tol, int max_iter, int* iters_out) {
    return solve_lanes(kss, rhs_pack, z_pack, nb, tol, max_iter, iters_out);
}

int b200fe_kss_solve(b200fe_kss* kss, const double* rhs, double* z, double tol, int max_iter,
                     int* iterations) {
    int it = -1;
    const int rc = solve_lanes(kss, rhs, z, 1, tol, max_iter, &it);
    if (iterations) *iterations = it;
    if (rc != B200FE_OK) return rc;
    return it >= 0 ? B200FE_OK : B200FE_NOT_CONVERGED;
}

int b200fe_stable_sort_u64(const uint64_t* keys, int64_t* order_out, int64_t n) {
    if (n == 0) return B200FE_OK;
    if (!keys || !order_out || n < 0 || n > INT_MAX) return B200FE_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    uint64_t *kin = nullptr, *kout = nullptr;
    int64_t *vin = nullptr, *vout = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaStream_t s = nullptr;
    const size_t nn = static_cast<size_t>(n);
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&kin, nn * sizeof(uint64_t)) == cudaSuccess &&
              cudaMalloc(&kout, nn * sizeof(uint64_t)) == cudaSuccess &&
              cudaMalloc(&vin, nn * sizeof(int64_t)) == cudaSuccess &&
              cudaMalloc(&vout, nn * sizeof(int64_t)) == cudaSuccess &&
              cudaMemcpyAsync(kin, keys, nn * sizeof(uint64_t), cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (ok) {
        kss_iota_kernel<<<1184, 256, 0, s>>>(vin, n);
        ok = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kin, kout, vin, vout, static_cast<int>(n),
                                             0, 64, s) == cudaSuccess &&
             cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 1)) == cudaSuccess &&
             cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kin, kout, vin, vout, static_cast<int>(n), 0, 64,
                                             s) == cudaSuccess &&
             cudaMemcpyAsync(order_out, vout, nn * sizeof(int64_t), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaStreamSynchronize(s) == cudaSuccess;
    }
    cudaGetLastError();
    cudaFree(tmp);
    cudaFree(vout);
    cudaFree(vin);
    cudaFree(kout);
    cudaFree(kin);
    if (s) cudaStreamDestroy(s);
    return ok ? B200FE_OK : B200FE_CUDA_ERROR;
}

}  // extern "C"
