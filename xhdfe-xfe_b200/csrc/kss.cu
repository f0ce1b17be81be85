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

// ---------------------------------------------------------------------------
// JLA leverages (b200fe_kss_jla).  Per draw d the reference's driver
// (src/akm_kss.cpp:2753-3160) draws one Rademacher sign per working row from
// the SplitMix64 stream (seed, 3d, row block of 64), scatters sqrt(c_r) g_r
// into worker and firm right-hand sides (tw1, tf1), draws per match the sum
// of cnt_m signs from the stream (seed, 3d + 1, m) and scatters its centred
// value su_m into (tw2, tf2), and solves K z = (tw1, tf1), (0, tf2) and
// (tw2, 0).  Per row it then accumulates, in ascending draw order,
//     Z = sqrt(c_r)(zw[w] + zf[f]), diff = g - Z:
//     Pacc += Z^2/p, Psq += Z^4/p, Macc += diff^2/p, Msq += diff^4/p,
//     PM += Z^2 diff^2/p, and Bfe += W2^2, Bpe += W1^2, Bcov += W1 W2
// with W2, W1 the same products of the (0, tf2) and (tw2, 0) solutions.  Here
// all of it runs on the device, a block of draws (three lanes each) per
// batched solve; the streams are the reference's bit for bit.
// ---------------------------------------------------------------------------

// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), the generator the reference's streams use.
__device__ __forceinline__ uint64_t jla_mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
// The reference's stream of (draw tag, unit): src/akm_kss.cpp:218-222.
__device__ __forceinline__ uint64_t jla_stream(uint64_t seed, uint64_t tag, uint64_t unit) {
    const uint64_t s = jla_mix(seed ^ (0xA24BAED4963EE407ULL * (tag + 1)));
    return jla_mix(s ^ (0x9FB21C651E98DF25ULL * (unit + 1)));
}
__device__ __forceinline__ double jla_sign(const uint64_t* words, int64_t r) {
    return ((words[r >> 6] >> (r & 63)) & 1ULL) ? 1.0 : -1.0;
}

// words[b][blk]: the sign words of draw d0 + b
__global__ void jla_bits_kernel(uint64_t seed, int d0, int B, int64_t nblk, uint64_t* __restrict__ words) {
    const int64_t total = static_cast<int64_t>(B) * nblk;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(e / nblk);
        const int64_t blk = e - static_cast<int64_t>(b) * nblk;
        words[e] = jla_stream(seed, 3ULL * static_cast<uint64_t>(d0 + b), static_cast<uint64_t>(blk));
    }
}

// su[b][m] = sum of cnt_m signs of the stream (seed, 3d + 1, m), 64 per state
// advance (src/akm_kss.cpp:224-238); tot[b] += that sum (integers: exact in
// any order)
__global__ void jla_msum_kernel(uint64_t seed, int d0, int B, int64_t M, const int64_t* __restrict__ cnt,
                                double* __restrict__ su, unsigned long long* __restrict__ tot) {
    const int64_t total = static_cast<int64_t>(B) * M;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(e / M);
        const int64_t m = e - static_cast<int64_t>(b) * M;
        uint64_t st = jla_stream(seed, 3ULL * static_cast<uint64_t>(d0 + b) + 1ULL, static_cast<uint64_t>(m));
        long long acc = 0;
        for (long long rem = cnt[m]; rem > 0;) {
            st = jla_mix(st);
            const int k = rem >= 64 ? 64 : static_cast<int>(rem);
            const uint64_t bits = k == 64 ? st : (st & ((1ULL << k) - 1ULL));
            acc += 2LL * __popcll(bits) - k;
            rem -= k;
        }
        su[e] = static_cast<double>(acc);
        atomicAdd(tot + b, static_cast<unsigned long long>(acc));
    }
}

// su[b][m] = msum * scale - vbar_b cnt_m, vbar_b = (tot_b / n_py) scale
__global__ void jla_su_kernel(int B, int64_t M, const int64_t* __restrict__ cnt,
                              const unsigned long long* __restrict__ tot, double n_py, double scale,
                              double* __restrict__ su) {
    const int64_t total = static_cast<int64_t>(B) * M;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(e / M);
        const int64_t m = e - static_cast<int64_t>(b) * M;
        const double vbar = (static_cast<double>(static_cast<long long>(tot[b])) / n_py) * scale;
        su[e] = su[e] * scale - vbar * static_cast<double>(cnt[m]);
    }
}

// xw[w][l] = tw[w][l] / Dw[w]: lanes [0,B) the rows' signed weights, [B,2B)
// zero, [2B,3B) su of the worker's matches; padding lanes zero
__global__ void jla_tw_kernel(int N, int LW, int B, const int64_t* __restrict__ rw_ptr,
                              const int32_t* __restrict__ rw_rows, const double* __restrict__ row_sw,
                              const uint64_t* __restrict__ words, int64_t nblk, const int64_t* __restrict__ w_ptr,
                              const double* __restrict__ su, int64_t M, const double* __restrict__ Dw,
                              double* __restrict__ xw) {
    const int64_t total = static_cast<int64_t>(N) * LW;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t w = e / LW;
        const int l = static_cast<int>(e - w * LW);
        double acc = 0.0;
        if (l < B) {
            const uint64_t* wd = words + static_cast<int64_t>(l) * nblk;
            for (int64_t a = rw_ptr[w]; a < rw_ptr[w + 1]; ++a) {
                const int64_t r = rw_rows[a];
                acc += (row_sw ? row_sw[r] : 1.0) * jla_sign(wd, r);
            }
        } else if (l >= 2 * B && l < 3 * B) {
            const double* sb = su + static_cast<int64_t>(l - 2 * B) * M;
            for (int64_t a = w_ptr[w]; a < w_ptr[w + 1]; ++a) acc += sb[a];
        }
        xw[e] = acc / Dw[w];
    }
}

// Firm-side scatters cut into chunks of at most kJlaChunk entries (a firm
// with a large share of the rows is summed by many threads), the chunk
// partials then added per firm in chunk order.
constexpr int kJlaChunk = 256;

__global__ void jla_chunk_count_kernel(int nseg, const int64_t* __restrict__ ptr, int32_t* __restrict__ count) {
    for (int64_t sg = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; sg <= nseg;
         sg += static_cast<int64_t>(gridDim.x) * blockDim.x)
        count[sg] = sg < nseg ? static_cast<int32_t>((ptr[sg + 1] - ptr[sg] + kJlaChunk - 1) / kJlaChunk) : 0;
}

__global__ void jla_chunk_fill_kernel(int nseg, const int64_t* __restrict__ ptr, const int32_t* __restrict__ first,
                                      int64_t* __restrict__ cbeg) {
    for (int64_t sg = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; sg < nseg;
         sg += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t k0 = first[sg], k1 = first[sg + 1];
        for (int32_t k = k0; k < k1; ++k) cbeg[k] = ptr[sg] + static_cast<int64_t>(k - k0) * kJlaChunk;
    }
}

// part[k][l], l in [0, B): the signed row weights of chunk k (rows: idx),
// or (su != null) the sums su[l][idx[a]] of chunk k
__global__ void jla_chunk_sum_kernel(int64_t nchunks, int LW, int B, const int64_t* __restrict__ cbeg,
                                     const int32_t* __restrict__ first, int nseg,
                                     const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx32,
                                     const int64_t* __restrict__ idx64, const double* __restrict__ row_sw,
                                     const uint64_t* __restrict__ words, int64_t nblk, const double* __restrict__ su,
                                     int64_t M, double* __restrict__ part) {
    const int64_t total = nchunks * B;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = e / B;
        const int l = static_cast<int>(e - k * B);
        // end of the chunk: the next chunk's start, or the end of its segment
        int lo = 0, hi = nseg;  // segment of chunk k: last sg with first[sg] <= k
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (first[mid] <= k) lo = mid;
            else hi = mid;
        }
        const int64_t a0 = cbeg[k];
        const int64_t a1 = min(a0 + kJlaChunk, ptr[lo + 1]);
        double acc = 0.0;
        if (su) {
            const double* sb = su + static_cast<int64_t>(l) * M;
            for (int64_t a = a0; a < a1; ++a) acc += sb[idx64[a]];
        } else {
            const uint64_t* wd = words + static_cast<int64_t>(l) * nblk;
            for (int64_t a = a0; a < a1; ++a) {
                const int64_t r = idx32[a];
                acc += (row_sw ? row_sw[r] : 1.0) * jla_sign(wd, r);
            }
        }
        part[k * LW + l] = acc;
    }
}

// out[sg][l0 + l] = sum of the chunk partials of segment sg, in chunk order
__global__ void jla_chunk_combine_kernel(int nseg, int LW, int B, int l0, const int32_t* __restrict__ first,
                                         const double* __restrict__ part, double* __restrict__ out) {
    const int64_t total = static_cast<int64_t>(nseg) * B;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t sg = e / B;
        const int l = static_cast<int>(e - sg * B);
        double acc = 0.0;
        for (int32_t k = first[sg]; k < first[sg + 1]; ++k) acc += part[static_cast<int64_t>(k) * LW + l];
        out[sg * LW + l0 + l] = acc;
    }
}

// lane-major stage [nl][J] = tf - B' xw (Ap holds -B' xw; ground entries zero)
__global__ void jla_rhs_kernel(int64_t J, int LW, int nl, int ground, const double* __restrict__ tf,
                               const double* __restrict__ Ap, double* __restrict__ stage) {
    const int64_t total = J * nl;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int l = static_cast<int>(e / J);
        const int64_t f = e - static_cast<int64_t>(l) * J;
        stage[e] = f == ground ? 0.0 : tf[f * LW + l] + Ap[f * LW + l];
    }
}

__global__ void jla_sub_kernel(int64_t total, const double* __restrict__ t, double* __restrict__ xw) {
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        xw[e] -= t[e];
}

// per row, ascending draw: the eight sums acc[k][r]
__global__ void jla_accum_kernel(int64_t R, int LW, int B, const int32_t* __restrict__ row_w,
                                 const int32_t* __restrict__ row_f, const double* __restrict__ row_sw,
                                 const uint64_t* __restrict__ words, int64_t nblk, const double* __restrict__ zw,
                                 const double* __restrict__ zf, double pd, double* __restrict__ acc) {
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t w = row_w[r], f = row_f[r];
        const double sw = row_sw ? row_sw[r] : 1.0;
        double pa = acc[r], ps = acc[R + r], ma = acc[2 * R + r], ms = acc[3 * R + r], pm = acc[4 * R + r];
        double bfe = acc[5 * R + r], bpe = acc[6 * R + r], bcov = acc[7 * R + r];
        for (int b = 0; b < B; ++b) {
            const double Z = sw * (zw[w * LW + b] + zf[f * LW + b]);
            const double g = jla_sign(words + static_cast<int64_t>(b) * nblk, r);
            const double diff = g - Z;
            const double z2 = Z * Z;
            const double m2 = diff * diff;
            pa += z2 / pd;
            ps += z2 * z2 / pd;
            ma += m2 / pd;
            ms += m2 * m2 / pd;
            pm += z2 * m2 / pd;
        }
        for (int b = 0; b < B; ++b) {
            const double W2 = sw * (zw[w * LW + B + b] + zf[f * LW + B + b]);
            const double W1 = sw * (zw[w * LW + 2 * B + b] + zf[f * LW + 2 * B + b]);
            bfe += W2 * W2;
            bpe += W1 * W1;
            bcov += W1 * W2;
        }
        acc[r] = pa;
        acc[R + r] = ps;
        acc[2 * R + r] = ma;
        acc[3 * R + r] = ms;
        acc[4 * R + r] = pm;
        acc[5 * R + r] = bfe;
        acc[6 * R + r] = bpe;
        acc[7 * R + r] = bcov;
    }
}

// ratio estimator and nonlinearity correction (src/akm_kss.cpp:3275-3289)
__global__ void jla_final_kernel(int64_t R, double pd, const double* __restrict__ acc, double* __restrict__ out) {
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double Pa = acc[r], Ps = acc[R + r], Ma = acc[2 * R + r], Ms = acc[3 * R + r], PM = acc[4 * R + r];
        const double denom = Pa + Ma;
        const double Ph = denom > 0.0 ? Pa / denom : 0.0;
        const double Mh = 1.0 - Ph;
        double corr = 0.0;
        if (Mh > 0.0) {
            const double Vi = (Mh * Mh * Ps + Ph * Ph * Ms - 2.0 * Mh * Ph * PM) / pd;
            const double Bi = (Mh * Ps - Ph * Ms + 2.0 * (Mh - Ph) * PM) / pd;
            corr = 1.0 - Vi / (Mh * Mh) + Bi / Mh;
        }
        out[r] = Ph;
        out[R + r] = Mh;
        out[2 * R + r] = corr;
    }
}

// CSR offsets of sorted keys: ptr[k] = first position with key >= k
__global__ void jla_ptr_kernel(int64_t R, int nkeys, const int32_t* __restrict__ keys, int64_t* __restrict__ ptr) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= R;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int kp = i == 0 ? -1 : keys[i - 1];
        const int kc = i == R ? nkeys : keys[i];
        for (int k = kp + 1; k <= kc && k <= nkeys; ++k) ptr[k] = i;
    }
}

__global__ void jla_iota_kernel(int32_t* out, int64_t n) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<int32_t>(i);
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
    double* Dw = nullptr;
    int64_t* f_ptr = nullptr;      // firm CSR over f_matches
    int64_t* f_matches = nullptr;  // match ids in firm order (ascending within a firm)
    KssScalars* sc_one = nullptr;  // nactive = 1: the matrix kernels outside a solve (JLA)
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

// Device buffers of one b200fe_kss_jla call, freed on every return.
struct JlaBufs {
    std::vector<void*> ptrs;
    ~JlaBufs() {
        for (void* q : ptrs) cudaFree(q);
    }
    template <typename T>
    cudaError_t get(T** out, size_t count) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1));
        if (e == cudaSuccess) ptrs.push_back(q);
        *out = static_cast<T*>(q);
        return e;
    }
};

struct JlaState {
    int64_t R = 0, M = 0, nblk = 0;
    const int32_t *row_w = nullptr, *row_f = nullptr;
    const double* row_sw = nullptr;
    const int64_t* cnt = nullptr;
    const int64_t *rw_ptr = nullptr, *rf_ptr = nullptr;
    const int32_t *rw_rows = nullptr, *rf_rows = nullptr;
    uint64_t* words = nullptr;
    double* su = nullptr;
    unsigned long long* tot = nullptr;
    double* xw = nullptr;  // tw / Dw, then zw
    double* tf = nullptr;
    double* acc = nullptr;  // [8][R]
    // firm chunks of the rows (r*) and of the matches (m*); part: their partials
    int32_t *rfirst = nullptr, *mfirst = nullptr;
    int64_t *rcbeg = nullptr, *mcbeg = nullptr;
    int64_t nrch = 0, nmch = 0;
    double* part = nullptr;
    uint64_t seed = 0;
    double n_py = 0.0, pd = 1.0, scale = 1.0;
    double tol = 1e-10;
    int max_iter = 1000;
    long long iters = 0;
    int failed = 0;
};

// draws [d0, d0 + B): the scatters, 3B batched solves and the row sums
template <int LW>
int jla_block(b200fe_kss* kss, JlaState& js, int d0, int B) {
    const cudaStream_t s = kss->stream;
    const int nl = 3 * B;
    const int64_t N = kss->N, J = kss->J;
    const int T = 256;
    auto grid = [&](int64_t work) { return grid_for(kss, work, 8); };
    jla_bits_kernel<<<grid(B * js.nblk), T, 0, s>>>(js.seed, d0, B, js.nblk, js.words);
    K_TRY(cudaMemsetAsync(js.tot, 0, sizeof(unsigned long long) * B, s));
    jla_msum_kernel<<<grid(B * js.M), T, 0, s>>>(js.seed, d0, B, js.M, js.cnt, js.su, js.tot);
    jla_su_kernel<<<grid(B * js.M), T, 0, s>>>(B, js.M, js.cnt, js.tot, js.n_py, js.scale, js.su);
    jla_tw_kernel<<<grid(N * LW), T, 0, s>>>(static_cast<int>(N), LW, B, js.rw_ptr, js.rw_rows, js.row_sw,
                                            js.words, js.nblk, kss->w_ptr, js.su, js.M, kss->Dw, js.xw);
    K_TRY(cudaMemsetAsync(js.tf, 0, sizeof(double) * J * LW, s));
    jla_chunk_sum_kernel<<<grid(js.nrch * B), T, 0, s>>>(js.nrch, LW, B, js.rcbeg, js.rfirst, static_cast<int>(J),
                                                         js.rf_ptr, js.rf_rows, nullptr, js.row_sw, js.words, js.nblk,
                                                         nullptr, js.M, js.part);
    jla_chunk_combine_kernel<<<grid(J * B), T, 0, s>>>(static_cast<int>(J), LW, B, 0, js.rfirst, js.part, js.tf);
    jla_chunk_sum_kernel<<<grid(js.nmch * B), T, 0, s>>>(js.nmch, LW, B, js.mcbeg, js.mfirst, static_cast<int>(J),
                                                         kss->f_ptr, nullptr, kss->f_matches, nullptr, js.words,
                                                         js.nblk, js.su, js.M, js.part);
    jla_chunk_combine_kernel<<<grid(J * B), T, 0, s>>>(static_cast<int>(J), LW, B, B, js.mfirst, js.part, js.tf);
    K_TRY(cudaGetLastError());
    // Ap = -B' xw (the firm pass at p = 0), then the lane-major right-hand sides
    constexpr int TG = LaneGeom<LW>::TG;
    K_TRY(cudaMemsetAsync(kss->z, 0, sizeof(double) * J * LW, s));
    kss_firm_kernel<LW><<<grid_for(kss, kss->nchunks * TG, 8), kKssThreads, 0, s>>>(
        kss->nchunks, kss->cbeg, kss->cfirm, kss->cslot, kss->mw_f, kss->mc_f, js.xw, kss->Df, kss->z, kss->Ap,
        kss->slot_part, kss->ground, kss->sc_one);
    if (kss->nmulti > 0)
        kss_firm_combine_kernel<LW><<<grid_for(kss, kss->nmulti * TG, 8), kKssThreads, 0, s>>>(
            kss->nmulti, kss->mfirm, kss->mslot0, kss->mnslot, kss->slot_part, kss->Df, kss->z, kss->Ap,
            kss->ground, kss->sc_one);
    jla_rhs_kernel<<<grid(J * nl), T, 0, s>>>(J, LW, nl, kss->ground, js.tf, kss->Ap, kss->stage);
    K_TRY(cudaGetLastError());
    // S zf = rhs for the 3B lanes
    KssScalars init;
    std::memset(&init, 0, sizeof(init));
    init.nb = nl;
    init.tol = js.tol;
    init.max_iter = js.max_iter;
    init.nactive = 1;
    *kss->h_sc = init;
    K_TRY(cudaMemcpyAsync(kss->sc, kss->h_sc, sizeof(KssScalars), cudaMemcpyHostToDevice, s));
    K_CHECK(run_solve<LW>(kss, nl));
    K_TRY(cudaMemcpyAsync(kss->h_sc, kss->sc, sizeof(KssScalars), cudaMemcpyDeviceToHost, s));
    // zf interleaved (failed lanes zero), zw = xw - Dw^-1 B zf
    kss_pack_in_kernel<<<grid(J * LW), T, 0, s>>>(J, LW, nl, kss->ground, kss->stage, kss->p);
    kss_worker_kernel<LW><<<grid_for(kss, N * TG, 8), kKssThreads, 0, s>>>(
        static_cast<int>(N), kss->w_ptr, kss->m_f, kss->m_c, kss->inv_dw, kss->p, kss->t, kss->sc_one);
    jla_sub_kernel<<<grid(N * LW), T, 0, s>>>(N * LW, kss->t, js.xw);
    jla_accum_kernel<<<grid(js.R), T, 0, s>>>(js.R, LW, B, js.row_w, js.row_f, js.row_sw, js.words, js.nblk,
                                             js.xw, kss->p, js.pd, js.acc);
    K_TRY(cudaGetLastError());
    K_TRY(cudaStreamSynchronize(s));
    for (int l = 0; l < nl; ++l) {
        if (kss->h_sc->ok[l]) js.iters += kss->h_sc->its[l];
        else ++js.failed;
    }
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
        (rc = upload(kss, &kss->Dw, Dw, static_cast<size_t>(n_workers))) ||
        (rc = upload(kss, &kss->f_ptr, f_ptr, static_cast<size_t>(n_firms) + 1)) ||
        (rc = upload(kss, &kss->f_matches, f_matches, M)) ||
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

int b200fe_kss_jla(b200fe_kss* kss, int64_t n_rows, const int32_t* row_w, const int32_t* row_f,
                   const double* row_sw, const int64_t* m_cnt, double n_py, uint64_t seed, int draws,
                   int block, double tol, int max_iter, double* pii, double* mii, double* corr,
                   double* bfe, double* bpe, double* bcov, int* failed_lanes, long long* iterations) {
    if (!kss || n_rows < 1 || n_rows >= INT_MAX || !row_w || !row_f || !m_cnt || draws < 1 || block < 0 ||
        !(tol >= 0.0) || max_iter < 1 || !(n_py > 0.0))
        return B200FE_INVALID_ARG;
    for (int64_t r = 0; r < n_rows; ++r)
        if (row_w[r] < 0 || row_w[r] >= kss->N || row_f[r] < 0 || row_f[r] >= kss->J) return B200FE_INVALID_ARG;
    for (int64_t m = 0; m < kss->M; ++m)
        if (m_cnt[m] < 0) return B200FE_INVALID_ARG;
    K_TRY(cudaSetDevice(kss->device));
    const cudaStream_t s = kss->stream;
    // draws per batched solve: three lanes each, at most kKssMaxLanes lanes
    const int B = std::max(1, std::min(block > 0 ? block : 8, kKssMaxLanes / 3));
    const int lw = lane_pitch(3 * B);
    K_CHECK(ensure_lanes(kss, lw));
    if (!kss->sc_one) {
        void* q = nullptr;
        K_TRY(cudaMalloc(&q, sizeof(KssScalars)));
        kss->owned.push_back(q);
        kss->sc_one = static_cast<KssScalars*>(q);
        KssScalars one;
        std::memset(&one, 0, sizeof(one));
        one.nactive = 1;
        K_TRY(cudaMemcpy(kss->sc_one, &one, sizeof(one), cudaMemcpyHostToDevice));
    }
    JlaBufs bufs;
    JlaState js;
    js.R = n_rows;
    js.M = kss->M;
    js.nblk = (n_rows + 63) / 64;
    js.seed = seed;
    js.n_py = n_py;
    js.pd = static_cast<double>(draws);
    js.scale = 1.0 / std::sqrt(js.pd);
    js.tol = tol;
    js.max_iter = max_iter;
    const size_t R = static_cast<size_t>(n_rows);
    int32_t *d_rw, *d_rf, *keys_sorted, *iota, *rw_rows, *rf_rows;
    double* d_sw = nullptr;
    int64_t *d_cnt, *rw_ptr, *rf_ptr;
    K_TRY(bufs.get(&d_rw, R));
    K_TRY(bufs.get(&d_rf, R));
    K_TRY(bufs.get(&keys_sorted, R));
    K_TRY(bufs.get(&iota, R));
    K_TRY(bufs.get(&rw_rows, R));
    K_TRY(bufs.get(&rf_rows, R));
    K_TRY(bufs.get(&d_cnt, static_cast<size_t>(kss->M)));
    K_TRY(bufs.get(&rw_ptr, static_cast<size_t>(kss->N) + 1));
    K_TRY(bufs.get(&rf_ptr, static_cast<size_t>(kss->J) + 1));
    K_TRY(cudaMemcpyAsync(d_rw, row_w, sizeof(int32_t) * R, cudaMemcpyHostToDevice, s));
    K_TRY(cudaMemcpyAsync(d_rf, row_f, sizeof(int32_t) * R, cudaMemcpyHostToDevice, s));
    K_TRY(cudaMemcpyAsync(d_cnt, m_cnt, sizeof(int64_t) * kss->M, cudaMemcpyHostToDevice, s));
    if (row_sw) {
        K_TRY(bufs.get(&d_sw, R));
        K_TRY(cudaMemcpyAsync(d_sw, row_sw, sizeof(double) * R, cudaMemcpyHostToDevice, s));
    }
    // rows grouped by worker and by firm, ascending row order within a group
    // (a stable sort), so every scatter adds in the reference's order
    jla_iota_kernel<<<grid_for(kss, n_rows, 8), 256, 0, s>>>(iota, n_rows);
    size_t tmp_bytes = 0;
    void* tmp = nullptr;
    K_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_rw, keys_sorted, iota, rw_rows,
                                          static_cast<int>(n_rows), 0, 32, s));
    K_TRY(bufs.get(reinterpret_cast<unsigned char**>(&tmp), tmp_bytes));
    K_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, d_rw, keys_sorted, iota, rw_rows,
                                          static_cast<int>(n_rows), 0, 32, s));
    jla_ptr_kernel<<<grid_for(kss, n_rows + 1, 8), 256, 0, s>>>(n_rows, kss->N, keys_sorted, rw_ptr);
    K_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, d_rf, keys_sorted, iota, rf_rows,
                                          static_cast<int>(n_rows), 0, 32, s));
    jla_ptr_kernel<<<grid_for(kss, n_rows + 1, 8), 256, 0, s>>>(n_rows, kss->J, keys_sorted, rf_ptr);
    K_TRY(cudaGetLastError());
    // firm chunks of the rows and of the matches
    auto chunks = [&](const int64_t* ptr, int32_t** first, int64_t** cbeg, int64_t* nch) -> int {
        int32_t* cnt;
        K_TRY(bufs.get(&cnt, static_cast<size_t>(kss->J) + 1));
        K_TRY(bufs.get(first, static_cast<size_t>(kss->J) + 1));
        jla_chunk_count_kernel<<<grid_for(kss, kss->J + 1, 8), 256, 0, s>>>(kss->J, ptr, cnt);
        size_t sb = 0;
        K_TRY(cub::DeviceScan::ExclusiveSum(nullptr, sb, cnt, *first, kss->J + 1, s));
        unsigned char* st;
        K_TRY(bufs.get(&st, sb));
        K_TRY(cub::DeviceScan::ExclusiveSum(st, sb, cnt, *first, kss->J + 1, s));
        int32_t tot = 0;
        K_TRY(cudaMemcpyAsync(&tot, *first + kss->J, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        K_TRY(cudaStreamSynchronize(s));
        *nch = tot;
        K_TRY(bufs.get(cbeg, static_cast<size_t>(std::max(tot, 1))));
        jla_chunk_fill_kernel<<<grid_for(kss, kss->J, 8), 256, 0, s>>>(kss->J, ptr, *first, *cbeg);
        K_TRY(cudaGetLastError());
        return B200FE_OK;
    };
    K_CHECK(chunks(rf_ptr, &js.rfirst, &js.rcbeg, &js.nrch));
    K_CHECK(chunks(kss->f_ptr, &js.mfirst, &js.mcbeg, &js.nmch));
    K_TRY(bufs.get(&js.part, static_cast<size_t>(std::max<int64_t>(std::max(js.nrch, js.nmch), 1)) * lw));
    js.row_w = d_rw;
    js.row_f = d_rf;
    js.row_sw = d_sw;
    js.cnt = d_cnt;
    js.rw_ptr = rw_ptr;
    js.rf_ptr = rf_ptr;
    js.rw_rows = rw_rows;
    js.rf_rows = rf_rows;
    K_TRY(bufs.get(&js.words, static_cast<size_t>(B) * js.nblk));
    K_TRY(bufs.get(&js.su, static_cast<size_t>(B) * std::max<int64_t>(kss->M, 1)));
    K_TRY(bufs.get(&js.tot, static_cast<size_t>(B)));
    K_TRY(bufs.get(&js.xw, static_cast<size_t>(std::max(kss->N, 1)) * lw));
    K_TRY(bufs.get(&js.tf, static_cast<size_t>(kss->J) * lw));
    K_TRY(bufs.get(&js.acc, 8 * R));
    K_TRY(cudaMemsetAsync(js.acc, 0, sizeof(double) * 8 * R, s));
    for (int d0 = 0; d0 < draws; d0 += B) {
        const int nb = std::min(B, draws - d0);
        int rc = B200FE_OK;
        switch (lw) {
            case 4: rc = jla_block<4>(kss, js, d0, nb); break;
            case 8: rc = jla_block<8>(kss, js, d0, nb); break;
            case 16: rc = jla_block<16>(kss, js, d0, nb); break;
            case 32: rc = jla_block<32>(kss, js, d0, nb); break;
            default: rc = jla_block<64>(kss, js, d0, nb); break;
        }
        if (rc != B200FE_OK) return rc;
    }
    double* fin;
    K_TRY(bufs.get(&fin, 3 * R));
    jla_final_kernel<<<grid_for(kss, n_rows, 8), 256, 0, s>>>(n_rows, js.pd, js.acc, fin);
    K_TRY(cudaGetLastError());
    double* const outs[6] = {pii, mii, corr, bfe, bpe, bcov};
    const double* const srcs[6] = {fin, fin + R, fin + 2 * R, js.acc + 5 * R, js.acc + 6 * R, js.acc + 7 * R};
    for (int k = 0; k < 6; ++k)
        if (outs[k]) K_TRY(cudaMemcpyAsync(outs[k], srcs[k], sizeof(double) * R, cudaMemcpyDeviceToHost, s));
    K_TRY(cudaStreamSynchronize(s));
    if (failed_lanes) *failed_lanes = js.failed;
    if (iterations) *iterations = js.iters;
    return js.failed == 0 ? B200FE_OK : B200FE_NOT_CONVERGED;
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
