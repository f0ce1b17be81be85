// FP64 data passes (kRhs, kFinal) fed by bulk asynchronous copies.
//
// One CTA per SM: a producer warp streams the regular tiles of this CTA
// (whole primary segments, at most kTileObs observations) into a ring of
// shared-memory stages with cp.async.bulk, each stage completing on its own
// mbarrier; kStreamWarps consumer warps work on the landed tiles.  A stage
// holds the tile's data columns and its record (tile_blob_kernel: work
// splits, segment and run offsets, run destinations, inverse segment
// weights, the order of its observations by small-dim level), plus in kFinal
// the ids the gather of D_r a needs and, when weighted, the weights.  A tile
// takes one copy per column, one for its record and one per id array; the
// producer lane of each copy computes its 16-byte-aligned span, and the
// consumers read each array from the offset of its first element in it.
// kFinal writes the within transform back in place in the stage; the
// producer stores the 16-byte-aligned interior of every output column with
// cp.async.bulk and the consumers store the at most two elements at its ends.
//
// Per tile, every consumer warp
//   1. takes the segments the record assigns to it (the ones starting in its
//      kStreamWarps-th of the tile's observations); lane c % 16 is data
//      column c, the warp's two halves take the even and odd observations of
//      every segment and run, and their sums meet in one shuffle: segment
//      means, z = w (v - mean) (kRhs) or d = v - D_r a - mean (kFinal) back
//      into the stage, the run sums R of every large dim, the column sums of
//      squares;
//   2. one tile later (after all warps are through step 1 of that tile, a
//      per-stage mbarrier that has normally completed by then), sums z over
//      the buckets of equal small-dim level (half-warp group g takes levels
//      g, g + 32, ...), each bucket a run of the tile's sorted order, into
//      the CTA's bins, so no two groups ever add to the same bin.
// Every reduction has a fixed order, so results do not depend on timing.
// Outputs are those of data_pass_kernel (kernels.cuh) in the same modes.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace b200fe {

#ifndef B200FE_STREAM_WARPS
#define B200FE_STREAM_WARPS 16
#endif
constexpr int kStreamWarps = B200FE_STREAM_WARPS;        // consumer warps per CTA
constexpr int kStreamThreads = (kStreamWarps + 1) * 32;  // + the producer warp
constexpr int kStreamMaxStages = 4;
constexpr int kStreamPitchD = kTileObs + 2;   // doubles per staged column (span of <= kTileObs - 1 obs)
constexpr int kStreamPitchI = kTileObs + 8;   // 4-byte words per staged int array
constexpr int kStreamHeader = 64;             // tile record at the start of every stage
constexpr int kStreamGather = 8;              // observations per half-warp and batch of the kFinal gather
constexpr int kStreamRunRows = 8;             // rows of dim 0 a consumer warp holds (kFinal, one large dim)
constexpr long long kStreamWaitCycles = 4000000000LL;  // bound of every mbarrier wait
static_assert(kStreamPitchD % 2 == 0 && kStreamPitchI % 4 == 0, "16-byte rows");

__host__ __device__ constexpr int round16(int b) { return (b + 15) & ~15; }

// Work splits and small-dim buckets, the first section of a tile record, in
// 16-bit words:
//   [0, W]                  first segment of consumer warp w (W = kStreamWarps)
//   [(1 + l)(W + 1), ...]   first run of dim l of consumer warp w
//   then per small dim s:   bucket offsets [sG[s] + 1] into the sorted order
__host__ __device__ constexpr int stream_aux_words(int nL, int SG, int nS) {
    return (1 + nL) * (kStreamWarps + 1) + SG + nS;
}
__host__ __device__ constexpr int stream_aux_stride(int nL, int SG, int nS) {
    return (stream_aux_words(nL, SG, nS) + 7) & ~7;  // 16 bytes
}

// Byte offsets of the sections of a tile record (each 16-byte aligned).
struct BlobLayout {
    int seg;                 // u16 [ns + 1] segment offsets from the tile's first observation
    int runs[kMaxLarge];     // u16 [nr + 1] run offsets of dim l
    int ord[kMaxSmall];      // u16 [nk] observations sorted by the level of small dim s
    int rd[kMaxLarge];       // i32 [nr] row of every run of dim l in R
    int rg;                  // i32 [nr] level of dim 0 of every run of dim 0
    int invw;                // f64 [ns] inverse segment weights
    int bytes;
};
__host__ __device__ inline BlobLayout blob_layout(int aux_stride, int nk, int ns, int nL, int nr0, int nr1,
                                                  int nS) {
    BlobLayout b{};
    int off = aux_stride * 2;
    b.seg = off;
    off += round16((ns + 1) * 2);
#pragma unroll
    for (int l = 0; l < kMaxLarge; ++l) {
        if (l < nL) {
            b.runs[l] = off;
            off += round16(((l == 0 ? nr0 : nr1) + 1) * 2);
        }
    }
#pragma unroll
    for (int s = 0; s < kMaxSmall; ++s) {
        if (s < nS) {
            b.ord[s] = off;
            off += round16(nk * 2);
        }
    }
#pragma unroll
    for (int l = 0; l < kMaxLarge; ++l) {
        if (l < nL) {
            b.rd[l] = off;
            off += round16((l == 0 ? nr0 : nr1) * 4);
        }
    }
    b.rg = off;
    if (nL > 0) off += round16(nr0 * 4);
    b.invw = off;
    off += round16(ns * 8);
    b.bytes = off;
    return b;
}

// Byte offsets of the staged arrays inside a stage (host-computed).
struct StreamLayout {
    const int4* tmeta;      // [nreg][2]: {k0, nk, s0, ns}, {rb0, nr0, rb1, nr1}
    const int32_t* boff;    // [nreg + 1] record offsets (16-byte units)
    const unsigned char* blob;
    int aux_stride;         // 16-bit words
    int64_t nreg;           // regular tiles
    int NS;                 // stages
    int stage_bytes;
    int off_cols, off_blob, off_wp, off_sid;
    int off_rid[kMaxLarge];
    int off_yt;             // kFinal: small-dim rows of a [SG][16]
    int off_afb;            // kFinal, one large dim: rows of dim 0 [kStreamWarps][kStreamRunRows][16]
    int off_stages;         // first stage from the start of shared memory
    int off_bins;           // bins [SG][16]
    int off_red;            // column-sum reduction [kStreamWarps][16]
    int* status;            // set to 1 when a wait ran out
};

// ---- PTX wrappers ----------------------------------------------------------
__device__ __forceinline__ uint32_t sm_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(sm_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            sm_addr(dst)),
        "l"(src), "r"(bytes), "r"(sm_addr(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(sm_addr(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on phase `parity` of `bar`; gives up when another warp has
// given up (abort) or after kStreamWaitCycles, then sets abort and status.
__device__ __forceinline__ bool stream_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                            int* status) {
    if (mbar_test(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > kStreamWaitCycles) {
            *abort_flag = 1;
            atomicExch(status, 1);
            return false;
        }
    }
    return true;
}
// The same for a whole warp: lane 0 waits, the outcome is broadcast.
__device__ __forceinline__ bool stream_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                                 int* status) {
    int got = 1;
    if ((threadIdx.x & 31) == 0) got = stream_wait(bar, parity, abort_flag, status);
    return __shfl_sync(0xffffffffu, got, 0) != 0;
}

// Element offset of element i0 of `base` inside its 16-byte-aligned span.
template <int E>
__device__ __forceinline__ int span_phase(const void* base, int64_t i0) {
    return static_cast<int>(((reinterpret_cast<uintptr_t>(base) + static_cast<uintptr_t>(i0) * E) & 15u) / E);
}
// The 16-byte-aligned span covering elements [i0, i0 + cnt) of `base`.
template <int E>
__device__ __forceinline__ void span_of(const void* base, int64_t i0, int64_t cnt, const unsigned char** src,
                                        uint32_t* bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(base) + static_cast<uintptr_t>(i0) * E;
    const uintptr_t a0 = a & ~static_cast<uintptr_t>(15);
    const uintptr_t a1 = (a + static_cast<uintptr_t>(cnt) * E + 15) & ~static_cast<uintptr_t>(15);
    *src = reinterpret_cast<const unsigned char*>(a0);
    *bytes = cnt > 0 ? static_cast<uint32_t>(a1 - a0) : 0u;
}

template <int MODE, bool WEIGHTED>
__global__ void __launch_bounds__(kStreamThreads, 1)
stream_pass_kernel(const PassArgs<double> a, const StreamLayout L) {
    constexpr unsigned kFull = 0xffffffffu;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kStreamMaxStages;
    uint64_t* mid = empty + kStreamMaxStages;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(mid + kStreamMaxStages);
    unsigned char* stages = smem + L.off_stages;
    double* bins = reinterpret_cast<double*>(smem + L.off_bins);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int NS = L.NS;
    const bool scatter = (MODE == kRhs) || a.scatter;
    const bool buckets = scatter && a.nS > 0;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kStreamWarps);
            mbar_init(&mid[i], kStreamWarps);
        }
        *abort_flag = 0;
        mbar_fence_init();
    }
    if (a.nS > 0)
        for (int i = threadIdx.x; i < a.SG * 16; i += kStreamThreads) bins[i] = 0.0;
    if (MODE == kFinal && a.nS > 0) {
        double* yt = reinterpret_cast<double*>(smem + L.off_yt);
        for (int i = threadIdx.x; i < a.SG * 16; i += kStreamThreads) {
            const int row = i >> 4, cc = i & 15;
            yt[i] = cc < a.CP ? a.x[(a.sbase[0] + row) * a.CP + cc] : 0.0;
        }
    }
    __syncthreads();

    if (warp == kStreamWarps) {
        // ------------------------------ producer ------------------------------
        // this lane's copy: column `lane`, the record, or one id array
        const int jc = lane - a.cols;  // 0: record, then weights, small ids, large ids
        int kind = lane < a.cols ? 0 : -1;
        int dst = 0;
        if (lane < a.cols) {
            dst = L.off_cols + lane * kStreamPitchD * 8;
        } else {
            int j = jc;
            if (j == 0) {
                kind = 1;
                dst = L.off_blob;
            }
            j -= 1;
            if (WEIGHTED) {
                if (j == 0) {
                    kind = 2;
                    dst = L.off_wp;
                }
                j -= 1;
            }
            if (MODE == kFinal && a.nS > 0) {
                if (j == 0) {
                    kind = 3;
                    dst = L.off_sid;
                }
                j -= 1;
            }
            if (MODE == kFinal && a.nL > 1 && j >= 0 && j < a.nL) {
                kind = 4 + j;
                dst = L.off_rid[j];
            }
        }
        const double* colbase = lane < a.cols ? a.v + static_cast<int64_t>(lane) * a.n : nullptr;
        const int32_t* ridbase = (kind >= 4) ? a.rid[kind - 4] : nullptr;

        auto load_batch = [&](int ib, int4& q0, int4& q1, int2& qb) {
            const int64_t t = blockIdx.x + static_cast<int64_t>(ib + lane) * gridDim.x;
            q0 = make_int4(0, 0, 0, 0);
            q1 = make_int4(0, 0, 0, 0);
            qb = make_int2(0, 0);
            if (t < L.nreg) {
                q0 = __ldg(L.tmeta + 2 * t);
                q1 = __ldg(L.tmeta + 2 * t + 1);
                qb.x = __ldg(L.boff + t);
                qb.y = __ldg(L.boff + t + 1);
            }
        };
        // the stage's 16-byte-aligned interior of every output column (kFinal)
        auto store_stage = [&](int slot) {
            const unsigned char* st = stages + static_cast<int64_t>(slot) * L.stage_bytes;
            const int4 m0 = *reinterpret_cast<const int4*>(st);
            if (lane < a.cols) {
                const int64_t e0 = static_cast<int64_t>(lane) * a.n + m0.x;
                const uintptr_t A = reinterpret_cast<uintptr_t>(a.out + e0);
                const uintptr_t B = A + static_cast<uintptr_t>(m0.y) * 8;
                const uintptr_t A16 = (A + 15) & ~static_cast<uintptr_t>(15);
                const uintptr_t B16 = B & ~static_cast<uintptr_t>(15);
                if (B16 > A16) {
                    const double* colp = reinterpret_cast<const double*>(st + dst) + span_phase<8>(a.v, e0);
                    bulk_store(reinterpret_cast<void*>(A16), colp + (A16 - A) / 8,
                               static_cast<uint32_t>(B16 - A16));
                }
                bulk_commit();
                bulk_wait_read();
            }
        };
        int issued = 0;  // tiles whose copies were issued
        int4 q0, q1, n0, n1;
        int2 qb, nb;
        load_batch(0, q0, q1, qb);
        load_batch(32, n0, n1, nb);
        for (;;) {
            const int64_t t = blockIdx.x + static_cast<int64_t>(issued) * gridDim.x;
            if (t >= L.nreg) break;
            const int qq = issued & 31;
            if (qq == 0 && issued > 0) {
                q0 = n0;
                q1 = n1;
                qb = nb;
                load_batch(issued + 32, n0, n1, nb);
            }
            const int k0 = __shfl_sync(kFull, q0.x, qq);
            const int nk = __shfl_sync(kFull, q0.y, qq);
            const int b0 = __shfl_sync(kFull, qb.x, qq);
            const int b1 = __shfl_sync(kFull, qb.y, qq);
            const int slot = issued % NS;
            if (issued >= NS) {
                if (!stream_wait_warp(&empty[slot], ((issued / NS) - 1) & 1, abort_flag, L.status)) break;
                if (MODE == kFinal) store_stage(slot);
                __syncwarp();
            }
            unsigned char* st = stages + static_cast<int64_t>(slot) * L.stage_bytes;
            const unsigned char* src = nullptr;
            uint32_t bytes = 0;
            if (kind == 0) span_of<8>(colbase, k0, nk, &src, &bytes);
            else if (kind == 1) {
                src = L.blob + static_cast<int64_t>(b0) * 16;
                bytes = static_cast<uint32_t>(b1 - b0) * 16u;
            } else if (kind == 2) span_of<8>(a.wp, k0, nk, &src, &bytes);
            else if (kind == 3) span_of<4>(a.sid, k0, nk, &src, &bytes);
            else if (kind >= 4) span_of<4>(ridbase, k0, nk, &src, &bytes);
            uint32_t total = bytes;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(kFull, total, o);
            if (lane == qq) {  // the lane holding this tile's record writes the header and arrives
                reinterpret_cast<int4*>(st)[0] = q0;
                reinterpret_cast<int4*>(st)[1] = q1;
                mbar_arrive_tx(&full[slot], total);
            }
            __syncwarp();
            if (bytes) bulk_load(st + dst, src, bytes, &full[slot]);
            ++issued;
        }
        if (*abort_flag) {
            // let the copies in flight land before the CTA exits
            if (lane == 0)
                for (int j = (issued > NS ? issued - NS : 0); j < issued; ++j) {
                    const long long t0 = clock64();
                    while (!mbar_test(&full[j % NS], (j / NS) & 1) && clock64() - t0 < kStreamWaitCycles) {
                    }
                }
        } else if (MODE == kFinal) {
            for (int j = (issued > NS ? issued - NS : 0); j < issued; ++j) {
                if (!stream_wait_warp(&empty[j % NS], (j / NS) & 1, abort_flag, L.status)) break;
                store_stage(j % NS);
                __syncwarp();
            }
        }
        bulk_wait_all();
        return;
    }

    // ------------------------------ consumers --------------------------------
    const int c = lane & 15;
    const int h = lane >> 4;
    const int grp = warp * 2 + h;  // half-warp group
    const bool col_lane = c < a.cols;
    const int CP = a.CP;
    double colsq = 0.0;

    // step 2 of the tile in `slot`: buckets of equal small-dim level
    auto buckets_of = [&](int slot) {
        unsigned char* st = stages + static_cast<int64_t>(slot) * L.stage_bytes;
        const int4 m0 = reinterpret_cast<const int4*>(st)[0];
        const int4 m1 = reinterpret_cast<const int4*>(st)[1];
        const int k0 = m0.x, nk = m0.y;
        const BlobLayout B = blob_layout(L.aux_stride, nk, m0.w, a.nL, m1.y, m1.w, a.nS);
        const unsigned char* blob = st + L.off_blob;
        const uint16_t* aux = reinterpret_cast<const uint16_t*>(blob);
        const double* col = reinterpret_cast<const double*>(st + L.off_cols + c * kStreamPitchD * 8) +
                            (col_lane ? span_phase<8>(a.v, static_cast<int64_t>(c) * a.n + k0) : 0);
        const double* wv = nullptr;
        if (MODE == kFinal && WEIGHTED)
            wv = reinterpret_cast<const double*>(st + L.off_wp) + span_phase<8>(a.wp, k0);
        int abase = (1 + a.nL) * (kStreamWarps + 1);
#pragma unroll
        for (int s = 0; s < kMaxSmall; ++s) {
            if (s >= a.nS) break;
            const uint16_t* ord = reinterpret_cast<const uint16_t*>(blob + B.ord[s]);
            const int levels = (s + 1 < a.nS ? a.sgoff[s + 1] : a.SG) - a.sgoff[s];
            for (int hh = grp; hh < levels; hh += 2 * kStreamWarps) {
                const int j0 = aux[abase + hh], j1 = aux[abase + hh + 1];
                if (j1 <= j0) continue;
                double acc = 0.0;
                for (int jj = j0; jj < j1; ++jj) {
                    const int k = ord[jj];
                    const double v = col_lane ? col[k] : 0.0;
                    acc += (MODE == kFinal && WEIGHTED) ? wv[k] * v : v;
                }
                bins[(a.sgoff[s] + hh) * 16 + c] += acc;
            }
            abase += levels + 1;
        }
    };

    int pend = -1;  // stage whose step 2 is still to do
    uint32_t pend_par = 0;
    for (int i = 0;; ++i) {
        const int64_t t = blockIdx.x + static_cast<int64_t>(i) * gridDim.x;
        if (t >= L.nreg) break;
        const int slot = i % NS;
        const uint32_t par = (i / NS) & 1;
        if (!stream_wait_warp(&full[slot], par, abort_flag, L.status)) break;
        unsigned char* st = stages + static_cast<int64_t>(slot) * L.stage_bytes;
        const int4 m0 = reinterpret_cast<const int4*>(st)[0];
        const int4 m1 = reinterpret_cast<const int4*>(st)[1];
        const int k0 = m0.x, nk = m0.y, s0 = m0.z;
        const BlobLayout B = blob_layout(L.aux_stride, nk, m0.w, a.nL, m1.y, m1.w, a.nS);
        const unsigned char* blob = st + L.off_blob;
        const uint16_t* aux = reinterpret_cast<const uint16_t*>(blob);
        const uint16_t* sego = reinterpret_cast<const uint16_t*>(blob + B.seg);
        const double* iw = reinterpret_cast<const double*>(blob + B.invw);
        const int64_t e0 = static_cast<int64_t>(c) * a.n + k0;
        double* col = reinterpret_cast<double*>(st + L.off_cols + c * kStreamPitchD * 8) +
                      (col_lane ? span_phase<8>(a.v, e0) : 0);
        const double* wv = nullptr;
        if (WEIGHTED) wv = reinterpret_cast<const double*>(st + L.off_wp) + span_phase<8>(a.wp, k0);
        const int sa = aux[warp], sb = aux[warp + 1];
        const int kb = sego[sa], ke = sego[sb];

        if (MODE == kFinal && a.nL > 1 && kb < ke) {
            // v - D_r a for this warp's observations, a batch of loads at a time
            const uint32_t* sidv = a.nS > 0 ? reinterpret_cast<const uint32_t*>(st + L.off_sid) +
                                                  span_phase<4>(a.sid, k0)
                                            : nullptr;
            const int32_t* ridv0 = a.nL > 0 ? reinterpret_cast<const int32_t*>(st + L.off_rid[0]) +
                                                  span_phase<4>(a.rid[0], k0)
                                            : nullptr;
            const int32_t* ridv1 = a.nL > 1 ? reinterpret_cast<const int32_t*>(st + L.off_rid[1]) +
                                                  span_phase<4>(a.rid[1], k0)
                                            : nullptr;
            for (int base = kb; base < ke; base += 2 * kStreamGather) {
                double u[kStreamGather];
#pragma unroll
                for (int q = 0; q < kStreamGather; ++q) {
                    const int k = base + 2 * q + h;
                    u[q] = 0.0;
                    if (k < ke && col_lane) {
                        if (a.nL > 0) u[q] += __ldg(a.x + (a.lbase[0] + ridv0[k]) * CP + c);
                        if (a.nL > 1) u[q] += __ldg(a.x + (a.lbase[1] + ridv1[k]) * CP + c);
                        if (a.nS > 0) {
                            const uint32_t packed = sidv[k];
                            for (int s = 0; s < a.nS; ++s)
                                u[q] += __ldg(a.x + (a.sbase[s] + ((packed >> (8 * s)) & 0xffu)) * CP + c);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kStreamGather; ++q) {
                    const int k = base + 2 * q + h;
                    if (k < ke && col_lane) col[k] -= u[q];
                }
            }
            __syncwarp();
        }

        // ---- 1. this warp's segments ------------------------------------------
        const uint16_t* rs0 = nullptr;
        const int32_t* rd0 = nullptr;
        const uint16_t* rs1 = nullptr;
        const int32_t* rd1 = nullptr;
        int r0c = 0, r1c = 0;
        if ((scatter || MODE == kFinal) && a.nL > 0) {
            rs0 = reinterpret_cast<const uint16_t*>(blob + B.runs[0]);
            rd0 = reinterpret_cast<const int32_t*>(blob + B.rd[0]);
            r0c = aux[(kStreamWarps + 1) + warp];
        }
        if (scatter && a.nL > 1) {
            rs1 = reinterpret_cast<const uint16_t*>(blob + B.runs[1]);
            rd1 = reinterpret_cast<const int32_t*>(blob + B.rd[1]);
            r1c = aux[2 * (kStreamWarps + 1) + warp];
        }
        if (MODE == kFinal && a.nL <= 1) {
            // v - D_r a - mean with one row of dim 0 per run (held in afb, up to
            // kStreamRunRows runs loaded at a time) and the small-dim rows from yt
            const uint32_t* sidv = a.nS > 0 ? reinterpret_cast<const uint32_t*>(st + L.off_sid) +
                                                  span_phase<4>(a.sid, k0)
                                            : nullptr;
            const double* yt = reinterpret_cast<const double*>(smem + L.off_yt);
            double* afb = reinterpret_cast<double*>(smem + L.off_afb) + warp * kStreamRunRows * 16;
            const int32_t* rg0 = reinterpret_cast<const int32_t*>(blob + B.rg);
            const int rend = a.nL > 0 ? aux[(kStreamWarps + 1) + warp + 1] : 0;
            int fb = r0c, fe = r0c;
            auto small_rows = [&](int k) {
                double y = 0.0;
                if (a.nS > 0) {
                    const uint32_t packed = sidv[k];
                    for (int s = 0; s < a.nS; ++s) y += yt[(a.sgoff[s] + ((packed >> (8 * s)) & 0xffu)) * 16 + c];
                }
                return y;
            };
            for (int j = sa; j < sb; ++j) {
                const int b = sego[j], e = sego[j + 1];
                const int rstart = r0c;
                double acc = 0.0;
                if (a.nL == 1) {
                    while (rs0[r0c] < e) {
                        if (r0c >= fe) {
                            __syncwarp();
                            fb = r0c;
                            fe = min(rend, r0c + kStreamRunRows);
                            double rows[kStreamRunRows / 2];
#pragma unroll
                            for (int q = 0; q < kStreamRunRows / 2; ++q) {
                                const int rr = fb + 2 * q + h;
                                rows[q] = (rr < fe && c < CP) ? __ldg(a.x + (a.lbase[0] + rg0[rr]) * CP + c) : 0.0;
                            }
#pragma unroll
                            for (int q = 0; q < kStreamRunRows / 2; ++q) afb[(2 * q + h) * 16 + c] = rows[q];
                            __syncwarp();
                        }
                        const double af = afb[(r0c - fb) * 16 + c];
                        const int q0 = rs0[r0c], q1 = rs0[r0c + 1];
                        for (int k = q0 + h; k < q1; k += 2) {
                            if (col_lane) {
                                const double u = col[k] - af - small_rows(k);
                                col[k] = u;
                                acc = WEIGHTED ? fma(wv[k], u, acc) : acc + u;
                            }
                        }
                        ++r0c;
                    }
                } else {
                    for (int k = b + h; k < e; k += 2) {
                        if (col_lane) {
                            const double u = col[k] - small_rows(k);
                            col[k] = u;
                            acc = WEIGHTED ? fma(wv[k], u, acc) : acc + u;
                        }
                    }
                }
                acc += __shfl_xor_sync(kFull, acc, 16);
                const double mean = acc * iw[j];
                if (a.mean_out && h == 0 && c < CP) a.mean_out[static_cast<int64_t>(s0 + j) * CP + c] = mean;
                double zs = 0.0;
                if (a.nL == 1) {
                    for (int r = rstart; r < r0c; ++r) {
                        const int q0 = rs0[r], q1 = rs0[r + 1];
                        double racc = 0.0;
                        for (int k = q0 + h; k < q1; k += 2) {
                            const double d = col_lane ? col[k] - mean : 0.0;
                            const double z = WEIGHTED ? wv[k] * d : d;
                            if (col_lane) col[k] = d;
                            racc += z;
                            zs += z;
                        }
                        if (scatter) {
                            racc += __shfl_xor_sync(kFull, racc, 16);
                            if (h == 0 && c < CP) __stcs(a.R[0] + static_cast<int64_t>(rd0[r]) * CP + c, racc);
                        }
                    }
                } else {
                    for (int k = b + h; k < e; k += 2) {
                        const double d = col_lane ? col[k] - mean : 0.0;
                        if (col_lane) col[k] = d;
                        zs += WEIGHTED ? wv[k] * d : d;
                    }
                }
                zs += __shfl_xor_sync(kFull, zs, 16);
                if (h == 0) colsq = fma(zs, zs, colsq);
            }
        } else
        for (int j = sa; j < sb; ++j) {
            const int b = sego[j], e = sego[j + 1];
            double acc = 0.0;
            for (int k = b + h; k < e; k += 2) {
                const double v = col_lane ? col[k] : 0.0;
                acc = WEIGHTED ? fma(wv[k], v, acc) : acc + v;
                if (MODE == kRhs) colsq = fma(v, v, colsq);
            }
            acc += __shfl_xor_sync(kFull, acc, 16);
            const double mean = acc * iw[j];
            if (MODE == kFinal && a.mean_out && h == 0 && c < CP)
                a.mean_out[static_cast<int64_t>(s0 + j) * CP + c] = mean;
            double zs = 0.0;
            if (rs0) {
                // runs of the first large dim: z (kRhs) or d (kFinal) into the stage
                while (rs0[r0c] < e) {
                    const int q0 = rs0[r0c], q1 = rs0[r0c + 1];
                    double racc = 0.0;
                    for (int k = q0 + h; k < q1; k += 2) {
                        const double d = col_lane ? col[k] - mean : 0.0;
                        const double z = WEIGHTED ? wv[k] * d : d;
                        racc += z;
                        if (col_lane) col[k] = MODE == kRhs ? z : d;
                        if (MODE == kFinal) zs += z;
                    }
                    racc += __shfl_xor_sync(kFull, racc, 16);
                    if (h == 0 && c < CP) __stcs(a.R[0] + static_cast<int64_t>(rd0[r0c]) * CP + c, racc);
                    ++r0c;
                }
                if (rs1) {
                    __syncwarp();  // z / d of the other half
                    while (rs1[r1c] < e) {
                        const int q0 = rs1[r1c], q1 = rs1[r1c + 1];
                        double racc = 0.0;
                        for (int k = q0 + h; k < q1; k += 2) {
                            const double d = col_lane ? col[k] : 0.0;
                            racc += (MODE == kFinal && WEIGHTED) ? wv[k] * d : d;
                        }
                        racc += __shfl_xor_sync(kFull, racc, 16);
                        if (h == 0 && c < CP) __stcs(a.R[1] + static_cast<int64_t>(rd1[r1c]) * CP + c, racc);
                        ++r1c;
                    }
                }
            } else {
                for (int k = b + h; k < e; k += 2) {
                    const double d = col_lane ? col[k] - mean : 0.0;
                    const double z = WEIGHTED ? wv[k] * d : d;
                    if (col_lane) col[k] = MODE == kRhs ? z : d;
                    if (MODE == kFinal) zs += z;
                }
            }
            if (MODE == kFinal) {
                zs += __shfl_xor_sync(kFull, zs, 16);
                if (h == 0) colsq = fma(zs, zs, colsq);
            }
        }
        if (MODE == kFinal && kb < ke) {
            __syncwarp();
            // the output elements outside the 16-byte interior the producer stores
            if (h == 0 && col_lane) {
                const uintptr_t A = reinterpret_cast<uintptr_t>(a.out + e0);
                if (kb == 0 && (A & 15u) != 0) a.out[e0] = col[0];
                if (ke == nk && ((A + static_cast<uintptr_t>(nk) * 8) & 15u) != 0) a.out[e0 + nk - 1] = col[nk - 1];
            }
        }
        __syncwarp();
        if (buckets) {
            // step 2 of the previous tile, then this tile waits for its own
            if (lane == 0) mbar_arrive(&mid[slot]);
            if (pend >= 0) {
                if (!stream_wait_warp(&mid[pend], pend_par, abort_flag, L.status)) break;
                buckets_of(pend);
                if (MODE == kFinal) fence_async_shared();
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[pend]);
            }
            pend = slot;
            pend_par = par;
        } else {
            if (MODE == kFinal) fence_async_shared();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot]);
        }
    }
    if (pend >= 0 && !*abort_flag) {
        if (stream_wait_warp(&mid[pend], pend_par, abort_flag, L.status)) {
            buckets_of(pend);
            if (MODE == kFinal) fence_async_shared();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[pend]);
        }
    }

    // ---- per-CTA partials (consumer warps only) -------------------------------
    double* red = reinterpret_cast<double*>(smem + L.off_red);
    colsq += __shfl_xor_sync(kFull, colsq, 16);
    if (h == 0) red[warp * 16 + c] = colsq;
    asm volatile("bar.sync 1, %0;" ::"r"(kStreamWarps * 32) : "memory");
    const int tid = threadIdx.x;
    const int cta = a.bins_cta0 + blockIdx.x;
    if (a.nS > 0 && scatter) {
        double* dst = a.bins_partial + static_cast<int64_t>(cta) * a.SG * CP;
        for (int idx = tid; idx < a.SG * CP; idx += kStreamWarps * 32) {
            const int row = idx / CP, cc = idx - row * CP;
            dst[idx] = bins[row * 16 + cc];
        }
    }
    if (tid < CP) {
        double sum = 0.0;
        for (int w = 0; w < kStreamWarps; ++w) sum += red[w * 16 + tid];
        a.colsq_partial[static_cast<int64_t>(cta) * CP + tid] = sum;
    }
}

// ---------------------------------------------------------------------------
// Setup: the regular tiles (those not holding a single long segment) in tile
// order, and one record per regular tile.
// ---------------------------------------------------------------------------
struct TileMetaArgs {
    int64_t ntiles;
    const int32_t* tile_seg;
    const uint8_t* tile_long;
    const int32_t* reg_idx;  // exclusive sum of the regular-tile flags
    const int32_t* seg_off;
    int nL, nS, aux_stride;
    const int32_t* run_base[kMaxLarge];
    int4* tmeta;
    int32_t* bsize;  // [nreg] record size in 16-byte units
    int* flags;      // [0] set when a regular tile exceeds the staged sizes; [1] largest record (bytes)
};

__global__ void tile_regular_flag_kernel(int64_t ntiles, const uint8_t* __restrict__ tile_long,
                                         int32_t* __restrict__ flag) {
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t <= ntiles;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flag[t] = (t < ntiles && !tile_long[t]) ? 1 : 0;
}

__global__ void tile_meta_kernel(const TileMetaArgs m) {
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < m.ntiles;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (m.tile_long[t]) continue;
        const int32_t s0 = m.tile_seg[t], s1 = m.tile_seg[t + 1];
        const int32_t k0 = m.seg_off[s0], k1 = m.seg_off[s1];
        const int4 a = make_int4(k0, k1 - k0, s0, s1 - s0);
        int4 b = make_int4(0, 0, 0, 0);
        if (m.nL > 0) {
            b.x = m.run_base[0][s0];
            b.y = m.run_base[0][s1] - b.x;
        }
        if (m.nL > 1) {
            b.z = m.run_base[1][s0];
            b.w = m.run_base[1][s1] - b.z;
        }
        if (a.y > kTileObs - 1 || a.w > kTileObs) atomicOr(m.flags, 1);
        const int bytes = blob_layout(m.aux_stride, a.y, a.w, m.nL, b.y, b.w, m.nS).bytes;
        atomicMax(m.flags + 1, bytes);
        const int64_t j = m.reg_idx[t];
        m.tmeta[2 * j] = a;
        m.tmeta[2 * j + 1] = b;
        m.bsize[j] = bytes / 16;
    }
}

struct TileBlobArgs {
    int64_t nreg;
    const int4* tmeta;
    const int32_t* boff;  // [nreg + 1] record offsets (16-byte units)
    const int32_t* seg_off;
    const double* inv_wp;
    int nL;
    const int32_t* run_base[kMaxLarge];
    const int32_t* run_start[kMaxLarge];
    const int32_t* run_dest[kMaxLarge];
    const int32_t* run_grp0;  // level of dim 0 of every run of dim 0
    const uint32_t* sid;  // packed small-dim levels in primary order
    int nS;
    int sG[kMaxSmall];
    int aux_stride;
    unsigned char* blob;
};

constexpr int kBlobWarps = 4;

// One warp per regular tile writes its record: the first segment and runs of
// every consumer warp (the segments starting in its kStreamWarps-th of the
// tile's observations), the bucket offsets and stable order of the tile's
// observations by every small dim's level (a counting sort), and the tile's
// segment offsets, run offsets, run destinations and inverse weights.
__global__ void __launch_bounds__(kBlobWarps * 32) tile_blob_kernel(const TileBlobArgs m) {
    __shared__ int cnt[kBlobWarps][kSmallLevels];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t t = static_cast<int64_t>(blockIdx.x) * kBlobWarps + w;
    if (t >= m.nreg) return;
    const int4 m0 = m.tmeta[2 * t], m1 = m.tmeta[2 * t + 1];
    const int k0 = m0.x, nk = m0.y, s0 = m0.z, ns = m0.w;
    const int rb[2] = {m1.x, m1.z}, nr[2] = {m1.y, m1.w};
    unsigned char* blob = m.blob + static_cast<int64_t>(m.boff[t]) * 16;
    const BlobLayout B = blob_layout(m.aux_stride, nk, ns, m.nL, nr[0], nr[1], m.nS);
    uint16_t* ax = reinterpret_cast<uint16_t*>(blob);
    for (int i = lane; i < m.aux_stride; i += 32) ax[i] = 0;
    __syncwarp();
    const int span = (nk + kStreamWarps - 1) / kStreamWarps;
    for (int q = lane; q <= kStreamWarps; q += 32) {
        int v = ns;
        const int lo = q * span;
        if (q < kStreamWarps && lo < nk) {
            int a = 0, b = ns;  // first local segment starting at or after k0 + lo
            while (a < b) {
                const int mid = (a + b) >> 1;
                if (m.seg_off[s0 + mid] < k0 + lo) a = mid + 1;
                else b = mid;
            }
            v = a;
        }
        ax[q] = static_cast<uint16_t>(v);
        for (int l = 0; l < m.nL; ++l)
            ax[(1 + l) * (kStreamWarps + 1) + q] = static_cast<uint16_t>(m.run_base[l][s0 + v] - rb[l]);
    }
    // segment offsets, run offsets and destinations, inverse weights
    uint16_t* sg = reinterpret_cast<uint16_t*>(blob + B.seg);
    for (int j = lane; j <= ns; j += 32) sg[j] = static_cast<uint16_t>(m.seg_off[s0 + j] - k0);
    for (int l = 0; l < m.nL; ++l) {
        uint16_t* rs = reinterpret_cast<uint16_t*>(blob + B.runs[l]);
        int32_t* rd = reinterpret_cast<int32_t*>(blob + B.rd[l]);
        for (int j = lane; j <= nr[l]; j += 32) {
            rs[j] = static_cast<uint16_t>(m.run_start[l][rb[l] + j] - k0);
            if (j < nr[l]) rd[j] = m.run_dest[l][rb[l] + j];
        }
    }
    if (m.nL > 0) {
        int32_t* rg = reinterpret_cast<int32_t*>(blob + B.rg);
        for (int j = lane; j < nr[0]; j += 32) rg[j] = m.run_grp0[rb[0] + j];
    }
    double* iw = reinterpret_cast<double*>(blob + B.invw);
    for (int j = lane; j < ns; j += 32) iw[j] = m.inv_wp[s0 + j];
    // buckets
    int base = (1 + m.nL) * (kStreamWarps + 1);
    const unsigned lt = (1u << lane) - 1u;
    for (int s = 0; s < m.nS; ++s) {
        const int Gs = m.sG[s];
        uint16_t* ord = reinterpret_cast<uint16_t*>(blob + B.ord[s]);
        for (int hh = lane; hh < kSmallLevels; hh += 32) cnt[w][hh] = 0;
        __syncwarp();
        for (int q0 = 0; q0 < nk; q0 += 32) {
            const int j = q0 + lane;
            const bool valid = j < nk;
            const uint32_t key = valid ? ((m.sid[k0 + j] >> (8 * s)) & 0xffu) : 0x100u + lane;
            const unsigned mm = __match_any_sync(0xffffffffu, key);
            if (valid && (mm & lt) == 0) cnt[w][key] += __popc(mm);
            __syncwarp();
        }
        if (lane == 0) {
            int run = 0;
            for (int hh = 0; hh < Gs; ++hh) {
                const int cc = cnt[w][hh];
                cnt[w][hh] = run;
                ax[base + hh] = static_cast<uint16_t>(run);
                run += cc;
            }
            ax[base + Gs] = static_cast<uint16_t>(run);
        }
        __syncwarp();
        for (int q0 = 0; q0 < nk; q0 += 32) {
            const int j = q0 + lane;
            const bool valid = j < nk;
            const uint32_t key = valid ? ((m.sid[k0 + j] >> (8 * s)) & 0xffu) : 0x100u + lane;
            const unsigned mm = __match_any_sync(0xffffffffu, key);
            const int pos = valid ? cnt[w][key] + __popc(mm & lt) : 0;
            __syncwarp();
            if (valid) {
                ord[pos] = static_cast<uint16_t>(j);
                if ((mm & lt) == 0) cnt[w][key] += __popc(mm);
            }
            __syncwarp();
        }
        base += Gs + 1;
    }
}

}  // namespace b200fe
