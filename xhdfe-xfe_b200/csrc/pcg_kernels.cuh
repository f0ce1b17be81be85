// Persistent preconditioned CG over the explicit Schur block (one launch per
// inner solve).
//
// Operator: rows [0, Gf) of the large dim (S_ff as CSR, sparse_kernels.cuh,
// plus the dense coupling C_fy x_small when a small dim is coupled) and rows
// [Gf, Gf + SG) of the small dim (C_fy' x_f + C_yy x_small).  Preconditioner:
// Jacobi (dinv).  Every column runs its own CG with its own mask; a column
// stops when r'r <= thr[c] (or r'z stops being positive) and then keeps its x.
//
// One cooperative launch of NB CTAs (all resident) runs every iteration:
//
//   A  q = S p for the large rows: "short" rows (<= kShortNnz nonzeros,
//      including empty ones) by one lane group each, "long" rows in chunks of
//      kLongChunk nonzeros by one warp each (partials).  The same warps form
//      C_fy' p_f: each stages its rows' p and C_fy rows in shared memory and
//      adds their outer product into registers (lane l keeps column l % CP of
//      levels l / CP, l / CP + 32 / CP, ...), so C_fy is read once per
//      iteration.  The dot p'q per CTA (by linearity also for long-row chunks
//      and the small rows).
//   -- grid barrier --
//   B  alpha = r'z / p'q (every CTA reduces the NB partials in the same order,
//      so all hold the same alpha); long rows and small rows are finished
//      round-robin over CTAs and updated; then every CTA updates its
//      contiguous range of short rows: x += alpha p, r -= alpha q, z = dinv r,
//      with per-CTA partials of r'z and r'r.
//   -- grid barrier --
//   C  new r'z, r'r, beta, masks (again the same in every CTA); p = z + beta p
//      over the CTA's contiguous range of all rows.
//   -- grid barrier --
//
// Data written by other CTAs during the launch is read with ld.global.cg (L2;
// L1 is not coherent across CTAs).  Every sum has a fixed order, so results
// are bitwise reproducible.  The barrier's wait is bounded (kBarrierCycles):
// on timeout it sets *status and every CTA leaves at its next barrier.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sparse_kernels.cuh"

namespace b200fe {

constexpr int kPcgThreads = 256;
constexpr int kShortNnz = 32;        // rows with at most this many nonzeros: one lane group
constexpr int kLongChunk = 256;      // nonzeros per warp chunk of a long row
constexpr int kPcgMaxSG = 64;        // small-dim rows the kernel handles (coupled levels)
constexpr int kHugeChunks = 32;      // long rows with more chunks: summed by a whole CTA
constexpr long long kBarrierCycles = 4000000000LL;  // ~2 s at 1.9 GHz

template <typename T>
struct PcgArgs {
    int CP;
    int64_t Gf;                 // rows of the large dim (alpha rows 0..Gf-1)
    int SG, SGP;                // small-dim rows (0 without coupling); C_fy row stride
    const int32_t* row_off;     // [Gf+1] CSR of S_ff
    const int32_t* col;
    const T* val;
    int64_t nshort;
    const int4* short_meta;     // rows with <= kShortNnz nonzeros, ascending: {row, begin, end, 0}
    int64_t nlchunks;           // chunks of long rows (kLongChunk nonzeros each)
    const int4* lchunk_meta;    // {row, begin, end, 1 for the row's first chunk}
    int64_t nlong;
    const int32_t* long_rows;   // [nlong] row of each long row
    const int32_t* long_c0;     // [nlong] its chunk range in lchunk_*
    const int32_t* long_c1;
    int64_t nhuge;              // long rows of more than kHugeChunks chunks
    const int32_t* huge_li;     // [nhuge] their index in long_rows
    const T* cfy;               // [Gf][SGP] or null
    const double* cyy;          // [SG][SG] or null
    const T* dinv;              // [GR]
    T* x;
    T* r;
    T* z;
    T* p;
    T* q;
    double* lpart;              // [nlchunks][CP]
    double* cta_part;           // [NB][part_stride]
    int part_stride;            // CP * (3 + SG): pq | C_fy'p [SG][CP] | rz | rr
    const double* thr;          // [CP] stop threshold on r'r (<= 0: column inactive)
    int max_iter;
    // outputs for the host
    double* rz_out;             // [CP]
    int* iters_out;             // [CP] iterations while active
    int* loops_out;             // [1] iterations run
    unsigned int* bar;          // [2] grid barrier: arrivals, generation (zero at launch)
    int* status;                // [1] 0 ok; 2 barrier timeout
};

__device__ __forceinline__ void v4_load_cg(const float* p, V4<float>& o) {
    const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
    o.v[0] = t.x; o.v[1] = t.y; o.v[2] = t.z; o.v[3] = t.w;
}
__device__ __forceinline__ void v4_load_cg(const double* p, V4<double>& o) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    o.v[0] = a.x; o.v[1] = a.y; o.v[2] = b.x; o.v[3] = b.y;
}
__device__ __forceinline__ void v4_store(float* p, const V4<float>& a) {
    *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ void v4_store(double* p, const V4<double>& a) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a.v[0], a.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(a.v[2], a.v[3]);
}

// Dynamic shared memory of pcg_persistent_kernel: small rows of p [64][CP],
// per-warp staging of GPW rows of p and C_fy, the CTA's C_fy' p_f partial.
template <typename T>
__host__ __device__ constexpr size_t pcg_smem_bytes(int CP, int SGP) {
    return align16(static_cast<size_t>(kPcgMaxSG) * CP * sizeof(T)) +
           align16(static_cast<size_t>(kPcgThreads / 32) * (32 / (CP / 4)) * (CP + SGP) * sizeof(T)) +
           static_cast<size_t>(kPcgMaxSG) * CP * sizeof(double);
}

// Grid-wide barrier for a cooperative launch, bounded: returns false (and
// sets *status) when the wait exceeds kBarrierCycles or another CTA gave up.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, int* status) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = bar + 1;
        const unsigned int g = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const long long t0 = clock64();
            while (*gen == g) {
                if (*reinterpret_cast<volatile int*>(status) != 0 || clock64() - t0 > kBarrierCycles) {
                    atomicOr(status, 2);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*reinterpret_cast<volatile int*>(status) != 0) ok = 0;
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// sum over CTAs b of part[b * stride + off + c] for c < CP, in CTA order
// within each thread's slice and a fixed tree across slices; the result is
// valid in threads c < CP.
__device__ __forceinline__ double cta_column_sum(const double* part, int nb, int stride, int off,
                                                 int CP, double* red) {
    const int t = threadIdx.x;
    const int J = kPcgThreads / CP;
    const int c = t % CP, j = t / CP;
    double s = 0.0;
    for (int b = j; b < nb; b += J) s += __ldcg(part + static_cast<int64_t>(b) * stride + off + c);
    red[t] = s;
    __syncthreads();
    for (int h = J / 2; h > 0; h >>= 1) {
        if (j < h) red[t] += red[t + h * CP];
        __syncthreads();
    }
    const double v = red[c];
    __syncthreads();
    return v;
}

// per-column sum of one value per thread (thread t holds column t % CP)
__device__ __forceinline__ double cta_reduce_by_column(double v, int CP, double* red) {
    const int t = threadIdx.x;
    const int J = kPcgThreads / CP;
    const int j = t / CP;
    red[t] = v;
    __syncthreads();
    for (int h = J / 2; h > 0; h >>= 1) {
        if (j < h) red[t] += red[t + h * CP];
        __syncthreads();
    }
    const double s = red[t % CP];
    __syncthreads();
    return s;
}

// 16-byte asynchronous copy global -> shared (cached in L2 only); the
// caller commits, waits and then __syncwarp()s before other lanes read it.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Per-column CTA sums of four values per thread: thread t holds columns
// 4 (t % CQ) .. 4 (t % CQ) + 3; fixed tree over the threads of one column
// quad.  out[c] (shared, CP entries) is valid after the call.
__device__ __forceinline__ void cta_reduce_quads(const double (&v)[4], int CQ, double* red, double* out) {
    const int t = threadIdx.x;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        red[t] = v[i];
        __syncthreads();
        for (int h = kPcgThreads / 2; h >= CQ; h >>= 1) {
            if (t < h) red[t] += red[t + h];
            __syncthreads();
        }
        if (t < CQ) out[4 * t + i] = red[t];
        __syncthreads();
    }
}

// q += sum over nonzeros j of val[j] p[col[j]] (4 columns of this lane) for
// j = j0, j0 + step, ... < je, U nonzeros per batch; the next batch's column
// ids and values are loaded while the current batch's rows of p are gathered.
template <typename T, int CP, int U>
__device__ __forceinline__ void gather_rows(const int32_t* __restrict__ col, const T* __restrict__ val,
                                            const T* p, int32_t j0, int32_t je, int step, int q4,
                                            Acc4& acc) {
    int32_t cj[U];
    T vj[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t j = j0 + u * step;
        cj[u] = j < je ? __ldg(col + j) : -1;
        vj[u] = j < je ? __ldg(val + j) : T(0);
    }
    for (int32_t jb = j0; jb < je; jb += U * step) {
        V4<T> xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (cj[u] >= 0) v4_load_cg(p + static_cast<int64_t>(cj[u]) * CP + 4 * q4, xv[u]);
            else v4_zero(xv[u]);
        }
        T vc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) vc[u] = vj[u];
        const int32_t jn = jb + U * step;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t j = jn + u * step;
            cj[u] = j < je ? __ldg(col + j) : -1;
            vj[u] = j < je ? __ldg(val + j) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                acc.v[i] = fma(static_cast<double>(vc[u]), static_cast<double>(xv[u].v[i]), acc.v[i]);
    }
}

// Per-warp outer-product accumulation of C_fy' p_f over the rows the warp
// staged (slab: nrows rows of [p (CP) | C_fy (SGP)]).  The [SGP/4][CP/4]
// blocks of 4 levels x 4 columns are dealt to the lanes (block l and l + 32),
// so a row costs a lane two 128-bit shared loads and 16 FMAs per block.
template <typename T>
__device__ __forceinline__ void lds4(const T* p, T (&v)[4]);
template <>
__device__ __forceinline__ void lds4<float>(const float* p, float (&v)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
template <>
__device__ __forceinline__ void lds4<double>(const double* p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <typename T, int CQ>
__device__ __forceinline__ void couple_rows(const T* slab, int nrows, int SGP, int lane,
                                            T (&cacc)[2][16]) {
    constexpr int CP = 4 * CQ;
    const int nblk = (SGP / 4) * CQ;
    for (int r = 0; r < nrows; ++r) {
        const T* row = slab + r * (CP + SGP);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int bk = lane + 32 * k;
            if (bk < nblk) {
                const int lq = bk / CQ, cq = bk % CQ;
                T pv[4], cv[4];
                lds4<T>(row + 4 * cq, pv);
                lds4<T>(row + CP + 4 * lq, cv);
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) cacc[k][4 * i + j] = fma(cv[i], pv[j], cacc[k][4 * i + j]);
            }
        }
    }
}

template <typename T, int CQ>
__global__ void __launch_bounds__(kPcgThreads, sizeof(T) == 4 ? 2 : 1)
pcg_persistent_kernel(const PcgArgs<T> a) {
    constexpr int CP = 4 * CQ;
    constexpr int GPW = 32 / CQ;  // lane groups per warp
    constexpr int U = 8;          // gathers in flight per lane group
    __shared__ double red[kPcgThreads];
    __shared__ double s_alpha[CP], s_beta[CP], s_rz[CP], s_pq[CP], s_q1[CP], s_q2[CP];
    __shared__ int s_active[CP], s_iters[CP];
    __shared__ int s_any;
    extern __shared__ __align__(16) unsigned char pcg_smem_raw[];
    T* s_xs = reinterpret_cast<T*>(pcg_smem_raw);  // [kPcgMaxSG][CP] small rows of p
    T* s_stage = reinterpret_cast<T*>(pcg_smem_raw + align16(static_cast<size_t>(kPcgMaxSG) * CP * sizeof(T)));
    double* s_cpart = reinterpret_cast<double*>(
        pcg_smem_raw + align16(static_cast<size_t>(kPcgMaxSG) * CP * sizeof(T)) +
        align16(static_cast<size_t>(kPcgThreads / 32) * GPW * (CP + a.SGP) * sizeof(T)));

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int gw = lane / CQ;
    const int q4 = lane % CQ;
    const int NB = gridDim.x;
    const int b = blockIdx.x;
    const int64_t GR = a.Gf + a.SG;
    const int PS = a.part_stride;
    const bool coupled = a.SG > 0;
    double* mypart = a.cta_part + static_cast<int64_t>(b) * PS;
    T* slab = s_stage + static_cast<size_t>(warp) * GPW * (CP + a.SGP);  // this warp's staging
    // contiguous row range owned by this CTA (updates, directions)
    const int64_t r0 = GR * b / NB, r1 = GR * (b + 1) / NB;
    const int c_of_t = tid % CP;  // column of this thread in flat row loops (256 % CP == 0)
    const int npairs = a.SG * CP;

    // ---- init: x = 0, z = dinv r, p = z; partials of r'z, r'r ----
    // (streaming loops: a thread owns column quad tq of rows in its CTA's
    // range, two quads in flight, every load issued before the stores)
    const int tq = tid % CQ;
    {
        double rz4[4] = {0.0, 0.0, 0.0, 0.0}, rr4[4] = {0.0, 0.0, 0.0, 0.0};
        const int64_t e1 = r1 * CQ;
        for (int64_t e = r0 * CQ + tid; e < e1; e += 2 * kPcgThreads) {
            const int64_t eb = e + kPcgThreads;
            const bool vb = eb < e1;
            V4<T> rv[2];
            T dv[2];
            v4_load_cg(a.r + 4 * e, rv[0]);
            dv[0] = __ldg(a.dinv + e / CQ);
            if (vb) {
                v4_load_cg(a.r + 4 * eb, rv[1]);
                dv[1] = __ldg(a.dinv + eb / CQ);
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !vb) break;
                const int64_t ee = k ? eb : e;
                V4<T> zv, xz;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const double ri = static_cast<double>(rv[k].v[i]);
                    zv.v[i] = static_cast<T>(static_cast<double>(dv[k]) * ri);
                    xz.v[i] = T(0);
                    rz4[i] = fma(ri, static_cast<double>(zv.v[i]), rz4[i]);
                    rr4[i] = fma(ri, ri, rr4[i]);
                }
                v4_store(a.x + 4 * ee, xz);
                v4_store(a.z + 4 * ee, zv);
                v4_store(a.p + 4 * ee, zv);
            }
        }
        cta_reduce_quads(rz4, CQ, red, s_q1);
        cta_reduce_quads(rr4, CQ, red, s_q2);
        if (tid < CP) {
            mypart[CP * (1 + a.SG) + tid] = s_q1[tid];
            mypart[CP * (2 + a.SG) + tid] = s_q2[tid];
        }
    }
    if (!grid_barrier(a.bar, a.status)) return;
    {
        const double rz = cta_column_sum(a.cta_part, NB, PS, CP * (1 + a.SG), CP, red);
        const double rr = cta_column_sum(a.cta_part, NB, PS, CP * (2 + a.SG), CP, red);
        if (tid < CP) {
            s_rz[tid] = rz;
            s_iters[tid] = 0;
            s_active[tid] = (a.thr[tid] > 0.0 && rr > a.thr[tid] && rz > 0.0) ? 1 : 0;
        }
        __syncthreads();
        if (tid == 0) {
            int any = 0;
            for (int c = 0; c < CP; ++c) any |= s_active[c];
            s_any = any;
        }
        __syncthreads();
    }

    int it = 0;
    while (s_any && it < a.max_iter) {
        // ================= A: q = S p, C_fy' p_f, dots =================
        if (coupled) {
            for (int i = tid; i < a.SGP * CP; i += kPcgThreads)
                s_xs[i] = i < a.SG * CP ? __ldcg(a.p + a.Gf * CP + i) : T(0);
            __syncthreads();
        }
        T cacc[2][16];  // this lane's 4x4 blocks of C_fy' p_f (see couple_rows)
#pragma unroll
        for (int k = 0; k < 2; ++k)
#pragma unroll
            for (int i = 0; i < 16; ++i) cacc[k][i] = T(0);
        double dot[4] = {0.0, 0.0, 0.0, 0.0};
        const int64_t nwarps = static_cast<int64_t>(NB) * (kPcgThreads / 32);
        const int64_t wid = static_cast<int64_t>(b) * (kPcgThreads / 32) + warp;
        // long-row chunks: a warp each, lane groups interleave the nonzeros;
        // the next chunk's record is loaded one chunk ahead
        int4 lm = wid < a.nlchunks ? __ldg(a.lchunk_meta + wid) : make_int4(0, 0, 0, 0);
        for (int64_t ch = wid; ch < a.nlchunks; ch += nwarps) {
            const int32_t g = lm.x, jb = lm.y, je = lm.z;
            const bool first = lm.w != 0;
            if (ch + nwarps < a.nlchunks) lm = __ldg(a.lchunk_meta + ch + nwarps);
            Acc4 acc;
            acc_zero(acc);
            gather_rows<T, CP, U>(a.col, a.val, a.p, jb + gw, je, GPW, q4, acc);
            // lane groups of the warp combined by a butterfly (every lane gets
            // the same sum)
#pragma unroll
            for (int o = 16; o >= CQ; o >>= 1)
#pragma unroll
                for (int i = 0; i < 4; ++i) acc.v[i] += __shfl_xor_sync(0xffffffffu, acc.v[i], o);
            V4<T> pv;
            v4_load_cg(a.p + static_cast<int64_t>(g) * CP + 4 * q4, pv);
            if (coupled && first) {
                // the row's first chunk carries C_fy[g] p_small, and adds the
                // row to the warp's C_fy' p_f
                const T* crow = a.cfy + static_cast<int64_t>(g) * a.SGP;
                if (gw == 0) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) slab[4 * q4 + i] = pv.v[i];
                }
                for (int h = lane; h < a.SGP; h += 32) slab[CP + h] = __ldg(crow + h);
                __syncwarp();
                T cs[4] = {T(0), T(0), T(0), T(0)};
                for (int h0 = 0; h0 < a.SGP; h0 += 4) {
                    T c4[4];
                    lds4<T>(slab + CP + h0, c4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        T xr[4];
                        lds4<T>(s_xs + (h0 + u) * CP + 4 * q4, xr);
#pragma unroll
                        for (int i = 0; i < 4; ++i) cs[i] = fma(c4[u], xr[i], cs[i]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) acc.v[i] += static_cast<double>(cs[i]);
                couple_rows<T, CQ>(slab, 1, a.SGP, lane, cacc);
                __syncwarp();
            }
            if (gw == 0) {
                double* dst = a.lpart + ch * CP + 4 * q4;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    dst[i] = acc.v[i];
                    dot[i] = fma(static_cast<double>(pv.v[i]), acc.v[i], dot[i]);
                }
            }
        }
        // short rows: GPW rows per warp, one lane group each.  With a coupled
        // small dim the row's C_fy row is copied into the warp's slab
        // (cp.async) while the gather runs.
        int4 sm = wid * GPW + gw < a.nshort ? __ldg(a.short_meta + wid * GPW + gw) : make_int4(0, 0, 0, 0);
        for (int64_t base = wid * GPW; base < a.nshort; base += nwarps * GPW) {
            const int64_t si = base + gw;
            const bool valid = si < a.nshort;
            const int32_t g = sm.x, jb = sm.y, je = sm.z;
            {  // the next step's record, one step ahead
                const int64_t sn = si + nwarps * GPW;
                sm = sn < a.nshort ? __ldg(a.short_meta + sn) : make_int4(0, 0, 0, 0);
            }
            T* srow = slab + gw * (CP + a.SGP);
            if (coupled) {
                constexpr int VT = 16 / sizeof(T);  // elements per 16-byte copy
                const T* crow = a.cfy + static_cast<int64_t>(g) * a.SGP;
                for (int v = q4; v < a.SGP / VT; v += CQ) {
                    if (valid) {
                        cp_async16(srow + CP + v * VT, crow + v * VT);
                    } else {
#pragma unroll
                        for (int u = 0; u < VT; ++u) srow[CP + v * VT + u] = T(0);
                    }
                }
                cp_async_commit();
            }
            Acc4 acc;
            acc_zero(acc);
            gather_rows<T, CP, U>(a.col, a.val, a.p, jb, je, 1, q4, acc);
            V4<T> pv;
            if (valid) v4_load_cg(a.p + static_cast<int64_t>(g) * CP + 4 * q4, pv);
            else v4_zero(pv);
            if (coupled) {
                cp_async_wait_all();
                __syncwarp();
                // C_fy[g] p_small (terms summed in the solve precision)
                T cs[4] = {T(0), T(0), T(0), T(0)};
                for (int h0 = 0; h0 < a.SGP; h0 += 4) {
                    T c4[4];
                    lds4<T>(srow + CP + h0, c4);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        T xr[4];
                        lds4<T>(s_xs + (h0 + u) * CP + 4 * q4, xr);
#pragma unroll
                        for (int i = 0; i < 4; ++i) cs[i] = fma(c4[u], xr[i], cs[i]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    acc.v[i] += static_cast<double>(cs[i]);
                    srow[4 * q4 + i] = pv.v[i];
                }
                __syncwarp();
                couple_rows<T, CQ>(slab, GPW, a.SGP, lane, cacc);
                __syncwarp();
            }
            if (valid) {
                V4<T> qs;
#pragma unroll
                for (int i = 0; i < 4; ++i) qs.v[i] = static_cast<T>(acc.v[i]);
                v4_store(a.q + static_cast<int64_t>(g) * CP + 4 * q4, qs);
#pragma unroll
                for (int i = 0; i < 4; ++i)  // dot with the stored (rounded) value
                    dot[i] = fma(static_cast<double>(pv.v[i]), static_cast<double>(qs.v[i]), dot[i]);
            }
        }
        // this CTA's C_fy' p_f: warps added in warp order
        if (coupled) {
            for (int i = tid; i < npairs; i += kPcgThreads) s_cpart[i] = 0.0;
            __syncthreads();
            for (int w = 0; w < kPcgThreads / 32; ++w) {
                if (warp == w) {
                    const int nblk = (a.SGP / 4) * CQ;
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        const int bk = lane + 32 * k;
                        if (bk < nblk) {
                            const int lq = bk / CQ, cq = bk % CQ;
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const int h = 4 * lq + i;
                                if (h < a.SG) {
#pragma unroll
                                    for (int j = 0; j < 4; ++j)
                                        s_cpart[h * CP + 4 * cq + j] += static_cast<double>(cacc[k][4 * i + j]);
                                }
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }
        // this CTA's pq partial: row dots (lane (gw, q4) holds columns 4 q4 + i,
        // summed over threads in thread order), plus p_small . (C_fy' p_f
        // partial), plus (CTA 0) p_small' C_yy p_small
        for (int i = 0; i < 4; ++i) {
            red[tid] = dot[i];
            __syncthreads();
            if (tid < CQ) {
                double sacc = 0.0;
                for (int t = tid; t < kPcgThreads; t += CQ) sacc += red[t];
                s_pq[4 * tid + i] = sacc;
            }
            __syncthreads();
        }
        double cdot = 0.0;  // column c_of_t
        if (coupled) {
            for (int pr = tid; pr < npairs; pr += kPcgThreads) {
                const int h = pr / CP;  // pr % CP == c_of_t
                mypart[CP + pr] = s_cpart[pr];
                cdot = fma(static_cast<double>(s_xs[pr]), s_cpart[pr], cdot);
                if (b == 0) {
                    double yq = 0.0;
                    for (int h2 = 0; h2 < a.SG; ++h2)
                        yq = fma(a.cyy[h * a.SG + h2], static_cast<double>(s_xs[h2 * CP + c_of_t]), yq);
                    cdot = fma(static_cast<double>(s_xs[pr]), yq, cdot);
                }
            }
        }
        {
            const double cs = cta_reduce_by_column(cdot, CP, red);
            if (tid < CP) mypart[tid] = s_pq[tid] + cs;
        }
        if (!grid_barrier(a.bar, a.status)) return;

        // ================= B: alpha, finish special rows, update =================
        {
            const double pq = cta_column_sum(a.cta_part, NB, PS, 0, CP, red);
            if (tid < CP) {
                const int act = s_active[tid];
                s_alpha[tid] = (act && pq > 0.0) ? s_rz[tid] / pq : 0.0;
            }
            __syncthreads();
        }
        double rzp = 0.0, rrp = 0.0;  // thread's column c_of_t
        // long rows of at most kHugeChunks chunks: a group of CP threads each
        // (thread c sums column c of the row's chunk partials in chunk order)
        {
            const int64_t ngrp = static_cast<int64_t>(NB) * (kPcgThreads / CP);
            const double al = s_alpha[c_of_t];
            for (int64_t li = static_cast<int64_t>(b) * (kPcgThreads / CP) + tid / CP; li < a.nlong;
                 li += ngrp) {
                const int32_t c0 = __ldg(a.long_c0 + li), c1 = __ldg(a.long_c1 + li);
                if (c1 - c0 > kHugeChunks) continue;
                const int64_t row = __ldg(a.long_rows + li);
                double qv = 0.0;
                for (int32_t k = c0; k < c1; ++k) qv += __ldcg(a.lpart + static_cast<int64_t>(k) * CP + c_of_t);
                const int64_t i = row * CP + c_of_t;
                double ri = static_cast<double>(__ldcg(a.r + i));
                if (al != 0.0) {
                    a.x[i] = static_cast<T>(static_cast<double>(__ldcg(a.x + i)) +
                                            al * static_cast<double>(__ldcg(a.p + i)));
                    ri -= al * static_cast<double>(static_cast<T>(qv));
                    const T rs = static_cast<T>(ri);
                    a.r[i] = rs;
                    ri = static_cast<double>(rs);
                }
                const T zi = static_cast<T>(static_cast<double>(__ldg(a.dinv + row)) * ri);
                a.z[i] = zi;
                rzp = fma(ri, static_cast<double>(zi), rzp);
                rrp = fma(ri, ri, rrp);
            }
        }
        // huge long rows and small rows, round-robin over CTAs; the CTA sums the
        // row's partials in a fixed order, thread c < CP updates column c
        const int64_t nspecial = a.nhuge + a.SG;
        for (int64_t sI = b; sI < nspecial; sI += NB) {
            int64_t row;
            double qv;
            if (sI < a.nhuge) {
                const int32_t li = __ldg(a.huge_li + sI);
                row = __ldg(a.long_rows + li);
                const int32_t c0 = __ldg(a.long_c0 + li), c1 = __ldg(a.long_c1 + li);
                qv = cta_column_sum(a.lpart + static_cast<int64_t>(c0) * CP, c1 - c0, CP, 0, CP, red);
            } else {
                const int h = static_cast<int>(sI - a.nhuge);
                row = a.Gf + h;
                qv = cta_column_sum(a.cta_part, NB, PS, CP + h * CP, CP, red);
                for (int h2 = 0; h2 < a.SG; ++h2)
                    qv = fma(a.cyy[h * a.SG + h2], static_cast<double>(s_xs[h2 * CP + c_of_t]), qv);
            }
            if (tid < CP) {
                const int64_t i = row * CP + tid;
                const T qs = static_cast<T>(qv);
                const double al = s_alpha[tid];
                double ri = static_cast<double>(__ldcg(a.r + i));
                if (al != 0.0) {
                    a.x[i] = static_cast<T>(static_cast<double>(__ldcg(a.x + i)) +
                                            al * static_cast<double>(__ldcg(a.p + i)));
                    ri -= al * static_cast<double>(qs);
                    const T rs = static_cast<T>(ri);
                    a.r[i] = rs;
                    ri = static_cast<double>(rs);
                }
                const T zi = static_cast<T>(static_cast<double>(__ldg(a.dinv + row)) * ri);
                a.z[i] = zi;
                rzp = fma(ri, static_cast<double>(zi), rzp);
                rrp = fma(ri, ri, rrp);
            }
        }
        // this CTA's short rows (contiguous range; long and small rows skipped)
        double rz4[4] = {0.0, 0.0, 0.0, 0.0}, rr4[4] = {0.0, 0.0, 0.0, 0.0};
        {
            double al4[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) al4[i] = s_alpha[4 * tq + i];
            const bool any_al = al4[0] != 0.0 || al4[1] != 0.0 || al4[2] != 0.0 || al4[3] != 0.0;
            const int64_t e1 = min(r1, a.Gf) * CQ;
            for (int64_t e = r0 * CQ + tid; e < e1; e += 2 * kPcgThreads) {
                const int64_t ev[2] = {e, e + kPcgThreads};
                bool use[2];
                V4<T> rv[2], xv[2], pv[2], qv[2];
                T dv[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    use[k] = ev[k] < e1;
                    if (use[k]) {
                        const int64_t row = ev[k] / CQ;
                        use[k] = __ldg(a.row_off + row + 1) - __ldg(a.row_off + row) <= kShortNnz;
                    }
                    if (use[k]) {
                        v4_load_cg(a.r + 4 * ev[k], rv[k]);
                        dv[k] = __ldg(a.dinv + ev[k] / CQ);
                        if (any_al) {
                            v4_load_cg(a.x + 4 * ev[k], xv[k]);
                            v4_load_cg(a.p + 4 * ev[k], pv[k]);
                            v4_load_cg(a.q + 4 * ev[k], qv[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (!use[k]) continue;
                    V4<T> zv;
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        double ri = static_cast<double>(rv[k].v[i]);
                        if (al4[i] != 0.0) {
                            xv[k].v[i] = static_cast<T>(static_cast<double>(xv[k].v[i]) +
                                                        al4[i] * static_cast<double>(pv[k].v[i]));
                            ri -= al4[i] * static_cast<double>(qv[k].v[i]);
                            rv[k].v[i] = static_cast<T>(ri);
                            ri = static_cast<double>(rv[k].v[i]);
                        }
                        zv.v[i] = static_cast<T>(static_cast<double>(dv[k]) * ri);
                        rz4[i] = fma(ri, static_cast<double>(zv.v[i]), rz4[i]);
                        rr4[i] = fma(ri, ri, rr4[i]);
                    }
                    if (any_al) {
                        v4_store(a.x + 4 * ev[k], xv[k]);
                        v4_store(a.r + 4 * ev[k], rv[k]);
                    }
                    v4_store(a.z + 4 * ev[k], zv);
                }
            }
        }
        rzp = cta_reduce_by_column(rzp, CP, red);
        rrp = cta_reduce_by_column(rrp, CP, red);
        cta_reduce_quads(rz4, CQ, red, s_q1);
        cta_reduce_quads(rr4, CQ, red, s_q2);
        if (tid < CP) {
            mypart[CP * (1 + a.SG) + tid] = rzp + s_q1[tid];
            mypart[CP * (2 + a.SG) + tid] = rrp + s_q2[tid];
        }
        if (!grid_barrier(a.bar, a.status)) return;

        // ================= C: beta, masks, directions =================
        {
            const double rz = cta_column_sum(a.cta_part, NB, PS, CP * (1 + a.SG), CP, red);
            const double rr = cta_column_sum(a.cta_part, NB, PS, CP * (2 + a.SG), CP, red);
            if (tid < CP) {
                s_beta[tid] = 0.0;
                if (s_active[tid]) {
                    const double old = s_rz[tid];
                    s_beta[tid] = old > 0.0 ? rz / old : 0.0;
                    s_rz[tid] = rz;
                    s_iters[tid] += 1;
                    if (!(rr > a.thr[tid]) || !(rz > 0.0)) s_active[tid] = 0;
                }
            }
            __syncthreads();
            if (tid == 0) {
                int any = 0;
                for (int c = 0; c < CP; ++c) any |= s_active[c];
                s_any = any;
            }
            __syncthreads();
        }
        {
            // a column that just stopped keeps p (its x and r no longer move)
            bool act4[4];
            double be4[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                act4[i] = s_active[4 * tq + i] != 0;
                be4[i] = s_beta[4 * tq + i];
            }
            if (act4[0] || act4[1] || act4[2] || act4[3]) {
                const int64_t e1 = r1 * CQ;
                for (int64_t e = r0 * CQ + tid; e < e1; e += 2 * kPcgThreads) {
                    const int64_t eb = e + kPcgThreads;
                    const bool vb = eb < e1;
                    V4<T> zv[2], pv[2];
                    v4_load_cg(a.z + 4 * e, zv[0]);
                    v4_load_cg(a.p + 4 * e, pv[0]);
                    if (vb) {
                        v4_load_cg(a.z + 4 * eb, zv[1]);
                        v4_load_cg(a.p + 4 * eb, pv[1]);
                    }
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        if (k == 1 && !vb) break;
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (act4[i])
                                pv[k].v[i] = static_cast<T>(static_cast<double>(zv[k].v[i]) +
                                                            be4[i] * static_cast<double>(pv[k].v[i]));
                        v4_store(a.p + 4 * (k ? eb : e), pv[k]);
                    }
                }
            }
        }
        ++it;
        if (!grid_barrier(a.bar, a.status)) return;
    }
    if (b == 0 && tid < CP) {
        a.rz_out[tid] = s_rz[tid];
        a.iters_out[tid] = s_iters[tid];
        if (tid == 0) *a.loops_out = it;
    }
}

}  // namespace b200fe

namespace b200fe {

// Work lists of pcg_persistent_kernel over the CSR rows of S_ff: per row g,
// is_short[g] (<= kShortNnz nonzeros), is_long[g] and its number of
// kLongChunk chunks.
__global__ void pcg_lists_count_kernel(const int32_t* __restrict__ row_off, int32_t G,
                                       int32_t* __restrict__ is_short, int32_t* __restrict__ is_long,
                                       int32_t* __restrict__ nchunks, int32_t* __restrict__ is_huge) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t len = row_off[g + 1] - row_off[g];
        const bool sh = len <= kShortNnz;
        const int32_t nc = sh ? 0 : (len + kLongChunk - 1) / kLongChunk;
        is_short[g] = sh ? 1 : 0;
        is_long[g] = sh ? 0 : 1;
        nchunks[g] = nc;
        is_huge[g] = nc > kHugeChunks ? 1 : 0;
    }
}

// Fills the lists from the exclusive scans of the three counts.
__global__ void pcg_lists_fill_kernel(const int32_t* __restrict__ row_off, int32_t G,
                                      const int32_t* __restrict__ is_short,
                                      const int32_t* __restrict__ short_idx,
                                      const int32_t* __restrict__ long_idx,
                                      const int32_t* __restrict__ chunk_off,
                                      int4* __restrict__ short_meta, int32_t* __restrict__ long_rows,
                                      int32_t* __restrict__ long_c0, int32_t* __restrict__ long_c1,
                                      int4* __restrict__ lchunk_meta,
                                      const int32_t* __restrict__ huge_idx, int32_t* __restrict__ huge_li) {
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < G;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (is_short[g]) {
            short_meta[short_idx[g]] = make_int4(static_cast<int32_t>(g), row_off[g], row_off[g + 1], 0);
            continue;
        }
        const int32_t li = long_idx[g];
        const int32_t c0 = chunk_off[g], c1 = chunk_off[g + 1];
        long_rows[li] = static_cast<int32_t>(g);
        long_c0[li] = c0;
        long_c1[li] = c1;
        if (c1 - c0 > kHugeChunks) huge_li[huge_idx[g]] = li;
        const int32_t b = row_off[g], e = row_off[g + 1];
        for (int32_t c = c0; c < c1; ++c) {
            const int32_t cb = b + (c - c0) * kLongChunk;
            lchunk_meta[c] = make_int4(static_cast<int32_t>(g), cb, min(e, cb + kLongChunk), c == c0 ? 1 : 0);
        }
    }
}

}  // namespace b200fe
