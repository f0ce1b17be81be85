// Host orchestration of the heterogeneous-slope and group/individual
// absorbers (kernels in slope_kernels.cuh) and their C ABI entry points
// (include/b200fe.h).

#include "context.cuh"
#include "slope_kernels.cuh"
#include "common_kernels.cuh"

using namespace b200fe;
using namespace b200fe_host;

// ---------------------------------------------------------------------------
// Heterogeneous slopes (slope_kernels.cuh): block-Jacobi CGLS over all FE
// blocks, the path the reference's absorb_fixed_effects_cuda takes when a
// GpuFeInput has is_slope set (src/fe_absorption_cuda.cu:2316-2420).
// ---------------------------------------------------------------------------
namespace {

// The stop test bounds the preconditioned gradient sqrt(s' M^-1 s) =
// sqrt(sum_d ||P_d r||_W^2); the distance to the exact projection is at most
// that over sqrt(lambda_min) of the preconditioned operator, so the gradient
// is driven two orders below the requested tolerance.
constexpr double kSlopeTolFactor = 1e-2;

// Device copy of a group/individual structure (rows = groups, original order).
struct GiDev {
    int32_t I;
    int64_t E;
    const int32_t* gptr;   // [n + 1]
    const int32_t* gind;   // [E]
    const int32_t* iptr;   // [I + 1]
    const int32_t* igrp;   // [E]
    const double* scale;   // [n]
};

int slopes_device_impl(b200fe_context* ctx, const double* d_v, int64_t n, int C, int nd,
                       const int32_t* const* d_gids, const int32_t* G,
                       const double* const* d_z, const unsigned char* icpt, const double* d_w,
                       const GiDev* gi, const b200fe_options& o, double* d_out,
                       b200fe_result* res) {
    const cudaStream_t s = ctx->stream;
    const int T = kSlopeThreads;
    cudaEvent_t e0, e1, e2;
    B_TRY(cudaEventCreate(&e0));
    B_TRY(cudaEventCreate(&e1));
    B_TRY(cudaEventCreate(&e2));
    B_TRY(cudaEventRecord(e0, s));
    ctx->profiling = o.profile != 0;
    ctx->prof.clear();
    ctx->ev_used = 0;
    std::unique_ptr<ProfScope> setup_scope(new ProfScope(ctx, B200FE_PROF_SETUP, 0.0));
    // ---- validation
    int* flags;
    B_CHECK(get_buf(ctx, "sl_flags", 8, &flags));
    B_TRY(cudaMemsetAsync(flags, 0, 8 * sizeof(int), s));
    int p = -1;  // primary: the FE dimension with the most groups (none: -1)
    for (int d = 0; d < nd; ++d)
        if (p < 0 || G[d] > G[p]) p = d;
    if (gi) {
        finite_values_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(gi->scale, n, flags);
        B_LAUNCHED();
    }
    for (int d = 0; d < nd; ++d) {
        validate_ids_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(d_gids[d], n, G[d], d == p, flags);
        B_LAUNCHED();
        if (d_z[d]) {
            finite_values_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(d_z[d], n, flags);
            B_LAUNCHED();
        }
    }
    if (d_w) {
        validate_weights_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(d_w, n, flags);
        B_LAUNCHED();
    }
    int hf[4];
    B_CHECK(sync_read_int(ctx, flags, 4, hf));
    if (hf[0]) {
        ctx->err = "group ids out of range";
        return B200FE_INVALID_ARG;
    }
    if (hf[2]) {
        ctx->err = "weights must be non-negative and finite";
        return B200FE_INVALID_ARG;
    }
    if (hf[3]) {
        ctx->err = gi ? "slope values and group scales must be finite" : "slope values must be finite";
        return B200FE_INVALID_ARG;
    }
    // ---- observations in primary order
    int32_t *pord = nullptr, *iota = nullptr, *gp = nullptr;
    B_CHECK(get_buf(ctx, "sl_iota", n, &iota));
    iota_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(iota, n);
    B_LAUNCHED();
    if (p >= 0 && hf[1]) {
        B_CHECK(get_buf(ctx, "sl_pord", n, &pord));
        B_CHECK(get_buf(ctx, "sl_gp", n, &gp));
        B_CHECK(cub_sort_pairs(ctx, d_gids[p], gp, iota, pord, n, G[p]));
    } else if (p >= 0) {
        gp = const_cast<int32_t*>(d_gids[p]);
    }
    const double* w = d_w;
    if (d_w && pord) {
        double* wp;
        B_CHECK(get_buf(ctx, "sl_w", n, &wp));
        gather_kernel<double><<<grid_for(ctx, n, T), T, 0, s>>>(d_w, pord, n, wp);
        B_LAUNCHED();
        w = wp;
    }
    double *R, *Q;
    B_CHECK(get_buf(ctx, "sl_R", static_cast<size_t>(n) * C, &R));
    B_CHECK(get_buf(ctx, "sl_Q", static_cast<size_t>(n) * C, &Q));
    {
        ProfScope ps(ctx, B200FE_PROF_RHS, 16.0 * n * C + (pord ? 4.0 * n : 0.0));
        slope_load_kernel<<<grid_for(ctx, n * C, T), T, 0, s>>>(d_v, pord, n, C, R);
        B_LAUNCHED();
    }
    // ---- per-dim structure
    const int ndt = nd + (gi ? 1 : 0);  // the individual dimension is dims[nd]
    SlopeDim dims[kSlopeMaxDims];
    int order[kSlopeMaxDims];  // segment passes: the primary (the writer) last
    int no = 0;
    for (int d = 0; d < ndt; ++d)
        if (d != p) order[no++] = d;
    if (p >= 0) order[no++] = p;
    double op_norm2 = 0.0;
    int present[kSlopeMaxDims] = {0};
    int fin_grid[kSlopeMaxDims] = {0};
    int32_t* big_list[kSlopeMaxDims] = {nullptr};  // groups of more than kFinSerialChunks chunks
    int n_big[kSlopeMaxDims] = {0};
    const int RB = T / C;
    int32_t* p_ch_grp = nullptr;
    int32_t* inv_pord = nullptr;
    if (gi && pord) {
        B_CHECK(get_buf(ctx, "sl_invp", n, &inv_pord));
        inverse_perm_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(pord, n, inv_pord);
        B_LAUNCHED();
    }
    for (int d = 0; d < ndt; ++d) {
        const std::string sx = std::to_string(d);
        const int32_t Gd = d < nd ? G[d] : gi->I;
        SlopeDim& D = dims[d];
        D = SlopeDim{};
        D.G = Gd;
        int32_t *sorted = gp, *off, *nch, *grp_ch;
        if (d == nd) {
            // individuals: positions are the edges in individual order, each
            // mapped to its row in primary order; multiplier the group scale
            D.has_a = 0;
            D.has_b = 1;
            D.nb = 1;
            int32_t* perm;
            B_CHECK(get_buf(ctx, "sl_perm" + sx, gi->E, &perm));
            map_rows_kernel<<<grid_for(ctx, gi->E, T), T, 0, s>>>(gi->igrp, gi->E, inv_pord, perm);
            B_LAUNCHED();
            D.perm = perm;
            double* z = const_cast<double*>(gi->scale);
            if (pord) {
                B_CHECK(get_buf(ctx, "sl_z" + sx, n, &z));
                gather_kernel<double><<<grid_for(ctx, n, T), T, 0, s>>>(gi->scale, pord, n, z);
                B_LAUNCHED();
            }
            D.z = z;
            off = const_cast<int32_t*>(gi->iptr);
        } else {
            D.has_b = d_z[d] ? 1 : 0;
            D.has_a = d_z[d] ? (icpt && icpt[d] ? 1 : 0) : 1;
            D.nb = D.has_a + D.has_b;
            if (d == p) {
                D.ids = gp;
            } else {
                int32_t* ids = const_cast<int32_t*>(d_gids[d]);
                if (pord) {
                    B_CHECK(get_buf(ctx, "sl_ids" + sx, n, &ids));
                    gather_kernel<int32_t><<<grid_for(ctx, n, T), T, 0, s>>>(d_gids[d], pord, n, ids);
                    B_LAUNCHED();
                }
                D.ids = ids;
                int32_t* perm;
                B_CHECK(get_buf(ctx, "sl_perm" + sx, n, &perm));
                B_CHECK(get_buf(ctx, "sl_sorted", n, &sorted));
                B_CHECK(cub_sort_pairs(ctx, ids, sorted, iota, perm, n, G[d]));
                D.perm = perm;
            }
            if (d_z[d]) {
                double* z = const_cast<double*>(d_z[d]);
                if (pord) {
                    B_CHECK(get_buf(ctx, "sl_z" + sx, n, &z));
                    gather_kernel<double><<<grid_for(ctx, n, T), T, 0, s>>>(d_z[d], pord, n, z);
                    B_LAUNCHED();
                }
                D.z = z;
            }
            B_CHECK(get_buf(ctx, "sl_off" + sx, static_cast<size_t>(G[d]) + 1, &off));
            segment_offsets_kernel<<<grid_for(ctx, n + 1, T), T, 0, s>>>(sorted, n, G[d], off);
            B_LAUNCHED();
        }
        B_CHECK(get_buf(ctx, "sl_nch", static_cast<size_t>(Gd) + 1, &nch));
        B_CHECK(get_buf(ctx, "sl_grpch" + sx, static_cast<size_t>(Gd) + 1, &grp_ch));
        slope_chunk_count_kernel<<<grid_for(ctx, Gd + 1, T), T, 0, s>>>(off, Gd, nch);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, nch, grp_ch, static_cast<int64_t>(Gd) + 1));
        int* cnt;
        B_CHECK(get_buf(ctx, "sl_cnt", 1, &cnt));
        B_TRY(cudaMemsetAsync(cnt, 0, sizeof(int), s));
        count_nonempty_kernel<<<grid_for(ctx, Gd, T), T, 0, s>>>(off, Gd, cnt);
        B_LAUNCHED();
        int hc[2];
        B_CHECK(sync_read_int(ctx, grp_ch + Gd, 1, &hc[0]));
        B_CHECK(sync_read_int(ctx, cnt, 1, &hc[1]));
        D.nch = hc[0];
        present[d] = hc[1];
        int32_t *cb, *ce;
        B_CHECK(get_buf(ctx, "sl_chb" + sx, D.nch, &cb));
        B_CHECK(get_buf(ctx, "sl_che" + sx, D.nch, &ce));
        int32_t* cg_of = nullptr;  // chunk -> group, kept for the primary (Schur gather)
        if (d == p) B_CHECK(get_buf(ctx, "sl_chgrp", D.nch, &cg_of));
        slope_chunk_fill_kernel<<<grid_for(ctx, Gd, T), T, 0, s>>>(off, Gd, grp_ch, cb, ce, cg_of);
        B_LAUNCHED();
        D.ch_beg = cb;
        D.ch_end = ce;
        D.grp_ch = grp_ch;
        if (d == p) p_ch_grp = cg_of;
        // moments and block inverses
        double *cm, *minv, *pop;
        B_CHECK(get_buf(ctx, "sl_cm", static_cast<size_t>(D.nch) * 5, &cm));
        B_CHECK(get_buf(ctx, "sl_minv" + sx, static_cast<size_t>(Gd) * 3, &minv));
        slope_moments_kernel<<<grid_for(ctx, static_cast<int64_t>(D.nch) * 32, T), T, 0, s>>>(D, w, cm);
        B_LAUNCHED();
        const int gb = grid_for(ctx, Gd, T, 4);
        B_CHECK(get_buf(ctx, "sl_pop", gb, &pop));
        slope_block_inverse_kernel<<<gb, T, 0, s>>>(D, cm, minv, pop);
        B_LAUNCHED();
        D.minv = minv;
        std::vector<double> hp(gb);
        B_TRY(cudaMemcpyAsync(hp.data(), pop, sizeof(double) * gb, cudaMemcpyDeviceToHost, s));
        B_TRY(cudaStreamSynchronize(s));
        for (double v : hp) op_norm2 += v;
        const size_t cw = static_cast<size_t>(Gd) * D.nb * C;
        B_CHECK(get_buf(ctx, "sl_part" + sx, static_cast<size_t>(D.nch) * D.nb * C, &D.part));
        B_CHECK(get_buf(ctx, "sl_zv" + sx, cw, &D.zv));
        B_CHECK(get_buf(ctx, "sl_p" + sx, cw, &D.p));
        fin_grid[d] = grid_for(ctx, (Gd + RB - 1) / RB, 1, 4);
        {
            int32_t *flag, *idx;
            B_CHECK(get_buf(ctx, "sl_bflag", Gd, &flag));
            B_CHECK(get_buf(ctx, "sl_bidx", Gd, &idx));
            multi_chunk_flags_kernel<<<grid_for(ctx, Gd, T), T, 0, s>>>(grp_ch, nullptr, Gd, flag,
                                                                        kFinSerialChunks);
            B_LAUNCHED();
            B_CHECK(cub_exclusive_sum(ctx, flag, idx, Gd));
            int hv[2];
            B_CHECK(sync_read_int(ctx, idx + (Gd - 1), 1, &hv[0]));
            B_CHECK(sync_read_int(ctx, flag + (Gd - 1), 1, &hv[1]));
            n_big[d] = hv[0] + hv[1];
            if (n_big[d] > 0) {
                B_CHECK(get_buf(ctx, "sl_blist" + sx, n_big[d], &big_list[d]));
                compact_kernel<<<grid_for(ctx, Gd, T), T, 0, s>>>(flag, idx, Gd, big_list[d]);
                B_LAUNCHED();
                B_CHECK(get_buf(ctx, "sl_big" + sx, cw, &D.big));
            }
        }
    }
    // ---- Schur form: the primary dimension eliminated exactly (auto, or
    // pass_kernel 1 for block Jacobi over every dimension)
    const bool schur = !gi && p >= 0 && nd >= 2 && o.pass_kernel != 1;
    std::vector<int> cg;  // dimensions the CG runs over, in pass order (writer last)
    for (int i = 0; i < no; ++i)
        if (!(schur && order[i] == p)) cg.push_back(order[i]);
    const int ncg = static_cast<int>(cg.size());
    // Schur form: the residual is updated by one coalesced pass in primary order
    // (slope_update_kernel) and the CG dims' passes read it through their
    // permutations; otherwise the primary's in-order segment pass stores it.
    const int writer = schur ? -1 : p;
    if (schur && dims[p].has_a && dims[p].has_b) {
        // the primary's slope in the centred basis (same span, well-conditioned
        // blocks); the certificate's primary share is then taken in that basis
        SlopeDim& P = dims[p];
        double *cm, *tbar, *zc, *minv_c;
        B_CHECK(get_buf(ctx, "sl_cm", static_cast<size_t>(P.nch) * 5, &cm));
        B_CHECK(get_buf(ctx, "sl_tbar", P.G, &tbar));
        B_CHECK(get_buf(ctx, "sl_zc", n, &zc));
        B_CHECK(get_buf(ctx, "sl_minvc", static_cast<size_t>(P.G) * 3, &minv_c));
        slope_moments_kernel<<<grid_for(ctx, static_cast<int64_t>(P.nch) * 32, T), T, 0, s>>>(P, w, cm);
        B_LAUNCHED();
        slope_group_center_kernel<<<grid_for(ctx, P.G, T), T, 0, s>>>(P, cm, tbar);
        B_LAUNCHED();
        slope_center_rows_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(P.ids, P.z, tbar, n, zc);
        B_LAUNCHED();
        P.z = zc;
        slope_moments_kernel<<<grid_for(ctx, static_cast<int64_t>(P.nch) * 32, T), T, 0, s>>>(P, w, cm);
        B_LAUNCHED();
        slope_centred_inverse_kernel<<<grid_for(ctx, P.G, T), T, 0, s>>>(P, cm, P.minv, minv_c);
        B_LAUNCHED();
        P.minv = minv_c;
    }
    if (schur) {
        for (int d : cg) {
            SlopeDim& D = dims[d];
            const std::string sx = std::to_string(d);
            int32_t *flag, *pid, *start, *off;
            double* contrib;
            B_CHECK(get_buf(ctx, "sl_pflag", n, &flag));
            B_CHECK(get_buf(ctx, "sl_pid", n, &pid));
            pair_flags_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(D.perm, D.ids, dims[p].ids, n, flag);
            B_LAUNCHED();
            B_CHECK(cub_inclusive_sum(ctx, flag, pid, n));
            int np = 0;
            B_CHECK(sync_read_int(ctx, pid + (n - 1), 1, &np));
            B_CHECK(get_buf(ctx, "sl_pstart", static_cast<size_t>(np) + 1, &start));
            pair_start_kernel<<<grid_for(ctx, n + 1, T), T, 0, s>>>(flag, pid, n, start);
            B_LAUNCHED();
            B_CHECK(get_buf(ctx, "sl_contrib", static_cast<size_t>(np) * 3, &contrib));
            pair_contrib_kernel<<<grid_for(ctx, np, T), T, 0, s>>>(D, dims[p], w, start, np,
                                                                   contrib);
            B_LAUNCHED();
            B_CHECK(get_buf(ctx, "sl_off" + sx, static_cast<size_t>(D.G) + 1, &off));
            // per group sums of the pair planes: one block per group, fixed order
            int32_t* poff;
            double* csum;
            B_CHECK(get_buf(ctx, "sl_poff", static_cast<size_t>(D.G) + 1, &poff));
            B_CHECK(get_buf(ctx, "sl_csum", static_cast<size_t>(D.G) * 3, &csum));
            pair_offsets_kernel<<<grid_for(ctx, static_cast<int64_t>(D.G) + 1, T), T, 0, s>>>(
                off, pid, D.G, n, np, poff);
            B_LAUNCHED();
            for (int m = 0; m < 3; ++m) {
                size_t tmp = 0;
                const double* in = contrib + static_cast<size_t>(m) * np;
                double* out = csum + static_cast<size_t>(m) * D.G;
                B_TRY(cub::DeviceSegmentedReduce::Sum(nullptr, tmp, in, out, D.G, poff, poff + 1, s));
                uint8_t* t;
                B_CHECK(get_buf(ctx, "cub_tmp", tmp, &t));
                B_TRY(cub::DeviceSegmentedReduce::Sum(t, tmp, in, out, D.G, poff, poff + 1, s));
                ++ctx->lib_calls;
            }
            double *cm, *pop;
            B_CHECK(get_buf(ctx, "sl_cm", static_cast<size_t>(D.nch) * 5, &cm));
            slope_moments_kernel<<<grid_for(ctx, static_cast<int64_t>(D.nch) * 32, T), T, 0, s>>>(D, w, cm);
            B_LAUNCHED();
            const int gb = grid_for(ctx, D.G, T, 4);
            B_CHECK(get_buf(ctx, "sl_pop", gb, &pop));
            schur_block_inverse_kernel<<<gb, T, 0, s>>>(D, cm, csum, const_cast<double*>(D.minv),
                                                        pop);
            B_LAUNCHED();
        }
    }
    // Schur gather: the primary groups spread over several chunks, and their chunks
    int32_t *multi_groups = nullptr, *multi_chunks = nullptr;
    int n_multi_groups = 0, n_multi_chunks = 0;
    if (schur) {
        const SlopeDim& P = dims[p];
        int32_t *flag, *idx;
        const int64_t m = std::max<int64_t>(P.G, P.nch);
        B_CHECK(get_buf(ctx, "sl_mflag", m, &flag));
        B_CHECK(get_buf(ctx, "sl_midx", m, &idx));
        for (int pass = 0; pass < 2; ++pass) {
            const int64_t cnt = pass == 0 ? P.G : P.nch;
            multi_chunk_flags_kernel<<<grid_for(ctx, cnt, T), T, 0, s>>>(
                P.grp_ch, pass == 0 ? nullptr : p_ch_grp, cnt, flag);
            B_LAUNCHED();
            B_CHECK(cub_exclusive_sum(ctx, flag, idx, cnt));
            int hv[2];
            B_CHECK(sync_read_int(ctx, idx + (cnt - 1), 1, &hv[0]));
            B_CHECK(sync_read_int(ctx, flag + (cnt - 1), 1, &hv[1]));
            const int total = hv[0] + hv[1];
            int32_t* list;
            B_CHECK(get_buf(ctx, pass == 0 ? "sl_mgroups" : "sl_mchunks", total, &list));
            compact_kernel<<<grid_for(ctx, cnt, T), T, 0, s>>>(flag, idx, cnt, list);
            B_LAUNCHED();
            if (pass == 0) {
                multi_groups = list;
                n_multi_groups = total;
            } else {
                multi_chunks = list;
                n_multi_chunks = total;
            }
        }
    }
    // ---- input norms and stop thresholds
    const int gN = grid_for(ctx, (n + RB - 1) / RB, 1, 8);
    double *pw, *pu;
    B_CHECK(get_buf(ctx, "sl_pw", static_cast<size_t>(gN) * C, &pw));
    B_CHECK(get_buf(ctx, "sl_pu", static_cast<size_t>(gN) * C, &pu));
    slope_norms_kernel<<<gN, C * RB, 0, s>>>(R, w, n, C, RB, pw, pu);
    B_LAUNCHED();
    std::vector<double> hpw(static_cast<size_t>(gN) * C), hpu(static_cast<size_t>(gN) * C);
    B_TRY(cudaMemcpyAsync(hpw.data(), pw, sizeof(double) * hpw.size(), cudaMemcpyDeviceToHost, s));
    B_TRY(cudaMemcpyAsync(hpu.data(), pu, sizeof(double) * hpu.size(), cudaMemcpyDeviceToHost, s));
    B_TRY(cudaStreamSynchronize(s));
    std::vector<double> vw(C, 0.0), vu(C, 0.0), thr(C);
    for (int b = 0; b < gN; ++b)
        for (int c = 0; c < C; ++c) {
            vw[c] += hpw[static_cast<size_t>(b) * C + c];
            vu[c] += hpu[static_cast<size_t>(b) * C + c];
        }
    const double ti = std::max(tol_eff(o), 0.0) * kSlopeTolFactor;
    for (int c = 0; c < C; ++c) thr[c] = ti * ti * vw[c];
    // scalars: thr, gamma, beta, nu, alpha [C] each; active [C]; done
    double* sc;
    int *active, *done;
    B_CHECK(get_buf(ctx, "sl_scal", static_cast<size_t>(5) * C, &sc));
    B_CHECK(get_buf(ctx, "sl_active", C, &active));
    B_CHECK(get_buf(ctx, "sl_done", 1, &done));
    double *d_thr = sc, *gamma = sc + C, *beta = sc + 2 * C, *nu = sc + 3 * C, *alpha = sc + 4 * C;
    B_TRY(cudaMemcpyAsync(d_thr, thr.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s));
    // finalize partials: slot i for cg[i], slot ncg for the primary (Schur form)
    int stride = 1;
    for (int d = 0; d < ndt; ++d) stride = std::max(stride, fin_grid[d]);
    double *pg, *pn, *pq;
    B_CHECK(get_buf(ctx, "sl_pg", static_cast<size_t>(ndt + 1) * stride * C, &pg));
    B_CHECK(get_buf(ctx, "sl_pn", static_cast<size_t>(ndt + 1) * stride * C, &pn));
    const int gG = gN;
    const int gS = schur ? grid_for(ctx, static_cast<int64_t>(dims[p].nch) * 32, T, 16) : 0;
    const int gF = n_multi_chunks ? grid_for(ctx, static_cast<int64_t>(n_multi_chunks) * 32, T, 16) : 0;
    double* pq2;
    B_CHECK(get_buf(ctx, "sl_pq", static_cast<size_t>(std::max(gG, gS)) * C, &pq));
    B_CHECK(get_buf(ctx, "sl_pq2", static_cast<size_t>(std::max(gF, 1)) * C, &pq2));
    setup_scope.reset();
    B_TRY(cudaEventRecord(e1, s));
    // algorithmic bytes per launch (profile categories)
    const double wb = w ? 8.0 : 0.0;
    double gather_bytes = 8.0 * n * C + wb * n;
    for (int d : cg)
        if (d < nd)
            gather_bytes += 4.0 * n + (dims[d].has_b ? 8.0 * n : 0.0) +
                            8.0 * dims[d].G * dims[d].nb * C;
    if (gi) gather_bytes += 16.0 * n + 4.0 * gi->E + 8.0 * gi->I * C;
    auto seg_bytes = [&](int d, bool update, bool write) {
        const SlopeDim& D = dims[d];
        const double pos = d == nd ? static_cast<double>(gi->E) : static_cast<double>(n);
        return pos * (8.0 * C * (update ? 2 : 1) + (write ? 8.0 * C : 0.0) + wb +
                      (D.has_b ? 8.0 : 0.0) + (D.perm ? 4.0 : 0.0)) +
               D.nch * (8.0 + 8.0 * D.nb * C);
    };
    auto fin_bytes = [&](int d) {
        const SlopeDim& D = dims[d];
        return D.nch * 8.0 * D.nb * C + D.G * (4.0 + 24.0 + 8.0 * D.nb * C);
    };

    // ---- iteration pieces
    const int CW = C <= 32 ? 1 : C <= 64 ? 2 : C <= 128 ? 4 : 8;
    // chunk sums of w x and w z x over dim d's groups, x = R - alpha Q (update)
    // or the rows of X (X given); the writer stores the updated residual
    auto segment = [&](int d, bool update, const double* X) -> int {
        SlopeSegArgs a{};
        a.d = dims[d];
        a.C = C;
        a.slots = CW == 1 ? 32 / C : 1;
        a.R = X ? const_cast<double*>(X) : R;
        a.Q = !X && update && writer >= 0 ? Q : nullptr;  // else R was updated first
        a.alpha = alpha;
        a.w = w;
        a.write = !X && update && d == writer;
        const int g = grid_for(ctx, static_cast<int64_t>(dims[d].nch) * 32, T, 16);
        ProfScope ps(ctx, B200FE_PROF_PASS, seg_bytes(d, a.Q != nullptr, a.write != 0));
        if (CW == 1) slope_segment_kernel<1><<<g, T, 0, s>>>(a);
        else if (CW == 2) slope_segment_kernel<2><<<g, T, 0, s>>>(a);
        else if (CW == 4) slope_segment_kernel<4><<<g, T, 0, s>>>(a);
        else slope_segment_kernel<8><<<g, T, 0, s>>>(a);
        B_LAUNCHED();
        return B200FE_OK;
    };
    auto finalize = [&](int d, int slot) -> int {
        ProfScope ps(ctx, B200FE_PROF_FINALIZE, fin_bytes(d));
        if (n_big[d] > 0) {
            const int64_t warps = static_cast<int64_t>(n_big[d]) * dims[d].nb * C;
            slope_big_reduce_kernel<<<grid_for(ctx, warps * 32, T, 16), T, 0, s>>>(
                dims[d], big_list[d], n_big[d], C);
            B_LAUNCHED();
        }
        slope_finalize_kernel<<<fin_grid[d], C * RB, 0, s>>>(
            dims[d], C, RB, pg + static_cast<size_t>(slot) * stride * C,
            pn + static_cast<size_t>(slot) * stride * C);
        B_LAUNCHED();
        return B200FE_OK;
    };
    // X -= its W-projection on the primary groups' bases (Schur form), with
    // partials of x' W x into pq when dots is set
    auto project = [&](double* X, bool dots) -> int {
        B_CHECK(segment(p, false, X));
        B_CHECK(finalize(p, ncg));  // zv of the primary = M_g^-1 B_g' W x
        ProfScope ps(ctx, B200FE_PROF_GATHER, n * (16.0 * C + 4.0 + wb + (dims[p].has_b ? 8.0 : 0.0)) +
                                                   8.0 * dims[p].G * dims[p].nb * C);
        slope_project_kernel<<<gG, C * RB, 0, s>>>(X, dims[p], w, n, C, RB, dots ? pq : nullptr);
        B_LAUNCHED();
        return B200FE_OK;
    };
    auto gradient = [&](bool update, bool init) -> int {
        if (update && writer < 0) {
            ProfScope ps(ctx, B200FE_PROF_VECTOR, 24.0 * n * C);
            slope_update_kernel<<<grid_for(ctx, n * C, T), T, 0, s>>>(R, Q, alpha, n, C);
            B_LAUNCHED();
        }
        for (int d : cg) B_CHECK(segment(d, update, nullptr));
        for (int i = 0; i < ncg; ++i) B_CHECK(finalize(cg[i], i));
        SlopeBetaArgs b{};
        b.nd = ncg;
        b.C = C;
        for (int i = 0; i < ncg; ++i) b.grid[i] = fin_grid[cg[i]];
        b.stride = stride;
        b.part_g = pg;
        b.part_n = pn;
        b.thr = d_thr;
        b.gamma = gamma;
        b.beta = beta;
        b.nu = nu;
        b.active = active;
        b.done = done;
        b.init = init ? 1 : 0;
        double vb = 0.0;
        for (int d = 0; d < ndt; ++d) vb += 24.0 * dims[d].G * dims[d].nb * C;
        ProfScope ps(ctx, B200FE_PROF_VECTOR, vb);
        slope_beta_kernel<<<1, T, 0, s>>>(b);
        B_LAUNCHED();
        for (int d = 0; d < ndt; ++d) {
            if (schur && d == p) continue;
            const int64_t tot = static_cast<int64_t>(dims[d].G) * dims[d].nb * C;
            slope_direction_kernel<<<grid_for(ctx, tot, T), T, 0, s>>>(dims[d], C, beta);
            B_LAUNCHED();
        }
        return B200FE_OK;
    };
    SlopeGatherArgs ga{};
    ga.nd = 0;
    for (int d = 0; d < nd; ++d)
        if (!(schur && d == p)) ga.dim[ga.nd++] = dims[d];
    ga.n = n;
    ga.C = C;
    ga.RB = RB;
    ga.w = w;
    ga.Q = Q;
    ga.part = pq;
    if (gi) {
        int32_t *rb, *re;
        B_CHECK(get_buf(ctx, "sl_gi_rb", n, &rb));
        B_CHECK(get_buf(ctx, "sl_gi_re", n, &re));
        row_edges_kernel<<<grid_for(ctx, n, T), T, 0, s>>>(gi->gptr, pord, n, rb, re);
        B_LAUNCHED();
        ga.has_gi = 1;
        ga.gi.beg = rb;
        ga.gi.end = re;
        ga.gi.ind = gi->gind;
        ga.gi.scale = dims[nd].z;
        ga.gi.p = dims[nd].p;
    }

    // Schur form: Q = (I - P_p) D_r p, fused for single-chunk primary groups
    SchurGatherArgs sga{};
    if (schur) {
        sga.nd = 0;
        for (int d : cg) sga.dim[sga.nd++] = dims[d];
        const SlopeDim& P = dims[p];
        sga.ch_beg = P.ch_beg;
        sga.ch_end = P.ch_end;
        sga.ch_grp = p_ch_grp;
        sga.grp_ch = P.grp_ch;
        sga.minv_p = P.minv;
        sga.z_p = P.z;
        sga.p_has_a = P.has_a;
        sga.p_has_b = P.has_b;
        sga.p_nb = P.nb;
        sga.nch = P.nch;
        sga.part_p = P.part;
        sga.n = n;
        sga.C = C;
        sga.slots = CW == 1 ? 32 / C : 1;
        sga.w = w;
        sga.Q = Q;
        sga.dpart = pq;
    }
    auto schur_gather = [&]() -> int {
        {
            ProfScope ps(ctx, B200FE_PROF_GATHER, gather_bytes);
            if (CW == 1) {
                if (sga.nd == 1) schur_gather_kernel<1, 1><<<gS, T, 0, s>>>(sga);
                else if (sga.nd == 2) schur_gather_kernel<1, 2><<<gS, T, 0, s>>>(sga);
                else if (sga.nd == 3) schur_gather_kernel<1, 3><<<gS, T, 0, s>>>(sga);
                else schur_gather_kernel<1, 0><<<gS, T, 0, s>>>(sga);
            } else if (CW == 2) {
                schur_gather_kernel<2, 0><<<gS, T, 0, s>>>(sga);
            } else if (CW == 4) {
                schur_gather_kernel<4, 0><<<gS, T, 0, s>>>(sga);
            } else {
                schur_gather_kernel<8, 0><<<gS, T, 0, s>>>(sga);
            }
            B_LAUNCHED();
        }
        if (n_multi_chunks) {
            ProfScope ps(ctx, B200FE_PROF_FINALIZE, 0.0);
            schur_fix_mean_kernel<<<grid_for(ctx, static_cast<int64_t>(n_multi_groups) * C, T), T, 0, s>>>(
                multi_groups, n_multi_groups, dims[p], C);
            B_LAUNCHED();
            const int S = CW == 1 ? 32 / C : 1;
            const SlopeDim& P = dims[p];
            if (CW == 1)
                schur_fix_apply_kernel<1><<<gF, T, 0, s>>>(multi_chunks, n_multi_chunks, p_ch_grp, P, w,
                                                            Q, C, S, pq2);
            else if (CW == 2)
                schur_fix_apply_kernel<2><<<gF, T, 0, s>>>(multi_chunks, n_multi_chunks, p_ch_grp, P, w,
                                                            Q, C, S, pq2);
            else if (CW == 4)
                schur_fix_apply_kernel<4><<<gF, T, 0, s>>>(multi_chunks, n_multi_chunks, p_ch_grp, P, w,
                                                            Q, C, S, pq2);
            else
                schur_fix_apply_kernel<8><<<gF, T, 0, s>>>(multi_chunks, n_multi_chunks, p_ch_grp, P, w,
                                                            Q, C, S, pq2);
            B_LAUNCHED();
        }
        return B200FE_OK;
    };

    if (schur) B_CHECK(project(R, false));
    B_CHECK(gradient(false, true));
    const int ci = std::max(1, o.check_interval);
    const int max_it = o.max_iter > 0 ? o.max_iter : 10000;
    int it = 0, hd = 0;
    B_CHECK(sync_read_int(ctx, done, 1, &hd));
    while (!hd && it < max_it) {
        const int steps = std::min(ci, max_it - it);
        for (int k = 0; k < steps; ++k) {
            if (schur) {
                B_CHECK(schur_gather());
            } else {
                ProfScope ps(ctx, B200FE_PROF_GATHER, gather_bytes);
                if (ga.nd == 1) slope_gather_kernel<1><<<gG, C * RB, 0, s>>>(ga);
                else if (ga.nd == 2) slope_gather_kernel<2><<<gG, C * RB, 0, s>>>(ga);
                else if (ga.nd == 3) slope_gather_kernel<3><<<gG, C * RB, 0, s>>>(ga);
                else slope_gather_kernel<0><<<gG, C * RB, 0, s>>>(ga);
                B_LAUNCHED();
            }
            {
                ProfScope ps(ctx, B200FE_PROF_VECTOR, 0.0);
                slope_alpha_kernel<<<1, T, 0, s>>>(pq, schur ? gS : gG, pq2, schur ? gF : 0, C,
                                                   gamma, active, alpha);
                B_LAUNCHED();
            }
            B_CHECK(gradient(true, false));
        }
        it += steps;
        B_CHECK(sync_read_int(ctx, done, 1, &hd));
    }
    // Schur form: the primary's share of the certificate, ||D_p' W r||^2
    std::vector<double> nu_p(C, 0.0);
    if (schur) {
        B_CHECK(segment(p, false, R));
        B_CHECK(finalize(p, ncg));
        std::vector<double> hq(static_cast<size_t>(fin_grid[p]) * C);
        B_TRY(cudaMemcpyAsync(hq.data(), pn + static_cast<size_t>(ncg) * stride * C,
                              sizeof(double) * hq.size(), cudaMemcpyDeviceToHost, s));
        B_TRY(cudaStreamSynchronize(s));
        for (int b = 0; b < fin_grid[p]; ++b)
            for (int c = 0; c < C; ++c) nu_p[c] += hq[static_cast<size_t>(b) * C + c];
    }
    {
        ProfScope ps(ctx, B200FE_PROF_FINAL, 16.0 * n * C + (pord ? 4.0 * n : 0.0));
        slope_store_kernel<<<grid_for(ctx, n * C, T), T, 0, s>>>(R, pord, n, C, d_out);
        B_LAUNCHED();
    }
    std::vector<double> hs(C);
    B_TRY(cudaMemcpyAsync(hs.data(), gamma, sizeof(double) * C, cudaMemcpyDeviceToHost, s));
    std::vector<double> hnu(C);
    B_TRY(cudaMemcpyAsync(hnu.data(), nu, sizeof(double) * C, cudaMemcpyDeviceToHost, s));
    B_TRY(cudaEventRecord(e2, s));
    B_TRY(cudaEventSynchronize(e2));
    res->setup_ms = elapsed_ms(e0, e1);
    res->solve_ms = elapsed_ms(e1, e2);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (ctx->profiling) {
        for (const auto& pr : ctx->prof) {
            if (pr.cat < 0 || pr.cat >= B200FE_PROF_CATEGORIES) continue;
            res->prof_ms[pr.cat] += elapsed_ms(pr.a, pr.b);
            res->prof_bytes[pr.cat] += pr.bytes;
            res->prof_launches[pr.cat] += 1;
        }
        ctx->prof.clear();
        ctx->profiling = false;
    }
    // ---- result fields
    const double opn = std::sqrt(std::max(0.0, op_norm2));
    double abs_res = 0.0, abs_rel = 0.0, rel = 0.0;
    for (int c = 0; c < C; ++c) {
        const double ab = std::sqrt(std::max(0.0, hnu[c] + nu_p[c]));
        const double scl = opn * std::sqrt(std::max(0.0, vu[c]));
        double r = 0.0;
        if (scl > 0.0) r = ab / scl;
        else if (ab > 0.0) r = std::numeric_limits<double>::max();
        abs_res = std::max(abs_res, ab);
        abs_rel = std::max(abs_rel, r);
        if (vw[c] > 0.0) rel = std::max(rel, std::sqrt(std::max(0.0, hs[c]) / vw[c]));
    }
    res->iterations = it;
    res->outer_iterations = 1;
    res->converged = hd ? 1 : 0;
    res->abs_residual = abs_res;
    res->abs_residual_rel = abs_rel;
    res->rel_residual = rel;
    res->primary_dim = p;
    for (int d = 0; d < nd; ++d) res->num_levels_present[d] = present[d];
    const double limit = std::max(8.0 * std::max(0.0, tol_eff(o)),
                                  64.0 * std::numeric_limits<double>::epsilon());
    res->precision_certified = res->converged && (o.certify ? abs_rel <= limit : 1);
    return res->converged ? B200FE_OK : B200FE_NOT_CONVERGED;
}

int check_slopes(b200fe_context* ctx, int cols, int num_dims) {
    if (cols > kSlopeMaxCols) {
        ctx->err = "the slope absorber takes at most 256 columns";
        return B200FE_INVALID_ARG;
    }
    if (num_dims < 1) {
        ctx->err = "need at least one FE dimension";
        return B200FE_INVALID_ARG;
    }
    return B200FE_OK;
}

}  // namespace

extern "C" {

int b200fe_absorb_slopes_device(b200fe_context* ctx, const double* d_v, int64_t n, int cols,
                                int num_dims, const int32_t* const* d_group_ids,
                                const int32_t* num_groups, const double* const* d_slope_values,
                                const unsigned char* slope_has_intercept, const double* d_weights,
                                const b200fe_options* opts, double* d_out, b200fe_result* res,
                                void* stream) {
    b200fe_result local;
    b200fe_result* r = res ? res : &local;
    clear_result(r);
    int rc = check_common(ctx, n, cols, num_dims, num_groups);
    if (rc != B200FE_OK) return r->status = rc;
    if (!d_v || !d_out || !d_group_ids) {
        ctx->err = "null pointer argument";
        return r->status = B200FE_INVALID_ARG;
    }
    rc = check_slopes(ctx, cols, num_dims);
    if (rc != B200FE_OK) return r->status = rc;
    const double* z[B200FE_MAX_DIMS] = {nullptr};
    for (int d = 0; d < num_dims; ++d) {
        if (!d_group_ids[d]) {
            ctx->err = "null group id array";
            return r->status = B200FE_INVALID_ARG;
        }
        z[d] = d_slope_values ? d_slope_values[d] : nullptr;
    }
    b200fe_options o;
    if (opts) o = *opts;
    else b200fe_default_options(&o);
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return r->status = B200FE_UNAVAILABLE;
    }
    const cudaStream_t own = ctx->stream;
    if (stream) ctx->stream = static_cast<cudaStream_t>(stream);
    const long long l0 = ctx->launches, c0 = ctx->lib_calls;
    rc = slopes_device_impl(ctx, d_v, n, cols, num_dims, d_group_ids, num_groups, z,
                            slope_has_intercept, d_weights, nullptr, o, d_out, r);
    ctx->stream = own;
    r->kernel_launches = ctx->launches - l0;
    r->library_calls = ctx->lib_calls - c0;
    return r->status = rc;
}

int b200fe_absorb_slopes(b200fe_context* ctx, const double* y, const double* X, int64_t n, int k,
                         int num_dims, const int32_t* const* group_ids, const int32_t* num_groups,
                         const double* const* slope_values, const unsigned char* slope_has_intercept,
                         const double* weights, const b200fe_options* opts, double* y_out,
                         double* X_out, b200fe_result* res) {
    b200fe_result local;
    b200fe_result* r = res ? res : &local;
    clear_result(r);
    int rc = check_common(ctx, n, k + 1, num_dims, num_groups);
    if (rc != B200FE_OK) return r->status = rc;
    if (!y || !y_out || (k > 0 && (!X || !X_out)) || !group_ids) {
        ctx->err = "null pointer argument";
        return r->status = B200FE_INVALID_ARG;
    }
    rc = check_slopes(ctx, k + 1, num_dims);
    if (rc != B200FE_OK) return r->status = rc;
    for (int d = 0; d < num_dims; ++d)
        if (!group_ids[d]) {
            ctx->err = "null group id array";
            return r->status = B200FE_INVALID_ARG;
        }
    b200fe_options o;
    if (opts) o = *opts;
    else b200fe_default_options(&o);
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return r->status = B200FE_UNAVAILABLE;
    }
    const cudaStream_t s = ctx->stream;
    const long long l0 = ctx->launches, c0 = ctx->lib_calls;
    const int cols = k + 1;
    auto run = [&]() -> int {
        double *dv, *dout, *dw = nullptr;
        B_CHECK(get_buf(ctx, "io_v", static_cast<size_t>(n) * cols, &dv));
        B_CHECK(get_buf(ctx, "io_out", static_cast<size_t>(n) * cols, &dout));
        int32_t* dg[B200FE_MAX_DIMS] = {nullptr};
        double* dz[B200FE_MAX_DIMS] = {nullptr};
        for (int d = 0; d < num_dims; ++d) {
            B_CHECK(get_buf(ctx, "io_g" + std::to_string(d), n, &dg[d]));
            if (slope_values && slope_values[d])
                B_CHECK(get_buf(ctx, "io_z" + std::to_string(d), n, &dz[d]));
        }
        if (weights) B_CHECK(get_buf(ctx, "io_w", n, &dw));
        cudaEvent_t h0, h1, d0, d1;
        B_TRY(cudaEventCreate(&h0));
        B_TRY(cudaEventCreate(&h1));
        B_TRY(cudaEventCreate(&d0));
        B_TRY(cudaEventCreate(&d1));
        B_TRY(cudaEventRecord(h0, s));
        for (int d = 0; d < num_dims; ++d) {
            B_TRY(cudaMemcpyAsync(dg[d], group_ids[d], sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
            if (dz[d])
                B_TRY(cudaMemcpyAsync(dz[d], slope_values[d], sizeof(double) * n, cudaMemcpyHostToDevice, s));
        }
        if (weights) B_TRY(cudaMemcpyAsync(dw, weights, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemcpyAsync(dv, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(dv + n, X, sizeof(double) * n * k, cudaMemcpyHostToDevice, s));
        B_TRY(cudaEventRecord(h1, s));
        const double* zc[B200FE_MAX_DIMS];
        for (int d = 0; d < B200FE_MAX_DIMS; ++d) zc[d] = dz[d];
        int rc2 = slopes_device_impl(ctx, dv, n, cols, num_dims, dg, num_groups, zc,
                                     slope_has_intercept, dw, nullptr, o, dout, r);
        if (rc2 != B200FE_OK && rc2 != B200FE_NOT_CONVERGED) return rc2;
        B_TRY(cudaEventRecord(d0, s));
        B_TRY(cudaMemcpyAsync(y_out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(X_out, dout + n, sizeof(double) * n * k, cudaMemcpyDeviceToHost, s));
        B_TRY(cudaEventRecord(d1, s));
        B_TRY(cudaEventSynchronize(d1));
        r->h2d_ms = elapsed_ms(h0, h1);
        r->d2h_ms = elapsed_ms(d0, d1);
        cudaEventDestroy(h0);
        cudaEventDestroy(h1);
        cudaEventDestroy(d0);
        cudaEventDestroy(d1);
        return rc2;
    };
    rc = run();
    r->kernel_launches = ctx->launches - l0;
    r->library_calls = ctx->lib_calls - c0;
    return r->status = rc;
}


int b200fe_absorb_group_individual(b200fe_context* ctx, const double* y, const double* X,
                                   int64_t n, int k, int num_dims,
                                   const int32_t* const* group_ids, const int32_t* num_groups,
                                   const b200fe_group_individual* gi, const double* weights,
                                   const b200fe_options* opts, double* y_out, double* X_out,
                                   b200fe_result* res) {
    b200fe_result local;
    b200fe_result* r = res ? res : &local;
    clear_result(r);
    int rc = check_common(ctx, n, k + 1, num_dims, num_groups);
    if (rc != B200FE_OK) return r->status = rc;
    if (!y || !y_out || (k > 0 && (!X || !X_out)) || (num_dims > 0 && !group_ids) || !gi) {
        ctx->err = "null pointer argument";
        return r->status = B200FE_INVALID_ARG;
    }
    if (k + 1 > kSlopeMaxCols) {
        ctx->err = "the group/individual absorber takes at most 256 columns";
        return r->status = B200FE_INVALID_ARG;
    }
    for (int d = 0; d < num_dims; ++d)
        if (!group_ids[d]) {
            ctx->err = "null group id array";
            return r->status = B200FE_INVALID_ARG;
        }
    // the structure's CSR arrays index each other: check every range on the host
    const int32_t I = gi->num_individuals;
    const int64_t E = gi->num_edges;
    if (I <= 0 || E < 0 || E >= (int64_t(1) << 31) - 1 || !gi->group_ptr || !gi->individual_ptr ||
        !gi->group_scale || (E > 0 && (!gi->group_individual || !gi->individual_group))) {
        ctx->err = "invalid group/individual structure";
        return r->status = B200FE_INVALID_ARG;
    }
    auto csr_ok = [](const int32_t* ptr, int64_t rows, int64_t edges) {
        if (ptr[0] != 0 || ptr[rows] != edges) return false;
        for (int64_t i = 0; i < rows; ++i)
            if (ptr[i + 1] < ptr[i]) return false;
        return true;
    };
    bool ok = csr_ok(gi->group_ptr, n, E) && csr_ok(gi->individual_ptr, I, E);
    for (int64_t e = 0; ok && e < E; ++e)
        ok = gi->group_individual[e] >= 0 && gi->group_individual[e] < I &&
             gi->individual_group[e] >= 0 && gi->individual_group[e] < n;
    if (!ok) {
        ctx->err = "invalid group/individual structure (pointer arrays or ids out of range)";
        return r->status = B200FE_INVALID_ARG;
    }
    b200fe_options o;
    if (opts) o = *opts;
    else b200fe_default_options(&o);
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return r->status = B200FE_UNAVAILABLE;
    }
    const cudaStream_t s = ctx->stream;
    const long long l0 = ctx->launches, c0 = ctx->lib_calls;
    const int cols = k + 1;
    auto run = [&]() -> int {
        double *dv, *dout, *dw = nullptr, *dscale;
        int32_t *gptr, *gind, *iptr, *igrp;
        B_CHECK(get_buf(ctx, "io_v", static_cast<size_t>(n) * cols, &dv));
        B_CHECK(get_buf(ctx, "io_out", static_cast<size_t>(n) * cols, &dout));
        B_CHECK(get_buf(ctx, "io_gptr", static_cast<size_t>(n) + 1, &gptr));
        B_CHECK(get_buf(ctx, "io_gind", E, &gind));
        B_CHECK(get_buf(ctx, "io_iptr", static_cast<size_t>(I) + 1, &iptr));
        B_CHECK(get_buf(ctx, "io_igrp", E, &igrp));
        B_CHECK(get_buf(ctx, "io_gscale", n, &dscale));
        int32_t* dg[B200FE_MAX_DIMS] = {nullptr};
        for (int d = 0; d < num_dims; ++d) B_CHECK(get_buf(ctx, "io_g" + std::to_string(d), n, &dg[d]));
        if (weights) B_CHECK(get_buf(ctx, "io_w", n, &dw));
        cudaEvent_t h0, h1, d0, d1;
        B_TRY(cudaEventCreate(&h0));
        B_TRY(cudaEventCreate(&h1));
        B_TRY(cudaEventCreate(&d0));
        B_TRY(cudaEventCreate(&d1));
        B_TRY(cudaEventRecord(h0, s));
        for (int d = 0; d < num_dims; ++d)
            B_TRY(cudaMemcpyAsync(dg[d], group_ids[d], sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        if (weights) B_TRY(cudaMemcpyAsync(dw, weights, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemcpyAsync(gptr, gi->group_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemcpyAsync(iptr, gi->individual_ptr, sizeof(int32_t) * (static_cast<size_t>(I) + 1),
                              cudaMemcpyHostToDevice, s));
        if (E > 0) {
            B_TRY(cudaMemcpyAsync(gind, gi->group_individual, sizeof(int32_t) * E, cudaMemcpyHostToDevice, s));
            B_TRY(cudaMemcpyAsync(igrp, gi->individual_group, sizeof(int32_t) * E, cudaMemcpyHostToDevice, s));
        }
        B_TRY(cudaMemcpyAsync(dscale, gi->group_scale, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemcpyAsync(dv, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(dv + n, X, sizeof(double) * n * k, cudaMemcpyHostToDevice, s));
        B_TRY(cudaEventRecord(h1, s));
        const double* zc[B200FE_MAX_DIMS] = {nullptr};
        GiDev g{I, E, gptr, gind, iptr, igrp, dscale};
        int rc2 = slopes_device_impl(ctx, dv, n, cols, num_dims, dg, num_groups, zc, nullptr, dw,
                                     &g, o, dout, r);
        if (rc2 != B200FE_OK && rc2 != B200FE_NOT_CONVERGED) return rc2;
        B_TRY(cudaEventRecord(d0, s));
        B_TRY(cudaMemcpyAsync(y_out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(X_out, dout + n, sizeof(double) * n * k, cudaMemcpyDeviceToHost, s));
        B_TRY(cudaEventRecord(d1, s));
        B_TRY(cudaEventSynchronize(d1));
        r->h2d_ms = elapsed_ms(h0, h1);
        r->d2h_ms = elapsed_ms(d0, d1);
        cudaEventDestroy(h0);
        cudaEventDestroy(h1);
        cudaEventDestroy(d0);
        cudaEventDestroy(d1);
        return rc2;
    };
    rc = run();
    r->kernel_launches = ctx->launches - l0;
    r->library_calls = ctx->lib_calls - c0;
    return r->status = rc;
}

}  // extern "C"
