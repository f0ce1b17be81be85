// Host orchestration and C ABI of the B200 fixed-effects absorber.
//
// Entry points are declared in include/b200fe.h.  The solver (see
// kernels.cuh for the math) runs entirely on one CUDA stream owned by the
// context; the host only reads a handful of per-column scalars between
// blocks of CG iterations.

#include "context.cuh"
#include "kernels.cuh"
#include "setup_kernels.cuh"
#include "ols_kernels.cuh"
#include "prep_kernels.cuh"
#include "sparse_kernels.cuh"
#include "pcg_kernels.cuh"
#include "ws_kernels.cuh"
#include "stream_kernels.cuh"

using namespace b200fe;
using namespace b200fe_host;

namespace {

// ---------------------------------------------------------------------------
// Structure build
// ---------------------------------------------------------------------------
// Chunk lists over groups whose items are [grp_off[g], grp_off[g+1]) (runs of
// a large dim, or nonzeros of a CSR row): chunks of at most CH items, the
// groups with several chunks ("multi" rows, summed by finalize_kernel) and
// their super-chunks (groups of more than kFinFewParts chunks: the Zipf-giant
// firm owns thousands).  Fills the chunk fields of L; L.G is set by the
// caller; buffer names end in sfx.
int build_chunks(b200fe_context* ctx, const int32_t* grp_off, int32_t CH, const std::string& sfx,
                 LargeDim& L) {
    const cudaStream_t s = ctx->stream;
    const int T256 = 256;
    // chunk list
    int32_t *nch, *ch_off, *mflag, *midx;
    B_CHECK(get_buf(ctx, "nch", static_cast<size_t>(L.G) + 1, &nch));
    B_CHECK(get_buf(ctx, "ch_off", static_cast<size_t>(L.G) + 1, &ch_off));
    B_CHECK(get_buf(ctx, "mflag", static_cast<size_t>(L.G) + 1, &mflag));
    B_CHECK(get_buf(ctx, "midx", static_cast<size_t>(L.G) + 1, &midx));
    B_TRY(cudaMemsetAsync(nch, 0, sizeof(int32_t) * (static_cast<size_t>(L.G) + 1), s));
    B_TRY(cudaMemsetAsync(mflag, 0, sizeof(int32_t) * (static_cast<size_t>(L.G) + 1), s));
    chunk_count_kernel<<<grid_for(ctx, L.G, T256), T256, 0, s>>>(grp_off, L.G, CH, nch);
    B_LAUNCHED();
    B_CHECK(cub_exclusive_sum(ctx, nch, ch_off, static_cast<int64_t>(L.G) + 1));
    multi_flag_kernel<<<grid_for(ctx, L.G, T256), T256, 0, s>>>(nch, L.G, mflag);
    B_LAUNCHED();
    B_CHECK(cub_exclusive_sum(ctx, mflag, midx, static_cast<int64_t>(L.G) + 1));
    int hc[2];
    B_CHECK(sync_read_int(ctx, ch_off + L.G, 1, &hc[0]));
    B_CHECK(sync_read_int(ctx, midx + L.G, 1, &hc[1]));
    L.nchunks = hc[0];
    L.nmulti = hc[1];
    B_CHECK(get_buf(ctx, "chunk_grp" + sfx, L.nchunks, &L.chunk_grp));
    B_CHECK(get_buf(ctx, "chunk_beg" + sfx, L.nchunks, &L.chunk_beg));
    B_CHECK(get_buf(ctx, "chunk_end" + sfx, L.nchunks, &L.chunk_end));
    B_CHECK(get_buf(ctx, "chunk_whole" + sfx, L.nchunks, &L.chunk_whole));
    B_CHECK(get_buf(ctx, "multi_grp" + sfx, L.nmulti, &L.multi_grp));
    B_CHECK(get_buf(ctx, "multi_c0" + sfx, L.nmulti, &L.multi_c0));
    B_CHECK(get_buf(ctx, "multi_c1" + sfx, L.nmulti, &L.multi_c1));
    chunk_fill_kernel<<<grid_for(ctx, L.G, T256), T256, 0, s>>>(
        grp_off, L.G, CH, ch_off, L.chunk_grp, L.chunk_beg, L.chunk_end,
        L.chunk_whole, midx, L.multi_grp, L.multi_c0, L.multi_c1);
    B_LAUNCHED();
    // super-chunks: a group with many chunks (Zipf sizes: one firm may own
    // 10%+ of the runs) has its chunk partials summed in slices of
    // kSuperParts by many lane groups before finalize adds the slices
    L.nsup = 0;
    if (L.nmulti > 0) {
        std::vector<int32_t> c0(L.nmulti), c1(L.nmulti);
        B_TRY(cudaMemcpyAsync(c0.data(), L.multi_c0, sizeof(int32_t) * L.nmulti, cudaMemcpyDeviceToHost, s));
        B_TRY(cudaMemcpyAsync(c1.data(), L.multi_c1, sizeof(int32_t) * L.nmulti, cudaMemcpyDeviceToHost, s));
        B_TRY(cudaStreamSynchronize(s));
        std::vector<int32_t> s0(L.nmulti), s1(L.nmulti), sb, se;
        for (int64_t r = 0; r < L.nmulti; ++r) {
            s0[r] = s1[r] = static_cast<int32_t>(sb.size());
            if (c1[r] - c0[r] <= kFinFewParts) continue;
            for (int32_t c = c0[r]; c < c1[r]; c += kSuperParts) {
                sb.push_back(c);
                se.push_back(std::min(c1[r], c + kSuperParts));
            }
            s1[r] = static_cast<int32_t>(sb.size());
        }
        L.nsup = static_cast<int64_t>(sb.size());
        B_CHECK(get_buf(ctx, "multi_s0" + sfx, L.nmulti, &L.multi_s0));
        B_CHECK(get_buf(ctx, "multi_s1" + sfx, L.nmulti, &L.multi_s1));
        B_CHECK(get_buf(ctx, "sup_c0" + sfx, std::max<int64_t>(L.nsup, 1), &L.sup_c0));
        B_CHECK(get_buf(ctx, "sup_c1" + sfx, std::max<int64_t>(L.nsup, 1), &L.sup_c1));
        B_TRY(cudaMemcpyAsync(L.multi_s0, s0.data(), sizeof(int32_t) * L.nmulti, cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemcpyAsync(L.multi_s1, s1.data(), sizeof(int32_t) * L.nmulti, cudaMemcpyHostToDevice, s));
        if (L.nsup > 0) {
            B_TRY(cudaMemcpyAsync(L.sup_c0, sb.data(), sizeof(int32_t) * L.nsup, cudaMemcpyHostToDevice, s));
            B_TRY(cudaMemcpyAsync(L.sup_c1, se.data(), sizeof(int32_t) * L.nsup, cudaMemcpyHostToDevice, s));
        }
        B_TRY(cudaStreamSynchronize(s));  // the host vectors leave scope
    }
    return B200FE_OK;
}

// Records of the regular tiles for the bulk-copy data passes
// (stream_kernels.cuh).  st.stream_ok stays false when a regular tile has
// more observations or segments than a stage holds.
int build_stream_meta(b200fe_context* ctx) {
    Structure& st = ctx->st;
    const cudaStream_t s = ctx->stream;
    st.stream_ok = false;
    st.stream_nreg = 0;
    if (st.ntiles <= 0) return B200FE_OK;
    int32_t *rflag, *ridx;
    int* flags;
    const size_t t1 = static_cast<size_t>(st.ntiles) + 1;
    B_CHECK(get_buf(ctx, "tmp_tile_flag", t1, &rflag));
    B_CHECK(get_buf(ctx, "tmp_tile_idx", t1, &ridx));
    B_CHECK(get_buf(ctx, "stream_flags", 4, &flags));
    B_TRY(cudaMemsetAsync(flags, 0, 4 * sizeof(int), s));
    tile_regular_flag_kernel<<<grid_for(ctx, st.ntiles + 1, 256), 256, 0, s>>>(st.ntiles, st.tile_long, rflag);
    B_LAUNCHED();
    B_CHECK(cub_exclusive_sum(ctx, rflag, ridx, static_cast<int64_t>(t1)));
    int nreg = 0;
    B_CHECK(sync_read_int(ctx, ridx + st.ntiles, 1, &nreg));
    st.stream_nreg = nreg;
    if (nreg == 0) return B200FE_OK;
    st.stream_aux_stride = stream_aux_stride(st.nL, st.SG, st.nS);
    int32_t* bsize;
    B_CHECK(get_buf(ctx, "stream_meta", 2 * static_cast<size_t>(nreg), &st.stream_meta));
    B_CHECK(get_buf(ctx, "tmp_blob_size", static_cast<size_t>(nreg) + 1, &bsize));
    B_CHECK(get_buf(ctx, "stream_boff", static_cast<size_t>(nreg) + 1, &st.stream_boff));
    B_TRY(cudaMemsetAsync(bsize + nreg, 0, sizeof(int32_t), s));
    TileMetaArgs m{};
    m.ntiles = st.ntiles;
    m.tile_seg = st.tile_seg;
    m.tile_long = st.tile_long;
    m.reg_idx = ridx;
    m.seg_off = st.seg_off;
    m.nL = st.nL;
    m.nS = st.nS;
    m.aux_stride = st.stream_aux_stride;
    for (int l = 0; l < st.nL; ++l) m.run_base[l] = st.L[l].run_base;
    m.tmeta = st.stream_meta;
    m.bsize = bsize;
    m.flags = flags;
    tile_meta_kernel<<<grid_for(ctx, st.ntiles, 256), 256, 0, s>>>(m);
    B_LAUNCHED();
    B_CHECK(cub_exclusive_sum(ctx, bsize, st.stream_boff, static_cast<int64_t>(nreg) + 1));
    int hf[2] = {0, 0}, units = 0;
    B_CHECK(sync_read_int(ctx, flags, 2, hf));
    B_CHECK(sync_read_int(ctx, st.stream_boff + nreg, 1, &units));
    if (hf[0] != 0) return B200FE_OK;
    st.stream_blob_max = hf[1];
    B_CHECK(get_buf(ctx, "stream_blob", static_cast<size_t>(std::max(units, 1)) * 16, &st.stream_blob));
    TileBlobArgs x{};
    x.nreg = nreg;
    x.tmeta = st.stream_meta;
    x.boff = st.stream_boff;
    x.seg_off = st.seg_off;
    x.inv_wp = st.inv_wp;
    x.nL = st.nL;
    for (int l = 0; l < st.nL; ++l) {
        x.run_base[l] = st.L[l].run_base;
        x.run_start[l] = st.L[l].run_start;
        x.run_dest[l] = st.L[l].run_dest;
    }
    x.run_grp0 = st.nL > 0 ? st.L[0].run_grp : nullptr;
    x.sid = st.sid;
    x.nS = st.nS;
    for (int j = 0; j < st.nS; ++j) x.sG[j] = st.sG[j];
    x.aux_stride = st.stream_aux_stride;
    x.blob = st.stream_blob;
    tile_blob_kernel<<<static_cast<int>((nreg + kBlobWarps - 1) / kBlobWarps), kBlobWarps * 32, 0, s>>>(x);
    B_LAUNCHED();
    st.stream_ok = true;
    return B200FE_OK;
}

// The explicit S_ff of the one large dim (see sparse_kernels.cuh).  Leaves
// st.sparse false (run-level matvec) when a segment has more than
// kSparseMaxRuns runs or the contributions would exceed eight per run.
int build_sparse_block(b200fe_context* ctx) {
    Structure& st = ctx->st;
    const cudaStream_t s = ctx->stream;
    const int T256 = 256;
    const int32_t Gp = st.G[st.p];
    LargeDim& L = st.L[0];
    int32_t *count, *flag;
    unsigned long long* total;
    B_CHECK(get_buf(ctx, "sp_count", static_cast<size_t>(Gp) + 1, &count));
    B_CHECK(get_buf(ctx, "sp_flag", 4, &flag));
    B_CHECK(get_buf(ctx, "sp_total", 1, &total));
    B_TRY(cudaMemsetAsync(flag, 0, sizeof(int32_t), s));
    B_TRY(cudaMemsetAsync(total, 0, sizeof(unsigned long long), s));
    B_TRY(cudaMemsetAsync(count + Gp, 0, sizeof(int32_t), s));
    sparse_pair_count_kernel<<<grid_for(ctx, Gp, T256), T256, 0, s>>>(Gp, L.run_base, L.run_grp,
                                                                        count, flag, total);
    B_LAUNCHED();
    unsigned long long htot = 0;
    int hflag = 0;
    B_TRY(cudaMemcpyAsync(&htot, total, sizeof(htot), cudaMemcpyDeviceToHost, s));
    B_CHECK(sync_read_int(ctx, flag, 1, &hflag));  // synchronises htot too
    const unsigned long long cap = std::min<unsigned long long>(
        8ull * static_cast<unsigned long long>(L.nruns) + (1ull << 20), (1ull << 31) - 1);
    if (hflag || htot > cap) return B200FE_OK;
    st.sp_pairs = static_cast<int64_t>(htot);
    st.sp.G = L.G;
    const int64_t np = std::max<int64_t>(st.sp_pairs, 1);
    int32_t* off;
    B_CHECK(get_buf(ctx, "sp_off", static_cast<size_t>(Gp) + 1, &off));
    B_CHECK(cub_exclusive_sum(ctx, count, off, static_cast<int64_t>(Gp) + 1));
    unsigned long long *k_in, *k_out;
    double *v_in, *v_out;
    B_CHECK(get_buf(ctx, "sp_kin", np, &k_in));
    B_CHECK(get_buf(ctx, "sp_kout", np, &k_out));
    B_CHECK(get_buf(ctx, "sp_vin", np, &v_in));
    B_CHECK(get_buf(ctx, "sp_vout", np, &v_out));
    int32_t *ustart, *urow;
    if (st.sp_pairs > 0) {
        sparse_pair_fill_kernel<<<grid_for(ctx, Gp, T256), T256, 0, s>>>(
            Gp, L.run_base, L.run_grp, L.cw_run, st.inv_wp, count, off, L.G, k_in, v_in);
        B_LAUNCHED();
        // stable sort by (row, column): equal keys keep segment order
        const unsigned long long gmax = static_cast<unsigned long long>(L.G) * L.G;
        int eb = 1;
        while (eb < 63 && (1ull << eb) < gmax) ++eb;
        size_t tmp = 0;
        B_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in, k_out, v_in, v_out, st.sp_pairs,
                                              0, eb, s));
        void* t;
        B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
        B_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, k_in, k_out, v_in, v_out, st.sp_pairs, 0, eb,
                                              s));
        ++ctx->lib_calls;
        int32_t *flags, *uid;
        B_CHECK(get_buf(ctx, "sp_flags", np, &flags));
        B_CHECK(get_buf(ctx, "sp_uid", np, &uid));
        sparse_key_flags_kernel<<<grid_for(ctx, st.sp_pairs, T256), T256, 0, s>>>(k_out, st.sp_pairs,
                                                                                   flags);
        B_LAUNCHED();
        B_CHECK(cub_inclusive_sum(ctx, flags, uid, st.sp_pairs));
        int nnz = 0;
        B_CHECK(sync_read_int(ctx, uid + (st.sp_pairs - 1), 1, &nnz));
        st.sp_nnz = nnz;
        B_CHECK(get_buf(ctx, "sp_ustart", static_cast<size_t>(nnz) + 1, &ustart));
        B_CHECK(get_buf(ctx, "sp_urow", nnz, &urow));
        B_CHECK(get_buf(ctx, "sp_col", nnz, &st.sp_col));
        sparse_unique_fill_kernel<<<grid_for(ctx, st.sp_pairs, T256), T256, 0, s>>>(
            k_out, st.sp_pairs, flags, uid, L.G, ustart, urow, st.sp_col);
        B_LAUNCHED();
        int32_t* long_list;
        B_CHECK(get_buf(ctx, "sp_val64", nnz, &st.sp_val64));
        B_CHECK(get_buf(ctx, "sp_val32", nnz, &st.sp_val32));
        B_CHECK(get_buf(ctx, "sp_long", nnz, &long_list));
        B_TRY(cudaMemsetAsync(flag + 1, 0, sizeof(int32_t), s));  // long-list counter
        sparse_merge_kernel<<<grid_for(ctx, nnz, T256), T256, 0, s>>>(nnz, ustart, v_out, st.sp_val64,
                                                                     long_list, flag + 1);
        B_LAUNCHED();
        sparse_merge_long_kernel<<<ctx->num_sms * 4, 256, 0, s>>>(long_list, flag + 1, ustart, v_out,
                                                                  st.sp_val64);
        B_LAUNCHED();
        to_float_kernel<<<grid_for(ctx, nnz, T256), T256, 0, s>>>(st.sp_val64, nnz, st.sp_val32);
        B_LAUNCHED();
    } else {
        st.sp_nnz = 0;
        B_CHECK(get_buf(ctx, "sp_urow", 1, &urow));
        B_CHECK(get_buf(ctx, "sp_col", 1, &st.sp_col));
        B_CHECK(get_buf(ctx, "sp_val64", 1, &st.sp_val64));
        B_CHECK(get_buf(ctx, "sp_val32", 1, &st.sp_val32));
    }
    // CSR row offsets over the large dim's levels (rows without movers are empty)
    B_CHECK(get_buf(ctx, "sp_row_off", static_cast<size_t>(L.G) + 1, &st.sp_row_off));
    segment_offsets_kernel<<<grid_for(ctx, st.sp_nnz + 1, T256), T256, 0, s>>>(urow, st.sp_nnz, L.G,
                                                                              st.sp_row_off);
    B_LAUNCHED();
    B_CHECK(build_chunks(ctx, st.sp_row_off, kSparseChunk, "_sp", st.sp));
    // work lists of the persistent PCG: short rows, long rows and their chunks
    {
        const size_t g1 = static_cast<size_t>(L.G) + 1;
        int32_t *is_short, *is_long, *nch, *short_idx, *long_idx, *chunk_off, *is_huge, *huge_idx;
        B_CHECK(get_buf(ctx, "pc_is_huge", g1, &is_huge));
        B_CHECK(get_buf(ctx, "pc_huge_idx", g1, &huge_idx));
        B_CHECK(get_buf(ctx, "pc_is_short", g1, &is_short));
        B_CHECK(get_buf(ctx, "pc_is_long", g1, &is_long));
        B_CHECK(get_buf(ctx, "pc_nch", g1, &nch));
        B_CHECK(get_buf(ctx, "pc_short_idx", g1, &short_idx));
        B_CHECK(get_buf(ctx, "pc_long_idx", g1, &long_idx));
        B_CHECK(get_buf(ctx, "pc_chunk_off", g1, &chunk_off));
        B_TRY(cudaMemsetAsync(is_short + L.G, 0, sizeof(int32_t), s));
        B_TRY(cudaMemsetAsync(is_long + L.G, 0, sizeof(int32_t), s));
        B_TRY(cudaMemsetAsync(nch + L.G, 0, sizeof(int32_t), s));
        B_TRY(cudaMemsetAsync(is_huge + L.G, 0, sizeof(int32_t), s));
        pcg_lists_count_kernel<<<grid_for(ctx, L.G, T256), T256, 0, s>>>(st.sp_row_off, L.G, is_short,
                                                                        is_long, nch, is_huge);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, is_huge, huge_idx, static_cast<int64_t>(g1)));
        B_CHECK(cub_exclusive_sum(ctx, is_short, short_idx, static_cast<int64_t>(g1)));
        B_CHECK(cub_exclusive_sum(ctx, is_long, long_idx, static_cast<int64_t>(g1)));
        B_CHECK(cub_exclusive_sum(ctx, nch, chunk_off, static_cast<int64_t>(g1)));
        int cnt[4];
        B_CHECK(sync_read_int(ctx, huge_idx + L.G, 1, &cnt[3]));
        st.pc_nhuge = cnt[3];
        B_CHECK(get_buf(ctx, "pc_huge_li", std::max<int64_t>(st.pc_nhuge, 1), &st.pc_huge_li));
        B_CHECK(sync_read_int(ctx, short_idx + L.G, 1, &cnt[0]));
        B_CHECK(sync_read_int(ctx, long_idx + L.G, 1, &cnt[1]));
        B_CHECK(sync_read_int(ctx, chunk_off + L.G, 1, &cnt[2]));
        st.pc_nshort = cnt[0];
        st.pc_nlong = cnt[1];
        st.pc_nlchunks = cnt[2];
        B_CHECK(get_buf(ctx, "pc_short_meta", std::max<int64_t>(st.pc_nshort, 1), &st.pc_short_meta));
        B_CHECK(get_buf(ctx, "pc_long_rows", std::max<int64_t>(st.pc_nlong, 1), &st.pc_long_rows));
        B_CHECK(get_buf(ctx, "pc_long_c0", std::max<int64_t>(st.pc_nlong, 1), &st.pc_long_c0));
        B_CHECK(get_buf(ctx, "pc_long_c1", std::max<int64_t>(st.pc_nlong, 1), &st.pc_long_c1));
        B_CHECK(get_buf(ctx, "pc_lchunk_meta", std::max<int64_t>(st.pc_nlchunks, 1), &st.pc_lchunk_meta));
        pcg_lists_fill_kernel<<<grid_for(ctx, L.G, T256), T256, 0, s>>>(
            st.sp_row_off, L.G, is_short, short_idx, long_idx, chunk_off, st.pc_short_meta,
            st.pc_long_rows, st.pc_long_c0, st.pc_long_c1, st.pc_lchunk_meta, huge_idx, st.pc_huge_li);
        B_LAUNCHED();
    }
    st.sparse = true;
    return B200FE_OK;
}

int build_structure(b200fe_context* ctx, int64_t n, int D, const int32_t* const* gids,
                    const int32_t* G, const double* w) {
    Structure& st = ctx->st;
    st = Structure();
    st.n = n;
    st.D = D;
    st.weighted = (w != nullptr);
    for (int d = 0; d < D; ++d) st.G[d] = G[d];
    // primary = most levels (first on ties)
    int p = 0;
    for (int d = 1; d < D; ++d)
        if (G[d] > G[p]) p = d;
    st.p = p;
    const cudaStream_t s = ctx->stream;
    const int T256 = 256;

    // validate ids, detect sortedness of the primary
    int32_t* flags;
    B_CHECK(get_buf(ctx, "flags", 4, &flags));
    B_TRY(cudaMemsetAsync(flags, 0, 4 * sizeof(int32_t), s));
    for (int d = 0; d < D; ++d) {
        validate_ids_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(gids[d], n, G[d], d == p,
                                                                      flags);
        B_LAUNCHED();
    }
    if (w) {
        validate_weights_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(w, n, flags);
        B_LAUNCHED();
    }
    int hf[4];
    B_CHECK(sync_read_int(ctx, flags, 4, hf));
    if (hf[0]) {
        ctx->err = "group id outside [0, num_groups)";
        return B200FE_INVALID_ARG;
    }
    if (hf[2]) {
        ctx->err = "weights must be finite and non-negative";
        return B200FE_INVALID_ARG;
    }
    const bool sorted = hf[1] == 0;

    // primary order
    int32_t* gp;
    B_CHECK(get_buf(ctx, "gp", n, &gp));
    if (sorted) {
        B_TRY(cudaMemcpyAsync(gp, gids[p], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
        st.pord = nullptr;
    } else {
        int32_t *iota, *pord;
        B_CHECK(get_buf(ctx, "tmp_n_a", n, &iota));
        B_CHECK(get_buf(ctx, "pord", n, &pord));
        iota_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(iota, n);
        B_LAUNCHED();
        B_CHECK(cub_sort_pairs(ctx, gids[p], gp, iota, pord, n, G[p]));
        st.pord = pord;
    }
    st.gp = gp;

    // primary segments
    int32_t* seg_off;
    B_CHECK(get_buf(ctx, "seg_off", static_cast<size_t>(G[p]) + 1, &seg_off));
    segment_offsets_kernel<<<grid_for(ctx, n + 1, T256), T256, 0, s>>>(gp, n, G[p], seg_off);
    B_LAUNCHED();
    st.seg_off = seg_off;

    // weights in primary order, segment weight sums
    if (w) {
        B_CHECK(get_buf(ctx, "wp64", n, &st.wp64));
        B_CHECK(get_buf(ctx, "wp32", n, &st.wp32));
        gather_kernel<double><<<grid_for(ctx, n, T256), T256, 0, s>>>(w, st.pord, n, st.wp64);
        B_LAUNCHED();
        to_float_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(st.wp64, n, st.wp32);
        B_LAUNCHED();
    }
    B_CHECK(get_buf(ctx, "inv_wp", G[p], &st.inv_wp));
    double* wsum_p;
    B_CHECK(get_buf(ctx, "wsum_p", G[p], &wsum_p));
    segment_inv_weight_kernel<<<grid_for(ctx, G[p], T256), T256, 0, s>>>(seg_off, G[p], st.wp64,
                                                                          wsum_p, st.inv_wp);
    B_LAUNCHED();

    // tiles of whole segments and the list of long segments
    {
        int32_t *tflag, *tidx, *lflag, *lidx;
        const size_t g1 = static_cast<size_t>(G[p]) + 1;
        B_CHECK(get_buf(ctx, "tflag", g1, &tflag));
        B_CHECK(get_buf(ctx, "tidx", g1, &tidx));
        B_CHECK(get_buf(ctx, "lflag", g1, &lflag));
        B_CHECK(get_buf(ctx, "lidx", g1, &lidx));
        tile_flag_kernel<<<grid_for(ctx, g1, T256), T256, 0, s>>>(seg_off, G[p], tflag, lflag);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, tflag, tidx, g1));
        B_CHECK(cub_exclusive_sum(ctx, lflag, lidx, g1));
        int cnt[2];
        B_CHECK(sync_read_int(ctx, tidx + G[p], 1, &cnt[0]));
        B_CHECK(sync_read_int(ctx, lidx + G[p], 1, &cnt[1]));
        st.ntiles = cnt[0];
        st.nlong = cnt[1];
        B_CHECK(get_buf(ctx, "tile_seg", static_cast<size_t>(st.ntiles) + 1, &st.tile_seg));
        B_CHECK(get_buf(ctx, "tile_long", static_cast<size_t>(st.ntiles) + 1, &st.tile_long));
        B_CHECK(get_buf(ctx, "long_segs", static_cast<size_t>(st.nlong) + 1, &st.long_segs));
        tile_fill_kernel<<<grid_for(ctx, g1, T256), T256, 0, s>>>(
            seg_off, G[p], tflag, tidx, lflag, lidx, st.tile_seg, st.tile_long, st.long_segs);
        B_LAUNCHED();
    }

    // classify the other dims
    for (int d = 0; d < D; ++d) {
        if (d == p) continue;
        int sg_total = 0;
        for (int j = 0; j < st.nS; ++j) sg_total += st.sG[j];
        if (G[d] <= kSmallLevels && st.nS < kMaxSmall && sg_total + G[d] <= kMaxSmallRows) {
            st.sdim[st.nS] = d;
            st.sG[st.nS] = G[d];
            ++st.nS;
        } else {
            if (st.nL >= kMaxLarge) {
                ctx->err = "more than 2 FE dimensions with over 64 levels besides the largest";
                return B200FE_INVALID_ARG;
            }
            st.L[st.nL].dim = d;
            st.L[st.nL].G = G[d];
            ++st.nL;
        }
    }
    int64_t row = 0;
    for (int l = 0; l < st.nL; ++l) {
        st.lbase[l] = row;
        row += st.L[l].G;
    }
    st.SG = 0;
    for (int j = 0; j < st.nS; ++j) {
        st.sbase[j] = row;
        st.sgoff[j] = st.SG;
        row += st.sG[j];
        st.SG += st.sG[j];
    }
    st.GR = row;

    double *Wall, *Eall;
    B_CHECK(get_buf(ctx, "diagW", std::max<int64_t>(st.GR, 1), &Wall));
    st.w_rows = Wall;
    B_CHECK(get_buf(ctx, "diagE", std::max<int64_t>(st.GR, 1), &Eall));

    // large dims: ids in primary order, runs, sorted run order, chunks, diagonal
    for (int l = 0; l < st.nL; ++l) {
        LargeDim& L = st.L[l];
        const std::string sfx = std::to_string(l);
        B_CHECK(get_buf(ctx, "rid" + sfx, n, &L.rid));
        gather_kernel<int32_t><<<grid_for(ctx, n, T256), T256, 0, s>>>(gids[L.dim], st.pord, n,
                                                                        L.rid);
        B_LAUNCHED();
        int32_t *rflags, *run_id;
        B_CHECK(get_buf(ctx, "tmp_n_a", n, &rflags));
        B_CHECK(get_buf(ctx, "tmp_n_b", n, &run_id));
        run_flags_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(gp, L.rid, n, rflags);
        B_LAUNCHED();
        B_CHECK(cub_inclusive_sum(ctx, rflags, run_id, n));
        int nr = 0;
        B_CHECK(sync_read_int(ctx, run_id + (n - 1), 1, &nr));
        L.nruns = nr;
        int32_t *run_grp, *run_start, *run_seg;
        B_CHECK(get_buf(ctx, "run_grp" + sfx, nr, &run_grp));
        L.run_grp = run_grp;
        B_CHECK(get_buf(ctx, "run_start" + sfx, static_cast<size_t>(nr) + 1, &run_start));
        B_CHECK(get_buf(ctx, "run_seg", nr, &run_seg));
        L.run_start = run_start;
        run_fill_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(rflags, run_id, gp, L.rid, n,
                                                                run_grp, run_start, run_seg);
        B_LAUNCHED();
        {
            const int32_t n32 = static_cast<int32_t>(n);
            B_TRY(cudaMemcpyAsync(run_start + nr, &n32, sizeof(int32_t), cudaMemcpyHostToDevice, s));
            B_TRY(cudaStreamSynchronize(s));  // n32 lives on this stack frame
        }
        B_CHECK(get_buf(ctx, "run_base" + sfx, static_cast<size_t>(G[p]) + 1, &L.run_base));
        run_base_kernel<<<grid_for(ctx, static_cast<int64_t>(G[p]) + 1, T256), T256, 0, s>>>(
            seg_off, G[p], run_id, n, nr, L.run_base);
        B_LAUNCHED();
        // sort runs by group (stable: primary order within a group)
        int32_t *riota, *sorted_runs, *sorted_grp;
        B_CHECK(get_buf(ctx, "tmp_n_a", n, &riota));  // flags no longer needed
        B_CHECK(get_buf(ctx, "sorted_runs", nr, &sorted_runs));
        B_CHECK(get_buf(ctx, "sorted_grp", nr, &sorted_grp));
        iota_kernel<<<grid_for(ctx, nr, T256), T256, 0, s>>>(riota, nr);
        B_LAUNCHED();
        B_CHECK(cub_sort_pairs(ctx, run_grp, sorted_grp, riota, sorted_runs, nr, L.G));
        // group offsets over sorted runs
        int32_t* grp_off;
        B_CHECK(get_buf(ctx, "grp_off" + sfx, static_cast<size_t>(L.G) + 1, &grp_off));
        segment_offsets_kernel<<<grid_for(ctx, static_cast<int64_t>(nr) + 1, T256), T256, 0, s>>>(
            sorted_grp, nr, L.G, grp_off);
        B_LAUNCHED();
        // run destinations and per-run diagonal terms
        B_CHECK(get_buf(ctx, "run_dest" + sfx, nr, &L.run_dest));
        double *cw, *ce, *cw_run;
        B_CHECK(get_buf(ctx, "run_cw", nr, &cw));
        B_CHECK(get_buf(ctx, "run_ce", nr, &ce));
        B_CHECK(get_buf(ctx, "run_cw_run" + sfx, nr, &cw_run));
        L.cw_run = cw_run;
        {
            double* ce_run;
            B_CHECK(get_buf(ctx, "run_ce_tmp", nr, &ce_run));
            run_weights_kernel<<<grid_for(ctx, nr, T256), T256, 0, s>>>(nr, run_start, n, run_seg,
                                                                        st.wp64, st.inv_wp, cw_run, ce_run);
            B_LAUNCHED();
            run_sorted_weights_kernel<<<grid_for(ctx, nr, T256), T256, 0, s>>>(sorted_runs, nr, cw_run, ce_run,
                                                                               L.run_dest, cw, ce);
            B_LAUNCHED();
        }
        // chunk lists (and super-chunks) of the groups' runs
        B_CHECK(build_chunks(ctx, grp_off, kChunkRuns, sfx, L));
        // diagonal terms W_g, E_g of the groups over the chunk list (balanced
        // however skewed the group sizes are)
        {
            double* part2;
            B_CHECK(get_buf(ctx, "wsum_part", static_cast<size_t>(L.nchunks) * 2, &part2));
            chunk_wsum_kernel<<<grid_for(ctx, L.nchunks, T256), T256, 0, s>>>(
                L.nchunks, L.chunk_grp, L.chunk_beg, L.chunk_end, L.chunk_whole, cw, ce,
                Wall + st.lbase[l], Eall + st.lbase[l], part2);
            B_LAUNCHED();
            if (L.nmulti > 0) {
                multi_wsum_kernel<<<static_cast<int>(std::min<int64_t>(
                                        L.nmulti, static_cast<int64_t>(ctx->num_sms) * 8)),
                                    256, 0, s>>>(L.nmulti, L.multi_grp, L.multi_c0, L.multi_c1, part2,
                                                 Wall + st.lbase[l], Eall + st.lbase[l]);
                B_LAUNCHED();
            }
        }
    }

    // the dense small-dim coupling of the CG matvec (block level, one small
    // dim with at most kCoupleMaxSG levels, coupling rows no larger than the
    // run rows): its setup also yields the exact small-dim diagonal
    const bool block_ok = st.GR > 0 && st.nL <= 1 && st.nS <= 1;
    const bool will_couple =
        block_ok && ctx->pass_kernel == 0 && st.nS == 1 && st.SG <= kCoupleMaxSG &&
        (st.nL == 0 || static_cast<int64_t>(st.L[0].G) * st.SG <= st.L[0].nruns * 16);

    // small dims: packed ids and diagonal
    if (st.nS > 0) {
        SmallPackArgs pa{};
        pa.nS = st.nS;
        for (int j = 0; j < st.nS; ++j) pa.ids[j] = gids[st.sdim[j]];
        B_CHECK(get_buf(ctx, "sid", n, &st.sid));
        pack_small_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(pa, st.pord, n, st.sid);
        B_LAUNCHED();
    }
    if (st.nS > 0 && !will_couple) {
        const int nb = ctx->num_sms * 4;
        double *part, *sw, *se;
        B_CHECK(get_buf(ctx, "small_part", static_cast<size_t>(nb) * kMaxSmall * kSmallLevels * 2,
                        &part));
        B_CHECK(get_buf(ctx, "small_w", kMaxSmall * kSmallLevels, &sw));
        B_CHECK(get_buf(ctx, "small_e", kMaxSmall * kSmallLevels, &se));
        small_diag_partial_kernel<<<nb, 128, 0, s>>>(st.sid, st.nS, n, gp, st.wp64, st.inv_wp,
                                                     part);
        B_LAUNCHED();
        small_diag_reduce_kernel<<<1, kMaxSmall * kSmallLevels, 0, s>>>(part, nb, st.nS, sw, se);
        B_LAUNCHED();
        for (int j = 0; j < st.nS; ++j) {
            B_TRY(cudaMemcpyAsync(Wall + st.sbase[j], sw + j * kSmallLevels,
                                  sizeof(double) * st.sG[j], cudaMemcpyDeviceToDevice, s));
            B_TRY(cudaMemcpyAsync(Eall + st.sbase[j], se + j * kSmallLevels,
                                  sizeof(double) * st.sG[j], cudaMemcpyDeviceToDevice, s));
        }
    }
    if (st.nS > 0) st.small_w = Wall + st.sbase[0];

    // blocks and packed metadata of the block-level pass
    st.block_ok = block_ok;
    if (st.block_ok) {
        int32_t *bflags, *bid, *bstart;
        B_CHECK(get_buf(ctx, "tmp_n_a", n, &bflags));
        B_CHECK(get_buf(ctx, "tmp_n_b", n, &bid));
        block_flags_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(
            gp, st.nL == 1 ? st.L[0].rid : nullptr, st.nS == 1 ? st.sid : nullptr, st.wp64, n, bflags);
        B_LAUNCHED();
        B_CHECK(cub_inclusive_sum(ctx, bflags, bid, n));
        int nb = 0;
        B_CHECK(sync_read_int(ctx, bid + (n - 1), 1, &nb));
        st.nblocks = nb;
        B_CHECK(get_buf(ctx, "block_start", nb, &bstart));
        block_start_kernel<<<grid_for(ctx, n, T256), T256, 0, s>>>(bflags, bid, n, bstart);
        B_LAUNCHED();
        B_CHECK(get_buf(ctx, "block_meta", nb, &st.block_meta));
        if (w) {
            B_CHECK(get_buf(ctx, "block_w64", nb, &st.block_w64));
            B_CHECK(get_buf(ctx, "block_w32", nb, &st.block_w32));
        }
        block_meta_kernel<<<grid_for(ctx, nb, T256), T256, 0, s>>>(
            bstart, nb, n, st.nS == 1 ? st.sid : nullptr, st.wp64, st.block_meta, st.block_w64,
            st.block_w32);
        B_LAUNCHED();
        const int64_t npr = st.nL == 1 ? st.L[0].nruns : static_cast<int64_t>(G[p]);
        B_CHECK(get_buf(ctx, "seg_meta", static_cast<size_t>(G[p]) + 1, &st.seg_meta));
        B_CHECK(get_buf(ctx, "run_meta", npr, &st.run_meta));
        B_CHECK(get_buf(ctx, "run_w64", npr, &st.run_w64));
        B_CHECK(get_buf(ctx, "run_w32", npr, &st.run_w32));
        const bool lg = st.nL == 1;
        pack_meta_kernel<<<grid_for(ctx, std::max<int64_t>(npr, static_cast<int64_t>(G[p]) + 1), T256),
                           T256, 0, s>>>(
            seg_off, lg ? st.L[0].run_base : nullptr, G[p], lg ? st.L[0].run_grp : nullptr,
            lg ? st.L[0].run_dest : nullptr, lg ? st.L[0].run_start : nullptr,
            lg ? st.L[0].nruns : 0, lg ? st.L[0].cw_run : nullptr, bid, nb, n, st.seg_meta,
            st.run_meta, st.run_w64, st.run_w32);
        B_LAUNCHED();
        // dense coupling of the small dim, when its rows are cheaper to stream
        // than one more pass over the runs
        const int64_t SG = st.SG;
        st.coupled = will_couple;
        if (st.coupled) {
            st.SGP = static_cast<int>((SG + 3) & ~int64_t(3));
            const int64_t SGP = st.SGP;
            if (lg) {
                const LargeDim& L = st.L[0];
                int32_t *sorted_grp, *run_seg, *grp_off;
                int4* frec;
                double* frec_cf;
                B_CHECK(get_buf(ctx, "sorted_grp", L.nruns, &sorted_grp));
                B_CHECK(get_buf(ctx, "fy_rec", L.nruns, &frec));
                B_CHECK(get_buf(ctx, "fy_rec_cf", L.nruns, &frec_cf));
                B_CHECK(get_buf(ctx, "run_seg", L.nruns, &run_seg));
                B_CHECK(get_buf(ctx, "grp_off0", static_cast<size_t>(L.G) + 1, &grp_off));
                const int64_t nranges = (L.nruns + kFyRangeRuns - 1) / kFyRangeRuns;
                double* cpart;
                B_CHECK(get_buf(ctx, "cfy64", static_cast<size_t>(L.G) * SGP, &st.cfy64));
                B_CHECK(get_buf(ctx, "cfy32", static_cast<size_t>(L.G) * SGP, &st.cfy32));
                B_CHECK(get_buf(ctx, "cfy_part", static_cast<size_t>(std::max<int64_t>(nranges, 1)) * 2 * SGP, &cpart));
                if (nranges == 0) {
                    B_TRY(cudaMemsetAsync(st.cfy64, 0, sizeof(double) * static_cast<size_t>(L.G) * SGP, s));
                } else {
                    const size_t fsmem = static_cast<size_t>(kCoupleWarps) * 32 * couple_pitch(static_cast<int>(SG)) * sizeof(double);
                    B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&coupling_fy_range_kernel), static_cast<int>(fsmem)));
                    int fps = 1;
                    B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fps, coupling_fy_range_kernel,
                                                                        kCoupleWarps * 32, fsmem));
                    const int fgrid = static_cast<int>(std::max<int64_t>(
                        1, std::min<int64_t>((nranges + kCoupleWarps - 1) / kCoupleWarps,
                                             static_cast<int64_t>(ctx->num_sms) * std::max(fps, 1))));
                    fy_run_record_kernel<<<grid_for(ctx, L.nruns, T256), T256, 0, s>>>(
                        L.nruns, L.run_dest, run_seg, st.run_meta, st.seg_meta, L.cw_run, st.inv_wp, frec,
                        frec_cf);
                    B_LAUNCHED();
                    coupling_fy_range_kernel<<<fgrid, kCoupleWarps * 32, fsmem, s>>>(
                        L.nruns, nranges, L.G, frec, frec_cf, sorted_grp, grp_off, st.block_meta,
                        st.block_w64, st.SG, st.SGP, st.cfy64, cpart);
                    B_LAUNCHED();
                    if (nranges > 1) {
                        coupling_fy_join_kernel<<<static_cast<int>(std::min<int64_t>(
                                                      nranges, static_cast<int64_t>(ctx->num_sms) * 8)),
                                                  256, 0, s>>>(L.nruns, nranges, sorted_grp, grp_off, cpart,
                                                               st.SGP, st.cfy64);
                        B_LAUNCHED();
                    }
                }
                to_float_kernel<<<grid_for(ctx, static_cast<int64_t>(L.G) * SGP, T256), T256, 0, s>>>(
                    st.cfy64, static_cast<int64_t>(L.G) * SGP, st.cfy32);
                B_LAUNCHED();
            }
            // C_yy partials: the register-tiled kernel where SG fits one of its
            // tiles, the shared-memory accumulator above that
            int ny = 1;
            double* ypart = nullptr;
            B_CHECK(get_buf(ctx, "cyy", static_cast<size_t>(SG) * SG, &st.cyy));
            auto launch_yy = [&](auto kern, int warps, size_t smem) -> int {
                B_TRY(raise_smem_limit(reinterpret_cast<const void*>(kern), static_cast<int>(smem)));
                int yps = 1;
                B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&yps, kern, warps * 32, smem));
                ny = static_cast<int>(std::max<int64_t>(
                    1, std::min<int64_t>((static_cast<int64_t>(G[p]) + 32 * warps - 1) / (32 * warps),
                                         static_cast<int64_t>(ctx->num_sms) * std::max(yps, 1))));
                B_CHECK(get_buf(ctx, "cyy_part", static_cast<size_t>(ny) * (SG * SG + SG), &ypart));
                kern<<<ny, warps * 32, smem, s>>>(G[p], st.seg_meta, st.run_meta, st.block_meta,
                                                  st.block_w64, st.inv_wp, st.SG, ypart);
                B_LAUNCHED();
                return B200FE_OK;
            };
            auto tile_smem = [&](int RT, int CT) {
                return static_cast<size_t>(SG * SG + SG + kCoupleTileWarps * 32 * couple_tile_pitch(RT, CT)) *
                       sizeof(double);
            };
            if (SG <= 12)
                B_CHECK(launch_yy(&coupling_yy_tile_kernel<2, 3>, kCoupleTileWarps, tile_smem(2, 3)));
            else if (SG <= 24)
                B_CHECK(launch_yy(&coupling_yy_tile_kernel<3, 6>, kCoupleTileWarps, tile_smem(3, 6)));
            else if (SG <= 36)
                B_CHECK(launch_yy(&coupling_yy_tile_kernel<5, 9>, kCoupleTileWarps, tile_smem(5, 9)));
            else
                B_CHECK(launch_yy(&coupling_yy_kernel, kCoupleYyWarps,
                                  static_cast<size_t>(kCoupleYyWarps) * couple_yy_warp_words(static_cast<int>(SG)) *
                                      sizeof(double)));
            coupling_yy_reduce_kernel<<<grid_for(ctx, SG * SG, T256), T256, 0, s>>>(
                ypart, ny, st.SG, st.cyy, Wall + st.sbase[0], Eall + st.sbase[0]);
            B_LAUNCHED();
        }
    }

    // explicit Schur block of the large dim (sparse_kernels.cuh): replaces the
    // per-iteration pass over the runs when the movers' pairs fit
    if (st.block_ok && ctx->sparse_schur && st.nL == 1 && (st.nS == 0 || st.coupled))
        B_CHECK(build_sparse_block(ctx));

    B_CHECK(build_stream_meta(ctx));

    if (st.GR > 0) {
        B_CHECK(get_buf(ctx, "dinv64", st.GR, &st.dinv64));
        B_CHECK(get_buf(ctx, "dinv32", st.GR, &st.dinv32));
        dinv_kernel<<<grid_for(ctx, st.GR, T256), T256, 0, s>>>(Wall, Eall, st.GR, st.dinv64,
                                                                 st.dinv32);
        B_LAUNCHED();
    }
    // ||D'W||_F^2 = D * sum w^2
    if (w) {
        double *part, *outv;
        unsigned int* ticket;
        B_CHECK(get_buf(ctx, "dot_part_w", static_cast<size_t>(ctx->num_sms) * 8, &part));
        B_CHECK(get_buf(ctx, "dot_out_w", 1, &outv));
        B_CHECK(get_buf(ctx, "ticket_w", 1, &ticket));
        B_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
        row_dot_kernel<double, double><<<grid_for(ctx, n, kRowThreads), kRowThreads, 0, s>>>(
            n, 1, w, w, part, ticket, outv);
        B_LAUNCHED();
        double sw2 = 0.0;
        B_CHECK(sync_read_double(ctx, outv, 1, &sw2));
        st.sum_w2 = sw2;
    } else {
        st.sum_w2 = static_cast<double>(n);
    }
    // levels present per dim (groups with positive weight): primary from
    // segment weights; the others from the diagonal's weight sums.
    for (int d = 0; d < D; ++d) st.present[d] = G[d];
    B_TRY(cudaStreamSynchronize(s));
    st.valid = true;
    return B200FE_OK;
}

// ---------------------------------------------------------------------------
// Solver
// ---------------------------------------------------------------------------
constexpr int kRunBatch = 2;  // runs per load batch of run_pass_kernel

template <typename T>
const T* pick_prec(const float* f32, const double* f64);
template <>
const float* pick_prec<float>(const float* f32, const double*) { return f32; }
template <>
const double* pick_prec<double>(const float*, const double* f64) { return f64; }

template <typename T>
struct Work {
    T* R[kMaxLarge];
    double* bins_partial;   // [nbins_ctas][SG][CP]
    double* colsq_partial;  // [nbins_ctas][CP]
    double* gather_partial[kMaxLarge];
    double* fin_partial;
    double* chunk_partial[kMaxLarge];
    double* super_partial[kMaxLarge];
    double* dot_out;
    unsigned int* ticket;
    int tile_grid, tile_smem;
    int data_grid, data_smem;  // FP64 data passes (double Work only)
    int run_grid, run_smem;  // block-level matvec grid/smem (0 when it does not apply)
    int long_grid, long_smem;
    int nbins_ctas;
    int couple_grid;  // CTAs of coupling_xf_kernel (coupled matvec), <= nbins_ctas
    int gather_grid[kMaxLarge];
    int fin_grid;
    int64_t fin_rows;
    // explicit Schur block (st.sparse): gather CTAs, their dot partials, the
    // chunk and super-chunk partials of multi-chunk rows, finalize rows/CTAs
    int sp_gather_grid;
    double* sp_gather_partial;
    double* sp_chunk_partial;
    double* sp_super_partial;
    int64_t sp_fin_rows;
    int sp_fin_grid;
};

template <typename T, int CQ, int MODE>
int set_pass_smem(b200fe_context* ctx, int tile_smem, int long_smem) {
    B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&tile_pass_kernel<T, CQ, MODE>), tile_smem));
    B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&segment_pass_kernel<T, CQ, MODE>), long_smem));
    return B200FE_OK;
}

template <typename T, int CQ>
int prepare_work(b200fe_context* ctx, const std::string& tag, Work<T>& wk) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    wk.tile_smem = static_cast<int>(tile_smem_bytes<T>(CP, st.SG));
    wk.long_smem = std::max<int>((kPassThreads / 32) * st.SG * CP * sizeof(double),
                                 kPassThreads * 4 * sizeof(double));
    B_CHECK((set_pass_smem<T, CQ, kMatvec>(ctx, wk.tile_smem, wk.long_smem)));
    B_CHECK((set_pass_smem<T, CQ, kRhs>(ctx, wk.tile_smem, wk.long_smem)));
    B_CHECK((set_pass_smem<T, CQ, kFinal>(ctx, wk.tile_smem, wk.long_smem)));
    int per_sm = 1;
    B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_pass_kernel<T, CQ, kMatvec>,
                                                        kTileThreads, wk.tile_smem));
    per_sm = std::max(1, per_sm);
    wk.tile_grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>(st.ntiles, static_cast<int64_t>(ctx->num_sms) * per_sm)));
    wk.data_grid = 0;
    wk.data_smem = 0;
    if (std::is_same<T, double>::value) {
        wk.data_smem = static_cast<int>(data_smem_bytes(CP, st.SG, st.nL));
        B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&data_pass_kernel<CP, kRhs>), wk.data_smem));
        B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&data_pass_kernel<CP, kFinal>), wk.data_smem));
        int dps = 1;
        B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dps, data_pass_kernel<CP, kRhs>, kDataThreads,
                                                            wk.data_smem));
        dps = std::max(1, dps);
        wk.data_grid = static_cast<int>(std::max<int64_t>(
            1, std::min<int64_t>(st.ntiles, static_cast<int64_t>(ctx->num_sms) * dps)));
    }
    wk.run_grid = 0;
    wk.run_smem = 0;
    if (st.block_ok && (ctx->pass_kernel == 0 || ctx->pass_kernel == 2)) {
        // the coupled matvec runs the pass without the small dim: no shared memory
        wk.run_smem = st.coupled ? 0 : static_cast<int>(block_smem_bytes<T>(CP, st.SG));
        B_TRY(raise_smem_limit(reinterpret_cast<const void*>(&block_pass_kernel<T, CQ>), wk.run_smem));
        int rps = 1;
        B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rps, block_pass_kernel<T, CQ>, kBlockThreads,
                                                            wk.run_smem));
        rps = std::max(1, rps);
        const int64_t warps = (static_cast<int64_t>(st.G[st.p]) + (32 / CQ) - 1) / (32 / CQ);
        wk.run_grid = static_cast<int>(std::max<int64_t>(
            1, std::min<int64_t>((warps + 3) / 4, static_cast<int64_t>(ctx->num_sms) * rps)));
    }
    wk.long_grid = 0;
    if (st.nlong > 0) {
        const int64_t groups = (st.nlong + (32 / CQ) - 1) / (32 / CQ);
        wk.long_grid = grid_for(ctx, groups * 32, kPassThreads, 4);
    }
    wk.nbins_ctas = std::max(std::max(wk.tile_grid, wk.run_grid), wk.data_grid) + wk.long_grid;
    wk.couple_grid = 0;
    if (st.coupled && wk.run_grid > 0 && st.nL == 1)
        wk.couple_grid = static_cast<int>(std::max<int64_t>(
            1, std::min<int64_t>({static_cast<int64_t>(wk.nbins_ctas),
                                  static_cast<int64_t>(ctx->num_sms) * 8, st.L[0].G})));
    B_CHECK(get_buf(ctx, tag + "bins", static_cast<size_t>(wk.nbins_ctas) * std::max(st.SG, 1) * CP,
                    &wk.bins_partial));
    B_CHECK(get_buf(ctx, tag + "colsq", static_cast<size_t>(wk.nbins_ctas) * CP, &wk.colsq_partial));
    for (int l = 0; l < st.nL; ++l) {
        const std::string sfx = std::to_string(l);
        // the FP32 run rows serve only the run-level matvec
        const bool need_R = !(st.sparse && std::is_same<T, float>::value);
        B_CHECK(get_buf(ctx, tag + "R" + sfx, need_R ? static_cast<size_t>(st.L[l].nruns) * CP : 1,
                        &wk.R[l]));
        wk.gather_grid[l] = grid_for(ctx, st.L[l].nchunks * CQ, kRowThreads, 8);
        B_CHECK(get_buf(ctx, tag + "gpart" + sfx, static_cast<size_t>(wk.gather_grid[l]) * CP,
                        &wk.gather_partial[l]));
        B_CHECK(get_buf(ctx, tag + "cpart" + sfx, static_cast<size_t>(st.L[l].nchunks) * CP,
                        &wk.chunk_partial[l]));
        B_CHECK(get_buf(ctx, tag + "spart" + sfx, static_cast<size_t>(std::max<int64_t>(st.L[l].nsup, 1)) * CP,
                        &wk.super_partial[l]));
    }
    wk.fin_rows = st.SG;
    for (int l = 0; l < st.nL; ++l) wk.fin_rows += st.L[l].nmulti;
    wk.fin_grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>(wk.fin_rows, static_cast<int64_t>(ctx->num_sms) * 8)));
    wk.sp_gather_grid = 0;
    wk.sp_fin_rows = 0;
    wk.sp_fin_grid = 0;
    if (st.sparse) {
        wk.sp_gather_grid = grid_for(ctx, st.sp.nchunks * CQ, kRowThreads, 8);
        B_CHECK(get_buf(ctx, tag + "sp_gpart", static_cast<size_t>(wk.sp_gather_grid) * CP,
                        &wk.sp_gather_partial));
        B_CHECK(get_buf(ctx, tag + "sp_cpart", static_cast<size_t>(st.sp.nchunks) * CP,
                        &wk.sp_chunk_partial));
        B_CHECK(get_buf(ctx, tag + "sp_spart",
                        static_cast<size_t>(std::max<int64_t>(st.sp.nsup, 1)) * CP,
                        &wk.sp_super_partial));
        wk.sp_fin_rows = st.SG + st.sp.nmulti;
        wk.sp_fin_grid = static_cast<int>(std::max<int64_t>(
            1, std::min<int64_t>(wk.sp_fin_rows, static_cast<int64_t>(ctx->num_sms) * 8)));
    }
    B_CHECK(get_buf(ctx, tag + "fpart", static_cast<size_t>(std::max(wk.fin_grid, wk.sp_fin_grid)) * CP,
                    &wk.fin_partial));
    B_CHECK(get_buf(ctx, tag + "dotout", CP, &wk.dot_out));
    B_CHECK(get_buf(ctx, tag + "ticket", 1, &wk.ticket));
    B_TRY(cudaMemsetAsync(wk.ticket, 0, sizeof(unsigned int), ctx->stream));
    return B200FE_OK;
}

template <typename T>
PassArgs<T> make_pass_args(const Structure& st, int cols, int CP, const Work<T>& wk) {
    PassArgs<T> a{};
    a.n = st.n;
    a.Gp = st.G[st.p];
    a.cols = cols;
    a.CP = CP;
    a.nL = st.nL;
    a.nS = st.nS;
    a.seg_off = st.seg_off;
    a.inv_wp = st.inv_wp;
    a.pord = st.pord;
    for (int l = 0; l < st.nL; ++l) {
        a.rid[l] = st.L[l].rid;
        a.run_base[l] = st.L[l].run_base;
        a.run_start[l] = st.L[l].run_start;
        a.run_dest[l] = st.L[l].run_dest;
        a.lbase[l] = st.lbase[l];
        a.R[l] = wk.R[l];
    }
    a.sid = st.sid;
    for (int j = 0; j < st.nS; ++j) {
        a.sbase[j] = st.sbase[j];
        a.sgoff[j] = st.sgoff[j];
    }
    a.SG = st.SG;
    a.bins_partial = wk.bins_partial;
    a.colsq_partial = wk.colsq_partial;
    a.tile_seg = st.tile_seg;
    a.tile_long = st.tile_long;
    a.ntiles = st.ntiles;
    a.long_segs = st.long_segs;
    a.nlong = st.nlong;
    return a;
}

// Bulk-copy FP64 data pass over the regular tiles (stream_kernels.cuh): one
// CTA per SM with as many stages as shared memory holds (at least two).
// *grid = 0 (nothing launched) when it does not apply: the pass is off, the
// observations are not in primary order, a tile exceeds the staged sizes, or
// (kFinal) input and output differ in their offset from a 16-byte boundary.
template <int MODE>
int launch_stream_pass(b200fe_context* ctx, const PassArgs<double>& a, int* grid) {
    const Structure& st = ctx->st;
    *grid = 0;
    if (!ctx->stream_pass || !st.stream_ok || a.pord || a.cols > 16 || a.CP > 16 || st.stream_nreg <= 0)
        return B200FE_OK;
    const uintptr_t pv = reinterpret_cast<uintptr_t>(a.v), po = reinterpret_cast<uintptr_t>(a.out);
    if ((pv & 7u) || (MODE == kFinal && (((pv ^ po) & 15u) || (po & 7u)))) return B200FE_OK;
    const bool weighted = a.wp != nullptr;
    StreamLayout L{};
    int off = kStreamHeader;
    L.off_cols = off;
    off += a.cols * kStreamPitchD * 8;
    L.off_blob = off;
    off += round16(st.stream_blob_max);
    if (weighted) {
        L.off_wp = off;
        off += kStreamPitchD * 8;
    }
    if (MODE == kFinal && a.nS > 0) {
        L.off_sid = off;
        off += kStreamPitchI * 4;
    }
    for (int l = 0; l < a.nL && MODE == kFinal && a.nL > 1; ++l) {
        L.off_rid[l] = off;
        off += kStreamPitchI * 4;
    }
    L.stage_bytes = (off + 127) & ~127;
    L.off_stages = 128;  // barriers and the abort flag
    const int bins_bytes = std::max(a.SG, 1) * 16 * 8;
    const int red_bytes = kStreamWarps * 16 * 8;
    const int yt_bytes = (MODE == kFinal && a.nS > 0) ? a.SG * 16 * 8 : 0;
    const int afb_bytes = (MODE == kFinal && a.nL == 1) ? kStreamWarps * kStreamRunRows * 16 * 8 : 0;
    int budget = 0;
    B_TRY(cudaDeviceGetAttribute(&budget, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const int ns = std::min(kStreamMaxStages, (budget - L.off_stages - bins_bytes - red_bytes - yt_bytes - afb_bytes) /
                                                  L.stage_bytes);
    if (ns < 2) return B200FE_OK;
    L.NS = ns;
    L.off_bins = L.off_stages + ns * L.stage_bytes;
    L.off_red = L.off_bins + bins_bytes;
    L.off_yt = L.off_red + red_bytes;
    L.off_afb = L.off_yt + yt_bytes;
    const int smem = L.off_afb + afb_bytes;
    L.tmeta = st.stream_meta;
    L.nreg = st.stream_nreg;
    L.boff = st.stream_boff;
    L.blob = st.stream_blob;
    L.aux_stride = st.stream_aux_stride;
    if (!ctx->stream_status) {
        B_CHECK(get_buf(ctx, "stream_status", 4, &ctx->stream_status));
        B_TRY(cudaMemsetAsync(ctx->stream_status, 0, 4 * sizeof(int), ctx->stream));
    }
    L.status = ctx->stream_status;
    auto kern = weighted ? stream_pass_kernel<MODE, true> : stream_pass_kernel<MODE, false>;
    const unsigned bit = 1u << (2 * (MODE == kFinal ? 1 : 0) + (weighted ? 1 : 0));
    if (!(ctx->stream_smem_set & bit)) {
        B_TRY(raise_smem_limit(reinterpret_cast<const void*>(kern), budget));
        ctx->stream_smem_set |= bit;
    }
    const int g = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(st.stream_nreg, ctx->num_sms)));
    kern<<<g, kStreamThreads, smem, ctx->stream>>>(a, L);
    B_LAUNCHED();
    *grid = g;
    return B200FE_OK;
}

// Reports a bulk-copy data pass whose pipeline wait ran out (and clears it).
int check_stream_status(b200fe_context* ctx) {
    if (!ctx->stream_status) return B200FE_OK;
    int hs = 0;
    B_CHECK(sync_read_int(ctx, ctx->stream_status, 1, &hs));
    if (hs != 0) {
        B_TRY(cudaMemsetAsync(ctx->stream_status, 0, sizeof(int), ctx->stream));
        ctx->err = "FP64 data pass: a pipeline wait timed out";
        return B200FE_CUDA_ERROR;
    }
    return B200FE_OK;
}

// Data pass (FP64: bulk-copy stream pass, else lane = column) or tile pass
// over the regular tiles, then the long segments (if any).  Partial slots beyond the launched grid are
// zeroed so finalize and the host sum a fixed number of slots.
template <typename T, int CQ, int MODE>
int launch_pass(b200fe_context* ctx, const Work<T>& wk, PassArgs<T> a) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const int slots = std::max(std::max(wk.tile_grid, wk.run_grid), wk.data_grid);
    int used;
    a.bins_cta0 = 0;
    if constexpr (std::is_same<T, double>::value && MODE != kMatvec) {
        B_CHECK(launch_stream_pass<MODE>(ctx, a, &used));
        if (used == 0) {
            data_pass_kernel<CP, MODE><<<wk.data_grid, kDataThreads, wk.data_smem, ctx->stream>>>(a);
            B_LAUNCHED();
            used = wk.data_grid;
        }
    } else {
        tile_pass_kernel<T, CQ, MODE><<<wk.tile_grid, kTileThreads, wk.tile_smem, ctx->stream>>>(a);
        B_LAUNCHED();
        used = wk.tile_grid;
    }
    if (used < slots) {
        if (st.nS > 0)
            B_TRY(cudaMemsetAsync(wk.bins_partial + static_cast<int64_t>(used) * st.SG * CP, 0,
                                  sizeof(double) * (slots - used) * st.SG * CP, ctx->stream));
        B_TRY(cudaMemsetAsync(wk.colsq_partial + static_cast<int64_t>(used) * CP, 0,
                              sizeof(double) * (slots - used) * CP, ctx->stream));
    }
    if (wk.long_grid > 0) {
        a.bins_cta0 = slots;
        segment_pass_kernel<T, CQ, MODE><<<wk.long_grid, kPassThreads, wk.long_smem, ctx->stream>>>(a);
        B_LAUNCHED();
    }
    return B200FE_OK;
}

// Matvec pass: run-level kernel when there is at most one large dim, else
// the tile kernel; then the long segments.  Bin partials of CTAs beyond the
// launched grid are zeroed so finalize can sum a fixed number of slots.
template <typename T, int CQ>
int launch_matvec_pass(b200fe_context* ctx, const Work<T>& wk, PassArgs<T> a, const T* run_w,
                       const T* block_w) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const int slots = std::max(std::max(wk.tile_grid, wk.run_grid), wk.data_grid);
    if (wk.run_grid > 0 && st.coupled) {
        // large dim only over every segment (C_fy' x_f follows in matvec)
        if (st.nL == 1) {
            BlockArgs<T> r{};
            r.Gp = st.G[st.p];
            r.CP = CP;
            r.has_large = 1;
            r.has_small = 0;
            r.SG = st.SG;
            r.seg_meta = st.seg_meta;
            r.inv_wp = st.inv_wp;
            r.run_meta = st.run_meta;
            r.run_w = run_w;
            r.block_meta = st.block_meta;
            r.block_w = block_w;
            r.lbase = st.lbase[0];
            r.sbase = st.sbase[0];
            r.x = a.x;
            r.R = wk.R[0];
            r.bins_partial = wk.bins_partial;
            r.bins_cta0 = 0;
            r.all_segs = 1;
            run_pass_kernel<T, CQ, kRunBatch><<<wk.run_grid, kBlockThreads, 0, ctx->stream>>>(r);
            B_LAUNCHED();
        }
        return B200FE_OK;
    }
    if (wk.run_grid > 0) {
        BlockArgs<T> r{};
        r.Gp = st.G[st.p];
        r.CP = CP;
        r.has_large = st.nL == 1;
        r.has_small = st.nS == 1;
        r.SG = st.SG;
        r.seg_meta = st.seg_meta;
        r.inv_wp = st.inv_wp;
        r.run_meta = st.run_meta;
        r.run_w = run_w;
        r.block_meta = st.block_meta;
        r.block_w = block_w;
        r.lbase = st.nL == 1 ? st.lbase[0] : 0;
        r.sbase = st.nS == 1 ? st.sbase[0] : 0;
        r.x = a.x;
        r.R = st.nL == 1 ? wk.R[0] : nullptr;
        r.bins_partial = wk.bins_partial;
        r.bins_cta0 = 0;
        r.all_segs = 0;
        if (st.nL == 1 && st.nS == 0)  // runs only (two-way)
            run_pass_kernel<T, CQ, kRunBatch><<<wk.run_grid, kBlockThreads, 0, ctx->stream>>>(r);
        else
            block_pass_kernel<T, CQ><<<wk.run_grid, kBlockThreads, wk.run_smem, ctx->stream>>>(r);
        B_LAUNCHED();
        if (st.nS > 0 && wk.run_grid < slots)
            B_TRY(cudaMemsetAsync(wk.bins_partial + static_cast<int64_t>(wk.run_grid) * st.SG * CP, 0,
                                  sizeof(double) * (slots - wk.run_grid) * st.SG * CP, ctx->stream));
    } else {
        a.bins_cta0 = 0;
        tile_pass_kernel<T, CQ, kMatvec><<<wk.tile_grid, kTileThreads, wk.tile_smem, ctx->stream>>>(a);
        B_LAUNCHED();
        if (st.nS > 0 && wk.tile_grid < slots)
            B_TRY(cudaMemsetAsync(wk.bins_partial + static_cast<int64_t>(wk.tile_grid) * st.SG * CP, 0,
                                  sizeof(double) * (slots - wk.tile_grid) * st.SG * CP, ctx->stream));
    }
    if (wk.long_grid > 0) {
        a.bins_cta0 = slots;
        a.bins_no_diag = wk.run_grid > 0 ? 1 : 0;
        segment_pass_kernel<T, CQ, kMatvec><<<wk.long_grid, kPassThreads, wk.long_smem, ctx->stream>>>(a);
        B_LAUNCHED();
    }
    return B200FE_OK;
}

// Algorithmic bytes of one launch (what the launch must read or write at
// least once from HBM); alpha vectors of the large dims are counted once.
double struct_obs_bytes(const Structure& st, size_t wsize) {
    return static_cast<double>(st.n) *
               (4.0 * st.nL + (st.nS ? 4.0 : 0.0) + (st.weighted ? double(wsize) : 0.0)) +
           static_cast<double>(st.G[st.p]) * (4.0 + 8.0 + 4.0 * st.nL);
}
double runs_write_bytes(const Structure& st, int CP, size_t tsize) {
    double b = 0.0;
    for (int l = 0; l < st.nL; ++l)
        b += static_cast<double>(st.L[l].nruns) * (4.0 + CP * double(tsize));
    return b;
}
double gather_bytes(const Structure& st, int l, int CP, size_t tsize, bool dot) {
    return static_cast<double>(st.L[l].nchunks) * 13.0 +
           static_cast<double>(st.L[l].nruns) * CP * double(tsize) +
           static_cast<double>(st.L[l].G) * CP * double(tsize) * (dot ? 2.0 : 1.0);
}

// Gathers runs and bins into alpha rows `out`; dot with `dotv` into wk.dot_out.
template <typename T, int CQ>
int reduce_runs(b200fe_context* ctx, const Work<T>& wk, T* out, const T* dotv,
                int cat_gather = B200FE_PROF_GATHER, int cat_fin = B200FE_PROF_FINALIZE,
                bool small_diag = false, bool coupled = false) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    for (int l = 0; l < st.nL; ++l) {
        GatherArgs<T> g{};
        g.CP = CP;
        g.nchunks = st.L[l].nchunks;
        g.chunk_grp = st.L[l].chunk_grp;
        g.chunk_beg = st.L[l].chunk_beg;
        g.chunk_end = st.L[l].chunk_end;
        g.chunk_whole = st.L[l].chunk_whole;
        g.R = wk.R[l];
        g.out = out + st.lbase[l] * CP;
        g.partial = wk.chunk_partial[l];
        g.dotv = dotv ? dotv + st.lbase[l] * CP : nullptr;
        g.dot_partial = wk.gather_partial[l];
        if (coupled && l == 0) {  // + C_fy x_small (x is the matvec input, dotv)
            g.cfy = pick_prec<T>(st.cfy32, st.cfy64);
            g.xs = dotv + st.sbase[0] * CP;
            g.SG = st.SG;
            g.SGP = st.SGP;
        }
        ProfScope ps(ctx, cat_gather, gather_bytes(st, l, CP, sizeof(T), dotv != nullptr));
        const size_t gsmem = g.cfy ? static_cast<size_t>(st.SGP) * CP * sizeof(T) : 0;
        run_gather_kernel<T, CQ><<<wk.gather_grid[l], kRowThreads, gsmem, s>>>(g);
        B_LAUNCHED();
        if (st.L[l].nsup > 0) {
            multi_super_kernel<<<grid_for(ctx, st.L[l].nsup * CP, kRowThreads), kRowThreads, 0, s>>>(
                st.L[l].nsup, st.L[l].sup_c0, st.L[l].sup_c1, wk.chunk_partial[l], CP,
                wk.super_partial[l]);
            B_LAUNCHED();
        }
    }
    FinalizeArgs<T> f{};
    f.CP = CP;
    f.nL = st.nL;
    f.nS = st.nS;
    for (int l = 0; l < st.nL; ++l) {
        f.nmulti[l] = st.L[l].nmulti;
        f.multi_grp[l] = st.L[l].multi_grp;
        f.multi_c0[l] = st.L[l].multi_c0;
        f.multi_c1[l] = st.L[l].multi_c1;
        f.partial[l] = wk.chunk_partial[l];
        f.multi_s0[l] = st.L[l].multi_s0;
        f.multi_s1[l] = st.L[l].multi_s1;
        f.super_partial[l] = wk.super_partial[l];
        f.lbase[l] = st.lbase[l];
        f.gather_dot_partial[l] = wk.gather_partial[l];
        f.gather_ctas[l] = dotv ? wk.gather_grid[l] : 0;
    }
    f.SG = st.SG;
    f.sgbase = st.nS > 0 ? st.sbase[0] : 0;
    f.bins_partial = wk.bins_partial;
    f.nbins_ctas = coupled ? wk.couple_grid : wk.nbins_ctas;
    f.small_diag = (small_diag && st.nS > 0 && !coupled) ? st.small_w : nullptr;
    f.small_dense = coupled ? st.cyy : nullptr;
    f.cfy = (coupled && st.nL == 1) ? pick_prec<T>(st.cfy32, st.cfy64) : nullptr;
    f.SGP = st.SGP;
    f.x = dotv;
    f.nrows = wk.fin_rows;
    f.out = out;
    f.dotv = dotv;
    f.dot_partial = wk.fin_partial;
    f.dot_out = dotv ? wk.dot_out : nullptr;
    f.ticket = wk.ticket;
    double fb = static_cast<double>(f.nbins_ctas) * st.SG * CP * 8.0;
    for (int l = 0; l < st.nL; ++l) fb += static_cast<double>(st.L[l].nmulti) * CP * (8.0 + sizeof(T));
    fb += static_cast<double>(st.SG) * CP * sizeof(T);
    ProfScope ps(ctx, cat_fin, fb);
    finalize_kernel<T><<<wk.fin_grid, kRowThreads, 0, s>>>(f);
    B_LAUNCHED();
    return B200FE_OK;
}

// q = S x over the explicit Schur block: the rows of the large dim by the
// sparse gather (+ C_fy x_small), then finalize (multi-chunk rows, small-dim
// rows from the coupling partials, the dot x'q into wk.dot_out).
template <typename T, int CQ>
int reduce_sparse(b200fe_context* ctx, const Work<T>& wk, const T* x, T* q) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    const LargeDim& L = st.sp;
    const bool coupled = st.coupled && st.nS == 1;
    SparseGatherArgs<T> g{};
    g.CP = CP;
    g.nchunks = L.nchunks;
    g.chunk_grp = L.chunk_grp;
    g.chunk_beg = L.chunk_beg;
    g.chunk_end = L.chunk_end;
    g.chunk_whole = L.chunk_whole;
    g.col = st.sp_col;
    g.val = pick_prec<T>(st.sp_val32, st.sp_val64);
    g.x = x + st.lbase[0] * CP;
    g.out = q + st.lbase[0] * CP;
    g.partial = wk.sp_chunk_partial;
    g.dot_partial = wk.sp_gather_partial;
    if (coupled) {
        g.cfy = pick_prec<T>(st.cfy32, st.cfy64);
        g.xs = x + st.sbase[0] * CP;
        g.SG = st.SG;
        g.SGP = st.SGP;
    }
    {
        // chunk meta, nonzeros (column + value), the large dim's rows of x
        // read and of q written once, and the coupling rows
        const double tb = static_cast<double>(sizeof(T));
        double pb = static_cast<double>(L.nchunks) * 13.0 + static_cast<double>(st.sp_nnz) * (4.0 + tb) +
                    2.0 * static_cast<double>(L.G) * CP * tb;
        if (coupled) pb += static_cast<double>(L.G) * st.SGP * tb;
        ProfScope ps(ctx, B200FE_PROF_GATHER, pb);
        const size_t gsmem = coupled ? static_cast<size_t>(st.SGP) * CP * sizeof(T) : 0;
        sparse_gather_kernel<T, CQ><<<wk.sp_gather_grid, kRowThreads, gsmem, s>>>(g);
        B_LAUNCHED();
        if (L.nsup > 0) {
            multi_super_kernel<<<grid_for(ctx, L.nsup * CP, kRowThreads), kRowThreads, 0, s>>>(
                L.nsup, L.sup_c0, L.sup_c1, wk.sp_chunk_partial, CP, wk.sp_super_partial);
            B_LAUNCHED();
        }
    }
    FinalizeArgs<T> f{};
    f.CP = CP;
    f.nL = 1;
    f.nS = st.nS;
    f.nmulti[0] = L.nmulti;
    f.multi_grp[0] = L.multi_grp;
    f.multi_c0[0] = L.multi_c0;
    f.multi_c1[0] = L.multi_c1;
    f.partial[0] = wk.sp_chunk_partial;
    f.multi_s0[0] = L.multi_s0;
    f.multi_s1[0] = L.multi_s1;
    f.super_partial[0] = wk.sp_super_partial;
    f.lbase[0] = st.lbase[0];
    f.gather_dot_partial[0] = wk.sp_gather_partial;
    f.gather_ctas[0] = wk.sp_gather_grid;
    f.SG = st.SG;
    f.sgbase = st.nS > 0 ? st.sbase[0] : 0;
    f.bins_partial = wk.bins_partial;
    f.nbins_ctas = coupled ? wk.couple_grid : 0;
    f.small_diag = nullptr;
    f.small_dense = coupled ? st.cyy : nullptr;
    f.cfy = coupled ? pick_prec<T>(st.cfy32, st.cfy64) : nullptr;
    f.SGP = st.SGP;
    f.x = x;
    f.nrows = wk.sp_fin_rows;
    f.out = q;
    f.dotv = x;
    f.dot_partial = wk.fin_partial;
    f.dot_out = wk.dot_out;
    f.ticket = wk.ticket;
    double fb = static_cast<double>(f.nbins_ctas) * st.SG * CP * 8.0 +
                static_cast<double>(L.nmulti) * CP * (8.0 + sizeof(T)) +
                static_cast<double>(st.SG) * CP * sizeof(T);
    ProfScope ps(ctx, B200FE_PROF_FINALIZE, fb);
    finalize_kernel<T><<<wk.sp_fin_grid, kRowThreads, 0, s>>>(f);
    B_LAUNCHED();
    return B200FE_OK;
}

// q = S x ; pq = x'q (per column) into wk.dot_out
template <typename T, int CQ>
int matvec(b200fe_context* ctx, const Work<T>& wk, const T* wp, const T* run_w,
           const T* block_w, const T* x, T* q) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    if (st.sparse) {
        if (st.coupled && st.nS == 1) {
            // C_fy' x_f into the coupling partials (read by finalize)
            ProfScope ps(ctx, B200FE_PROF_COUPLE,
                         static_cast<double>(st.L[0].G) * (st.SGP + CP) * double(sizeof(T)) +
                             static_cast<double>(wk.couple_grid) * st.SG * CP * 8.0);
            coupling_xf_kernel<T, CQ><<<wk.couple_grid, 256, 0, ctx->stream>>>(
                st.L[0].G, st.SG, st.SGP, pick_prec<T>(st.cfy32, st.cfy64), x + st.lbase[0] * CP,
                wk.bins_partial);
            B_LAUNCHED();
        }
        return reduce_sparse<T, CQ>(ctx, wk, x, q);
    }
    PassArgs<T> a = make_pass_args<T>(st, 0, CP, wk);
    a.wp = wp;
    a.x = x;
    {
        double pb;
        if (wk.run_grid > 0 && st.coupled) {  // large-dim runs (segment meta, run meta + weight, R, x_f)
            pb = static_cast<double>(st.G[st.p]) * 16.0;
            if (st.nL == 1)
                pb += static_cast<double>(st.L[0].nruns) * (16.0 + sizeof(T) + CP * double(sizeof(T))) +
                      static_cast<double>(st.L[0].G) * CP * double(sizeof(T));
        } else if (wk.run_grid > 0) {  // block-level pass: per segment, run and block
            pb = static_cast<double>(st.G[st.p]) * 16.0 + static_cast<double>(st.GR) * CP * sizeof(T) +
                 static_cast<double>(st.nblocks) * (8.0 + (st.weighted ? sizeof(T) : 0.0));
            const int64_t npr = st.nL == 1 ? st.L[0].nruns : st.G[st.p];
            pb += static_cast<double>(npr) * (16.0 + sizeof(T));
            if (st.nL == 1) pb += static_cast<double>(st.L[0].nruns) * CP * double(sizeof(T));
        } else {
            pb = struct_obs_bytes(st, sizeof(T)) + runs_write_bytes(st, CP, sizeof(T)) +
                 static_cast<double>(st.GR) * CP * sizeof(T);
        }
        ProfScope ps(ctx, B200FE_PROF_PASS, pb);
        B_CHECK((launch_matvec_pass<T, CQ>(ctx, wk, a, run_w, block_w)));
    }
    if (wk.run_grid > 0 && st.coupled && st.nL == 1) {
        // C_fy' x_f into the bin partials (rows of C_fy and x_f once, partials written)
        ProfScope ps(ctx, B200FE_PROF_COUPLE,
                     static_cast<double>(st.L[0].G) * (st.SGP + CP) * double(sizeof(T)) +
                         static_cast<double>(wk.couple_grid) * st.SG * CP * 8.0);
        coupling_xf_kernel<T, CQ><<<wk.couple_grid, 256, 0, ctx->stream>>>(
            st.L[0].G, st.SG, st.SGP, pick_prec<T>(st.cfy32, st.cfy64), x + st.lbase[0] * CP,
            wk.bins_partial);
        B_LAUNCHED();
    }
    return reduce_runs<T, CQ>(ctx, wk, q, x, B200FE_PROF_GATHER, B200FE_PROF_FINALIZE,
                              wk.run_grid > 0, wk.run_grid > 0 && st.coupled);
}

struct ColState {
    double* rz;
    double* pq;
    double* rr;
    double* thr;
    double* beta;
    int* active;
    int* iters;
    double* partial;
    unsigned int* ticket;
    int* n_active;
};

// Inner PCG on S x = rhs (rows already in r), T precision.
// thr_host[c]: stop column c when r'r <= thr (0 or negative: column inactive).
template <typename T, int CQ>
int pcg(b200fe_context* ctx, const Work<T>& wk, const T* wp, const T* run_w, const T* block_w,
        const T* dinv, T* x, T* r, T* z,
        T* p, T* q, const std::vector<double>& thr_host, int max_iter, int check_interval,
        int* iters_out) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    const int64_t GR = st.GR;
    ColState cs{};
    B_CHECK(get_buf(ctx, "cs_rz", CP, &cs.rz));
    B_CHECK(get_buf(ctx, "cs_pq", CP, &cs.pq));
    B_CHECK(get_buf(ctx, "cs_rr", CP, &cs.rr));
    B_CHECK(get_buf(ctx, "cs_thr", CP, &cs.thr));
    B_CHECK(get_buf(ctx, "cs_beta", CP, &cs.beta));
    B_CHECK(get_buf(ctx, "cs_active", CP, &cs.active));
    B_CHECK(get_buf(ctx, "cs_iters", CP, &cs.iters));
    B_CHECK(get_buf(ctx, "cs_nactive", 1, &cs.n_active));
    B_CHECK(get_buf(ctx, "cs_ticket", 1, &cs.ticket));
    const int rgrid = grid_for(ctx, GR * CP, kRowThreads, 8);
    B_CHECK(get_buf(ctx, "cs_partial", static_cast<size_t>(rgrid) * 2 * CP, &cs.partial));
    std::vector<int> act(CP, 0);
    for (int c = 0; c < CP; ++c) act[c] = thr_host[c] > 0.0 ? 1 : 0;
    B_CHECK(small_h2d(ctx, cs.thr, thr_host.data(), sizeof(double) * CP));
    B_CHECK(small_h2d(ctx, cs.active, act.data(), sizeof(int) * CP));
    B_TRY(cudaMemsetAsync(cs.rz, 0, sizeof(double) * CP, s));
    B_TRY(cudaMemsetAsync(cs.pq, 0, sizeof(double) * CP, s));
    B_TRY(cudaMemsetAsync(cs.iters, 0, sizeof(int) * CP, s));
    B_TRY(cudaMemsetAsync(cs.ticket, 0, sizeof(unsigned int), s));
    B_TRY(cudaMemsetAsync(x, 0, sizeof(T) * GR * CP, s));
    B_TRY(cudaStreamSynchronize(s));  // act/thr host vectors are stack-owned

    CgScalars sc{};
    sc.rz = cs.rz;
    sc.pq = cs.pq;
    sc.rr = cs.rr;
    sc.bb = cs.thr;
    sc.beta = cs.beta;
    sc.active = cs.active;
    sc.iters = cs.iters;
    sc.partial = cs.partial;
    sc.ticket = cs.ticket;
    sc.n_active = cs.n_active;
    // z = M^-1 r, rz, rr; alpha = 0 because pq = 0
    cg_update_kernel<T><<<rgrid, kRowThreads, 0, s>>>(GR, CP, x, r, z, p, q, dinv, sc, 1.0, -1);
    B_LAUNCHED();
    cg_direction_kernel<T><<<rgrid, kRowThreads, 0, s>>>(GR, CP, p, z, sc, 1);
    B_LAUNCHED();
    // one block of nit iterations on ctx->stream: every scalar (alpha, beta,
    // the column masks) lives on the device, nothing is read back inside it
    auto run_block = [&](int nit) -> int {
        const cudaStream_t bs = ctx->stream;
        for (int j = 0; j < nit; ++j) {
            B_CHECK((matvec<T, CQ>(ctx, wk, wp, run_w, block_w, p, q)));
            // pq is in wk.dot_out: copy into the scalar slot
            B_TRY(cudaMemcpyAsync(cs.pq, wk.dot_out, sizeof(double) * CP, cudaMemcpyDeviceToDevice, bs));
            {
                ProfScope ps(ctx, B200FE_PROF_VECTOR,
                             static_cast<double>(GR) * (CP * 10.0 + 1.0) * sizeof(T));
                cg_update_kernel<T><<<rgrid, kRowThreads, 0, bs>>>(GR, CP, x, r, z, p, q, dinv, sc,
                                                                  1.0, 0);
                B_LAUNCHED();
                cg_direction_kernel<T><<<rgrid, kRowThreads, 0, bs>>>(GR, CP, p, z, sc, 0);
                B_LAUNCHED();
            }
        }
        return B200FE_OK;
    };
    // Full blocks after the first run as one CUDA graph: captured once per
    // call (the first block has allocated every buffer), the executable kept
    // in the context and updated in place when the next call's kernels match.
    // Without the event profiler only; any capture failure falls back to
    // plain launches.
    cudaGraphExec_t exec = nullptr;
    long long graph_launches = 0;
    bool graph_ok = ctx->graphs && !ctx->profiling;
    auto capture = [&]() {
        if (!ctx->cap_stream &&
            cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            ctx->cap_stream = nullptr;
            graph_ok = false;
            return;
        }
        if (cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            graph_ok = false;
            return;
        }
        const cudaStream_t saved = ctx->stream;
        const long long l0 = ctx->launches;
        const std::string err0 = ctx->err;
        ctx->stream = ctx->cap_stream;
        const int rc = run_block(check_interval);
        ctx->stream = saved;
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(ctx->cap_stream, &g);
        graph_launches = ctx->launches - l0;
        ctx->launches = l0;
        if (rc != B200FE_OK || ee != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            ctx->err = err0;
            graph_ok = false;
            return;
        }
        const int key = static_cast<int>(sizeof(T)) * 64 + CQ;
        auto found = ctx->graph_exec.find(key);
        if (found != ctx->graph_exec.end()) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(found->second, g, &info) == cudaSuccess) {
                exec = found->second;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(found->second);
                ctx->graph_exec.erase(found);
            }
        }
        if (!exec) {
            if (cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
                ctx->graph_exec[key] = exec;
            } else {
                cudaGetLastError();
                exec = nullptr;
                graph_ok = false;
            }
        }
        cudaGraphDestroy(g);
    };
    int it = 0;
    int na = 0;
    B_CHECK(sync_read_int(ctx, cs.n_active, 1, &na));
    while (na > 0 && it < max_iter) {
        const int block = std::min(check_interval, max_iter - it);
        if (graph_ok && !exec && it > 0 && block == check_interval) capture();
        if (exec && block == check_interval) {
            B_TRY(cudaGraphLaunch(exec, s));
            ctx->launches += graph_launches;
        } else {
            B_CHECK(run_block(block));
        }
        it += block;
        B_CHECK(sync_read_int(ctx, cs.n_active, 1, &na));
    }
    *iters_out = it;
    return B200FE_OK;
}

// Algorithmic bytes of one persistent PCG iteration: the explicit block
// (column and value per nonzero, row offsets, the p rows gathered and the q
// rows written once), the coupling rows, and the vector updates (x, r, z, p,
// q, dinv read; x, r, z written; z, p read and p written for the directions).
double pcg_iter_bytes(const Structure& st, int CP, size_t tsize) {
    const double tb = static_cast<double>(tsize);
    const double gf = static_cast<double>(st.L[0].G);
    const double gr = static_cast<double>(st.GR);
    double b = static_cast<double>(st.sp_nnz) * (4.0 + tb) + gf * 4.0 + 2.0 * gf * CP * tb;
    if (st.coupled && st.nS == 1) b += gf * st.SGP * tb;
    b += gr * CP * tb * 11.0 + gr * tb;
    return b;
}

// Inner PCG as one cooperative launch (pcg_kernels.cuh).  Returns
// B200FE_UNAVAILABLE (nothing run) when the launch cannot be made, so the
// caller falls back to the multi-kernel PCG.
template <typename T, int CQ>
int pcg_persistent(b200fe_context* ctx, const Work<T>& wk, const T* dinv, T* x, T* r, T* z, T* p,
                   T* q, const std::vector<double>& thr_host, int max_iter, int* iters_out) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    const bool coupled = st.coupled && st.nS == 1;
    const int SG = coupled ? st.SG : 0;
    const int SGP = coupled ? st.SGP : 0;
    if (SG > kPcgMaxSG) return B200FE_UNAVAILABLE;
    const size_t smem = pcg_smem_bytes<T>(CP, SGP);
    auto kern = pcg_persistent_kernel<T, CQ>;
    B_TRY(raise_smem_limit(reinterpret_cast<const void*>(kern), static_cast<int>(smem)));
    int per_sm = 0;
    B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPcgThreads, smem));
    if (per_sm < 1) return B200FE_UNAVAILABLE;
    const int nb = ctx->num_sms * std::min(per_sm, 2);
    PcgArgs<T> a{};
    a.CP = CP;
    a.Gf = st.L[0].G;
    a.SG = SG;
    a.SGP = SGP;
    a.row_off = st.sp_row_off;
    a.col = st.sp_col;
    a.val = pick_prec<T>(st.sp_val32, st.sp_val64);
    a.nshort = st.pc_nshort;
    a.short_meta = st.pc_short_meta;
    a.nlchunks = st.pc_nlchunks;
    a.lchunk_meta = st.pc_lchunk_meta;
    a.nlong = st.pc_nlong;
    a.long_rows = st.pc_long_rows;
    a.long_c0 = st.pc_long_c0;
    a.long_c1 = st.pc_long_c1;
    a.nhuge = st.pc_nhuge;
    a.huge_li = st.pc_huge_li;
    a.cfy = coupled ? pick_prec<T>(st.cfy32, st.cfy64) : nullptr;
    a.cyy = coupled ? st.cyy : nullptr;
    a.dinv = dinv;
    a.x = x;
    a.r = r;
    a.z = z;
    a.p = p;
    a.q = q;
    a.part_stride = CP * (3 + SG);
    a.max_iter = max_iter;
    const std::string tag = std::is_same<T, float>::value ? "pc32_" : "pc64_";
    B_CHECK(get_buf(ctx, tag + "lpart", static_cast<size_t>(std::max<int64_t>(st.pc_nlchunks, 1)) * CP, &a.lpart));
    B_CHECK(get_buf(ctx, tag + "cta_part", static_cast<size_t>(nb) * a.part_stride, &a.cta_part));
    double* thr_d;
    B_CHECK(get_buf(ctx, tag + "thr", CP, &thr_d));
    B_CHECK(get_buf(ctx, tag + "rz", CP, &a.rz_out));
    int32_t *iters_d, *ctl;
    B_CHECK(get_buf(ctx, tag + "iters", CP, &iters_d));
    B_CHECK(get_buf(ctx, tag + "ctl", 4, &ctl));  // loops, status, barrier[2]
    a.iters_out = iters_d;
    a.loops_out = ctl;
    a.status = ctl + 1;
    a.bar = reinterpret_cast<unsigned int*>(ctl + 2);
    a.thr = thr_d;
    B_CHECK(small_h2d(ctx, thr_d, thr_host.data(), sizeof(double) * CP));
    B_TRY(cudaMemsetAsync(ctl, 0, 4 * sizeof(int32_t), s));
    void* args[] = {&a};
    {
        ProfScope ps(ctx, B200FE_PROF_PASS, 0.0);
        const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(nb),
                                                          dim3(kPcgThreads), args, smem, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            B_TRY(cudaStreamSynchronize(s));  // thr_host copy done before the caller's fallback
            return B200FE_UNAVAILABLE;
        }
        ++ctx->launches;
        int hc[2] = {0, 0};
        B_CHECK(sync_read_int(ctx, ctl, 2, hc));
        if (hc[1] != 0) {
            ctx->err = "persistent PCG: grid barrier wait timed out";
            return B200FE_CUDA_ERROR;
        }
        *iters_out = hc[0];
        ps.bytes = static_cast<double>(hc[0]) * pcg_iter_bytes(st, CP, sizeof(T));
    }
    return B200FE_OK;
}

// Learned warm start (ws_kernels.cuh): the Jacobi iterates a1..a3 of S a = b
// in FP64, the column scales and the network's features [GR * cols][8].
template <int CQ>
int ws_features(b200fe_context* ctx, const Work<double>& w64, const double* b64, int cols, double* q64,
                double* dot_part, unsigned int* dot_ticket, double* dot_res, double** a1o, double** a3o,
                double** sigmao, float** feato) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    const int64_t GR = st.GR;
    double *a1, *a2, *a3, *sigma;
    float* feat;
    B_CHECK(get_buf(ctx, "ws_a1", GR * CP, &a1));
    B_CHECK(get_buf(ctx, "ws_a2", GR * CP, &a2));
    B_CHECK(get_buf(ctx, "ws_a3", GR * CP, &a3));
    B_CHECK(get_buf(ctx, "ws_sigma", CP, &sigma));
    B_CHECK(get_buf(ctx, "ws_feat", static_cast<size_t>(GR) * cols * kWsFeatures, &feat));
    const int g = grid_for(ctx, GR * CP, 256);
    ws_jacobi_kernel<<<g, 256, 0, s>>>(GR, CP, nullptr, b64, nullptr, st.dinv64, a1);
    B_LAUNCHED();
    B_CHECK((matvec<double, CQ>(ctx, w64, st.wp64, st.run_w64, st.block_w64, a1, q64)));
    ws_jacobi_kernel<<<g, 256, 0, s>>>(GR, CP, a1, b64, q64, st.dinv64, a2);
    B_LAUNCHED();
    B_CHECK((matvec<double, CQ>(ctx, w64, st.wp64, st.run_w64, st.block_w64, a2, q64)));
    ws_jacobi_kernel<<<g, 256, 0, s>>>(GR, CP, a2, b64, q64, st.dinv64, a3);
    B_LAUNCHED();
    const int rgrid = grid_for(ctx, std::max<int64_t>(GR, 1) * CP, kRowThreads, 8);
    row_dot_kernel<double, double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, a1, a1, dot_part, dot_ticket, dot_res);
    B_LAUNCHED();
    ws_sigma_kernel<<<1, 32, 0, s>>>(dot_res, GR, CP, sigma);
    B_LAUNCHED();
    ws_features_kernel<<<grid_for(ctx, GR * cols, 256), 256, 0, s>>>(
        GR, CP, cols, a1, a2, a3, sigma, st.w_rows, st.dinv64, st.nS > 0 ? st.sbase[0] : GR, feat);
    B_LAUNCHED();
    *a1o = a1;
    *a3o = a3;
    *sigmao = sigma;
    *feato = feat;
    return B200FE_OK;
}

template <int CQ>
int solve_block(b200fe_context* ctx, const double* d_v, int cols, double* d_out,
                const b200fe_options& o, b200fe_result* res) {
    const Structure& st = ctx->st;
    constexpr int CP = 4 * CQ;
    const cudaStream_t s = ctx->stream;
    const int64_t GR = st.GR;
    Work<double> w64{};
    B_CHECK(prepare_work<double, CQ>(ctx, "w64_", w64));
    const bool mixed = (o.precision == B200FE_PREC_MIXED) && GR > 0;
    Work<float> w32{};
    if (mixed) B_CHECK(prepare_work<float, CQ>(ctx, "w32_", w32));

    double *b64, *a64, *r64, *q64, *z64 = nullptr, *p64 = nullptr, *x64 = nullptr,
           *rin64 = nullptr;
    B_CHECK(get_buf(ctx, "b64", GR * CP, &b64));
    B_CHECK(get_buf(ctx, "a64", GR * CP, &a64));
    B_CHECK(get_buf(ctx, "r64", GR * CP, &r64));
    B_CHECK(get_buf(ctx, "q64", GR * CP, &q64));
    float *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *q32 = nullptr;
    if (mixed) {
        B_CHECK(get_buf(ctx, "x32", GR * CP, &x32));
        B_CHECK(get_buf(ctx, "r32", GR * CP, &r32));
        B_CHECK(get_buf(ctx, "z32", GR * CP, &z32));
        B_CHECK(get_buf(ctx, "p32", GR * CP, &p32));
        B_CHECK(get_buf(ctx, "q32", GR * CP, &q32));
    } else {
        B_CHECK(get_buf(ctx, "rin64", GR * CP, &rin64));
        B_CHECK(get_buf(ctx, "x64", GR * CP, &x64));
        B_CHECK(get_buf(ctx, "z64", GR * CP, &z64));
        B_CHECK(get_buf(ctx, "p64", GR * CP, &p64));
    }
    double *scale_d, *inv_scale_d, *dot_part;
    unsigned int* dot_ticket;
    double* dot_res;
    B_CHECK(get_buf(ctx, "scale_d", CP, &scale_d));
    B_CHECK(get_buf(ctx, "inv_scale_d", CP, &inv_scale_d));
    const int rgrid = grid_for(ctx, std::max<int64_t>(GR, 1) * CP, kRowThreads, 8);
    B_CHECK(get_buf(ctx, "rowdot_part", static_cast<size_t>(rgrid) * CP, &dot_part));
    B_CHECK(get_buf(ctx, "rowdot_ticket", 1, &dot_ticket));
    B_CHECK(get_buf(ctx, "rowdot_res", CP, &dot_res));
    B_TRY(cudaMemsetAsync(dot_ticket, 0, sizeof(unsigned int), s));

    // 1. RHS pass: b = D_r' W (I - P_p) v ; ||v||^2 per column
    {
        PassArgs<double> a = make_pass_args<double>(st, cols, CP, w64);
        a.wp = st.wp64;
        a.v = d_v;
        ProfScope ps(ctx, B200FE_PROF_RHS,
                     static_cast<double>(st.n) * cols * 8.0 + struct_obs_bytes(st, 8) +
                         runs_write_bytes(st, CP, 8));
        B_CHECK((launch_pass<double, CQ, kRhs>(ctx, w64, a)));
    }
    std::vector<double> vnorm2(CP, 0.0);
    {
        std::vector<double> hp(static_cast<size_t>(w64.nbins_ctas) * CP);
        if (GR > 0)
            B_CHECK(reduce_runs<double, CQ>(ctx, w64, b64, nullptr, B200FE_PROF_RHS, B200FE_PROF_RHS));
        B_CHECK(small_d2h(ctx, w64.colsq_partial, sizeof(double) * hp.size(), hp.data()));
        for (int b = 0; b < w64.nbins_ctas; ++b)
            for (int c = 0; c < CP; ++c) vnorm2[c] += hp[static_cast<size_t>(b) * CP + c];
    }

    int total_iters = 0, outer = 0;
    bool converged = true;
    const double* dinv64_use = st.dinv64;  // Jacobi diagonal (scaled by the learned warm start)
    const float* dinv32_use = st.dinv32;
    double rel_res = 0.0;
    std::vector<double> bb(CP, 0.0), rr(CP, 0.0);
    if (GR > 0) {
        row_dot_kernel<double, double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, b64, b64, dot_part,
                                                                     dot_ticket, dot_res);
        B_LAUNCHED();
        B_CHECK(sync_read_double(ctx, dot_res, CP, bb.data()));
        B_TRY(cudaMemsetAsync(a64, 0, sizeof(double) * GR * CP, s));
        B_TRY(cudaMemcpyAsync(r64, b64, sizeof(double) * GR * CP, cudaMemcpyDeviceToDevice, s));
        rr = bb;
        // learned warm start: start from the network's prediction (columns
        // whose predicted start has a larger residual than zero start cold),
        // optionally with its per-row scaling of the Jacobi diagonal
        if (ctx->ws_mode != 0 && ctx->ws_packed) {
            ProfScope ps(ctx, B200FE_PROF_SETUP, 0.0);
            double *wa1, *wa3, *wsig;
            float *feat, *wy;
            B_CHECK(ws_features<CQ>(ctx, w64, b64, cols, q64, dot_part, dot_ticket, dot_res, &wa1, &wa3,
                                    &wsig, &feat));
            B_CHECK(get_buf(ctx, "ws_y", static_cast<size_t>(GR) * cols * 2, &wy));
            B_CHECK(mlp_forward_device(ctx, ctx->ws_packed, feat, GR * cols, wy));
            if (ctx->ws_mode & 1) {
                double* a0;
                B_CHECK(get_buf(ctx, "ws_a0", GR * CP, &a0));
                ws_apply_kernel<<<grid_for(ctx, GR * CP, 256), 256, 0, s>>>(GR, CP, cols, wa3, wsig, wy, a0);
                B_LAUNCHED();
                B_CHECK((matvec<double, CQ>(ctx, w64, st.wp64, st.run_w64, st.block_w64, a0, q64)));
                double* r0;
                B_CHECK(get_buf(ctx, "ws_r0", GR * CP, &r0));
                sub_kernel<<<rgrid, kRowThreads, 0, s>>>(GR * CP, b64, q64, r0);
                B_LAUNCHED();
                row_dot_kernel<double, double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, r0, r0, dot_part,
                                                                             dot_ticket, dot_res);
                B_LAUNCHED();
                std::vector<double> r0r0(CP, 0.0);
                B_CHECK(sync_read_double(ctx, dot_res, CP, r0r0.data()));
                for (int c = 0; c < cols && c < CP; ++c) {
                    if (!(r0r0[c] < bb[c])) continue;  // keep the cold start of this column
                    B_TRY(cudaMemcpy2DAsync(a64 + c, CP * sizeof(double), a0 + c, CP * sizeof(double),
                                            sizeof(double), GR, cudaMemcpyDeviceToDevice, s));
                    B_TRY(cudaMemcpy2DAsync(r64 + c, CP * sizeof(double), r0 + c, CP * sizeof(double),
                                            sizeof(double), GR, cudaMemcpyDeviceToDevice, s));
                    rr[c] = r0r0[c];
                    ++res->warm_columns;
                }
            }
            if (ctx->ws_mode & 2) {
                double* d64s;
                float* d32s;
                B_CHECK(get_buf(ctx, "ws_dinv64", GR, &d64s));
                B_CHECK(get_buf(ctx, "ws_dinv32", GR, &d32s));
                ws_scale_kernel<<<grid_for(ctx, GR, 256), 256, 0, s>>>(GR, cols, wy, st.dinv64, d64s, d32s);
                B_LAUNCHED();
                dinv64_use = d64s;
                dinv32_use = d32s;
            }
        }
        const double tol = o.tol;
        // Stop column c when ||r_c||^2 <= thr_c = max(tol^2 ||b_c||^2, floor_c^2).
        // The floor, 1e3 eps ||D'W||_F ||v_c||, sits four orders of magnitude
        // below the certificate limit; it only binds for a column (almost) in
        // the span of the FEs, whose b_c is rounding noise that partly lies in
        // the null space of S and cannot be reduced relative to itself.
        std::vector<double> thr64(CP, 0.0);
        {
            const double fl = 1e3 * std::numeric_limits<double>::epsilon();
            const double opn2 = static_cast<double>(st.D) * st.sum_w2;
            for (int c = 0; c < cols && c < CP; ++c)
                thr64[c] = std::max(tol * tol * bb[c], fl * fl * opn2 * vnorm2[c]);
        }
        // fe_linf_tol: the largest group mean of the within transform, per column
        const bool linf_on = o.fe_linf_tol > 0.0 && st.w_rows != nullptr;
        std::vector<double> linf(CP, 0.0);
        unsigned long long* linf_d = nullptr;
        if (linf_on) B_CHECK(get_buf(ctx, "linf_bits", CP, &linf_d));
        auto read_linf = [&]() -> int {
            B_TRY(cudaMemsetAsync(linf_d, 0, sizeof(unsigned long long) * CP, s));
            row_linf_kernel<<<rgrid, kRowThreads, 0, s>>>(GR, CP, cols, r64, st.w_rows, linf_d);
            B_LAUNCHED();
            std::vector<unsigned long long> bits(CP);
            B_CHECK(small_d2h(ctx, linf_d, sizeof(unsigned long long) * CP, bits.data()));
            for (int c = 0; c < CP; ++c) std::memcpy(&linf[c], &bits[c], sizeof(double));
            return B200FE_OK;
        };
        if (linf_on) B_CHECK(read_linf());
        // rounds driven by the group-mean bound alone get a bounded inner budget,
        // and one that raises the residual (its rhs was rounding noise) is undone
        double* a_prev = nullptr;
        double* r_prev = nullptr;
        if (linf_on) {
            B_CHECK(get_buf(ctx, "a64_prev", GR * CP, &a_prev));
            B_CHECK(get_buf(ctx, "r64_prev", GR * CP, &r_prev));
        }
        int first_round_its = 0;
        bool linf_stuck = false;
        const int max_outer = std::max(1, o.max_outer);
        converged = false;
        for (outer = 0; outer < max_outer; ++outer) {
            bool all = true, linf_only = true;
            std::vector<double> scale(CP, 0.0), inv_scale(CP, 0.0), thr(CP, 0.0);
            for (int c = 0; c < cols && c < CP; ++c) {
                const bool l2_done = !(rr[c] > thr64[c]);
                const bool linf_done = !linf_on || linf_stuck || !(linf[c] > o.fe_linf_tol);
                if (!(l2_done && linf_done) && rr[c] > 0.0) {
                    all = false;
                    if (!l2_done) linf_only = false;
                    scale[c] = std::sqrt(rr[c]);
                    inv_scale[c] = 1.0 / scale[c];
                    // inner target relative to this round's rhs
                    double t_in = l2_done ? 0.5 : 0.5 * std::sqrt(thr64[c] / rr[c]);
                    if (!linf_done) t_in = std::min(t_in, 0.1 * o.fe_linf_tol / linf[c]);
                    if (mixed) t_in = std::max(t_in, o.inner_tol);
                    t_in = std::min(t_in, 0.5);
                    thr[c] = t_in * t_in;  // rhs is normalised to unit norm
                }
            }
            if (all) {
                converged = true;
                break;
            }
            if (total_iters >= o.max_iter) break;
            int round_cap = o.max_iter - total_iters;
            const std::vector<double> rr_before = rr;
            if (linf_on && linf_only) {
                round_cap = std::min(round_cap, std::max(50, 2 * first_round_its));
                B_TRY(cudaMemcpyAsync(a_prev, a64, sizeof(double) * GR * CP, cudaMemcpyDeviceToDevice, s));
                B_TRY(cudaMemcpyAsync(r_prev, r64, sizeof(double) * GR * CP, cudaMemcpyDeviceToDevice, s));
            }
            B_CHECK(small_h2d(ctx, scale_d, scale.data(), sizeof(double) * CP));
            B_CHECK(small_h2d(ctx, inv_scale_d, inv_scale.data(), sizeof(double) * CP));
            int its = 0;
            if (mixed) {
                scale_rows_kernel<float><<<rgrid, kRowThreads, 0, s>>>(GR, CP, r64, inv_scale_d, r32);
                B_LAUNCHED();
                int prc = B200FE_UNAVAILABLE;
                if (st.sparse && ctx->persistent)
                    prc = pcg_persistent<float, CQ>(ctx, w32, dinv32_use, x32, r32, z32, p32, q32, thr,
                                                    round_cap, &its);
                if (prc == B200FE_UNAVAILABLE)
                    B_CHECK((pcg<float, CQ>(ctx, w32, st.wp32, st.run_w32, st.block_w32, dinv32_use, x32, r32, z32, p32, q32, thr,
                                            round_cap, std::max(1, o.check_interval),
                                            &its)));
                else if (prc != B200FE_OK)
                    return prc;
                axpy_rows_kernel<float><<<rgrid, kRowThreads, 0, s>>>(GR, CP, x32, scale_d, a64);
                B_LAUNCHED();
            } else {
                scale_rows_kernel<double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, r64, inv_scale_d, rin64);
                B_LAUNCHED();
                int prc = B200FE_UNAVAILABLE;
                if (st.sparse && ctx->persistent)
                    prc = pcg_persistent<double, CQ>(ctx, w64, dinv64_use, x64, rin64, z64, p64, q64, thr,
                                                     round_cap, &its);
                if (prc == B200FE_UNAVAILABLE)
                    B_CHECK((pcg<double, CQ>(ctx, w64, st.wp64, st.run_w64, st.block_w64, dinv64_use, x64, rin64, z64, p64, q64, thr,
                                             round_cap, std::max(1, o.check_interval),
                                             &its)));
                else if (prc != B200FE_OK)
                    return prc;
                axpy_rows_kernel<double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, x64, scale_d, a64);
                B_LAUNCHED();
            }
            total_iters += its;
            // true residual in FP64: r = b - S a
            B_CHECK((matvec<double, CQ>(ctx, w64, st.wp64, st.run_w64, st.block_w64, a64, q64)));
            sub_kernel<<<rgrid, kRowThreads, 0, s>>>(GR * CP, b64, q64, r64);
            B_LAUNCHED();
            row_dot_kernel<double, double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, r64, r64, dot_part,
                                                                         dot_ticket, dot_res);
            B_LAUNCHED();
            B_CHECK(sync_read_double(ctx, dot_res, CP, rr.data()));
            if (outer == 0) first_round_its = its;
            if (linf_on && linf_only) {
                bool worse = false;
                for (int c = 0; c < cols && c < CP; ++c) worse = worse || rr[c] > rr_before[c];
                if (worse) {  // the bound is below what rounding allows: keep the last a
                    B_TRY(cudaMemcpyAsync(a64, a_prev, sizeof(double) * GR * CP, cudaMemcpyDeviceToDevice, s));
                    B_TRY(cudaMemcpyAsync(r64, r_prev, sizeof(double) * GR * CP, cudaMemcpyDeviceToDevice, s));
                    rr = rr_before;
                    linf_stuck = true;
                    continue;
                }
            }
            if (linf_on) B_CHECK(read_linf());
        }
        if (!converged) {
            bool all = true;
            for (int c = 0; c < cols && c < CP; ++c) {
                if (rr[c] > thr64[c]) all = false;
                if (linf_on && !linf_stuck && linf[c] > o.fe_linf_tol && rr[c] > 0.0) all = false;
            }
            converged = all;
        }
        // residual relative to the scale the stop rule uses (||b_c|| or the floor)
        for (int c = 0; c < cols && c < CP; ++c)
            if (thr64[c] > 0.0) rel_res = std::max(rel_res, tol * std::sqrt(rr[c] / thr64[c]));
    }

    // training samples of the learned warm start (b200fe_warmstart_samples):
    // features of this right-hand side and targets from the converged a
    if (ctx->ws_feat && GR > 0) {
        double *wa1, *wa3, *wsig;
        float* feat;
        B_CHECK(ws_features<CQ>(ctx, w64, b64, cols, q64, dot_part, dot_ticket, dot_res, &wa1, &wa3, &wsig,
                                &feat));
        const int64_t ns = GR * cols;
        if (ctx->ws_count + ns > ctx->ws_cap) {
            ctx->err = "warm-start sample capacity exceeded";
            return B200FE_INVALID_ARG;
        }
        B_TRY(cudaMemcpyAsync(ctx->ws_feat + ctx->ws_count * kWsFeatures, feat,
                              sizeof(float) * ns * kWsFeatures, cudaMemcpyDeviceToDevice, s));
        ws_targets_kernel<<<grid_for(ctx, ns, 256), 256, 0, s>>>(GR, CP, cols, a64, wa1, wa3, wsig,
                                                                 ctx->ws_targ + ctx->ws_count * 4);
        B_LAUNCHED();
        ctx->ws_count += ns;
    }

    // final pass: out = (I - P_p)(v - D_r a); certificate scatter; with saved
    // FEs also the primary segment means (the primary dim's coefficients)
    const bool cert = o.certify != 0;
    const bool save_fe = ctx->fe_dev[0] != nullptr;
    double* means = nullptr;
    if (save_fe) {
        B_CHECK(get_buf(ctx, "fe_means", static_cast<size_t>(st.G[st.p]) * CP, &means));
        B_TRY(cudaMemsetAsync(means, 0, sizeof(double) * st.G[st.p] * CP, s));
    }
    {
        PassArgs<double> a = make_pass_args<double>(st, cols, CP, w64);
        a.wp = st.wp64;
        a.v = d_v;
        a.out = d_out;
        a.x = a64;
        a.scatter = cert ? 1 : 0;
        a.mean_out = means;
        ProfScope ps(ctx, B200FE_PROF_FINAL,
                     static_cast<double>(st.n) * cols * 16.0 + struct_obs_bytes(st, 8) +
                         static_cast<double>(GR) * CP * 8.0 +
                         (cert ? runs_write_bytes(st, CP, 8) : 0.0));
        B_CHECK((launch_pass<double, CQ, kFinal>(ctx, w64, a)));
    }
    B_CHECK(check_stream_status(ctx));
    double abs_res = 0.0, abs_rel = 0.0;
    if (cert) {
        std::vector<double> hp(static_cast<size_t>(w64.nbins_ctas) * CP);
        std::vector<double> res2(CP, 0.0);
        if (GR > 0) {
            B_CHECK(reduce_runs<double, CQ>(ctx, w64, q64, nullptr, B200FE_PROF_FINAL,
                                            B200FE_PROF_FINAL));
            row_dot_kernel<double, double><<<rgrid, kRowThreads, 0, s>>>(GR, CP, q64, q64, dot_part,
                                                                         dot_ticket, dot_res);
            B_LAUNCHED();
            B_CHECK(sync_read_double(ctx, dot_res, CP, res2.data()));
        }
        B_CHECK(small_d2h(ctx, w64.colsq_partial, sizeof(double) * hp.size(), hp.data()));
        for (int b = 0; b < w64.nbins_ctas; ++b)
            for (int c = 0; c < CP; ++c) res2[c] += hp[static_cast<size_t>(b) * CP + c];
        const double opn = std::sqrt(static_cast<double>(st.D) * st.sum_w2);
        for (int c = 0; c < cols; ++c) {
            const double ab = std::sqrt(std::max(0.0, res2[c]));
            const double sc = opn * std::sqrt(std::max(0.0, vnorm2[c]));
            double rel = 0.0;
            if (sc > 0.0) rel = ab / sc;
            else if (ab > 0.0) rel = std::numeric_limits<double>::max();
            abs_res = std::max(abs_res, ab);
            abs_rel = std::max(abs_rel, rel);
        }
    }
    if (save_fe) {
        FeLayoutArgs f{};
        f.nd = st.D;
        for (int d = 0; d < st.D; ++d) {
            f.G[d] = st.G[d];
            f.out[d] = ctx->fe_dev[d];
            f.row0[d] = d == st.p ? -1 : -2;
        }
        for (int l = 0; l < st.nL; ++l) f.row0[st.L[l].dim] = st.lbase[l];
        for (int j = 0; j < st.nS; ++j) f.row0[st.sdim[j]] = st.sbase[j];
        f.cols_total = ctx->fe_cols;
        f.c0 = ctx->fe_c0;
        f.cb = cols;
        f.CP = CP;
        f.a = a64;
        f.means = means;
        fe_layout_kernel<<<grid_for(ctx, static_cast<int64_t>(st.n) + GR, 256), 256, 0, s>>>(f);
        B_LAUNCHED();
    }
    B_TRY(cudaStreamSynchronize(s));
    res->iterations += total_iters;
    res->outer_iterations = std::max(res->outer_iterations, outer);
    res->converged = res->converged && converged;
    res->rel_residual = std::max(res->rel_residual, rel_res);
    res->abs_residual = std::max(res->abs_residual, abs_res);
    res->abs_residual_rel = std::max(res->abs_residual_rel, abs_rel);
    return B200FE_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {


template <int CQ>
int solve_dispatch_cq(b200fe_context* ctx, const double* d_v, int cols, double* d_out,
                      const b200fe_options& o, b200fe_result* res) {
    return solve_block<CQ>(ctx, d_v, cols, d_out, o, res);
}

int solve_all(b200fe_context* ctx, const double* d_v, int cols, double* d_out,
              const b200fe_options& o, b200fe_result* res) {
    const int64_t n = ctx->st.n;
    // column blocks of at most 16 (CP <= 16 bounds the staged tile in shared memory)
    for (int c0 = 0; c0 < cols; c0 += 16) {
        const int cb = std::min(16, cols - c0);
        const double* v = d_v + static_cast<int64_t>(c0) * n;
        double* out = d_out + static_cast<int64_t>(c0) * n;
        const int cq = (cb + 3) / 4;
        ctx->fe_c0 = c0;
        int rc;
        if (cq <= 1) rc = solve_dispatch_cq<1>(ctx, v, cb, out, o, res);
        else if (cq <= 2) rc = solve_dispatch_cq<2>(ctx, v, cb, out, o, res);
        else rc = solve_dispatch_cq<4>(ctx, v, cb, out, o, res);
        if (rc != B200FE_OK) return rc;
    }
    return B200FE_OK;
}



int absorb_device_impl(b200fe_context* ctx, const double* d_v, int64_t n, int cols, int num_dims,
                       const int32_t* const* d_gids, const int32_t* G, const double* d_w,
                       const b200fe_options& o, double* d_out, b200fe_result* res) {
    const cudaStream_t s = ctx->stream;
    if (num_dims == 0) {
        if (d_out != d_v)
            B_TRY(cudaMemcpyAsync(d_out, d_v, sizeof(double) * n * cols, cudaMemcpyDeviceToDevice, s));
        B_TRY(cudaStreamSynchronize(s));
        res->converged = 1;
        res->precision_certified = 1;
        return B200FE_OK;
    }
    cudaEvent_t e0, e1, e2;
    B_TRY(cudaEventCreate(&e0));
    B_TRY(cudaEventCreate(&e1));
    B_TRY(cudaEventCreate(&e2));
    B_TRY(cudaEventRecord(e0, s));
    const bool reuse = o.reuse_structure && ctx->st.valid && ctx->st.n == n &&
                       ctx->st.D == num_dims && ctx->st.weighted == (d_w != nullptr);
    ctx->profiling = o.profile != 0;
    // 3: the run-level matvec of the automatic choice, without the explicit block
    ctx->pass_kernel = o.pass_kernel == 3 ? 0 : o.pass_kernel;
    ctx->sparse_schur = o.pass_kernel == 0;
    ctx->prof.clear();
    ctx->ev_used = 0;
    if (!reuse) {
        int rc;
        {
            ProfScope ps(ctx, B200FE_PROF_SETUP, 0.0);
            rc = build_structure(ctx, n, num_dims, d_gids, G, d_w);
        }
        if (rc != B200FE_OK) {
            ctx->st.valid = false;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaEventDestroy(e2);
            return rc;
        }
    }
    B_TRY(cudaEventRecord(e1, s));
    res->converged = 1;
    int rc = solve_all(ctx, d_v, cols, d_out, o, res);
    B_TRY(cudaEventRecord(e2, s));
    B_TRY(cudaEventSynchronize(e2));
    res->setup_ms = reuse ? 0.0 : elapsed_ms(e0, e1);
    res->solve_ms = elapsed_ms(e1, e2);
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
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (rc != B200FE_OK) return rc;
    res->primary_dim = ctx->st.p;
    for (int d = 0; d < num_dims; ++d) res->num_levels_present[d] = ctx->st.present[d];
    const double limit = std::max(8.0 * std::max(0.0, tol_eff(o)),
                                  64.0 * std::numeric_limits<double>::epsilon());
    res->precision_certified =
        res->converged && (o.certify ? res->abs_residual_rel <= limit : 1);
    return res->converged ? B200FE_OK : B200FE_NOT_CONVERGED;
}


// Host arrays in and out with the copies overlapped: the ids (and weights)
// go in first, then the columns in groups (two columns, then kPipeCols) on
// the copy-in stream; the compute stream builds the FE structure as soon as
// the ids are in and solves group after group on it, each group waiting for its own
// columns; each group's within transform goes out on the copy-out stream as
// soon as its solve is done, while later groups are still coming in (PCIe
// copies in both directions at once).  Every group is solved to the same
// tolerance as one batched call; results merge: iterations, rounds and
// residuals as maxima over the groups, converged and certified only if every
// group is, setup and solve times summed.
constexpr int kPipeCols = 4;
// Large copies are issued in pieces of this size: the solver's own small
// device<->host reads share the copy engines with them, and a read queued
// behind a whole gigabyte-sized copy would stall the compute stream until it
// finished.
constexpr size_t kCopyPiece = size_t(8) << 20;

int copy_pieces(b200fe_context* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                cudaStream_t st) {
    for (size_t o = 0; o < bytes; o += kCopyPiece)
        B_TRY(cudaMemcpyAsync(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o,
                              std::min(kCopyPiece, bytes - o), kind, st));
    return B200FE_OK;
}

int absorb_host_pipelined(b200fe_context* ctx, const double* y, const double* X, int64_t n, int k,
                          int num_dims, const int32_t* const* group_ids, const int32_t* G,
                          const double* weights, const b200fe_options& o, double* y_out, double* X_out,
                          b200fe_result* r) {
    const cudaStream_t s = ctx->stream;
    const int cols = k + 1;
    for (cudaStream_t* cs : {&ctx->copy_in, &ctx->copy_out})
        if (!*cs) B_TRY(cudaStreamCreateWithFlags(cs, cudaStreamNonBlocking));
    const cudaStream_t sin = ctx->copy_in, sout = ctx->copy_out;
    double *dv, *dout, *dw = nullptr;
    B_CHECK(get_buf(ctx, "io_v", static_cast<size_t>(n) * cols, &dv));
    B_CHECK(get_buf(ctx, "io_out", static_cast<size_t>(n) * cols, &dout));
    int32_t* dg[B200FE_MAX_DIMS] = {nullptr};
    for (int d = 0; d < num_dims; ++d) B_CHECK(get_buf(ctx, "io_g" + std::to_string(d), n, &dg[d]));
    if (weights) B_CHECK(get_buf(ctx, "io_w", n, &dw));
    B_TRY(cudaStreamSynchronize(s));  // buffers may have been reallocated
    // column groups: a small first group (its output copies can start early),
    // then groups of kPipeCols
    std::vector<int> gb{0};
    gb.push_back(std::min(cols, 2));
    while (gb.back() < cols) gb.push_back(std::min(cols, gb.back() + kPipeCols));
    const int ngroups = static_cast<int>(gb.size()) - 1;
    std::vector<cudaEvent_t> ev_in(ngroups), ev_done(ngroups);
    cudaEvent_t h0, h1, d0, d1;
    for (auto* e : {&h0, &h1, &d0, &d1}) B_TRY(cudaEventCreate(e));
    for (int g = 0; g < ngroups; ++g) {
        B_TRY(cudaEventCreateWithFlags(&ev_in[g], cudaEventDisableTiming));
        B_TRY(cudaEventCreateWithFlags(&ev_done[g], cudaEventDisableTiming));
    }
    auto host_col = [&](int c) { return c == 0 ? y : X + static_cast<int64_t>(c - 1) * n; };
    auto out_col = [&](int c) { return c == 0 ? y_out : X_out + static_cast<int64_t>(c - 1) * n; };
    // copies in: ids and weights, then the column groups
    cudaEvent_t ev_ids;
    B_TRY(cudaEventCreateWithFlags(&ev_ids, cudaEventDisableTiming));
    B_TRY(cudaEventRecord(h0, sin));
    for (int d = 0; d < num_dims; ++d)
        B_CHECK(copy_pieces(ctx, dg[d], group_ids[d], sizeof(int32_t) * n, cudaMemcpyHostToDevice, sin));
    if (weights) B_CHECK(copy_pieces(ctx, dw, weights, sizeof(double) * n, cudaMemcpyHostToDevice, sin));
    B_TRY(cudaEventRecord(ev_ids, sin));
    for (int g = 0; g < ngroups; ++g) {
        const int c0 = gb[g], c1 = gb[g + 1];
        for (int c = c0; c < c1; ++c)
            B_CHECK(copy_pieces(ctx, dv + static_cast<int64_t>(c) * n, host_col(c), sizeof(double) * n,
                                cudaMemcpyHostToDevice, sin));
        B_TRY(cudaEventRecord(ev_in[g], sin));
    }
    B_TRY(cudaEventRecord(h1, sin));
    // the FE structure as soon as the ids are in, while the columns arrive
    int rc = B200FE_OK;
    if (!(o.reuse_structure && ctx->st.valid && ctx->st.n == n && ctx->st.D == num_dims &&
          ctx->st.weighted == (dw != nullptr)) && num_dims > 0) {
        B_TRY(cudaStreamWaitEvent(s, ev_ids, 0));
        cudaEvent_t e0, e1;
        B_TRY(cudaEventCreate(&e0));
        B_TRY(cudaEventCreate(&e1));
        ctx->pass_kernel = o.pass_kernel == 3 ? 0 : o.pass_kernel;
        ctx->sparse_schur = o.pass_kernel == 0;
        B_TRY(cudaEventRecord(e0, s));
        rc = build_structure(ctx, n, num_dims, dg, G, dw);
        B_TRY(cudaEventRecord(e1, s));
        B_TRY(cudaEventSynchronize(e1));
        r->setup_ms = elapsed_ms(e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc != B200FE_OK) {
            ctx->st.valid = false;
            B_TRY(cudaStreamSynchronize(sin));
            cudaEventDestroy(ev_ids);
            return rc;
        }
    }
    cudaEventDestroy(ev_ids);
    bool first_out = true;
    for (int g = 0; g < ngroups && (rc == B200FE_OK || rc == B200FE_NOT_CONVERGED); ++g) {
        const int c0 = gb[g], c1 = gb[g + 1];
        B_TRY(cudaStreamWaitEvent(s, ev_in[g], 0));
        b200fe_options og = o;
        og.reuse_structure = num_dims > 0 ? 1 : o.reuse_structure;
        b200fe_result rg;
        clear_result(&rg);
        const int rcg = absorb_device_impl(ctx, dv + static_cast<int64_t>(c0) * n, n, c1 - c0, num_dims, dg, G,
                                           dw, og, dout + static_cast<int64_t>(c0) * n, &rg);
        if (rcg != B200FE_OK && rcg != B200FE_NOT_CONVERGED) {
            rc = rcg;
            break;
        }
        if (rcg == B200FE_NOT_CONVERGED) rc = rcg;
        B_TRY(cudaEventRecord(ev_done[g], s));
        B_TRY(cudaStreamWaitEvent(sout, ev_done[g], 0));
        if (first_out) {
            B_TRY(cudaEventRecord(d0, sout));
            first_out = false;
        }
        for (int c = c0; c < c1; ++c)
            B_CHECK(copy_pieces(ctx, out_col(c), dout + static_cast<int64_t>(c) * n, sizeof(double) * n,
                                cudaMemcpyDeviceToHost, sout));
        // merge
        r->iterations = std::max(r->iterations, rg.iterations);
        r->outer_iterations = std::max(r->outer_iterations, rg.outer_iterations);
        r->converged = (g == 0 ? 1 : r->converged) && rg.converged;
        r->precision_certified = (g == 0 ? 1 : r->precision_certified) && rg.precision_certified;
        r->primary_dim = rg.primary_dim;
        for (int d = 0; d < num_dims; ++d) r->num_levels_present[d] = rg.num_levels_present[d];
        r->abs_residual = std::max(r->abs_residual, rg.abs_residual);
        r->abs_residual_rel = std::max(r->abs_residual_rel, rg.abs_residual_rel);
        r->rel_residual = std::max(r->rel_residual, rg.rel_residual);
        r->setup_ms += rg.setup_ms;
        r->solve_ms += rg.solve_ms;
        r->warm_columns += rg.warm_columns;
        for (int c = 0; c < B200FE_PROF_CATEGORIES; ++c) {
            r->prof_ms[c] += rg.prof_ms[c];
            r->prof_bytes[c] += rg.prof_bytes[c];
            r->prof_launches[c] += rg.prof_launches[c];
        }
    }
    B_TRY(cudaEventRecord(d1, sout));
    const cudaError_t e1 = cudaStreamSynchronize(sout);
    const cudaError_t e2 = cudaStreamSynchronize(sin);
    if (e1 == cudaSuccess && e2 == cudaSuccess && !first_out) {
        r->h2d_ms = elapsed_ms(h0, h1);
        r->d2h_ms = elapsed_ms(d0, d1);
    }
    for (auto e : {h0, h1, d0, d1}) cudaEventDestroy(e);
    for (int g = 0; g < ngroups; ++g) {
        cudaEventDestroy(ev_in[g]);
        cudaEventDestroy(ev_done[g]);
    }
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        cudaGetLastError();
        ctx->err = std::string("pipelined copies: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2);
        return B200FE_CUDA_ERROR;
    }
    if (rc == B200FE_OK || rc == B200FE_NOT_CONVERGED) rc = r->converged ? B200FE_OK : B200FE_NOT_CONVERGED;
    return rc;
}

}  // namespace

extern "C" {

int b200fe_version(void) { return 10000; }

int b200fe_device_available(void) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

void b200fe_default_options(b200fe_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-8;
    o->max_iter = 10000;
    o->precision = B200FE_PREC_MIXED;
    o->certify = 1;
    o->check_interval = 4;
    o->reuse_structure = 0;
    o->inner_tol = 1e-5;
    o->tolerance_mode = 1;
    o->max_outer = 12;
    o->profile = 0;
    o->pass_kernel = 0;
}

int b200fe_context_create(int device, b200fe_context** out) {
    if (!out) return B200FE_INVALID_ARG;
    *out = nullptr;
    if (!b200fe_device_available()) return B200FE_UNAVAILABLE;
    cudaGetLastError();
    b200fe_context* ctx = new (std::nothrow) b200fe_context();
    if (!ctx) return B200FE_CUDA_ERROR;
    ctx->device = device;
    if (const char* g = std::getenv("B200FE_GRAPHS")) ctx->graphs = std::strcmp(g, "0") != 0;
    if (const char* g = std::getenv("B200FE_PERSISTENT")) ctx->persistent = std::strcmp(g, "0") != 0;
    if (const char* g = std::getenv("B200FE_PIPELINE")) ctx->pipeline = std::strcmp(g, "0") != 0;
    if (const char* g = std::getenv("B200FE_STREAM")) ctx->stream_pass = std::strcmp(g, "0") != 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_pinned, 64 * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_pinned_d, 64 * sizeof(double));
    if (e == cudaSuccess) e = cudaHostAlloc(&ctx->h_xout, kXferOutBytes, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->h_xout_dev), ctx->h_xout, 0);
    if (e == cudaSuccess) e = cudaHostAlloc(&ctx->h_xin, kXferInBytes, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->h_xin_dev), ctx->h_xin, 0);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b200fe_context_destroy(ctx);
        return B200FE_CUDA_ERROR;
    }
    // place the no-alloc entry point's scratch array on this device now, so
    // that its later calls here load nothing (a failure is reported by them)
    if (noalloc_scratch_for_current_device(nullptr) != B200FE_OK) cudaGetLastError();
    *out = ctx;
    return B200FE_OK;
}

void b200fe_context_destroy(b200fe_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    for (auto& kv : ctx->graph_exec) cudaGraphExecDestroy(kv.second);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    for (cudaStream_t cs : {ctx->copy_in, ctx->copy_out})
        if (cs) {
            cudaStreamSynchronize(cs);
            cudaStreamDestroy(cs);
        }
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->h_pinned_d) cudaFreeHost(ctx->h_pinned_d);
    if (ctx->h_xout) cudaFreeHost(ctx->h_xout);
    if (ctx->h_xin) cudaFreeHost(ctx->h_xin);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    cudaGetLastError();
    delete ctx;
}

const char* b200fe_last_error(const b200fe_context* ctx) {
    return ctx ? ctx->err.c_str() : "null context";
}

void* b200fe_context_stream(b200fe_context* ctx) {
    return ctx ? static_cast<void*>(ctx->stream) : nullptr;
}

int b200fe_absorb_device(b200fe_context* ctx, const double* d_v, int64_t n, int cols,
                         int num_dims, const int32_t* const* d_group_ids,
                         const int32_t* num_groups, const double* d_weights,
                         const b200fe_options* opts, double* d_out, b200fe_result* res,
                         void* stream) {
    b200fe_result local;
    b200fe_result* r = res ? res : &local;
    clear_result(r);
    int rc = check_common(ctx, n, cols, num_dims, num_groups);
    if (rc != B200FE_OK) return r->status = rc;
    if (!d_v || !d_out || (num_dims > 0 && !d_group_ids)) {
        ctx->err = "null pointer argument";
        return r->status = B200FE_INVALID_ARG;
    }
    b200fe_options o;
    if (opts) o = *opts;
    else b200fe_default_options(&o);
    cudaGetLastError();  // clear a stale non-sticky error from an earlier call
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return r->status = B200FE_UNAVAILABLE;
    }
    const cudaStream_t own = ctx->stream;
    if (stream) ctx->stream = static_cast<cudaStream_t>(stream);
    const long long l0 = ctx->launches, c0 = ctx->lib_calls;
    rc = absorb_device_impl(ctx, d_v, n, cols, num_dims, d_group_ids, num_groups, d_weights, o,
                            d_out, r);
    ctx->stream = own;
    r->kernel_launches = ctx->launches - l0;
    r->library_calls = ctx->lib_calls - c0;
    return r->status = rc;
}

int b200fe_warmstart_samples(b200fe_context* ctx, const double* d_v, int64_t n, int cols,
                             int num_dims, const int32_t* const* d_group_ids,
                             const int32_t* num_groups, const double* d_weights,
                             const b200fe_options* opts, double* d_out, float* d_features,
                             float* d_targets, int64_t capacity, int64_t* count,
                             b200fe_result* res) {
    if (!ctx || !d_features || !d_targets || !count || capacity < 0) return B200FE_INVALID_ARG;
    *count = 0;
    const int saved_mode = ctx->ws_mode;
    ctx->ws_mode = 0;  // samples come from the plain solver
    ctx->ws_feat = d_features;
    ctx->ws_targ = d_targets;
    ctx->ws_cap = capacity;
    ctx->ws_count = 0;
    const int rc = b200fe_absorb_device(ctx, d_v, n, cols, num_dims, d_group_ids, num_groups, d_weights,
                                        opts, d_out, res, nullptr);
    *count = ctx->ws_count;
    ctx->ws_feat = nullptr;
    ctx->ws_targ = nullptr;
    ctx->ws_cap = ctx->ws_count = 0;
    ctx->ws_mode = saved_mode;
    return rc;
}

int b200fe_absorb_fe(b200fe_context* ctx, const double* y, const double* X, int64_t n, int k,
                     int num_dims, const int32_t* const* group_ids, const int32_t* num_groups,
                     const double* weights, const b200fe_options* opts, double* y_out,
                     double* X_out, double* const* fe_out, b200fe_result* res) {
    b200fe_result local;
    b200fe_result* r = res ? res : &local;
    clear_result(r);
    int rc = check_common(ctx, n, k + 1, num_dims, num_groups);
    if (rc != B200FE_OK) return r->status = rc;
    if (!y || !y_out || (k > 0 && (!X || !X_out)) || (num_dims > 0 && !group_ids)) {
        ctx->err = "null pointer argument";
        return r->status = B200FE_INVALID_ARG;
    }
    for (int d = 0; d < num_dims; ++d)
        if (!group_ids[d] || (fe_out && !fe_out[d])) {
            ctx->err = "null group id or FE output array";
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
    if (!fe_out && ctx->pipeline && cols > kPipeCols) {
        rc = absorb_host_pipelined(ctx, y, X, n, k, num_dims, group_ids, num_groups, weights, o, y_out,
                                   X_out, r);
        r->kernel_launches = ctx->launches - l0;
        r->library_calls = ctx->lib_calls - c0;
        return r->status = rc;
    }
    auto run = [&]() -> int {
        double *dv, *dout, *dw = nullptr;
        B_CHECK(get_buf(ctx, "io_v", static_cast<size_t>(n) * cols, &dv));
        B_CHECK(get_buf(ctx, "io_out", static_cast<size_t>(n) * cols, &dout));
        int32_t* dg[B200FE_MAX_DIMS] = {nullptr};
        for (int d = 0; d < num_dims; ++d)
            B_CHECK(get_buf(ctx, "io_g" + std::to_string(d), n, &dg[d]));
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
        B_TRY(cudaMemcpyAsync(dv, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(dv + n, X, sizeof(double) * n * k, cudaMemcpyHostToDevice, s));
        B_TRY(cudaEventRecord(h1, s));
        if (fe_out) {
            for (int d = 0; d < num_dims; ++d)
                B_CHECK(get_buf(ctx, "fe_out" + std::to_string(d), static_cast<size_t>(num_groups[d]) * cols,
                                &ctx->fe_dev[d]));
            ctx->fe_cols = cols;
        }
        int rc2 = absorb_device_impl(ctx, dv, n, cols, num_dims, dg, num_groups, dw, o, dout, r);
        if (rc2 != B200FE_OK && rc2 != B200FE_NOT_CONVERGED) {
            for (double*& q : ctx->fe_dev) q = nullptr;
            return rc2;
        }
        B_TRY(cudaEventRecord(d0, s));
        B_TRY(cudaMemcpyAsync(y_out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        if (k > 0)
            B_TRY(cudaMemcpyAsync(X_out, dout + n, sizeof(double) * n * k, cudaMemcpyDeviceToHost, s));
        if (fe_out) {
            for (int d = 0; d < num_dims; ++d)
                B_TRY(cudaMemcpyAsync(fe_out[d], ctx->fe_dev[d], sizeof(double) * num_groups[d] * cols,
                                      cudaMemcpyDeviceToHost, s));
            for (double*& q : ctx->fe_dev) q = nullptr;
        }
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

}

int b200fe_absorb(b200fe_context* ctx, const double* y, const double* X, int64_t n, int k,
                  int num_dims, const int32_t* const* group_ids, const int32_t* num_groups,
                  const double* weights, const b200fe_options* opts, double* y_out,
                  double* X_out, b200fe_result* res) {
    return b200fe_absorb_fe(ctx, y, X, n, k, num_dims, group_ids, num_groups, weights, opts, y_out,
                            X_out, nullptr, res);
}  // extern "C"

namespace {
thread_local b200fe_context* tl_ctx = nullptr;

b200fe_context* thread_context() {
    if (!tl_ctx) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            dev = 0;
        }
        if (b200fe_context_create(dev, &tl_ctx) != B200FE_OK) tl_ctx = nullptr;
    }
    return tl_ctx;
}

int fe_recovery_impl(b200fe_context* ctx, const double* residual, int64_t n, int num_dims,
                     const int32_t* const* group_ids, const int32_t* num_groups,
                     const double* weights, const int32_t* sweep_order, double* out) {
    const cudaStream_t s = ctx->stream;
    double *dv, *dw = nullptr, *mean;
    int32_t *dg, *iota, *sorted_keys, *ord, *counts, *off;
    B_CHECK(get_buf(ctx, "rec_v", n, &dv));
    B_CHECK(get_buf(ctx, "rec_g", n, &dg));
    B_CHECK(get_buf(ctx, "rec_iota", n, &iota));
    B_CHECK(get_buf(ctx, "rec_keys", n, &sorted_keys));
    B_CHECK(get_buf(ctx, "rec_ord", n, &ord));
    if (weights) {
        B_CHECK(get_buf(ctx, "rec_w", n, &dw));
        B_TRY(cudaMemcpyAsync(dw, weights, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    }
    B_TRY(cudaMemcpyAsync(dv, residual, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    int32_t* flags;
    B_CHECK(get_buf(ctx, "flags", 4, &flags));
    double best = 0.0;
    for (int j = 0; j < num_dims; ++j) {
        const int d = sweep_order ? sweep_order[j] : j;
        if (d < 0 || d >= num_dims) {
            ctx->err = "sweep_order entry out of range";
            return B200FE_INVALID_ARG;
        }
        const int32_t G = num_groups[d];
        B_TRY(cudaMemcpyAsync(dg, group_ids[d], sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        B_TRY(cudaMemsetAsync(flags, 0, 4 * sizeof(int32_t), s));
        validate_ids_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(dg, n, G, 0, flags);
        B_LAUNCHED();
        int hf[4];
        B_CHECK(sync_read_int(ctx, flags, 4, hf));
        if (hf[0]) {
            ctx->err = "group id outside [0, num_groups)";
            return B200FE_INVALID_ARG;
        }
        iota_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(iota, n);
        B_LAUNCHED();
        B_CHECK(cub_sort_pairs(ctx, dg, sorted_keys, iota, ord, n, G));
        B_CHECK(get_buf(ctx, "rec_counts", static_cast<size_t>(G) + 1, &counts));
        B_CHECK(get_buf(ctx, "rec_off", static_cast<size_t>(G) + 1, &off));
        B_CHECK(get_buf(ctx, "rec_mean", G, &mean));
        B_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * (static_cast<size_t>(G) + 1), s));
        histogram_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(dg, n, counts);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, counts, off, static_cast<int64_t>(G) + 1));
        const int gg = grid_for(ctx, G, 256, 4);
        double* part;
        B_CHECK(get_buf(ctx, "rec_part", gg, &part));
        group_mean_csr_kernel<<<gg, 256, 0, s>>>(off, ord, G, dv, dw, mean, part);
        B_LAUNCHED();
        std::vector<double> hp(gg);
        B_TRY(cudaMemcpyAsync(hp.data(), part, sizeof(double) * gg, cudaMemcpyDeviceToHost, s));
        subtract_mean_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(dv, dg, mean, n);
        B_LAUNCHED();
        B_TRY(cudaStreamSynchronize(s));
        for (double v : hp) best = std::max(best, v);
    }
    *out = best;
    return B200FE_OK;
}

}  // namespace

extern "C" {

int b200fe_demean_raw(double* Y, double* X, int64_t n, int k, int num_dims,
                      const int32_t* const* fe, const int32_t* nlev, double tol, int max_iter,
                      int* iters_out) {
    b200fe_context* ctx = thread_context();
    if (!ctx) return B200FE_UNAVAILABLE;
    b200fe_options o;
    b200fe_default_options(&o);
    if (tol > 0.0) o.tol = tol;
    if (max_iter > 0) o.max_iter = max_iter;
    o.certify = 0;
    b200fe_result r;
    const int rc = b200fe_absorb(ctx, Y, X, n, k, num_dims, fe, nlev, nullptr, &o, Y, X, &r);
    if (iters_out) *iters_out = r.iterations;
    return rc;
}

int b200fe_fe_recovery_max_delta(b200fe_context* ctx, const double* residual, int64_t n,
                                 int num_dims, const int32_t* const* group_ids,
                                 const int32_t* num_groups, const double* weights,
                                 const int32_t* sweep_order, double* out_max_delta) {
    if (!ctx || !residual || !out_max_delta || n <= 0 || num_dims < 0 ||
        num_dims > B200FE_MAX_DIMS || (num_dims > 0 && (!group_ids || !num_groups)))
        return B200FE_INVALID_ARG;
    *out_max_delta = 0.0;
    if (num_dims == 0) return B200FE_OK;
    for (int d = 0; d < num_dims; ++d)
        if (num_groups[d] <= 0 || !group_ids[d]) return B200FE_INVALID_ARG;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    return fe_recovery_impl(ctx, residual, n, num_dims, group_ids, num_groups, weights,
                            sweep_order, out_max_delta);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// OLS (run_ols): moments on the device, p x p algebra on the host
// ---------------------------------------------------------------------------
namespace {

// Symmetric-pivoted LDL' of the p x p symmetric matrix A (column-major), in
// long double: at step k the largest remaining diagonal entry is the pivot
// (the rule of the robust Cholesky in Eigen's LDLT, which the reference's
// run_ols uses).  Solves apply the pseudo-inverse of D: a pivot of magnitude
// at most DBL_MIN is treated as zero and its component set to zero, so a
// rank-deficient X'X yields zero coefficients in its null directions, as the
// reference's solve does, instead of failing.
struct Ldlt {
    int p = 0;
    std::vector<long double> L;  // unit lower, column-major
    std::vector<long double> D;
    std::vector<int> perm;       // row k of the factor is row perm[k] of A
};

Ldlt ldlt_factor(const std::vector<double>& A, int p) {
    Ldlt f;
    f.p = p;
    std::vector<long double> M(A.begin(), A.end());
    f.perm.resize(p);
    for (int i = 0; i < p; ++i) f.perm[i] = i;
    auto at = [&](int i, int j) -> long double& { return M[static_cast<size_t>(j) * p + i]; };
    f.D.assign(p, 0.0L);
    for (int k = 0; k < p; ++k) {
        int piv = k;
        for (int i = k + 1; i < p; ++i)
            if (fabsl(at(i, i)) > fabsl(at(piv, piv))) piv = i;
        if (piv != k) {
            for (int j = 0; j < p; ++j) std::swap(at(k, j), at(piv, j));
            for (int i = 0; i < p; ++i) std::swap(at(i, k), at(i, piv));
            std::swap(f.perm[k], f.perm[piv]);
        }
        const long double d = at(k, k);
        f.D[k] = d;
        const bool zero = fabsl(d) <= static_cast<long double>(DBL_MIN);
        for (int i = k + 1; i < p; ++i) at(i, k) = zero ? 0.0L : at(i, k) / d;
        for (int j = k + 1; j < p; ++j)
            for (int i = j; i < p; ++i) {
                at(i, j) -= at(i, k) * at(j, k) * d;
                at(j, i) = at(i, j);
            }
    }
    f.L = M;
    return f;
}

// x = A^+ b through the factor (b of length p, overwritten)
void ldlt_solve(const Ldlt& f, std::vector<long double>& b) {
    const int p = f.p;
    std::vector<long double> y(p);
    for (int k = 0; k < p; ++k) y[k] = b[f.perm[k]];
    for (int i = 0; i < p; ++i)
        for (int k = 0; k < i; ++k) y[i] -= f.L[static_cast<size_t>(k) * p + i] * y[k];
    for (int i = 0; i < p; ++i)
        y[i] = fabsl(f.D[i]) > static_cast<long double>(DBL_MIN) ? y[i] / f.D[i] : 0.0L;
    for (int i = p - 1; i >= 0; --i)
        for (int k = i + 1; k < p; ++k) y[i] -= f.L[static_cast<size_t>(i) * p + k] * y[k];
    for (int k = 0; k < p; ++k) b[f.perm[k]] = y[k];
}

// sum_i f_i a_i b_i over the column pairs, summed over CTAs; out [npairs]
int run_moments(b200fe_context* ctx, MomentArgs m, std::vector<double>& out, double* rss) {
    const cudaStream_t s = ctx->stream;
    const int npairs = m.P * (m.P + 1) / 2;
    const int grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((m.n + kOlsTile - 1) / kOlsTile, static_cast<int64_t>(ctx->num_sms) * 4)));
    double *part, *sum, *rpart = nullptr, *rsum = nullptr;
    B_CHECK(get_buf(ctx, "ols_part", static_cast<size_t>(grid) * npairs, &part));
    B_CHECK(get_buf(ctx, "ols_sum", static_cast<size_t>(npairs) + 1, &sum));
    if (rss) {
        B_CHECK(get_buf(ctx, "ols_rpart", grid, &rpart));
        B_CHECK(get_buf(ctx, "ols_rsum", 1, &rsum));
    }
    m.partial = part;
    m.rss_partial = rpart;
    moments_kernel<<<grid, kOlsThreads, 0, s>>>(m);
    B_LAUNCHED();
    partial_sum_kernel<<<grid_for(ctx, npairs, 256, 1), 256, 0, s>>>(part, grid, npairs, sum);
    B_LAUNCHED();
    if (rss) {
        partial_sum_kernel<<<1, 32, 0, s>>>(rpart, grid, 1, rsum);
        B_LAUNCHED();
    }
    out.assign(npairs, 0.0);
    B_TRY(cudaMemcpyAsync(out.data(), sum, sizeof(double) * npairs, cudaMemcpyDeviceToHost, s));
    if (rss) B_TRY(cudaMemcpyAsync(rss, rsum, sizeof(double), cudaMemcpyDeviceToHost, s));
    B_TRY(cudaStreamSynchronize(s));
    return B200FE_OK;
}

// upper-triangle pair list -> symmetric P x P (column-major)
std::vector<double> unpack_pairs(const std::vector<double>& v, int P) {
    std::vector<double> M(static_cast<size_t>(P) * P);
    int t = 0;
    for (int a = 0; a < P; ++a)
        for (int b = a; b < P; ++b, ++t) {
            M[static_cast<size_t>(b) * P + a] = v[t];
            M[static_cast<size_t>(a) * P + b] = v[t];
        }
    return M;
}

int ols_impl(b200fe_context* ctx, const double* d_y, const double* d_X, int64_t n, int p,
             const double* d_w, const int32_t* d_cl, int32_t G, int se_type, double n_effective,
             int wfreq, b200fe_ols_result* out) {
    const cudaStream_t s = ctx->stream;
    std::memset(out, 0, sizeof(*out));
    out->p = p;
    // 1. Gram [X y]' W [X y]
    MomentArgs m{};
    m.n = n;
    m.P = p + 1;
    m.p = p;
    m.X = d_X;
    m.cs = n;
    m.rs = 1;
    m.y = d_y;
    m.w = d_w;
    m.mode = kMomGram;
    std::vector<double> g;
    B_CHECK(run_moments(ctx, m, g, nullptr));
    const std::vector<double> GM = unpack_pairs(g, p + 1);
    std::vector<double> xtx(static_cast<size_t>(p) * p);
    std::vector<long double> xty(p);
    for (int j = 0; j < p; ++j) {
        for (int i = 0; i < p; ++i) xtx[static_cast<size_t>(j) * p + i] = GM[static_cast<size_t>(j) * (p + 1) + i];
        xty[j] = GM[static_cast<size_t>(p) * (p + 1) + j];
    }
    for (int i = 0; i < p * p; ++i)
        if (!std::isfinite(xtx[i])) {
            ctx->err = "Failed to factorize X'X; matrix may be singular";
            return B200FE_INVALID_ARG;
        }
    const Ldlt fac = ldlt_factor(xtx, p);
    ldlt_solve(fac, xty);
    for (int j = 0; j < p; ++j) out->coef[j] = static_cast<double>(xty[j]);
    std::vector<double> inv(static_cast<size_t>(p) * p);
    for (int j = 0; j < p; ++j) {
        std::vector<long double> e(p, 0.0L);
        e[j] = 1.0L;
        ldlt_solve(fac, e);
        for (int i = 0; i < p; ++i) inv[static_cast<size_t>(j) * p + i] = static_cast<double>(e[i]);
    }
    for (int i = 0; i < p * p; ++i) out->xtx_inv[i] = inv[i];
    // 2. residual pass: RSS, and the meat for robust inference
    m.P = p;
    m.mode = se_type == 1 ? kMomRobust : kMomRss;
    m.wfreq = wfreq;
    for (int j = 0; j < p; ++j) m.beta[j] = out->coef[j];
    std::vector<double> rm;
    double rss = 0.0;
    B_CHECK(run_moments(ctx, m, rm, &rss));
    const double n_eff = n_effective > 0.0 ? n_effective : static_cast<double>(n);
    const double df_resid = std::max(0.0, n_eff - p);
    out->rss = rss;
    out->df_resid = df_resid;
    out->sigma2 = df_resid > 0.0 ? rss / df_resid : 0.0;
    out->cov_scale = 1.0;
    std::vector<double> meat;
    if (se_type == 1) {
        meat = unpack_pairs(rm, p);
    } else if (se_type == 2) {
        // 3. cluster scores in cluster order (stable sort by cluster id)
        int32_t *keys, *perm, *skeys, *iota, *off;
        B_CHECK(get_buf(ctx, "ols_keys", n, &keys));
        B_CHECK(get_buf(ctx, "ols_perm", n, &perm));
        B_CHECK(get_buf(ctx, "ols_skeys", n, &skeys));
        B_CHECK(get_buf(ctx, "ols_iota", n, &iota));
        B_CHECK(get_buf(ctx, "ols_off", static_cast<size_t>(G) + 1, &off));
        iota_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(iota, n);
        B_LAUNCHED();
        B_CHECK(cub_sort_pairs(ctx, d_cl, skeys, iota, perm, n, G));
        segment_offsets_kernel<<<grid_for(ctx, n + 1, 256), 256, 0, s>>>(skeys, n, G, off);
        B_LAUNCHED();
        (void)keys;
        int32_t *nch, *ch_off, *mflag, *midx;
        B_CHECK(get_buf(ctx, "ols_nch", static_cast<size_t>(G) + 1, &nch));
        B_CHECK(get_buf(ctx, "ols_choff", static_cast<size_t>(G) + 1, &ch_off));
        B_CHECK(get_buf(ctx, "ols_mflag", static_cast<size_t>(G) + 1, &mflag));
        B_CHECK(get_buf(ctx, "ols_midx", static_cast<size_t>(G) + 1, &midx));
        B_TRY(cudaMemsetAsync(nch, 0, sizeof(int32_t) * (static_cast<size_t>(G) + 1), s));
        B_TRY(cudaMemsetAsync(mflag, 0, sizeof(int32_t) * (static_cast<size_t>(G) + 1), s));
        chunk_count_kernel<<<grid_for(ctx, G, 256), 256, 0, s>>>(off, G, kOlsChunk, nch);
        B_LAUNCHED();
        drop_small_chunks_kernel<<<grid_for(ctx, G, 256), 256, 0, s>>>(off, G, kOlsSmallCluster, nch);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, nch, ch_off, static_cast<int64_t>(G) + 1));
        multi_flag_kernel<<<grid_for(ctx, G, 256), 256, 0, s>>>(nch, G, mflag);
        B_LAUNCHED();
        B_CHECK(cub_exclusive_sum(ctx, mflag, midx, static_cast<int64_t>(G) + 1));
        int hc[2];
        B_CHECK(sync_read_int(ctx, ch_off + G, 1, &hc[0]));
        B_CHECK(sync_read_int(ctx, midx + G, 1, &hc[1]));
        const int64_t nchunks = hc[0], nmulti = hc[1];
        int32_t *cgrp, *cbeg, *cend, *mgrp, *mc0, *mc1;
        uint8_t* cwhole;
        B_CHECK(get_buf(ctx, "ols_cgrp", nchunks, &cgrp));
        B_CHECK(get_buf(ctx, "ols_cbeg", nchunks, &cbeg));
        B_CHECK(get_buf(ctx, "ols_cend", nchunks, &cend));
        B_CHECK(get_buf(ctx, "ols_cwhole", nchunks, &cwhole));
        B_CHECK(get_buf(ctx, "ols_mgrp", std::max<int64_t>(nmulti, 1), &mgrp));
        B_CHECK(get_buf(ctx, "ols_mc0", std::max<int64_t>(nmulti, 1), &mc0));
        B_CHECK(get_buf(ctx, "ols_mc1", std::max<int64_t>(nmulti, 1), &mc1));
        chunk_fill_kernel<<<grid_for(ctx, G, 256), 256, 0, s>>>(off, G, kOlsChunk, ch_off, cgrp, cbeg,
                                                                cend, cwhole, midx, mgrp, mc0, mc1);
        B_LAUNCHED();
        double *scores, *cpart;
        const int width = p + 1;
        B_CHECK(get_buf(ctx, "ols_scores", static_cast<size_t>(G) * width, &scores));
        B_CHECK(get_buf(ctx, "ols_cpart", static_cast<size_t>(nchunks) * width, &cpart));
        ClusterArgs c{};
        c.nchunks = nchunks;
        c.chunk_grp = cgrp;
        c.chunk_beg = cbeg;
        c.chunk_end = cend;
        c.chunk_whole = cwhole;
        c.perm = perm;
        c.p = p;
        c.X = d_X;
        c.ld = n;
        c.y = d_y;
        c.w = d_w;
        for (int j = 0; j < p; ++j) c.beta[j] = out->coef[j];
        c.scores = scores;
        c.chunk_part = cpart;
        c.small_max = kOlsSmallCluster;
        cluster_small_kernel<<<grid_for(ctx, G, kOlsThreads, 8), kOlsThreads, 0, s>>>(c, off, G);
        B_LAUNCHED();
        cluster_chunk_kernel<<<grid_for(ctx, nchunks * 32, kOlsThreads, 8), kOlsThreads, 0, s>>>(c);
        B_LAUNCHED();
        if (nmulti > 0) {
            cluster_combine_kernel<<<grid_for(ctx, nmulti * width, 256), 256, 0, s>>>(
                nmulti, mgrp, mc0, mc1, cpart, width, scores);
            B_LAUNCHED();
        }
        int* cnt;
        B_CHECK(get_buf(ctx, "ols_cnt", 1, &cnt));
        B_TRY(cudaMemsetAsync(cnt, 0, sizeof(int), s));
        count_nonempty_kernel<<<grid_for(ctx, G, 256), 256, 0, s>>>(off, G, cnt);
        B_LAUNCHED();
        int ncl = 0;
        B_CHECK(sync_read_int(ctx, cnt, 1, &ncl));
        // meat = sum_g s_g s_g', cluster_u2 = sum_g u_g^2: moments of the scores
        MomentArgs q{};
        q.n = G;
        q.P = p + 1;
        q.p = p;
        q.X = scores;
        q.cs = 1;
        q.rs = width;
        q.y = scores + p;
        q.mode = kMomPlain;
        std::vector<double> sm;
        B_CHECK(run_moments(ctx, q, sm, nullptr));
        const std::vector<double> SM = unpack_pairs(sm, p + 1);
        meat.assign(static_cast<size_t>(p) * p, 0.0);
        for (int j = 0; j < p; ++j)
            for (int i = 0; i < p; ++i) meat[static_cast<size_t>(j) * p + i] = SM[static_cast<size_t>(j) * (p + 1) + i];
        out->cluster_u2 = SM[static_cast<size_t>(p) * (p + 1) + p];
        out->num_clusters = ncl;
        if (ncl > 1 && df_resid > 0.0)
            out->cov_scale = (static_cast<double>(ncl) / (ncl - 1.0)) * ((n_eff - 1.0) / df_resid);
    }
    // 4. covariance
    if (se_type == 0) {
        for (int i = 0; i < p * p; ++i) out->cov[i] = out->sigma2 * inv[i];
    } else {
        std::vector<long double> t(static_cast<size_t>(p) * p, 0.0L);  // inv * meat
        for (int j = 0; j < p; ++j)
            for (int k = 0; k < p; ++k) {
                const long double mk = meat[static_cast<size_t>(j) * p + k];
                for (int i = 0; i < p; ++i) t[static_cast<size_t>(j) * p + i] += inv[static_cast<size_t>(k) * p + i] * mk;
            }
        for (int j = 0; j < p; ++j)
            for (int i = 0; i < p; ++i) {
                long double v = 0.0L;
                for (int k = 0; k < p; ++k) v += t[static_cast<size_t>(k) * p + i] * inv[static_cast<size_t>(j) * p + k];
                out->cov[static_cast<size_t>(j) * p + i] = static_cast<double>(v) * out->cov_scale;
            }
    }
    for (int j = 0; j < p; ++j) out->se[j] = std::sqrt(std::max(0.0, out->cov[static_cast<size_t>(j) * p + j]));
    return B200FE_OK;
}

int ols_check(b200fe_context* ctx, int64_t n, int p, const void* y, const void* X, int se_type,
              const void* cl, int32_t G, b200fe_ols_result* out) {
    if (!ctx || !out || !y || !X || n <= 0 || n >= (int64_t(1) << 31) - 1 || p <= 0 ||
        p > B200FE_OLS_MAX_P || se_type < 0 || se_type > 2 || (se_type == 2 && (!cl || G <= 0))) {
        if (ctx) ctx->err = "invalid OLS arguments";
        return B200FE_INVALID_ARG;
    }
    return B200FE_OK;
}

}  // namespace

extern "C" {

int b200fe_ols_device(b200fe_context* ctx, const double* d_y, const double* d_X, int64_t n, int p,
                      const double* d_weights, const int32_t* d_clusters, int32_t num_clusters,
                      int se_type, double n_effective, int weights_are_frequencies,
                      b200fe_ols_result* out) {
    int rc = ols_check(ctx, n, p, d_y, d_X, se_type, d_clusters, num_clusters, out);
    if (rc != B200FE_OK) return rc;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    if (se_type == 2) {  // cluster ids must be dense in [0, G)
        int* bad;
        B_CHECK(get_buf(ctx, "ols_bad", 3, &bad));
        B_TRY(cudaMemsetAsync(bad, 0, 3 * sizeof(int), ctx->stream));
        validate_ids_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(d_clusters, n, num_clusters, 0, bad);
        B_LAUNCHED();
        int hb = 0;
        B_CHECK(sync_read_int(ctx, bad, 1, &hb));
        if (hb) {
            ctx->err = "cluster ids out of range";
            return B200FE_INVALID_ARG;
        }
    }
    return ols_impl(ctx, d_y, d_X, n, p, d_weights, se_type == 2 ? d_clusters : nullptr,
                    num_clusters, se_type, n_effective, weights_are_frequencies, out);
}

int b200fe_ols(b200fe_context* ctx, const double* y, const double* X, int64_t n, int p,
               const double* weights, const int32_t* clusters, int32_t num_clusters, int se_type,
               double n_effective, int weights_are_frequencies, b200fe_ols_result* out) {
    int rc = ols_check(ctx, n, p, y, X, se_type, clusters, num_clusters, out);
    if (rc != B200FE_OK) return rc;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    const cudaStream_t s = ctx->stream;
    double *dy, *dX, *dw = nullptr;
    int32_t* dc = nullptr;
    B_CHECK(get_buf(ctx, "ols_y", n, &dy));
    B_CHECK(get_buf(ctx, "ols_X", static_cast<size_t>(n) * p, &dX));
    B_TRY(cudaMemcpyAsync(dy, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    B_TRY(cudaMemcpyAsync(dX, X, sizeof(double) * n * p, cudaMemcpyHostToDevice, s));
    if (weights) {
        B_CHECK(get_buf(ctx, "ols_w", n, &dw));
        B_TRY(cudaMemcpyAsync(dw, weights, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    }
    if (se_type == 2) {
        B_CHECK(get_buf(ctx, "ols_c", n, &dc));
        B_TRY(cudaMemcpyAsync(dc, clusters, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    }
    return b200fe_ols_device(ctx, dy, dX, n, p, dw, dc, num_clusters, se_type, n_effective,
                             weights_are_frequencies, out);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Preprocessing on the device: dense ids (build_indexer) and singleton drop
// ---------------------------------------------------------------------------
namespace {

int dense_ids_impl(b200fe_context* ctx, const int32_t* d_raw, int64_t n, int32_t* d_out,
                   int32_t* G_out, int32_t* present_out) {
    const cudaStream_t s = ctx->stream;
    int* mm;
    B_CHECK(get_buf(ctx, "prep_mm", 4, &mm));
    const int init[2] = {INT_MAX, INT_MIN};
    B_TRY(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, s));
    minmax_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_raw, n, mm);
    B_LAUNCHED();
    int hm[2];
    B_CHECK(sync_read_int(ctx, mm, 2, hm));
    const int lo = hm[0], hi = hm[1];
    const long long range = static_cast<long long>(hi) - lo + 1;
    if (range > 0 && range <= kDenseRangeCap && range <= 2LL * n) {
        int32_t *seen, *remap;
        int* cnt;
        B_CHECK(get_buf(ctx, "prep_seen", range, &seen));
        B_CHECK(get_buf(ctx, "prep_remap", range + 1, &remap));
        B_CHECK(get_buf(ctx, "prep_cnt", 1, &cnt));
        B_TRY(cudaMemsetAsync(seen, 0, sizeof(int32_t) * range, s));
        B_TRY(cudaMemsetAsync(cnt, 0, sizeof(int), s));
        mark_seen_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_raw, n, lo, seen);
        B_LAUNCHED();
        count_ones_kernel<<<grid_for(ctx, range, 256), 256, 0, s>>>(seen, range, cnt);
        B_LAUNCHED();
        int unique = 0;
        B_CHECK(sync_read_int(ctx, cnt, 1, &unique));
        *present_out = unique;
        if (static_cast<long long>(unique) * 10 < range * 9) {  // compact in raw order
            B_CHECK(cub_exclusive_sum(ctx, seen, remap, range));
            map_ids_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_raw, n, lo, remap, d_out);
            *G_out = unique;
        } else {
            map_ids_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_raw, n, lo, nullptr, d_out);
            *G_out = static_cast<int32_t>(range);
        }
        B_LAUNCHED();
        B_TRY(cudaStreamSynchronize(s));
        return B200FE_OK;
    }
    // sparse range: rank of the raw value among the distinct values
    uint32_t *key, *skey;
    int32_t *iota, *perm, *flag, *rank;
    B_CHECK(get_buf(ctx, "prep_key", n, &key));
    B_CHECK(get_buf(ctx, "prep_skey", n, &skey));
    B_CHECK(get_buf(ctx, "prep_iota", n, &iota));
    B_CHECK(get_buf(ctx, "prep_perm", n, &perm));
    B_CHECK(get_buf(ctx, "prep_flag", n, &flag));
    B_CHECK(get_buf(ctx, "prep_rank", n, &rank));
    flip_sign_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_raw, n, key);
    B_LAUNCHED();
    iota_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(iota, n);
    B_LAUNCHED();
    size_t tmp = 0;
    B_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, skey, iota, perm, n, 0, 32, s));
    void* t;
    B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
    B_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, key, skey, iota, perm, n, 0, 32, s));
    ++ctx->lib_calls;
    new_key_flags_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(skey, n, flag);
    B_LAUNCHED();
    B_CHECK(cub_inclusive_sum(ctx, flag, rank, n));
    scatter_rank_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(rank, perm, n, d_out);
    B_LAUNCHED();
    int last = 0;
    B_CHECK(sync_read_int(ctx, rank + (n - 1), 1, &last));
    *G_out = last;
    *present_out = last;
    return B200FE_OK;
}

int drop_singletons_impl(b200fe_context* ctx, int nd, const int32_t* const* d_ids, const int32_t* G,
                         int64_t n, uint8_t* d_keep, int max_iter, int64_t* dropped, int* rounds) {
    const cudaStream_t s = ctx->stream;
    SingletonArgs a{};
    a.nd = nd;
    for (int d = 0; d < nd; ++d) {
        a.ids[d] = d_ids[d];
        B_CHECK(get_buf(ctx, "prep_cnt" + std::to_string(d), G[d], &a.counts[d]));
    }
    unsigned long long* dcount;
    B_CHECK(get_buf(ctx, "prep_dropped", 1, &dcount));
    B_TRY(cudaMemsetAsync(d_keep, 1, n, s));
    int64_t total = 0;
    int r = 0;
    for (; r < std::max(1, max_iter); ++r) {
        for (int d = 0; d < nd; ++d)
            B_TRY(cudaMemsetAsync(a.counts[d], 0, sizeof(int32_t) * G[d], s));
        B_TRY(cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), s));
        singleton_count_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(a, n, d_keep);
        B_LAUNCHED();
        singleton_drop_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(a, n, d_keep, dcount);
        B_LAUNCHED();
        unsigned long long h = 0;
        B_TRY(cudaMemcpyAsync(&h, dcount, sizeof(h), cudaMemcpyDeviceToHost, s));
        B_TRY(cudaStreamSynchronize(s));
        if (h == 0) break;
        total += static_cast<int64_t>(h);
    }
    if (dropped) *dropped = total;
    if (rounds) *rounds = r;
    return B200FE_OK;
}

int component_stats_impl(b200fe_context* ctx, const int32_t* d_fe1, const int32_t* d_fe2, int64_t n,
                         const double* d_w, int* num_components, int64_t* largest_n_obs,
                         double* obs_share, double* weight_share) {
    const cudaStream_t s = ctx->stream;
    int32_t *g1, *g2;
    B_CHECK(get_buf(ctx, "cc_g1", n, &g1));
    B_CHECK(get_buf(ctx, "cc_g2", n, &g2));
    int32_t G1 = 0, G2 = 0, p1 = 0, p2 = 0;
    B_CHECK(dense_ids_impl(ctx, d_fe1, n, g1, &G1, &p1));
    B_CHECK(dense_ids_impl(ctx, d_fe2, n, g2, &G2, &p2));
    const int64_t N = static_cast<int64_t>(G1) + G2;
    if (N >= INT32_MAX) {
        ctx->err = "too many groups";
        return B200FE_INVALID_ARG;
    }
    int32_t *parent, *label, *slabel, *off;
    int* flags;
    B_CHECK(get_buf(ctx, "cc_parent", N, &parent));
    B_CHECK(get_buf(ctx, "cc_label", n, &label));
    B_CHECK(get_buf(ctx, "cc_slabel", n, &slabel));
    B_CHECK(get_buf(ctx, "cc_off", N + 1, &off));
    B_CHECK(get_buf(ctx, "cc_flags", 4, &flags));
    iota_kernel<<<grid_for(ctx, N, 256), 256, 0, s>>>(parent, N);
    B_LAUNCHED();
    int rounds = 0;
    for (;; ++rounds) {
        if (rounds >= 1000) {  // min-label hooking converges in a few rounds
            ctx->err = "connected components did not converge";
            return B200FE_CUDA_ERROR;
        }
        B_TRY(cudaMemsetAsync(flags, 0, sizeof(int), s));
        cc_hook_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(g1, g2, n, G1, parent, flags);
        B_LAUNCHED();
        cc_compress_kernel<<<grid_for(ctx, N, 256), 256, 0, s>>>(parent, static_cast<int32_t>(N));
        B_LAUNCHED();
        int changed = 0;
        B_CHECK(sync_read_int(ctx, flags, 1, &changed));
        if (!changed) break;
    }
    cc_label_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(g1, n, parent, label);
    B_LAUNCHED();
    // observations sorted by component (stable), offsets per node: exact counts
    // and, with weights, per-component sums in a fixed order
    double *w_sorted = nullptr, *wsum = nullptr, *tot = nullptr;
    int32_t *iota = nullptr, *perm = nullptr;
    if (d_w) {
        B_TRY(cudaMemsetAsync(flags + 1, 0, sizeof(int), s));
        positive_weights_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(d_w, n, flags + 1);
        B_LAUNCHED();
        int bad = 0;
        B_CHECK(sync_read_int(ctx, flags + 1, 1, &bad));
        if (bad) {
            ctx->err = "First-pair component weights must be finite and positive";
            return B200FE_INVALID_ARG;
        }
        B_CHECK(get_buf(ctx, "cc_iota", n, &iota));
        B_CHECK(get_buf(ctx, "cc_perm", n, &perm));
        iota_kernel<<<grid_for(ctx, n, 256), 256, 0, s>>>(iota, n);
        B_LAUNCHED();
    }
    {
        size_t tmp = 0;
        const uint32_t* ki = reinterpret_cast<const uint32_t*>(label);
        uint32_t* ko = reinterpret_cast<uint32_t*>(slabel);
        const int eb = bits_for(static_cast<int32_t>(N));
        if (d_w) {
            B_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ki, ko, iota, perm, n, 0, eb, s));
        } else {
            B_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp, ki, ko, n, 0, eb, s));
        }
        void* t;
        B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
        if (d_w) {
            B_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, ki, ko, iota, perm, n, 0, eb, s));
        } else {
            B_TRY(cub::DeviceRadixSort::SortKeys(t, tmp, ki, ko, n, 0, eb, s));
        }
        ++ctx->lib_calls;
    }
    segment_offsets_kernel<<<grid_for(ctx, n + 1, 256), 256, 0, s>>>(slabel, n, static_cast<int32_t>(N), off);
    B_LAUNCHED();
    B_TRY(cudaMemsetAsync(flags + 2, 0, 2 * sizeof(int), s));
    cc_count_kernel<<<grid_for(ctx, N, 256), 256, 0, s>>>(off, static_cast<int32_t>(N), flags + 2, flags + 3);
    B_LAUNCHED();
    int hc[2];
    B_CHECK(sync_read_int(ctx, flags + 2, 2, hc));
    *num_components = hc[0];
    *largest_n_obs = hc[1];
    *obs_share = static_cast<double>(hc[1]) / static_cast<double>(n);
    *weight_share = *obs_share;
    if (d_w) {
        B_CHECK(get_buf(ctx, "cc_wsorted", n, &w_sorted));
        B_CHECK(get_buf(ctx, "cc_wsum", N, &wsum));
        B_CHECK(get_buf(ctx, "cc_tot", 1, &tot));
        gather_kernel<double><<<grid_for(ctx, n, 256), 256, 0, s>>>(d_w, perm, n, w_sorted);
        B_LAUNCHED();
        size_t tmp = 0;
        B_TRY(cub::DeviceSegmentedReduce::Sum(nullptr, tmp, w_sorted, wsum, static_cast<int>(N), off, off + 1, s));
        void* t;
        B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
        B_TRY(cub::DeviceSegmentedReduce::Sum(t, tmp, w_sorted, wsum, static_cast<int>(N), off, off + 1, s));
        B_TRY(cub::DeviceReduce::Max(nullptr, tmp, wsum, tot, static_cast<int>(N), s));
        B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
        B_TRY(cub::DeviceReduce::Max(t, tmp, wsum, tot, static_cast<int>(N), s));
        ctx->lib_calls += 2;
        double largest_w = 0.0;
        B_CHECK(sync_read_double(ctx, tot, 1, &largest_w));
        // total weight: the component sums in node order
        B_TRY(cub::DeviceReduce::Sum(nullptr, tmp, wsum, tot, static_cast<int>(N), s));
        B_CHECK(get_buf(ctx, "cub_tmp", tmp, reinterpret_cast<uint8_t**>(&t)));
        B_TRY(cub::DeviceReduce::Sum(t, tmp, wsum, tot, static_cast<int>(N), s));
        ++ctx->lib_calls;
        double total_w = 0.0;
        B_CHECK(sync_read_double(ctx, tot, 1, &total_w));
        *weight_share = total_w > 0.0 ? largest_w / total_w : 0.0;
    }
    return B200FE_OK;
}

}  // namespace

extern "C" {

int b200fe_first_pair_components_device(b200fe_context* ctx, const int32_t* d_fe1,
                                        const int32_t* d_fe2, int64_t n, const double* d_weights,
                                        int* num_components, int64_t* largest_component_n_obs,
                                        double* largest_component_obs_share,
                                        double* largest_component_weight_share) {
    if (!ctx || !d_fe1 || !d_fe2 || n <= 0 || n >= (int64_t(1) << 31) - 1 || !num_components ||
        !largest_component_n_obs || !largest_component_obs_share || !largest_component_weight_share)
        return B200FE_INVALID_ARG;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    return component_stats_impl(ctx, d_fe1, d_fe2, n, d_weights, num_components,
                                largest_component_n_obs, largest_component_obs_share,
                                largest_component_weight_share);
}

int b200fe_dense_ids_device(b200fe_context* ctx, const int32_t* d_raw, int64_t n, int32_t* d_out,
                            int32_t* num_groups, int32_t* num_levels_present) {
    if (!ctx || !d_raw || !d_out || !num_groups || !num_levels_present || n <= 0 ||
        n >= (int64_t(1) << 31) - 1)
        return B200FE_INVALID_ARG;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    return dense_ids_impl(ctx, d_raw, n, d_out, num_groups, num_levels_present);
}

int b200fe_drop_singletons_device(b200fe_context* ctx, int num_dims, const int32_t* const* d_ids,
                                  const int32_t* num_groups, int64_t n, uint8_t* d_keep,
                                  int max_iter, int64_t* dropped, int* rounds) {
    if (!ctx || !d_keep || n <= 0 || num_dims < 1 || num_dims > B200FE_MAX_DIMS || !d_ids ||
        !num_groups)
        return B200FE_INVALID_ARG;
    for (int d = 0; d < num_dims; ++d)
        if (!d_ids[d] || num_groups[d] <= 0) return B200FE_INVALID_ARG;
    cudaGetLastError();
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return B200FE_UNAVAILABLE;
    }
    // ids must be dense in [0, G_d)
    int* bad;
    B_CHECK(get_buf(ctx, "prep_bad", 3, &bad));
    B_TRY(cudaMemsetAsync(bad, 0, 3 * sizeof(int), ctx->stream));
    for (int d = 0; d < num_dims; ++d) {
        validate_ids_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(d_ids[d], n, num_groups[d], 0, bad);
        B_LAUNCHED();
    }
    int hb = 0;
    B_CHECK(sync_read_int(ctx, bad, 1, &hb));
    if (hb) {
        ctx->err = "group ids out of range";
        return B200FE_INVALID_ARG;
    }
    return drop_singletons_impl(ctx, num_dims, d_ids, num_groups, n, d_keep,
                                max_iter > 0 ? max_iter : 100, dropped, rounds);
}

}  // extern "C"

