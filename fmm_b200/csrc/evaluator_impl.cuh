// The device evaluator of one expansion order P and one precision T: plan upload, the
// level-by-level pass sequence on one stream, the level calls.  Included by
// evaluator_order.cu, which instantiates it for one order.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "evaluator_base.hpp"
#include "helmholtz.cuh"
#include "helmholtz_far.cuh"
#include "helmholtz_st.cuh"
#include "kernels.cuh"
#include "m2l_fused.cuh"
#include "m2l_tc.cuh"
#include "p2p_x2.cuh"

namespace fmmb {

static_assert(kX2Warps == 4, "EvaluatorBase::p2p_warps starts at the mixed P2P's static block");

// The Helmholtz FMM's state in an evaluator: complex multipoles and locals (row pairs), the
// translation products, the per-level tables of one wavenumber, the far partials.
struct HhState {
    double k = -1.0;  // the wavenumber of the tables held
    DevBuf M, L, Y, Yo, m2l, m2m, l2l, far_phi, far_g;
    HhLevels lv{};
    bool built = false;
    // the mixed form's tensor-core M2L (p <= 10): tiles over every level, (level, offset,
    // half) as the table index, the table images, and the multipoles' tensor maps
    DevBuf tc_d, tc_begin, tc_count, tc_img;
    int64_t tc_ntiles = 0;
    CUtensorMap mmap{}, vmap{};
};

// ----------------------------------------------------------------------------------
// The evaluator of one precision T and one degree P.
// ----------------------------------------------------------------------------------
template <int P, typename T>
struct Evaluator final : EvaluatorBase {
    static constexpr int NC = nc_of(P);
    using T4 = typename Vec4<T>::type;
    const Plan& plan;
    DevPlan dp{};
    cudaStream_t stream;
    int m;
    bool gradients;
    // plan arrays
    DevBuf level, idx, parent, child_first, box_leaf, src_below, tgt_below, leaf_box, src_start,
        tgt_start, tgt_perm, src_perm, near_row, near_col, w_row, w_col, x_row, x_col, v_row, v_col,
        v_off, box_side;
    // data
    DevBuf m2l_tab, m2m_tab, l2l_tab, spos, tpos, sq, M, Lc, far_phi, far_g, Y;
    // interior boxes per level with a source below (M2M parents), CSR by level
    DevBuf m2m_par;
    std::vector<int64_t> m2m_start;
    // per-level octant batches of the M2M (children with a source) and L2L (children with a
    // target) products, tiles of kGemmPairs; Yo holds one product row per child box
    DevBuf oct_tile_d, oct_tile_begin, oct_tile_count, oct_pair_e, oct_pair_src, Yo;
    std::vector<int64_t> m2m_tiles, l2l_tiles;  // tile ranges per level (nlevels + 1)
    // M2L batches: pairs of all levels grouped by offset, in tiles
    DevBuf tile_d, tile_begin, tile_count, pair_e, pair_src, v_pos;
    int64_t ntiles = 0;
    // the same pairs in per-level tiles, for the level calls
    DevBuf ltile_d, ltile_begin, ltile_count;
    std::vector<int64_t> lvl_tiles;
    // tensor-core M2L (mixed form, p <= 12; above p = 10 in two output-slot halves):
    // tiles of TcTs<P>::NT columns and the table images; the fused form needs p <= 8
    // (tensor memory holds two tables there)
    static constexpr bool kTensor = sizeof(T) == 4 && P <= 12;
    static constexpr int kTcHalves = kTensor ? TcTs<P>::H : 1;
    static constexpr bool kFusedOk = kTensor && P <= 8;
    DevBuf tc_tile_d, tc_tile_begin, tc_tile_count, tc_pair_e, tc_pair_src, tc_bimg, tc_error;
    DevBuf tc_ltile_d, tc_ltile_begin, tc_ltile_count;
    std::vector<int64_t> tc_lvl_tiles;
    int64_t tc_ntiles = 0;
    // the same with the tuner's alternative tile (tc_alt_columns<P>() columns; m2l_tile 1)
    static constexpr int kTcAlt = kTensor ? tc_alt_columns<(P <= 12 ? P : 12)>() : 0;
    DevBuf tc2_tile_d, tc2_tile_begin, tc2_tile_count, tc2_ltile_d, tc2_ltile_begin, tc2_ltile_count;
    std::vector<int64_t> tc2_lvl_tiles;
    int64_t tc2_ntiles = 0;
    int num_sms = 148;
    // fused tensor-core M2L: per level, chunks of consecutive target boxes cut into tiles
    // of one offset (pairs in (chunk, offset, target) order), CTA c of level l taking the
    // tiles fu_cta[fu_lvl_cta[l] + c] .. fu_cta[fu_lvl_cta[l] + c + 1]
    DevBuf fu_tile_d, fu_tile_begin, fu_tile_np, fu_cta, fu_pair_src, fu_pair_tgt, fu_img;
    std::vector<int64_t> fu_lvl_cta;
    std::vector<int> fu_lvl_grid;
    bool product_path_built = false;  // the product paths' tiles and Y (built on first use)
    // chunked product path: when the products of every V pair and vector do not fit the
    // product budget (ybudget bytes), each level's boxes are cut into chunks whose products
    // fit; a chunk's pairs are ordered by (offset, target) at positions local to the chunk
    // (v_pos), tensor-core tiles (NT / m pairs) and SIMT tiles (kGemmPairs pairs) per chunk
    struct Chunk {
        int level;
        int64_t b0, b1, base, npairs, tc_t0, tc_nt, s_t0, s_nt;
    };
    std::vector<Chunk> chunks;
    int64_t ybudget = 0;
    DevBuf ck_tc_d, ck_tc_begin, ck_tc_count, ck_s_d, ck_s_begin, ck_s_count, ck_pair_src;
    std::vector<uint32_t> tc_img;     // host copy of the tensor-memory table images
    CUtensorMap mmap{};               // the multipoles, for the tensor-core M2L's row gathers
    CUtensorMap vmap{};               // the same, boxes of m rows (a pair's vectors)
    // P2P work items (32 targets of one leaf each) and, for the mixed form, the
    // near-singular pairs evaluated in f64
    DevBuf item_leaf, item_t0, close_row, close_src, close_leaf, spos64, tpos64, sq64, near_rec, close_y;
    // the near rows' source streams in the target leaves' frames (mixed form, P2pStream)
    DevBuf st_rowpair, st_xy, st_zz, st_idx;
    // the near-singular pairs' weights (per pair) and, per evaluation, their f64 sums per
    // target and vector (close_weights_kernel, close_sum_kernel)
    DevBuf close_w, close_acc, close_src32;
    // boxes with a nonempty X list, level by level (the P2L launches), the f32 P2L's
    // per-entry records (XRec), and the X-list sums of the f32 P2L when it runs apart (Lx,
    // a box's rows as in Lc): in the evaluation with the near-singular sums on near_stream,
    // the P2L of every level runs there too, beside the upward pass, and the local reduce
    // adds Lx last (the same floats as adding P2L into the stored locals)
    DevBuf xbox, xrec, Lx;
    bool p2l_apart = false;  // set for one evaluation of that form
    std::vector<int64_t> xbox_start;
    // the near field summed apart on a second, lower-priority stream, joined by output_kernel
    DevBuf near_phi, near_g;
    cudaStream_t near_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    P2pItems items{};
    std::vector<int64_t> item_lstart;  // first work item of each level's leaves (nlevels + 1)
    std::vector<int32_t> item_leaf_h;  // the items' leaves (host copy, ascending)
    // The mixed P2P's own work lists, by item slots: every item of 32 targets (one target a
    // lane), then the remainders of the leaves cut into items of 16 and of 8 targets and a
    // last one of up to 8 in 8 slots or up to 4 in 4 slots (K = 32 / slots lanes a target
    // split its pair-steps, so lanes idle only in the last item); each list in leaf order,
    // with explicit targets and slots, on a kernel with K fixed at compile time.
    static constexpr int kP2pClasses = 4;
    DevBuf pitem_leaf, pitem_t0, pitem_n;
    P2pItems plist[kP2pClasses]{};
    std::vector<int64_t> plist_lstart[kP2pClasses];  // first item of each level (nlevels + 1)
    ClosePairs close{};
    int64_t nclose = 0;
    static constexpr bool kMixed = sizeof(T) == 4;
    // register P2M (f32, vectors one after another) up to p = 10; above, its (p+1)^2
    // accumulators a lane exceed the register file (255 registers at p = 11, 12) and the
    // shared-memory column sums run instead (p = 11, sphere 1e6: 0.19 against 0.24 ms).
    // P2L keeps the register kernel at every order: its boxes sum many more sources, and
    // the shared-memory form measured slower there (p = 11: 0.60 against 0.28 ms)
    static constexpr bool kBfly = sizeof(T) == 4 && P <= 10;
    static constexpr bool kBflyP2L = sizeof(T) == 4;

    // near-singular threshold of the mixed form: r2 < 1/16 in target-leaf units (|d| < r_t/4)
    static constexpr float kTheta2 = 0.0625f;
    static constexpr float kRmax = 4.0f;  // 1 / theta: the mixed P2P's clamp of 1/r

    Evaluator(const Plan& pl, const std::vector<double>& m2l, const std::vector<double>& m2m,
              const std::vector<double>& l2l, cudaStream_t s, int m_, bool grad, const std::vector<double>& us,
              const std::vector<double>& ut, bool fused, int64_t ybudget_)
        : plan(pl), stream(s), m(m_), gradients(grad), ybudget(ybudget_) {
        timer.stream = s;
        level.upload(pl.level);
        idx.upload(pl.idx);
        parent.upload(pl.parent);
        child_first.upload(pl.child_first);
        box_leaf.upload(pl.box_leaf);
        src_below.upload(pl.src_below);
        tgt_below.upload(pl.tgt_below);
        leaf_box.upload(pl.leaf_box);
        src_start.upload(pl.src_start);
        tgt_start.upload(pl.tgt_start);
        tgt_perm.upload(pl.tgt_perm);
        src_perm.upload(pl.src_perm);
        near_row.upload(pl.near.row);
        near_col.upload(pl.near.col);
        w_row.upload(pl.w.row);
        w_col.upload(pl.w.col);
        x_row.upload(pl.x.row);
        x_col.upload(pl.x.col);
        v_row.upload(pl.v.row);
        v_col.upload(pl.v.col);
        v_off.upload(pl.v.aux);
        dp.nlevels = pl.nlevels;
        dp.side = pl.side;
        dp.level = level.as<int32_t>();
        dp.idx = idx.as<uint32_t>();
        dp.parent = parent.as<int32_t>();
        dp.child_first = child_first.as<int32_t>();
        dp.box_leaf = box_leaf.as<int32_t>();
        dp.src_below = src_below.as<int64_t>();
        dp.tgt_below = tgt_below.as<int64_t>();
        dp.leaf_box = leaf_box.as<int32_t>();
        dp.src_start = src_start.as<int64_t>();
        dp.tgt_start = tgt_start.as<int64_t>();
        dp.tgt_perm = tgt_perm.as<int64_t>();
        dp.src_perm = src_perm.as<int64_t>();
        dp.near_row = near_row.as<int64_t>();
        dp.near_col = near_col.as<int32_t>();
        dp.w_row = w_row.as<int64_t>();
        dp.w_col = w_col.as<int32_t>();
        dp.x_row = x_row.as<int64_t>();
        dp.x_col = x_col.as<int32_t>();
        dp.v_row = v_row.as<int64_t>();
        dp.v_col = v_col.as<int32_t>();
        dp.v_off = v_off.as<int32_t>();
        if (!pl.box_side.empty()) box_side.upload(pl.box_side);
        dp.box_side = pl.box_side.empty() ? nullptr : box_side.as<double>();
        dp.nsrc = (int64_t)pl.src_perm.size();
        dp.ntgt = (int64_t)pl.tgt_perm.size();
        // tables rounded entry by entry to T (fmm-tables/src/matrix_set.rs:150 cast)
        auto up_tab = [](DevBuf& b, const std::vector<double>& t) {
            std::vector<T> c(t.begin(), t.end());
            b.upload(c);
        };
        up_tab(m2l_tab, m2l);
        up_tab(m2m_tab, m2m);
        up_tab(l2l_tab, l2l);
        // leaf-scaled coordinates, rounded once to T
        auto up_pos = [](DevBuf& b, const std::vector<double>& u) {
            size_t n = u.size() / 3;
            std::vector<T4> v(n);
            for (size_t i = 0; i < n; ++i) {
                v[i].x = (T)u[3 * i];
                v[i].y = (T)u[3 * i + 1];
                v[i].z = (T)u[3 * i + 2];
                v[i].w = T(0);
            }
            b.upload(v);
        };
        up_pos(spos, us);
        up_pos(tpos, ut);
        const size_t nb = pl.nboxes();
        sq.alloc(sizeof(T) * (size_t)m * (dp.nsrc + 1));
        M.alloc(sizeof(T) * (size_t)m * ms_of(P) * nb);
        Lc.alloc(sizeof(T) * (size_t)m * ms_of(P) * nb);
        far_phi.alloc(sizeof(double) * (size_t)m * (dp.ntgt + 1));
        far_g.alloc(sizeof(double) * 3 * (size_t)m * (dp.ntgt + 1));
        CUDA_TRY(cudaMemset(M.ptr, 0, M.bytes));
        build_parent_lists();
        if (kTensor) build_tensor_m2l(m2l);
        if (kFusedOk && fused && m <= fused_tile_columns(P)) {
            build_fused_m2l();
            m2l_path = 2;
        } else {
            m2l_path = kTensor ? 1 : 0;
            ensure_product_path();
        }
        build_p2p_items();
        {
            std::vector<int32_t> xb;
            xbox_start.assign(pl.nlevels + 1, 0);
            for (int l = 0; l < pl.nlevels; ++l) {
                xbox_start[l] = (int64_t)xb.size();
                for (int64_t b = pl.level_start[l]; b < pl.level_start[l + 1]; ++b)
                    if (pl.x.row[b + 1] > pl.x.row[b]) xb.push_back((int32_t)b);
            }
            xbox_start[pl.nlevels] = (int64_t)xb.size();
            xbox.upload(xb);
            if (kMixed && !xb.empty()) {  // the f32 P2L's entry records and its apart sums
                Lx.alloc(sizeof(float) * (size_t)m * ms_of(P) * pl.nboxes());
                xrec.alloc(sizeof(XRec) * (pl.x.nnz() + 1));
                x_record_kernel<<<(unsigned)((xb.size() + 127) / 128), 128>>>(dp, xbox.as<int32_t>(),
                                                                              (int64_t)xb.size(), xrec.as<XRec>());
                CUDA_TRY(cudaGetLastError());
            }
        }
        int least = 0, greatest = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_TRY(cudaStreamCreateWithPriority(&near_stream, cudaStreamNonBlocking, least));
        CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        near_phi.alloc(sizeof(double) * (size_t)m * (dp.ntgt + 1));
        if (gradients) near_g.alloc(sizeof(double) * 3 * (size_t)m * (dp.ntgt + 1));
        if (kMixed) {
            for (size_t j = 0; j < pl.nleaves(); ++j)  // a row fits the kernel's shared memory
                if (pl.near.row[j + 1] - pl.near.row[j] > kX2Recs)
                    throw Failure(FMMGPU_INVALID_ARGUMENT, "a near row longer than " + std::to_string(kX2Recs) +
                                                              " leaves (the tree is not 2:1 balanced)");
            build_close_pairs(us, ut);
            near_rec.alloc(sizeof(NearRec) * (pl.near.nnz() + 1));
            if (pl.nleaves())
                near_record_kernel<<<(unsigned)((pl.nleaves() + 127) / 128), 128>>>(dp, (int64_t)pl.nleaves(),
                                                                                   near_rec.as<NearRec>());
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaDeviceSynchronize());
            build_p2p_stream();
        }
        close_pairs = nclose;
        gemm_smem = GemmShape<P, T>::SMEM;
        if (gemm_smem > 48 * 1024)
            CUDA_TRY(cudaFuncSetAttribute(m2l_gemm_kernel<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem));
        // shared memory opt-in beyond 48 KB where a kernel needs it
        size_t exp_smem = sizeof(T) * (NC * 32 + (size_t)m * 32);
        if (exp_smem > 48 * 1024) {
            CUDA_TRY(cudaFuncSetAttribute(expand_kernel<P, T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)exp_smem));
            CUDA_TRY(cudaFuncSetAttribute(expand_kernel<P, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)exp_smem));
        }
    }

    size_t gemm_smem = 0;

    ~Evaluator() override {
        if (near_stream) {
            cudaStreamSynchronize(near_stream);
            cudaStreamDestroy(near_stream);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
    }

    // The product paths (1 and 0): offset-sorted tiles, the position map and the product
    // array Y, built when a product path is first used.
    void ensure_product_path() {
        if (product_path_built) return;
        const int64_t row_bytes = (int64_t)sizeof(T) * m * ys_of(P);
        if (ybudget > 0 && ((int64_t)plan.v.nnz() + 1) * row_bytes > ybudget) {
            build_product_chunks(row_bytes);
            product_path_built = true;
            return;
        }
        build_m2l_batches(kGemmPairs);
        if constexpr (kTensor) {
            Tiles all, lvl;
            std::vector<int64_t> pe;
            std::vector<int32_t> ps;
            batches(TcTs<P>::NT / m, all, lvl, tc_lvl_tiles, pe, ps);
            tc_halves(all, nullptr);
            tc_halves(lvl, &tc_lvl_tiles);
            tc_ntiles = (int64_t)all.d.size();
            tc_tile_d.upload(all.d);
            tc_tile_begin.upload(all.begin);
            tc_tile_count.upload(all.count);
            tc_ltile_d.upload(lvl.d);
            tc_ltile_begin.upload(lvl.begin);
            tc_ltile_count.upload(lvl.count);
            tc_pair_src.upload(ps);
            // the alternative tile's lists (the pair order is the same)
            Tiles all2, lvl2;
            std::vector<int64_t> pe2;
            std::vector<int32_t> ps2;
            batches(std::max(1, kTcAlt / m), all2, lvl2, tc2_lvl_tiles, pe2, ps2);
            tc_halves(all2, nullptr);
            tc_halves(lvl2, &tc2_lvl_tiles);
            tc2_ntiles = (int64_t)all2.d.size();
            tc2_tile_d.upload(all2.d);
            tc2_tile_begin.upload(all2.begin);
            tc2_tile_count.upload(all2.count);
            tc2_ltile_d.upload(lvl2.d);
            tc2_ltile_begin.upload(lvl2.begin);
            tc2_ltile_count.upload(lvl2.count);
        }
        Y.alloc(sizeof(T) * (size_t)m * ys_of(P) * (plan.v.nnz() + 1));
        product_path_built = true;
    }

    void build_product_chunks(int64_t row_bytes) {
        const Plan& pl = plan;
        const int ppt_tc = kTensor ? std::max(1, tc_tile_columns(P) / m) : 1;
        const int64_t max_pairs = std::max<int64_t>(1, ybudget / row_bytes - 1);
        std::vector<int32_t> ps, tcd, tcn, sd, sn;
        std::vector<int64_t> tcb, sb, vp(pl.v.nnz());
        std::vector<int64_t> cnt(317), fill(316);
        int64_t ymax = 0;
        chunks.clear();
        for (int l = 0; l < pl.nlevels; ++l) {
            int64_t b = pl.level_start[l];
            const int64_t bend = pl.level_start[l + 1];
            while (b < bend) {
                int64_t e = b, np = 0;
                for (; e < bend; ++e) {
                    const int64_t nv = pl.v.row[e + 1] - pl.v.row[e];
                    if (np > 0 && np + nv > max_pairs) break;
                    np += nv;
                }
                Chunk c{l, b, e, (int64_t)ps.size(), np, (int64_t)tcd.size(), 0, (int64_t)sd.size(), 0};
                if (np > 0) {
                    std::fill(cnt.begin(), cnt.end(), 0);
                    for (int64_t x = b; x < e; ++x)
                        for (int64_t q = pl.v.row[x]; q < pl.v.row[x + 1]; ++q) cnt[pl.v.aux[q] + 1]++;
                    for (int d = 0; d < 316; ++d) cnt[d + 1] += cnt[d];
                    ps.resize(c.base + np);
                    for (int d = 0; d < 316; ++d) fill[d] = cnt[d];
                    // boxes in order: each offset's pairs come out ordered by target
                    for (int64_t x = b; x < e; ++x)
                        for (int64_t q = pl.v.row[x]; q < pl.v.row[x + 1]; ++q) {
                            const int64_t pos = fill[pl.v.aux[q]]++;
                            ps[c.base + pos] = pl.v.col[q];
                            vp[q] = pos;
                        }
                    for (int d = 0; d < 316; ++d) {
                        for (int h = 0; h < kTcHalves; ++h)  // table index d * halves + half
                            for (int64_t j = cnt[d]; j < cnt[d + 1]; j += ppt_tc) {
                                tcd.push_back(d * kTcHalves + h);
                                tcb.push_back(j);
                                tcn.push_back((int32_t)std::min<int64_t>(ppt_tc, cnt[d + 1] - j));
                            }
                        for (int64_t j = cnt[d]; j < cnt[d + 1]; j += kGemmPairs) {
                            sd.push_back(d);
                            sb.push_back(j);
                            sn.push_back((int32_t)std::min<int64_t>(kGemmPairs, cnt[d + 1] - j));
                        }
                    }
                    c.tc_nt = (int64_t)tcd.size() - c.tc_t0;
                    c.s_nt = (int64_t)sd.size() - c.s_t0;
                    ymax = std::max(ymax, np);
                }
                chunks.push_back(c);
                b = e;
            }
        }
        ck_tc_d.upload(tcd);
        ck_tc_begin.upload(tcb);
        ck_tc_count.upload(tcn);
        ck_s_d.upload(sd);
        ck_s_begin.upload(sb);
        ck_s_count.upload(sn);
        ck_pair_src.upload(ps);
        v_pos.upload(vp);
        Y.alloc((size_t)row_bytes * (size_t)(ymax + 1));
    }

    // M2L products of one chunk into the product buffer, then its boxes' locals
    void m2l_chunk(const Chunk& c) {
        if (c.npairs == 0) return;
        if (kTensor && m2l_path == 1) {
            if constexpr (kTensor) {
                const unsigned grid = (unsigned)std::min<int64_t>(c.tc_nt, num_sms);
                m2l_tc_kernel<P><<<counted(grid), 32 * kTcWarps, TcTs<P>::SMEM, stream>>>(
                    ck_tc_d.as<int32_t>() + c.tc_t0, ck_tc_begin.as<int64_t>() + c.tc_t0,
                    ck_tc_count.as<int32_t>() + c.tc_t0, c.tc_nt, ck_pair_src.as<int32_t>() + c.base, m,
                    tc_bimg.as<uint32_t>(), mmap, vmap, reinterpret_cast<float*>(Y.ptr), tc_error.as<int>());
            }
            return;
        }
        m2l_gemm_kernel<P, T><<<counted((unsigned)c.s_nt), 256, gemm_smem, stream>>>(
            ck_s_d.as<int32_t>() + c.s_t0, ck_s_begin.as<int64_t>() + c.s_t0, ck_s_count.as<int32_t>() + c.s_t0,
            nullptr, ck_pair_src.as<int32_t>() + c.base, m, m2l_tab.as<T>(), M.as<T>(), Y.as<T>());
    }
    void reduce_chunk(const Chunk& c, int with_l2l, int with_v, int accumulate) {
        reduce_range(c.b0, c.b1, with_l2l, with_v, accumulate);
    }

    // the local reduce of boxes [b0, b1): f32 a warp per box with 16-byte accesses, f64 a
    // block per box (the same order of additions either way)
    void reduce_range(int64_t b0, int64_t b1, int with_l2l, int with_v, int accumulate, bool with_x = false) {
        if (b1 <= b0) return;
        if constexpr (kMixed) {
            const unsigned g = counted((unsigned)((b1 - b0 + 3) / 4));
            const auto* yo = reinterpret_cast<const float*>(Yo.ptr);
            const auto* yv = reinterpret_cast<const float*>(Y.ptr);
            auto* lc = reinterpret_cast<float*>(Lc.ptr);
            const auto* lx = with_x ? reinterpret_cast<const float*>(Lx.ptr) : nullptr;
            if (m == 1)
                local_reduce4_kernel<P, true><<<g, 128, 0, stream>>>(dp, b0, b1, m, with_l2l, with_v, accumulate, yo,
                                                                     yv, v_pos.as<int64_t>(), lc, lx);
            else
                local_reduce4_kernel<P, false><<<g, 128, 0, stream>>>(dp, b0, b1, m, with_l2l, with_v, accumulate,
                                                                      yo, yv, v_pos.as<int64_t>(), lc, lx);
        } else
            local_reduce_kernel<P, T><<<counted((unsigned)(b1 - b0)), round32(NC), 0, stream>>>(
                dp, b0, b1, m, with_l2l, with_v, accumulate, Yo.as<T>(), Y.as<T>(), v_pos.as<int64_t>(),
                Lc.as<T>());
    }

    // The fused path's tiles (see m2l_fused.cuh).  A chunk closes once it holds about
    // three full tiles per offset, or a 1 / (2 num_sms) share of its level's columns (so
    // that every level spreads over the SMs), or before its locals pass kFuChunkBytes (they
    // stay in L2 while its CTA walks the offsets); each level's chunks are dealt to at most
    // num_sms CTAs in contiguous runs of about equal tile counts.
    static constexpr int64_t kFuChunkBytes = 384 * 1024;
    void build_fused_m2l() {
        if constexpr (kFusedOk) {
            using S = FuShape<P>;
            const Plan& pl = plan;
            const int ppt = S::NT / m;
            const int64_t col_full = 3 * 316 * (int64_t)S::NT;
            const int64_t box_bytes = (int64_t)m * ms_of(P) * (int64_t)sizeof(float);
            std::vector<int32_t> td, tn, ps, pt;
            std::vector<int64_t> tb, cta;
            fu_lvl_cta.assign(pl.nlevels + 1, 0);
            fu_lvl_grid.assign(pl.nlevels, 0);
            std::vector<int64_t> cnt(317), fill(316);
            for (int l = 0; l < pl.nlevels; ++l) {
                std::vector<int64_t> chunk_tiles{(int64_t)td.size()};
                int64_t b = pl.level_start[l];
                const int64_t bend = pl.level_start[l + 1];
                const int64_t level_cols = (pl.v.row[bend] - pl.v.row[b]) * m;
                const int64_t col_target =
                    std::min<int64_t>(col_full, std::max<int64_t>(S::NT, level_cols / (2 * (int64_t)num_sms)));
                while (b < bend) {
                    int64_t e = b, cols = 0, nbox = 0;
                    for (; e < bend; ++e) {
                        const int64_t nv = pl.v.row[e + 1] - pl.v.row[e];
                        if (nv == 0) continue;
                        if (nbox > 0 && (cols >= col_target || (nbox + 1) * box_bytes > kFuChunkBytes)) break;
                        cols += nv * m;
                        ++nbox;
                    }
                    if (nbox > 0) {
                        std::fill(cnt.begin(), cnt.end(), 0);
                        for (int64_t x = b; x < e; ++x)
                            for (int64_t q = pl.v.row[x]; q < pl.v.row[x + 1]; ++q) cnt[pl.v.aux[q] + 1]++;
                        for (int d = 0; d < 316; ++d) cnt[d + 1] += cnt[d];
                        const int64_t base = (int64_t)ps.size();
                        ps.resize(base + cnt[316]);
                        pt.resize(base + cnt[316]);
                        for (int d = 0; d < 316; ++d) fill[d] = cnt[d];
                        // boxes in order: each offset's pairs come out ordered by target
                        for (int64_t x = b; x < e; ++x)
                            for (int64_t q = pl.v.row[x]; q < pl.v.row[x + 1]; ++q) {
                                const int64_t pos = base + fill[pl.v.aux[q]]++;
                                ps[pos] = pl.v.col[q];
                                pt[pos] = (int32_t)x;
                            }
                        for (int d = 0; d < 316; ++d)
                            for (int64_t j = cnt[d]; j < cnt[d + 1]; j += ppt) {
                                td.push_back(d);
                                tb.push_back(base + j);
                                tn.push_back((int32_t)std::min<int64_t>(ppt, cnt[d + 1] - j));
                            }
                        chunk_tiles.push_back((int64_t)td.size());
                    }
                    b = e;
                }
                const int64_t nch = (int64_t)chunk_tiles.size() - 1;
                const int G = (int)std::min<int64_t>(num_sms, nch);
                fu_lvl_cta[l] = (int64_t)cta.size();
                fu_lvl_grid[l] = G;
                if (G > 0) {
                    const int64_t t0 = chunk_tiles[0], tt = chunk_tiles[nch] - t0;
                    int64_t ci = 0;
                    cta.push_back(t0);
                    for (int c = 1; c < G; ++c) {
                        const int64_t want = t0 + tt * c / G;
                        while (ci < nch && chunk_tiles[ci] < want) ++ci;
                        cta.push_back(std::max(cta.back(), chunk_tiles[ci]));
                    }
                    cta.push_back(chunk_tiles[nch]);
                }
            }
            fu_lvl_cta[pl.nlevels] = (int64_t)cta.size();
            fu_tile_d.upload(td);
            fu_tile_begin.upload(tb);
            fu_tile_np.upload(tn);
            fu_cta.upload(cta);
            fu_pair_src.upload(ps);
            fu_pair_tgt.upload(pt);
            std::vector<uint32_t> img;
            build_fused_table_images<P>(tc_img, img);
            fu_img.upload(img);
            CUDA_TRY(cudaFuncSetAttribute(m2l_fused_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          FuShape<P>::SMEM));
        }
    }

    void build_tensor_m2l(const std::vector<double>& m2l) {
        if constexpr (kTensor) {
            build_tc_table_images<P>(m2l, tc_img);
            tc_bimg.upload(tc_img);
            encode_multipole_map<P>(&mmap, reinterpret_cast<const float*>(M.ptr), (int64_t)plan.nboxes() * m);
            encode_multipole_map<P>(&vmap, reinterpret_cast<const float*>(M.ptr), (int64_t)plan.nboxes() * m, m);
            tc_error.alloc(sizeof(int));
            CUDA_TRY(cudaMemset(tc_error.ptr, 0, sizeof(int)));
            CUDA_TRY(cudaFuncSetAttribute(m2l_tc_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          TcTs<P>::SMEM));
            CUDA_TRY(cudaFuncSetAttribute(m2l_tc_kernel<P, false, kTcAlt>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, TcTs<P, false, kTcAlt>::SMEM));
            int dev = 0;
            CUDA_TRY(cudaGetDevice(&dev));
            CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
        }
    }

    // Tile lists over the V pairs grouped by offset index, then by target box (pair
    // positions pe/ps shared by both lists):
    //  - the evaluation's list: tiles of up to `tile` pairs of one offset, all levels;
    //  - the level calls' list: the same pairs cut at level boundaries too, ordered by
    //    (level, offset), with its tile range per level in lstart.
    struct Tiles {
        std::vector<int32_t> d, count;
        std::vector<int64_t> begin;
        void add(int dd, int64_t b, int64_t n, int tile) {
            for (int64_t x = b; x < b + n; x += tile) {
                d.push_back(dd);
                begin.push_back(x);
                count.push_back((int32_t)std::min<int64_t>(tile, b + n - x));
            }
        }
    };
    // Tensor-core tiles with two output-slot halves (TcTs<P>::H == 2, p = 11, 12): every run
    // of tiles of one offset d is listed twice, with table index 2d (slots 0..127) and then
    // 2d + 1 (slots 128..255), so a CTA swaps tables as rarely as with one half; lstart
    // (per-level tile ranges, when given) is remapped.  With one half the index is d.
    static void tc_halves(Tiles& t, std::vector<int64_t>* lstart) {
        if constexpr (TcTs<P>::H == 2) {
            std::vector<int64_t> seg = lstart ? *lstart : std::vector<int64_t>{0, (int64_t)t.d.size()};
            Tiles o;
            std::vector<int64_t> nseg(seg.size(), 0);
            for (size_t sgi = 0; sgi + 1 < seg.size(); ++sgi) {
                nseg[sgi] = (int64_t)o.d.size();
                for (int64_t i = seg[sgi]; i < seg[sgi + 1];) {
                    int64_t j = i;
                    while (j < seg[sgi + 1] && t.d[j] == t.d[i]) ++j;
                    for (int h = 0; h < 2; ++h)
                        for (int64_t x = i; x < j; ++x) {
                            o.d.push_back(2 * t.d[x] + h);
                            o.begin.push_back(t.begin[x]);
                            o.count.push_back(t.count[x]);
                        }
                    i = j;
                }
            }
            nseg.back() = (int64_t)o.d.size();
            if (lstart) *lstart = nseg;
            t = std::move(o);
        } else {
            (void)t;
            (void)lstart;
        }
    }

    void batches(int tile, Tiles& all, Tiles& lvl, std::vector<int64_t>& lstart, std::vector<int64_t>& pe,
                 std::vector<int32_t>& ps) {
        const Plan& pl = plan;
        const size_t nnz = pl.v.nnz();
        std::vector<int64_t> cnt(317, 0);
        for (size_t e2 = 0; e2 < nnz; ++e2) cnt[pl.v.aux[e2] + 1]++;
        for (int d = 0; d < 316; ++d) cnt[d + 1] += cnt[d];
        pe.assign(nnz, 0);
        ps.assign(nnz, 0);
        std::vector<int64_t> tbox(nnz, 0);
        std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
        // rows are boxes in order, so pairs of one offset come out ordered by target
        for (size_t b = 0; b + 1 < pl.v.row.size(); ++b)
            for (int64_t e2 = pl.v.row[b]; e2 < pl.v.row[b + 1]; ++e2) {
                int64_t pos = fill[pl.v.aux[e2]]++;
                pe[pos] = e2;
                ps[pos] = pl.v.col[e2];
                tbox[pos] = (int64_t)b;
            }
        for (int d = 0; d < 316; ++d) all.add(d, cnt[d], cnt[d + 1] - cnt[d], tile);
        lstart.assign(pl.nlevels + 1, 0);
        for (int l = 0; l < pl.nlevels; ++l) {
            lstart[l] = (int64_t)lvl.d.size();
            for (int d = 0; d < 316; ++d) {
                auto b0 = std::lower_bound(tbox.begin() + cnt[d], tbox.begin() + cnt[d + 1], pl.level_start[l]);
                auto b1 = std::lower_bound(b0, tbox.begin() + cnt[d + 1], pl.level_start[l + 1]);
                lvl.add(d, b0 - tbox.begin(), b1 - b0, tile);
            }
        }
        lstart[pl.nlevels] = (int64_t)lvl.d.size();
    }

    void build_m2l_batches(int tile) {
        Tiles all, lvl;
        std::vector<int64_t> pe;
        std::vector<int32_t> ps;
        batches(tile, all, lvl, lvl_tiles, pe, ps);
        ntiles = (int64_t)all.d.size();
        tile_d.upload(all.d);
        tile_begin.upload(all.begin);
        tile_count.upload(all.count);
        ltile_d.upload(lvl.d);
        ltile_begin.upload(lvl.begin);
        ltile_count.upload(lvl.count);
        pair_e.upload(pe);
        pair_src.upload(ps);
        // the row of each V entry's product in Y: its position in the offset-sorted list
        std::vector<int64_t> vp(pe.size());
        for (size_t pos = 0; pos < pe.size(); ++pos) vp[pe[pos]] = (int64_t)pos;
        v_pos.upload(vp);
    }

    void build_parent_lists() {
        std::vector<int32_t> a;
        m2m_start.assign(plan.nlevels + 1, 0);
        for (int l = 0; l < plan.nlevels; ++l) {
            for (int64_t x = plan.level_start[l]; x < plan.level_start[l + 1]; ++x)
                if (plan.child_first[x] >= 0 && plan.src_below[x] > 0) a.push_back((int32_t)x);
            m2m_start[l + 1] = (int64_t)a.size();
        }
        m2m_par.upload(a);
        // octant batches: M2M of level l takes children (level l + 1) with a source, L2L of
        // level l takes children (level l) with a target; pairs grouped by octant per level
        std::vector<int32_t> td, tc, ps;
        std::vector<int64_t> tb, pe;
        m2m_tiles.assign(plan.nlevels + 1, 0);
        l2l_tiles.assign(plan.nlevels + 1, 0);
        auto octant = [&](int64_t c) {
            return (int)(((plan.idx[3 * c] & 1) << 2) | ((plan.idx[3 * c + 1] & 1) << 1) | (plan.idx[3 * c + 2] & 1));
        };
        for (int pass = 0; pass < 2; ++pass) {
            std::vector<int64_t>& ranges = pass == 0 ? m2m_tiles : l2l_tiles;
            for (int l = 0; l < plan.nlevels; ++l) {
                ranges[l] = (int64_t)td.size();
                const int cl = pass == 0 ? l + 1 : l;  // level of the children
                if (cl >= plan.nlevels || (pass == 1 && l < 3)) continue;
                std::vector<std::vector<int64_t>> by(8);
                for (int64_t c = plan.level_start[cl]; c < plan.level_start[cl + 1]; ++c) {
                    if (pass == 0 ? plan.src_below[c] == 0 : plan.tgt_below[c] == 0) continue;
                    by[octant(c)].push_back(c);
                }
                for (int o = 0; o < 8; ++o)
                    for (size_t s0 = 0; s0 < by[o].size(); s0 += kGemmPairs) {
                        td.push_back(o);
                        tb.push_back((int64_t)pe.size());
                        const size_t cnt = std::min<size_t>(kGemmPairs, by[o].size() - s0);
                        tc.push_back((int32_t)cnt);
                        for (size_t q = s0; q < s0 + cnt; ++q) {
                            const int64_t c = by[o][q];
                            pe.push_back(c);
                            ps.push_back(pass == 0 ? (int32_t)c : plan.parent[c]);
                        }
                    }
            }
            ranges[plan.nlevels] = (int64_t)td.size();
        }
        oct_tile_d.upload(td);
        oct_tile_begin.upload(tb);
        oct_tile_count.upload(tc);
        oct_pair_e.upload(pe);
        oct_pair_src.upload(ps);
        Yo.alloc(sizeof(T) * (size_t)m * ys_of(P) * plan.nboxes());
    }

    // The near rows' source streams (P2pStream), built when they take at most a quarter of
    // the free device memory; otherwise the P2P maps its sources per flush (the same floats).
    void build_p2p_stream() {
        const size_t nl = plan.nleaves();
        std::vector<int64_t> rp(nl + 1, 0);
        for (size_t j = 0; j < nl; ++j) {
            int64_t S = 0;
            for (int64_t e = plan.near.row[j]; e < plan.near.row[j + 1]; ++e) {
                const int sl = plan.near.col[e];
                S += plan.src_start[sl + 1] - plan.src_start[sl];
            }
            rp[j + 1] = rp[j] + (S + 1) / 2;
        }
        const size_t pairs = (size_t)rp[nl];
        const size_t bytes = pairs * (sizeof(float4) + sizeof(float2) + sizeof(int2)) + 8 * (nl + 1);
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        if (dp.nsrc >= ((int64_t)1 << 31) || bytes > free_b / 4) return;
        st_rowpair.upload(rp);
        st_xy.alloc(sizeof(float4) * (pairs + 1));
        st_zz.alloc(sizeof(float2) * (pairs + 1));
        st_idx.alloc(sizeof(int2) * (pairs + 1));
        if (nl)
            near_stream_kernel<<<(unsigned)((nl + 3) / 4), 128>>>(dp, (int64_t)nl, near_rec.as<NearRec>(),
                                                                  reinterpret_cast<const float4*>(spos.ptr),
                                                                  st_rowpair.as<int64_t>(), st_xy.as<float4>(),
                                                                  st_zz.as<float2>(), st_idx.as<int2>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaDeviceSynchronize());
        p2p_stream_bytes = (int64_t)(st_rowpair.bytes + st_xy.bytes + st_zz.bytes + st_idx.bytes);
        p2p_path = 1;
    }

    void set_p2p_path(int path) override {
        if (path < 0 || path > 1 || (path == 1 && !p2p_stream_bytes))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "P2P path " + std::to_string(path) + " not available");
        p2p_path = path;
    }

    void build_p2p_items() {
        std::vector<int32_t> il;
        std::vector<int64_t> it;
        for (size_t j = 0; j < plan.nleaves(); ++j)
            for (int64_t t = plan.tgt_start[j]; t < plan.tgt_start[j + 1]; t += 32) {
                il.push_back((int32_t)j);
                it.push_back(t);
            }
        item_lstart.assign(plan.nlevels + 1, (int64_t)il.size());
        for (int l = plan.nlevels - 1; l >= 0; --l) {
            int64_t first = plan.leaf_level_start[l];
            item_lstart[l] = std::lower_bound(il.begin(), il.end(), (int32_t)first) - il.begin();
        }
        item_leaf.upload(il);
        item_t0.upload(it);
        item_leaf_h = il;
        items.leaf = item_leaf.as<int32_t>();
        items.t0 = item_t0.as<int64_t>();
        items.count = (int64_t)il.size();
        if constexpr (kMixed) build_p2p_lists();
    }

    void build_p2p_lists() {
        std::vector<int32_t> lv[kP2pClasses], nv[kP2pClasses];
        std::vector<int64_t> tv[kP2pClasses];
        auto add = [&](int c, size_t j, int64_t t, int n) {
            lv[c].push_back((int32_t)j);
            tv[c].push_back(t);
            nv[c].push_back(n);
        };
        for (size_t j = 0; j < plan.nleaves(); ++j) {
            int64_t t = plan.tgt_start[j];
            const int64_t t1 = plan.tgt_start[j + 1];
            for (; t + 32 <= t1; t += 32) add(0, j, t, 32 | 32 << 8);
            // a remainder of 25 to 31 targets as one item of 32 slots (a lane a target, the
            // rest idle): cheaper than the three partial items it would split into, each of
            // which reads the near row and pays an item's fixed cost
            if (t1 - t >= 25) add(0, j, t, (int)(t1 - t) | 32 << 8), t = t1;
            if (t + 16 <= t1) add(1, j, t, 16 | 16 << 8), t += 16;
            if (t + 8 <= t1) add(2, j, t, 8 | 8 << 8), t += 8;
            const int r = (int)(t1 - t);  // 0 to 7 left
            if (r > 4) add(2, j, t, r | 8 << 8);
            else if (r > 0) add(3, j, t, r | 4 << 8);
        }
        std::vector<int32_t> al, an;
        std::vector<int64_t> at;
        int64_t base[kP2pClasses];
        for (int c = 0; c < kP2pClasses; ++c) {
            plist_lstart[c].assign(plan.nlevels + 1, (int64_t)lv[c].size());
            for (int l = plan.nlevels - 1; l >= 0; --l)
                plist_lstart[c][l] =
                    std::lower_bound(lv[c].begin(), lv[c].end(), (int32_t)plan.leaf_level_start[l]) - lv[c].begin();
            base[c] = (int64_t)al.size();
            al.insert(al.end(), lv[c].begin(), lv[c].end());
            at.insert(at.end(), tv[c].begin(), tv[c].end());
            an.insert(an.end(), nv[c].begin(), nv[c].end());
        }
        pitem_leaf.upload(al);
        pitem_t0.upload(at);
        pitem_n.upload(an);
        for (int c = 0; c < kP2pClasses; ++c)
            plist[c] = P2pItems{pitem_leaf.as<int32_t>() + base[c], pitem_t0.as<int64_t>() + base[c],
                                (int64_t)lv[c].size(), pitem_n.as<int32_t>() + base[c]};
    }

    // The mixed form's f64 pairs: found on the device with the f32 arithmetic of the P2P
    // kernel itself, then sorted per target (source order) into a CSR.
    void build_close_pairs(const std::vector<double>& us, const std::vector<double>& ut) {
        auto up64 = [](DevBuf& b, const std::vector<double>& u) {
            size_t n = u.size() / 3;
            std::vector<double4> v(n);
            for (size_t i = 0; i < n; ++i) v[i] = make_double4(u[3 * i], u[3 * i + 1], u[3 * i + 2], 0.0);
            b.upload(v);
        };
        up64(spos64, us);
        up64(tpos64, ut);
        sq64.alloc(sizeof(double) * (size_t)m * (dp.nsrc + 1));
        int64_t cap = std::max<int64_t>(1 << 20, dp.ntgt * 2);
        DevBuf cnt, ot, os, ol;
        cnt.alloc(sizeof(unsigned long long));
        unsigned long long found = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
            ot.alloc(sizeof(int64_t) * cap);
            os.alloc(sizeof(int64_t) * cap);
            ol.alloc(sizeof(int32_t) * cap);
            CUDA_TRY(cudaMemset(cnt.ptr, 0, sizeof(unsigned long long)));
            if (items.count)
                close_pairs_kernel<T><<<(unsigned)((items.count + kP2pWarps - 1) / kP2pWarps), 32 * kP2pWarps>>>(
                    dp, items, (T)kTheta2, spos.as<T4>(), tpos.as<T4>(), cnt.as<unsigned long long>(), cap,
                    ot.as<int64_t>(), os.as<int64_t>(), ol.as<int32_t>());
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaMemcpy(&found, cnt.ptr, sizeof(found), cudaMemcpyDeviceToHost));
            if ((int64_t)found <= cap) break;
            cap = (int64_t)found + 1024;
        }
        nclose = (int64_t)found;
        // sorted by (target, source) into a CSR by target, on the device (plan_gpu.cu; the
        // pair's key packs both indices in 64 bits)
        if (dp.nsrc >= ((int64_t)1 << 32)) throw Failure(FMMGPU_UNSUPPORTED, "more than 2^32 sources");
        close_row.alloc(sizeof(int64_t) * (size_t)(dp.ntgt + 2));
        close_src.alloc(sizeof(int64_t) * (size_t)(nclose + 1));
        close_leaf.alloc(sizeof(int32_t) * (size_t)(nclose + 1));
        sort_close_pairs(nclose, ot.as<int64_t>(), os.as<int64_t>(), ol.as<int32_t>(), dp.ntgt, close_row.as<int64_t>(),
                         close_src.as<int64_t>(), close_leaf.as<int32_t>());
        close.row = close_row.as<int64_t>();
        close.src = close_src.as<int64_t>();
        close.leaf = close_leaf.as<int32_t>();
        close.spos = spos64.as<double4>();
        close.tpos = tpos64.as<double4>();
        close_y.alloc(sizeof(double4) * (size_t)(nclose + 1));
        close.y = close_y.as<double4>();
        if (plan.nleaves()) close_map_kernel<<<(unsigned)plan.nleaves(), 64>>>(dp, close, close_y.as<double4>());
        CUDA_TRY(cudaGetLastError());
        close.q = sq64.as<double>();
        const size_t wd = gradients ? 4 : 1;  // floats a pair, doubles a target and vector
        close_w.alloc(sizeof(float) * wd * (size_t)(nclose + 1));
        close_acc.alloc(sizeof(double) * wd * (size_t)m * (dp.ntgt + 1));
        close_src32.alloc(sizeof(uint32_t) * (size_t)(nclose + 1));
        if (nclose)
            close_src32_kernel<<<(unsigned)((nclose + 255) / 256), 256>>>(close_src.as<int64_t>(), nclose,
                                                                          close_src32.as<uint32_t>());
        close.acc = nclose ? close_acc.as<double>() : nullptr;  // no pairs: nothing to add
        if (plan.nleaves() && nclose) {
            const auto* s32 = reinterpret_cast<const float4*>(spos.ptr);
            const auto* t32 = reinterpret_cast<const float4*>(tpos.ptr);
            if (gradients)
                close_weights_kernel<true><<<(unsigned)plan.nleaves(), 64>>>(dp, close, s32, t32, kRmax,
                                                                             close_w.as<float>());
            else
                close_weights_kernel<false><<<(unsigned)plan.nleaves(), 64>>>(dp, close, s32, t32, kRmax,
                                                                              close_w.as<float>());
        }
        CUDA_TRY(cudaGetLastError());
    }

    // The near-singular pairs' f64 sums of this pass's charges (mixed form).
    void close_sums(cudaStream_t s) {
        if (!kMixed || !nclose || !dp.ntgt) return;
        const unsigned g = (unsigned)((dp.ntgt + 255) / 256);
        if (gradients)
            close_sum_kernel<true><<<counted(g), 256, 0, s>>>(close, close_w.as<float>(), close_src32.as<uint32_t>(),
                                                             m, dp.nsrc, dp.ntgt,
                                                             close_acc.as<double>());
        else
            close_sum_kernel<false><<<counted(g), 256, 0, s>>>(close, close_w.as<float>(), close_src32.as<uint32_t>(),
                                                              m, dp.nsrc, dp.ntgt,
                                                              close_acc.as<double>());
    }

    const int* device_status_word() const override {
        if constexpr (kTensor) return tc_error.as<int>();
        return nullptr;
    }

    int device_status() override {
        if constexpr (kTensor) {
            int err = 0;
            CUDA_TRY(cudaMemcpy(&err, tc_error.ptr, sizeof(int), cudaMemcpyDeviceToHost));
            return err;
        }
        return 0;
    }

    size_t device_bytes() const {
        const DevBuf* all[] = {&level, &idx, &parent, &child_first, &box_leaf, &src_below, &tgt_below,
                               &leaf_box, &src_start, &tgt_start, &tgt_perm, &src_perm, &near_row,
                               &near_col, &w_row, &w_col, &x_row, &x_col, &v_row, &v_col, &v_off,
                               &m2l_tab, &m2m_tab, &l2l_tab, &spos, &tpos, &sq, &M, &Lc, &far_phi, &far_g,
                               &Y, &m2m_par, &oct_tile_d, &oct_tile_begin, &oct_tile_count, &oct_pair_e, &pitem_leaf, &pitem_t0, &pitem_n,
                               &oct_pair_src, &Yo, &tile_d, &tile_begin, &tile_count, &pair_e, &pair_src, &item_leaf, &item_t0,
                               &close_row, &close_src, &close_leaf, &spos64, &tpos64, &sq64, &close_y, &tc_tile_d,
                               &tc_tile_begin, &tc_tile_count, &tc_pair_e, &tc_pair_src, &tc_bimg, &tc_error, &near_rec,
                               &ltile_d, &ltile_begin, &ltile_count, &tc_ltile_d, &tc_ltile_begin, &tc_ltile_count,
                               &near_phi, &near_g, &box_side, &v_pos, &xbox, &xrec, &Lx, &fu_tile_d, &fu_tile_begin,
                               &fu_tile_np, &fu_cta, &fu_pair_src, &fu_pair_tgt, &fu_img, &ck_tc_d, &ck_tc_begin,
                               &ck_tc_count, &ck_s_d, &ck_s_begin, &ck_s_count, &ck_pair_src, &st_rowpair,
                               &st_xy, &st_zz, &st_idx, &close_w, &close_acc, &close_src32};
        size_t s = 0;
        for (auto* b : all) s += b->bytes;
        return s;
    }

    // ---- evaluation: every pass, fused where the level structure allows ----
    void evaluate(const double* d_charges, double* d_phi, double* d_grad) override {
        if (first_pass) {
            timer.begin();
            launches = 0;
        }
        // the near-singular sums (mixed) need only the charges: beside the far field on
        // near_stream, or with the charge load when kinds are timed
        const bool sums = kMixed && nclose && (kinds & 1) && items.count;
        // charge load into leaf order
        timer.run(kLoad, [&] {
            load_charges(d_charges);
            if (sums && timer.on) close_sums(stream);
            // locals of levels 0 and 1 stay zero (no V or L2L reaches them)
            int64_t top = plan.nlevels > 2 ? plan.level_start[2] : (int64_t)plan.nboxes();
            CUDA_TRY(cudaMemsetAsync(Lc.ptr, 0, sizeof(T) * (size_t)m * ms_of(P) * top, stream));
        });
        if (overlap && !timer.on && kinds == 3 && items.count) {
            // the near field on near_stream (it needs only the charges) beside the far-field
            // chain on the evaluator's stream; output_kernel adds them: far + near, the same
            // addition as the fused P2P epilogue, so the same floats
            CUDA_TRY(cudaEventRecord(ev_fork, stream));
            CUDA_TRY(cudaStreamWaitEvent(near_stream, ev_fork, 0));
            close_sums(near_stream);
            p2p_levels(0, plan.nlevels, 1, 2, near_phi.as<double>(), gradients ? near_g.as<double>() : nullptr,
                       near_stream);
            CUDA_TRY(cudaEventRecord(ev_join, near_stream));
            run_far();
            CUDA_TRY(cudaStreamWaitEvent(stream, ev_join, 0));
            output(d_phi, d_grad, true);
            CUDA_TRY(cudaGetLastError());
            return;
        }
        const bool forked = sums && !timer.on;
        // P2L apart on near_stream: the product path (all levels' M2L products at once)
        p2l_apart = forked && (kinds & 2) && m2l_path == 1 && chunks.empty() && Lx.ptr;
        if (forked) {
            CUDA_TRY(cudaEventRecord(ev_fork, stream));
            CUDA_TRY(cudaStreamWaitEvent(near_stream, ev_fork, 0));
            if (p2l_apart)  // first: the first local reduce waits for it
                for (int l = 2; l < plan.nlevels; ++l) p2l_level(l, true, near_stream);
            close_sums(near_stream);
            CUDA_TRY(cudaEventRecord(ev_join, near_stream));
        }
        if (!(kinds & 2)) {
            // far field off: zero partials, then the near field and the output pass only
            CUDA_TRY(cudaMemsetAsync(far_phi.ptr, 0, far_phi.bytes, stream));
            CUDA_TRY(cudaMemsetAsync(far_g.ptr, 0, far_g.bytes, stream));
        } else {
            run_far();
        }
        if (forked && !p2l_apart) CUDA_TRY(cudaStreamWaitEvent(stream, ev_join, 0));
        p2l_apart = false;
        if (items.count) timer.run(kP2P, [&] { p2p_levels(0, plan.nlevels, kinds & 1, 0, d_phi, d_grad); });
        CUDA_TRY(cudaGetLastError());
    }

    // Times the launch shapes that change no float (every P2P target and every L2P / M2P
    // target sums the same terms in the same order whatever the block) on this plan and
    // device, and keeps the fastest: warps a block of the mixed P2P kernel, threads a block
    // of the L2P / M2P kernel.  One evaluation first leaves the far partials in place; the
    // P2P launches with accumulate 0 only read them and rewrite the output, the L2P / M2P
    // launches rewrite the same partials.  A last evaluation leaves the output and the
    // launch count as a plain evaluation does.
    int64_t product_chunks() const override { return (int64_t)chunks.size(); }
    int m2l_tile_columns(int tile) const override {
        if constexpr (kTensor) return tile ? kTcAlt : TcTs<P>::NT;
        return 0;
    }

    void set_m2l_path(int path) override {
        if (path < 0 || path > 2 || (path >= 1 && !kTensor) || (path == 2 && !kFusedOk))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "M2L path " + std::to_string(path) + " not available");
        if (path == 2 && fu_lvl_grid.empty()) {
            if (m > fused_tile_columns(P))
                throw Failure(FMMGPU_INVALID_ARGUMENT, "the fused M2L takes at most " +
                                                           std::to_string(fused_tile_columns(P)) + " vectors a pass");
            build_fused_m2l();
        }
        if (path <= 1) ensure_product_path();
        m2l_path = path;
    }

    void autotune(const double* d_charges, double* d_phi, double* d_grad) override {
        const bool timing = timer.on;
        timer.on = false;
        first_pass = true;
        evaluate(d_charges, d_phi, d_grad);
        cudaEvent_t e0, e1;
        CUDA_TRY(cudaEventCreate(&e0));
        CUDA_TRY(cudaEventCreate(&e1));
        auto time = [&](auto&& launch) {
            launch();  // warm-up
            CUDA_TRY(cudaEventRecord(e0, stream));
            for (int r = 0; r < 3; ++r) launch();
            CUDA_TRY(cudaEventRecord(e1, stream));
            CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            return ms;
        };
        if (kMixed && items.count) {
            float best = 0.f;
            int pick = p2p_warps;
            for (int w : {1, 2, 4}) {
                p2p_warps = w;
                const float ms = time([&] { p2p_levels(0, plan.nlevels, kinds & 1, 0, d_phi, d_grad); });
                if (w == 1 || ms < best) best = ms, pick = w;
            }
            p2p_warps = pick;
        }
        if (plan.nleaves() && (kinds & 2)) {
            float best = 0.f;
            int pick = leaf_block;
            for (int b : {32, 64, 128}) {
                leaf_block = b;
                const float ms = time([&] { leaf_far(0, (int64_t)plan.nleaves(), 3); });
                if (b == 32 || ms < best) best = ms, pick = b;
            }
            leaf_block = pick;
        }
        // the tensor-core M2L tile (the products are the same floats for either: every
        // column is its own MMA column with the same K order)
        if (kTensor && m2l_path == 1 && chunks.empty() && tc_ntiles && (kinds & 2)) {
            float best = 0.f;
            int pick = m2l_tile;
            for (int t : {0, 1}) {
                m2l_tile = t;
                const float ms = time([&] { m2l_products(-1); });
                if (t == 0 || ms < best) best = ms, pick = t;
            }
            m2l_tile = pick;
        }
        CUDA_TRY(cudaEventDestroy(e0));
        CUDA_TRY(cudaEventDestroy(e1));
        timer.on = timing;
        first_pass = true;
        evaluate(d_charges, d_phi, d_grad);
    }

    void output(double* d_phi, double* d_grad, bool with_near) {
        if (plan.nleaves())
            output_kernel<<<counted((unsigned)plan.nleaves()), 128, 0, stream>>>(
                dp, m, far_phi.as<double>(), far_g.as<double>(), with_near ? near_phi.as<double>() : nullptr,
                with_near && gradients ? near_g.as<double>() : nullptr, d_phi, gradients ? d_grad : nullptr);
    }

    void run_far() {
        const int L = plan.nlevels - 1;
        // upward: P2M of every leaf, then M2M from level L-1 up to 0
        timer.run(kP2M, [&] { p2m_rows(0, (int64_t)plan.nleaves()); });
        for (int l = L - 1; l >= 0; --l) timer.run(kM2M, [&] { m2m_level(l); });
        if (m2l_path == 2) {
            // downward, fused: per level the L2L part of the locals, then the V products
            // added into them in row order, then P2L
            for (int l = 2; l <= L; ++l) {
                timer.run(kL2L, [&] {
                    if (l >= 3) l2l_products(l);
                    reduce_locals(l, l >= 3, 0, 0);
                });
                timer.run(kM2L, [&] { m2l_fused(l); });
                timer.run(kP2L, [&] { p2l_level(l); });
            }
            timer.run(kFar, [&] { leaf_far(0, (int64_t)plan.nleaves(), 3); });
            return;
        }
        if (!chunks.empty()) {
            // downward, chunked: per level the L2L products, then chunk by chunk the M2L
            // products and the locals (L2L + V in offset order), then P2L
            for (int l = 2; l <= L; ++l) {
                timer.run(kL2L, [&] {
                    if (l >= 3) l2l_products(l);
                });
                for (const Chunk& c : chunks) {
                    if (c.level != l) continue;
                    timer.run(kM2L, [&] { m2l_chunk(c); });
                    timer.run(kL2L, [&] { reduce_chunk(c, l >= 3, 1, 0); });
                }
                timer.run(kP2L, [&] { p2l_level(l); });
            }
            timer.run(kFar, [&] { leaf_far(0, (int64_t)plan.nleaves(), 3); });
            return;
        }
        // M2L products of every level at once (all multipoles are final here)
        timer.run(kM2L, [&] { m2l_products(-1); });
        // P2L apart: its sums (on near_stream) are read by the first reduce
        if (p2l_apart) CUDA_TRY(cudaStreamWaitEvent(stream, ev_join, 0));
        // downward: for l = 2..L: L2L products, the local (L2L + V in offset order), then P2L
        for (int l = 2; l <= L; ++l) {
            timer.run(kL2L, [&] {
                l2l_products(l);
                reduce_locals(l, l >= 3, 1, 0, p2l_apart);
            });
            if (!p2l_apart) timer.run(kP2L, [&] { p2l_level(l); });
        }
        // leaves: L2P + M2P
        timer.run(kFar, [&] { leaf_far(0, (int64_t)plan.nleaves(), 3); });
    }

    // ---- the pieces, shared by the evaluation and the level calls ----
    void load_charges(const double* d_charges) {
        const int64_t ns = dp.nsrc;
        if (ns > 0)
            charge_load_kernel<T><<<counted((unsigned)((ns + 255) / 256)), 256, 0, stream>>>(
                d_charges, src_perm.as<int64_t>(), ns, m, qstride, sq.as<T>(), kMixed ? sq64.as<double>() : nullptr);
    }

    size_t exp_smem() const { return sizeof(T) * (NC * 32 + (size_t)m * 32); }

    void p2m_rows(int64_t r0, int64_t r1) {  // P2M of leaves [r0, r1)
        if (r1 <= r0) return;
        if (kBfly && m == 1)
            expand_bfly_kernel<P, false, false><<<counted((unsigned)(r1 - r0)), 32, 0, stream>>>(
                dp, r0, r1, nullptr, reinterpret_cast<const float4*>(spos.ptr), m,
                reinterpret_cast<const float*>(sq.ptr), reinterpret_cast<float*>(M.ptr));
        else if (kBfly)
            expand_bfly_kernel<P, false, true><<<counted((unsigned)(r1 - r0)), 32, 0, stream>>>(
                dp, r0, r1, nullptr, reinterpret_cast<const float4*>(spos.ptr), m,
                reinterpret_cast<const float*>(sq.ptr), reinterpret_cast<float*>(M.ptr));
        else
            expand_kernel<P, T, false><<<counted((unsigned)(r1 - r0)), 32, exp_smem(), stream>>>(
                dp, r0, r1, nullptr, m, spos.as<T4>(), sq.as<T>(), M.as<T>());
    }

    void m2m_level(int l) {  // parents on level l from their children on level l + 1
        const int64_t t0 = m2m_tiles[l], nt = m2m_tiles[l + 1] - m2m_tiles[l];
        const int64_t n = m2m_start[l + 1] - m2m_start[l];
        if (nt)
            m2l_gemm_kernel<P, T><<<counted((unsigned)nt), 256, gemm_smem, stream>>>(
                oct_tile_d.as<int32_t>() + t0, oct_tile_begin.as<int64_t>() + t0, oct_tile_count.as<int32_t>() + t0,
                oct_pair_e.as<int64_t>(), oct_pair_src.as<int32_t>(), m, m2m_tab.as<T>(), M.as<T>(), Yo.as<T>());
        if (n)
            m2m_reduce_kernel<P, T><<<counted((unsigned)n), round32(NC), 0, stream>>>(
                dp, m2m_par.as<int32_t>() + m2m_start[l], n, m, Yo.as<T>(), M.as<T>());
    }

    // fused M2L of level l: L += the V products, in row order (after the L2L part)
    void m2l_fused(int l) {
        if constexpr (kFusedOk) {
            const int G = fu_lvl_grid[l];
            if (G == 0) return;
            m2l_fused_kernel<P><<<counted((unsigned)G), 32 * kFuWarps, FuShape<P>::SMEM, stream>>>(
                fu_tile_d.as<int32_t>(), fu_tile_begin.as<int64_t>(), fu_tile_np.as<int32_t>(),
                fu_cta.as<int64_t>() + fu_lvl_cta[l], fu_pair_src.as<int32_t>(), fu_pair_tgt.as<int32_t>(), m,
                fu_img.as<uint32_t>(), reinterpret_cast<const float*>(M.ptr), reinterpret_cast<float*>(Lc.ptr),
                tc_error.as<int>());
        }
    }

    // M2L products Y of the V pairs of level l (l < 0: every level in one launch)
    void m2l_products(int l) {
        if (kTensor && m2l_path == 1) {
            if constexpr (kTensor) {
                const bool alt = m2l_tile == 1;
                const std::vector<int64_t>& ls = alt ? tc2_lvl_tiles : tc_lvl_tiles;
                const int64_t t0 = l < 0 ? 0 : ls[l];
                const int64_t nt = l < 0 ? (alt ? tc2_ntiles : tc_ntiles) : ls[l + 1] - ls[l];
                const DevBuf& td = l < 0 ? (alt ? tc2_tile_d : tc_tile_d) : (alt ? tc2_ltile_d : tc_ltile_d);
                const DevBuf& tb = l < 0 ? (alt ? tc2_tile_begin : tc_tile_begin) : (alt ? tc2_ltile_begin : tc_ltile_begin);
                const DevBuf& tn = l < 0 ? (alt ? tc2_tile_count : tc_tile_count) : (alt ? tc2_ltile_count : tc_ltile_count);
                if (nt == 0) return;
                const unsigned grid = (unsigned)std::min<int64_t>(nt, num_sms);
                if (alt)
                    m2l_tc_kernel<P, false, kTcAlt><<<counted(grid), 32 * kTcWarps, TcTs<P, false, kTcAlt>::SMEM,
                                                      stream>>>(
                        td.as<int32_t>() + t0, tb.as<int64_t>() + t0, tn.as<int32_t>() + t0, nt,
                        tc_pair_src.as<int32_t>(), m, tc_bimg.as<uint32_t>(), mmap, vmap,
                        reinterpret_cast<float*>(Y.ptr), tc_error.as<int>());
                else
                    m2l_tc_kernel<P><<<counted(grid), 32 * kTcWarps, TcTs<P>::SMEM, stream>>>(
                        td.as<int32_t>() + t0, tb.as<int64_t>() + t0, tn.as<int32_t>() + t0, nt,
                        tc_pair_src.as<int32_t>(), m, tc_bimg.as<uint32_t>(), mmap, vmap,
                        reinterpret_cast<float*>(Y.ptr), tc_error.as<int>());
            }
            return;
        }
        const int64_t t0 = l < 0 ? 0 : lvl_tiles[l];
        const int64_t nt = l < 0 ? ntiles : lvl_tiles[l + 1] - lvl_tiles[l];
        const DevBuf& td = l < 0 ? tile_d : ltile_d;
        const DevBuf& tb = l < 0 ? tile_begin : ltile_begin;
        const DevBuf& tn = l < 0 ? tile_count : ltile_count;
        if (nt)
            m2l_gemm_kernel<P, T><<<counted((unsigned)nt), 256, gemm_smem, stream>>>(
                td.as<int32_t>() + t0, tb.as<int64_t>() + t0, tn.as<int32_t>() + t0, nullptr,
                pair_src.as<int32_t>(), m, m2l_tab.as<T>(), M.as<T>(), Y.as<T>());
    }

    void l2l_products(int l) {  // L2L products Yo of the children on level l (l >= 3)
        const int64_t t0 = l2l_tiles[l], nt = l2l_tiles[l + 1] - l2l_tiles[l];
        if (nt)
            m2l_gemm_kernel<P, T><<<counted((unsigned)nt), 256, gemm_smem, stream>>>(
                oct_tile_d.as<int32_t>() + t0, oct_tile_begin.as<int64_t>() + t0, oct_tile_count.as<int32_t>() + t0,
                oct_pair_e.as<int64_t>(), oct_pair_src.as<int32_t>(), m, l2l_tab.as<T>(), Lc.as<T>(), Yo.as<T>());
    }

    void reduce_locals(int l, int with_l2l, int with_v, int accumulate, bool with_x = false) {
        reduce_range(plan.level_start[l], plan.level_start[l + 1], with_l2l, with_v, accumulate, with_x);
    }

    // P2L of the boxes of level l with an X list: added into the locals, or (apart, true)
    // written into Lx on stream s for the local reduce to add (mixed form)
    void p2l_level(int l, bool apart = false, cudaStream_t s = nullptr) {
        const int64_t b0 = xbox_start[l], b1 = xbox_start[l + 1];
        if (b1 <= b0) return;
        if (!s) s = stream;
        float* out = reinterpret_cast<float*>(apart ? Lx.ptr : Lc.ptr);
        if (kBflyP2L && m == 1)
            expand_bfly_kernel<P, true, false><<<counted((unsigned)(b1 - b0)), 32, 0, s>>>(
                dp, b0, b1, xbox.as<int32_t>(), reinterpret_cast<const float4*>(spos.ptr), m,
                reinterpret_cast<const float*>(sq.ptr), out, xrec.as<XRec>(), apart ? 1 : 0);
        else if (kBflyP2L)
            expand_bfly_kernel<P, true, true><<<counted((unsigned)(b1 - b0)), 32, 0, s>>>(
                dp, b0, b1, xbox.as<int32_t>(), reinterpret_cast<const float4*>(spos.ptr), m,
                reinterpret_cast<const float*>(sq.ptr), out, xrec.as<XRec>(), apart ? 1 : 0);
        else  // (f64: never apart)
            expand_kernel<P, T, true><<<counted((unsigned)(b1 - b0)), 32, exp_smem(), s>>>(
                dp, b0, b1, xbox.as<int32_t>(), m, spos.as<T4>(), sq.as<T>(), Lc.as<T>());
    }

    void leaf_far(int64_t r0, int64_t r1, int mode) {  // L2P / M2P of leaves [r0, r1)
        if (r1 <= r0) return;
        const size_t smem = sizeof(T) == 8 ? NC * sizeof(T) : 0;
        if constexpr (kMixed) {
            // a warp per P2P work item of these leaves (items are in leaf order); leaf_block
            // threads a block
            const int64_t i0 = std::lower_bound(item_leaf_h.begin(), item_leaf_h.end(), (int32_t)r0) - item_leaf_h.begin();
            const int64_t i1 = std::lower_bound(item_leaf_h.begin(), item_leaf_h.end(), (int32_t)r1) - item_leaf_h.begin();
            if (i1 <= i0) return;
            const P2pItems it{items.leaf + i0, items.t0 + i0, i1 - i0};
            const int wpb = leaf_block / 32;
            const unsigned g = (unsigned)((it.count + wpb - 1) / wpb);
            const auto* tp = reinterpret_cast<const float4*>(tpos.ptr);
            const auto* Mf = reinterpret_cast<const float*>(M.ptr);
            const auto* Lf = reinterpret_cast<const float*>(Lc.ptr);
            if (!gradients)  // potentials: the harmonics shared by up to 8 vectors (any m: the same floats)
                leaf_far_mv_items_kernel<P, 8><<<counted(g), leaf_block, 0, stream>>>(dp, it, mode, m, tp, Mf, Lf,
                                                                                     far_phi.as<double>());
            else
                leaf_far_items_kernel<P, true><<<counted(g), leaf_block, 0, stream>>>(
                    dp, it, mode, m, tp, Mf, Lf, far_phi.as<double>(), far_g.as<double>());
            return;
        }
        if (gradients)
            leaf_far_kernel<P, T, true><<<counted((unsigned)(r1 - r0)), leaf_block, smem, stream>>>(
                dp, r0, mode, m, tpos.as<T4>(), M.as<T>(), Lc.as<T>(), far_phi.as<double>(), far_g.as<double>());
        else
            leaf_far_kernel<P, T, false><<<counted((unsigned)(r1 - r0)), leaf_block, smem, stream>>>(
                dp, r0, mode, m, tpos.as<T4>(), M.as<T>(), Lc.as<T>(), far_phi.as<double>(), far_g.as<double>());
    }

    template <int W, int KS>
    void p2p_x2_launch(const P2pItems& it, int near, int accumulate, double* d_phi, double* fg, double* og,
                       cudaStream_t s) {
        const unsigned g = (unsigned)((it.count + W - 1) / W);
        const auto* sp = reinterpret_cast<const float4*>(spos.ptr);
        const auto* tp = reinterpret_cast<const float4*>(tpos.ptr);
        const auto* q = reinterpret_cast<const float*>(sq.ptr);
        if (p2p_path == 1) {
            const P2pStream st{st_rowpair.as<int64_t>(), st_xy.as<float4>(), st_zz.as<float2>(), st_idx.as<int2>()};
            if (!gradients) {
                p2p_st_mv_kernel<W><<<counted(g), 32 * W, 0, s>>>(dp, it, m, near, kRmax, st, q, tp, close,
                                                                 far_phi.as<double>(), accumulate, d_phi);
                return;
            }
            const P2pStArgs a{dp, it, m, near, kRmax, st, q, tp, close, far_phi.as<double>(), fg, accumulate, d_phi, og};
            launch_p2p_st(a, W, KS, counted(g), s);
            return;
        }
        if (!gradients) {  // potentials: the pair geometry shared by up to kX2Vb vectors (any m)
            p2p_x2_mv_kernel<W><<<counted(g), 32 * W, 0, s>>>(dp, it, m, near, kRmax, near_rec.as<NearRec>(), sp, q,
                                                             tp, close, far_phi.as<double>(), accumulate, d_phi);
            return;
        }
        if (gradients)
            p2p_x2_kernel<true, W><<<counted(g), 32 * W, 0, s>>>(dp, it, m, near, kRmax, near_rec.as<NearRec>(), sp,
                                                               q, tp, close, far_phi.as<double>(), fg, accumulate,
                                                               d_phi, og);
        else
            p2p_x2_kernel<false, W><<<counted(g), 32 * W, 0, s>>>(dp, it, m, near, kRmax, near_rec.as<NearRec>(),
                                                                sp, q, tp, close, far_phi.as<double>(), fg,
                                                                accumulate, d_phi, og);
    }

    template <int KS>
    void p2p_x2_shape(const P2pItems& it, int near, int accumulate, double* d_phi, double* fg, double* og,
                      cudaStream_t s) {
        if (!it.count) return;
        if (p2p_warps == 1)
            p2p_x2_launch<1, KS>(it, near, accumulate, d_phi, fg, og, s);
        else if (p2p_warps == 2)
            p2p_x2_launch<2, KS>(it, near, accumulate, d_phi, fg, og, s);
        else
            p2p_x2_launch<4, KS>(it, near, accumulate, d_phi, fg, og, s);
    }
    static P2pItems item_range(const P2pItems& a, int64_t i0, int64_t i1) {
        return P2pItems{a.leaf + i0, a.t0 + i0, i1 - i0, a.n ? a.n + i0 : nullptr};
    }

    // P2P of the leaves of levels [l0, l1); accumulate = 0 adds the far partial and writes
    // the scaled output in caller order, 1 adds into the leaf-order store (level calls), 2
    // writes the near field alone in leaf order into d_phi / d_grad.  The mixed form runs
    // its two work lists (items of 32 targets, then the split remainders).
    void p2p_levels(int l0, int l1, int near, int accumulate, double* d_phi, double* d_grad,
                    cudaStream_t s = nullptr) {
        if (!s) s = stream;
        double* fg = gradients ? far_g.as<double>() : nullptr;
        double* og = gradients ? d_grad : nullptr;
        if constexpr (kMixed) {
            auto range = [&](int c) { return item_range(plist[c], plist_lstart[c][l0], plist_lstart[c][l1]); };
            p2p_x2_shape<1>(range(0), near, accumulate, d_phi, fg, og, s);
            p2p_x2_shape<2>(range(1), near, accumulate, d_phi, fg, og, s);
            p2p_x2_shape<4>(range(2), near, accumulate, d_phi, fg, og, s);
            p2p_x2_shape<8>(range(3), near, accumulate, d_phi, fg, og, s);
        } else {
            const int64_t i0 = item_lstart[l0], i1 = item_lstart[l1];
            if (i1 <= i0) return;
            P2pItems it{items.leaf + i0, items.t0 + i0, i1 - i0};
            const unsigned g = (unsigned)((it.count + kP2pWarps - 1) / kP2pWarps);
            if (gradients)
                p2p_kernel<T, true><<<counted(g), 32 * kP2pWarps, 0, s>>>(
                    dp, it, m, near, (T)kTheta2, spos.as<T4>(), sq.as<T>(), tpos.as<T4>(), close,
                    far_phi.as<double>(), fg, accumulate, d_phi, og);
            else
                p2p_kernel<T, false><<<counted(g), 32 * kP2pWarps, 0, s>>>(
                    dp, it, m, near, (T)kTheta2, spos.as<T4>(), sq.as<T>(), tpos.as<T4>(), close,
                    far_phi.as<double>(), fg, accumulate, d_phi, og);
        }
    }

    // ---- the Helmholtz FMM (real k): complex expansions as row pairs, per-level tables ----
    static constexpr int NE = 2 * NC;  // order of a complex translation as a real matrix
    // the mixed form's Helmholtz M2L on the tensor cores ((p+1)^2 <= 128: p <= 10)
    static constexpr bool kHhTensor = kMixed && P <= 10;
    HhState hh;

    // the complex translation of a host table (a real 2n x n matrix per set, column-major,
    // column j the image of the unit real input e_j, the real plane over the imaginary
    // plane) as the real 2n x 2n block [[A_r, -A_i], [A_i, A_r]], column-major, in T,
    // scaled by `scale` (exact: a power of two)
    static void hh_block(const std::vector<double>& host, int sets, double scale, std::vector<T>& out, size_t at) {
        const int n = NC;
        for (int d = 0; d < sets; ++d) {
            const double* h = host.data() + (size_t)d * 2 * n * n;
            T* o = out.data() + at + (size_t)d * NE * NE;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    const double ar = h[(size_t)j * 2 * n + i], ai = h[(size_t)j * 2 * n + n + i];
                    o[(size_t)j * NE + i] = (T)(scale * ar);
                    o[(size_t)j * NE + n + i] = (T)(scale * ai);
                    o[(size_t)(n + j) * NE + i] = (T)(-scale * ai);
                    o[(size_t)(n + j) * NE + n + i] = (T)(scale * ar);
                }
        }
    }

    // Buffers (first use) and the tables of wavenumber k (when it changed): per level l the
    // M2L set of boxes of half-width 1 at k_l = k r_l (l >= 2), the M2M set of parent level
    // l (l < L) and the L2L set of child level l (l >= 3, its parent's octant tables times
    // 1/2: a local in box units is r_l times the absolute one).
    void hh_setup(double k) {
        const int NL = plan.nlevels;
        if (NL > 32) throw Failure(FMMGPU_UNSUPPORTED, "more than 32 levels");
        if (!hh.built) {
            const size_t nb = plan.nboxes();
            const size_t mv = 2 * (size_t)m;
            hh.M.alloc(sizeof(T) * mv * ms_of(P) * nb);
            hh.L.alloc(sizeof(T) * mv * ms_of(P) * nb);
            hh.Y.alloc(sizeof(T) * mv * (kHhTensor ? 256 : ys_of(P)) * (plan.v.nnz() + 1));
            hh.Yo.alloc(sizeof(T) * mv * ys_of(P) * nb);
            hh.far_phi.alloc(sizeof(double) * 2 * (size_t)m * (dp.ntgt + 1));
            if (gradients) hh.far_g.alloc(sizeof(double) * 6 * (size_t)m * (dp.ntgt + 1));
            if (!hq.ptr) {
                hq.alloc(sizeof(Cplx<T>) * (size_t)m * (dp.nsrc + 1));
                if (kMixed) hq64.alloc(sizeof(double2) * (size_t)m * (dp.nsrc + 1));
            }
            size_t smem = sizeof(double) * (2 * NC * 32 + 2 * (size_t)m * 32);
            if (smem > 227 * 1024) throw Failure(FMMGPU_UNSUPPORTED, "too many charge vectors a pass for P2L");
            CUDA_TRY(cudaFuncSetAttribute(hh_expand_kernel<P, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            CUDA_TRY(cudaFuncSetAttribute(hh_expand_kernel<P, T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            if (GemmShape<P, T, true>::SMEM > 48 * 1024)
                CUDA_TRY(cudaFuncSetAttribute(m2l_gemm_kernel<P, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              GemmShape<P, T, true>::SMEM));
            if constexpr (kHhTensor) hh_tc_tiles();
            hh.built = true;
        }
        if (k == hh.k) return;
        const auto t0 = std::chrono::steady_clock::now();
        for (int l = 0; l < NL; ++l) hh.lv.kl[l] = k * plan.side * std::ldexp(1.0, -(l + 1));
        const size_t set = (size_t)NE * NE;
        std::vector<T> m2l(kHhTensor ? 0 : (size_t)std::max(NL - 2, 1) * 316 * set), m2m((size_t)NL * 8 * set),
            l2l((size_t)NL * 8 * set);
        std::vector<double> host, hm, hl;
        std::vector<uint32_t> tc_img;
        for (int l = 2; l < NL; ++l) {
            bool any = false;
            for (int64_t b = plan.level_start[l]; b < plan.level_start[l + 1] && !any; ++b)
                any = plan.v.row[b + 1] > plan.v.row[b];
            if (!any) continue;  // no V pair on this level: its tables are never read
            const size_t cnt = (size_t)316 * 2 * NC * NC;
            std::string why;
            if (table_cache_dir.empty() ||
                !table_cache_load(table_cache_dir, kTableHelmholtzM2l, P, hh.lv.kl[l], cnt, host, &why)) {
                build_helmholtz_m2l_tables(P, hh.lv.kl[l], 1.0, host);
                if (!table_cache_dir.empty())
                    table_cache_store(table_cache_dir, kTableHelmholtzM2l, P, hh.lv.kl[l], host, &why);
            }
            if constexpr (kHhTensor) {
                tc_img.resize((size_t)(l - 2) * 316 * 2 * TcTs<P, true>::IMG_WORDS);
                append_tc_complex_images<P>(host, tc_img);
            } else {
                hh_block(host, 316, 1.0, m2l, (size_t)(l - 2) * 316 * set);
            }
        }
        for (int l = 0; l + 1 < NL; ++l) {
            const size_t half = (size_t)8 * 2 * NC * NC;
            std::string why;
            if (!table_cache_dir.empty() &&
                table_cache_load(table_cache_dir, kTableHelmholtzOctant, P, hh.lv.kl[l], 2 * half, host, &why)) {
                hm.assign(host.begin(), host.begin() + half);
                hl.assign(host.begin() + half, host.end());
            } else {
                build_helmholtz_octant_tables(P, hh.lv.kl[l], 1.0, hm, hl);
                if (!table_cache_dir.empty()) {
                    host = hm;
                    host.insert(host.end(), hl.begin(), hl.end());
                    table_cache_store(table_cache_dir, kTableHelmholtzOctant, P, hh.lv.kl[l], host, &why);
                }
            }
            hh_block(hm, 8, 1.0, m2m, (size_t)l * 8 * set);
            hh_block(hl, 8, 0.5, l2l, (size_t)(l + 1) * 8 * set);
        }
        if constexpr (kHhTensor) {
            tc_img.resize((size_t)std::max(NL - 2, 1) * 316 * 2 * TcTs<P, true>::IMG_WORDS);
            hh.tc_img.upload(tc_img);
            std::vector<uint32_t>().swap(tc_img);
        } else {
            hh.m2l.upload(m2l);
        }
        hh.m2m.upload(m2m);
        hh.l2l.upload(l2l);
        hh.k = k;
        hh_table_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // The mixed form's tensor-core Helmholtz M2L: tiles of NT / (2m) pairs (each pair's 2m
    // columns: the real and imaginary planes of its vectors) over the V pairs of every
    // level, by (level, offset), each run listed twice (halves A_r and A_i), table index
    // ((level - 2) * 316 + d) * 2 + half; the multipoles' tensor maps over the complex rows.
    void hh_tc_tiles() {
        if constexpr (kHhTensor) {
            using S = TcTs<P, true>;
            Tiles all, lvl;
            std::vector<int64_t> pe, lstart;
            std::vector<int32_t> ps;
            batches(std::max(1, S::NT / (2 * m)), all, lvl, lstart, pe, ps);
            tc_halves_force(lvl, lstart);
            for (int l = 0; l < plan.nlevels; ++l)
                for (int64_t i = lstart[l]; i < lstart[l + 1]; ++i) lvl.d[i] += (l - 2) * 316 * 2;
            hh.tc_ntiles = (int64_t)lvl.d.size();
            hh.tc_d.upload(lvl.d);
            hh.tc_begin.upload(lvl.begin);
            hh.tc_count.upload(lvl.count);
            const int64_t rows = (int64_t)plan.nboxes() * 2 * m;
            encode_multipole_map<P>(&hh.mmap, reinterpret_cast<const float*>(hh.M.ptr), rows);
            encode_multipole_map<P>(&hh.vmap, reinterpret_cast<const float*>(hh.M.ptr), rows, 2 * m);
            CUDA_TRY(cudaFuncSetAttribute(m2l_tc_kernel<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          S::SMEM));
        }
    }

    // every run of tiles of one table index d listed twice, as 2d then 2d + 1 (per level)
    static void tc_halves_force(Tiles& t, std::vector<int64_t>& lstart) {
        Tiles o;
        std::vector<int64_t> nseg(lstart.size(), 0);
        for (size_t sgi = 0; sgi + 1 < lstart.size(); ++sgi) {
            nseg[sgi] = (int64_t)o.d.size();
            for (int64_t i = lstart[sgi]; i < lstart[sgi + 1];) {
                int64_t j = i;
                while (j < lstart[sgi + 1] && t.d[j] == t.d[i]) ++j;
                for (int h = 0; h < 2; ++h)
                    for (int64_t x = i; x < j; ++x) {
                        o.d.push_back(2 * t.d[x] + h);
                        o.begin.push_back(t.begin[x]);
                        o.count.push_back(t.count[x]);
                    }
                i = j;
            }
        }
        nseg.back() = (int64_t)o.d.size();
        lstart = nseg;
        t = std::move(o);
    }

    void helmholtz_fmm(double kre, double kim, const double* d_q, double* d_phi, double* d_grad) override {
        if (kim != 0.0)
            throw Failure(FMMGPU_UNSUPPORTED, "the Helmholtz far field is built for a real wavenumber (Im k = 0)");
        if (!(kre > 0.0)) throw Failure(FMMGPU_INVALID_ARGUMENT, "the Helmholtz FMM needs k > 0");
        if (!plan.box_side.empty())
            throw Failure(FMMGPU_UNSUPPORTED, "the Helmholtz FMM is not offered for multi-cloud batches");
        if (!chunks.empty())
            throw Failure(FMMGPU_UNSUPPORTED,
                          "the Helmholtz far field needs every M2L product at once (the plan was built chunked)");
        ensure_product_path();
        if (!chunks.empty())
            throw Failure(FMMGPU_UNSUPPORTED, "the Helmholtz far field needs every M2L product at once");
        hh_setup(kre);
        if (first_pass) launches = 0;
        const int64_t ns = dp.nsrc;
        const int L = plan.nlevels - 1;
        const int mv = 2 * m;
        const size_t set = (size_t)NE * NE;
        T* hM = hh.M.as<T>();
        T* hL = hh.L.as<T>();
        if (ns > 0)
            helm_charge_kernel<T><<<counted((unsigned)((ns + 255) / 256)), 256, 0, stream>>>(
                d_q, src_perm.as<int64_t>(), ns, m, qstride, hq.as<Cplx<T>>(), kMixed ? hq64.as<double2>() : nullptr);
        CUDA_TRY(cudaMemsetAsync(hh.M.ptr, 0, hh.M.bytes, stream));
        const int64_t top = plan.nlevels > 2 ? plan.level_start[2] : (int64_t)plan.nboxes();
        CUDA_TRY(cudaMemsetAsync(hh.L.ptr, 0, sizeof(T) * (size_t)mv * ms_of(P) * top, stream));
        const size_t esmem = sizeof(double) * (2 * NC * 32 + 2 * (size_t)m * 32);
        // upward: P2M of every leaf, then M2M from level L-1 up to 0
        if (plan.nleaves())
            hh_expand_kernel<P, T, false><<<counted((unsigned)plan.nleaves()), 32, esmem, stream>>>(
                dp, hh.lv, 0, (int64_t)plan.nleaves(), nullptr, m, spos.as<T4>(), hq.as<Cplx<T>>(), hM);
        constexpr int gsm = GemmShape<P, T, true>::SMEM;
        for (int l = L - 1; l >= 0; --l) {
            const int64_t t0 = m2m_tiles[l], nt = m2m_tiles[l + 1] - m2m_tiles[l];
            const int64_t n = m2m_start[l + 1] - m2m_start[l];
            if (nt)
                m2l_gemm_kernel<P, T, true><<<counted((unsigned)nt), 256, gsm, stream>>>(
                    oct_tile_d.as<int32_t>() + t0, oct_tile_begin.as<int64_t>() + t0,
                    oct_tile_count.as<int32_t>() + t0, oct_pair_e.as<int64_t>(), oct_pair_src.as<int32_t>(), m,
                    hh.m2m.as<T>() + (size_t)l * 8 * set, hM, hh.Yo.as<T>());
            if (n)
                m2m_reduce_kernel<P, T><<<counted((unsigned)n), round32(NC), 0, stream>>>(
                    dp, m2m_par.as<int32_t>() + m2m_start[l], n, mv, hh.Yo.as<T>(), hM);
        }
        // M2L products of every level (their tables are per level): the mixed form on the
        // tensor cores in one launch over every level, f64 on the SIMT GEMM level by level
        if constexpr (kHhTensor) {
            if (hh.tc_ntiles) {
                const unsigned grid = (unsigned)std::min<int64_t>(hh.tc_ntiles, num_sms);
                m2l_tc_kernel<P, true><<<counted(grid), 32 * kTcWarps, TcTs<P, true>::SMEM, stream>>>(
                    hh.tc_d.as<int32_t>(), hh.tc_begin.as<int64_t>(), hh.tc_count.as<int32_t>(), hh.tc_ntiles,
                    pair_src.as<int32_t>(), 2 * m, hh.tc_img.as<uint32_t>(), hh.mmap, hh.vmap,
                    reinterpret_cast<float*>(hh.Y.ptr), tc_error.as<int>());
            }
        } else {
            for (int l = 2; l <= L; ++l) {
                const int64_t t0 = lvl_tiles[l], nt = lvl_tiles[l + 1] - lvl_tiles[l];
                if (nt)
                    m2l_gemm_kernel<P, T, true><<<counted((unsigned)nt), 256, gsm, stream>>>(
                        ltile_d.as<int32_t>() + t0, ltile_begin.as<int64_t>() + t0, ltile_count.as<int32_t>() + t0,
                        nullptr, pair_src.as<int32_t>(), m, hh.m2l.as<T>() + (size_t)(l - 2) * 316 * set, hM,
                        hh.Y.as<T>());
            }
        }
        // downward: per level the L2L products, the locals (L2L + V in offset order), P2L
        for (int l = 2; l <= L; ++l) {
            if (l >= 3) {
                const int64_t t0 = l2l_tiles[l], nt = l2l_tiles[l + 1] - l2l_tiles[l];
                if (nt)
                    m2l_gemm_kernel<P, T, true><<<counted((unsigned)nt), 256, gsm, stream>>>(
                        oct_tile_d.as<int32_t>() + t0, oct_tile_begin.as<int64_t>() + t0,
                        oct_tile_count.as<int32_t>() + t0, oct_pair_e.as<int64_t>(), oct_pair_src.as<int32_t>(), m,
                        hh.l2l.as<T>() + (size_t)l * 8 * set, hL, hh.Yo.as<T>());
            }
            const int64_t b0 = plan.level_start[l], b1 = plan.level_start[l + 1];
            if (b1 > b0) {
                if constexpr (kHhTensor)
                    hh_local_reduce_tc_kernel<P><<<counted((unsigned)(b1 - b0)), round32(NC), 0, stream>>>(
                        dp, b0, b1, m, l >= 3, reinterpret_cast<const float*>(hh.Yo.ptr),
                        reinterpret_cast<const float*>(hh.Y.ptr), v_pos.as<int64_t>(),
                        reinterpret_cast<float*>(hh.L.ptr));
                else if constexpr (kMixed)
                    local_reduce4_kernel<P, false><<<counted((unsigned)((b1 - b0 + 3) / 4)), 128, 0, stream>>>(
                        dp, b0, b1, mv, l >= 3, 1, 0, reinterpret_cast<const float*>(hh.Yo.ptr),
                        reinterpret_cast<const float*>(hh.Y.ptr), v_pos.as<int64_t>(),
                        reinterpret_cast<float*>(hh.L.ptr));
                else
                    local_reduce_kernel<P, T><<<counted((unsigned)(b1 - b0)), round32(NC), 0, stream>>>(
                        dp, b0, b1, mv, l >= 3, 1, 0, hh.Yo.as<T>(), hh.Y.as<T>(), v_pos.as<int64_t>(), hL);
            }
            const int64_t x0 = xbox_start[l], x1 = xbox_start[l + 1];
            if (x1 > x0)
                hh_expand_kernel<P, T, true><<<counted((unsigned)(x1 - x0)), 32, esmem, stream>>>(
                    dp, hh.lv, x0, x1, xbox.as<int32_t>(), m, spos.as<T4>(), hq.as<Cplx<T>>(), hL);
        }
        // leaves: L2P + M2P into the far partials, then the near field and the output pass
        if (plan.nleaves()) {
            if (gradients)
                hh_leaf_far_kernel<P, T, true><<<counted((unsigned)plan.nleaves()), 128, 0, stream>>>(
                    dp, hh.lv, 0, m, tpos.as<T4>(), hM, hL, hh.far_phi.as<double>(), hh.far_g.as<double>());
            else
                hh_leaf_far_kernel<P, T, false><<<counted((unsigned)plan.nleaves()), 128, 0, stream>>>(
                    dp, hh.lv, 0, m, tpos.as<T4>(), hM, hL, hh.far_phi.as<double>(), nullptr);
        }
        helm_near_launch(kre, kim, d_phi, d_grad, hh.far_phi.as<double>(), gradients ? hh.far_g.as<double>() : nullptr);
        CUDA_TRY(cudaGetLastError());
    }

    // the Helmholtz P2P of every leaf into the caller-order outputs, after adding the far
    // partials when given (far_phi [v][t][2], far_g [v][t][6], leaf order)
    void helm_near_launch(double kre, double kim, double* d_phi, double* d_grad, const double* far_phi,
                          const double* far_g) {
        if (!items.count) return;
        if constexpr (kMixed) {
            // one vector, a real wavenumber and the near rows' streams built: the streamed
            // kernel over the P2P work lists (item slots 32, 16, 8, 4)
            if (m == 1 && kim == 0.0 && p2p_path == 1) {
                const P2pStream st{st_rowpair.as<int64_t>(), st_xy.as<float4>(), st_zz.as<float2>(),
                                   st_idx.as<int2>()};
                for (int c = 0; c < kP2pClasses; ++c) {
                    const P2pItems it = plist[c];
                    if (!it.count) continue;
                    const HelmStArgs a{dp, it, kTheta2, kre, st, hq.as<Cplx<float>>(),
                                       reinterpret_cast<const float4*>(tpos.ptr), close, hq64.as<double2>(),
                                       far_phi, far_g, d_phi, gradients ? d_grad : nullptr};
                    const unsigned g = counted((unsigned)it.count);
                    if (gradients) {
                        if (c == 0) helm_st_kernel<true, 1><<<g, 32, 0, stream>>>(a);
                        else if (c == 1) helm_st_kernel<true, 2><<<g, 32, 0, stream>>>(a);
                        else if (c == 2) helm_st_kernel<true, 4><<<g, 32, 0, stream>>>(a);
                        else helm_st_kernel<true, 8><<<g, 32, 0, stream>>>(a);
                    } else {
                        if (c == 0) helm_st_kernel<false, 1><<<g, 32, 0, stream>>>(a);
                        else if (c == 1) helm_st_kernel<false, 2><<<g, 32, 0, stream>>>(a);
                        else if (c == 2) helm_st_kernel<false, 4><<<g, 32, 0, stream>>>(a);
                        else helm_st_kernel<false, 8><<<g, 32, 0, stream>>>(a);
                    }
                }
                return;
            }
        }
        const unsigned g = (unsigned)((items.count + kHelmWarps - 1) / kHelmWarps);
        if (gradients)
            helm_p2p_kernel<T, true, kMixed><<<counted(g), 32 * kHelmWarps, 0, stream>>>(
                dp, items, m, (T)kTheta2, kre, kim, spos.as<T4>(), hq.as<Cplx<T>>(), tpos.as<T4>(), close,
                hq64.as<double2>(), far_phi, far_g, d_phi, d_grad);
        else
            helm_p2p_kernel<T, false, kMixed><<<counted(g), 32 * kHelmWarps, 0, stream>>>(
                dp, items, m, (T)kTheta2, kre, kim, spos.as<T4>(), hq.as<Cplx<T>>(), tpos.as<T4>(), close,
                hq64.as<double2>(), far_phi, nullptr, d_phi, nullptr);
    }

    // ---- the Helmholtz near field (all leaves' P2P level calls) ----
    DevBuf hq, hq64;
    void helmholtz_near(double kre, double kim, const double* d_q, double* d_phi, double* d_grad) override {
        if (first_pass) launches = 0;
        const int64_t ns = dp.nsrc;
        if (!hq.ptr) {
            hq.alloc(sizeof(Cplx<T>) * (size_t)m * (ns + 1));
            if (kMixed) hq64.alloc(sizeof(double2) * (size_t)m * (ns + 1));
        }
        if (ns > 0)
            helm_charge_kernel<T><<<counted((unsigned)((ns + 255) / 256)), 256, 0, stream>>>(
                d_q, src_perm.as<int64_t>(), ns, m, qstride, hq.as<Cplx<T>>(), kMixed ? hq64.as<double2>() : nullptr);
        helm_near_launch(kre, kim, d_phi, d_grad, nullptr, nullptr);
        CUDA_TRY(cudaGetLastError());
    }

    // ---- level calls (the FmmOperator trait, fmm-plan/src/operator.rs:434-492) ----
    void op_begin(const double* d_charges) override {
        launches = 0;
        load_charges(d_charges);
        close_sums(stream);
        CUDA_TRY(cudaMemsetAsync(Lc.ptr, 0, Lc.bytes, stream));
        CUDA_TRY(cudaMemsetAsync(far_phi.ptr, 0, far_phi.bytes, stream));
        CUDA_TRY(cudaMemsetAsync(far_g.ptr, 0, far_g.bytes, stream));
    }

    void op_level(int kind, int l) override {
        const int L = plan.nlevels - 1;
        const int64_t f0 = plan.leaf_level_start[l], f1 = plan.leaf_level_start[l + 1];
        switch (kind) {
            case FMMGPU_OP_P2M: p2m_rows(f0, f1); break;
            case FMMGPU_OP_M2M: if (l < L) m2m_level(l); break;
            case FMMGPU_OP_L2L:
                if (l >= 3) {
                    l2l_products(l);
                    reduce_locals(l, 1, 0, 1);
                }
                break;
            case FMMGPU_OP_M2L:
                if (l >= 2 && m2l_path == 2) {
                    m2l_fused(l);
                } else if (l >= 2 && !chunks.empty()) {
                    for (const Chunk& c : chunks)
                        if (c.level == l) {
                            m2l_chunk(c);
                            reduce_chunk(c, 0, 1, 1);
                        }
                } else if (l >= 2) {
                    m2l_products(l);
                    reduce_locals(l, 0, 1, 1);
                }
                break;
            case FMMGPU_OP_P2L: if (l >= 2) p2l_level(l); break;
            case FMMGPU_OP_L2P: leaf_far(f0, f1, 5); break;
            case FMMGPU_OP_M2P: leaf_far(f0, f1, 6); break;
            case FMMGPU_OP_P2P: p2p_levels(l, l + 1, 1, 1, nullptr, nullptr); break;
            default: throw Failure(FMMGPU_INVALID_ARGUMENT, "unknown operator kind");
        }
        CUDA_TRY(cudaGetLastError());
    }

    void op_output(double* d_phi, double* d_grad) override {
        output(d_phi, d_grad, false);
        CUDA_TRY(cudaGetLastError());
    }
};

template <int P>
std::unique_ptr<EvaluatorBase> make_evaluator_at(bool mixed, const EvaluatorArgs& a, size_t* bytes) {
    if (mixed) {
        auto e = std::make_unique<Evaluator<P, float>>(a.plan, a.m2l, a.m2m, a.l2l, a.stream, a.m, a.gradients, a.us,
                                                       a.ut, a.fused, a.ybudget);
        *bytes = e->device_bytes();
        return e;
    }
    auto e = std::make_unique<Evaluator<P, double>>(a.plan, a.m2l, a.m2m, a.l2l, a.stream, a.m, a.gradients, a.us,
                                                    a.ut, false, a.ybudget);
    *bytes = e->device_bytes();
    return e;
}

}  // namespace fmmb
