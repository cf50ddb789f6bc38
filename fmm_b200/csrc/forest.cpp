// Multi-cloud batching: independent octrees merged into one level-major forest plan, so
// that every pass of an evaluation is one launch over all the clouds (the M2L batches by
// offset then span every cloud: one GEMM per offset for the whole batch).
//
// Boxes of level l are those of every tree's level l, tree by tree, each tree's boxes in
// their own order; leaves likewise; points follow the merged leaf order.  Every index map
// is monotone within a tree, so the rows of the lists keep their accumulation order
// (fmm-plan/src/operator.rs:34-45) and each cloud's results are those of its own plan.
// The reference batches only charge vectors (FmmBuilder::vectors, fmm-exec/src/fmm.rs:
// 200-227); the forest is this library's own form of its clouds-in-one-launch target.
#include <algorithm>
#include <stdexcept>

#include "plan.hpp"

namespace fmmb {

Plan merge_plans(std::vector<TreePart>& parts, std::vector<double>& us, std::vector<double>& ut) {
    const size_t T = parts.size();
    if (T == 0) throw std::runtime_error("no clouds");
    Plan M;
    int L = 0;
    size_t nbox = 0, nleaf = 0, nsrc = 0, ntgt = 0;
    for (auto& p : parts) {
        L = std::max(L, p.plan.nlevels);
        nbox += p.plan.nboxes();
        nleaf += p.plan.nleaves();
        nsrc += p.plan.src_perm.size();
        ntgt += p.plan.tgt_perm.size();
    }
    if (nbox >= ((size_t)1 << 31)) throw std::runtime_error("too many boxes for 32-bit box indices");
    M.nlevels = L;
    M.side = parts[0].plan.side;
    for (int k = 0; k < 3; ++k) M.lower[k] = parts[0].plan.lower[k];
    for (int k = 0; k < 6; ++k) M.box6[k] = parts[0].plan.box6[k];
    // boxes, level by level, tree by tree
    std::vector<std::vector<int32_t>> bmap(T), lmap(T);
    std::vector<int32_t> box_tree(nbox), box_old(nbox), leaf_tree(nleaf), leaf_old(nleaf);
    for (size_t t = 0; t < T; ++t) {
        bmap[t].assign(parts[t].plan.nboxes(), -1);
        lmap[t].assign(parts[t].plan.nleaves(), -1);
    }
    M.level_start.assign(L + 1, 0);
    M.leaf_level_start.assign(L + 1, 0);
    int32_t nb = 0, nl = 0;
    for (int l = 0; l < L; ++l) {
        M.level_start[l] = nb;
        M.leaf_level_start[l] = nl;
        for (size_t t = 0; t < T; ++t) {
            const Plan& P = parts[t].plan;
            if (l >= P.nlevels) continue;
            for (int64_t b = P.level_start[l]; b < P.level_start[l + 1]; ++b) {
                bmap[t][b] = nb;
                box_tree[nb] = (int32_t)t;
                box_old[nb] = (int32_t)b;
                ++nb;
            }
            for (int64_t j = P.leaf_level_start[l]; j < P.leaf_level_start[l + 1]; ++j) {
                lmap[t][j] = nl;
                leaf_tree[nl] = (int32_t)t;
                leaf_old[nl] = (int32_t)j;
                ++nl;
            }
        }
    }
    M.level_start[L] = nb;
    M.leaf_level_start[L] = nl;
    // per box (every output slot written by exactly one chunk: the same arrays for any
    // number of host threads)
    M.key.resize(nbox);
    M.level.resize(nbox);
    M.idx.resize(3 * nbox);
    M.parent.resize(nbox);
    M.child_first.resize(nbox);
    M.box_leaf.resize(nbox);
    M.src_below.resize(nbox);
    M.tgt_below.resize(nbox);
    M.box_side.resize(nbox);
    for_chunks(nbox, stage_threads(nbox), [&](size_t, size_t n0, size_t n1) {
        for (size_t n = n0; n < n1; ++n) {
            const int t = box_tree[n], b = box_old[n];
            const Plan& P = parts[t].plan;
            M.key[n] = P.key[b];
            M.level[n] = P.level[b];
            for (int k = 0; k < 3; ++k) M.idx[3 * n + k] = P.idx[3 * b + k];
            M.parent[n] = P.parent[b] < 0 ? -1 : bmap[t][P.parent[b]];
            M.child_first[n] = P.child_first[b] < 0 ? -1 : bmap[t][P.child_first[b]];
            M.box_leaf[n] = P.box_leaf[b] < 0 ? -1 : lmap[t][P.box_leaf[b]];
            M.src_below[n] = P.src_below[b];
            M.tgt_below[n] = P.tgt_below[b];
            M.box_side[n] = P.side;
        }
    });
    // per leaf, with the points in merged leaf order: each leaf's first position from the
    // counts of the leaves before it, then the leaves filled independently
    M.leaf_box.resize(nleaf);
    M.src_start.assign(nleaf + 1, 0);
    M.tgt_start.assign(nleaf + 1, 0);
    for (size_t n = 0; n < nleaf; ++n) {
        const Plan& P = parts[leaf_tree[n]].plan;
        const int j = leaf_old[n];
        M.src_start[n + 1] = M.src_start[n] + (P.src_start[j + 1] - P.src_start[j]);
        M.tgt_start[n + 1] = M.tgt_start[n] + (P.tgt_start[j + 1] - P.tgt_start[j]);
    }
    M.src_perm.resize(nsrc);
    M.tgt_perm.resize(ntgt);
    us.resize(3 * nsrc);
    ut.resize(3 * ntgt);
    for_chunks(nleaf, stage_threads(nleaf), [&](size_t, size_t n0, size_t n1) {
        for (size_t n = n0; n < n1; ++n) {
            const int t = leaf_tree[n], j = leaf_old[n];
            const TreePart& tp = parts[t];
            const Plan& P = tp.plan;
            M.leaf_box[n] = bmap[t][P.leaf_box[j]];
            int64_t ps = M.src_start[n];
            for (int64_t a = P.src_start[j]; a < P.src_start[j + 1]; ++a, ++ps) {
                M.src_perm[ps] = P.src_perm[a] + tp.src_offset;
                for (int k = 0; k < 3; ++k) us[3 * ps + k] = tp.us[3 * a + k];
            }
            int64_t pt = M.tgt_start[n];
            for (int64_t a = P.tgt_start[j]; a < P.tgt_start[j + 1]; ++a, ++pt) {
                M.tgt_perm[pt] = P.tgt_perm[a] + tp.tgt_offset;
                for (int k = 0; k < 3; ++k) ut[3 * pt + k] = tp.ut[3 * a + k];
            }
        }
    });
    M.src_pos_of.assign(nsrc, 0);
    M.tgt_pos_of.assign(ntgt, 0);
    for_chunks(nsrc, stage_threads(nsrc), [&](size_t, size_t a0, size_t a1) {
        for (size_t a = a0; a < a1; ++a) M.src_pos_of[M.src_perm[a]] = (int64_t)a;
    });
    for_chunks(ntgt, stage_threads(ntgt), [&](size_t, size_t a0, size_t a1) {
        for (size_t a = a0; a < a1; ++a) M.tgt_pos_of[M.tgt_perm[a]] = (int64_t)a;
    });
    // lists: rows in merged order, columns through the maps (monotone within a tree); the
    // row ends from the rows' lengths, then the rows filled independently
    auto remap = [&](Csr& out, bool leaf_rows, const Csr Plan::*which, bool leaf_cols) {
        const size_t nrows = leaf_rows ? nleaf : nbox;
        out.row.assign(nrows + 1, 0);
        bool with_aux = false;
        for (size_t t = 0; t < T; ++t) with_aux |= !(parts[t].plan.*which).aux.empty();
        for (size_t n = 0; n < nrows; ++n) {
            const int t = leaf_rows ? leaf_tree[n] : box_tree[n];
            const int r = leaf_rows ? leaf_old[n] : box_old[n];
            const Csr& c = parts[t].plan.*which;
            out.row[n + 1] = out.row[n] + (c.row[r + 1] - c.row[r]);
        }
        out.col.assign((size_t)out.row[nrows], 0);
        out.aux.assign(with_aux ? (size_t)out.row[nrows] : 0, 0);
        for_chunks(nrows, stage_threads(nrows), [&](size_t, size_t n0, size_t n1) {
            for (size_t n = n0; n < n1; ++n) {
                const int t = leaf_rows ? leaf_tree[n] : box_tree[n];
                const int r = leaf_rows ? leaf_old[n] : box_old[n];
                const Csr& c = parts[t].plan.*which;
                const std::vector<int32_t>& map = leaf_cols ? lmap[t] : bmap[t];
                int64_t o = out.row[n];
                for (int64_t e = c.row[r]; e < c.row[r + 1]; ++e, ++o) {
                    out.col[o] = map[c.col[e]];
                    if (!c.aux.empty()) out.aux[o] = c.aux[e];
                }
            }
        });
    };
    remap(M.near, true, &Plan::near, true);
    remap(M.w, true, &Plan::w, false);
    remap(M.x, false, &Plan::x, true);
    remap(M.v, false, &Plan::v, false);
    return M;
}

}  // namespace fmmb
