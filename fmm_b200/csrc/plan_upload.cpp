// A plan given by the caller in the reference's layout (fmmgpu_plan_arrays of
// include/fmm_b200.h: fmm-plan's one-rank Plan and the CSR views its level calls receive,
// fmm-plan/src/operator.rs:170-317, fmm-plan/src/lists.rs:172-282), checked and turned
// into the evaluator's Plan; and the export of a Plan in the same layout.
//
// The checks are those the evaluator's kernels rely on (every index in range, the tree
// complete with its children consecutive, lists between the levels the operators assume,
// V offsets equal to the boxes' displacement) and the accumulation order of the rows
// (operator.rs:34-45); a failed check throws std::runtime_error naming it.
#include <cmath>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fmm_b200.h"
#include "plan.hpp"

namespace fmmb {

namespace {

[[noreturn]] void bad(const std::string& what) { throw std::runtime_error("uploaded plan: " + what); }

void check_rows(const int64_t* rows, size_t nrows, const char* name) {
    if (!rows) bad(std::string("null ") + name + " rows");
    if (rows[0] != 0) bad(std::string(name) + " rows must start at 0");
    for (size_t r = 0; r < nrows; ++r)
        if (rows[r + 1] < rows[r]) bad(std::string(name) + " rows decrease at row " + std::to_string(r));
}

Csr copy_csr(const int64_t* rows, const int32_t* cols, const int32_t* aux, size_t nrows) {
    Csr c;
    c.row.assign(rows, rows + nrows + 1);
    const size_t nnz = (size_t)rows[nrows];
    if (nnz && !cols) bad("null list entries");
    c.col.assign(cols, cols + nnz);
    if (aux) c.aux.assign(aux, aux + nnz);
    return c;
}

}  // namespace

Plan plan_from_arrays(const fmmgpu_plan_arrays& a, size_t ns, size_t nt) {
    if (a.nlevels < 1 || a.nlevels > kDeepest + 1) bad("nlevels must be 1 to 17");
    if (!a.level_start || !a.keys || !a.is_leaf) bad("null box arrays");
    if (!(a.side > 0.0) || !std::isfinite(a.side) || !std::isfinite(a.lower[0]) || !std::isfinite(a.lower[1]) ||
        !std::isfinite(a.lower[2]))
        bad("the domain must be finite with a positive side");
    Plan P;
    P.nlevels = a.nlevels;
    P.side = a.side;
    for (int k = 0; k < 3; ++k) {
        P.lower[k] = a.lower[k];
        P.box6[k] = a.lower[k];
        P.box6[k + 3] = a.lower[k] + a.side;
    }
    // ---- boxes ----
    P.level_start.assign(a.level_start, a.level_start + a.nlevels + 1);
    if (P.level_start[0] != 0 || P.level_start[1] != 1) bad("level 0 must hold the root alone");
    for (int l = 0; l < a.nlevels; ++l)
        if (P.level_start[l + 1] < P.level_start[l]) bad("level_start decreases");
    const size_t nb = (size_t)P.level_start[a.nlevels];
    if (nb >= ((size_t)1 << 31)) bad("too many boxes");
    P.key.assign(a.keys, a.keys + nb);
    P.level.assign(nb, 0);
    P.idx.assign(3 * nb, 0);
    std::unordered_map<uint64_t, int32_t> at;
    at.reserve(nb * 2);
    for (int l = 0; l < a.nlevels; ++l)
        for (int64_t b = P.level_start[l]; b < P.level_start[l + 1]; ++b) {
            const uint64_t k = P.key[b];
            if (morton_level(k) != l) bad("box " + std::to_string(b) + ": its key is not of level " + std::to_string(l));
            if (b > P.level_start[l] && !(P.key[b - 1] < k)) bad("keys of level " + std::to_string(l) + " not ascending");
            P.level[b] = l;
            morton_decode(k, &P.idx[3 * b]);
            if (morton_encode(P.idx[3 * b], P.idx[3 * b + 1], P.idx[3 * b + 2], l) != k)
                bad("box " + std::to_string(b) + ": not a valid key");
            at.emplace(k, (int32_t)b);
        }
    P.parent.assign(nb, -1);
    P.child_first.assign(nb, -1);
    P.box_leaf.assign(nb, -1);
    P.leaf_level_start.assign(a.nlevels + 1, 0);
    for (size_t b = 0; b < nb; ++b) {
        if (a.is_leaf[b] > 1) bad("is_leaf must be 0 or 1");
        const int l = P.level[b];
        if (l > 0) {
            uint32_t pi[3] = {P.idx[3 * b] >> 1, P.idx[3 * b + 1] >> 1, P.idx[3 * b + 2] >> 1};
            auto it = at.find(morton_encode(pi[0], pi[1], pi[2], l - 1));
            if (it == at.end()) bad("box " + std::to_string(b) + " has no parent");
            P.parent[b] = it->second;
            if (a.is_leaf[it->second]) bad("box " + std::to_string(b) + " has a leaf for parent");
        }
        if (!a.is_leaf[b]) {
            if (l + 1 >= a.nlevels) bad("box " + std::to_string(b) + " is no leaf but has no level below");
            int32_t first = -1;
            for (int o = 0; o < 8; ++o) {
                const uint32_t ci = 2 * P.idx[3 * b] + ((o >> 2) & 1), cj = 2 * P.idx[3 * b + 1] + ((o >> 1) & 1),
                               ck = 2 * P.idx[3 * b + 2] + (o & 1);
                auto it = at.find(morton_encode(ci, cj, ck, l + 1));
                if (it == at.end()) bad("box " + std::to_string(b) + " lacks child " + std::to_string(o));
                if (o == 0) first = it->second;
                else if (it->second != first + o) bad("the children of box " + std::to_string(b) + " are not consecutive");
            }
            P.child_first[b] = first;
        } else {
            P.box_leaf[b] = (int32_t)P.leaf_box.size();
            P.leaf_box.push_back((int32_t)b);
            P.leaf_level_start[l + 1] = (int64_t)P.leaf_box.size();
        }
    }
    for (int l = 1; l <= a.nlevels; ++l) P.leaf_level_start[l] = std::max(P.leaf_level_start[l], P.leaf_level_start[l - 1]);
    const size_t nl = P.leaf_box.size();
    // ---- points ----
    if (!a.source_offsets || !a.target_offsets || (ns && !a.source_order) || (nt && !a.target_order))
        bad("null point arrays");
    for (int s = 0; s < 2; ++s) {
        const int64_t* off = s ? a.target_offsets : a.source_offsets;
        const int64_t* order = s ? a.target_order : a.source_order;
        const size_t n = s ? nt : ns;
        const char* name = s ? "target" : "source";
        if (off[0] != 0 || off[nl] != (int64_t)n) bad(std::string(name) + " offsets must run from 0 to the count");
        for (size_t j = 0; j < nl; ++j)
            if (off[j + 1] < off[j]) bad(std::string(name) + " offsets decrease");
        std::vector<int64_t> pos_of(n, -1);
        for (size_t i = 0; i < n; ++i) {
            const int64_t c = order[i];
            if (c < 0 || c >= (int64_t)n || pos_of[c] >= 0) bad(std::string(name) + " order is not a permutation");
            pos_of[c] = (int64_t)i;
        }
        std::vector<int64_t> start(off, off + nl + 1), perm(order, order + n);
        if (s) {
            P.tgt_start.swap(start);
            P.tgt_perm.swap(perm);
            P.tgt_pos_of.swap(pos_of);
        } else {
            P.src_start.swap(start);
            P.src_perm.swap(perm);
            P.src_pos_of.swap(pos_of);
        }
    }
    P.src_below.assign(nb, 0);
    P.tgt_below.assign(nb, 0);
    for (size_t j = 0; j < nl; ++j) {
        P.src_below[P.leaf_box[j]] = P.src_start[j + 1] - P.src_start[j];
        P.tgt_below[P.leaf_box[j]] = P.tgt_start[j + 1] - P.tgt_start[j];
    }
    for (size_t b = nb; b-- > 1;) {
        P.src_below[P.parent[b]] += P.src_below[b];
        P.tgt_below[P.parent[b]] += P.tgt_below[b];
    }
    // ---- lists ----
    check_rows(a.near_rows, nl, "near");
    check_rows(a.w_rows, nl, "W");
    check_rows(a.x_rows, nb, "X");
    check_rows(a.v_rows, nb, "V");
    P.near = copy_csr(a.near_rows, a.near, nullptr, nl);
    P.w = copy_csr(a.w_rows, a.w, nullptr, nl);
    P.x = copy_csr(a.x_rows, a.x, nullptr, nb);
    if (a.v_rows[nb] && !a.v_offsets) bad("null V offsets");
    P.v = copy_csr(a.v_rows, a.v, a.v_offsets, nb);
    for (size_t j = 0; j < nl; ++j) {
        const int lt = P.level[P.leaf_box[j]];
        for (int64_t e = P.near.row[j]; e < P.near.row[j + 1]; ++e) {
            const int32_t s = P.near.col[e];
            if (s < 0 || (size_t)s >= nl) bad("near entry out of range in row " + std::to_string(j));
            if (e > P.near.row[j] && P.near.col[e - 1] >= s) bad("near row " + std::to_string(j) + " not ascending");
            const int ls = P.level[P.leaf_box[s]];
            if (ls < lt - 1 || ls > lt + 1) bad("near row " + std::to_string(j) + " reaches beyond one level");
        }
        for (int64_t e = P.w.row[j]; e < P.w.row[j + 1]; ++e) {
            const int32_t s = P.w.col[e];
            if (s < 0 || (size_t)s >= nb || P.level[s] != lt + 1)
                bad("W entry of row " + std::to_string(j) + " is no box of the next level");
            if (e > P.w.row[j] && P.w.col[e - 1] >= s) bad("W row " + std::to_string(j) + " not ascending");
        }
    }
    for (size_t b = 0; b < nb; ++b) {
        const int l = P.level[b];
        for (int64_t e = P.x.row[b]; e < P.x.row[b + 1]; ++e) {
            const int32_t s = P.x.col[e];
            if (s < 0 || (size_t)s >= nl || P.level[P.leaf_box[s]] != l - 1)
                bad("X entry of box " + std::to_string(b) + " is no leaf of the level above");
            if (e > P.x.row[b] && P.x.col[e - 1] >= s) bad("X row " + std::to_string(b) + " not ascending");
        }
        for (int64_t e = P.v.row[b]; e < P.v.row[b + 1]; ++e) {
            const int32_t s = P.v.col[e];
            if (s < 0 || (size_t)s >= nb || P.level[s] != l) bad("V entry of box " + std::to_string(b) + " is no box of its level");
            const int d = P.v.aux[e];
            const int want = offset_index((int)P.idx[3 * b] - (int)P.idx[3 * s], (int)P.idx[3 * b + 1] - (int)P.idx[3 * s + 1],
                                          (int)P.idx[3 * b + 2] - (int)P.idx[3 * s + 2]);
            if (d < 0 || d >= 316 || d != want) bad("V offset of box " + std::to_string(b) + " is not its displacement's");
            if (e > P.v.row[b] && P.v.aux[e - 1] >= d) bad("V row " + std::to_string(b) + " not by offset index");
        }
    }
    return P;
}

}  // namespace fmmb
