// Host-side plan of the B200 FMM evaluator: the octree, the box index, the per-leaf
// point order and the U/V/W/X interaction lists, flattened into arrays that are
// uploaded once and read by the device kernels.
//
// Conventions follow the reference (tbetcke/fmm):
//  - Morton keys: octree/src/morton.rs (3 interleaved index bits per level, x highest,
//    << 15, level in the low 15 bits); child octant o = 4x + 2y + z.
//  - boxes are numbered level-major, key order within a level; leaves likewise
//    (the leaf numbering of fmm-plan/src/index.rs, one rank).
//  - list rule: fmm-plan/src/interaction_manager.rs:15-27; rows are sorted as the
//    accumulation rule of fmm-plan/src/operator.rs:34-45 orders them (V by offset
//    index, W by box index, X and near by source leaf).
//  - boxes with no source below them are left out of every source-side list and
//    boxes with no target below them get empty target rows (their contributions
//    are exact zeros in the reference).
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fmm_b200.h"

namespace fmmb {

constexpr int kDeepest = 16;

struct Csr {
    std::vector<int64_t> row;  // nrows + 1
    std::vector<int32_t> col;  // entries
    std::vector<int32_t> aux;  // optional per-entry payload (the offset index for V)
    size_t nnz() const { return col.size(); }
};

struct Plan {
    int nlevels = 0;
    double lower[3] = {0, 0, 0};
    double side = 0;
    double box6[6] = {0, 0, 0, 0, 0, 0};

    // boxes, level-major
    std::vector<uint64_t> key;
    std::vector<int32_t> level;          // per box
    std::vector<uint32_t> idx;           // 3 per box
    std::vector<int64_t> level_start;    // nlevels + 1
    std::vector<int32_t> parent;         // -1 for the root
    std::vector<int32_t> child_first;    // first of 8 consecutive children, -1 for leaves
    std::vector<int32_t> box_leaf;       // leaf index or -1
    std::vector<int64_t> src_below, tgt_below;

    // leaves, level-major
    std::vector<int32_t> leaf_box;
    std::vector<int64_t> leaf_level_start;  // nlevels + 1
    std::vector<int64_t> src_start, tgt_start;  // nleaves + 1 (points in leaf order)
    std::vector<int64_t> src_perm, tgt_perm;    // leaf-order position -> caller index
    std::vector<int64_t> src_pos_of, tgt_pos_of;  // caller index -> leaf-order position

    // interaction lists (rows: leaves for near/W, boxes for V/X)
    Csr near;  // source leaves, U-list and the leaf itself, by leaf index
    Csr w;     // source boxes on level l + 1, by box index
    Csr x;     // source leaves on level l - 1, by leaf index
    Csr v;     // source boxes with aux = offset index, by offset index

    // forests (merge_plans): the domain side of each box's tree; empty for one tree
    std::vector<double> box_side;

    size_t nboxes() const { return key.size(); }
    size_t nleaves() const { return leaf_box.size(); }
};

// One cloud of a batch: its plan, its leaf-scaled coordinates (plan leaf order) and the
// offsets of its points in the batch's concatenated caller order.
struct TreePart {
    Plan plan;
    std::vector<double> us, ut;
    int64_t src_offset = 0, tgt_offset = 0;
};

// Host threads for a stage over n independent items: one below 2^16 items, else up to
// `limit` (0: the host's cores, at most 16).
size_t stage_threads(size_t n, int limit = 0);
// fn(t, begin, end) for the chunks t = 0..nth-1 of [0, n), chunk t on its own thread (chunk
// 0 on the calling one).  A thread that cannot be started has its chunk run on the calling
// thread, so every chunk runs exactly once; an exception from a chunk is rethrown here once
// every chunk has ended (the first chunk's that threw).
void for_chunks(size_t n, size_t nth, const std::function<void(size_t, size_t, size_t)>& fn);

// The forest of several clouds' plans (forest.cpp): level-major over all trees, with the
// merged leaf-scaled coordinates in us / ut.
Plan merge_plans(std::vector<TreePart>& parts, std::vector<double>& us, std::vector<double>& ut);

// Builds the cubic domain, the tree of the distinct level-16 keys of sources ++ targets
// (refined while a box holds more than max_keys keys, then 2:1 balanced), the box
// index, the point order and the lists.  Throws std::runtime_error on bad input.
// device_points: the point stages (keys, sort, each point's leaf, the order by leaf) on the
// current CUDA device (plan_gpu.cu), with the same results.  Otherwise they run on up to
// host_threads host threads (0: the host's cores, at most 16; 1: this thread only), with
// the same results for every thread count.
Plan build_plan(size_t ns, const double* src, size_t nt, const double* tgt, int max_level,
                int max_keys, bool device_points = false, int host_threads = 0);

// The point stages of a build: the level-16 keys of sources ++ targets sorted and made
// distinct, then, once the leaves are known (their first level-16 keys ascending and their
// leaf indices), each point's leaf and the stable order of the points by leaf.
struct PointSort {
    virtual ~PointSort() = default;
    virtual std::vector<uint64_t> distinct_keys() = 0;
    virtual void leaf_order(const std::vector<uint64_t>& firsts, const std::vector<int32_t>& leaf_index, size_t nl,
                            Plan& P) = 0;
};
std::unique_ptr<PointSort> device_point_sort(size_t ns, const double* src, size_t nt, const double* tgt,
                                             const double box6[6]);
// The mixed P2P's near-singular pairs (target t[i], source s[i], source leaf l[i], device
// arrays of n) sorted by (target, source) into a CSR by target: row[ntgt + 1], src[n],
// leaf[n], device arrays (plan_gpu.cu); synchronises.
void sort_close_pairs(int64_t n, const int64_t* t, const int64_t* s, const int32_t* l, int64_t ntgt, int64_t* row,
                      int64_t* src, int32_t* leaf);

// Leaf-scaled coordinate of CONVENTIONS 3.13: fl(fl(fl(x - a) * 2^(l+1)) / w) - (2i + 1).
double leaf_coordinate(double x, double a, double w, int level, uint32_t index);

// M2L offset index of d = index(target) - index(source) (fmm-tables/src/geometry.rs:90)
int offset_index(int dx, int dy, int dz);

// Morton keys (octree/src/morton.rs): encode the integer coordinates of a box of a level,
// decode them, read the level
uint64_t morton_encode(uint32_t i, uint32_t j, uint32_t k, int level);
void morton_decode(uint64_t key, uint32_t out[3]);
int morton_level(uint64_t key);

// A plan given in the reference's flattened layout (fmmgpu_plan_arrays), checked
// (plan_upload.cpp); throws std::runtime_error naming the first failed check.
Plan plan_from_arrays(const fmmgpu_plan_arrays& a, size_t ns, size_t nt);

// Operator tables (column-major, (p+1)^2 x (p+1)^2 each), built in f64 from the direct
// translations applied to unit vectors (fmm-tables/src/m2l.rs:67-96, octant.rs:150-174).
void build_m2l_tables(int p, std::vector<double>& out);  // 316 matrices
void build_m2m_tables(int p, std::vector<double>& out);  // 8
void build_l2l_tables(int p, std::vector<double>& out);  // 8
// Helmholtz (real k): the dense M2L tables of one level of boxes of half-width r, 316 real
// 2n x n matrices in offset index order (helmholtz_tables.cpp)
void build_helmholtz_m2l_tables(int p, double k, double r, std::vector<double>& out);
// and the 8 octants' M2M (child multipole -> parent) and L2L (parent local -> child) tables
// of a parent level of half-width r, real 2n x n matrices each
void build_helmholtz_octant_tables(int p, double k, double r, std::vector<double>& m2m, std::vector<double>& l2l);

// On-disk caches (table_cache.cpp): the operator tables in the reference's TableCache
// format (fmm-tables/src/cache.rs; kind codes 1 M2M, 2 L2L, 3 M2L; the Helmholtz tables of
// a level under codes 65 and 66 with k_l in the name), f64, and the autotuner's choices in
// the layout of its TuningCache (fmm-exec/src/tune.rs:118-140).  Loads return false with
// the reason in *why (missing, or which check rejected the file); stores are atomic.
enum { kTableM2m = 1, kTableL2l = 2, kTableM2l = 3, kTableHelmholtzM2l = 65, kTableHelmholtzOctant = 66 };
std::string table_cache_file_name(int kind, int p, double k = 0.0);
bool table_cache_store(const std::string& dir, int kind, int p, double k, const std::vector<double>& values,
                       std::string* why);
bool table_cache_load(const std::string& dir, int kind, int p, double k, size_t count, std::vector<double>& values,
                      std::string* why);
struct TuningKey {
    std::string device, compiler, precision;
    int p = 0;
};
std::string tuning_cache_file_name(const TuningKey& key);
bool tuning_cache_load(const std::string& dir, const TuningKey& key, std::map<std::string, int>& entries,
                       std::string* why);
bool tuning_cache_store(const std::string& dir, const TuningKey& key, const std::map<std::string, int>& entries,
                        std::string* why);

}  // namespace fmmb
