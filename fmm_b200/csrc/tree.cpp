// Host plan build: domain, Morton keys, refinement, 2:1 balance, box index, point
// order and interaction lists (see plan.hpp for the conventions it follows).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>

#include "morton.hpp"
#include "plan.hpp"

namespace fmmb {

namespace {

constexpr uint64_t kLevelMask = 0x7FFF;

inline uint64_t compact3(uint64_t x) {
    x &= 0x1249249249249249ULL;
    x = (x ^ (x >> 2)) & 0x10C30C30C30C30C3ULL;
    x = (x ^ (x >> 4)) & 0x100F00F00F00F00FULL;
    x = (x ^ (x >> 8)) & 0x1F0000FF0000FFULL;
    x = (x ^ (x >> 16)) & 0x1F00000000FFFFULL;
    x = (x ^ (x >> 32)) & 0x1FFFFFULL;
    return x;
}

inline uint64_t encode(uint32_t i, uint32_t j, uint32_t k, int level) { return morton_encode_hd(i, j, k, level); }

inline int key_level(uint64_t key) { return (int)(key & kLevelMask); }

inline void decode(uint64_t key, uint32_t out[3]) {
    int l = key_level(key);
    uint64_t m = key >> 15;
    out[0] = (uint32_t)(compact3(m >> 2) >> (kDeepest - l));
    out[1] = (uint32_t)(compact3(m >> 1) >> (kDeepest - l));
    out[2] = (uint32_t)(compact3(m) >> (kDeepest - l));
}

inline uint64_t parent_key(uint64_t key) {
    int l = key_level(key);
    uint64_t keep = ~0ULL << (15 + 3 * (kDeepest - l + 1));
    return (key & keep) | (uint64_t)(l - 1);
}

inline uint64_t child_key(uint64_t key, int o) {
    int l = key_level(key);
    return ((key & ~kLevelMask) | ((uint64_t)o << (15 + 3 * (kDeepest - l - 1)))) | (uint64_t)(l + 1);
}

inline uint64_t first_fine(uint64_t key) { return (key & ~kLevelMask) | (uint64_t)kDeepest; }

void sort_unique(std::vector<uint64_t>& v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

// sort_unique with the chunks sorted on nth threads and merged pairwise (the same values)
void sort_unique_threads(std::vector<uint64_t>& v, size_t nth) {
    if (nth <= 1) return sort_unique(v);
    const size_t n = v.size();
    std::vector<size_t> edge(nth + 1);
    for (size_t t = 0; t <= nth; ++t) edge[t] = n * t / nth;
    for_chunks(nth, nth, [&](size_t t, size_t, size_t) { std::sort(v.begin() + edge[t], v.begin() + edge[t + 1]); });
    for (size_t w = 1; w < nth; w *= 2) {
        const size_t pairs = (nth + 2 * w - 1) / (2 * w);
        for_chunks(pairs, pairs, [&](size_t i, size_t, size_t) {
            const size_t a = 2 * w * i, b = std::min(a + w, nth), c = std::min(a + 2 * w, nth);
            if (b < c) std::inplace_merge(v.begin() + edge[a], v.begin() + edge[b], v.begin() + edge[c]);
        });
    }
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

// LSD radix sort of level-16 keys with their point numbers, 8 bits a pass over bits 15..62
// (the Morton code; the level bits are the same in every key): stable, so equal keys keep
// their points' order.  A pass whose byte is the same in every key is skipped.
void radix_sort_keys(std::vector<uint64_t>& key, std::vector<uint32_t>& id) {
    const size_t n = key.size();
    std::vector<uint64_t> k2(n);
    std::vector<uint32_t> i2(n);
    for (int shift = 15; shift < 63; shift += 8) {
        size_t start[257] = {0};
        for (size_t i = 0; i < n; ++i) start[((key[i] >> shift) & 0xFF) + 1]++;
        bool one_bucket = false;
        for (int b = 0; b < 256; ++b) one_bucket |= start[b + 1] == n;
        if (one_bucket) continue;
        for (int b = 0; b < 256; ++b) start[b + 1] += start[b];
        for (size_t i = 0; i < n; ++i) {
            const size_t d = start[(key[i] >> shift) & 0xFF]++;
            k2[d] = key[i];
            i2[d] = id[i];
        }
        key.swap(k2);
        id.swap(i2);
    }
}

// create_local_tree of octree/src/octree/implementation.rs:682-730 from the root:
// a box splits while it holds more than max_keys distinct keys and lies above max_level.
void refine(const uint64_t* fine, size_t n, uint64_t box, int max_level, size_t max_keys,
            std::vector<uint64_t>& out) {
    if (key_level(box) < max_level && n > max_keys) {
        const uint64_t* begin = fine;
        for (int o = 0; o < 8; ++o) {
            const uint64_t* end = fine + n;
            if (o < 7) end = std::lower_bound(begin, fine + n, first_fine(child_key(box, o + 1)));
            refine(begin, (size_t)(end - begin), child_key(box, o), max_level, max_keys, out);
            begin = end;
        }
    } else {
        out.push_back(box);
    }
}

// 2:1 balance over all 26 directions, as the closure of
// octree/src/octree/implementation.rs:1069-1103: from the deepest level up, every
// parent of a required box is split (its 8 children exist), and the neighbours of that
// parent become required on the level above.  Returns the balanced leaves, sorted.
std::vector<uint64_t> balance(const std::vector<uint64_t>& leaves) {
    int deepest = 0;
    for (uint64_t k : leaves) deepest = std::max(deepest, key_level(k));
    if (deepest == 0) return leaves;
    std::vector<std::vector<uint64_t>> by_level(deepest + 1);
    for (uint64_t k : leaves) by_level[key_level(k)].push_back(k);
    std::vector<uint64_t> interior, generated;
    std::vector<uint64_t> work = by_level[deepest];
    for (int l = deepest; l >= 1; --l) {
        std::vector<uint64_t> parents;
        parents.reserve(work.size());
        for (uint64_t k : work) parents.push_back(parent_key(k));
        sort_unique(parents);
        std::vector<uint64_t> next = by_level[l - 1];
        for (uint64_t par : parents) {
            interior.push_back(par);
            for (int o = 0; o < 8; ++o) generated.push_back(child_key(par, o));
            uint32_t ix[3];
            decode(par, ix);
            int pl = l - 1;
            int64_t size = (int64_t)1 << pl;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        if (!dx && !dy && !dz) continue;
                        int64_t a = (int64_t)ix[0] + dx, b = (int64_t)ix[1] + dy, c = (int64_t)ix[2] + dz;
                        if (a < 0 || b < 0 || c < 0 || a >= size || b >= size || c >= size) continue;
                        next.push_back(encode((uint32_t)a, (uint32_t)b, (uint32_t)c, pl));
                    }
        }
        sort_unique(next);
        work.swap(next);
    }
    sort_unique(interior);
    sort_unique(generated);
    std::vector<uint64_t> out;
    out.reserve(generated.size());
    for (uint64_t k : generated)
        if (!std::binary_search(interior.begin(), interior.end(), k)) out.push_back(k);
    return out;
}

struct KeyMap {
    std::unordered_map<uint64_t, int32_t> map;
    int32_t find(uint64_t k) const {
        auto it = map.find(k);
        return it == map.end() ? -1 : it->second;
    }
};

inline bool is_ancestor(uint64_t a, uint64_t b) {
    int la = key_level(a), lb = key_level(b);
    if (la >= lb) return false;
    uint64_t mask = ~0ULL << (15 + 3 * (kDeepest - la));
    return ((a ^ b) & mask) == 0;
}

// closed cubes intersect and neither is an ancestor of the other
bool adjacent(const Plan& P, int32_t a, int32_t b) {
    if (a == b || is_ancestor(P.key[a], P.key[b]) || is_ancestor(P.key[b], P.key[a])) return false;
    int la = P.level[a], lb = P.level[b], L = std::max(la, lb);
    for (int k = 0; k < 3; ++k) {
        int64_t a0 = (int64_t)P.idx[3 * a + k] << (L - la), a1 = (int64_t)(P.idx[3 * a + k] + 1) << (L - la);
        int64_t b0 = (int64_t)P.idx[3 * b + k] << (L - lb), b1 = (int64_t)(P.idx[3 * b + k] + 1) << (L - lb);
        if (std::max(a0, b0) > std::min(a1, b1)) return false;
    }
    return true;
}

}  // namespace

double leaf_coordinate(double x, double a, double w, int level, uint32_t index) {
    double scale = std::ldexp(1.0, level + 1);
    double d = x - a;
    return d * scale / w - (double)(2 * (uint64_t)index + 1);
}

int offset_index(int x, int y, int z) {
    auto adj = [](int t) { return -1 <= t && t <= 1; };
    auto kappa = [](int t) { return std::min(std::max(t + 1, 0), 3); };
    if (x < -3 || x > 3 || y < -3 || y > 3 || z < -3 || z > 3) return -1;
    if (adj(x) && adj(y) && adj(z)) return -1;
    return 49 * (x + 3) + 7 * (y + 3) + (z + 3) - 9 * kappa(x) -
           (adj(x) ? 1 : 0) * (3 * kappa(y) + (adj(y) ? 1 : 0) * kappa(z));
}

size_t stage_threads(size_t n, int limit) {
    if (n < ((size_t)1 << 16)) return 1;
    const size_t cap = limit > 0 ? (size_t)limit : 16;
    return std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), cap));
}

void for_chunks(size_t n, size_t nth, const std::function<void(size_t, size_t, size_t)>& fn) {
    std::vector<std::exception_ptr> failed(nth);
    auto chunk = [&fn, &failed, n, nth](size_t t) {
        try {
            fn(t, n * t / nth, n * (t + 1) / nth);
        } catch (...) {
            failed[t] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    size_t t = 1;
    try {
        for (; t < nth; ++t) pool.emplace_back(chunk, t);
    } catch (...) {
    }
    chunk(0);
    for (; t < nth; ++t) chunk(t);
    for (auto& th : pool) th.join();
    for (const auto& e : failed)
        if (e) std::rethrow_exception(e);
}

Plan build_plan(size_t ns, const double* src, size_t nt, const double* tgt, int max_level,
                int max_keys, bool device_points, int host_threads) {
    if (ns + nt == 0) throw std::runtime_error("no points");
    if (max_keys < 1) throw std::runtime_error("max_points_per_leaf must be at least 1");
    if (max_level > kDeepest) max_level = kDeepest;
    Plan P;
    // ---- domain: octree/src/octree.rs:1278-1370 and fmm-exec/src/geometry.rs:120-147 ----
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k) {
        mn[k] = std::numeric_limits<double>::max();
        mx[k] = std::numeric_limits<double>::lowest();
    }
    // per-chunk bounds on host threads, then combined (min and max are exact in any order)
    for (int s = 0; s < 2; ++s) {
        const size_t n = s ? nt : ns;
        const double* x = s ? tgt : src;
        const size_t nth = stage_threads(n, host_threads);
        std::vector<double> lo(3 * nth, std::numeric_limits<double>::max()),
            hi(3 * nth, std::numeric_limits<double>::lowest());
        for_chunks(n, nth, [&](size_t t, size_t i0, size_t i1) {
            double l[3], h[3];  // this chunk's bounds, stored once at its end
            for (int k = 0; k < 3; ++k) {
                l[k] = std::numeric_limits<double>::max();
                h[k] = std::numeric_limits<double>::lowest();
            }
            for (size_t i = i0; i < i1; ++i)
                for (int k = 0; k < 3; ++k) {
                    double v = x[3 * i + k];
                    if (!std::isfinite(v)) throw std::runtime_error("non-finite point coordinate");
                    l[k] = std::fmin(l[k], v);
                    h[k] = std::fmax(h[k], v);
                }
            for (int k = 0; k < 3; ++k) {
                lo[3 * t + k] = l[k];
                hi[3 * t + k] = h[k];
            }
        });
        for (size_t t = 0; t < nth; ++t)
            for (int k = 0; k < 3; ++k) {
                mn[k] = std::fmin(mn[k], lo[3 * t + k]);
                mx[k] = std::fmax(mx[k], hi[3 * t + k]);
            }
    }
    double diam[3], mean[3];
    for (int k = 0; k < 3; ++k) {
        diam[k] = mx[k] - mn[k];
        mean[k] = mn[k] + 0.5 * diam[k];
    }
    double md = std::fmax(std::fmax(diam[0], diam[1]), diam[2]);
    if (!(md > 0.0) || !std::isfinite(md)) throw std::runtime_error("points span no volume");
    md = md * (1.0 + 1.0 / (double)(1 << kDeepest));
    double sides[3];
    for (int k = 0; k < 3; ++k) {
        P.box6[k] = mean[k] - 0.5 * md;
        P.box6[k + 3] = mean[k] + 0.5 * md;
        P.lower[k] = P.box6[k];
        sides[k] = P.box6[k + 3] - P.box6[k];
    }
    P.side = std::fmax(std::fmax(sides[0], sides[1]), sides[2]);

    // ---- level-16 keys (morton.rs:255-272) ----
    const uint32_t size16 = 1u << kDeepest;
    auto point_key = [&](const double* x) {
        uint32_t id[3];
        for (int k = 0; k < 3; ++k) {
            double ref = (x[k] - P.box6[k]) / (P.box6[k + 3] - P.box6[k]);
            double s = ref * (double)size16;
            uint64_t i = s <= 0.0 ? 0 : (uint64_t)s;
            id[k] = (uint32_t)std::min<uint64_t>(i, size16 - 1);
        }
        return encode(id[0], id[1], id[2], kDeepest);
    };
    // the point stages (keys, their distinct sorted set, later each point's leaf and the
    // order by leaf) on the device when asked (plan_gpu.cu: the same keys and order), else here
    std::unique_ptr<PointSort> dev = device_points ? device_point_sort(ns, src, nt, tgt, P.box6) : nullptr;
    const bool same_points = src == tgt && ns == nt;  // one point set: the targets' stages are the sources'
    std::vector<uint64_t> skey, tkey, fine;
    // on one host thread the keys are radix-sorted with their point numbers (sources, then
    // targets after ns) once: that gives the distinct keys here and each point's leaf below
    // by one sweep against the leaves' first keys (the leaf a binary search would find)
    const bool sweep = !dev && stage_threads(ns + nt, host_threads) == 1 && ns + nt < ((size_t)1 << 32);
    std::vector<uint32_t> sorted_id;
    if (dev) {
        fine = dev->distinct_keys();
    } else {
        skey.resize(ns);
        for_chunks(ns, stage_threads(ns, host_threads), [&](size_t, size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) skey[i] = point_key(src + 3 * i);
        });
        if (!same_points) {
            tkey.resize(nt);
            for_chunks(nt, stage_threads(nt, host_threads), [&](size_t, size_t i0, size_t i1) {
                for (size_t i = i0; i < i1; ++i) tkey[i] = point_key(tgt + 3 * i);
            });
        }
        // targets that are the sources add no key of their own
        fine.reserve(ns + (same_points ? 0 : nt));
        fine.insert(fine.end(), skey.begin(), skey.end());
        fine.insert(fine.end(), tkey.begin(), tkey.end());
        if (sweep) {
            sorted_id.resize(fine.size());
            for (size_t i = 0; i < sorted_id.size(); ++i) sorted_id[i] = (uint32_t)i;
            radix_sort_keys(fine, sorted_id);
            fine.erase(std::unique(fine.begin(), fine.end()), fine.end());
        } else {
            sort_unique_threads(fine, stage_threads(fine.size(), host_threads));  // distinct keys (route_keys on one rank)
        }
    }

    std::vector<uint64_t> refined;
    refine(fine.data(), fine.size(), 0ULL, max_level, (size_t)max_keys, refined);
    std::vector<uint64_t> leaves = balance(refined);

    // ---- boxes: leaves and their ancestors, level-major ----
    std::vector<uint64_t> all = leaves;
    for (uint64_t k : leaves)
        while (key_level(k) > 0) {
            k = parent_key(k);
            all.push_back(k);
        }
    sort_unique(all);
    std::stable_sort(all.begin(), all.end(),
                     [](uint64_t a, uint64_t b) { return key_level(a) < key_level(b); });
    const size_t nb = all.size();
    if (nb >= ((size_t)1 << 31)) throw std::runtime_error("too many boxes for 32-bit box indices");
    P.key = all;
    P.nlevels = key_level(all.back()) + 1;
    P.level.resize(nb);
    P.idx.resize(3 * nb);
    P.level_start.assign(P.nlevels + 1, 0);
    KeyMap km;
    km.map.reserve(nb * 2);
    for (size_t b = 0; b < nb; ++b) {
        P.level[b] = key_level(all[b]);
        decode(all[b], &P.idx[3 * b]);
        P.level_start[P.level[b] + 1] = (int64_t)b + 1;
        km.map.emplace(all[b], (int32_t)b);
    }
    for (int l = 1; l <= P.nlevels; ++l) P.level_start[l] = std::max(P.level_start[l], P.level_start[l - 1]);
    P.parent.assign(nb, -1);
    P.child_first.assign(nb, -1);
    P.box_leaf.assign(nb, -1);
    std::vector<uint8_t> is_leaf(nb, 0);
    for (uint64_t k : leaves) is_leaf[km.find(k)] = 1;
    for (size_t b = 0; b < nb; ++b) {
        if (P.level[b] > 0) P.parent[b] = km.find(parent_key(all[b]));
        if (!is_leaf[b]) {
            int32_t c0 = km.find(child_key(all[b], 0));
            if (c0 < 0) throw std::runtime_error("incomplete tree");
            P.child_first[b] = c0;
        }
    }
    // leaves level-major
    P.leaf_level_start.assign(P.nlevels + 1, 0);
    for (size_t b = 0; b < nb; ++b)
        if (is_leaf[b]) {
            P.box_leaf[b] = (int32_t)P.leaf_box.size();
            P.leaf_box.push_back((int32_t)b);
            P.leaf_level_start[P.level[b] + 1] = (int64_t)P.leaf_box.size();
        }
    for (int l = 1; l <= P.nlevels; ++l)
        P.leaf_level_start[l] = std::max(P.leaf_level_start[l], P.leaf_level_start[l - 1]);
    const size_t nl = P.leaf_box.size();

    // ---- points -> leaves: the leaf (Morton order partitions the key space) ----
    std::vector<uint64_t> morton_leaves = leaves;  // sorted by key value
    std::vector<int32_t> morton_leaf_index(morton_leaves.size());
    for (size_t i = 0; i < morton_leaves.size(); ++i)
        morton_leaf_index[i] = P.box_leaf[km.find(morton_leaves[i])];
    std::vector<uint64_t> firsts(morton_leaves.size());
    for (size_t i = 0; i < morton_leaves.size(); ++i) firsts[i] = first_fine(morton_leaves[i]);
    auto leaf_of = [&](uint64_t fk) {
        size_t pos = (size_t)(std::upper_bound(firsts.begin(), firsts.end(), fk) - firsts.begin()) - 1;
        return morton_leaf_index[pos];
    };
    if (dev) dev->leaf_order(firsts, morton_leaf_index, nl, P);
    std::vector<int32_t> swept;  // each point's leaf, sources then targets
    if (sweep) {
        swept.resize(sorted_id.size());
        size_t at = 0;
        for (uint32_t id : sorted_id) {
            const uint64_t k = id < ns ? skey[id] : tkey[id - ns];
            while (at + 1 < firsts.size() && firsts[at + 1] <= k) ++at;
            swept[id] = morton_leaf_index[at];
        }
    }
    for (int s = 0; s < (dev ? 0 : same_points ? 1 : 2); ++s) {
        const std::vector<uint64_t>& keys = s ? tkey : skey;
        size_t n = keys.size();
        const size_t nth = stage_threads(n, host_threads);
        std::vector<int32_t> lf(n);
        // each chunk counts its points per leaf; a chunk's points of leaf j then go after
        // those of the chunks before it (a stable counting sort: the order of the points'
        // indices within a leaf, for every thread count)
        std::vector<std::vector<int64_t>> next(nth, std::vector<int64_t>(nl, 0));
        for_chunks(n, nth, [&](size_t t, size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) {
                lf[i] = sweep ? swept[(s ? ns : 0) + i] : leaf_of(keys[i]);
                next[t][lf[i]]++;
            }
        });
        std::vector<int64_t> start(nl + 1, 0);
        int64_t run = 0;
        for (size_t j = 0; j < nl; ++j) {
            start[j] = run;
            for (size_t t = 0; t < nth; ++t) {
                const int64_t c = next[t][j];
                next[t][j] = run;
                run += c;
            }
        }
        start[nl] = run;
        std::vector<int64_t> perm(n), pos_of(n);
        for_chunks(n, nth, [&](size_t t, size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) {
                const int64_t pos = next[t][lf[i]]++;
                perm[pos] = (int64_t)i;
                pos_of[i] = pos;
            }
        });
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
    if (!dev && same_points) {
        P.tgt_start = P.src_start;
        P.tgt_perm = P.src_perm;
        P.tgt_pos_of = P.src_pos_of;
    }
    // counts below every box (children come after parents, level-major)
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

    // ---- lists (interaction_manager.rs:15-27) ----
    auto same_level = [&](int32_t b, int dx, int dy, int dz) -> int32_t {
        int l = P.level[b];
        int64_t size = (int64_t)1 << l;
        int64_t a = (int64_t)P.idx[3 * b] + dx, c = (int64_t)P.idx[3 * b + 1] + dy,
                e = (int64_t)P.idx[3 * b + 2] + dz;
        if (a < 0 || c < 0 || e < 0 || a >= size || c >= size || e >= size) return -2;
        return km.find(encode((uint32_t)a, (uint32_t)c, (uint32_t)e, l));
    };
    // the rows of two lists at once, in parallel over chunks of rows (each row depends on
    // the tree only); the chunks' rows are joined in row order, so the lists are the
    // same whatever the number of threads
    struct Rows {
        std::vector<int32_t> a, aux, b;
        std::vector<int64_t> arow, brow;  // row ends within the chunk
    };
    auto two_lists = [host_threads](size_t nrows, Csr& A, Csr& B, bool with_aux, auto&& row_fn) {
        const size_t cap = host_threads > 0 ? (size_t)host_threads : 16;
        const size_t nth = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), cap));
        const size_t nch = std::min(nrows, nth * 4) ? std::min(nrows, nth * 4) : 1;
        std::vector<Rows> parts(nch);
        std::vector<std::string> errors(nch);
        std::atomic<size_t> next{0};
        auto work = [&] {
            for (size_t c; (c = next.fetch_add(1)) < nch;) {
                try {
                    for (size_t r = nrows * c / nch; r < nrows * (c + 1) / nch; ++r) row_fn(r, parts[c]);
                } catch (const std::exception& e) {
                    errors[c] = e.what();
                }
            }
        };
        std::vector<std::thread> pool;
        for (size_t i = 1; i < nth; ++i) pool.emplace_back(work);
        work();
        for (auto& th : pool) th.join();
        for (const auto& e : errors)
            if (!e.empty()) throw std::runtime_error(e);
        A.row.assign(nrows + 1, 0);
        B.row.assign(nrows + 1, 0);
        A.col.clear();
        B.col.clear();
        A.aux.clear();
        size_t r = 0;
        for (const Rows& pr : parts) {
            const int64_t a0 = (int64_t)A.col.size(), b0 = (int64_t)B.col.size();
            A.col.insert(A.col.end(), pr.a.begin(), pr.a.end());
            if (with_aux) A.aux.insert(A.aux.end(), pr.aux.begin(), pr.aux.end());
            B.col.insert(B.col.end(), pr.b.begin(), pr.b.end());
            for (size_t i = 0; i < pr.arow.size(); ++i, ++r) {
                A.row[r + 1] = a0 + pr.arow[i];
                B.row[r + 1] = b0 + pr.brow[i];
            }
        }
    };
    // near and W, per leaf
    two_lists(nl, P.near, P.w, false, [&](size_t j, Rows& out) {
        int32_t b = P.leaf_box[j];
        std::vector<int32_t> nearj, wj;
        if (P.tgt_below[b] > 0) {
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        if (!dx && !dy && !dz) continue;
                        int32_t N = same_level(b, dx, dy, dz);
                        if (N == -2) continue;
                        if (N >= 0 && P.child_first[N] >= 0) {
                            for (int o = 0; o < 8; ++o) {
                                int32_t c = P.child_first[N] + o;
                                if (P.src_below[c] == 0) continue;
                                if (adjacent(P, c, b)) {
                                    if (P.box_leaf[c] < 0) throw std::runtime_error("tree not 2:1 balanced");
                                    nearj.push_back(P.box_leaf[c]);
                                } else {
                                    wj.push_back(c);
                                }
                            }
                        } else if (N >= 0) {
                            if (P.src_below[N] > 0) nearj.push_back(P.box_leaf[N]);
                        } else {
                            // the neighbour cell is no box: the leaf on the level above holds it
                            int64_t a = ((int64_t)P.idx[3 * b] + dx) >> 1, c = ((int64_t)P.idx[3 * b + 1] + dy) >> 1,
                                    e = ((int64_t)P.idx[3 * b + 2] + dz) >> 1;
                            int32_t C = km.find(encode((uint32_t)a, (uint32_t)c, (uint32_t)e, P.level[b] - 1));
                            if (C < 0 || P.box_leaf[C] < 0) throw std::runtime_error("tree not 2:1 balanced");
                            if (P.src_below[C] > 0) nearj.push_back(P.box_leaf[C]);
                        }
                    }
            if (P.src_below[b] > 0) nearj.push_back((int32_t)j);
            std::sort(nearj.begin(), nearj.end());
            nearj.erase(std::unique(nearj.begin(), nearj.end()), nearj.end());
            std::sort(wj.begin(), wj.end());
        }
        out.a.insert(out.a.end(), nearj.begin(), nearj.end());
        out.arow.push_back((int64_t)out.a.size());
        out.b.insert(out.b.end(), wj.begin(), wj.end());
        out.brow.push_back((int64_t)out.b.size());
        });
    // V and X, per box
    two_lists(nb, P.v, P.x, true, [&](size_t bb, Rows& out) {
        int32_t b = (int32_t)bb;
        std::vector<std::pair<int32_t, int32_t>> vtmp;
        std::vector<int32_t> tmp;
        if (P.level[b] >= 1 && P.tgt_below[b] > 0) {
            int32_t par = P.parent[b];
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        if (!dx && !dy && !dz) continue;
                        int32_t C = same_level(par, dx, dy, dz);
                        if (C < 0) continue;
                        if (P.child_first[C] >= 0) {
                            for (int o = 0; o < 8; ++o) {
                                int32_t s = P.child_first[C] + o;
                                if (P.src_below[s] == 0 || adjacent(P, s, b)) continue;
                                int d = offset_index((int)P.idx[3 * b] - (int)P.idx[3 * s],
                                                     (int)P.idx[3 * b + 1] - (int)P.idx[3 * s + 1],
                                                     (int)P.idx[3 * b + 2] - (int)P.idx[3 * s + 2]);
                                if (d < 0) throw std::runtime_error("V pair outside the 316 offsets");
                                vtmp.emplace_back(d, s);
                            }
                        } else if (P.src_below[C] > 0 && !adjacent(P, C, b)) {
                            tmp.push_back(P.box_leaf[C]);
                        }
                    }
            std::sort(vtmp.begin(), vtmp.end());
            std::sort(tmp.begin(), tmp.end());
        }
        for (auto& e : vtmp) {
            out.a.push_back(e.second);
            out.aux.push_back(e.first);
        }
        out.arow.push_back((int64_t)out.a.size());
        out.b.insert(out.b.end(), tmp.begin(), tmp.end());
        out.brow.push_back((int64_t)out.b.size());
        });
    return P;
}

uint64_t morton_encode(uint32_t i, uint32_t j, uint32_t k, int level) { return encode(i, j, k, level); }
void morton_decode(uint64_t key, uint32_t out[3]) { decode(key, out); }
int morton_level(uint64_t key) { return key_level(key); }

}  // namespace fmmb
