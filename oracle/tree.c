/*
 * Oracle (test infrastructure only): Morton keys, the cubic domain, the single-rank
 * octree (refinement + 2:1 balance) and the U/V/W/X interaction lists, restated from
 *   octree/src/morton.rs (key layout: 3 interleaved index bits per level, x highest,
 *     shifted left by 15, level in the low 15 bits; from_physical_point :255),
 *   octree/src/octree.rs:1278-1370 (compute_global_bounding_box),
 *   octree/src/octree/implementation.rs:682-730 (create_local_tree) and :1014-1103
 *     (balance / balance_closure), morton.rs:795 (linearize),
 *   fmm-plan/src/interaction_manager.rs:1-40 (the list rule).
 * Simple and serial by design: it is the checker of the product's tree and lists.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fmm_oracle.h"

#define DEEPEST 16
#define LEVEL_MASK 0x7FFFULL

static uint64_t spread3(uint64_t v) { /* bit b of v -> bit 3b */
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> b) & 1ULL) << (3 * b);
    return r;
}

uint64_t orc_key_from_index(const uint32_t idx[3], int level) {
    int d = DEEPEST - level;
    uint64_t x = (uint64_t)idx[0] << d, y = (uint64_t)idx[1] << d, z = (uint64_t)idx[2] << d;
    uint64_t k = (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    return (k << 15) | (uint64_t)level;
}

void orc_key_decode(uint64_t key, int *level, uint32_t idx[3]) {
    int l = (int)(key & LEVEL_MASK);
    uint64_t k = key >> 15;
    uint32_t v[3] = {0, 0, 0};
    for (int b = 0; b < 16; ++b) {
        v[0] |= (uint32_t)((k >> (3 * b + 2)) & 1ULL) << b;
        v[1] |= (uint32_t)((k >> (3 * b + 1)) & 1ULL) << b;
        v[2] |= (uint32_t)((k >> (3 * b)) & 1ULL) << b;
    }
    for (int a = 0; a < 3; ++a) idx[a] = v[a] >> (DEEPEST - l);
    *level = l;
}

static int key_level(uint64_t k) { return (int)(k & LEVEL_MASK); }

static uint64_t key_parent(uint64_t k) {
    int l;
    uint32_t i[3];
    orc_key_decode(k, &l, i);
    uint32_t pi[3] = {i[0] >> 1, i[1] >> 1, i[2] >> 1};
    return orc_key_from_index(pi, l - 1);
}

static void key_children(uint64_t k, uint64_t c[8]) {
    int l;
    uint32_t i[3];
    orc_key_decode(k, &l, i);
    for (int o = 0; o < 8; ++o) {
        uint32_t ci[3] = {2 * i[0] + ((o >> 2) & 1), 2 * i[1] + ((o >> 1) & 1), 2 * i[2] + (o & 1)};
        c[o] = orc_key_from_index(ci, l + 1);
    }
}

/* morton.rs is_ancestor: a is a strict ancestor of b */
static int is_ancestor(uint64_t a, uint64_t b) {
    int la = key_level(a), lb = key_level(b);
    if (la >= lb) return 0;
    uint64_t mask = ~0ULL << (15 + 3 * (DEEPEST - la));
    return ((a ^ b) & mask) == 0;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

/* ---- domain (octree.rs:1278-1370) ---- */
void orc_domain(size_t ns, const double *src, size_t nt, const double *tgt, double lower[3],
                double *side, double box6[6]) {
    double mn[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    double mx[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    for (int s = 0; s < 2; ++s) {
        size_t n = s ? nt : ns;
        const double *x = s ? tgt : src;
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                mn[k] = fmin(mn[k], x[3 * i + k]);
                mx[k] = fmax(mx[k], x[3 * i + k]);
            }
    }
    double diam[3], mean[3];
    for (int k = 0; k < 3; ++k) {
        diam[k] = mx[k] - mn[k];
        mean[k] = mn[k] + 0.5 * diam[k];
    }
    double deepest_box = 1.0 / (double)(1 << DEEPEST);
    double md = fmax(fmax(diam[0], diam[1]), diam[2]);
    md = md * (1.0 + deepest_box);
    for (int k = 0; k < 3; ++k) {
        box6[k] = mean[k] - 0.5 * md;
        box6[k + 3] = mean[k] + 0.5 * md;
    }
    /* fmm-exec/src/geometry.rs:120-147 Domain::new */
    double sides[3];
    for (int k = 0; k < 3; ++k) {
        lower[k] = box6[k];
        sides[k] = box6[k + 3] - box6[k];
    }
    *side = fmax(fmax(sides[0], sides[1]), sides[2]);
}

/* morton.rs:255-272 from_physical_point with geometry.rs:73 physical_to_reference */
uint64_t orc_point_key(const double x[3], const double box6[6], int level) {
    uint32_t size = 1u << level, idx[3];
    for (int k = 0; k < 3; ++k) {
        double ref = (x[k] - box6[k]) / (box6[k + 3] - box6[k]);
        double s = ref * (double)size;
        uint64_t i = s <= 0.0 ? 0 : (uint64_t)s; /* Rust `as usize` saturates at 0 */
        if (i > size - 1) i = size - 1;
        idx[k] = (uint32_t)i;
    }
    return orc_key_from_index(idx, level);
}

/* ---- refinement (implementation.rs:682-730) ---- */
typedef struct { uint64_t *data; size_t len, cap; } vec64;

static void vpush(vec64 *v, uint64_t x) {
    if (v->len == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 64;
        v->data = (uint64_t *)realloc(v->data, v->cap * sizeof(uint64_t));
    }
    v->data[v->len++] = x;
}

/* first and one-past-last level-16 key under `box` */
static uint64_t first_fine(uint64_t box) { return (box & ~LEVEL_MASK) | DEEPEST; }

static void refine(const uint64_t *fine, size_t nfine, uint64_t box, int max_level, size_t max_keys,
                   vec64 *out) {
    int level = key_level(box);
    if (level < max_level && nfine > max_keys) {
        uint64_t ch[8];
        key_children(box, ch);
        size_t start = 0;
        for (int o = 0; o < 8; ++o) {
            /* keys under child o are contiguous; find the end by the next child's first key */
            size_t end = start;
            uint64_t limit = o < 7 ? first_fine(ch[o + 1]) : ~0ULL;
            while (end < nfine && (o == 7 || fine[end] < limit)) ++end;
            refine(fine + start, end - start, ch[o], max_level, max_keys, out);
            start = end;
        }
    } else {
        vpush(out, box);
    }
}

/* ---- balance (implementation.rs:1069-1103) and linearize (morton.rs:795-811) ---- */
static int contains_u64(const uint64_t *a, size_t n, uint64_t x) {
    return bsearch(&x, a, n, sizeof(uint64_t), cmp_u64) != NULL;
}

static void neighbours(uint64_t key, uint64_t out[26], int *count) {
    int l;
    uint32_t i[3];
    orc_key_decode(key, &l, i);
    *count = 0;
    if (l == 0) return;
    long size = 1L << l;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                long n[3] = {(long)i[0] + dx, (long)i[1] + dy, (long)i[2] + dz};
                if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= size || n[1] >= size || n[2] >= size)
                    continue;
                uint32_t ni[3] = {(uint32_t)n[0], (uint32_t)n[1], (uint32_t)n[2]};
                out[(*count)++] = orc_key_from_index(ni, l);
            }
}

static vec64 linearize(uint64_t *keys, size_t n) {
    vec64 out = {0, 0, 0};
    if (!n) return out;
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    for (size_t i = 0; i + 1 < n; ++i) {
        if (keys[i] == keys[i + 1] || is_ancestor(keys[i], keys[i + 1])) continue;
        vpush(&out, keys[i]);
    }
    vpush(&out, keys[n - 1]);
    return out;
}

static vec64 balance(const uint64_t *leaves, size_t n) {
    int deepest = 0;
    for (size_t i = 0; i < n; ++i)
        if (key_level(leaves[i]) > deepest) deepest = key_level(leaves[i]);
    vec64 result = {0, 0, 0};
    if (deepest == 0) {
        for (size_t i = 0; i < n; ++i) vpush(&result, leaves[i]);
        return result;
    }
    vec64 work = {0, 0, 0};
    for (size_t i = 0; i < n; ++i)
        if (key_level(leaves[i]) == deepest) vpush(&work, leaves[i]);
    for (int level = deepest; level >= 1; --level) {
        /* the distinct parents of the work list (a set in the reference; the order of
         * `result` is irrelevant because it is linearised, and `next` is a set too) */
        uint64_t *par = (uint64_t *)malloc((work.len ? work.len : 1) * sizeof(uint64_t));
        for (size_t w = 0; w < work.len; ++w) par[w] = key_parent(work.data[w]);
        qsort(par, work.len, sizeof(uint64_t), cmp_u64);
        size_t np = 0;
        for (size_t w = 0; w < work.len; ++w)
            if (np == 0 || par[np - 1] != par[w]) par[np++] = par[w];
        vec64 next = {0, 0, 0};
        for (size_t j = 0; j < np; ++j) {
            uint64_t ch[8];
            key_children(par[j], ch);
            for (int o = 0; o < 8; ++o) vpush(&result, ch[o]);
            uint64_t nb[26];
            int c;
            neighbours(par[j], nb, &c);
            for (int a = 0; a < c; ++a) vpush(&next, nb[a]);
        }
        free(par);
        for (size_t i = 0; i < n; ++i)
            if (key_level(leaves[i]) == level - 1) vpush(&next, leaves[i]);
        free(work.data);
        work = next;
    }
    free(work.data);
    vec64 lin = linearize(result.data, result.len);
    free(result.data);
    return lin;
}

/* ---- the tree object ---- */
struct orc_tree {
    int nlevels;
    double box6[6], lower[3], side;
    uint64_t *keys; /* all boxes, sorted by key value */
    uint8_t *leaf;
    size_t nboxes, nleaves;
};

orc_tree *orc_tree_build(size_t ns, const double *src, size_t nt, const double *tgt, int max_level,
                         int max_keys) {
    orc_tree *t = (orc_tree *)calloc(1, sizeof(orc_tree));
    orc_domain(ns, src, nt, tgt, t->lower, &t->side, t->box6);
    size_t n = ns + nt;
    uint64_t *fine = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    for (size_t i = 0; i < ns; ++i) fine[i] = orc_point_key(src + 3 * i, t->box6, DEEPEST);
    for (size_t i = 0; i < nt; ++i) fine[ns + i] = orc_point_key(tgt + 3 * i, t->box6, DEEPEST);
    qsort(fine, n, sizeof(uint64_t), cmp_u64);
    size_t nd = 0; /* distinct keys (route_keys on one rank, implementation.rs:83-125) */
    for (size_t i = 0; i < n; ++i)
        if (nd == 0 || fine[nd - 1] != fine[i]) fine[nd++] = fine[i];
    vec64 refined = {0, 0, 0};
    refine(fine, nd, 0ULL, max_level > DEEPEST ? DEEPEST : max_level, (size_t)max_keys, &refined);
    free(fine);
    vec64 leaves = balance(refined.data, refined.len);
    free(refined.data);
    /* all boxes: leaves and every ancestor */
    vec64 all = {0, 0, 0};
    for (size_t i = 0; i < leaves.len; ++i) {
        uint64_t k = leaves.data[i];
        vpush(&all, k);
        while (key_level(k) > 0) {
            k = key_parent(k);
            vpush(&all, k);
        }
    }
    qsort(all.data, all.len, sizeof(uint64_t), cmp_u64);
    size_t nb = 0;
    for (size_t i = 0; i < all.len; ++i)
        if (nb == 0 || all.data[nb - 1] != all.data[i]) all.data[nb++] = all.data[i];
    t->keys = all.data;
    t->nboxes = nb;
    t->leaf = (uint8_t *)calloc(nb, 1);
    t->nlevels = 1;
    for (size_t i = 0; i < leaves.len; ++i) {
        uint64_t *p = (uint64_t *)bsearch(&leaves.data[i], t->keys, nb, sizeof(uint64_t), cmp_u64);
        t->leaf[p - t->keys] = 1;
        if (key_level(leaves.data[i]) + 1 > t->nlevels) t->nlevels = key_level(leaves.data[i]) + 1;
    }
    t->nleaves = leaves.len;
    free(leaves.data);
    return t;
}

void orc_tree_free(orc_tree *t) {
    if (!t) return;
    free(t->keys);
    free(t->leaf);
    free(t);
}

int orc_tree_nlevels(const orc_tree *t) { return t->nlevels; }
size_t orc_tree_nboxes(const orc_tree *t) { return t->nboxes; }
size_t orc_tree_nleaves(const orc_tree *t) { return t->nleaves; }
void orc_tree_domain(const orc_tree *t, double lower[3], double *side) {
    memcpy(lower, t->lower, sizeof(t->lower));
    *side = t->side;
}

/* boxes level-major, key order within a level */
void orc_tree_boxes(const orc_tree *t, uint64_t *keys, uint8_t *is_leaf) {
    size_t o = 0;
    for (int l = 0; l < t->nlevels; ++l)
        for (size_t i = 0; i < t->nboxes; ++i)
            if (key_level(t->keys[i]) == l) {
                keys[o] = t->keys[i];
                if (is_leaf) is_leaf[o] = t->leaf[i];
                ++o;
            }
}

static long find_box(const orc_tree *t, uint64_t k) {
    uint64_t *p = (uint64_t *)bsearch(&k, t->keys, t->nboxes, sizeof(uint64_t), cmp_u64);
    return p ? (long)(p - t->keys) : -1;
}

/* closed cubes intersect and neither is an ancestor of the other (interaction_manager.rs:10-13) */
static int adjacent(uint64_t a, uint64_t b) {
    if (a == b || is_ancestor(a, b) || is_ancestor(b, a)) return 0;
    int la, lb;
    uint32_t ia[3], ib[3];
    orc_key_decode(a, &la, ia);
    orc_key_decode(b, &lb, ib);
    int L = la > lb ? la : lb;
    for (int k = 0; k < 3; ++k) {
        long a0 = (long)ia[k] << (L - la), a1 = (long)(ia[k] + 1) << (L - la);
        long b0 = (long)ib[k] << (L - lb), b1 = (long)(ib[k] + 1) << (L - lb);
        long lo = a0 > b0 ? a0 : b0, hi = a1 < b1 ? a1 : b1;
        if (lo > hi) return 0;
    }
    return 1;
}

static void add_unique(vec64 *v, uint64_t k) {
    for (size_t i = 0; i < v->len; ++i)
        if (v->data[i] == k) return;
    vpush(v, k);
}

/* The list rule (interaction_manager.rs:15-27), stated as a search over the tree. */
size_t orc_tree_list(const orc_tree *t, size_t box_level_major, int kind, uint64_t *out,
                     size_t cap) {
    /* map level-major position to the key */
    uint64_t *lm = (uint64_t *)malloc(t->nboxes * sizeof(uint64_t));
    orc_tree_boxes(t, lm, NULL);
    uint64_t b = lm[box_level_major];
    free(lm);
    long bi = find_box(t, b);
    int is_leaf = t->leaf[bi];
    int lb = key_level(b);
    vec64 res = {0, 0, 0};
    if (kind == 0 && is_leaf) { /* U: all leaves adjacent to B */
        for (size_t i = 0; i < t->nboxes; ++i)
            if (t->leaf[i] && adjacent(b, t->keys[i])) vpush(&res, t->keys[i]);
    } else if (kind == 1 && lb > 0) { /* V: level of B, parent adjacent to P, not adjacent to B */
        uint64_t P = key_parent(b);
        for (size_t i = 0; i < t->nboxes; ++i) {
            uint64_t c = t->keys[i];
            if (key_level(c) != lb || c == b) continue;
            if (adjacent(key_parent(c), P) && !adjacent(c, b)) vpush(&res, c);
        }
    } else if (kind == 2 && is_leaf) { /* W: finer than B, parent adjacent to B, not adjacent */
        for (size_t i = 0; i < t->nboxes; ++i) {
            uint64_t c = t->keys[i];
            if (key_level(c) <= lb) continue;
            if (adjacent(key_parent(c), b) && !adjacent(c, b)) vpush(&res, c);
        }
    } else if (kind == 3 && lb > 0) { /* X: leaves at level of P, adjacent to P, not adjacent to B */
        uint64_t P = key_parent(b);
        for (size_t i = 0; i < t->nboxes; ++i) {
            uint64_t c = t->keys[i];
            if (!t->leaf[i] || key_level(c) != lb - 1) continue;
            if (adjacent(c, P) && !adjacent(c, b)) vpush(&res, c);
        }
    }
    (void)add_unique;
    qsort(res.data, res.len, sizeof(uint64_t), cmp_u64);
    size_t n = res.len;
    for (size_t i = 0; i < n && i < cap; ++i) out[i] = res.data[i];
    free(res.data);
    return n;
}

double orc_leaf_coordinate(double x, double lower, double side, int level, uint32_t index) {
    double scale = ldexp(1.0, level + 1);
    double d = x - lower;
    return d * scale / side - (double)(2 * index + 1);
}
