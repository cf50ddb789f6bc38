/*
 * Oracle (test infrastructure only): the reference's host FMM on one rank, restated:
 *   - build: fmm-exec/src/fmm.rs:17-93 steps 3-8 (domain, keys of sources ++ targets,
 *     octree, points in leaf order = caller order within a leaf, leaf-scaled
 *     coordinates per fmm-exec/src/geometry.rs:291-298);
 *   - lists: fmm-plan/src/interaction_manager.rs:15-27, found by neighbour lookups
 *     (the brute-force search of tree.c checks them in the tests);
 *   - evaluation order: fmm-plan/src/evaluator.rs:368-527 (upward L..0: p2m then m2m;
 *     downward 1..L: l2l, m2l by offset index, p2l by source leaf; leaves 0..L: l2p,
 *     m2p by box index, p2p by source leaf), accumulation rule operator.rs:34-45;
 *   - operators: fmm-ref leaf/direct/p2p restated in operators.c, M2M/L2L/M2L by
 *     tables applied as fmm-tables/src/matrix_set.rs:128;
 *   - frames: CONVENTIONS 3.13 "Relative frames" (integer centres, exact dyadics);
 *   - output: fmm-exec/src/fmm.rs:4750-4778 (phi / (4 pi r), g / ((4 pi r) r)).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fmm_oracle.h"

#define DEEPEST 16

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

typedef struct {
    int nlevels;
    size_t nboxes;
    uint64_t *key;      /* level-major key order */
    int *level;
    uint32_t (*idx)[3];
    uint8_t *leaf;
    size_t *level_start; /* nlevels + 1 */
    uint64_t *sorted;    /* keys sorted by value, with their box index */
    size_t *sorted_box;
} boxes_t;

static long find(const boxes_t *b, uint64_t k) {
    uint64_t *p = (uint64_t *)bsearch(&k, b->sorted, b->nboxes, sizeof(uint64_t), cmp_u64);
    return p ? (long)b->sorted_box[p - b->sorted] : -1;
}

static int is_anc(uint64_t a, uint64_t b) {
    int la = (int)(a & 0x7FFF), lb = (int)(b & 0x7FFF);
    if (la >= lb) return 0;
    uint64_t mask = ~0ULL << (15 + 3 * (DEEPEST - la));
    return ((a ^ b) & mask) == 0;
}

static int adjacent_boxes(const boxes_t *B, size_t a, size_t b) {
    if (a == b || is_anc(B->key[a], B->key[b]) || is_anc(B->key[b], B->key[a])) return 0;
    int la = B->level[a], lb = B->level[b], L = la > lb ? la : lb;
    for (int k = 0; k < 3; ++k) {
        long a0 = (long)B->idx[a][k] << (L - la), a1 = (long)(B->idx[a][k] + 1) << (L - la);
        long b0 = (long)B->idx[b][k] << (L - lb), b1 = (long)(B->idx[b][k] + 1) << (L - lb);
        if ((a0 > b0 ? a0 : b0) > (a1 < b1 ? a1 : b1)) return 0;
    }
    return 1;
}

static long neighbour(const boxes_t *B, size_t b, int dx, int dy, int dz) {
    int l = B->level[b];
    long size = 1L << l;
    long n[3] = {(long)B->idx[b][0] + dx, (long)B->idx[b][1] + dy, (long)B->idx[b][2] + dz};
    for (int k = 0; k < 3; ++k)
        if (n[k] < 0 || n[k] >= size) return -2; /* outside the domain */
    uint32_t ni[3] = {(uint32_t)n[0], (uint32_t)n[1], (uint32_t)n[2]};
    return find(B, orc_key_from_index(ni, l));
}

static long parent_box(const boxes_t *B, size_t b) {
    if (B->level[b] == 0) return -1;
    uint32_t pi[3] = {B->idx[b][0] >> 1, B->idx[b][1] >> 1, B->idx[b][2] >> 1};
    return find(B, orc_key_from_index(pi, B->level[b] - 1));
}

static long child_box(const boxes_t *B, size_t b, int o) {
    uint32_t ci[3] = {2 * B->idx[b][0] + ((o >> 2) & 1), 2 * B->idx[b][1] + ((o >> 1) & 1),
                      2 * B->idx[b][2] + (o & 1)};
    return find(B, orc_key_from_index(ci, B->level[b] + 1));
}

typedef struct { size_t *data; size_t len, cap; } vecz;
static void zpush(vecz *v, size_t x) {
    if (v->len == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 32;
        v->data = (size_t *)realloc(v->data, v->cap * sizeof(size_t));
    }
    v->data[v->len++] = x;
}
static int cmp_z(const void *a, const void *b) {
    size_t x = *(const size_t *)a, y = *(const size_t *)b;
    return x < y ? -1 : x > y;
}
static void sort_unique(vecz *v) {
    qsort(v->data, v->len, sizeof(size_t), cmp_z);
    size_t n = 0;
    for (size_t i = 0; i < v->len; ++i)
        if (n == 0 || v->data[n - 1] != v->data[i]) v->data[n++] = v->data[i];
    v->len = n;
}

/* relative frame of box s seen from box t (CONVENTIONS 3.13 "Relative frames") */
static void rel_frame(const boxes_t *B, size_t s, size_t t, double c[3], double *r) {
    int ls = B->level[s], lt = B->level[t], L = ls > lt ? ls : lt;
    for (int k = 0; k < 3; ++k) {
        long Cs = (2L * B->idx[s][k] + 1) << (L - ls);
        long Ct = (2L * B->idx[t][k] + 1) << (L - lt);
        c[k] = ldexp((double)(Cs - Ct), lt - L);
    }
    *r = ldexp(1.0, lt - ls);
}

static int offset_of(const boxes_t *B, size_t t, size_t s) {
    return orc_offset_index((int64_t)B->idx[t][0] - (int64_t)B->idx[s][0],
                            (int64_t)B->idx[t][1] - (int64_t)B->idx[s][1],
                            (int64_t)B->idx[t][2] - (int64_t)B->idx[s][2]);
}

static int cmp_pair(const void *a, const void *b) {
    const size_t *x = (const size_t *)a, *y = (const size_t *)b;
    return x[0] < y[0] ? -1 : x[0] > y[0] ? 1 : (x[1] < y[1] ? -1 : x[1] > y[1]);
}

/* The plan shared by the Laplace FMM and the Helmholtz near field: the octree (boxes
 * level-major), the leaves, the points in leaf order and their leaf-scaled coordinates. */
typedef struct {
    boxes_t B;
    double lower[3], side;
    size_t nleaves;
    long *leaf_of_box;
    size_t *leaf_box, *s_off, *t_off, *s_perm, *t_perm;
    double *us, *ut;
} plan_t;

static void plan_setup(plan_t *P, size_t ns, const double *src, size_t nt, const double *tgt, int max_keys) {
    memset(P, 0, sizeof(*P));
    boxes_t *Bp = &P->B;
    orc_tree *tree = orc_tree_build(ns, src, nt, tgt, DEEPEST, max_keys);
    Bp->nlevels = orc_tree_nlevels(tree);
    Bp->nboxes = orc_tree_nboxes(tree);
    Bp->key = (uint64_t *)malloc(Bp->nboxes * sizeof(uint64_t));
    Bp->leaf = (uint8_t *)malloc(Bp->nboxes);
    orc_tree_boxes(tree, Bp->key, Bp->leaf);
    orc_tree_domain(tree, P->lower, &P->side);
    double box6[6];
    { double lw[3], sd; orc_domain(ns, src, nt, tgt, lw, &sd, box6); }
    orc_tree_free(tree);
    Bp->level = (int *)malloc(Bp->nboxes * sizeof(int));
    Bp->idx = malloc(Bp->nboxes * sizeof(*Bp->idx));
    Bp->level_start = (size_t *)calloc(Bp->nlevels + 1, sizeof(size_t));
    for (size_t b = 0; b < Bp->nboxes; ++b) {
        orc_key_decode(Bp->key[b], &Bp->level[b], Bp->idx[b]);
        Bp->level_start[Bp->level[b] + 1] = b + 1;
    }
    for (int l = 1; l <= Bp->nlevels; ++l)
        if (Bp->level_start[l] < Bp->level_start[l - 1]) Bp->level_start[l] = Bp->level_start[l - 1];
    Bp->sorted = (uint64_t *)malloc(Bp->nboxes * sizeof(uint64_t));
    Bp->sorted_box = (size_t *)malloc(Bp->nboxes * sizeof(size_t));
    {
        size_t *pr = (size_t *)malloc(2 * Bp->nboxes * sizeof(size_t));
        for (size_t b = 0; b < Bp->nboxes; ++b) { pr[2 * b] = (size_t)Bp->key[b]; pr[2 * b + 1] = b; }
        qsort(pr, Bp->nboxes, 2 * sizeof(size_t), cmp_pair);
        for (size_t i = 0; i < Bp->nboxes; ++i) { Bp->sorted[i] = pr[2 * i]; Bp->sorted_box[i] = pr[2 * i + 1]; }
        free(pr);
    }
    /* leaves in level-major order (the leaf numbering); box -> leaf */
    size_t nleaves = 0;
    long *leaf_of_box = (long *)malloc(Bp->nboxes * sizeof(long));
    for (size_t b = 0; b < Bp->nboxes; ++b) leaf_of_box[b] = Bp->leaf[b] ? (long)nleaves++ : -1;
    size_t *leaf_box = (size_t *)malloc((nleaves + 1) * sizeof(size_t));
    for (size_t b = 0; b < Bp->nboxes; ++b)
        if (Bp->leaf[b]) leaf_box[leaf_of_box[b]] = b;

    /* points -> leaves, caller order within each leaf */
    size_t *s_leaf = (size_t *)malloc((ns + 1) * sizeof(size_t));
    size_t *t_leaf = (size_t *)malloc((nt + 1) * sizeof(size_t));
    for (int s = 0; s < 2; ++s) {
        size_t n = s ? nt : ns;
        const double *x = s ? tgt : src;
        size_t *out = s ? t_leaf : s_leaf;
        for (size_t i = 0; i < n; ++i) {
            uint64_t fine = orc_point_key(x + 3 * i, box6, DEEPEST);
            long found = -1;
            for (int l = Bp->nlevels - 1; l >= 0 && found < 0; --l) {
                int fl;
                uint32_t fi[3];
                orc_key_decode(fine, &fl, fi);
                uint32_t ai[3] = {fi[0] >> (DEEPEST - l), fi[1] >> (DEEPEST - l), fi[2] >> (DEEPEST - l)};
                long b = find(Bp, orc_key_from_index(ai, l));
                if (b >= 0 && Bp->leaf[b]) found = leaf_of_box[b];
            }
            out[i] = (size_t)found;
        }
    }
    size_t *s_off = (size_t *)calloc(nleaves + 1, sizeof(size_t));
    size_t *t_off = (size_t *)calloc(nleaves + 1, sizeof(size_t));
    for (size_t i = 0; i < ns; ++i) s_off[s_leaf[i] + 1]++;
    for (size_t i = 0; i < nt; ++i) t_off[t_leaf[i] + 1]++;
    for (size_t j = 0; j < nleaves; ++j) { s_off[j + 1] += s_off[j]; t_off[j + 1] += t_off[j]; }
    size_t *s_perm = (size_t *)malloc((ns + 1) * sizeof(size_t)); /* leaf-order pos -> caller */
    size_t *t_perm = (size_t *)malloc((nt + 1) * sizeof(size_t));
    {
        size_t *fill = (size_t *)calloc(nleaves + 1, sizeof(size_t));
        for (size_t i = 0; i < ns; ++i) s_perm[s_off[s_leaf[i]] + fill[s_leaf[i]]++] = i;
        memset(fill, 0, (nleaves + 1) * sizeof(size_t));
        for (size_t i = 0; i < nt; ++i) t_perm[t_off[t_leaf[i]] + fill[t_leaf[i]]++] = i;
        free(fill);
    }
    free(s_leaf);
    free(t_leaf);
    /* leaf-scaled coordinates in leaf order */
    double *us = (double *)malloc((3 * ns + 1) * sizeof(double));
    double *ut = (double *)malloc((3 * nt + 1) * sizeof(double));
    for (size_t j = 0; j < nleaves; ++j) {
        size_t b = leaf_box[j];
        for (size_t a = s_off[j]; a < s_off[j + 1]; ++a) {
            size_t i = s_perm[a];
            for (int k = 0; k < 3; ++k)
                us[3 * a + k] = orc_leaf_coordinate(src[3 * i + k], P->lower[k], P->side, Bp->level[b], Bp->idx[b][k]);
        }
        for (size_t a = t_off[j]; a < t_off[j + 1]; ++a) {
            size_t i = t_perm[a];
            for (int k = 0; k < 3; ++k)
                ut[3 * a + k] = orc_leaf_coordinate(tgt[3 * i + k], P->lower[k], P->side, Bp->level[b], Bp->idx[b][k]);
        }
    }
    P->nleaves = nleaves;
    P->leaf_of_box = leaf_of_box;
    P->leaf_box = leaf_box;
    P->s_off = s_off;
    P->t_off = t_off;
    P->s_perm = s_perm;
    P->t_perm = t_perm;
    P->us = us;
    P->ut = ut;
}

static void plan_free(plan_t *P) {
    free(P->B.key); free(P->B.leaf); free(P->B.level); free(P->B.idx); free(P->B.level_start);
    free(P->B.sorted); free(P->B.sorted_box);
    free(P->leaf_of_box); free(P->leaf_box); free(P->s_off); free(P->t_off); free(P->s_perm); free(P->t_perm);
    free(P->us); free(P->ut);
}

/* The W list (boxes, by index) and the near list (leaves: U and the leaf itself, by leaf
 * index) of leaf box b (fmm-plan/src/interaction_manager.rs:15-27). */
static void leaf_lists(const plan_t *P, size_t b, vecz *wl, vecz *near) {
    const boxes_t *Bp = &P->B;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                long N = neighbour(Bp, b, dx, dy, dz);
                if (N == -2) continue;
                if (N >= 0 && !Bp->leaf[N]) {
                    for (int co = 0; co < 8; ++co) {
                        long c = child_box(Bp, (size_t)N, co);
                        if (adjacent_boxes(Bp, (size_t)c, b)) zpush(near, (size_t)P->leaf_of_box[c]);
                        else zpush(wl, (size_t)c);
                    }
                } else if (N >= 0) {
                    zpush(near, (size_t)P->leaf_of_box[N]);
                } else {
                    /* the neighbour cell is not a box: its parent is a coarser leaf */
                    int l1 = Bp->level[b];
                    uint32_t ni[3] = {(uint32_t)((long)Bp->idx[b][0] + dx) >> 1,
                                      (uint32_t)((long)Bp->idx[b][1] + dy) >> 1,
                                      (uint32_t)((long)Bp->idx[b][2] + dz) >> 1};
                    long C = find(Bp, orc_key_from_index(ni, l1 - 1));
                    if (C >= 0 && Bp->leaf[C]) zpush(near, (size_t)P->leaf_of_box[C]);
                }
            }
    zpush(near, (size_t)P->leaf_of_box[b]);
    sort_unique(wl);
    sort_unique(near);
}

/* seconds of the last orc_fmm_kinds without its plan and table builds (the evaluation the
 * reference's benchmark times, fmm-bench/src/measure.rs: build and tables excluded) */
static double g_eval_seconds = 0.0;
double orc_fmm_last_eval_seconds(void) { return g_eval_seconds; }

int orc_fmm(size_t ns, const double *src, const double *q, int m, size_t nt, const double *tgt,
            int p, int max_keys, int gradients, int threads, double *phi_out, double *grad_out) {
    return orc_fmm_kinds(ns, src, q, m, nt, tgt, p, max_keys, gradients, threads, 3, phi_out, grad_out);
}

/* A built oracle FMM: the plan and the f64 tables, kept for repeated evaluations (the
 * reference's Fmm, fmm-exec/src/fmm.rs:1853 build then :3691 evaluate). */
struct orc_fmm_handle {
    plan_t PL;
    int p, m, gradients;
    size_t ns, nt;
    double *m2l_t, *m2m_t, *l2l_t;
    /* the host path (orc_fmm_set_host_path): lists made once, batched M2L, SIMD P2P */
    int host_path;
    size_t *v_row, *v_box, *v_off;     /* V list of every box, by offset index */
    size_t *near_row, *near_leaf;      /* near list of every leaf (itself included) */
    size_t *w_row, *w_box;             /* W list of every leaf */
};

/* the V list of box b: children of its parent's colleagues not adjacent to b, as
 * (offset index, box) sorted by offset index (fmm-plan/src/interaction_manager.rs:15-27) */
static int v_list(const boxes_t *B, size_t b, size_t vl[189][2]) {
    long P = parent_box(B, b);
    int nv = 0;
    if (P < 0) return 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                long C = neighbour(B, (size_t)P, dx, dy, dz);
                if (C < 0 || B->leaf[C]) continue;
                for (int co = 0; co < 8; ++co) {
                    long s = child_box(B, (size_t)C, co);
                    if (adjacent_boxes(B, (size_t)s, b)) continue;
                    vl[nv][0] = (size_t)offset_of(B, b, (size_t)s);
                    vl[nv][1] = (size_t)s;
                    ++nv;
                }
            }
    qsort(vl, nv, sizeof(vl[0]), cmp_pair);
    return nv;
}

orc_fmm_handle *orc_fmm_new(size_t ns, const double *src, size_t nt, const double *tgt, int p, int max_keys,
                            int m, int gradients) {
    orc_fmm_handle *h = (orc_fmm_handle *)calloc(1, sizeof(orc_fmm_handle));
    int nc = (p + 1) * (p + 1);
    plan_setup(&h->PL, ns, src, nt, tgt, max_keys);
    h->p = p;
    h->m = m;
    h->gradients = gradients;
    h->ns = ns;
    h->nt = nt;
    h->m2l_t = (double *)malloc((size_t)316 * nc * nc * sizeof(double));
    h->m2m_t = (double *)malloc((size_t)8 * nc * nc * sizeof(double));
    h->l2l_t = (double *)malloc((size_t)8 * nc * nc * sizeof(double));
    orc_build_m2l_tables(p, h->m2l_t);
    orc_build_m2m_tables(p, h->m2m_t);
    orc_build_l2l_tables(p, h->l2l_t);
    return h;
}

/* The reference's host path instead of its scalar operators (hostpath.c): the lists made
 * once here (the reference's plan holds them), the batched M2L in blocks of 64 targets and
 * the AVX-512 P2P; the same FMM to rounding (the P2P terms differ in the last bits). */
void orc_fmm_set_host_path(orc_fmm_handle *h, int on) {
    h->host_path = on;
    if (!on || h->v_row) return;
    const boxes_t *B = &h->PL.B;
    const size_t nb = B->nboxes, nl = h->PL.nleaves;
    h->v_row = (size_t *)calloc(nb + 1, sizeof(size_t));
    size_t (*vl)[2] = malloc(sizeof(size_t[189][2]));
    for (size_t b = 0; b < nb; ++b) h->v_row[b + 1] = h->v_row[b] + (size_t)(B->level[b] >= 2 ? v_list(B, b, vl) : 0);
    h->v_box = (size_t *)malloc((h->v_row[nb] + 1) * sizeof(size_t));
    h->v_off = (size_t *)malloc((h->v_row[nb] + 1) * sizeof(size_t));
    for (size_t b = 0; b < nb; ++b) {
        if (B->level[b] < 2) continue;
        int nv = v_list(B, b, vl);
        for (int e = 0; e < nv; ++e) {
            h->v_off[h->v_row[b] + e] = vl[e][0];
            h->v_box[h->v_row[b] + e] = vl[e][1];
        }
    }
    free(vl);
    vecz *nears = calloc(nl, sizeof(vecz)), *ws = calloc(nl, sizeof(vecz));
    h->near_row = (size_t *)calloc(nl + 1, sizeof(size_t));
    h->w_row = (size_t *)calloc(nl + 1, sizeof(size_t));
    for (size_t j = 0; j < nl; ++j) {
        leaf_lists(&h->PL, h->PL.leaf_box[j], &ws[j], &nears[j]);
        h->near_row[j + 1] = h->near_row[j] + nears[j].len;
        h->w_row[j + 1] = h->w_row[j] + ws[j].len;
    }
    h->near_leaf = (size_t *)malloc((h->near_row[nl] + 1) * sizeof(size_t));
    h->w_box = (size_t *)malloc((h->w_row[nl] + 1) * sizeof(size_t));
    for (size_t j = 0; j < nl; ++j) {
        if (nears[j].len) memcpy(h->near_leaf + h->near_row[j], nears[j].data, nears[j].len * sizeof(size_t));
        if (ws[j].len) memcpy(h->w_box + h->w_row[j], ws[j].data, ws[j].len * sizeof(size_t));
        free(nears[j].data);
        free(ws[j].data);
    }
    free(nears);
    free(ws);
}

void orc_fmm_free(orc_fmm_handle *h) {
    if (!h) return;
    free(h->v_row);
    free(h->v_box);
    free(h->v_off);
    free(h->near_row);
    free(h->near_leaf);
    free(h->w_row);
    free(h->w_box);
    free(h->m2l_t);
    free(h->m2m_t);
    free(h->l2l_t);
    plan_free(&h->PL);
    free(h);
}

/* One evaluation of a built FMM: charges q[i][v] in caller order, outputs in caller order
 * (phi[v][nt], grad[v][nt][3]); kinds bit 0 the near field, bit 1 the far field.  Its
 * wall time is orc_fmm_last_eval_seconds(). */
int orc_fmm_eval(orc_fmm_handle *h, const double *q, int threads, int kinds, double *phi_out, double *grad_out) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    const double t_start = omp_get_wtime();
    const int p = h->p, m = h->m, gradients = h->gradients;
    const size_t ns = h->ns, nt = h->nt;
    int nc = (p + 1) * (p + 1);
    const plan_t PL = h->PL;
    boxes_t B = PL.B;
    const double side = PL.side;
    size_t nleaves = PL.nleaves;
    long *leaf_of_box = PL.leaf_of_box;
    size_t *leaf_box = PL.leaf_box, *s_off = PL.s_off, *t_off = PL.t_off, *t_perm = PL.t_perm, *s_perm = PL.s_perm;
    double *us = PL.us, *ut = PL.ut;
    const double *m2l_t = h->m2l_t, *m2m_t = h->m2m_t, *l2l_t = h->l2l_t;
    /* charges in leaf order */
    double *qs = (double *)malloc((ns * m + 1) * sizeof(double));
    for (size_t a = 0; a < ns; ++a)
        for (int v = 0; v < m; ++v) qs[a * m + v] = q[s_perm[a] * m + v];

    double *M = (double *)calloc(B.nboxes * m * nc, sizeof(double));
    double *Lc = (double *)calloc(B.nboxes * m * nc, sizeof(double));
    double *phi = (double *)calloc(nt * m + 1, sizeof(double));
    double *grad = (double *)calloc(3 * nt * m + 1, sizeof(double));
    const double zero3[3] = {0.0, 0.0, 0.0};
    int L = B.nlevels - 1;

    /* ---- upward: for l = L..0: p2m(l); m2m(l-1) ---- */
    for (int l = L; l >= 0; --l) {
#pragma omp parallel for schedule(dynamic, 4)
        for (long b = (long)B.level_start[l]; b < (long)B.level_start[l + 1]; ++b) {
            if (!B.leaf[b]) continue;
            size_t j = (size_t)leaf_of_box[b];
            size_t n = s_off[j + 1] - s_off[j];
            orc_p2m(p, zero3, 1.0, n, us + 3 * s_off[j], qs + m * s_off[j], m, M + (size_t)b * m * nc);
        }
        if (l > 0) {
#pragma omp parallel for schedule(dynamic, 4)
            for (long b = (long)B.level_start[l - 1]; b < (long)B.level_start[l]; ++b) {
                if (B.leaf[b]) continue;
                for (int o = 0; o < 8; ++o) {
                    long c = child_box(&B, (size_t)b, o);
                    for (int v = 0; v < m; ++v)
                        orc_matvec(nc, m2m_t + (size_t)o * nc * nc, M + ((size_t)c * m + v) * nc,
                                   M + ((size_t)b * m + v) * nc);
                }
            }
        }
    }

    /* ---- downward: for l = 1..L: l2l, m2l (V by offset), p2l (X by source leaf) ---- */
    for (int l = 1; l <= L; ++l) {
        if (h->host_path) {
            /* the reference's batched M2L: L2L of every box, then the V products of blocks of
             * 64 consecutive targets, offset by offset, four columns at a time (each box's
             * chain: L2L, then V by offset index, then X, as below) */
#pragma omp parallel for schedule(dynamic, 4)
            for (long b = (long)B.level_start[l]; b < (long)B.level_start[l + 1]; ++b) {
                long P = parent_box(&B, (size_t)b);
                int o = (int)(((B.idx[b][0] & 1) << 2) | ((B.idx[b][1] & 1) << 1) | (B.idx[b][2] & 1));
                for (int v = 0; v < m; ++v)
                    orc_matvec(nc, l2l_t + (size_t)o * nc * nc, Lc + ((size_t)P * m + v) * nc,
                               Lc + ((size_t)b * m + v) * nc);
            }
            const long b0 = (long)B.level_start[l], b1 = (long)B.level_start[l + 1];
#pragma omp parallel for schedule(dynamic, 1)
            for (long blk = b0; blk < b1; blk += 64) {
                const long be = blk + 64 < b1 ? blk + 64 : b1;
                size_t npair = h->v_row[be] - h->v_row[blk];
                size_t *ord = (size_t *)malloc((npair + 1) * sizeof(size_t));
                for (size_t e = 0; e < npair; ++e) ord[e] = h->v_row[blk] + e;
                /* by offset index, then target (a V row is by offset: a stable merge) */
                size_t cnt[317] = {0};
                for (size_t e = 0; e < npair; ++e) cnt[h->v_off[ord[e]] + 1]++;
                for (int d = 0; d < 316; ++d) cnt[d + 1] += cnt[d];
                size_t *sorted = (size_t *)malloc((npair + 1) * sizeof(size_t)), fill[316];
                for (int d = 0; d < 316; ++d) fill[d] = cnt[d];
                for (size_t e = 0; e < npair; ++e) sorted[fill[h->v_off[ord[e]]]++] = ord[e];
                const double **bc = (const double **)malloc((npair + 1) * sizeof(double *));
                double **cc = (double **)malloc((npair + 1) * sizeof(double *));
                size_t *tbox = (size_t *)malloc((npair + 1) * sizeof(size_t));
                for (long t2 = blk; t2 < be; ++t2)
                    for (size_t e = h->v_row[t2]; e < h->v_row[t2 + 1]; ++e) tbox[e - h->v_row[blk]] = (size_t)t2;
                for (int v = 0; v < m; ++v)
                    for (int d = 0; d < 316; ++d) {
                        const int nq = (int)(cnt[d + 1] - cnt[d]);
                        if (!nq) continue;
                        for (int i = 0; i < nq; ++i) {
                            const size_t e = sorted[cnt[d] + i];
                            bc[i] = M + (h->v_box[e] * m + v) * nc;
                            cc[i] = Lc + (tbox[e - h->v_row[blk]] * m + v) * nc;
                        }
                        orc_hp_columns(nc, m2l_t + (size_t)d * nc * nc, bc, cc, nq);
                    }
                free(ord);
                free(sorted);
                free(bc);
                free(cc);
                free(tbox);
            }
#pragma omp parallel for schedule(dynamic, 4)
            for (long b = b0; b < b1; ++b) {
                long P = parent_box(&B, (size_t)b);
                double *Lb = Lc + (size_t)b * m * nc;
                vecz xl = {0, 0, 0};
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -1; dz <= 1; ++dz) {
                            if (!dx && !dy && !dz) continue;
                            long C = neighbour(&B, (size_t)P, dx, dy, dz);
                            if (C < 0 || !B.leaf[C] || adjacent_boxes(&B, (size_t)C, (size_t)b)) continue;
                            zpush(&xl, (size_t)leaf_of_box[C]);
                        }
                sort_unique(&xl);
                for (size_t e = 0; e < xl.len; ++e) {
                    size_t j = xl.data[e], s = leaf_box[j];
                    double c[3], r;
                    rel_frame(&B, (size_t)b, s, c, &r);
                    orc_p2l(p, c, r, s_off[j + 1] - s_off[j], us + 3 * s_off[j], qs + m * s_off[j], m, Lb);
                }
                free(xl.data);
            }
            continue;
        }
#pragma omp parallel for schedule(dynamic, 4)
        for (long b = (long)B.level_start[l]; b < (long)B.level_start[l + 1]; ++b) {
            long P = parent_box(&B, (size_t)b);
            int o = (int)(((B.idx[b][0] & 1) << 2) | ((B.idx[b][1] & 1) << 1) | (B.idx[b][2] & 1));
            double *Lb = Lc + (size_t)b * m * nc;
            for (int v = 0; v < m; ++v)
                orc_matvec(nc, l2l_t + (size_t)o * nc * nc, Lc + ((size_t)P * m + v) * nc, Lb + v * nc);
            /* V: children of the parent's colleagues, not adjacent to b, by offset index */
            size_t vl[189][2];
            int nv = 0;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        if (!dx && !dy && !dz) continue;
                        long C = neighbour(&B, (size_t)P, dx, dy, dz);
                        if (C < 0 || B.leaf[C]) continue;
                        for (int co = 0; co < 8; ++co) {
                            long s = child_box(&B, (size_t)C, co);
                            if (adjacent_boxes(&B, (size_t)s, (size_t)b)) continue;
                            vl[nv][0] = (size_t)offset_of(&B, (size_t)b, (size_t)s);
                            vl[nv][1] = (size_t)s;
                            ++nv;
                        }
                    }
            qsort(vl, nv, sizeof(vl[0]), cmp_pair);
            for (int e = 0; e < nv; ++e)
                for (int v = 0; v < m; ++v)
                    orc_matvec(nc, m2l_t + vl[e][0] * nc * nc, M + (vl[e][1] * m + v) * nc, Lb + v * nc);
            /* X: leaves among the parent's colleagues, not adjacent to b, by leaf index */
            vecz xl = {0, 0, 0};
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        if (!dx && !dy && !dz) continue;
                        long C = neighbour(&B, (size_t)P, dx, dy, dz);
                        if (C < 0 || !B.leaf[C] || adjacent_boxes(&B, (size_t)C, (size_t)b)) continue;
                        zpush(&xl, (size_t)leaf_of_box[C]);
                    }
            sort_unique(&xl);
            for (size_t e = 0; e < xl.len; ++e) {
                size_t j = xl.data[e], s = leaf_box[j];
                double c[3], r;
                rel_frame(&B, (size_t)b, s, c, &r); /* (c(t|s), r(t|s)) */
                orc_p2l(p, c, r, s_off[j + 1] - s_off[j], us + 3 * s_off[j], qs + m * s_off[j], m, Lb);
            }
            free(xl.data);
        }
    }

    /* ---- leaves: for l = 0..L: l2p, m2p (W by box index), p2p (near by source leaf) ---- */
    for (int l = 0; l <= L; ++l) {
#pragma omp parallel for schedule(dynamic, 2)
        for (long b = (long)B.level_start[l]; b < (long)B.level_start[l + 1]; ++b) {
            if (!B.leaf[b]) continue;
            size_t j = (size_t)leaf_of_box[b];
            size_t n = t_off[j + 1] - t_off[j];
            if (n == 0) continue;
            /* chunk-local outputs: phi[v][n], grad[v][n][3] */
            double *cphi = (double *)calloc(m * n, sizeof(double));
            double *cg = gradients ? (double *)calloc(3 * m * n, sizeof(double)) : NULL;
            const double *u = ut + 3 * t_off[j];
            if (kinds & 2) orc_l2p(p, zero3, 1.0, Lc + (size_t)b * m * nc, m, n, u, cphi, cg);
            vecz wl = {0, 0, 0}, near = {0, 0, 0};
            if (h->host_path) {  /* the lists the reference's plan holds */
                wl.data = h->w_box + h->w_row[j];
                wl.len = h->w_row[j + 1] - h->w_row[j];
                near.data = h->near_leaf + h->near_row[j];
                near.len = h->near_row[j + 1] - h->near_row[j];
            } else {
                leaf_lists(&PL, (size_t)b, &wl, &near);
            }
            for (size_t e = 0; e < ((kinds & 2) ? wl.len : 0); ++e) {
                size_t s = wl.data[e];
                double c[3], r;
                rel_frame(&B, s, (size_t)b, c, &r); /* (c(s|t), r(s|t)) */
                orc_m2p(p, c, r, M + s * m * nc, m, n, u, cphi, cg);
            }
            double *ys = NULL;
            size_t ys_cap = 0;
            for (size_t e = 0; e < ((kinds & 1) ? near.len : 0); ++e) {
                size_t sj = near.data[e], s = leaf_box[sj];
                size_t nsrc = s_off[sj + 1] - s_off[sj];
                const double *y = us + 3 * s_off[sj];
                if (sj != j) {
                    if (nsrc > ys_cap) { ys_cap = nsrc; ys = (double *)realloc(ys, 3 * nsrc * sizeof(double)); }
                    double c[3], r;
                    rel_frame(&B, s, (size_t)b, c, &r);
                    for (size_t a = 0; a < nsrc; ++a)
                        for (int k = 0; k < 3; ++k) ys[3 * a + k] = c[k] + r * us[3 * (s_off[sj] + a) + k];
                    y = ys;
                }
                double *qv = (double *)malloc((nsrc + 1) * sizeof(double));
                for (int v = 0; v < m; ++v) {
                    for (size_t a = 0; a < nsrc; ++a) qv[a] = qs[(s_off[sj] + a) * m + v];
                    if (h->host_path)
                        orc_hp_p2p(nsrc, y, qv, n, u, cphi + v * n, cg ? cg + 3 * v * n : NULL);
                    else
                        orc_p2p(nsrc, y, qv, n, u, cphi + v * n, cg ? cg + 3 * v * n : NULL);
                }
                free(qv);
            }
            free(ys);
            if (!h->host_path) {
                free(wl.data);
                free(near.data);
            }
            for (int v = 0; v < m; ++v)
                for (size_t a = 0; a < n; ++a) {
                    phi[v * nt + t_off[j] + a] = cphi[v * n + a];
                    if (cg)
                        for (int k = 0; k < 3; ++k) grad[3 * (v * nt + t_off[j] + a) + k] = cg[3 * (v * n + a) + k];
                }
            free(cphi);
            free(cg);
        }
    }

    /* ---- output pass ---- */
    for (size_t j = 0; j < nleaves; ++j) {
        double r = ldexp(side, -(B.level[leaf_box[j]] + 1));
        double ps = 4.0 * M_PI * r, gs = 4.0 * M_PI * r * r;
        for (size_t a = t_off[j]; a < t_off[j + 1]; ++a) {
            size_t i = t_perm[a];
            for (int v = 0; v < m; ++v) {
                phi_out[v * nt + i] = phi[v * nt + a] / ps;
                if (gradients && grad_out)
                    for (int k = 0; k < 3; ++k)
                        grad_out[3 * (v * nt + i) + k] = grad[3 * (v * nt + a) + k] / gs;
            }
        }
    }

    g_eval_seconds = omp_get_wtime() - t_start;
    free(M); free(Lc); free(phi); free(grad);
    free(qs);
    return 0;
}

int orc_fmm_kinds(size_t ns, const double *src, const double *q, int m, size_t nt, const double *tgt,
                  int p, int max_keys, int gradients, int threads, int kinds, double *phi_out,
                  double *grad_out) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    orc_fmm_handle *h = orc_fmm_new(ns, src, nt, tgt, p, max_keys, m, gradients);
    int rc = orc_fmm_eval(h, q, threads, kinds, phi_out, grad_out);
    orc_fmm_free(h);
    return rc;
}

/* The Helmholtz near field on the plan (see helmholtz.c for the term): charges q[i][v]
 * complex (2 m doubles per source), outputs phi[v][nt] and grad[v][nt][3] complex, caller
 * order, with 1/(4 pi r_t) (and r_t again for the gradient). */
int orc_helmholtz_near(size_t ns, const double *src, const double *q, int m, size_t nt, const double *tgt,
                       int max_keys, double kre, double kim, int gradients, int threads, double *phi_out,
                       double *grad_out) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    plan_t PL;
    plan_setup(&PL, ns, src, nt, tgt, max_keys);
    const boxes_t *Bp = &PL.B;
    const double r0 = ldexp(PL.side, -1);
    const double kr0[2] = {kre * r0, kim * r0};
    int L = Bp->nlevels - 1;
    for (int l = 0; l <= L; ++l) {
        const double kl[2] = {ldexp(kr0[0], -l), ldexp(kr0[1], -l)};
#pragma omp parallel for schedule(dynamic, 2)
        for (long b = (long)Bp->level_start[l]; b < (long)Bp->level_start[l + 1]; ++b) {
            if (!Bp->leaf[b]) continue;
            size_t j = (size_t)PL.leaf_of_box[b];
            size_t n = PL.t_off[j + 1] - PL.t_off[j];
            if (n == 0) continue;
            double *cphi = (double *)calloc(2 * m * n, sizeof(double));
            double *cg = gradients ? (double *)calloc(6 * m * n, sizeof(double)) : NULL;
            const double *u = PL.ut + 3 * PL.t_off[j];
            vecz wl = {0, 0, 0}, near = {0, 0, 0};
            leaf_lists(&PL, (size_t)b, &wl, &near);
            double *ys = NULL, *qv = NULL;
            size_t cap = 0;
            for (size_t e = 0; e < near.len; ++e) {
                size_t sj = near.data[e], s = PL.leaf_box[sj];
                size_t nsrc = PL.s_off[sj + 1] - PL.s_off[sj];
                if (nsrc > cap) {
                    cap = nsrc;
                    ys = (double *)realloc(ys, 3 * cap * sizeof(double));
                    qv = (double *)realloc(qv, 2 * cap * sizeof(double));
                }
                double c[3] = {0.0, 0.0, 0.0}, r = 1.0;
                if (sj != j) rel_frame(Bp, s, (size_t)b, c, &r);
                for (size_t a = 0; a < nsrc; ++a)
                    for (int k = 0; k < 3; ++k) {
                        double uu = PL.us[3 * (PL.s_off[sj] + a) + k];
                        ys[3 * a + k] = sj != j ? c[k] + r * uu : uu;
                    }
                for (int v = 0; v < m; ++v) {
                    for (size_t a = 0; a < nsrc; ++a) {
                        size_t i = PL.s_perm[PL.s_off[sj] + a];
                        qv[2 * a] = q[2 * (i * m + v)];
                        qv[2 * a + 1] = q[2 * (i * m + v) + 1];
                    }
                    orc_helmholtz_p2p(kl[0], kl[1], nsrc, ys, qv, n, u, cphi + 2 * v * n, cg ? cg + 6 * v * n : NULL);
                }
            }
            free(ys);
            free(qv);
            free(wl.data);
            free(near.data);
            double rt = ldexp(PL.side, -(l + 1));
            double ps = 4.0 * M_PI * rt, gs = 4.0 * M_PI * rt * rt;
            for (int v = 0; v < m; ++v)
                for (size_t a = 0; a < n; ++a) {
                    size_t i = PL.t_perm[PL.t_off[j] + a];
                    for (int c2 = 0; c2 < 2; ++c2) phi_out[2 * (v * nt + i) + c2] = cphi[2 * (v * n + a) + c2] / ps;
                    if (cg && grad_out)
                        for (int c2 = 0; c2 < 6; ++c2)
                            grad_out[6 * (v * nt + i) + c2] = cg[6 * (v * n + a) + c2] / gs;
                }
            free(cphi);
            free(cg);
        }
    }
    plan_free(&PL);
    return 0;
}
