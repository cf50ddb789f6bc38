/*
 * fmm_oracle.h -- CPU restatement of the tbetcke/fmm Laplace FMM, used ONLY as test
 * infrastructure: the parity checker of the tests, of __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  Nothing in the product (fmm_b200/) links or calls it.
 *
 * Everything here is f64 and serial unless stated, and follows the reference operation
 * by operation where the reference fixes an order (cited per function).  It is pinned
 * against the reference's own golden vectors: tests/golden/ holds the mpmath fixtures
 * of fmm-math/fixtures/harmonics_{A,B,C}.json (subset), the doc examples of
 * fmm-ref/src/p2p.rs:48-64 and fmm-ref/src/harmonics.rs, and the SplitMix64 seed-0
 * outputs of fmm-validate/src/rng.rs:58-64.
 *
 * Storage conventions (reference docs/CONVENTIONS.md section 3.6): coefficients of
 * degree <= p occupy (p+1)^2 reals at index n*n + n + m, slot m >= 0 the real part and
 * slot -m the imaginary part of the order-m value.
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- SplitMix64 and point distributions (fmm-validate/src/rng.rs, points.rs) ---- */
typedef struct { uint64_t state; } orc_rng;
uint64_t orc_rng_next(orc_rng *r);
double orc_rng_uniform(orc_rng *r);
double orc_rng_range(orc_rng *r, double lo, double hi);
double orc_rng_normal(orc_rng *r);
/* cube: centre + h * U[-1,1)^3 per component (points.rs:28) */
void orc_points_cube(orc_rng *r, size_t n, const double c[3], double h, double *xyz);
/* sphere as the reference draws it: ball rejection with min norm 1e-3, normalised (points.rs:48) */
void orc_points_sphere_ball(orc_rng *r, size_t n, const double c[3], double radius, double *xyz);
/* sphere from normalised Gaussian 3-vectors (the sphere workload's own rule) */
void orc_points_sphere_gauss(orc_rng *r, size_t n, const double c[3], double radius, double *xyz);
/* Plummer sphere truncated at `trunc` scale radii (points.rs:78, truncation 10) */
void orc_points_plummer(orc_rng *r, size_t n, const double c[3], double scale, double trunc, double *xyz);
/* isotropic Gaussian clusters truncated at 4 sigma (points.rs:108) */
void orc_points_gaussian_clusters(orc_rng *r, size_t n, const double *centres, size_t k,
                                  double width, double *xyz);
void orc_charges(orc_rng *r, size_t n, double *q); /* U[-1,1) (points.rs:138) */
/* partial Fisher-Yates sample of `sampled` indices (fmm-bench/src/measure.rs:49-56) */
void orc_sample(orc_rng *r, size_t n, size_t sampled, uint32_t *out);

/* ---- solid harmonics (fmm-math/src/harmonics.rs) ---- */
static inline int orc_idx(int n, int m) { return n * n + n + m; }
void orc_regular(int p, const double x[3], double *out);
void orc_irregular(int p, const double x[3], double *out);
void orc_regular_grad(int p, const double x[3], double *value, double *gx, double *gy, double *gz);
void orc_irregular_grad(int p, const double x[3], double *value, double *gx, double *gy, double *gz);

/* ---- leaf operators (fmm-ref/src/leaf.rs); frame = (centre, radius) ---- */
void orc_p2m(int p, const double centre[3], double radius, size_t ns, const double *src,
             const double *q, int m, double *multipoles);
void orc_p2l(int p, const double centre[3], double radius, size_t ns, const double *src,
             const double *q, int m, double *locals);
/* potential[v*nt + i], gradient[(v*nt + i)*3 + k]; gradient may be NULL */
void orc_l2p(int p, const double centre[3], double radius, const double *locals, int m,
             size_t nt, const double *tgt, double *potential, double *gradient);
void orc_m2p(int p, const double centre[3], double radius, const double *multipoles, int m,
             size_t nt, const double *tgt, double *potential, double *gradient);

/* ---- direct O(p^4) translations (fmm-ref/src/direct.rs) ---- */
void orc_m2m(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out);
void orc_l2l(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out);
void orc_m2l(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out);

/* ---- tables (fmm-tables/src/m2l.rs:67-160, octant.rs:59-174) ----
 * m2l: 316 matrices, m2m/l2l: 8 each, each (p+1)^2 x (p+1)^2 column-major. */
void orc_offsets(int64_t *offsets /* 316*3 */);
int orc_offset_index(int64_t dx, int64_t dy, int64_t dz);
void orc_build_m2l_tables(int p, double *tables);
void orc_build_m2m_tables(int p, double *tables);
void orc_build_l2l_tables(int p, double *tables);
/* y += A x, k ascending (fmm-tables/src/matrix_set.rs:128) */
void orc_matvec(int nc, const double *A, const double *x, double *y);

/* ---- P2P (fmm-ref/src/p2p.rs); orc_p2p_ref is the same sums one target at a time ---- */
void orc_p2p_ref(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
                 double *potential, double *gradient);
/* the sums of orc_p2p on targets split into coordinate and accumulator arrays */
void orc_p2p_lanes(size_t ns, const double *src, const double *q, size_t nt, const double *restrict tx,
                   const double *restrict ty, const double *restrict tz, double *restrict ph,
                   double *restrict g0, double *restrict g1, double *restrict g2);
void orc_p2p(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
             double *potential, double *gradient);
void orc_direct_sum(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
                    double *potential, double *gradient);
/* same as direct_sum, OpenMP over targets (bit-identical per target) */
void orc_direct_sum_omp(size_t ns, const double *src, const double *q, size_t nt,
                        const double *tgt, double *potential, double *gradient);

/* ---- Morton keys and the octree (octree/src/morton.rs, octree/implementation.rs) ---- */
uint64_t orc_key_from_index(const uint32_t idx[3], int level);
void orc_key_decode(uint64_t key, int *level, uint32_t idx[3]);
/* cubic domain of sources ++ targets (octree.rs:1278-1370, fmm-exec/src/geometry.rs:120) */
void orc_domain(size_t ns, const double *src, size_t nt, const double *tgt, double lower[3],
                double *side, double box6[6]);
uint64_t orc_point_key(const double x[3], const double box6[6], int level);

/* A built tree + its interaction lists, all boxes level-major in key order. */
typedef struct orc_tree orc_tree;
orc_tree *orc_tree_build(size_t ns, const double *src, size_t nt, const double *tgt,
                         int max_level, int max_keys);
void orc_tree_free(orc_tree *t);
int orc_tree_nlevels(const orc_tree *t);
size_t orc_tree_nboxes(const orc_tree *t);
size_t orc_tree_nleaves(const orc_tree *t);
void orc_tree_boxes(const orc_tree *t, uint64_t *keys, uint8_t *is_leaf);
void orc_tree_domain(const orc_tree *t, double lower[3], double *side);
/* lists of box b as sorted key arrays; kind 0=U 1=V 2=W 3=X; returns count, writes up to cap */
size_t orc_tree_list(const orc_tree *t, size_t box, int kind, uint64_t *out, size_t cap);

/* ---- the host FMM (fmm-exec operator bodies, fmm-plan evaluator order) ----
 * Returns phi[v*nt + i] and grad[(v*nt + i)*3 + k] in caller order, with 1/(4 pi r_t)
 * applied as fmm-exec/src/fmm.rs:4750-4778.  `threads` > 1 uses OpenMP over targets
 * and boxes (bit-identical to serial).  Returns 0 on success. */
int orc_fmm(size_t ns, const double *src, const double *q, int m, size_t nt, const double *tgt,
            int p, int max_keys, int gradients, int threads, double *phi, double *grad);

/* seconds of the last orc_fmm / orc_fmm_kinds call without its plan and table builds */
double orc_fmm_last_eval_seconds(void);

/* the same with a kinds mask: bit 0 the near field (P2P), bit 1 the far field (L2P, M2P
 * and everything upstream of them); 3 is the whole FMM */
int orc_fmm_kinds(size_t ns, const double *src, const double *q, int m, size_t nt,
                  const double *tgt, int p, int max_keys, int gradients, int threads, int kinds,
                  double *phi, double *grad);

/* A built FMM kept for repeated evaluations (plan and tables once, the reference's
 * FmmBuilder::build then Fmm::evaluate): orc_fmm_eval takes caller-order charges q[i][v]
 * and writes caller-order outputs as orc_fmm; its wall time is orc_fmm_last_eval_seconds(). */
typedef struct orc_fmm_handle orc_fmm_handle;
orc_fmm_handle *orc_fmm_new(size_t ns, const double *src, size_t nt, const double *tgt, int p, int max_keys,
                            int m, int gradients);
int orc_fmm_eval(orc_fmm_handle *h, const double *q, int threads, int kinds, double *phi, double *grad);
void orc_fmm_free(orc_fmm_handle *h);
/* on = 1: the reference's host path (hostpath.c: lists made once, batched M2L, AVX-512 P2P)
 * in the following evaluations; 0: the scalar operators (the parity oracle) */
void orc_fmm_set_host_path(orc_fmm_handle *h, int on);
/* hostpath.c */
int orc_hp_has_avx512(void);
void orc_hp_p2p(size_t ns, const double *src, const double *q, size_t nt, const double *tgt, double *potential,
                double *gradient);
void orc_hp_columns(int n, const double *A, const double *const *bcols, double *const *ccols, int ncol);
void orc_matvec(int nc, const double *A, const double *x, double *y);

/* Helmholtz (helmholtz.c): complex values are (re, im) double pairs.  p2p and the
 * Neumaier direct sum of e^{ikr}/r (no 1/(4 pi)), potential[nt] and gradient[nt][3]
 * complex, += into the outputs */
void orc_helmholtz_p2p(double kre, double kim, size_t ns, const double *src, const double *q, size_t nt,
                       const double *tgt, double *potential, double *gradient);
void orc_helmholtz_direct_sum(double kre, double kim, size_t ns, const double *src, const double *q, size_t nt,
                              const double *tgt, double *potential, double *gradient);
/* Helmholtz expansions for a real k (helmholtz_ops.c): complex expansions are two real
 * planes of (p + 1)^2 (real parts, then imaginary parts) in the layout n^2 + n + m; a box
 * is its centre and half-width r; phi and grad as orc_helmholtz_p2p (e^{ikr}/r sums). */
void orc_hh_harmonics(int p, const double *x, double *Y, double *dt, double *df);
void orc_hh_radial(int p, double z, double s, double *jh, double *jhp, double *hh, double *hhp);
void orc_hh_p2m(int p, double k, double r, const double *c, size_t ns, const double *src, const double *q,
                double *M);
void orc_hh_p2l(int p, double k, double r, const double *c, size_t ns, const double *src, const double *q,
                double *L);
void orc_hh_l2p(int p, double k, double r, const double *c, const double *L, size_t nt, const double *tgt,
                double *phi, double *grad);
void orc_hh_m2p(int p, double k, double r, const double *c, const double *M, size_t nt, const double *tgt,
                double *phi, double *grad);
void orc_hh_m2m(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *M_in, double *M_out);
void orc_hh_l2l(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *L_in, double *L_out);
void orc_hh_m2l(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *M_in, double *L_out);
/* the dense M2L of offset (dx, dy, dz) on a level of half-width r: a real 2n x n matrix,
 * column-major, column j the local (real plane over imaginary plane) of the unit real
 * multipole e_j (n = (p + 1)^2) */
void orc_hh_m2l_dense(int p, double k, double r, int dx, int dy, int dz, double *table);
/* the Helmholtz near field on the plan (fmm.c), with 1/(4 pi) */
int orc_helmholtz_near(size_t ns, const double *src, const double *q, int m, size_t nt, const double *tgt,
                       int max_keys, double kre, double kim, int gradients, int threads, double *phi,
                       double *grad);

/* the oracle's own scaling of one leaf-scaled coordinate (fmm-exec/src/geometry.rs:291) */
double orc_leaf_coordinate(double x, double lower, double side, int level, uint32_t index);

#ifdef __cplusplus
}
#endif
#endif
