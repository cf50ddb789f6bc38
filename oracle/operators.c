/*
 * Oracle (test infrastructure only): SplitMix64 and point distributions, the leaf
 * operators, the direct translations, P2P / direct sum and the operator tables of the
 * reference, restated in C.  Each function cites the reference lines it follows.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fmm_oracle.h"

/* ------------------------------------------------------------------------------------
 * SplitMix64 (fmm-validate/src/rng.rs:24-45) and distributions (points.rs)
 * ---------------------------------------------------------------------------------- */
uint64_t orc_rng_next(orc_rng *r) {
    r->state += 0x9e3779b97f4a7c15ULL;
    uint64_t z = r->state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

double orc_rng_uniform(orc_rng *r) {
    return (double)(orc_rng_next(r) >> 11) * (1.0 / (double)(1ULL << 53));
}

double orc_rng_range(orc_rng *r, double lo, double hi) { return lo + (hi - lo) * orc_rng_uniform(r); }

/* points.rs:148-152: Box-Muller cosine branch, 1 - U in (0, 1] */
double orc_rng_normal(orc_rng *r) {
    double radius = sqrt(-2.0 * log(1.0 - orc_rng_uniform(r)));
    return radius * cos(2.0 * M_PI * orc_rng_uniform(r));
}

void orc_points_cube(orc_rng *r, size_t n, const double c[3], double h, double *xyz) {
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = c[k] + h * orc_rng_range(r, -1.0, 1.0);
}

/* points.rs:154-163 */
static void in_unit_ball(orc_rng *r, double min_norm, double v[3]) {
    for (;;) {
        for (int k = 0; k < 3; ++k) v[k] = orc_rng_range(r, -1.0, 1.0);
        double s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (s <= 1.0 && s >= min_norm * min_norm) return;
    }
}

void orc_points_sphere_ball(orc_rng *r, size_t n, const double c[3], double radius, double *xyz) {
    for (size_t i = 0; i < n; ++i) {
        double v[3];
        in_unit_ball(r, 1e-3, v);
        double norm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = c[k] + radius * (v[k] / norm);
    }
}

void orc_points_sphere_gauss(orc_rng *r, size_t n, const double c[3], double radius, double *xyz) {
    for (size_t i = 0; i < n; ++i) {
        double v[3], s;
        do {
            for (int k = 0; k < 3; ++k) v[k] = orc_rng_normal(r);
            s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        } while (s < 1e-12);
        double norm = sqrt(s);
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = c[k] + radius * (v[k] / norm);
    }
}

/* points.rs:78-98 */
void orc_points_plummer(orc_rng *r, size_t n, const double c[3], double scale, double trunc,
                        double *xyz) {
    double x = trunc;
    double mass = x * x * x / pow(1.0 + x * x, 1.5);
    for (size_t i = 0; i < n; ++i) {
        double u = mass * orc_rng_uniform(r);
        double rad = u > 0.0 ? scale / sqrt(pow(u, -2.0 / 3.0) - 1.0) : 0.0;
        double v[3];
        in_unit_ball(r, 1e-3, v);
        double norm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = c[k] + rad * (v[k] / norm);
    }
}

/* points.rs:108-136 */
void orc_points_gaussian_clusters(orc_rng *r, size_t n, const double *centres, size_t k,
                                  double width, double *xyz) {
    size_t out = 0;
    for (size_t j = 0; j < k; ++j) {
        size_t count = n / k + (j < n % k ? 1 : 0);
        for (size_t i = 0; i < count; ++i) {
            double z[3];
            for (;;) {
                for (int a = 0; a < 3; ++a) z[a] = orc_rng_normal(r);
                if (z[0] * z[0] + z[1] * z[1] + z[2] * z[2] <= 16.0) break;
            }
            for (int a = 0; a < 3; ++a) xyz[3 * out + a] = centres[3 * j + a] + width * z[a];
            ++out;
        }
    }
}

void orc_charges(orc_rng *r, size_t n, double *q) {
    for (size_t i = 0; i < n; ++i) q[i] = orc_rng_range(r, -1.0, 1.0);
}

/* fmm-bench/src/measure.rs:49-56 */
void orc_sample(orc_rng *r, size_t n, size_t sampled, uint32_t *out) {
    uint32_t *order = (uint32_t *)malloc(n * sizeof(uint32_t));
    for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    if (sampled > n) sampled = n;
    for (size_t i = 0; i < sampled; ++i) {
        size_t j = i + (size_t)(((orc_rng_next(r) >> 32) * (uint64_t)(n - i)) >> 32);
        uint32_t t = order[i];
        order[i] = order[j];
        order[j] = t;
    }
    memcpy(out, order, sampled * sizeof(uint32_t));
    free(order);
}

/* ------------------------------------------------------------------------------------
 * Leaf operators (fmm-ref/src/leaf.rs)
 * ---------------------------------------------------------------------------------- */
static inline void frame_scaled(const double c[3], double r, const double x[3], double u[3]) {
    for (int k = 0; k < 3; ++k) u[k] = (x[k] - c[k]) / r; /* frame.rs Frame::scaled */
}

/* leaf.rs:509-517 add_conjugate */
static void add_conjugate(int p, double q, const double *values, double *out) {
    for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
            int i = orc_idx(n, m);
            out[i] = m < 0 ? out[i] - q * values[i] : out[i] + q * values[i];
        }
}

/* leaf.rs:521-540 contract (doubling rule) */
static double contract(int p, const double *c, const double *v) {
    double sum = 0.0;
    for (int n = 0; n <= p; ++n) {
        int z = orc_idx(n, 0);
        double orders = 0.0;
        for (int m = 1; m <= n; ++m) {
            int re = orc_idx(n, m), im = orc_idx(n, -m);
            orders = orders + c[re] * v[re] - c[im] * v[im];
        }
        sum = sum + c[z] * v[z] + 2.0 * orders;
    }
    return sum;
}

/* leaf.rs:113-145 p2m_many */
void orc_p2m(int p, const double centre[3], double radius, size_t ns, const double *src,
             const double *q, int m, double *multipoles) {
    int nc = (p + 1) * (p + 1);
    double *values = (double *)malloc(nc * sizeof(double));
    for (size_t j = 0; j < ns; ++j) {
        double u[3];
        frame_scaled(centre, radius, src + 3 * j, u);
        orc_regular(p, u, values);
        for (int v = 0; v < m; ++v) add_conjugate(p, q[j * m + v], values, multipoles + v * nc);
    }
    free(values);
}

/* leaf.rs:185-211 p2l_many */
void orc_p2l(int p, const double centre[3], double radius, size_t ns, const double *src,
             const double *q, int m, double *locals) {
    int nc = (p + 1) * (p + 1);
    double *values = (double *)malloc(nc * sizeof(double));
    for (size_t j = 0; j < ns; ++j) {
        double u[3];
        frame_scaled(centre, radius, src + 3 * j, u);
        orc_irregular(p, u, values);
        for (int v = 0; v < m; ++v) add_conjugate(p, q[j * m + v], values, locals + v * nc);
    }
    free(values);
}

/* leaf.rs:443-505 Expansion::evaluate */
static void evaluate(int regular, int p, const double centre[3], double radius,
                     const double *coeffs, int m, size_t nt, const double *tgt,
                     double *potential, double *gradient) {
    int nc = (p + 1) * (p + 1);
    double *vals = (double *)malloc(4 * nc * sizeof(double));
    double *gx = vals + nc, *gy = gx + nc, *gz = gy + nc;
    double r = radius, r2 = r * r;
    for (size_t i = 0; i < nt; ++i) {
        double v[3];
        frame_scaled(centre, radius, tgt + 3 * i, v);
        if (!gradient) {
            if (regular) orc_regular(p, v, vals);
            else orc_irregular(p, v, vals);
        } else {
            if (regular) orc_regular_grad(p, v, vals, gx, gy, gz);
            else orc_irregular_grad(p, v, vals, gx, gy, gz);
        }
        for (int c = 0; c < m; ++c) {
            const double *e = coeffs + c * nc;
            double *phi = potential + c * nt + i;
            *phi = *phi + contract(p, e, vals) / r;
            if (gradient) {
                double *g = gradient + 3 * (c * nt + i);
                g[0] = g[0] + contract(p, e, gx) / r2;
                g[1] = g[1] + contract(p, e, gy) / r2;
                g[2] = g[2] + contract(p, e, gz) / r2;
            }
        }
    }
    free(vals);
}

void orc_l2p(int p, const double centre[3], double radius, const double *locals, int m,
             size_t nt, const double *tgt, double *potential, double *gradient) {
    evaluate(1, p, centre, radius, locals, m, nt, tgt, potential, gradient);
}

void orc_m2p(int p, const double centre[3], double radius, const double *multipoles, int m,
             size_t nt, const double *tgt, double *potential, double *gradient) {
    evaluate(0, p, centre, radius, multipoles, m, nt, tgt, potential, gradient);
}

/* ------------------------------------------------------------------------------------
 * Direct translations (fmm-ref/src/direct.rs:75-240)
 * ---------------------------------------------------------------------------------- */
typedef struct { double re, im; } cx;

static inline cx cx_mul(cx a, cx b) {
    cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}

/* direct.rs read(): order q of degree n from real storage, zero beyond the degree */
static inline cx read_q(const double *v, int n, int q) {
    int m = q < 0 ? -q : q;
    cx z = {0.0, 0.0};
    if (m > n) return z;
    z.re = v[orc_idx(n, m)];
    z.im = m == 0 ? 0.0 : v[orc_idx(n, -m)];
    if (q < 0) {
        z.im = -z.im;
        if (m % 2 == 1) { z.re = -z.re; z.im = -z.im; }
    }
    return z;
}

static inline void add_out(double *out, int j, int i, cx v) {
    int re = orc_idx(j, i);
    out[re] = out[re] + v.re;
    if (i > 0) {
        int im = orc_idx(j, -i);
        out[im] = out[im] + v.im;
    }
}

static inline double power(double x, int k) {
    double acc = 1.0;
    for (int i = 0; i < k; ++i) acc = acc * x;
    return acc;
}

void orc_m2m(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out) {
    int np = (p + 1) * (p + 1);
    double b[3];
    frame_scaled(to_c, to_r, from_c, b);
    double rho = from_r / to_r;
    double *shift = (double *)malloc(np * sizeof(double));
    orc_regular(p, b, shift);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cx sum = {0.0, 0.0};
            for (int k = 0; k <= j; ++k) {
                cx orders = {0.0, 0.0};
                for (int l = -k; l <= k; ++l) {
                    cx a = read_q(in, k, l);
                    cx r = read_q(shift, j - k, i - l);
                    r.im = -r.im;
                    cx pr = cx_mul(a, r);
                    orders.re = orders.re + pr.re;
                    orders.im = orders.im + pr.im;
                }
                double s = power(rho, k);
                sum.re = sum.re + s * orders.re;
                sum.im = sum.im + s * orders.im;
            }
            add_out(out, j, i, sum);
        }
    free(shift);
}

void orc_l2l(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out) {
    int np = (p + 1) * (p + 1);
    double t[3];
    frame_scaled(from_c, from_r, to_c, t);
    double sigma = to_r / from_r;
    double *shift = (double *)malloc(np * sizeof(double));
    orc_regular(p, t, shift);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cx sum = {0.0, 0.0};
            for (int n = j; n <= p; ++n)
                for (int m = -n; m <= n; ++m) {
                    cx pr = cx_mul(read_q(in, n, m), read_q(shift, n - j, m - i));
                    sum.re = sum.re + pr.re;
                    sum.im = sum.im + pr.im;
                }
            double s = power(sigma, j + 1);
            cx v = {s * sum.re, s * sum.im};
            add_out(out, j, i, v);
        }
    free(shift);
}

void orc_m2l(int p, const double from_c[3], double from_r, const double to_c[3], double to_r,
             const double *in, double *out) {
    int p2 = 2 * p;
    int ns = (p2 + 1) * (p2 + 1);
    double b[3];
    frame_scaled(from_c, from_r, to_c, b);
    double sigma = to_r / from_r;
    double *shift = (double *)malloc(ns * sizeof(double));
    orc_irregular(p2, b, shift);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cx sum = {0.0, 0.0};
            for (int n = 0; n <= p; ++n)
                for (int m = -n; m <= n; ++m) {
                    cx pr = cx_mul(read_q(in, n, m), read_q(shift, n + j, m - i));
                    sum.re = sum.re + pr.re;
                    sum.im = sum.im + pr.im;
                }
            double sign = ((j + i) % 2 == 0) ? 1.0 : -1.0;
            double s = sign * power(sigma, j + 1);
            cx v = {s * sum.re, s * sum.im};
            add_out(out, j, i, v);
        }
    free(shift);
}

/* ------------------------------------------------------------------------------------
 * Tables (fmm-tables/src/geometry.rs:57-175, m2l.rs:67-96, octant.rs:150-174)
 * ---------------------------------------------------------------------------------- */
static int adjacent1(int64_t t) { return -1 <= t && t <= 1; }

void orc_offsets(int64_t *offsets) {
    int next = 0;
    for (int64_t x = -3; x <= 3; ++x)
        for (int64_t y = -3; y <= 3; ++y)
            for (int64_t z = -3; z <= 3; ++z)
                if (!(adjacent1(x) && adjacent1(y) && adjacent1(z))) {
                    offsets[3 * next] = x;
                    offsets[3 * next + 1] = y;
                    offsets[3 * next + 2] = z;
                    ++next;
                }
}

static int64_t kappa(int64_t t) {
    int64_t v = t + 1;
    if (v < 0) v = 0;
    if (v > 3) v = 3;
    return v;
}

int orc_offset_index(int64_t x, int64_t y, int64_t z) {
    if (x < -3 || x > 3 || y < -3 || y > 3 || z < -3 || z > 3) return -1;
    if (adjacent1(x) && adjacent1(y) && adjacent1(z)) return -1;
    return (int)(49 * (x + 3) + 7 * (y + 3) + (z + 3) - 9 * kappa(x) -
                 adjacent1(x) * (3 * kappa(y) + adjacent1(y) * kappa(z)));
}

void orc_build_m2l_tables(int p, double *tables) {
    int nc = (p + 1) * (p + 1);
    int64_t off[316 * 3];
    orc_offsets(off);
    double *unit = (double *)calloc(nc, sizeof(double));
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < 316; ++t) {
        double tc[3] = {2.0 * (double)off[3 * t], 2.0 * (double)off[3 * t + 1],
                        2.0 * (double)off[3 * t + 2]};
        for (int k = 0; k < nc; ++k) {
            double *col = tables + (size_t)t * nc * nc + (size_t)k * nc;
            memset(col, 0, nc * sizeof(double));
            unit[k] = 1.0;
            orc_m2l(p, zero, 1.0, tc, 1.0, unit, col);
            unit[k] = 0.0;
        }
    }
    free(unit);
}

/* child octant o = 4x + 2y + z, sign vector s_o = (2x-1, 2y-1, 2z-1) (CONVENTIONS 3.12) */
static void child_frame(int o, double c[3]) {
    int bits[3] = {(o >> 2) & 1, (o >> 1) & 1, o & 1};
    for (int k = 0; k < 3; ++k) c[k] = 0.5 * (double)(2 * bits[k] - 1);
}

void orc_build_m2m_tables(int p, double *tables) {
    int nc = (p + 1) * (p + 1);
    double *unit = (double *)calloc(nc, sizeof(double));
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int o = 0; o < 8; ++o) {
        double cc[3];
        child_frame(o, cc);
        for (int k = 0; k < nc; ++k) {
            double *col = tables + (size_t)o * nc * nc + (size_t)k * nc;
            memset(col, 0, nc * sizeof(double));
            unit[k] = 1.0;
            orc_m2m(p, cc, 0.5, zero, 1.0, unit, col);
            unit[k] = 0.0;
        }
    }
    free(unit);
}

void orc_build_l2l_tables(int p, double *tables) {
    int nc = (p + 1) * (p + 1);
    double *unit = (double *)calloc(nc, sizeof(double));
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int o = 0; o < 8; ++o) {
        double cc[3];
        child_frame(o, cc);
        for (int k = 0; k < nc; ++k) {
            double *col = tables + (size_t)o * nc * nc + (size_t)k * nc;
            memset(col, 0, nc * sizeof(double));
            unit[k] = 1.0;
            orc_l2l(p, zero, 1.0, cc, 0.5, unit, col);
            unit[k] = 0.0;
        }
    }
    free(unit);
}

/* ------------------------------------------------------------------------------------
 * P2P and the direct sum (fmm-ref/src/p2p.rs:90-186, Term at :400-433, Neumaier :436-460)
 * ---------------------------------------------------------------------------------- */
/* The reference's loop order, one target at a time (kept as the statement of the rule and
 * to check orc_p2p against). */
void orc_p2p_ref(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
                 double *potential, double *gradient) {
    for (size_t i = 0; i < nt; ++i) {
        const double *x = tgt + 3 * i;
        for (size_t j = 0; j < ns; ++j) {
            const double *y = src + 3 * j;
            if (x[0] == y[0] && x[1] == y[1] && x[2] == y[2]) continue;
            double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            double r = sqrt(r2);
            potential[i] = potential[i] + q[j] / r;
            if (gradient) {
                double r3 = r2 * r;
                for (int k = 0; k < 3; ++k)
                    gradient[3 * i + k] = gradient[3 * i + k] + -(q[j] * d[k] / r3);
            }
        }
    }
}

void orc_p2p(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
             double *potential, double *gradient) {
    if (nt == 0) return;
    double *w = (double *)malloc(7 * nt * sizeof(double));
    double *tx = w, *ty = w + nt, *tz = w + 2 * nt, *ph = w + 3 * nt, *g0 = w + 4 * nt, *g1 = w + 5 * nt,
           *g2 = w + 6 * nt;
    for (size_t i = 0; i < nt; ++i) {
        tx[i] = tgt[3 * i];
        ty[i] = tgt[3 * i + 1];
        tz[i] = tgt[3 * i + 2];
        ph[i] = potential[i];
        g0[i] = gradient ? gradient[3 * i] : 0.0;
        g1[i] = gradient ? gradient[3 * i + 1] : 0.0;
        g2[i] = gradient ? gradient[3 * i + 2] : 0.0;
    }
    orc_p2p_lanes(ns, src, q, nt, tx, ty, tz, ph, g0, g1, g2);  /* the gradient sums are dropped without one */
    for (size_t i = 0; i < nt; ++i) {
        potential[i] = ph[i];
        if (gradient) {
            gradient[3 * i] = g0[i];
            gradient[3 * i + 1] = g1[i];
            gradient[3 * i + 2] = g2[i];
        }
    }
    free(w);
}

typedef struct { double sum, comp; } neumaier;

static inline void nm_add(neumaier *s, double term) {
    double t = s->sum + term;
    if (fabs(s->sum) >= fabs(term)) s->comp += (s->sum - t) + term;
    else s->comp += (term - t) + s->sum;
    s->sum = t;
}

static void direct_one(size_t ns, const double *src, const double *q, const double *x,
                       double *phi, double *g) {
    neumaier s = {0, 0}, gs[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (size_t j = 0; j < ns; ++j) {
        const double *y = src + 3 * j;
        if (x[0] == y[0] && x[1] == y[1] && x[2] == y[2]) continue;
        double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double r = sqrt(r2);
        nm_add(&s, q[j] / r);
        if (g) {
            double r3 = r2 * r;
            for (int k = 0; k < 3; ++k) nm_add(&gs[k], -(q[j] * d[k] / r3));
        }
    }
    *phi += s.sum + s.comp;
    if (g)
        for (int k = 0; k < 3; ++k) g[k] += gs[k].sum + gs[k].comp;
}

void orc_direct_sum(size_t ns, const double *src, const double *q, size_t nt, const double *tgt,
                    double *potential, double *gradient) {
    for (size_t i = 0; i < nt; ++i)
        direct_one(ns, src, q, tgt + 3 * i, potential + i, gradient ? gradient + 3 * i : NULL);
}

void orc_direct_sum_omp(size_t ns, const double *src, const double *q, size_t nt,
                        const double *tgt, double *potential, double *gradient) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < (long)nt; ++i)
        direct_one(ns, src, q, tgt + 3 * i, potential + i, gradient ? gradient + 3 * i : NULL);
}
