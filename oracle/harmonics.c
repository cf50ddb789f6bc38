/*
 * Oracle (test infrastructure only): solid harmonics R_n^m, I_n^m and their gradients in
 * real storage, restating fmm-math/src/harmonics.rs:118-440 operation by operation
 * (built with -ffp-contract=off so no product is fused, as in the reference).
 */
#include <math.h>
#include <string.h>

#include "fmm_oracle.h"

typedef struct { double re, im; } cplx;

static inline void store(double *out, int n, int m, cplx v) {
    out[orc_idx(n, m)] = v.re;
    if (m > 0) out[orc_idx(n, -m)] = v.im;
}

static inline cplx load(const double *v, int n, int m) {
    cplx c;
    c.re = v[orc_idx(n, m)];
    c.im = m == 0 ? 0.0 : v[orc_idx(n, -m)];
    return c;
}

/* X_n^{-k} = (-1)^k conj(X_n^k)  (harmonics.rs:50-57) */
static inline cplx negate_order(int k, cplx v) {
    cplx r;
    if (k % 2 == 0) { r.re = v.re; r.im = -v.im; }
    else { r.re = -v.re; r.im = v.im; }
    return r;
}

static inline cplx value_at(const double *v, int n, int m) {
    int k = m < 0 ? -m : m;
    cplx z = {0.0, 0.0};
    if (k > n) return z;
    z = load(v, n, k);
    return m < 0 ? negate_order(k, z) : z;
}

static inline void three_term(double *out, int n, int m, double c1, double c2) {
    cplx a = load(out, n - 1, m), b = load(out, n - 2, m);
    cplx r = {c1 * a.re + c2 * b.re, c1 * a.im + c2 * b.im};
    store(out, n, m, r);
}

/* rho (re, im) scaled by s, rho = x + iy  (harmonics.rs:80-83) */
static inline cplx times_rho(double x, double y, double s, cplx v) {
    cplx r = {(x * v.re - y * v.im) * s, (x * v.im + y * v.re) * s};
    return r;
}

/* harmonics.rs:118-140 */
void orc_regular(int p, const double xv[3], double *out) {
    double x = xv[0], y = xv[1], z = xv[2];
    double r2 = x * x + y * y + z * z;
    cplx diag = {1.0, 0.0};
    for (int m = 0; m <= p; ++m) {
        if (m > 0) diag = times_rho(x, y, 1.0 / (double)(2 * m), diag);
        store(out, m, m, diag);
        if (m == p) break;
        cplx nxt = {z * diag.re, z * diag.im};
        store(out, m + 1, m, nxt);
        for (int n = m + 2; n <= p; ++n) {
            double den = (double)((n + m) * (n - m));
            double c1 = (double)(2 * n - 1) * z / den;
            double c2 = -r2 / den;
            three_term(out, n, m, c1, c2);
        }
    }
}

/* harmonics.rs:163-187 */
void orc_irregular(int p, const double xv[3], double *out) {
    double x = xv[0], y = xv[1], z = xv[2];
    double r2 = x * x + y * y + z * z;
    double inv_r2 = 1.0 / r2;
    cplx diag = {1.0 / sqrt(r2), 0.0};
    for (int m = 0; m <= p; ++m) {
        if (m > 0) diag = times_rho(x, y, (double)(2 * m - 1) * inv_r2, diag);
        store(out, m, m, diag);
        if (m == p) break;
        double c = (double)(2 * m + 1) * z * inv_r2;
        cplx nxt = {c * diag.re, c * diag.im};
        store(out, m + 1, m, nxt);
        for (int n = m + 2; n <= p; ++n) {
            double c1 = (double)(2 * n - 1) * z * inv_r2;
            double c2 = -(double)((n - 1 - m) * (n - 1 + m)) * inv_r2;
            three_term(out, n, m, c1, c2);
        }
    }
}

/* harmonics.rs:193-205: from [A, B, C] = [X_s^{m-1}, X_s^{m+1}, X_s^m] */
static inline void store_ladder(double *gx, double *gy, double *gz, int n, int m, cplx a,
                                cplx b, cplx c, double sigma) {
    const double half = 0.5;
    cplx vx = {(a.re - b.re) * half, (a.im - b.im) * half};
    cplx vy = {-(a.im + b.im) * half, (a.re + b.re) * half};
    cplx vz = {sigma * c.re, sigma * c.im};
    store(gx, n, m, vx);
    store(gy, n, m, vy);
    store(gz, n, m, vz);
}

/* harmonics.rs:228-245 */
void orc_regular_grad(int p, const double x[3], double *value, double *gx, double *gy,
                      double *gz) {
    orc_regular(p, x, value);
    cplx zero = {0.0, 0.0};
    store_ladder(gx, gy, gz, 0, 0, zero, zero, zero, 1.0);
    for (int n = 1; n <= p; ++n)
        for (int m = 0; m <= n; ++m) {
            cplx a = value_at(value, n - 1, m - 1);
            cplx b = value_at(value, n - 1, m + 1);
            cplx c = value_at(value, n - 1, m);
            store_ladder(gx, gy, gz, n, m, a, b, c, 1.0);
        }
}

/* I_{p+1}^k from degrees p and p-1 (harmonics.rs:250-286) */
static cplx irregular_above(const double *values, int p, int k, const double xv[3],
                            double inv_r2) {
    double x = xv[0], y = xv[1], z = xv[2];
    int j = k < 0 ? -k : k;
    cplx v = {0.0, 0.0};
    if (j > p + 1) return v;
    if (j == p + 1) {
        v = times_rho(x, y, (double)(2 * p + 1) * inv_r2, load(values, p, p));
    } else if (j == p) {
        double c = (double)(2 * p + 1) * z * inv_r2;
        cplx a = load(values, p, p);
        v.re = c * a.re;
        v.im = c * a.im;
    } else {
        double c1 = (double)(2 * p + 1) * z * inv_r2;
        double c2 = -(double)((p - j) * (p + j)) * inv_r2;
        cplx a = load(values, p, j), b = load(values, p - 1, j);
        v.re = c1 * a.re + c2 * b.re;
        v.im = c1 * a.im + c2 * b.im;
    }
    return k < 0 ? negate_order(j, v) : v;
}

/* harmonics.rs:328-355 */
void orc_irregular_grad(int p, const double x[3], double *value, double *gx, double *gy,
                        double *gz) {
    orc_irregular(p, x, value);
    for (int n = 0; n < p; ++n)
        for (int m = 0; m <= n; ++m) {
            cplx a = value_at(value, n + 1, m - 1);
            cplx b = value_at(value, n + 1, m + 1);
            cplx c = value_at(value, n + 1, m);
            store_ladder(gx, gy, gz, n, m, a, b, c, -1.0);
        }
    double inv_r2 = 1.0 / (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    for (int m = 0; m <= p; ++m) {
        cplx a = irregular_above(value, p, m - 1, x, inv_r2);
        cplx b = irregular_above(value, p, m + 1, x, inv_r2);
        cplx c = irregular_above(value, p, m, x, inv_r2);
        store_ladder(gx, gy, gz, p, m, a, b, c, -1.0);
    }
}
