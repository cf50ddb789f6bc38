/*
 * Oracle (test infrastructure only): the expansions of the Helmholtz family restated for
 * a real wavenumber k > 0 (Im k = 0, so the reference's damping exponents are zero).
 *   - real orthonormal harmonics, fmm-math/src/orthonormal/harmonics.rs:7-16 (CONVENTIONS
 *     §3.15 "Angular basis"): layout idx(n, m) = n^2 + n + m, the cos part in slot +m and
 *     the sin part in slot -m, no Condon-Shortley phase,
 *       Y_n^0 = sqrt((2n+1)/(4 pi)) Pb_n^0(cos t),
 *       Y_n^{+-m} = sqrt(2) sqrt((2n+1)/(4 pi)) Pb_n^m(cos t) {cos m f, sin m f},
 *     Pb_n^m = sqrt((n-m)!/(n+m)!) P_n^m; angular derivatives as harmonics_derivatives
 *     (harmonics.rs:62-78): d_t Pb_n^0 = -sqrt(n(n+1)) Pb_n^1,
 *     d_t Pb_n^m = (sqrt((n+m)(n-m+1)) Pb_n^{m-1} - sqrt((n-m)(n+m+1)) Pb_n^{m+1}) / 2, and
 *     (1/sin t) d_f from Pb_n^m / sin t (no division by sin t);
 *   - scaled radial functions, fmm-math/src/radial.rs:4-33: jh_n(z) = j_n(z) / s^n,
 *     hh_n(z) = h_n(z) s^n with h_n = j_n + i y_n, derivatives from the neighbouring orders
 *     (j_n' = (n j_{n-1} - (n+1) j_{n+1}) / (2n+1), h_n' = h_{n-1} - (n+1) h_n / z,
 *     j_0' = -j_1, h_0' = -h_1); j_n by Miller's backward recursion started where the
 *     forward recursion from the requested length has grown by 1e20, normalised by j_0 or
 *     j_1 (the larger), y_n upward from its closed forms;
 *   - a level of half-width r: circumradius a = sqrt(3) r, power scale s = min(k a, 1)
 *     (fmm-ref/src/helmholtz/level.rs:10-20);
 *   - leaf operators, fmm-ref/src/helmholtz/leaf.rs:6-33 (v = x - c, rho_j = y_j - c):
 *       P2M  M += sum_j q_j jh_n(k rho_j) Y(rho_j)
 *       L2P  phi += sum L jh_n(k |v|) Y(v)
 *       P2L  L += 4 pi i k sum_j q_j hh_n(k rho_j) Y(rho_j)
 *       M2P  phi += 4 pi i k sum M hh_n(k |v|) Y(v)
 *     the gradient that of the sum, f' Y r^ + (f/|v|)(d_t Y t^ + (1/sin t) d_f Y f^), with
 *     the limit k/(3s) of jh_1(k|v|)/|v| at the centre of a local; phi is the sum of
 *     q e^{ikr}/r (no 1/(4 pi)); a complex expansion is two real planes of (p+1)^2, the
 *     real parts then the imaginary parts;
 *   - translations by projection, fmm-ref/src/helmholtz/direct.rs:5-25: the input's field
 *     at the nodes of a product rule on the output's sphere (radius rho = the output's
 *     circumradius; Gauss-Legendre in cos t with Q nodes, uniform in f with 2Q,
 *     Q = p_in + p_out + ceil(k rho) + 40), A = int phi Y, B = int rho d_rho phi Y;
 *     multipole M = A / (4 pi i k hh_n(k rho)), local L = (f A + g B) / (f^2 + g^2) with
 *     f = jh_n(k rho), g = rho k jh_n'(k rho) (least squares: j_n has zeros).
 * The radial start order and the three-term harmonics recurrence are this file's own (the
 * reference forms the harmonics by a Cartesian recursion): these functions are pinned
 * against the direct sum (orc_helmholtz_direct_sum), not bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fmm_oracle.h"

#define HIDX(n, m) ((n) * (n) + (n) + (m))
#define HMAX 64 /* largest degree these functions take */

static const double kPi = 3.14159265358979323846;

/* ---- harmonics ---------------------------------------------------------------------- */

/* Y (and, when dt / df are given, d_t Y and (1/sin t) d_f Y) of the direction of x,
 * n <= p.  On the z-axis f = 0; at x = 0 also t = 0. */
void orc_hh_harmonics(int p, const double *x, double *Y, double *dt, double *df) {
    const double rho = sqrt(x[0] * x[0] + x[1] * x[1]);
    const double r = sqrt(rho * rho + x[2] * x[2]);
    const double c = r > 0.0 ? x[2] / r : 1.0, s = r > 0.0 ? rho / r : 0.0;
    const double cf = rho > 0.0 ? x[0] / rho : 1.0, sf = rho > 0.0 ? x[1] / rho : 0.0;
    /* Pb_n^m and Pb_n^m / sin t for m <= n <= p + 1: every entry read below is written */
    double pb[HMAX + 2][HMAX + 2], po[HMAX + 2][HMAX + 2];
    double pmm = 1.0, omm = 0.0; /* Pb_m^m and Pb_m^m / sin t */
    for (int m = 0; m <= p + 1; ++m) {
        if (m > 0) {
            const double f = sqrt((2.0 * m - 1.0) / (2.0 * m));
            omm = pmm * f; /* Pb_{m-1}^{m-1} sqrt((2m-1)/(2m)): one factor of sin t short */
            pmm = pmm * f * s;
        }
        pb[m][m] = pmm;
        po[m][m] = omm;
        if (m + 1 <= p + 1) {
            pb[m + 1][m] = c * sqrt(2.0 * m + 1.0) * pmm;
            po[m + 1][m] = c * sqrt(2.0 * m + 1.0) * omm;
        }
        for (int n = m + 2; n <= p + 1; ++n) {
            const double a = (2.0 * n - 1.0) * c, b = sqrt((double)(n - 1) * (n - 1) - (double)m * m);
            const double d = sqrt((double)n * n - (double)m * m);
            pb[n][m] = (a * pb[n - 1][m] - b * pb[n - 2][m]) / d;
            po[n][m] = (a * po[n - 1][m] - b * po[n - 2][m]) / d;
        }
    }
    double cm = 1.0, sm = 0.0; /* cos m f, sin m f */
    for (int m = 0; m <= p; ++m) {
        if (m > 0) {
            const double c2 = cm * cf - sm * sf, s2 = sm * cf + cm * sf;
            cm = c2;
            sm = s2;
        }
        for (int n = m; n <= p; ++n) {
            const double cn = sqrt((2.0 * n + 1.0) / (4.0 * kPi)) * (m ? sqrt(2.0) : 1.0);
            Y[HIDX(n, m)] = cn * pb[n][m] * cm;
            if (m) Y[HIDX(n, -m)] = cn * pb[n][m] * sm;
            if (!dt) continue;
            double d;
            if (m == 0)
                d = -sqrt((double)n * (n + 1)) * pb[n][1];
            else
                d = 0.5 * (sqrt((double)(n + m) * (n - m + 1)) * pb[n][m - 1] -
                           sqrt((double)(n - m) * (n + m + 1)) * (m + 1 <= n ? pb[n][m + 1] : 0.0));
            dt[HIDX(n, m)] = cn * d * cm;
            df[HIDX(n, m)] = -m * cn * po[n][m] * sm;
            if (m) {
                dt[HIDX(n, -m)] = cn * d * sm;
                df[HIDX(n, -m)] = m * cn * po[n][m] * cm;
            }
        }
    }
}

/* ---- radial functions ---------------------------------------------------------------- */

/* j_n(x), n = 0..nmax + 1 (x >= 0). */
static void sph_j(int nmax, double x, double *j) {
    const int len = nmax + 2;
    if (x == 0.0) {
        j[0] = 1.0;
        for (int n = 1; n < len; ++n) j[n] = 0.0;
        return;
    }
    /* start: where the forward recursion from the requested length has grown by 1e20 */
    double f0 = 0.0, f1 = 1.0;
    int n = len;
    while (fabs(f1) < 1e20 && n < len + 100000) {
        const double f2 = (2.0 * n + 1.0) / x * f1 - f0;
        f0 = f1;
        f1 = f2;
        ++n;
    }
    const int start = n + 1;
    double hi = 0.0, cur = 1e-250; /* f_{start+1}, f_start */
    for (int k = 0; k < len; ++k) j[k] = 0.0;
    for (int m = start; m >= 1; --m) {
        const double lo = (2.0 * m + 1.0) / x * cur - hi; /* f_{m-1} */
        hi = cur;
        cur = lo;
        if (m - 1 < len) j[m - 1] = cur;
        if (m < len) j[m] = hi;
        if (fabs(cur) > 1e200) { /* rescale what is stored and the running pair */
            cur *= 1e-200;
            hi *= 1e-200;
            for (int k = m - 1; k < len; ++k) j[k] *= 1e-200;
        }
    }
    /* normalise by j_0 or j_1, whichever is larger */
    double j0, j1;
    if (x < 1e-3) {
        const double x2 = x * x;
        j0 = 1.0 - x2 / 6.0 * (1.0 - x2 / 20.0 * (1.0 - x2 / 42.0));
        j1 = x / 3.0 * (1.0 - x2 / 10.0 * (1.0 - x2 / 28.0));
    } else {
        j0 = sin(x) / x;
        j1 = sin(x) / (x * x) - cos(x) / x;
    }
    const double scale = fabs(j0) >= fabs(j1) ? j0 / j[0] : j1 / j[1];
    for (int k = 0; k < len; ++k) j[k] *= scale;
}

/* y_n(x), n = 0..nmax + 1 (x > 0), upward (the stable direction). */
static void sph_y(int nmax, double x, double *y) {
    y[0] = -cos(x) / x;
    y[1] = -cos(x) / (x * x) - sin(x) / x;
    for (int n = 1; n <= nmax; ++n) y[n + 1] = (2.0 * n + 1.0) / x * y[n] - y[n - 1];
}

/* Scaled jh_n and jh_n' at z (n = 0..p); hh_n and hh_n' as (re, im) pairs when hh is given
 * (z > 0). */
void orc_hh_radial(int p, double z, double s, double *jh, double *jhp, double *hh, double *hhp) {
    double j[HMAX + 2], y[HMAX + 2];
    sph_j(p, z, j);
    double sn = 1.0;
    for (int n = 0; n <= p; ++n) {
        const double d = n == 0 ? -j[1] : (n * j[n - 1] - (n + 1) * j[n + 1]) / (2.0 * n + 1.0);
        jh[n] = j[n] / sn;
        if (jhp) jhp[n] = d / sn;
        sn *= s;
    }
    if (!hh) return;
    sph_y(p, z, y);
    sn = 1.0;
    for (int n = 0; n <= p; ++n) {
        hh[2 * n] = j[n] * sn;
        hh[2 * n + 1] = y[n] * sn;
        if (hhp) {
            double dr, di;
            if (n == 0) {
                dr = -j[1];
                di = -y[1];
            } else {
                dr = j[n - 1] - (n + 1) * j[n] / z;
                di = y[n - 1] - (n + 1) * y[n] / z;
            }
            hhp[2 * n] = dr * sn;
            hhp[2 * n + 1] = di * sn;
        }
        sn *= s;
    }
}

static double level_scale(double k, double half_width) {
    const double a = sqrt(3.0) * half_width;
    return k * a < 1.0 ? k * a : 1.0;
}

/* ---- leaf operators ------------------------------------------------------------------ */

static void cmul(const double a[2], const double b[2], double out[2]) {
    const double re = a[0] * b[0] - a[1] * b[1], im = a[0] * b[1] + a[1] * b[0];
    out[0] = re;
    out[1] = im;
}

/* P2M (regular) or P2L (singular) of complex charges q about centre c. */
static void form(int p, double k, double r, const double *c, size_t ns, const double *src, const double *q,
                 int singular, double *E) {
    const int nc = (p + 1) * (p + 1);
    const double s = level_scale(k, r);
    double Y[(HMAX + 1) * (HMAX + 1)], jh[HMAX + 1], hh[2 * (HMAX + 1)];
    for (size_t i = 0; i < ns; ++i) {
        const double v[3] = {src[3 * i] - c[0], src[3 * i + 1] - c[1], src[3 * i + 2] - c[2]};
        const double rho = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        orc_hh_harmonics(p, v, Y, NULL, NULL);
        orc_hh_radial(p, k * rho, s, jh, NULL, singular ? hh : NULL, NULL);
        for (int n = 0; n <= p; ++n) {
            double w[2]; /* the complex factor of degree n for this charge */
            if (singular) { /* 4 pi i k q hh_n */
                double qh[2];
                cmul(q + 2 * i, hh + 2 * n, qh);
                w[0] = -4.0 * kPi * k * qh[1];
                w[1] = 4.0 * kPi * k * qh[0];
            } else {
                w[0] = q[2 * i] * jh[n];
                w[1] = q[2 * i + 1] * jh[n];
            }
            for (int m = -n; m <= n; ++m) {
                E[HIDX(n, m)] += w[0] * Y[HIDX(n, m)];
                E[nc + HIDX(n, m)] += w[1] * Y[HIDX(n, m)];
            }
        }
    }
}

void orc_hh_p2m(int p, double k, double r, const double *c, size_t ns, const double *src, const double *q,
                double *M) {
    form(p, k, r, c, ns, src, q, 0, M);
}

void orc_hh_p2l(int p, double k, double r, const double *c, size_t ns, const double *src, const double *q,
                double *L) {
    form(p, k, r, c, ns, src, q, 1, L);
}

/* Field (and gradient) of an expansion about c at one point: a local (regular, factor 1)
 * or a multipole (singular, factor 4 pi i k). phi (re, im); grad 6 doubles
 * (re x, im x, re y, im y, re z, im z) when given. */
static void eval_point(int p, double k, double r, const double *c, const double *E, int singular, const double *x,
                       double *phi, double *grad) {
    const int nc = (p + 1) * (p + 1);
    const double s = level_scale(k, r);
    const double v[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
    const double d = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double Y[(HMAX + 1) * (HMAX + 1)], Dt[(HMAX + 1) * (HMAX + 1)], Df[(HMAX + 1) * (HMAX + 1)];
    double jh[HMAX + 1], jhp[HMAX + 1], hh[2 * (HMAX + 1)], hhp[2 * (HMAX + 1)];
    orc_hh_harmonics(p, v, Y, grad ? Dt : NULL, grad ? Df : NULL);
    orc_hh_radial(p, k * d, s, jh, jhp, singular ? hh : NULL, singular ? hhp : NULL);
    double f[2] = {0.0, 0.0}, gr[2] = {0.0, 0.0}, gt[2] = {0.0, 0.0}, gf[2] = {0.0, 0.0};
    for (int n = 0; n <= p; ++n) {
        double R[2], Rp[2], Rt[2]; /* radial value, k * derivative, value / |v| */
        if (singular) {
            R[0] = hh[2 * n];
            R[1] = hh[2 * n + 1];
            Rp[0] = k * hhp[2 * n];
            Rp[1] = k * hhp[2 * n + 1];
            Rt[0] = R[0] / d;
            Rt[1] = R[1] / d;
        } else {
            R[0] = jh[n];
            R[1] = 0.0;
            Rp[0] = k * jhp[n];
            Rp[1] = 0.0;
            Rt[0] = d > 0.0 ? jh[n] / d : (n == 1 ? k / (3.0 * s) : 0.0);
            Rt[1] = 0.0;
        }
        for (int m = -n; m <= n; ++m) {
            const double e[2] = {E[HIDX(n, m)], E[nc + HIDX(n, m)]};
            double t[2];
            cmul(e, R, t);
            f[0] += t[0] * Y[HIDX(n, m)];
            f[1] += t[1] * Y[HIDX(n, m)];
            if (!grad) continue;
            cmul(e, Rp, t);
            gr[0] += t[0] * Y[HIDX(n, m)];
            gr[1] += t[1] * Y[HIDX(n, m)];
            cmul(e, Rt, t);
            gt[0] += t[0] * Dt[HIDX(n, m)];
            gt[1] += t[1] * Dt[HIDX(n, m)];
            gf[0] += t[0] * Df[HIDX(n, m)];
            gf[1] += t[1] * Df[HIDX(n, m)];
        }
    }
    double out[8] = {f[0], f[1], 0, 0, 0, 0, 0, 0};
    if (grad) {
        /* spherical unit vectors of v's direction (the frame f = 0 on the z-axis) */
        const double rho = sqrt(v[0] * v[0] + v[1] * v[1]);
        const double ct = d > 0.0 ? v[2] / d : 1.0, st = d > 0.0 ? rho / d : 0.0;
        const double cf = rho > 0.0 ? v[0] / rho : 1.0, sf = rho > 0.0 ? v[1] / rho : 0.0;
        const double er[3] = {st * cf, st * sf, ct}, et[3] = {ct * cf, ct * sf, -st}, ef[3] = {-sf, cf, 0.0};
        if (d > 0.0) {
            for (int a = 0; a < 3; ++a) {
                out[2 + 2 * a] = gr[0] * er[a] + gt[0] * et[a] + gf[0] * ef[a];
                out[3 + 2 * a] = gr[1] * er[a] + gt[1] * et[a] + gf[1] * ef[a];
            }
        } else if (p >= 1) { /* at the centre: the gradient of the degree-1 part */
            const double g = sqrt(3.0 / (4.0 * kPi)) * k / (3.0 * s);
            const int slot[3] = {HIDX(1, 1), HIDX(1, -1), HIDX(1, 0)}; /* x, y, z */
            for (int a = 0; a < 3; ++a) {
                out[2 + 2 * a] = g * E[slot[a]];
                out[3 + 2 * a] = g * E[nc + slot[a]];
            }
        }
    }
    if (singular) { /* times 4 pi i k */
        for (int i = 0; i < 8; i += 2) {
            const double re = out[i], im = out[i + 1];
            out[i] = -4.0 * kPi * k * im;
            out[i + 1] = 4.0 * kPi * k * re;
        }
    }
    phi[0] += out[0];
    phi[1] += out[1];
    if (grad)
        for (int a = 0; a < 6; ++a) grad[a] += out[2 + a];
}

void orc_hh_l2p(int p, double k, double r, const double *c, const double *L, size_t nt, const double *tgt,
                double *phi, double *grad) {
    for (size_t i = 0; i < nt; ++i) eval_point(p, k, r, c, L, 0, tgt + 3 * i, phi + 2 * i, grad ? grad + 6 * i : NULL);
}

void orc_hh_m2p(int p, double k, double r, const double *c, const double *M, size_t nt, const double *tgt,
                double *phi, double *grad) {
    for (size_t i = 0; i < nt; ++i) eval_point(p, k, r, c, M, 1, tgt + 3 * i, phi + 2 * i, grad ? grad + 6 * i : NULL);
}

/* ---- translations by projection ----------------------------------------------------- */

/* Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_q from the Chebyshev guesses). */
static void gauss_legendre(int q, double *x, double *w) {
    for (int i = 0; i < q; ++i) {
        double z = cos(kPi * (i + 0.75) / (q + 0.5)), pp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = 0.0;
            for (int j = 1; j <= q; ++j) {
                const double p2 = p1;
                p1 = p0;
                p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
            }
            pp = q * (z * p0 - p1) / (z * z - 1.0);
            const double dz = p0 / pp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

/* in: expansion E_in about c_in (half-width r_in, degree p_in, singular or regular);
 * out: multipole (out_singular) or local about c_out (half-width r_out, degree p_out),
 * added into E_out. */
static void project(int p_in, double k, double r_in, const double *c_in, const double *E_in, int in_singular,
                    int p_out, double r_out, const double *c_out, int out_singular, double *E_out) {
    const int nc = (p_out + 1) * (p_out + 1);
    const double rho = sqrt(3.0) * r_out, s = level_scale(k, r_out);
    const int Q = p_in + p_out + (int)ceil(k * rho) + 40;
    double *gx = malloc(sizeof(double) * Q), *gw = malloc(sizeof(double) * Q);
    double *A = calloc(2 * (size_t)nc, sizeof(double)), *B = calloc(2 * (size_t)nc, sizeof(double));
    double Y[(HMAX + 1) * (HMAX + 1)];
    gauss_legendre(Q, gx, gw);
    for (int i = 0; i < Q; ++i) {
        const double ct = gx[i], st = sqrt(1.0 - ct * ct);
        for (int j = 0; j < 2 * Q; ++j) {
            const double f = 2.0 * kPi * j / (2.0 * Q), w = gw[i] * 2.0 * kPi / (2.0 * Q);
            const double u[3] = {st * cos(f), st * sin(f), ct};
            const double x[3] = {c_out[0] + rho * u[0], c_out[1] + rho * u[1], c_out[2] + rho * u[2]};
            double phi[2] = {0.0, 0.0}, g[6] = {0, 0, 0, 0, 0, 0};
            eval_point(p_in, k, r_in, c_in, E_in, in_singular, x, phi, out_singular ? NULL : g);
            /* rho d_rho phi = rho (grad phi . u) */
            const double b[2] = {rho * (g[0] * u[0] + g[2] * u[1] + g[4] * u[2]),
                                 rho * (g[1] * u[0] + g[3] * u[1] + g[5] * u[2])};
            orc_hh_harmonics(p_out, u, Y, NULL, NULL);
            for (int t = 0; t < nc; ++t) {
                A[t] += w * phi[0] * Y[t];
                A[nc + t] += w * phi[1] * Y[t];
                B[t] += w * b[0] * Y[t];
                B[nc + t] += w * b[1] * Y[t];
            }
        }
    }
    double jh[HMAX + 1], jhp[HMAX + 1], hh[2 * (HMAX + 1)];
    orc_hh_radial(p_out, k * rho, s, jh, jhp, out_singular ? hh : NULL, NULL);
    for (int n = 0; n <= p_out; ++n)
        for (int m = -n; m <= n; ++m) {
            const int t = HIDX(n, m);
            if (out_singular) { /* A / (4 pi i k hh_n) */
                const double dr = -4.0 * kPi * k * hh[2 * n + 1], di = 4.0 * kPi * k * hh[2 * n];
                const double den = dr * dr + di * di;
                E_out[t] += (A[t] * dr + A[nc + t] * di) / den;
                E_out[nc + t] += (A[nc + t] * dr - A[t] * di) / den;
            } else { /* (f A + g B) / (f^2 + g^2), f and g real for a real k */
                const double fv = jh[n], gv = rho * k * jhp[n], den = fv * fv + gv * gv;
                E_out[t] += (fv * A[t] + gv * B[t]) / den;
                E_out[nc + t] += (fv * A[nc + t] + gv * B[nc + t]) / den;
            }
        }
    free(gx);
    free(gw);
    free(A);
    free(B);
}

void orc_hh_m2m(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *M_in, double *M_out) {
    project(p_in, k, r_in, c_in, M_in, 1, p_out, r_out, c_out, 1, M_out);
}

void orc_hh_l2l(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *L_in, double *L_out) {
    project(p_in, k, r_in, c_in, L_in, 0, p_out, r_out, c_out, 0, L_out);
}

void orc_hh_m2l(int p_in, int p_out, double k, double r_in, const double *c_in, double r_out, const double *c_out,
                const double *M_in, double *L_out) {
    project(p_in, k, r_in, c_in, M_in, 1, p_out, r_out, c_out, 0, L_out);
}

/* ---- dense M2L tables by projection -------------------------------------------------- */

/* The M2L of one V-list offset on one level as one real 2n x n matrix (n = (p+1)^2),
 * column-major, the layout of fmm-tables/src/helmholtz/dense.rs:5-14: column j is the
 * local (real plane in rows 0..n, imaginary plane in rows n..2n) about the box at
 * 2r (dx, dy, dz) of the unit real multipole e_j about the box at the origin, both of
 * half-width r.  Each column is orc_hh_m2l of e_j (the same projection and quadrature);
 * the phi sums of a ring of nodes are taken per order first, so a table costs
 * O(Q^2 n p) instead of n projections. */
void orc_hh_m2l_dense(int p, double k, double r, int dx, int dy, int dz, double *table) {
    const int n = (p + 1) * (p + 1);
    const double rho = sqrt(3.0) * r, s = level_scale(k, r);
    const double cout[3] = {2.0 * r * dx, 2.0 * r * dy, 2.0 * r * dz};
    const int Q = 2 * p + (int)ceil(k * rho) + 40, NP = 2 * Q;
    double *gx = malloc(sizeof(double) * Q), *gw = malloc(sizeof(double) * Q);
    gauss_legendre(Q, gx, gw);
    /* per ring: F[j][m] = sum_l w_l field_j(node l) trig_m(phi_l), m = -p..p (A and B) */
    const int nm = 2 * p + 1;
    double *FA = malloc(sizeof(double) * 2 * (size_t)n * nm), *FB = malloc(sizeof(double) * 2 * (size_t)n * nm);
    double *A = calloc(2 * (size_t)n * n, sizeof(double)), *B = calloc(2 * (size_t)n * n, sizeof(double));
    double Y[(HMAX + 1) * (HMAX + 1)], Dt[(HMAX + 1) * (HMAX + 1)], Df[(HMAX + 1) * (HMAX + 1)], Yo[(HMAX + 1) * (HMAX + 1)];
    double jh[HMAX + 1], jhp[HMAX + 1], hh[2 * (HMAX + 1)], hhp[2 * (HMAX + 1)];
    double *fj = malloc(sizeof(double) * 2 * (size_t)n), *bj = malloc(sizeof(double) * 2 * (size_t)n);
    for (int i = 0; i < Q; ++i) {
        const double ct = gx[i], st = sqrt(1.0 - ct * ct);
        memset(FA, 0, sizeof(double) * 2 * (size_t)n * nm);
        memset(FB, 0, sizeof(double) * 2 * (size_t)n * nm);
        for (int l = 0; l < NP; ++l) {
            const double f = 2.0 * kPi * l / NP, wl = 2.0 * kPi / NP;
            const double u[3] = {st * cos(f), st * sin(f), ct};
            const double v[3] = {cout[0] + rho * u[0], cout[1] + rho * u[1], cout[2] + rho * u[2]};
            const double d = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            orc_hh_harmonics(p, v, Y, Dt, Df);
            orc_hh_radial(p, k * d, s, jh, jhp, hh, hhp);
            /* spherical unit vectors of v */
            const double rr = sqrt(v[0] * v[0] + v[1] * v[1]);
            const double c2 = v[2] / d, s2 = rr / d, cf = rr > 0.0 ? v[0] / rr : 1.0, sf = rr > 0.0 ? v[1] / rr : 0.0;
            const double er[3] = {s2 * cf, s2 * sf, c2}, et[3] = {c2 * cf, c2 * sf, -s2}, ef[3] = {-sf, cf, 0.0};
            const double uer = u[0] * er[0] + u[1] * er[1] + u[2] * er[2];
            const double uet = u[0] * et[0] + u[1] * et[1] + u[2] * et[2];
            const double uef = u[0] * ef[0] + u[1] * ef[1] + u[2] * ef[2];
            /* the unit multipole's field and rho d_rho of it: 4 pi i k times
             * hh Y and rho (k hh' Y u.er + (hh / d)(Dt u.et + Df u.ef)) */
            for (int dn = 0; dn <= p; ++dn)
                for (int m = -dn; m <= dn; ++m) {
                    const int j = HIDX(dn, m);
                    const double h0 = hh[2 * dn], h1 = hh[2 * dn + 1];
                    const double rad = k * uer * Y[j], tan = (uet * Dt[j] + uef * Df[j]) / d;
                    const double vr = h0 * Y[j], vi = h1 * Y[j];
                    const double br = rho * (rad * hhp[2 * dn] + tan * h0), bi = rho * (rad * hhp[2 * dn + 1] + tan * h1);
                    fj[2 * j] = -4.0 * kPi * k * vi; /* times i */
                    fj[2 * j + 1] = 4.0 * kPi * k * vr;
                    bj[2 * j] = -4.0 * kPi * k * bi;
                    bj[2 * j + 1] = 4.0 * kPi * k * br;
                }
            for (int m = -p; m <= p; ++m) {
                const double tr = wl * (m >= 0 ? cos(m * f) : sin(-m * f));
                double *fa = FA + 2 * (size_t)n * (m + p), *fb = FB + 2 * (size_t)n * (m + p);
                for (int j = 0; j < 2 * n; ++j) {
                    fa[j] += tr * fj[j];
                    fb[j] += tr * bj[j];
                }
            }
        }
        /* the output harmonics at this ring: Y_t(t_i, phi) = Yo_t(phi = 0 part) trig(m phi) */
        const double ud[3] = {st, 0.0, ct};
        orc_hh_harmonics(p, ud, Yo, NULL, NULL); /* at phi = 0: cos part = N Pb, sin part 0 */
        for (int tn = 0; tn <= p; ++tn)
            for (int tm = -tn; tm <= tn; ++tm) {
                const int t = HIDX(tn, tm);
                const double yt = gw[i] * Yo[HIDX(tn, tm < 0 ? -tm : tm)]; /* N Pb_n^|m| */
                const double *fa = FA + 2 * (size_t)n * (tm + p), *fb = FB + 2 * (size_t)n * (tm + p);
                for (int j = 0; j < n; ++j) {
                    A[2 * ((size_t)j * n + t)] += yt * fa[2 * j];
                    A[2 * ((size_t)j * n + t) + 1] += yt * fa[2 * j + 1];
                    B[2 * ((size_t)j * n + t)] += yt * fb[2 * j];
                    B[2 * ((size_t)j * n + t) + 1] += yt * fb[2 * j + 1];
                }
            }
    }
    orc_hh_radial(p, k * rho, s, jh, jhp, NULL, NULL);
    for (int j = 0; j < n; ++j)
        for (int tn = 0; tn <= p; ++tn) {
            const double fv = jh[tn], gv = rho * k * jhp[tn], den = fv * fv + gv * gv;
            for (int tm = -tn; tm <= tn; ++tm) {
                const int t = HIDX(tn, tm);
                const size_t a = 2 * ((size_t)j * n + t);
                table[(size_t)j * 2 * n + t] = (fv * A[a] + gv * B[a]) / den;
                table[(size_t)j * 2 * n + n + t] = (fv * A[a + 1] + gv * B[a + 1]) / den;
            }
        }
    free(gx);
    free(gw);
    free(FA);
    free(FB);
    free(A);
    free(B);
    free(fj);
    free(bj);
}
