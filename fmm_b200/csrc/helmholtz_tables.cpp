// Dense M2L tables of the Helmholtz family for a real wavenumber, built on the host in f64
// (the reference's DenseM2l, fmm-tables/src/helmholtz/dense.rs:1-30): per level and V-list
// offset d (the 316 offsets in index order, target box at 2 r d from the source box) one
// real 2n x n matrix, n = (p+1)^2, column-major, column j the local of the unit real
// multipole e_j: the real plane in rows 0..n, the imaginary plane in rows n..2n.  A complex
// multipole M = M_r + i M_i then gives L_r = A_r M_r - A_i M_i, L_i = A_i M_r + A_r M_i.
//
// Expansions (fmm-ref/src/helmholtz/leaf.rs:6-33, real k): about a box centre, with
// v = x - c, a multipole is phi(x) = 4 pi i k sum M_n^m hh_n(k|v|) Y_n^m(v^) and a local
// phi(x) = sum L_n^m jh_n(k|v|) Y_n^m(v^), jh_n = j_n / s^n, hh_n = h_n s^n, h_n = j_n + i y_n,
// s = min(k a, 1), a = sqrt(3) r (fmm-ref/src/helmholtz/level.rs:10-20); Y_n^m the real
// orthonormal harmonics of fmm-math/src/orthonormal/harmonics.rs:7-16 (layout n^2 + n + m,
// cos part in slot +m, sin part in slot -m, no Condon-Shortley phase).
//
// Each column is the M2L by projection (fmm-ref/src/helmholtz/direct.rs:5-25): the unit
// multipole's field phi and rho d_rho phi at the nodes of a product rule on the target's
// sphere (radius rho = a; Gauss-Legendre in cos t with Q nodes, uniform in f with 2Q,
// Q = 2p + ceil(k rho) + 40), projected on Y, and the local by least squares from value
// and radial derivative, L = (f A + g B) / (f^2 + g^2), f = jh_n(k rho),
// g = rho k jh_n'(k rho).  The f sums of a ring of nodes are taken per order m first, so
// all n columns of an offset cost O(Q^2 n p); the offsets run on the host's threads.
#include <algorithm>
#include <cmath>
#include <exception>
#include <functional>
#include <thread>
#include <vector>

#include "plan.hpp"

namespace fmmb {

namespace {

constexpr double kPi = 3.14159265358979323846;

inline int hidx(int n, int m) { return n * n + n + m; }

// Y, d_t Y and (1/sin t) d_f Y of the direction of x (f = 0 on the z-axis).
void harmonics(int p, const double* x, double* Y, double* dt, double* df) {
    const double rho = std::sqrt(x[0] * x[0] + x[1] * x[1]);
    const double r = std::sqrt(rho * rho + x[2] * x[2]);
    const double c = r > 0.0 ? x[2] / r : 1.0, s = r > 0.0 ? rho / r : 0.0;
    const double cf = rho > 0.0 ? x[0] / rho : 1.0, sf = rho > 0.0 ? x[1] / rho : 0.0;
    const int P1 = p + 2;
    // normalised Legendre Pb_n^m (and Pb_n^m / sin t) for m <= n <= p + 1
    std::vector<double> pb((size_t)P1 * P1, 0.0), po((size_t)P1 * P1, 0.0);
    auto at = [&](std::vector<double>& a, int n, int m) -> double& { return a[(size_t)n * P1 + m]; };
    double pmm = 1.0, omm = 0.0;
    for (int m = 0; m <= p + 1; ++m) {
        if (m > 0) {
            const double f = std::sqrt((2.0 * m - 1.0) / (2.0 * m));
            omm = pmm * f;
            pmm = pmm * f * s;
        }
        at(pb, m, m) = pmm;
        at(po, m, m) = omm;
        if (m + 1 <= p + 1) {
            at(pb, m + 1, m) = c * std::sqrt(2.0 * m + 1.0) * pmm;
            at(po, m + 1, m) = c * std::sqrt(2.0 * m + 1.0) * omm;
        }
        for (int n = m + 2; n <= p + 1; ++n) {
            const double a = (2.0 * n - 1.0) * c, b = std::sqrt((double)(n - 1) * (n - 1) - (double)m * m);
            const double d = std::sqrt((double)n * n - (double)m * m);
            at(pb, n, m) = (a * at(pb, n - 1, m) - b * at(pb, n - 2, m)) / d;
            at(po, n, m) = (a * at(po, n - 1, m) - b * at(po, n - 2, m)) / d;
        }
    }
    double cm = 1.0, sm = 0.0;
    for (int m = 0; m <= p; ++m) {
        if (m > 0) {
            const double c2 = cm * cf - sm * sf, s2 = sm * cf + cm * sf;
            cm = c2;
            sm = s2;
        }
        for (int n = m; n <= p; ++n) {
            const double cn = std::sqrt((2.0 * n + 1.0) / (4.0 * kPi)) * (m ? std::sqrt(2.0) : 1.0);
            Y[hidx(n, m)] = cn * at(pb, n, m) * cm;
            if (m) Y[hidx(n, -m)] = cn * at(pb, n, m) * sm;
            if (!dt) continue;
            const double d = m == 0 ? -std::sqrt((double)n * (n + 1)) * at(pb, n, 1)
                                    : 0.5 * (std::sqrt((double)(n + m) * (n - m + 1)) * at(pb, n, m - 1) -
                                             std::sqrt((double)(n - m) * (n + m + 1)) * (m + 1 <= n ? at(pb, n, m + 1) : 0.0));
            dt[hidx(n, m)] = cn * d * cm;
            df[hidx(n, m)] = -m * cn * at(po, n, m) * sm;
            if (m) {
                dt[hidx(n, -m)] = cn * d * sm;
                df[hidx(n, -m)] = m * cn * at(po, n, m) * cm;
            }
        }
    }
}

// j_n(x), n = 0..nmax + 1: Miller's backward recursion from where the forward recursion has
// grown by 1e20, normalised by the larger of j_0 and j_1.
void sph_j(int nmax, double x, double* j) {
    const int len = nmax + 2;
    if (x == 0.0) {
        j[0] = 1.0;
        for (int n = 1; n < len; ++n) j[n] = 0.0;
        return;
    }
    double f0 = 0.0, f1 = 1.0;
    int n = len;
    while (std::fabs(f1) < 1e20 && n < len + 100000) {
        const double f2 = (2.0 * n + 1.0) / x * f1 - f0;
        f0 = f1;
        f1 = f2;
        ++n;
    }
    double hi = 0.0, cur = 1e-250;
    for (int k = 0; k < len; ++k) j[k] = 0.0;
    for (int m = n + 1; m >= 1; --m) {
        const double lo = (2.0 * m + 1.0) / x * cur - hi;
        hi = cur;
        cur = lo;
        if (m - 1 < len) j[m - 1] = cur;
        if (m < len) j[m] = hi;
        if (std::fabs(cur) > 1e200) {
            cur *= 1e-200;
            hi *= 1e-200;
            for (int k = m - 1; k < len; ++k) j[k] *= 1e-200;
        }
    }
    double j0, j1;
    if (x < 1e-3) {
        const double x2 = x * x;
        j0 = 1.0 - x2 / 6.0 * (1.0 - x2 / 20.0 * (1.0 - x2 / 42.0));
        j1 = x / 3.0 * (1.0 - x2 / 10.0 * (1.0 - x2 / 28.0));
    } else {
        j0 = std::sin(x) / x;
        j1 = std::sin(x) / (x * x) - std::cos(x) / x;
    }
    const double scale = std::fabs(j0) >= std::fabs(j1) ? j0 / j[0] : j1 / j[1];
    for (int k = 0; k < len; ++k) j[k] *= scale;
}

// jh, jh' (n = 0..p) and, when given, hh and hh' as (re, im) pairs, at z > 0 (z = 0 for jh).
void radial(int p, double z, double s, double* jh, double* jhp, double* hh, double* hhp) {
    std::vector<double> j(p + 2), y(p + 2);
    sph_j(p, z, j.data());
    double sn = 1.0;
    for (int n = 0; n <= p; ++n) {
        const double d = n == 0 ? -j[1] : (n * j[n - 1] - (n + 1) * j[n + 1]) / (2.0 * n + 1.0);
        jh[n] = j[n] / sn;
        jhp[n] = d / sn;
        sn *= s;
    }
    if (!hh) return;
    y[0] = -std::cos(z) / z;
    y[1] = -std::cos(z) / (z * z) - std::sin(z) / z;
    for (int n = 1; n <= p; ++n) y[n + 1] = (2.0 * n + 1.0) / z * y[n] - y[n - 1];
    sn = 1.0;
    for (int n = 0; n <= p; ++n) {
        hh[2 * n] = j[n] * sn;
        hh[2 * n + 1] = y[n] * sn;
        const double dr = n == 0 ? -j[1] : j[n - 1] - (n + 1) * j[n] / z;
        const double di = n == 0 ? -y[1] : y[n - 1] - (n + 1) * y[n] / z;
        hhp[2 * n] = dr * sn;
        hhp[2 * n + 1] = di * sn;
        sn *= s;
    }
}

void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& w) {
    x.assign(q, 0.0);
    w.assign(q, 0.0);
    for (int i = 0; i < q; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (q + 0.5)), pp = 0.0;
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
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

// One table (2n x n, column-major): column j the output expansion of the unit real input
// expansion e_j.  Input: a multipole (singular) or local about c_in, boxes of half-width
// r_in; output: a multipole or local about c_out, half-width r_out, projected on the
// output's sphere (radius the output's circumradius).
void dense_translation(int p, double k, bool in_singular, double r_in, const double* c_in, bool out_singular,
                       double r_out, const double* c_out, double* table) {
    const int n = (p + 1) * (p + 1), nm = 2 * p + 1;
    const double rho = std::sqrt(3.0) * r_out;
    const double s_in = std::min(k * std::sqrt(3.0) * r_in, 1.0), s_out = std::min(k * rho, 1.0);
    const int Q = 2 * p + (int)std::ceil(k * rho) + 40, NP = 2 * Q;
    std::vector<double> gx, gw;
    gauss_legendre(Q, gx, gw);
    std::vector<double> FA(2 * (size_t)n * nm), FB(2 * (size_t)n * nm), A(2 * (size_t)n * n, 0.0),
        B(2 * (size_t)n * n, 0.0), Y(n), Dt(n), Df(n), Yo(n), jh(p + 1), jhp(p + 1), hh(2 * (p + 1)),
        hhp(2 * (p + 1)), fj(2 * (size_t)n), bj(2 * (size_t)n);
    for (int i = 0; i < Q; ++i) {
        const double ct = gx[i], st = std::sqrt(1.0 - ct * ct);
        std::fill(FA.begin(), FA.end(), 0.0);
        std::fill(FB.begin(), FB.end(), 0.0);
        for (int l = 0; l < NP; ++l) {
            const double f = 2.0 * kPi * l / NP, wl = 2.0 * kPi / NP;
            const double u[3] = {st * std::cos(f), st * std::sin(f), ct};
            const double v[3] = {c_out[0] + rho * u[0] - c_in[0], c_out[1] + rho * u[1] - c_in[1],
                                 c_out[2] + rho * u[2] - c_in[2]};
            const double dv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            harmonics(p, v, Y.data(), Dt.data(), Df.data());
            radial(p, k * dv, s_in, jh.data(), jhp.data(), in_singular ? hh.data() : nullptr,
                   in_singular ? hhp.data() : nullptr);
            const double rr = std::sqrt(v[0] * v[0] + v[1] * v[1]);
            const double c2 = dv > 0.0 ? v[2] / dv : 1.0, s2 = dv > 0.0 ? rr / dv : 0.0;
            const double cf = rr > 0.0 ? v[0] / rr : 1.0, sf = rr > 0.0 ? v[1] / rr : 0.0;
            const double uer = u[0] * s2 * cf + u[1] * s2 * sf + u[2] * c2;
            const double uet = u[0] * c2 * cf + u[1] * c2 * sf - u[2] * s2;
            const double uef = -u[0] * sf + u[1] * cf;
            for (int dn = 0; dn <= p; ++dn) {
                // the radial value R, k R' and R / |v| of degree dn (complex for a multipole)
                double R[2], Rp[2], Rt[2];
                if (in_singular) {
                    R[0] = hh[2 * dn];
                    R[1] = hh[2 * dn + 1];
                    Rp[0] = k * hhp[2 * dn];
                    Rp[1] = k * hhp[2 * dn + 1];
                    Rt[0] = R[0] / dv;
                    Rt[1] = R[1] / dv;
                } else {
                    R[0] = jh[dn];
                    R[1] = 0.0;
                    Rp[0] = k * jhp[dn];
                    Rp[1] = 0.0;
                    Rt[0] = dv > 0.0 ? jh[dn] / dv : (dn == 1 ? k / (3.0 * s_in) : 0.0);
                    Rt[1] = 0.0;
                }
                for (int m = -dn; m <= dn; ++m) {
                    const int jj = hidx(dn, m);
                    const double rad = uer * Y[jj], tan = uet * Dt[jj] + uef * Df[jj];
                    double fv[2] = {R[0] * Y[jj], R[1] * Y[jj]};
                    double bv[2] = {rho * (Rp[0] * rad + Rt[0] * tan), rho * (Rp[1] * rad + Rt[1] * tan)};
                    if (in_singular) {  // times 4 pi i k
                        const double a0 = fv[0], b0 = bv[0];
                        fv[0] = -4.0 * kPi * k * fv[1];
                        fv[1] = 4.0 * kPi * k * a0;
                        bv[0] = -4.0 * kPi * k * bv[1];
                        bv[1] = 4.0 * kPi * k * b0;
                    }
                    fj[2 * jj] = fv[0];
                    fj[2 * jj + 1] = fv[1];
                    bj[2 * jj] = bv[0];
                    bj[2 * jj + 1] = bv[1];
                }
            }
            for (int m = -p; m <= p; ++m) {
                const double tr = wl * (m >= 0 ? std::cos(m * f) : std::sin(-m * f));
                double* fa = &FA[2 * (size_t)n * (m + p)];
                double* fb = &FB[2 * (size_t)n * (m + p)];
                for (int e = 0; e < 2 * n; ++e) {
                    fa[e] += tr * fj[e];
                    fb[e] += tr * bj[e];
                }
            }
        }
        const double ud[3] = {st, 0.0, ct};
        harmonics(p, ud, Yo.data(), nullptr, nullptr);
        for (int tn = 0; tn <= p; ++tn)
            for (int tm = -tn; tm <= tn; ++tm) {
                const int t = hidx(tn, tm);
                const double yt = gw[i] * Yo[hidx(tn, tm < 0 ? -tm : tm)];
                const double* fa = &FA[2 * (size_t)n * (tm + p)];
                const double* fb = &FB[2 * (size_t)n * (tm + p)];
                for (int jj = 0; jj < n; ++jj) {
                    const size_t o = 2 * ((size_t)jj * n + t);
                    A[o] += yt * fa[2 * jj];
                    A[o + 1] += yt * fa[2 * jj + 1];
                    B[o] += yt * fb[2 * jj];
                    B[o + 1] += yt * fb[2 * jj + 1];
                }
            }
    }
    radial(p, k * rho, s_out, jh.data(), jhp.data(), out_singular ? hh.data() : nullptr,
           out_singular ? hhp.data() : nullptr);
    for (int jj = 0; jj < n; ++jj)
        for (int tn = 0; tn <= p; ++tn) {
            for (int tm = -tn; tm <= tn; ++tm) {
                const int t = hidx(tn, tm);
                const size_t o = 2 * ((size_t)jj * n + t);
                double re, im;
                if (out_singular) {  // A / (4 pi i k hh_n)
                    const double dr = -4.0 * kPi * k * hh[2 * tn + 1], di = 4.0 * kPi * k * hh[2 * tn];
                    const double den = dr * dr + di * di;
                    re = (A[o] * dr + A[o + 1] * di) / den;
                    im = (A[o + 1] * dr - A[o] * di) / den;
                } else {  // (f A + g B) / (f^2 + g^2)
                    const double fv = jh[tn], gv = rho * k * jhp[tn], den = fv * fv + gv * gv;
                    re = (fv * A[o] + gv * B[o]) / den;
                    im = (fv * A[o + 1] + gv * B[o + 1]) / den;
                }
                table[(size_t)jj * 2 * n + t] = re;
                table[(size_t)jj * 2 * n + n + t] = im;
            }
        }
}

// One offset's M2L table: source box at the origin, target at 2 r d.
void dense_m2l(int p, double k, double r, const int d[3], double* table) {
    const double c0[3] = {0.0, 0.0, 0.0}, ct[3] = {2.0 * r * d[0], 2.0 * r * d[1], 2.0 * r * d[2]};
    dense_translation(p, k, true, r, c0, false, r, ct, table);
}

// Runs work(t) for t = 0..count-1 on up to `threads` host threads; an exception in any of
// them (an allocation failure) is rethrown here after all have joined.
void parallel_for(int count, int threads, const std::function<void(int)>& work) {
    const int nt = std::max(1, std::min(threads, count));
    std::vector<std::exception_ptr> err(nt);
    std::vector<std::thread> pool;
    for (int w = 0; w < nt; ++w)
        pool.emplace_back([&, w] {
            try {
                for (int t = w; t < count; t += nt) work(t);
            } catch (...) {
                err[w] = std::current_exception();
            }
        });
    for (auto& th : pool) th.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

int host_threads() { return (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 64u)); }

}  // namespace

// The 8 octants' M2M and L2L tables of a parent level of half-width r (child o at the
// parent centre + r/2 (+-1, +-1, +-1), the sign of x from bit 2 of o, y bit 1, z bit 0):
// M2M takes a child's multipole to the parent's, L2L the parent's local to the child's.
void build_helmholtz_octant_tables(int p, double k, double r, std::vector<double>& m2m, std::vector<double>& l2l) {
    const int n = (p + 1) * (p + 1);
    const size_t per = 2 * (size_t)n * n;
    m2m.assign(8 * per, 0.0);
    l2l.assign(8 * per, 0.0);
    parallel_for(16, host_threads(), [&](int t) {
        const int o = t >> 1;
        const double c0[3] = {0.0, 0.0, 0.0};
        const double cc[3] = {((o >> 2) & 1) ? 0.5 * r : -0.5 * r, ((o >> 1) & 1) ? 0.5 * r : -0.5 * r,
                              (o & 1) ? 0.5 * r : -0.5 * r};
        if (t & 1)
            dense_translation(p, k, false, r, c0, false, 0.5 * r, cc, &l2l[per * o]);
        else
            dense_translation(p, k, true, 0.5 * r, cc, true, r, c0, &m2m[per * o]);
    });
}

// The 316 offsets' tables of one level (boxes of half-width r), one after the other in
// offset index order: 316 * 2 n^2 doubles.
void build_helmholtz_m2l_tables(int p, double k, double r, std::vector<double>& out) {
    std::vector<int> off;
    for (int x = -3; x <= 3; ++x)
        for (int y = -3; y <= 3; ++y)
            for (int z = -3; z <= 3; ++z)
                if (offset_index(x, y, z) >= 0) {
                    off.push_back(x);
                    off.push_back(y);
                    off.push_back(z);
                }
    const int n = (p + 1) * (p + 1), count = (int)off.size() / 3;
    const size_t per = 2 * (size_t)n * n;
    out.assign(per * count, 0.0);
    parallel_for(count, host_threads(), [&](int t) { dense_m2l(p, k, r, &off[3 * t], &out[per * t]); });
}

}  // namespace fmmb
