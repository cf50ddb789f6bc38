// Helmholtz far field on the device, e^{ikr}/(4 pi r) for a real wavenumber: the leaf
// operators (P2M, P2L, L2P, M2P) of complex expansions in the reference's real
// orthonormal harmonics and scaled radial functions (fmm-ref/src/helmholtz/leaf.rs:6-33;
// fmm-math/src/orthonormal/harmonics.rs:7-16; fmm-math/src/radial.rs:4-33).
//
// Units.  Every box works in its own leaf-scaled frame (half-width 1) with the level's
// wavenumber k_l = k r_l and power scale s_l = min(sqrt(3) k_l, 1) (fmm-ref/src/
// helmholtz/level.rs:10-20 in box units).  Since the radial arguments are products k r,
// a multipole formed in box units is the multipole of absolute units, and a local in box
// units is r_l times the absolute one; the near field and the output pass then follow the
// Laplace path (phi / (4 pi r_t), grad / ((4 pi r_t) r_t)).  Expansions:
//   P2M   M += sum_j q_j jh_n(k_l rho_j) Y(rho_j)
//   P2L   L += 4 pi i k_l sum_j q_j hh_n(k_l rho_j) Y(rho_j)      (rho_j in the box's frame)
//   L2P   phi += sum L jh_n(k_l |u|) Y(u)
//   M2P   phi += (1 / r) 4 pi i k_s sum M hh_n(k_s |v|) Y(v),      v = (u - c) / r,
// (c, r) the source box's frame seen from the target leaf, the gradient (1 / r^2) times
// the source frame's.  A complex expansion of vector v is two rows of the expansion
// array: row 2v its real parts, row 2v + 1 its imaginary parts (each (p+1)^2 slots in
// the layout idx(n, m) = n^2 + n + m, cos part in slot +m, sin part in slot -m).
//
// The harmonics and the radial functions are formed in f64 in both precisions (the mixed
// form stores and translates its expansions in f32).
#pragma once

#include "helmholtz.cuh"
#include "kernels.cuh"

namespace fmmb {

// sqrt of a compile-time constant by Newton's iteration (Heron's method), for the tables
// below; converges to within an ulp of the rounded root
constexpr double ce_sqrt(double x) {
    if (x <= 0.0) return 0.0;
    double g = x > 1.0 ? x : 1.0;
    for (int i = 0; i < 200; ++i) g = 0.5 * (g + x / g);
    return g;
}

// Constants of the real orthonormal harmonics to degree P (Pb_n^m = sqrt((n-m)!/(n+m)!)
// P_n^m, no Condon-Shortley phase), formed at compile time.
template <int P>
struct HhConst {
    double ra[P + 1][P + 1];  // (2n - 1) / sqrt(n^2 - m^2):      Pb_n^m = ra c Pb_{n-1}^m - rb Pb_{n-2}^m
    double rb[P + 1][P + 1];  // sqrt((n-1)^2 - m^2) / sqrt(n^2 - m^2)
    double rc[P + 1];         // sqrt(2m + 1):                     Pb_{m+1}^m = c rc Pb_m^m
    double rf[P + 1];         // sqrt((2m - 1) / (2m)):            Pb_m^m = rf s Pb_{m-1}^{m-1}
    double cn[P + 1][P + 1];  // sqrt((2n + 1) / (4 pi)), times sqrt(2) for m > 0
    double dm[P + 1][P + 1];  // d_t Pb_n^m = dm Pb_n^{m-1} - dp Pb_n^{m+1}; m = 0: dm = 0, dp = sqrt(n (n+1))
    double dp[P + 1][P + 1];
    constexpr HhConst() : ra{}, rb{}, rc{}, rf{}, cn{}, dm{}, dp{} {
        const double pi4 = 4.0 * 3.14159265358979323846;
        for (int m = 0; m <= P; ++m) {
            rc[m] = ce_sqrt(2.0 * m + 1.0);
            rf[m] = m > 0 ? ce_sqrt((2.0 * m - 1.0) / (2.0 * m)) : 0.0;
            for (int n = m; n <= P; ++n) {
                if (n >= m + 2) {
                    const double d = ce_sqrt((double)n * n - (double)m * m);
                    ra[n][m] = (2.0 * n - 1.0) / d;
                    rb[n][m] = ce_sqrt((double)(n - 1) * (n - 1) - (double)m * m) / d;
                }
                cn[n][m] = ce_sqrt((2.0 * n + 1.0) / pi4) * (m ? ce_sqrt(2.0) : 1.0);
                if (m == 0) {
                    dm[n][m] = 0.0;
                    dp[n][m] = ce_sqrt((double)n * (n + 1));
                } else {
                    dm[n][m] = 0.5 * ce_sqrt((double)(n + m) * (n - m + 1));
                    dp[n][m] = 0.5 * ce_sqrt((double)(n - m) * (n + m + 1));
                }
            }
        }
    }
};

template <int P>
__constant__ HhConst<P> kHhConst = HhConst<P>();

// The real orthonormal harmonics of the direction of (x, y, z), streamed column by
// column: f(n, m, yc, ys, tc, ts, fc, fs) for m = 0..P, n = m..P, with yc / ys the cos /
// sin parts of Y_n^m (slots +m / -m; ys = 0 for m = 0) and, with DERIV, tc / ts their
// theta derivatives and fc / fs their phi derivatives over sin theta.  On the z-axis
// phi = 0; at the origin theta = 0 as well.  Three columns of Pb (m - 1, m, m + 1) are
// held in registers.
template <int P, bool DERIV, class F>
__device__ __forceinline__ void hh_harmonics(double x, double y, double z, F&& f) {
    const HhConst<P>& K = kHhConst<P>;
    const double rho = sqrt(x * x + y * y);
    const double r = sqrt(rho * rho + z * z);
    const double c = r > 0.0 ? z / r : 1.0, s = r > 0.0 ? rho / r : 0.0;
    const double cf = rho > 0.0 ? x / rho : 1.0, sf = rho > 0.0 ? y / rho : 0.0;
    double prev[P + 2], cur[P + 2], nxt[P + 2], ocur[P + 2], onxt[P + 2];
#pragma unroll
    for (int n = 0; n < P + 2; ++n) prev[n] = cur[n] = nxt[n] = ocur[n] = onxt[n] = 0.0;
    double pmm = 1.0, omm = 0.0;  // Pb_m^m and Pb_m^m / sin t of the last column formed
    auto column = [&](int m, double (&pb)[P + 2], double (&po)[P + 2]) {
        if (m > 0) {
            omm = pmm * K.rf[m];
            pmm = omm * s;
        }
#pragma unroll
        for (int n = 0; n < P + 2; ++n) pb[n] = po[n] = 0.0;
        pb[m] = pmm;
        po[m] = omm;
        if (m + 1 <= P) {
            pb[m + 1] = c * K.rc[m] * pmm;
            po[m + 1] = c * K.rc[m] * omm;
        }
#pragma unroll
        for (int n = m + 2; n <= P; ++n) {
            pb[n] = K.ra[n][m] * c * pb[n - 1] - K.rb[n][m] * pb[n - 2];
            po[n] = K.ra[n][m] * c * po[n - 1] - K.rb[n][m] * po[n - 2];
        }
    };
    column(0, cur, ocur);
    if (P >= 1) column(1, nxt, onxt);
    double cm = 1.0, sm = 0.0;  // cos m phi, sin m phi
#pragma unroll
    for (int m = 0; m <= P; ++m) {
        if (m > 0) {
            const double c2 = cm * cf - sm * sf, s2 = sm * cf + cm * sf;
            cm = c2;
            sm = s2;
        }
#pragma unroll
        for (int n = m; n <= P; ++n) {
            const double a = K.cn[n][m] * cur[n];
            double tc = 0.0, ts = 0.0, fc = 0.0, fs = 0.0;
            if (DERIV) {
                const double d = K.dm[n][m] * prev[n] - (m + 1 <= n ? K.dp[n][m] * nxt[n] : 0.0);
                tc = K.cn[n][m] * d * cm;
                ts = K.cn[n][m] * d * sm;
                const double o = (double)m * K.cn[n][m] * ocur[n];
                fc = -o * sm;
                fs = o * cm;
            }
            f(n, m, a * cm, a * sm, tc, ts, fc, fs);
        }
        // shift the columns: m + 1 becomes current, m + 2 is formed
#pragma unroll
        for (int n = 0; n < P + 2; ++n) {
            prev[n] = cur[n];
            cur[n] = nxt[n];
            ocur[n] = onxt[n];
        }
        if (m + 2 <= P) column(m + 2, nxt, onxt);
        else {
#pragma unroll
            for (int n = 0; n < P + 2; ++n) nxt[n] = onxt[n] = 0.0;
        }
    }
}

// Spherical Bessel j_n(x), n = 0..P+1, x >= 0: Miller's backward recursion started where
// the forward recursion from n = P + 2 has grown by 1e20, rescaled on the way down, then
// normalised by j_0 or j_1 (whichever is larger in magnitude), with their series below
// x = 1e-3.
template <int P>
__device__ __forceinline__ void sph_bessel_j(double x, double (&j)[P + 2]) {
    constexpr int len = P + 2;
#pragma unroll
    for (int n = 0; n < len; ++n) j[n] = 0.0;
    if (x == 0.0) {
        j[0] = 1.0;
        return;
    }
    const double ix = 1.0 / x;
    double f0 = 0.0, f1 = 1.0;
    int n = len;
    while (fabs(f1) < 1e20 && n < len + 100000) {
        const double f2 = (2.0 * n + 1.0) * ix * f1 - f0;
        f0 = f1;
        f1 = f2;
        ++n;
    }
    double hi = 0.0, cur = 1e-250;  // f_{m+1}, f_m
    for (int m = n + 1; m > len; --m) {  // down to f_len, nothing stored
        const double lo = (2.0 * m + 1.0) * ix * cur - hi;
        hi = cur;
        cur = lo;
        if (fabs(cur) > 1e200) {
            cur *= 1e-200;
            hi *= 1e-200;
        }
    }
#pragma unroll
    for (int m = len; m >= 1; --m) {
        const double lo = (2.0 * m + 1.0) * ix * cur - hi;
        hi = cur;
        cur = lo;
        j[m - 1] = cur;
        if (fabs(cur) > 1e200) {
            cur *= 1e-200;
            hi *= 1e-200;
#pragma unroll
            for (int k = m - 1; k < len; ++k) j[k] *= 1e-200;
        }
    }
    double j0, j1;
    if (x < 1e-3) {
        const double x2 = x * x;
        j0 = 1.0 - x2 / 6.0 * (1.0 - x2 / 20.0 * (1.0 - x2 / 42.0));
        j1 = x / 3.0 * (1.0 - x2 / 10.0 * (1.0 - x2 / 28.0));
    } else {
        double sx, cx;
        sincos(x, &sx, &cx);
        j0 = sx * ix;
        j1 = sx * ix * ix - cx * ix;
    }
    const double scale = fabs(j0) >= fabs(j1) ? j0 / j[0] : j1 / j[1];
#pragma unroll
    for (int k = 0; k < len; ++k) j[k] *= scale;
}

// The scaled radial functions at z (n = 0..P): jh_n = j_n / s^n and jh_n' = j_n' / s^n;
// with SINGULAR also hh_n = h_n s^n and hh_n' = h_n' s^n, h_n = j_n + i y_n (z > 0):
// j_n' = (n j_{n-1} - (n+1) j_{n+1}) / (2n+1), h_n' = h_{n-1} - (n+1) h_n / z, j_0' = -j_1,
// h_0' = -h_1; y_n upward from its closed forms.
template <int P, bool SINGULAR>
struct HhRadial {
    double jh[P + 1], jhp[P + 1];
    double hr[SINGULAR ? P + 1 : 1], hi[SINGULAR ? P + 1 : 1], hpr[SINGULAR ? P + 1 : 1], hpi[SINGULAR ? P + 1 : 1];
    __device__ __forceinline__ void eval(double z, double s, bool deriv) {
        double j[P + 2];
        sph_bessel_j<P>(z, j);
        double sn = 1.0;
#pragma unroll
        for (int n = 0; n <= P; ++n) {
            const double d = n == 0 ? -j[1] : ((double)n * j[n - 1] - (double)(n + 1) * j[n + 1]) / (2.0 * n + 1.0);
            jh[n] = j[n] / sn;
            jhp[n] = deriv ? d / sn : 0.0;
            sn *= s;
        }
        if constexpr (SINGULAR) {
            double y[P + 2];
            double sz, cz;
            sincos(z, &sz, &cz);
            const double iz = 1.0 / z;
            y[0] = -cz * iz;
            y[1] = -cz * iz * iz - sz * iz;
#pragma unroll
            for (int n = 1; n <= P; ++n) y[n + 1] = (2.0 * n + 1.0) * iz * y[n] - y[n - 1];
            sn = 1.0;
#pragma unroll
            for (int n = 0; n <= P; ++n) {
                hr[n] = j[n] * sn;
                hi[n] = y[n] * sn;
                if (deriv) {
                    const double dr = n == 0 ? -j[1] : j[n - 1] - (double)(n + 1) * j[n] * iz;
                    const double di = n == 0 ? -y[1] : y[n - 1] - (double)(n + 1) * y[n] * iz;
                    hpr[n] = dr * sn;
                    hpi[n] = di * sn;
                }
                sn *= s;
            }
        }
    }
};

// power scale of a box of half-width 1 at wavenumber k_l (level.rs:10-20)
__device__ __forceinline__ double hh_scale(double kl) {
    const double a = 1.7320508075688772 * kl;
    return a < 1.0 ? a : 1.0;
}

// per-level Helmholtz data of an evaluation: k_l of every level (k times the level's
// half-width)
struct HhLevels {
    double kl[32];
};

// ---------------------------------------------------------------------------------
// P2M (rows = leaves, sources of the leaf, unit frame) and P2L (rows = boxes with an X
// list, sources of the X leaves in the box's frame): one warp per row.  Each lane forms
// the harmonics and radial factors of one source into shared memory (B[t][lane], complex
// for P2L), then the lanes add q B over the chunk's 32 sources per coefficient in source
// order, into rows 2v (real) and 2v + 1 (imaginary) of the box's expansion.
// ---------------------------------------------------------------------------------
template <int P, typename T, bool SINGULAR>
__global__ void __launch_bounds__(32) hh_expand_kernel(DevPlan plan, HhLevels lv, int64_t row_begin, int64_t row_end,
                                                       const int32_t* __restrict__ rows, int m,
                                                       const typename Vec4<T>::type* __restrict__ spos,
                                                       const Cplx<T>* __restrict__ sq, T* __restrict__ out) {
    constexpr int NC = nc_of(P), MS = ms_of(P);
    constexpr int NB = SINGULAR ? 2 * NC : NC;  // real base (P2M) or complex base (P2L)
    extern __shared__ unsigned char smem_raw[];
    double* B = reinterpret_cast<double*>(smem_raw);  // [NB][32]
    double* Q = B + NB * 32;                          // [m][2][32]
    const int lane = threadIdx.x;
    const int64_t idx = row_begin + blockIdx.x;
    if (idx >= row_end) return;
    const int64_t row = rows ? rows[idx] : idx;
    int box, nent;
    int64_t ent0;
    if (!SINGULAR) {
        box = plan.leaf_box[row];
        nent = 1;
        ent0 = 0;
        if (plan.src_below[box] == 0) return;
    } else {
        box = (int)row;
        ent0 = plan.x_row[row];
        nent = (int)(plan.x_row[row + 1] - ent0);
        if (nent == 0) return;
    }
    const double kl = lv.kl[plan.level[box]], s = hh_scale(kl);
    const double pik = 4.0 * 3.14159265358979323846 * kl;
    T* outb = out + (int64_t)box * 2 * m * MS;
    for (int e = 0; e < nent; ++e) {
        const int sleaf = SINGULAR ? plan.x_col[ent0 + e] : (int)row;
        double fc[3] = {0.0, 0.0, 0.0}, fr = 1.0;
        if (SINGULAR) rel_frame<double>(plan, box, plan.leaf_box[sleaf], fc, fr);  // (c(t|s), r(t|s))
        const double finv = 1.0 / fr;
        const int64_t s0 = plan.src_start[sleaf], s1 = plan.src_start[sleaf + 1];
        for (int64_t cb = s0; cb < s1; cb += 32) {
            const int64_t si = cb + lane;
            const bool valid = si < s1;
            double x = 0.0, y = 0.0, z = 0.0;
            if (valid) {
                const auto p4 = spos[si];
                x = ((double)p4.x - fc[0]) * finv;
                y = ((double)p4.y - fc[1]) * finv;
                z = ((double)p4.z - fc[2]) * finv;
            }
            for (int v = 0; v < m; ++v) {
                const Cplx<T> q = valid ? sq[(int64_t)v * plan.nsrc + si] : Cplx<T>{T(0), T(0)};
                Q[(2 * v) * 32 + lane] = (double)q.re;
                Q[(2 * v + 1) * 32 + lane] = (double)q.im;
            }
            HhRadial<P, SINGULAR> rad;
            const double rr = sqrt(x * x + y * y + z * z);
            rad.eval(kl * rr, s, false);
            hh_harmonics<P, false>(x, y, z, [&](int n, int mm, double yc, double ys, double, double, double, double) {
                const int tp = n * n + n + mm, tn = n * n + n - mm;
                if (!SINGULAR) {
                    const double w = valid ? rad.jh[n] : 0.0;
                    B[tp * 32 + lane] = w * yc;
                    if (mm) B[tn * 32 + lane] = w * ys;
                } else {
                    // 4 pi i k hh_n Y
                    const double wr = valid ? -pik * rad.hi[n] : 0.0, wi = valid ? pik * rad.hr[n] : 0.0;
                    B[tp * 32 + lane] = wr * yc;
                    B[(NC + tp) * 32 + lane] = wi * yc;
                    if (mm) {
                        B[tn * 32 + lane] = wr * ys;
                        B[(NC + tn) * 32 + lane] = wi * ys;
                    }
                }
            });
            __syncwarp();
            const int cnt = (int)((s1 - cb) < 32 ? (s1 - cb) : 32);
            for (int v = 0; v < m; ++v) {
                const double* qr = Q + (2 * v) * 32;
                const double* qi = Q + (2 * v + 1) * 32;
                for (int t = lane; t < NC; t += 32) {
                    double ar = 0.0, ai = 0.0;
                    if (!SINGULAR) {
                        for (int j = 0; j < cnt; ++j) {
                            const double b = B[t * 32 + j];
                            ar += qr[j] * b;
                            ai += qi[j] * b;
                        }
                    } else {
                        for (int j = 0; j < cnt; ++j) {
                            const double br = B[t * 32 + j], bi = B[(NC + t) * 32 + j];
                            ar += qr[j] * br - qi[j] * bi;
                            ai += qr[j] * bi + qi[j] * br;
                        }
                    }
                    T* o = outb + (int64_t)(2 * v) * MS + t;
                    o[0] = (T)((double)o[0] + ar);
                    o[MS] = (T)((double)o[MS] + ai);
                }
            }
            __syncwarp();
        }
    }
}

// One complex expansion (rows E and E + MS) at one point v of its box's frame:
// phi (re, im) and, with GRAD, the gradient (re x, im x, re y, im y, re z, im z), of
//   sum E jh_n(k |v|) Y(v)                 (regular, a local)
//   4 pi i k sum E hh_n(k |v|) Y(v)        (singular, a multipole).
template <int P, bool GRAD, bool SINGULAR, typename T>
__device__ __forceinline__ void hh_eval(const T* __restrict__ E, double k, double s, double vx, double vy, double vz,
                                        double (&out)[8]) {
    constexpr int NC = nc_of(P), MS = ms_of(P);
    const double d = sqrt(vx * vx + vy * vy + vz * vz);
    HhRadial<P, SINGULAR> rad;
    rad.eval(k * d, s, GRAD);
    // per degree: S_n = sum_m E Y, and with GRAD T_n = sum_m E d_t Y, F_n = sum_m E d_f Y / sin t
    double Sr[P + 1], Si[P + 1], Tr[P + 1], Ti[P + 1], Fr[P + 1], Fi[P + 1];
#pragma unroll
    for (int n = 0; n <= P; ++n) Sr[n] = Si[n] = Tr[n] = Ti[n] = Fr[n] = Fi[n] = 0.0;
    hh_harmonics<P, GRAD>(vx, vy, vz, [&](int n, int mm, double yc, double ys, double tc, double ts, double fc, double fs) {
        const int tp = n * n + n + mm, tn = n * n + n - mm;
        const double er = (double)E[tp], ei = (double)E[MS + tp];
        Sr[n] += er * yc;
        Si[n] += ei * yc;
        if (GRAD) {
            Tr[n] += er * tc;
            Ti[n] += ei * tc;
            Fr[n] += er * fc;
            Fi[n] += ei * fc;
        }
        if (mm) {
            const double nr = (double)E[tn], ni = (double)E[MS + tn];
            Sr[n] += nr * ys;
            Si[n] += ni * ys;
            if (GRAD) {
                Tr[n] += nr * ts;
                Ti[n] += ni * ts;
                Fr[n] += nr * fs;
                Fi[n] += ni * fs;
            }
        }
    });
    (void)NC;
    double f[2] = {0.0, 0.0}, gr[2] = {0.0, 0.0}, gt[2] = {0.0, 0.0}, gf[2] = {0.0, 0.0};
#pragma unroll
    for (int n = 0; n <= P; ++n) {
        double Rr, Ri, Pr, Pi, Ur, Ui;  // value, k * derivative, value / |v|
        if (SINGULAR) {
            Rr = rad.hr[n];
            Ri = rad.hi[n];
            Pr = GRAD ? k * rad.hpr[n] : 0.0;
            Pi = GRAD ? k * rad.hpi[n] : 0.0;
            Ur = Rr / d;
            Ui = Ri / d;
        } else {
            Rr = rad.jh[n];
            Ri = 0.0;
            Pr = k * rad.jhp[n];
            Pi = 0.0;
            Ur = d > 0.0 ? rad.jh[n] / d : (n == 1 ? k / (3.0 * s) : 0.0);
            Ui = 0.0;
        }
        f[0] += Sr[n] * Rr - Si[n] * Ri;
        f[1] += Sr[n] * Ri + Si[n] * Rr;
        if (GRAD) {
            gr[0] += Sr[n] * Pr - Si[n] * Pi;
            gr[1] += Sr[n] * Pi + Si[n] * Pr;
            gt[0] += Tr[n] * Ur - Ti[n] * Ui;
            gt[1] += Tr[n] * Ui + Ti[n] * Ur;
            gf[0] += Fr[n] * Ur - Fi[n] * Ui;
            gf[1] += Fr[n] * Ui + Fi[n] * Ur;
        }
    }
    out[0] = f[0];
    out[1] = f[1];
#pragma unroll
    for (int a = 2; a < 8; ++a) out[a] = 0.0;
    if (GRAD) {
        const double rho = sqrt(vx * vx + vy * vy);
        const double ct = d > 0.0 ? vz / d : 1.0, st = d > 0.0 ? rho / d : 0.0;
        const double cf = rho > 0.0 ? vx / rho : 1.0, sf = rho > 0.0 ? vy / rho : 0.0;
        const double er[3] = {st * cf, st * sf, ct}, et[3] = {ct * cf, ct * sf, -st}, ef[3] = {-sf, cf, 0.0};
        if (d > 0.0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                out[2 + 2 * a] = gr[0] * er[a] + gt[0] * et[a] + gf[0] * ef[a];
                out[3 + 2 * a] = gr[1] * er[a] + gt[1] * et[a] + gf[1] * ef[a];
            }
        } else if (P >= 1) {  // at the centre of a local: the gradient of its degree-1 part
            const double g = 0.4886025119029199 * k / (3.0 * s);  // sqrt(3 / (4 pi)) k / (3 s)
            const int slot[3] = {3, 1, 2};                         // idx(1, 1), idx(1, -1), idx(1, 0): x, y, z
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                out[2 + 2 * a] = g * (double)E[slot[a]];
                out[3 + 2 * a] = g * (double)E[MS + slot[a]];
            }
        }
    }
    if (SINGULAR) {  // times 4 pi i k
        const double pik = 4.0 * 3.14159265358979323846 * k;
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
            const double re = out[i], im = out[i + 1];
            out[i] = -pik * im;
            out[i + 1] = pik * re;
        }
    }
}

// L2P (the leaf's own local, unit frame) and M2P (its W list, by box index) for every
// target of a leaf: a block per leaf, a thread per target.  Partials in f64 complex:
// far_phi [v][t][2], far_g [v][t][6] (leaf order), overwritten.
template <int P, typename T, bool GRAD>
__global__ void __launch_bounds__(128) hh_leaf_far_kernel(DevPlan plan, HhLevels lv, int64_t leaf0, int m,
                                                         const typename Vec4<T>::type* __restrict__ tpos,
                                                         const T* __restrict__ M, const T* __restrict__ Lc,
                                                         double* __restrict__ far_phi, double* __restrict__ far_g) {
    constexpr int MS = ms_of(P);
    const int64_t leaf = leaf0 + blockIdx.x;
    const int box = plan.leaf_box[leaf];
    const int64_t t0 = plan.tgt_start[leaf], t1 = plan.tgt_start[leaf + 1];
    if (t1 == t0) return;
    const int64_t w0 = plan.w_row[leaf], w1 = plan.w_row[leaf + 1];
    const int64_t nt = plan.ntgt;
    const double kt = lv.kl[plan.level[box]], st = hh_scale(kt);
    for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        const auto p4 = tpos[t];
        const double ux = (double)p4.x, uy = (double)p4.y, uz = (double)p4.z;
        for (int v = 0; v < m; ++v) {
            double acc[8];
            hh_eval<P, GRAD, false, T>(Lc + ((int64_t)box * 2 * m + 2 * v) * MS, kt, st, ux, uy, uz, acc);
            for (int64_t e = w0; e < w1; ++e) {
                const int sb = plan.w_col[e];
                double c[3], r;
                rel_frame<double>(plan, sb, box, c, r);
                const double rinv = 1.0 / r;
                const double ks = lv.kl[plan.level[sb]];
                double o[8];
                hh_eval<P, GRAD, true, T>(M + ((int64_t)sb * 2 * m + 2 * v) * MS, ks, hh_scale(ks),
                                          (ux - c[0]) * rinv, (uy - c[1]) * rinv, (uz - c[2]) * rinv, o);
                acc[0] += o[0] * rinv;
                acc[1] += o[1] * rinv;
                if (GRAD)
                    for (int a = 2; a < 8; ++a) acc[a] += o[a] * rinv * rinv;
            }
            double* fp = far_phi + 2 * ((int64_t)v * nt + t);
            fp[0] = acc[0];
            fp[1] = acc[1];
            if (GRAD) {
                double* fg = far_g + 6 * ((int64_t)v * nt + t);
                for (int a = 0; a < 6; ++a) fg[a] = acc[2 + a];
            }
        }
    }
}

// The locals of one level from the tensor-core complex M2L's products (f32): for every box
// with a target below it and every vector v,
//   L_re = (L2L part) + sum_V (A_r x_re - A_i x_im),  L_im = (L2L part) + sum_V (A_i x_re + A_r x_im)
// with a pair's products Y[pos][2v + c][0..n) = A_r x_c and [128..128+n) = A_i x_c (row
// stride 256), V entries in row order; the L2L part (with_l2l) from the SIMT complex GEMM's
// rows 2v, 2v + 1 of stride ys_of(P).  Block per box, thread per slot.
template <int P>
__global__ void hh_local_reduce_tc_kernel(DevPlan plan, int64_t b0, int64_t b1, int m, int with_l2l,
                                          const float* __restrict__ Yo, const float* __restrict__ Yv,
                                          const int64_t* __restrict__ vpos, float* __restrict__ L) {
    constexpr int NC = nc_of(P), YS = ys_of(P), MS = ms_of(P);
    const int64_t b = b0 + blockIdx.x;
    if (b >= b1 || plan.tgt_below[b] == 0) return;
    const int64_t e0 = plan.v_row[b], e1 = plan.v_row[b + 1];
    for (int v = 0; v < m; ++v)
        for (int t = threadIdx.x; t < NC; t += blockDim.x) {
            float sr = 0.0f, si = 0.0f;
            if (with_l2l) {
                sr = Yo[((int64_t)b * 2 * m + 2 * v) * YS + t];
                si = Yo[((int64_t)b * 2 * m + 2 * v + 1) * YS + t];
            }
            for (int64_t e = e0; e < e1; ++e) {
                const float* y = Yv + (vpos[e] * 2 * m + 2 * v) * 256;
                const float rr = __ldcs(y + t), ir = __ldcs(y + 128 + t);        // A_r x_re, A_i x_re
                const float ri = __ldcs(y + 256 + t), ii = __ldcs(y + 384 + t);  // A_r x_im, A_i x_im
                sr += rr - ii;
                si += ir + ri;
            }
            L[((int64_t)b * 2 * m + 2 * v) * MS + t] = sr;
            L[((int64_t)b * 2 * m + 2 * v + 1) * MS + t] = si;
        }
}

}  // namespace fmmb
