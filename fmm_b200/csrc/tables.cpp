// Operator tables in f64 (CONVENTIONS 3.11-3.12 of the reference): each table column
// is the translation of a unit coefficient vector at the canonical frames
//   M2M(o): child (s_o/2, 1/2) -> parent (0, 1);  L2L(o): parent -> child;
//   M2L(d): source (0, 1) -> target (2d, 1), d the 316 V-list offsets in index order,
// as fmm-tables/src/m2l.rs:67-96 and octant.rs:150-174 define them.  The translations
// are evaluated with the real-storage order sums of CONVENTIONS 3.11 "Real storage"
// (stored orders m >= 0 of the input only), in complex arithmetic on (re, im) pairs.
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

#include "plan.hpp"

namespace fmmb {

namespace {

struct cd {
    double re, im;
};
inline cd operator*(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cd operator+(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
inline cd conj(cd a) { return {a.re, -a.im}; }
inline cd scale(cd a, double s) { return {a.re * s, a.im * s}; }

inline int idx(int n, int m) { return n * n + n + m; }

// complex harmonic values X_n^m, m >= 0, held as (re, im) per (n, m)
struct Harm {
    int p;
    std::vector<cd> v;  // (p+1)(p+2)/2 entries, n-major
    explicit Harm(int p_) : p(p_), v((p_ + 1) * (p_ + 2) / 2) {}
    cd& at(int n, int m) { return v[n * (n + 1) / 2 + m]; }
    // any order q, from the (-1)^q conjugate rule; zero beyond the degree
    cd get(int n, int q) {
        int m = q < 0 ? -q : q;
        if (m > n) return {0.0, 0.0};
        cd z = at(n, m);
        if (q < 0) {
            z = conj(z);
            if (m & 1) z = scale(z, -1.0);
        }
        return z;
    }
};

// Cartesian recursions of CONVENTIONS 3.5
void regular(Harm& h, double x, double y, double z) {
    int p = h.p;
    double r2 = x * x + y * y + z * z;
    cd diag{1.0, 0.0};
    for (int m = 0; m <= p; ++m) {
        if (m > 0) {
            double s = 1.0 / (2.0 * m);
            diag = {(x * diag.re - y * diag.im) * s, (x * diag.im + y * diag.re) * s};
        }
        h.at(m, m) = diag;
        if (m == p) break;
        h.at(m + 1, m) = {z * diag.re, z * diag.im};
        for (int n = m + 2; n <= p; ++n) {
            double den = (double)((n + m) * (n - m));
            double c1 = (2.0 * n - 1.0) * z / den, c2 = -r2 / den;
            cd a = h.at(n - 1, m), b = h.at(n - 2, m);
            h.at(n, m) = {c1 * a.re + c2 * b.re, c1 * a.im + c2 * b.im};
        }
    }
}

void irregular(Harm& h, double x, double y, double z) {
    int p = h.p;
    double r2 = x * x + y * y + z * z, inv = 1.0 / r2;
    cd diag{1.0 / std::sqrt(r2), 0.0};
    for (int m = 0; m <= p; ++m) {
        if (m > 0) {
            double s = (2.0 * m - 1.0) * inv;
            diag = {(x * diag.re - y * diag.im) * s, (x * diag.im + y * diag.re) * s};
        }
        h.at(m, m) = diag;
        if (m == p) break;
        double c = (2.0 * m + 1.0) * z * inv;
        h.at(m + 1, m) = {c * diag.re, c * diag.im};
        for (int n = m + 2; n <= p; ++n) {
            double c1 = (2.0 * n - 1.0) * z * inv, c2 = -(double)((n - 1 - m) * (n - 1 + m)) * inv;
            cd a = h.at(n - 1, m), b = h.at(n - 2, m);
            h.at(n, m) = {c1 * a.re + c2 * b.re, c1 * a.im + c2 * b.im};
        }
    }
}

// input coefficient of degree n, stored order m >= 0
inline cd coef(const double* c, int n, int m) { return {c[idx(n, m)], m ? c[idx(n, -m)] : 0.0}; }

inline void add_out(double* out, int j, int i, cd v) {
    out[idx(j, i)] += v.re;
    if (i > 0) out[idx(j, -i)] += v.im;
}

// M2M (CONVENTIONS 3.11): M'_j^i = sum_k rho^k sum_l M_k^l conj R_{j-k}^{i-l}(b),
// the order sum over stored l >= 0: A^0 B^i + sum_l>=1 (A^l B^{i-l} + (-1)^l conj(A^l) B^{i+l})
void m2m(int p, const double b[3], double rho, const double* in, double* out) {
    Harm R(p);
    regular(R, b[0], b[1], b[2]);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cd sum{0.0, 0.0};
            double rk = 1.0;
            for (int k = 0; k <= j; ++k) {
                cd s = coef(in, k, 0) * conj(R.get(j - k, i));
                for (int l = 1; l <= k; ++l) {
                    cd A = coef(in, k, l);
                    cd t1 = A * conj(R.get(j - k, i - l));
                    cd t2 = scale(conj(A) * conj(R.get(j - k, i + l)), (l & 1) ? -1.0 : 1.0);
                    s = s + t1 + t2;
                }
                sum = sum + scale(s, rk);
                rk *= rho;
            }
            add_out(out, j, i, sum);
        }
}

// L2L: L'_j^i = sigma^{j+1} sum_{n>=j} sum_m L_n^m R_{n-j}^{m-i}(t)
// order sum: A^0 B^{-i} + sum_m>=1 (A^m B^{m-i} + (-1)^m conj(A^m) B^{-m-i})
void l2l(int p, const double t[3], double sigma, const double* in, double* out) {
    Harm R(p);
    regular(R, t[0], t[1], t[2]);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cd sum{0.0, 0.0};
            for (int n = j; n <= p; ++n) {
                cd s = coef(in, n, 0) * R.get(n - j, -i);
                for (int m = 1; m <= n; ++m) {
                    cd A = coef(in, n, m);
                    s = s + A * R.get(n - j, m - i) +
                        scale(conj(A) * R.get(n - j, -m - i), (m & 1) ? -1.0 : 1.0);
                }
                sum = sum + s;
            }
            add_out(out, j, i, scale(sum, std::pow(sigma, j + 1)));
        }
}

// M2L: L'_j^i = (-1)^{j+i} sigma^{j+1} sum_n sum_m M_n^m I_{n+j}^{m-i}(b)
void m2l(int p, const double b[3], double sigma, const double* in, double* out) {
    Harm I(2 * p);
    irregular(I, b[0], b[1], b[2]);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= j; ++i) {
            cd sum{0.0, 0.0};
            for (int n = 0; n <= p; ++n) {
                cd s = coef(in, n, 0) * I.get(n + j, -i);
                for (int m = 1; m <= n; ++m) {
                    cd A = coef(in, n, m);
                    s = s + A * I.get(n + j, m - i) +
                        scale(conj(A) * I.get(n + j, -m - i), (m & 1) ? -1.0 : 1.0);
                }
                sum = sum + s;
            }
            double sign = ((j + i) & 1) ? -1.0 : 1.0;
            add_out(out, j, i, scale(sum, sign * std::pow(sigma, j + 1)));
        }
}

// The tables are independent (each writes its own nc x nc slice), so they are built in
// chunks on host threads: the same values for any number of threads.
template <class F>
void build(int p, int count, std::vector<double>& out, F&& apply) {
    int nc = (p + 1) * (p + 1);
    out.assign((size_t)count * nc * nc, 0.0);
    const size_t nth = std::max<size_t>(1, std::min<size_t>({std::thread::hardware_concurrency(), 16, (size_t)count}));
    std::vector<std::vector<double>> units(nth, std::vector<double>(nc, 0.0));  // allocated here, not in a thread
    for_chunks((size_t)count, nth, [&](size_t c, size_t t0, size_t t1) {
        std::vector<double>& unit = units[c];
        for (size_t t = t0; t < t1; ++t)
            for (int k = 0; k < nc; ++k) {
                unit[k] = 1.0;
                apply((int)t, unit.data(), out.data() + (t * nc + k) * nc);
                unit[k] = 0.0;
            }
    });
}

inline void octant_half(int o, double c[3]) {
    c[0] = ((o >> 2) & 1) ? 0.5 : -0.5;
    c[1] = ((o >> 1) & 1) ? 0.5 : -0.5;
    c[2] = (o & 1) ? 0.5 : -0.5;
}

}  // namespace

void build_m2l_tables(int p, std::vector<double>& out) {
    std::vector<int> off;
    for (int x = -3; x <= 3; ++x)
        for (int y = -3; y <= 3; ++y)
            for (int z = -3; z <= 3; ++z)
                if (offset_index(x, y, z) >= 0) {
                    off.push_back(x);
                    off.push_back(y);
                    off.push_back(z);
                }
    build(p, 316, out, [&](int t, const double* in, double* col) {
        // source frame (0, 1), target (2d, 1): b = (c' - c)/r = 2d, sigma = 1
        double b[3] = {2.0 * off[3 * t], 2.0 * off[3 * t + 1], 2.0 * off[3 * t + 2]};
        m2l(p, b, 1.0, in, col);
    });
}

void build_m2m_tables(int p, std::vector<double>& out) {
    build(p, 8, out, [&](int o, const double* in, double* col) {
        // child (s_o/2, 1/2) -> parent (0, 1): b = (c - c')/r' = s_o/2, rho = 1/2
        double b[3];
        octant_half(o, b);
        m2m(p, b, 0.5, in, col);
    });
}

void build_l2l_tables(int p, std::vector<double>& out) {
    build(p, 8, out, [&](int o, const double* in, double* col) {
        // parent (0, 1) -> child (s_o/2, 1/2): t = (c' - c)/r = s_o/2, sigma = 1/2
        double t[3];
        octant_half(o, t);
        l2l(p, t, 0.5, in, col);
    });
}

}  // namespace fmmb
