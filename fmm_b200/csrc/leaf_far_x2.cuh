// L2P and M2P with gradients for the mixed form on the packed f32x2 pipe of sm_100
// (FFMA2 / FADD2 / FMUL2): the sums of l2p_eval / m2p_eval (kernels.cuh) taken
// coefficient by coefficient, each complex harmonic one float2 (re, im).
//
// l2p_eval / m2p_eval visit the harmonics and, for each, read the coefficients of the
// potential and of the ladder identities.  Taken per coefficient c = (a, b) of degree n and
// order mu instead, the same terms are
//   potential        w Re(c H)            H the harmonic of (n, mu)
//   d/dz             w Re(c W)            W the harmonic of (n -+ 1, mu)      (M2P: minus)
//   d/dx - i d/dy    c U - conj(c V)      U, V the harmonics of (n -+ 1, mu -+ 1)
// with w = 1 for mu = 0 and 2 otherwise, L2P taking the row below (n - 1) and M2P the row
// above (n + 1): the ladder terms of l2p_eval (up, the coefficient of (k + 1, mu + 1), and
// dn, that of (k + 1, mu - 1), with R_k^mu) and of m2p_eval (those of (k - 1, mu +- 1) with
// I_k^mu), re-indexed by coefficient.  With S = U - V and T = U + V,
//   Re(c U - conj(c V)) = a S.re - b S.im,   Im(c U - conj(c V)) = a T.im + b T.re,
// so a coefficient costs four packed fused multiply-adds ((a, b) times H, W and S, (b, a)
// times T, into float2 sums whose real and imaginary products are summed apart) and S, T
// two packed adds; the harmonic rows come from the recursions of RegularRows /
// IrregularRows with both parts in one packed instruction.  The terms are those of
// l2p_eval / m2p_eval; the order of the f32 additions differs.
#pragma once

#include <cuda_runtime.h>

#include "harmonics.cuh"

namespace fmmb {

__device__ __forceinline__ float2 x2(float a) { return make_float2(a, a); }

// The row recursions of RegularRows / IrregularRows (harmonics.cuh) in f32 with both parts
// of a harmonic in one packed instruction and the recursion's constants folded at compile
// time (a multiplication by 1 / ((n + m)(n - m)), no division): step(n) forms row n into
// c (m = 0..n), keeping rows n - 1 (pr) and n - 2 (pp); rows in order n = 0, 1, 2, ...
template <int PMAX>
struct RegularRows2 {
    float x, y, z;
    float2 nr2;
    float2 pp[PMAX + 2], pr[PMAX + 2], c[PMAX + 2];  // one spare slot
    __device__ __forceinline__ void init(float x_, float y_, float z_) {
        x = x_;
        y = y_;
        z = z_;
        nr2 = x2(-(x * x + y * y + z * z));
    }
    __device__ __forceinline__ void step(int n) {
#pragma unroll
        for (int m = 0; m < n; ++m) {
            pp[m] = pr[m];
            pr[m] = c[m];
        }
        if (n == 0) {
            c[0] = make_float2(1.0f, 0.0f);
            return;
        }
        const float2 zn = x2((float)(2 * n - 1) * z);
#pragma unroll
        for (int m = 0; m <= n; ++m) {
            if (m + 2 <= n) {
                // R_n^m = ((2n - 1) z R_{n-1}^m - r^2 R_{n-2}^m) / ((n + m)(n - m))
                const float inv_den = 1.0f / (float)((n + m) * (n - m));
                c[m] = __fmul2_rn(x2(inv_den), __ffma2_rn(zn, pr[m], __fmul2_rn(nr2, pp[m])));
            } else if (m + 1 == n) {
                c[m] = __fmul2_rn(x2(z), pr[m]);
            } else {
                const float sc = 1.0f / (float)(2 * n);
                const float a = pr[n - 1].x, b = pr[n - 1].y;
                c[m] = make_float2((x * a - y * b) * sc, (x * b + y * a) * sc);
            }
        }
    }
};

template <int PMAX>
struct IrregularRows2 {
    float x, y, z, inv_r, inv_r2;
    float2 ir2;
    float2 pp[PMAX + 2], pr[PMAX + 2], c[PMAX + 2];
    __device__ __forceinline__ void init(float x_, float y_, float z_, float inv_r_) {
        x = x_;
        y = y_;
        z = z_;
        inv_r = inv_r_;
        inv_r2 = inv_r * inv_r;
        ir2 = x2(inv_r2);
    }
    __device__ __forceinline__ void step(int n) {
#pragma unroll
        for (int m = 0; m < n; ++m) {
            pp[m] = pr[m];
            pr[m] = c[m];
        }
        if (n == 0) {
            c[0] = make_float2(inv_r, 0.0f);
            return;
        }
        // I_n^m = ((2n - 1) z I_{n-1}^m - (n - 1 - m)(n - 1 + m) I_{n-2}^m) / r^2
        const float2 zn = x2((float)(2 * n - 1) * z);
#pragma unroll
        for (int m = 0; m <= n; ++m) {
            if (m + 2 <= n) {
                const float2 k2 = x2(-(float)((n - 1 - m) * (n - 1 + m)));
                c[m] = __fmul2_rn(ir2, __ffma2_rn(zn, pr[m], __fmul2_rn(k2, pp[m])));
            } else if (m + 1 == n) {
                c[m] = __fmul2_rn(ir2, __fmul2_rn(zn, pr[m]));
            } else {
                const float sc = (float)(2 * n - 1) * inv_r2;
                const float a = pr[n - 1].x, b = pr[n - 1].y;
                c[m] = make_float2((x * a - y * b) * sc, (x * b + y * a) * sc);
            }
        }
    }
};

// The sums of one evaluation; the orders mu > 0 weighted 2 at the end.
struct LadderSums {
    float f0 = 0.0f, d0 = 0.0f, gxs = 0.0f, gys = 0.0f;  // mu = 0 (b = 0, H and W real)
    float2 f1 = make_float2(0.0f, 0.0f), d1 = make_float2(0.0f, 0.0f);
    float2 sa = make_float2(0.0f, 0.0f), tb = make_float2(0.0f, 0.0f);

    // coefficient (a, b) of order mu with harmonics H (potential), W (d/dz) and U, V (the
    // ladder); HAS_*: that harmonic exists for this coefficient
    template <bool MU0, bool HAS_W, bool HAS_U, bool HAS_V>
    __device__ __forceinline__ void add(float a, float b, float2 H, float2 W, float2 U, float2 V) {
        float2 S = make_float2(0.0f, 0.0f), T = make_float2(0.0f, 0.0f);
        if (HAS_U && HAS_V) {
            S = __ffma2_rn(V, x2(-1.0f), U);
            T = __fadd2_rn(U, V);
        } else if (HAS_U) {
            S = U;
            T = U;
        } else if (HAS_V) {
            S = make_float2(-V.x, -V.y);
            T = V;
        }
        if (MU0) {
            f0 = fmaf(a, H.x, f0);
            if (HAS_W) d0 = fmaf(a, W.x, d0);
            if (HAS_U || HAS_V) {
                gxs = fmaf(a, S.x, gxs);
                gys = fmaf(a, T.y, gys);
            }
        } else {
            const float2 ab = make_float2(a, b);
            f1 = __ffma2_rn(ab, H, f1);
            if (HAS_W) d1 = __ffma2_rn(ab, W, d1);
            if (HAS_U || HAS_V) {
                sa = __ffma2_rn(ab, S, sa);
                tb = __ffma2_rn(make_float2(b, a), T, tb);
            }
        }
    }
    __device__ __forceinline__ void finish(float dz_sign, float& phi, float& gx, float& gy, float& gz) const {
        phi = f0 + 2.0f * (f1.x - f1.y);
        gz = dz_sign * (d0 + 2.0f * (d1.x - d1.y));
        gx = gxs + (sa.x - sa.y);
        gy = -(gys + (tb.x + tb.y));
    }
};

// L2P with gradients at (x, y, z) in the box's unit frame; L the local (real storage)
template <int P>
__device__ __forceinline__ void l2p_x2(const float* __restrict__ L, float x, float y, float z, float& phi,
                                       float& gx, float& gy, float& gz) {
    const float2 zero = make_float2(0.0f, 0.0f);
    RegularRows2<P> h;
    h.init(x, y, z);
    LadderSums s;
#pragma unroll
    for (int n = 0; n <= P; ++n) {
        h.step(n);
        // the coefficients of degree n: H = R_n^mu, W = R_{n-1}^mu, U = R_{n-1}^{mu-1},
        // V = R_{n-1}^{mu+1}
#pragma unroll
        for (int mu = 0; mu <= n; ++mu) {
            const float a = L[slot(n, mu)], b = mu ? L[slot(n, -mu)] : 0.0f;
            const float2 W = mu <= n - 1 ? h.pr[mu] : zero;
            const float2 U = mu >= 1 ? h.pr[mu >= 1 ? mu - 1 : 0] : zero;
            const float2 V = mu + 1 <= n - 1 ? h.pr[mu + 1] : zero;
            if (mu == 0) {
                if (n >= 2)
                    s.add<true, true, false, true>(a, b, h.c[0], W, U, V);
                else if (n == 1)
                    s.add<true, true, false, false>(a, b, h.c[0], W, U, V);
                else
                    s.add<true, false, false, false>(a, b, h.c[0], W, U, V);
            } else if (mu + 1 <= n - 1) {
                s.add<false, true, true, true>(a, b, h.c[mu], W, U, V);
            } else if (mu <= n - 1) {
                s.add<false, true, true, false>(a, b, h.c[mu], W, U, V);
            } else {
                s.add<false, false, true, false>(a, b, h.c[mu], W, U, V);
            }
        }
    }
    s.finish(1.0f, phi, gx, gy, gz);
}

// M2P with gradients at (x, y, z) in the source box's unit frame; M the multipole
template <int P>
__device__ __forceinline__ void m2p_x2(const float* __restrict__ M, float x, float y, float z, float& phi,
                                       float& gx, float& gy, float& gz) {
    constexpr int K = P + 1;
    const float2 zero = make_float2(0.0f, 0.0f);
    IrregularRows2<K> h;
    h.init(x, y, z, 1.0f / sqrtf(x * x + y * y + z * z));
    LadderSums s;
#pragma unroll
    for (int n = 0; n <= K; ++n) {
        h.step(n);
        if (n == 0) continue;
        // the coefficients of degree d = n - 1: H = I_d^mu, W = I_n^mu, U = I_n^{mu-1},
        // V = I_n^{mu+1}
        const int d = n - 1;
#pragma unroll
        for (int mu = 0; mu <= d; ++mu) {
            const float a = M[slot(d, mu)], b = mu ? M[slot(d, -mu)] : 0.0f;
            if (mu == 0)
                s.add<true, true, false, true>(a, b, h.pr[0], h.c[0], zero, h.c[1]);
            else
                s.add<false, true, true, true>(a, b, h.pr[mu], h.c[mu], h.c[mu - 1], h.c[mu + 1]);
        }
    }
    s.finish(-1.0f, phi, gx, gy, gz);
}

}  // namespace fmmb
