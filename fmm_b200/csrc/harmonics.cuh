// Solid harmonics evaluated degree by degree in registers (CONVENTIONS 3.5 of the
// reference: fmm-math/src/harmonics.rs:118-187 defines the same recursions, there
// m-major into a full array).  Degree n is formed from degrees n-1 and n-2 only, so
// a kernel holds two rows of (P+2) complex values and consumes each row as it is made:
// P2M/P2L scatter it into coefficient slots, L2P/M2P contract it with coefficients.
#pragma once

#include <cuda_runtime.h>

namespace fmmb {

__host__ __device__ constexpr int nc_of(int p) { return (p + 1) * (p + 1); }
// row stride of the translation products (Y, Yo): (p+1)^2 rounded up to whole 16-byte
// groups of f32, as the expansions' rows, so that the rows of a tile are one contiguous
// run with no padding to write and read back (measured: 32-slot rows cost 12 % more of
// the product traffic at p = 8)
__host__ __device__ constexpr int ys_of(int p) { return ((nc_of(p) + 3) / 4) * 4; }
// row stride of one expansion (one box, one vector) in the multipole and local arrays:
// (p+1)^2 rounded up to whole 16-byte groups in f32, so that every row starts on a
// 16-byte boundary (the tensor-memory-access gathers of the tensor-core M2L need it)
__host__ __device__ constexpr int ms_of(int p) { return ((nc_of(p) + 3) / 4) * 4; }
__host__ __device__ constexpr int slot(int n, int m) { return n * n + n + m; }

template <typename T>
struct Cx {
    T re, im;
};

// Row recursion state for the regular harmonics R_n^m, m = 0..n.
template <int PMAX, typename T>
struct RegularRows {
    T x, y, z, r2;
    T pre[PMAX + 2], pim[PMAX + 2];    // row n - 1
    T ppre[PMAX + 2], ppim[PMAX + 2];  // row n - 2
    T cre[PMAX + 2], cim[PMAX + 2];    // row n
    __device__ __forceinline__ void init(T x_, T y_, T z_) {
        x = x_;
        y = y_;
        z = z_;
        r2 = x * x + y * y + z * z;
    }
    // forms row n into (cre, cim); rows must be formed in order n = 0, 1, 2, ...
    __device__ __forceinline__ void step(int n) {
#pragma unroll
        for (int m = 0; m <= PMAX + 1; ++m) {
            ppre[m] = pre[m];
            ppim[m] = pim[m];
            pre[m] = cre[m];
            pim[m] = cim[m];
        }
        if (n == 0) {
            cre[0] = T(1);
            cim[0] = T(0);
            return;
        }
#pragma unroll
        for (int m = 0; m <= PMAX + 1; ++m) {
            if (m + 2 <= n) {
                T den = T((n + m) * (n - m));
                T c1 = T(2 * n - 1) * z / den, c2 = -r2 / den;
                cre[m] = c1 * pre[m] + c2 * ppre[m];
                cim[m] = c1 * pim[m] + c2 * ppim[m];
            } else if (m + 1 == n) {
                cre[m] = z * pre[m];
                cim[m] = z * pim[m];
            } else if (m == n) {
                T s = T(1) / T(2 * n);
                T a = pre[n - 1], b = pim[n - 1];
                cre[m] = (x * a - y * b) * s;
                cim[m] = (x * b + y * a) * s;
            }
        }
    }
};

// Row recursion state for the irregular harmonics I_n^m, m = 0..n.
template <int PMAX, typename T>
struct IrregularRows {
    T x, y, z, inv_r2, inv_r;
    T pre[PMAX + 3], pim[PMAX + 3];
    T ppre[PMAX + 3], ppim[PMAX + 3];
    T cre[PMAX + 3], cim[PMAX + 3];
    __device__ __forceinline__ void init(T x_, T y_, T z_, T inv_r_) {
        x = x_;
        y = y_;
        z = z_;
        inv_r = inv_r_;
        inv_r2 = inv_r * inv_r;
    }
    __device__ __forceinline__ void step(int n) {
#pragma unroll
        for (int m = 0; m <= PMAX + 2; ++m) {
            ppre[m] = pre[m];
            ppim[m] = pim[m];
            pre[m] = cre[m];
            pim[m] = cim[m];
        }
        if (n == 0) {
            cre[0] = inv_r;
            cim[0] = T(0);
            return;
        }
#pragma unroll
        for (int m = 0; m <= PMAX + 2; ++m) {
            if (m + 2 <= n) {
                T c1 = T(2 * n - 1) * z * inv_r2;
                T c2 = -T((n - 1 - m) * (n - 1 + m)) * inv_r2;
                cre[m] = c1 * pre[m] + c2 * ppre[m];
                cim[m] = c1 * pim[m] + c2 * ppim[m];
            } else if (m + 1 == n) {
                T c = T(2 * n - 1) * z * inv_r2;
                cre[m] = c * pre[m];
                cim[m] = c * pim[m];
            } else if (m == n) {
                T s = T(2 * n - 1) * inv_r2;
                T a = pre[n - 1], b = pim[n - 1];
                cre[m] = (x * a - y * b) * s;
                cim[m] = (x * b + y * a) * s;
            }
        }
    }
};

// coefficient of degree n, stored order m >= 0, from real storage (zero beyond degree)
template <typename T>
__device__ __forceinline__ Cx<T> coef_at(const T* c, int n, int m) {
    Cx<T> z;
    if (m < 0 || m > n || n < 0) {
        z.re = T(0);
        z.im = T(0);
        return z;
    }
    z.re = c[slot(n, m)];
    z.im = m ? c[slot(n, -m)] : T(0);
    return z;
}

}  // namespace fmmb
