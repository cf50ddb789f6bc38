/*
 * Oracle side (test infrastructure and the timed CPU baseline only): the two kernels of the
 * reference's host path that differ from its trusted scalar operators, restated so the CPU
 * baseline times what the reference's LaplaceOperator runs on x86_64 with AVX-512F:
 *
 *  - the P2P of nd-fmm-simd on AVX-512 (fmm-simd/src/lib.rs:56-79, the table there;
 *    fmm-simd/src/arch/avx512.rs:1-40): targets in vector lanes, two vectors of 8 f64
 *    targets a block (K = 2), each source broadcast and visited in input order; per pair
 *    and lane d = x - y, r^2 = fma(d2, d2, fma(d1, d1, d0 d0)), rho = 1/sqrt(r^2) from the
 *    estimate vrsqrt14pd and two Newton steps y <- y + y (1/2 - h y^2) with h = r^2 / 2,
 *    cleared to +0 where r^2 = 0; phi += q rho and, with gradients, grad -= ((q rho) rho^2) d.
 *    The last partial block runs on a copy padded with the last target.  Each term is within
 *    8 u (potential) and 16 u (gradient) of the scalar loop's (fmm-simd/src/lib.rs:103-109),
 *    so sums agree with orc_p2p to rounding, not bit for bit.  Without AVX-512F the exact
 *    loop of orc_p2p runs.
 *  - the batched M2L (fmm-exec/src/operator.rs:417-419, M2L_BLOCK_TARGETS = 64;
 *    fmm-simd/src/matrix.rs:95-200, MatrixKernel::accumulate_columns in its Separate
 *    mode): the targets of a level in blocks of 64 consecutive boxes; within a block, for
 *    each offset index in turn, the columns C[:, t] += A_d M[:, s] of its pairs, four
 *    columns at a time so each column of A_d is read once per four; every element adds
 *    its terms with k ascending, a product and a sum rounded apart, so the result is that
 *    of the matrix-vector loop bit for bit (orc_matvec).
 */
#include <immintrin.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "fmm_oracle.h"

__attribute__((target("avx512f,fma"))) static void p2p_avx512(size_t ns, const double *src, const double *q, size_t nt,
                                                              const double *tx, const double *ty, const double *tz,
                                                              double *ph, double *g0, double *g1, double *g2,
                                                              int grad) {
    const __m512d half = _mm512_set1_pd(0.5), zero = _mm512_setzero_pd();
    for (size_t b = 0; b < nt; b += 16) {
        double lx[16], ly[16], lz[16], lp[16], l0[16], l1[16], l2[16];
        const size_t cnt = nt - b < 16 ? nt - b : 16;
        for (size_t i = 0; i < 16; ++i) {
            const size_t s = b + (i < cnt ? i : cnt - 1);  /* the tail padded with the last target */
            lx[i] = tx[s];
            ly[i] = ty[s];
            lz[i] = tz[s];
            lp[i] = ph[s];
            l0[i] = g0[s];
            l1[i] = g1[s];
            l2[i] = g2[s];
        }
        __m512d x[2], y[2], z[2], p[2], a0[2], a1[2], a2[2];
        for (int v = 0; v < 2; ++v) {
            x[v] = _mm512_loadu_pd(lx + 8 * v);
            y[v] = _mm512_loadu_pd(ly + 8 * v);
            z[v] = _mm512_loadu_pd(lz + 8 * v);
            p[v] = _mm512_loadu_pd(lp + 8 * v);
            a0[v] = _mm512_loadu_pd(l0 + 8 * v);
            a1[v] = _mm512_loadu_pd(l1 + 8 * v);
            a2[v] = _mm512_loadu_pd(l2 + 8 * v);
        }
        for (size_t j = 0; j < ns; ++j) {
            const __m512d sx = _mm512_set1_pd(src[3 * j]), sy = _mm512_set1_pd(src[3 * j + 1]),
                          sz = _mm512_set1_pd(src[3 * j + 2]), sq = _mm512_set1_pd(q[j]);
            for (int v = 0; v < 2; ++v) {
                const __m512d d0 = _mm512_sub_pd(x[v], sx), d1 = _mm512_sub_pd(y[v], sy), d2 = _mm512_sub_pd(z[v], sz);
                const __m512d r2 = _mm512_fmadd_pd(d2, d2, _mm512_fmadd_pd(d1, d1, _mm512_mul_pd(d0, d0)));
                const __mmask8 coincident = _mm512_cmp_pd_mask(r2, zero, _CMP_EQ_OQ);
                const __m512d h = _mm512_mul_pd(r2, half);
                __m512d rho = _mm512_rsqrt14_pd(r2);
                __m512d e = _mm512_fnmadd_pd(h, _mm512_mul_pd(rho, rho), half);
                rho = _mm512_fmadd_pd(rho, e, rho);
                e = _mm512_fnmadd_pd(h, _mm512_mul_pd(rho, rho), half);
                rho = _mm512_fmadd_pd(rho, e, rho);
                rho = _mm512_maskz_mov_pd((__mmask8)~coincident, rho);
                const __m512d qr = _mm512_mul_pd(sq, rho);
                p[v] = _mm512_add_pd(p[v], qr);
                if (grad) {
                    const __m512d w = _mm512_mul_pd(qr, _mm512_mul_pd(rho, rho));
                    a0[v] = _mm512_fnmadd_pd(w, d0, a0[v]);
                    a1[v] = _mm512_fnmadd_pd(w, d1, a1[v]);
                    a2[v] = _mm512_fnmadd_pd(w, d2, a2[v]);
                }
            }
        }
        for (int v = 0; v < 2; ++v) {
            _mm512_storeu_pd(lp + 8 * v, p[v]);
            _mm512_storeu_pd(l0 + 8 * v, a0[v]);
            _mm512_storeu_pd(l1 + 8 * v, a1[v]);
            _mm512_storeu_pd(l2 + 8 * v, a2[v]);
        }
        for (size_t i = 0; i < cnt; ++i) {
            ph[b + i] = lp[i];
            g0[b + i] = l0[i];
            g1[b + i] = l1[i];
            g2[b + i] = l2[i];
        }
    }
}

int orc_hp_has_avx512(void) {
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("fma");
}

void orc_hp_p2p(size_t ns, const double *src, const double *q, size_t nt, const double *tgt, double *potential,
                double *gradient) {
    if (nt == 0) return;
    if (!orc_hp_has_avx512()) {
        orc_p2p(ns, src, q, nt, tgt, potential, gradient);
        return;
    }
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
    p2p_avx512(ns, src, q, nt, tx, ty, tz, ph, g0, g1, g2, gradient != NULL);
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

/* C[:, c_j] += A B[:, b_j] for ncol columns (A column-major n x n), four at a time: each
 * column of A is read once per four columns, every element sums k ascending with the
 * product and the sum rounded apart (the bits of orc_matvec). */
__attribute__((target_clones("avx512f", "avx2", "default")))
void orc_hp_columns(int n, const double *restrict A, const double *const *bcols, double *const *ccols, int ncol) {
    int j = 0;
    for (; j + 4 <= ncol; j += 4) {
        double *restrict c0 = ccols[j], *restrict c1 = ccols[j + 1], *restrict c2 = ccols[j + 2],
                         *restrict c3 = ccols[j + 3];
        const double *b0 = bcols[j], *b1 = bcols[j + 1], *b2 = bcols[j + 2], *b3 = bcols[j + 3];
        for (int k = 0; k < n; ++k) {
            const double *restrict a = A + (size_t)k * n;
            const double x0 = b0[k], x1 = b1[k], x2 = b2[k], x3 = b3[k];
            for (int r = 0; r < n; ++r) {
                const double ar = a[r];
                c0[r] = c0[r] + x0 * ar;
                c1[r] = c1[r] + x1 * ar;
                c2[r] = c2[r] + x2 * ar;
                c3[r] = c3[r] + x3 * ar;
            }
        }
    }
    for (; j < ncol; ++j) orc_matvec(n, A, bcols[j], ccols[j]);
}
