/*
 * Oracle (test infrastructure only): the two loops of the oracle that run in vector lanes,
 * the table product y += A x (fmm-tables/src/matrix_set.rs:128, rows in lanes) and the P2P
 * sums of orc_p2p (targets in lanes).  Built apart with -O3 -fno-trapping-math
 * -fno-math-errno (oracle/Makefile): they only let the compiler vectorise and compute a
 * lane's square root and division before the select that drops a coincident pair; the
 * values are the same IEEE results, and -ffp-contract=off still forbids fma, so every sum
 * is bit for bit that of the scalar loop (orc_p2p_ref, fmm-ref/src/p2p.rs:90-140).  One
 * clone per ISA, chosen at load time.
 */
#include <math.h>
#include <stddef.h>

#include "fmm_oracle.h"

/* rows in vector lanes: every row's sum runs over k in the same ascending order, so the
 * clones give the same bits (no fma: -ffp-contract=off) */
__attribute__((target_clones("avx512f", "avx2", "default")))
void orc_matvec(int nc, const double *restrict A, const double *restrict x, double *restrict y) {
    for (int k = 0; k < nc; ++k) {
        double xk = x[k];
        const double *col = A + (size_t)k * nc;
        for (int r = 0; r < nc; ++r) y[r] = y[r] + xk * col[r];
    }
}

/* The same sums with the targets in vector lanes: sources outer, targets inner, so every
 * target still adds its terms in source order with the same operations (sqrt and division
 * correctly rounded, no fma), and a coincident pair leaves the sums as they were (a select
 * on r^2 = 0; x - y = 0 exactly when x = y).  The bits equal orc_p2p_ref's. */
__attribute__((target_clones("avx512f", "avx2", "default")))
void orc_p2p_lanes(size_t ns, const double *src, const double *q, size_t nt, const double *restrict tx,
                      const double *restrict ty, const double *restrict tz, double *restrict ph,
                      double *restrict g0, double *restrict g1, double *restrict g2) {
    for (size_t j = 0; j < ns; ++j) {
        const double y0 = src[3 * j], y1 = src[3 * j + 1], y2 = src[3 * j + 2], qj = q[j];
#pragma GCC ivdep
        for (size_t i = 0; i < nt; ++i) {
            const double d0 = tx[i] - y0, d1 = ty[i] - y1, d2 = tz[i] - y2;
            const int same = (d0 == 0.0) & (d1 == 0.0) & (d2 == 0.0);
            const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
            const double r2s = same ? 1.0 : r2;
            const double r = sqrt(r2s);
            const double r3 = r2s * r;
            const double p = ph[i] + qj / r;
            const double a0 = g0[i] + -(qj * d0 / r3), a1 = g1[i] + -(qj * d1 / r3), a2 = g2[i] + -(qj * d2 / r3);
            ph[i] = same ? ph[i] : p;
            g0[i] = same ? g0[i] : a0;
            g1[i] = same ? g1[i] : a1;
            g2[i] = same ? g2[i] : a2;
        }
    }
}

