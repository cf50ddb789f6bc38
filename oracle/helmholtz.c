/*
 * Oracle (test infrastructure only): the Helmholtz P2P of the reference, restated.
 *   - the pair term: fmm-ref/src/helmholtz/p2p.rs:315-375 (Term): d = x - y,
 *     r2 = d0^2 + d1^2 + d2^2, r = sqrt(r2), damping = -(Im k r), phase = Re k r,
 *     e = exp(damping) (cos phase, sin phase), factor = (damping - 1, phase);
 *     potential (q e) / r; gradient q ((factor e) / (r2 r)) d_k; exactly coincident
 *     pairs skipped;
 *   - p2p: fmm-ref/src/helmholtz/p2p.rs:102-140, sources in input order, plain additions;
 *   - direct_sum: the same terms, Neumaier per real component, one final addition;
 *   - near field on the plan: the P2P level calls of the Helmholtz operator
 *     (fmm-exec/src/helmholtz/operator.rs:2571-2615): leaf-scaled coordinates, the near
 *     row (U list and the leaf itself, by source leaf), sources mapped by the relative
 *     frame, wavenumber k_l = k r_0 2^-l (fmm-tables/src/helmholtz.rs:472,
 *     fmm-exec/src/helmholtz/fmm.rs:1146-1149), output phi / (4 pi r_t),
 *     grad / ((4 pi r_t) r_t) in caller order.
 * Complex numbers are (re, im) pairs of doubles; complex products are the textbook ones
 * (ac - bd, ad + bc), built with -ffp-contract=off like the rest of the oracle.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fmm_oracle.h"

typedef struct {
    double d[3], r, r3, e[2], f[2];
} hterm;

static int term(const double k[2], const double *x, const double *y, hterm *t) {
    if (x[0] == y[0] && x[1] == y[1] && x[2] == y[2]) return 0;
    for (int i = 0; i < 3; ++i) t->d[i] = x[i] - y[i];
    double r2 = t->d[0] * t->d[0] + t->d[1] * t->d[1] + t->d[2] * t->d[2];
    t->r = sqrt(r2);
    double damping = -(k[1] * t->r);
    double phase = k[0] * t->r;
    double decay = exp(damping);
    t->r3 = r2 * t->r;
    t->e[0] = decay * cos(phase);
    t->e[1] = decay * sin(phase);
    t->f[0] = damping - 1.0;
    t->f[1] = phase;
    return 1;
}

static void cmul(const double a[2], const double b[2], double out[2]) {
    double re = a[0] * b[0] - a[1] * b[1];
    double im = a[0] * b[1] + a[1] * b[0];
    out[0] = re;
    out[1] = im;
}

/* (q e) / r, and the three complex gradient terms q g d_k */
static void term_values(const hterm *t, const double q[2], double pot[2], double grad[6]) {
    double qe[2];
    cmul(q, t->e, qe);
    pot[0] = qe[0] / t->r;
    pot[1] = qe[1] / t->r;
    if (grad) {
        double fe[2], g[2], qg[2];
        cmul(t->f, t->e, fe);
        g[0] = fe[0] / t->r3;
        g[1] = fe[1] / t->r3;
        cmul(q, g, qg);
        for (int k = 0; k < 3; ++k) {
            grad[2 * k] = qg[0] * t->d[k];
            grad[2 * k + 1] = qg[1] * t->d[k];
        }
    }
}

void orc_helmholtz_p2p(double kre, double kim, size_t ns, const double *src, const double *q, size_t nt,
                       const double *tgt, double *potential, double *gradient) {
    const double k[2] = {kre, kim};
    for (size_t i = 0; i < nt; ++i)
        for (size_t j = 0; j < ns; ++j) {
            hterm t;
            if (!term(k, tgt + 3 * i, src + 3 * j, &t)) continue;
            double p[2], g[6];
            term_values(&t, q + 2 * j, p, gradient ? g : NULL);
            potential[2 * i] = potential[2 * i] + p[0];
            potential[2 * i + 1] = potential[2 * i + 1] + p[1];
            if (gradient)
                for (int c = 0; c < 6; ++c) gradient[6 * i + c] = gradient[6 * i + c] + g[c];
        }
}

typedef struct { double sum, comp; } nsum;

static void nadd(nsum *s, double term) {
    double t = s->sum + term;
    if (fabs(s->sum) >= fabs(term)) s->comp += (s->sum - t) + term;
    else s->comp += (term - t) + s->sum;
    s->sum = t;
}

void orc_helmholtz_direct_sum(double kre, double kim, size_t ns, const double *src, const double *q, size_t nt,
                              const double *tgt, double *potential, double *gradient) {
    const double k[2] = {kre, kim};
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < (long)nt; ++i) {
        nsum s[8];
        memset(s, 0, sizeof(s));
        for (size_t j = 0; j < ns; ++j) {
            hterm t;
            if (!term(k, tgt + 3 * i, src + 3 * j, &t)) continue;
            double p[2], g[6];
            term_values(&t, q + 2 * j, p, gradient ? g : NULL);
            nadd(&s[0], p[0]);
            nadd(&s[1], p[1]);
            if (gradient)
                for (int c = 0; c < 6; ++c) nadd(&s[2 + c], g[c]);
        }
        potential[2 * i] = potential[2 * i] + (s[0].sum + s[0].comp);
        potential[2 * i + 1] = potential[2 * i + 1] + (s[1].sum + s[1].comp);
        if (gradient)
            for (int c = 0; c < 6; ++c) gradient[6 * i + c] = gradient[6 * i + c] + (s[2 + c].sum + s[2 + c].comp);
    }
}
