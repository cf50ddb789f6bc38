// Helmholtz near field (P2P) of e^{ikr}/(4 pi r) on the plan, potential and gradient,
// complex charges; f64 or f32 (complex64) with the mixed form's f64 near-singular pairs.
//
// The pair term restates fmm-ref/src/helmholtz/p2p.rs:315-375 (Term): with d = x - y,
// r2 = |d|^2, r = sqrt(r2), damping = -(Im k r), phase = Re k r,
//   e = exp(damping) (cos phase + i sin phase),  phi += (q e) / r,
//   g = ((damping - 1) + i phase) e / (r2 r),    grad_k += (q g) d_k,
// exactly coincident pairs skipped.  As the reference's Helmholtz P2P level call
// (fmm-exec/src/helmholtz/operator.rs:2571-2615) it runs in leaf-scaled coordinates with
// the level's wavenumber k_l = k r_0 2^-l (fmm-tables/src/helmholtz.rs:472), sources
// mapped into the target leaf by y = fma(r, u, c); the output is phi / (4 pi r_t) and
// grad / ((4 pi r_t) r_t) in caller order, as for Laplace.
// Work split as p2p_kernel: one warp per item of up to 32 targets of one leaf, source
// leaves of the near row staged in shared memory, a partial per source leaf added into
// f64 per-target sums.
#pragma once

#include "kernels.cuh"

namespace fmmb {

template <typename T>
struct Cplx {
    T re, im;
};

template <typename T>
__device__ __forceinline__ Cplx<T> cmul(Cplx<T> a, Cplx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

template <typename T>
__device__ __forceinline__ void helm_exp_sincos(T damping, T phase, T& decay, T& s, T& c);
template <>
__device__ __forceinline__ void helm_exp_sincos<float>(float damping, float phase, float& decay, float& s, float& c) {
    decay = expf(damping);
    sincosf(phase, &s, &c);
}
template <>
__device__ __forceinline__ void helm_exp_sincos<double>(double damping, double phase, double& decay, double& s,
                                                        double& c) {
    decay = exp(damping);
    sincos(phase, &s, &c);
}

// one pair: adds (q e)/r into phi and (q g) d into g3 (T precision)
template <typename T, bool GRAD>
__device__ __forceinline__ void helm_pair(T kre, T kim, T dx, T dy, T dz, T r2, Cplx<T> q, Cplx<T>& phi,
                                          Cplx<T> (&g3)[3]) {
    const T r = sqrt(r2);
    const T damping = -(kim * r), phase = kre * r;
    T decay, s, c;
    helm_exp_sincos<T>(damping, phase, decay, s, c);
    const Cplx<T> e{decay * c, decay * s};
    const Cplx<T> qe = cmul(q, e);
    phi.re += qe.re / r;
    phi.im += qe.im / r;
    if (GRAD) {
        const T r3 = r2 * r;
        const Cplx<T> fe = cmul(Cplx<T>{damping - T(1), phase}, e);
        const Cplx<T> qg = cmul(q, Cplx<T>{fe.re / r3, fe.im / r3});
        g3[0].re += qg.re * dx;
        g3[0].im += qg.im * dx;
        g3[1].re += qg.re * dy;
        g3[1].im += qg.im * dy;
        g3[2].re += qg.re * dz;
        g3[2].im += qg.im * dz;
    }
}

// The same term in f32 (the mixed form's far-from-singular pairs): 1/r and 1/r^3 from one
// rsqrt instead of divisions, and the decay exp(-Im(k) r) not formed for a real wavenumber
// (it is exactly 1 there)
template <bool GRAD>
__device__ __forceinline__ void helm_pair_f32(float kre, float kim, float dx, float dy, float dz, float r2,
                                              Cplx<float> q, Cplx<float>& phi, Cplx<float> (&g3)[3]) {
    const float rinv = rsqrtf(r2);
    const float r = r2 * rinv;
    const float damping = -(kim * r), phase = kre * r;
    // the phase reduced to [-pi, pi] by Cody and Waite's two-step reduction (2 pi as a float
    // head and its remainder), then the hardware sine and cosine, whose error there is
    // below 2^-21 absolute: the f32 pair terms' own level
    const float turns = rintf(phase * 0.159154943091895336f);  // 1 / (2 pi)
    float pr = fmaf(-turns, 6.28318548202514648f, phase);     // 2 pi rounded to float
    pr = fmaf(-turns, -1.74845553146951640e-7f, pr);           // 2 pi minus that float
    float s, c;
    __sincosf(pr, &s, &c);
    const float decay = kim == 0.0f ? 1.0f : expf(damping);
    const Cplx<float> e{decay * c, decay * s};
    const Cplx<float> qe = cmul(q, e);
    phi.re += qe.re * rinv;
    phi.im += qe.im * rinv;
    if (GRAD) {
        const float rinv3 = rinv * rinv * rinv;
        const Cplx<float> fe = cmul(Cplx<float>{damping - 1.0f, phase}, e);
        const Cplx<float> qg = cmul(q, Cplx<float>{fe.re * rinv3, fe.im * rinv3});
        g3[0].re += qg.re * dx;
        g3[0].im += qg.im * dx;
        g3[1].re += qg.re * dy;
        g3[1].im += qg.im * dy;
        g3[2].re += qg.re * dz;
        g3[2].im += qg.im * dz;
    }
}

// Charges of the Helmholtz calls: caller order, m complex charges per point adjacent
// ((re, im) doubles) -> leaf order [v][point] in T, and in f64 for the near-singular pairs.
template <typename T>
__global__ void helm_charge_kernel(const double* __restrict__ q_caller, const int64_t* __restrict__ perm, int64_t n,
                                   int m, int stride, Cplx<T>* __restrict__ q_leaf, double2* __restrict__ q64) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t c = perm[i];
    for (int v = 0; v < m; ++v) {
        const double re = q_caller[2 * (c * stride + v)], im = q_caller[2 * (c * stride + v) + 1];
        q_leaf[(int64_t)v * n + i] = Cplx<T>{(T)re, (T)im};
        if (q64) q64[(int64_t)v * n + i] = make_double2(re, im);
    }
}

constexpr int kHelmWarps = 4;
constexpr int kHelmStage = 64;

// k the physical wavenumber; out_phi [v][nt] and out_g [v][nt][3], complex as (re, im)
// doubles, caller order; far_phi / far_g (when given) the far field's partials of the
// FMM in leaf order ([v][t] complex, [v][t][3] complex), added to each target's sum
template <typename T, bool GRAD, bool CLOSE>
__global__ void __launch_bounds__(32 * kHelmWarps) helm_p2p_kernel(
    DevPlan plan, P2pItems items, int m, T theta2, double k_re, double k_im,
    const typename Vec4<T>::type* __restrict__ spos, const Cplx<T>* __restrict__ sq,
    const typename Vec4<T>::type* __restrict__ tpos, ClosePairs close, const double2* __restrict__ q64,
    const double* __restrict__ far_phi, const double* __restrict__ far_g, double* __restrict__ out_phi,
    double* __restrict__ out_g) {
    using T4 = typename Vec4<T>::type;
    __shared__ T4 stage[kHelmWarps][kHelmStage];
    __shared__ Cplx<T> qstage[kHelmWarps][kHelmStage];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * kHelmWarps + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    const int64_t t = items.t0[item] + lane;
    const bool valid = t < t1;
    const int64_t n0 = plan.near_row[leaf], n1 = plan.near_row[leaf + 1];
    const int64_t nt = plan.ntgt, nsrc = plan.nsrc;
    const int lt = plan.level[box];
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(lt + 1));
    // k_l = k r_l: the reference's (k r_0) 2^-l, the same double (scaling by 2^-l is exact)
    const double kl_re = k_re * rt, kl_im = k_im * rt;
    const T kre = (T)kl_re, kim = (T)kl_im;
    T tx = T(0), ty = T(0), tz = T(0);
    if (valid) {
        const T4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    for (int v = 0; v < m; ++v) {
        double aphi[2] = {0.0, 0.0}, ag[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t e = n0; e < n1; ++e) {
            const int sl = plan.near_col[e];
            T c[3] = {T(0), T(0), T(0)}, r = T(1);
            const bool self = sl == leaf;
            if (!self) rel_frame<T>(plan, plan.leaf_box[sl], box, c, r);
            const int64_t s0 = plan.src_start[sl], s1 = plan.src_start[sl + 1];
            for (int64_t sb = s0; sb < s1; sb += kHelmStage) {
                const int cnt = (int)((s1 - sb) < kHelmStage ? (s1 - sb) : kHelmStage);
                for (int j = lane; j < cnt; j += 32) {
                    const T4 p4 = spos[sb + j];
                    T4 y;
                    y.x = self ? p4.x : map_coord<T>(r, p4.x, c[0]);
                    y.y = self ? p4.y : map_coord<T>(r, p4.y, c[1]);
                    y.z = self ? p4.z : map_coord<T>(r, p4.z, c[2]);
                    y.w = T(0);
                    stage[warp][j] = y;
                    qstage[warp][j] = sq[(int64_t)v * nsrc + sb + j];
                }
                __syncwarp();
                Cplx<T> pphi{T(0), T(0)};
                Cplx<T> pg[3] = {{T(0), T(0)}, {T(0), T(0)}, {T(0), T(0)}};
                for (int s = 0; s < cnt; ++s) {
                    const T4 y = stage[warp][s];
                    const T dx = sub_rn<T>(tx, y.x), dy = sub_rn<T>(ty, y.y), dz = sub_rn<T>(tz, y.z);
                    const T r2 = pair_r2<T>(dx, dy, dz);
                    const bool skip = CLOSE ? (r2 < theta2) : (r2 == T(0));
                    if (!skip) {
                        if constexpr (sizeof(T) == 4)
                            helm_pair_f32<GRAD>(kre, kim, dx, dy, dz, r2, qstage[warp][s], pphi, pg);
                        else
                            helm_pair<T, GRAD>(kre, kim, dx, dy, dz, r2, qstage[warp][s], pphi, pg);
                    }
                }
                aphi[0] += (double)pphi.re;
                aphi[1] += (double)pphi.im;
                if (GRAD)
                    for (int k = 0; k < 3; ++k) {
                        ag[2 * k] += (double)pg[k].re;
                        ag[2 * k + 1] += (double)pg[k].im;
                    }
                __syncwarp();
            }
        }
        if (!valid) continue;
        if (far_phi) {  // the far field's partials (the FMM): added after the near sums
            aphi[0] += far_phi[2 * ((int64_t)v * nt + t)];
            aphi[1] += far_phi[2 * ((int64_t)v * nt + t) + 1];
            if (GRAD)
                for (int k = 0; k < 6; ++k) ag[k] += far_g[6 * ((int64_t)v * nt + t) + k];
        }
        if (CLOSE) {
            // near-singular pairs in f64 with the reference's coincidence rule
            const double4 u = close.tpos[t];
            for (int64_t c2 = close.row[t]; c2 < close.row[t + 1]; ++c2) {
                const int64_t sp = close.src[c2];
                const double4 yv = close.y[c2];  // the source point in the target's frame
                const double yx = yv.x, yy = yv.y, yz = yv.z;
                if (u.x == yx && u.y == yy && u.z == yz) continue;
                const double dx = u.x - yx, dy = u.y - yy, dz = u.z - yz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double2 qq = q64[(int64_t)v * nsrc + sp];
                Cplx<double> p{0.0, 0.0};
                Cplx<double> g3[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
                helm_pair<double, GRAD>(kl_re, kl_im, dx, dy, dz, r2, Cplx<double>{qq.x, qq.y}, p, g3);
                aphi[0] += p.re;
                aphi[1] += p.im;
                if (GRAD)
                    for (int k = 0; k < 3; ++k) {
                        ag[2 * k] += g3[k].re;
                        ag[2 * k + 1] += g3[k].im;
                    }
            }
        }
        const int64_t i = plan.tgt_perm[t];
        out_phi[2 * ((int64_t)v * nt + i)] = aphi[0] / phi_scale;
        out_phi[2 * ((int64_t)v * nt + i) + 1] = aphi[1] / phi_scale;
        if (GRAD)
            for (int k = 0; k < 6; ++k) out_g[6 * ((int64_t)v * nt + i) + k] = ag[k] / g_scale;
    }
}

}  // namespace fmmb
