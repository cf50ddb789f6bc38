// The mixed Helmholtz near field from the near rows' source streams (the mixed Laplace
// P2P's P2pStream: every near row's sources mapped into the target leaf's frame once, at
// build), on the packed f32x2 pipe: the term of helm_pair_f32 for two sources per lane
// and step, e^{ik r} q / r and its gradient, for a real wavenumber and one charge vector.
//
// The work lists and the flush pipeline are the Laplace streamed P2P's (p2p_x2.cuh): items
// of 32 / KS slots of one leaf, flushes of 64 source pairs copied asynchronously, the
// complex charges gathered by index (real parts beside the z coordinates, imaginary parts
// apart).  Pairs with f32 r^2 < theta^2 (the near-singular pairs, found at build with this
// same r^2) take 1/r = 0 here and are summed in f64 per target from the close-pair CSR,
// as helm_p2p_kernel does; the f32 partials of a flush are added into f64 per-target sums.
#pragma once

#include "helmholtz.cuh"
#include "p2p_x2.cuh"

namespace fmmb {

struct HelmStArgs {
    DevPlan plan;
    P2pItems items;
    float theta2;
    double k_re;  // real k (at leaf level k_l = k r_l)
    P2pStream st;
    const Cplx<float>* sq;  // complex charges in leaf order (one vector)
    const float4* tpos;
    ClosePairs close;
    const double2* q64;     // the same charges in f64, for the near-singular pairs
    const double *far_phi, *far_g;  // far partials (null: the near field alone)
    double *out_phi, *out_g;
};

template <bool GRAD, int KS>
__global__ void __launch_bounds__(32, 24) helm_st_kernel(HelmStArgs a) {
    constexpr int NB = 2;
    __shared__ float4 sxy[NB][kStPairs];  // (x0, x1, y0, y1)
    __shared__ float4 szq[NB][kStPairs];  // (z0, z1, Re q0, Re q1)
    __shared__ float2 sqi[NB][kStPairs];  // (Im q0, Im q1)
    const int lane = threadIdx.x & 31;
    const int64_t item = blockIdx.x;
    if (item >= a.items.count) return;
    const DevPlan& plan = a.plan;
    const P2pStream& st = a.st;
    const int leaf = a.items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t0 = a.items.t0[item];
    int ni, ns;
    item_shape(a.items, item, plan.tgt_start[leaf + 1], ni, ns);
    constexpr int NIS = 32 / KS;
    ns = NIS;
    const int kk = lane / NIS, ti = lane % NIS;
    const int64_t t = t0 + ti;
    const bool valid = lane < ni;
    const bool has_target = ti < ni;
    const int64_t nt = plan.ntgt;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (has_target) {
        const float4 p4 = a.tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double kl = a.k_re * rt;  // k_l = k r_l, as helm_p2p_kernel forms it
    const float kf = (float)kl;
    const float2 k2 = f2(kf, kf);
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    const float theta2 = a.theta2;
    const int64_t pb = st.row_pair[leaf];
    const int np_row = (int)(st.row_pair[leaf + 1] - pb);
    const int nfl = np_row > 0 ? (np_row + kStPairs - 1) / kStPairs : 1;
    int ifl = 0;
    int2 ix0 = make_int2(-1, -1), ix1 = make_int2(-1, -1);
    auto load_idx = [&]() {
        const int i0 = ifl * kStPairs + lane, i1 = i0 + 32;
        ix0 = i0 < np_row ? st.idx[pb + i0] : make_int2(-1, -1);
        ix1 = i1 < np_row ? st.idx[pb + i1] : make_int2(-1, -1);
    };
    const float* qf = reinterpret_cast<const float*>(a.sq);  // (re, im) a source
    auto issue = [&](int b) {
        const int64_t base = pb + (int64_t)ifl * kStPairs;
        const int npf = np_row - ifl * kStPairs;
        float* zq = reinterpret_cast<float*>(&szq[b][0]);
        float* qi = reinterpret_cast<float*>(&sqi[b][0]);
        auto pair = [&](int i, int2 ix) {
            cp_async16_cg(&sxy[b][i], st.xy + base + i);
            cp_async8(zq + 4 * i, st.zz + base + i);
            const int s0 = ix.x < 0 ? 0 : ix.x, s1 = ix.y < 0 ? 0 : ix.y;
            cp_async4_zf(zq + 4 * i + 2, qf + 2 * (int64_t)s0, ix.x < 0 ? 0 : 4);
            cp_async4_zf(zq + 4 * i + 3, qf + 2 * (int64_t)s1, ix.y < 0 ? 0 : 4);
            cp_async4_zf(qi + 2 * i, qf + 2 * (int64_t)s0 + 1, ix.x < 0 ? 0 : 4);
            cp_async4_zf(qi + 2 * i + 1, qf + 2 * (int64_t)s1 + 1, ix.y < 0 ? 0 : 4);
        };
        if (lane < npf) pair(lane, ix0);
        if (lane + 32 < npf) pair(lane + 32, ix1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        if (++ifl < nfl) load_idx();
    };
    load_idx();
    issue(0);
    // f64 sums of the target: phi (re, im), then grad (x re, x im, y re, y im, z re, z im)
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const float2 inv2pi = f2(0.159154943091895336f, 0.159154943091895336f);     // 1 / (2 pi)
    const float2 twopi_hi = f2(-6.28318548202514648f, -6.28318548202514648f);  // -(2 pi rounded to float)
    const float2 twopi_lo = f2(1.74845553146951640e-7f, 1.74845553146951640e-7f);  // -(2 pi minus that)
    for (int f = 0; f < nfl; ++f) {
        const int b = f & 1;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        if (f + 1 < nfl) issue(b ^ 1);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        const int rem = np_row - f * kStPairs;
        const int npairs = rem < kStPairs ? rem : kStPairs;
        float2 pr = f2(0.f, 0.f), pi = f2(0.f, 0.f);  // phi partials (two sources' lanes)
        float2 g[6] = {f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f), f2(0.f, 0.f)};
        auto step = [&](int i) {
            const float4 p = sxy[b][i];
            const float4 c = szq[b][i];
            const float2 qim = sqi[b][i];
            const float2 qre = f2(c.z, c.w);
            // d = y - t (the close-pair search's r^2; the gradient's sign is fixed at the end)
            const float2 dx = __fadd2_rn(f2(p.x, p.y), ntx);
            const float2 dy = __fadd2_rn(f2(p.z, p.w), nty);
            const float2 dz = __fadd2_rn(f2(c.x, c.y), ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float ri0 = r2.x < theta2 ? 0.f : rsqrtf(r2.x);
            const float ri1 = r2.y < theta2 ? 0.f : rsqrtf(r2.y);
            const float2 rinv = f2(ri0, ri1);
            const float2 ph = __fmul2_rn(k2, __fmul2_rn(r2, rinv));  // k r (0 for a skipped pair)
            // the phase reduced to [-pi, pi] (Cody and Waite), then the hardware sine / cosine
            const float2 turns = f2(rintf(ph.x * inv2pi.x), rintf(ph.y * inv2pi.y));
            const float2 red = __ffma2_rn(turns, twopi_lo, __ffma2_rn(turns, twopi_hi, ph));
            float s0, c0, s1, c1;
            __sincosf(red.x, &s0, &c0);
            __sincosf(red.y, &s1, &c1);
            const float2 sn = f2(s0, s1), cs = f2(c0, c1);
            // q e = (qre c - qim s) + i (qre s + qim c); phi += q e / r
            const float2 qer = __ffma2_rn(qre, cs, __fmul2_rn(f2(-qim.x, -qim.y), sn));
            const float2 qei = __ffma2_rn(qre, sn, __fmul2_rn(qim, cs));
            pr = __ffma2_rn(qer, rinv, pr);
            pi = __ffma2_rn(qei, rinv, pi);
            if (GRAD) {
                // (-1 + i k r) e / r^3 = -(c + kr s) + i (kr c - s), times q, over r^3
                const float2 u = __ffma2_rn(ph, sn, cs);
                const float2 w = __ffma2_rn(ph, cs, f2(-sn.x, -sn.y));
                const float2 rinv3 = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
                // q (-u + i w) = -(qre u + qim w) + i (qre w - qim u)
                const float2 gr = __fmul2_rn(__ffma2_rn(qre, u, __fmul2_rn(qim, w)), rinv3);   // -Re
                const float2 gi = __fmul2_rn(__ffma2_rn(qre, w, __fmul2_rn(f2(-qim.x, -qim.y), u)), rinv3);
                // grad += (q g) (t - y) = Re: gr (y - t), Im: -gi (y - t)
                g[0] = __ffma2_rn(gr, dx, g[0]);
                g[1] = __ffma2_rn(gi, dx, g[1]);
                g[2] = __ffma2_rn(gr, dy, g[2]);
                g[3] = __ffma2_rn(gi, dy, g[3]);
                g[4] = __ffma2_rn(gr, dz, g[4]);
                g[5] = __ffma2_rn(gi, dz, g[5]);
            }
        };
        if (KS == 1) {
#pragma unroll 8
            for (int i = 0; i < npairs; ++i) step(i);
        } else {
#pragma unroll 4
            for (int i = kk; i < npairs; i += KS) step(i);
        }
        acc[0] += (double)pr.x;
        acc[0] += (double)pr.y;
        acc[1] += (double)pi.x;
        acc[1] += (double)pi.y;
        if (GRAD) {
            // the sums above are of (q g)(y - t) with g's real part negated: undo both here
            for (int k = 0; k < 3; ++k) {
                acc[2 + 2 * k] += (double)g[2 * k].x;
                acc[2 + 2 * k] += (double)g[2 * k].y;
                acc[3 + 2 * k] -= (double)g[2 * k + 1].x;
                acc[3 + 2 * k] -= (double)g[2 * k + 1].y;
            }
        }
        __syncwarp();  // buffer b read before it is refilled
    }
    if (KS > 1) {  // a target's KS partial sums, in kk order, through the (idle) pair buffers
        double(*red)[32] = reinterpret_cast<double(*)[32]>(&sxy[0][0]);
#pragma unroll
        for (int j = 0; j < 8; ++j) red[j][lane] = acc[j];
        __syncwarp();
        if (valid)
            for (int j = 1; j < KS; ++j)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[c] += red[c][ti + NIS * j];
        __syncwarp();
    }
    if (!valid) return;
    if (a.far_phi) {  // the far field's partials (the FMM), added after the near sums
        acc[0] += a.far_phi[2 * t];
        acc[1] += a.far_phi[2 * t + 1];
        if (GRAD)
            for (int k = 0; k < 6; ++k) acc[2 + k] += a.far_g[6 * t + k];
    }
    {  // the near-singular pairs in f64 with the reference's coincidence rule
        const ClosePairs& close = a.close;
        const double4 u = close.tpos[t];
        for (int64_t c2 = close.row[t]; c2 < close.row[t + 1]; ++c2) {
            const double4 yv = close.y[c2];
            if (u.x == yv.x && u.y == yv.y && u.z == yv.z) continue;
            const double dx = u.x - yv.x, dy = u.y - yv.y, dz = u.z - yv.z;
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double2 qq = a.q64[close.src[c2]];
            Cplx<double> p{0.0, 0.0};
            Cplx<double> g3[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
            helm_pair<double, GRAD>(kl, 0.0, dx, dy, dz, r2, Cplx<double>{qq.x, qq.y}, p, g3);
            acc[0] += p.re;
            acc[1] += p.im;
            if (GRAD)
                for (int k = 0; k < 3; ++k) {
                    acc[2 + 2 * k] += g3[k].re;
                    acc[3 + 2 * k] += g3[k].im;
                }
        }
    }
    const int64_t i = plan.tgt_perm[t];
    a.out_phi[2 * i] = acc[0] / phi_scale;
    a.out_phi[2 * i + 1] = acc[1] / phi_scale;
    if (GRAD)
        for (int k = 0; k < 6; ++k) a.out_g[6 * i + k] = acc[2 + k] / g_scale;
    (void)nt;
}

}  // namespace fmmb
