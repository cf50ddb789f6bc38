// Mixed-precision P2P on the packed f32x2 pipe of sm_100 (FFMA2 / FADD2 / FMUL2).
//
// One warp per work item of up to 32 targets of one leaf (lane = target; an item of fewer
// targets splits the sources over several lanes per target), the near row of that leaf
// (source leaves in row order, points in leaf order), sources mapped into the target
// leaf's frame by y = fma(r, u, c) (fmm-kernels/src/p2p.rs:320-340 frame_centre /
// frame_ratio), f32 pair terms with 1/r clamped to 4 (the near-singular pairs, f32
// r2 < theta2 = 1/16, found at build time by close_pairs_kernel with this r2, are then
// corrected by their f64 weights: close_sum_kernel below), f32 partials added into f64
// per-target accumulators.  The schedule:
//  - each lane takes two sources per instruction: the stage holds sources in pairs,
//    (x0, x1, y0, y1) and (z0, z1, q0, q1), so one LDS.128 yields aligned float2
//    operands and every add / multiply / fma of a pair-step is one f32x2 instruction;
//    the difference is formed as d = y + (-t) = -(t - y) exactly, so r2 is the float the
//    close-pair search forms and the gradient term fma(qr3, d, g) equals g - qr3 (t - y);
//  - the frame, start and size of every near entry are precomputed at build time
//    (NearRec, from rel_frame<float>, the same function the close-pair search uses), so
//    a source leaf costs no dependent index loads;
//  - the stage is filled across source-leaf boundaries (128 sources per flush), the next
//    flush's points and charges copied asynchronously (cp.async) while one is computed;
//    the streamed form (p2p_st_kernel) copies flushes already mapped at build time;
//  - an item of fewer than 32 targets splits the sources over several lanes per target.
// The f32 partial of a flush (at most 64 sources per half) is added into the f64 sums.
#pragma once

#include "kernels.cuh"

namespace fmmb {

struct __align__(16) NearRec {
    float4 frame;   // (c0, c1, c2, r): y = fma(r, u, c) maps the source leaf into the target leaf
    long long s0;   // first source point of the source leaf (leaf order)
    int ns;         // its points
    int off;        // position of its first point in the row's concatenated source stream
};

// Build time: one record per near-list entry (row = target leaf).
static __global__ void near_record_kernel(DevPlan plan, int64_t nleaves, NearRec* __restrict__ rec) {
    const int64_t leaf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (leaf >= nleaves) return;
    const int box = plan.leaf_box[leaf];
    int off = 0;
    for (int64_t e = plan.near_row[leaf]; e < plan.near_row[leaf + 1]; ++e) {
        const int sl = plan.near_col[e];
        float c[3], r;
        rel_frame<float>(plan, plan.leaf_box[sl], box, c, r);
        NearRec x;
        x.frame = make_float4(c[0], c[1], c[2], r);
        x.s0 = plan.src_start[sl];
        x.ns = (int)(plan.src_start[sl + 1] - plan.src_start[sl]);
        x.off = off;
        off += x.ns;
        rec[e] = x;
    }
}

// The near-singular pairs as a fixed sparse operator.  In the f32 pair loop every pair's
// 1/r is clamped to rmax = 1/theta = 4: a pair with f32 r^2 >= theta^2 = 1/16 is unchanged
// (its 1/r is at most 4), a near-singular one (f32 r^2 < 1/16, the pairs close_pairs_kernel
// finds with the same arithmetic) contributes exactly 4 q to phi and 64 q d32 to the
// gradient sum, d32 its f32 difference y - t.  The exact term minus that clamp term is q
// times a weight fixed by the geometry, formed at build time in f64 from f64 coordinates
// with the reference's coincidence rule (a coincident pair has no exact term):
// w = (1/r - 4, (y - u)/r^3 - 64 d32).  Each evaluation forms the f64 sum of q_s w over a
// target's near-singular pairs in CSR order (close_sum_kernel, q the f64 charges) and the
// P2P epilogue adds it once, after the f32 partials.  The clamp terms carry the f32
// charge and the weights the f64 one: the difference is 4 |q32 - q64| <= 2^-22 |q| a pair.
// A weight is formed in f64 and stored rounded to f32 (relative 2^-24 of that pair's
// term; in range for any two distinct f64 points, whose leaf-unit distance is far above
// the 1e-19 where 1/r^2 would leave f32), and the sums stay f64: the sparse operator reads
// 20 bytes a pair (weights and a 32-bit source index) where f64 weights took 40.

// Build time: block per leaf, thread per target; w is 4 floats a pair (GRAD) or 1.
template <bool GRAD>
__global__ void close_weights_kernel(DevPlan plan, ClosePairs close, const float4* __restrict__ spos32,
                                     const float4* __restrict__ tpos32, float rmax, float* __restrict__ w) {
    const int64_t leaf = blockIdx.x;
    const int box = plan.leaf_box[leaf];
    const double R = rmax, R3 = (double)rmax * rmax * rmax;
    for (int64_t t = plan.tgt_start[leaf] + threadIdx.x; t < plan.tgt_start[leaf + 1]; t += blockDim.x) {
        const double4 u = close.tpos[t];
        const float4 t32 = tpos32[t];
        for (int64_t c2 = close.row[t]; c2 < close.row[t + 1]; ++c2) {
            // the f32 difference of the pair loop: the near entry's frame (NearRec), y + (-t)
            float fc[3], fr;
            rel_frame<float>(plan, plan.leaf_box[close.leaf[c2]], box, fc, fr);
            const float4 p = spos32[close.src[c2]];
            const double d32x = __fadd_rn(__fmaf_rn(fr, p.x, fc[0]), -t32.x);
            const double d32y = __fadd_rn(__fmaf_rn(fr, p.y, fc[1]), -t32.y);
            const double d32z = __fadd_rn(__fmaf_rn(fr, p.z, fc[2]), -t32.z);
            const double4 y = close.y[c2];
            double rinv = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
            if (!(u.x == y.x && u.y == y.y && u.z == y.z)) {
                dx = y.x - u.x;
                dy = y.y - u.y;
                dz = y.z - u.z;
                rinv = rsqrt(dx * dx + dy * dy + dz * dz);
            }
            const double r3 = rinv * rinv * rinv;
            if (GRAD)
                reinterpret_cast<float4*>(w)[c2] =
                    make_float4(__double2float_rn(rinv - R), __double2float_rn(r3 * dx - R3 * d32x),
                                __double2float_rn(r3 * dy - R3 * d32y), __double2float_rn(r3 * dz - R3 * d32z));
            else
                w[c2] = __double2float_rn(rinv - R);
        }
    }
}

// Build time: each pair's source index as 32 bits.
static __global__ void close_src32_kernel(const int64_t* __restrict__ src, int64_t n, uint32_t* __restrict__ src32) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) src32[i] = (uint32_t)src[i];
}

// Evaluation: thread per target, every vector of the pass; acc [vector][target].
// src32: each pair's source as 32 bits (the plan has fewer than 2^32 sources).
template <bool GRAD>
__global__ void close_sum_kernel(ClosePairs close, const float* __restrict__ w, const uint32_t* __restrict__ src32,
                                 int m, int64_t nsrc, int64_t nt, double* __restrict__ acc) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int64_t c0 = close.row[t], c1 = close.row[t + 1];
    for (int v = 0; v < m; ++v) {
        const double* qv = close.q + (int64_t)v * nsrc;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll 4
        for (int64_t c = c0; c < c1; ++c) {
            const double q = qv[src32[c]];
            if (GRAD) {
                const float4 wc = reinterpret_cast<const float4*>(w)[c];
                a0 = __fma_rn(q, (double)wc.x, a0);
                a1 = __fma_rn(q, (double)wc.y, a1);
                a2 = __fma_rn(q, (double)wc.z, a2);
                a3 = __fma_rn(q, (double)wc.w, a3);
            } else {
                a0 = __fma_rn(q, (double)w[c], a0);
            }
        }
        if (GRAD)
            reinterpret_cast<double4*>(acc)[(int64_t)v * nt + t] = make_double4(a0, a1, a2, a3);
        else
            acc[(int64_t)v * nt + t] = a0;
    }
}

// The P2P epilogue's addition of a target's near-singular sum (entry vt = v nt + t); no
// sums (acc null) when the plan has no near-singular pair.
template <bool GRAD>
__device__ __forceinline__ void close_sum_add(const ClosePairs& close, int64_t vt, double& aphi, double& ag0,
                                              double& ag1, double& ag2) {
    if (!close.acc) return;
    if (GRAD) {
        const double4 c = reinterpret_cast<const double4*>(close.acc)[vt];
        aphi += c.x;
        ag0 += c.y;
        ag1 += c.z;
        ag2 += c.w;
    } else {
        aphi += close.acc[vt];
    }
}
__device__ __forceinline__ void close_sum_add1(const ClosePairs& close, int64_t vt, double& aphi) {
    if (close.acc) aphi += close.acc[vt];
}

constexpr int kX2Warps = 4;      // warps a block until the autotuner chooses
constexpr int kX2Stage = 128;  // sources per flush (64 pairs)
constexpr int kX2Recs = 58;    // a near row's entries, all in shared memory (2:1 balance: at most 57)

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async16_cg(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
// 4 bytes, or zeros when src_bytes is 0 (the address is then not read)
__device__ __forceinline__ void cp_async4_zf(void* smem, const void* gmem, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem), "r"(src_bytes)
                 : "memory");
}

// Flushes run over (vector, position in the row's source stream); while flush f is
// computed, the raw points and charges of flush f + 1 are in flight (cp.async), so a
// warp does not wait on global memory for its sources.
// W warps a block (1, 2 or 4; the autotuner picks one): 6.8 KB of shared memory and
// at most 64 registers a thread, so 32 warps are resident on an SM for every W.
template <bool GRAD, int W>
__global__ void __launch_bounds__(32 * W, 32 / W) p2p_x2_kernel(
    DevPlan plan, P2pItems items, int m, int near, float rmax, const NearRec* __restrict__ recs,
    const float4* __restrict__ spos, const float* __restrict__ sq, const float4* __restrict__ tpos, ClosePairs close,
    double* __restrict__ far_phi, double* __restrict__ far_g, int accumulate, double* __restrict__ out_phi,
    double* __restrict__ out_g) {
    __shared__ float4 sxy[W][kX2Stage / 2];  // (x0, x1, y0, y1) in the target's frame
    __shared__ float4 szq[W][kX2Stage / 2];  // (z0, z1, q0, q1)
    __shared__ float4 raw[W][kX2Stage];      // the next flush's points, as loaded
    __shared__ float rawq[W][kX2Stage];
    __shared__ int rawrec[W][kX2Stage];      // their near entries
    __shared__ NearRec srec[W][kX2Recs];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the split lanes' sums, reduced per target, in the pair buffer (idle at that point)
    double(*red)[32] = reinterpret_cast<double(*)[32]>(&sxy[warp][0]);
    const int64_t item = (int64_t)blockIdx.x * W + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    // an item of ni targets in ns >= ni slots splits each flush's pair-steps over K = 32 / ns
    // lanes per target: lane = slot + ns * kk takes the pair-steps i = kk (mod K); the K
    // sums of a target are added in kk order at the end (slots past ni hold no target)
    int ni, ns;
    item_shape(items, item, t1, ni, ns);
    const int K = 32 / ns;
    const int kk = lane < ns * K && lane % ns < ni ? lane / ns : K;  // lanes without a target take no pair-steps
    const int ti = lane < ns * K ? lane % ns : 0;
    const int64_t t = items.t0[item] + ti;
    const bool valid = lane < ni;  // the lanes that finish their target (kk = 0)
    const int64_t n0 = plan.near_row[leaf], n1 = near ? plan.near_row[leaf + 1] : n0;
    const int64_t nt = plan.ntgt, nsrc = plan.nsrc;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (kk < K) {
        const float4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
    float* sxy_f = reinterpret_cast<float*>(sxy[warp]);
    float* szq_f = reinterpret_cast<float*>(szq[warp]);
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    const int nr = (int)(n1 - n0);  // <= kX2Recs, checked when the plan is uploaded
    for (int j = lane; j < nr; j += 32) srec[warp][j] = recs[n0 + j];
    __syncwarp();
    const int S = nr ? srec[warp][nr - 1].off + srec[warp][nr - 1].ns : 0;  // the row's sources
    const int nfl = S > 0 ? (S + kX2Stage - 1) / kX2Stage : 1;              // flushes per vector
    const int total = nfl * m;
    int epf = 0;  // this lane's near entry in the prefetch walk (monotone within a vector)
    auto issue = [&](int f) {
        const int v = f / nfl, base = (f - v * nfl) * kX2Stage;
        const int cnt = (S - base) < kX2Stage ? (S - base) : kX2Stage;
        const float* qv = sq + (int64_t)v * nsrc;
        if (base == 0) epf = 0;
#pragma unroll
        for (int i = 0; i < kX2Stage / 32; ++i) {
            const int k = lane + 32 * i;
            if (k < cnt) {
                const int pos = base + k;
                // the entries are contiguous in the stream and pos < S: epf stays < nr
                while (srec[warp][epf].off + srec[warp][epf].ns <= pos) ++epf;
                const int64_t s = srec[warp][epf].s0 + (pos - srec[warp][epf].off);
                cp_async16(&raw[warp][k], spos + s);
                cp_async4(&rawq[warp][k], qv + s);
                rawrec[warp][k] = epf;
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    double aphi = 0.0, ag0 = 0.0, ag1 = 0.0, ag2 = 0.0;
    issue(0);
    for (int f = 0; f < total; ++f) {
        const int v = f / nfl, base = (f - v * nfl) * kX2Stage;
        const int cnt = (S - base) < kX2Stage ? (S - base) : kX2Stage;
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        // map the flush's sources into the target's frame, in pairs
#pragma unroll
        for (int i = 0; i < kX2Stage / 32; ++i) {
            const int k = lane + 32 * i;
            if (k < cnt) {
                const float4 p = raw[warp][k];
                const float4 fr = srec[warp][rawrec[warp][k]].frame;
                const int slot = (k >> 1) * 4 + (k & 1);
                sxy_f[slot] = __fmaf_rn(fr.w, p.x, fr.x);
                sxy_f[slot + 2] = __fmaf_rn(fr.w, p.y, fr.y);
                szq_f[slot] = __fmaf_rn(fr.w, p.z, fr.z);
                szq_f[slot + 2] = rawq[warp][k];
            }
        }
        if ((cnt & 1) && lane == 0) {  // odd count: a zero charge completes the last pair
            const int slot = (cnt >> 1) * 4 + 1;
            sxy_f[slot] = 0.f;
            sxy_f[slot + 2] = 0.f;
            szq_f[slot] = 0.f;
            szq_f[slot + 2] = 0.f;
        }
        __syncwarp();
        if (f + 1 < total) issue(f + 1);  // the raw buffers are free again
        float2 pphi = f2(0.f, 0.f), pg0 = f2(0.f, 0.f), pg1 = f2(0.f, 0.f), pg2 = f2(0.f, 0.f);
        const int npairs = (cnt + 1) >> 1;
#pragma unroll 2
        for (int i = kk; i < npairs; i += K) {
            const float4 a = sxy[warp][i];
            const float4 b = szq[warp][i];
            const float2 dx = __fadd2_rn(f2(a.x, a.y), ntx);
            const float2 dy = __fadd2_rn(f2(a.z, a.w), nty);
            const float2 dz = __fadd2_rn(f2(b.x, b.y), ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float ri0 = fminf(rsqrtf(r2.x), rmax);
            const float ri1 = fminf(rsqrtf(r2.y), rmax);
            const float2 rinv = f2(ri0, ri1);
            const float2 qr = __fmul2_rn(f2(b.z, b.w), rinv);
            pphi = __fadd2_rn(pphi, qr);
            if (GRAD) {
                const float2 qr3 = __fmul2_rn(__fmul2_rn(qr, rinv), rinv);
                pg0 = __ffma2_rn(qr3, dx, pg0);
                pg1 = __ffma2_rn(qr3, dy, pg1);
                pg2 = __ffma2_rn(qr3, dz, pg2);
            }
        }
        aphi += (double)pphi.x;
        aphi += (double)pphi.y;
        if (GRAD) {
            ag0 += (double)pg0.x;
            ag0 += (double)pg0.y;
            ag1 += (double)pg1.x;
            ag1 += (double)pg1.y;
            ag2 += (double)pg2.x;
            ag2 += (double)pg2.y;
        }
        __syncwarp();  // the pairs are read before the next map overwrites them
        if (f - v * nfl != nfl - 1) continue;
        // ---- the last flush of vector v: finish its targets ----
        if (K > 1) {  // the target's K partial sums, in kk order
            red[0][lane] = aphi;
            red[1][lane] = ag0;
            red[2][lane] = ag1;
            red[3][lane] = ag2;
            __syncwarp();
            if (valid)
                for (int j = 1; j < K; ++j) {
                    aphi += red[0][ti + ns * j];
                    ag0 += red[1][ti + ns * j];
                    ag1 += red[2][ti + ns * j];
                    ag2 += red[3][ti + ns * j];
                }
            __syncwarp();
        }
        if (valid) {
            if (near) close_sum_add<GRAD>(close, (int64_t)v * nt + t, aphi, ag0, ag1, ag2);
            // both gradient sums hold -sum qr3 (t - y), as p2p_kernel's
            if (accumulate == 2) {  // near field alone, leaf order (added to the far field by output_kernel)
                out_phi[(int64_t)v * nt + t] = aphi;
                if (GRAD) {
                    double* o = out_g + ((int64_t)v * nt + t) * 3;
                    o[0] = ag0;
                    o[1] = ag1;
                    o[2] = ag2;
                }
            } else if (accumulate) {  // level calls: add into the leaf-order store, scaled by output_kernel
                far_phi[(int64_t)v * nt + t] = far_phi[(int64_t)v * nt + t] + aphi;
                if (GRAD) {
                    double* fg = far_g + ((int64_t)v * nt + t) * 3;
                    fg[0] = fg[0] + ag0;
                    fg[1] = fg[1] + ag1;
                    fg[2] = fg[2] + ag2;
                }
            } else {
                const double ph = far_phi[(int64_t)v * nt + t] + aphi;
                const int64_t i = plan.tgt_perm[t];
                out_phi[(int64_t)v * nt + i] = ph / phi_scale;
                if (GRAD) {
                    const double* fg = far_g + ((int64_t)v * nt + t) * 3;
                    double* o = out_g + ((int64_t)v * nt + i) * 3;
                    o[0] = (fg[0] + ag0) / g_scale;
                    o[1] = (fg[1] + ag1) / g_scale;
                    o[2] = (fg[2] + ag2) / g_scale;
                }
            }
        }
        aphi = ag0 = ag1 = ag2 = 0.0;
    }
}

// Potentials of several charge vectors (no gradients): the flush stages the sources'
// positions once and the charges of VB vectors; a pair-step forms the pair geometry (d, r2,
// the rsqrt and its near-singular select) once and adds q rinv for each vector.  Per
// vector every operation and its order are p2p_x2_kernel<false, W>'s (the same flushes,
// the same pair-steps, the same f64 additions), so the floats do not depend on how many
// vectors a pass holds; the evaluation uses this kernel for every vector count.
constexpr int kX2Vb = 4;  // vectors a flush

template <int W>
__global__ void __launch_bounds__(32 * W, 20 / W) p2p_x2_mv_kernel(
    DevPlan plan, P2pItems items, int m, int near, float rmax, const NearRec* __restrict__ recs,
    const float4* __restrict__ spos, const float* __restrict__ sq, const float4* __restrict__ tpos, ClosePairs close,
    double* __restrict__ far_phi, int accumulate, double* __restrict__ out_phi) {
    constexpr int VB = kX2Vb;
    __shared__ float4 sxy[W][kX2Stage / 2];       // (x0, x1, y0, y1) in the target's frame
    __shared__ float2 szz[W][kX2Stage / 2];       // (z0, z1)
    __shared__ float2 sqq[W][VB][kX2Stage / 2];   // (q0, q1) of each vector
    __shared__ float4 raw[W][kX2Stage];           // the next flush's points, as loaded
    __shared__ float rawq[W][VB][kX2Stage];
    __shared__ int rawrec[W][kX2Stage];
    __shared__ NearRec srec[W][kX2Recs];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the split lanes' sums (VB x 32 doubles), reduced per target, in the pair buffer
    double(*red)[32] = reinterpret_cast<double(*)[32]>(&sxy[warp][0]);
    static_assert(VB * 32 * sizeof(double) <= sizeof(float4) * (kX2Stage / 2), "reduction buffer");
    const int64_t item = (int64_t)blockIdx.x * W + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    int ni, ns;
    item_shape(items, item, t1, ni, ns);
    const int K = 32 / ns;
    const int kk = lane < ns * K && lane % ns < ni ? lane / ns : K;
    const int ti = lane < ns * K ? lane % ns : 0;
    const int64_t t = items.t0[item] + ti;
    const bool valid = lane < ni;
    const int64_t n0 = plan.near_row[leaf], n1 = near ? plan.near_row[leaf + 1] : n0;
    const int64_t nt = plan.ntgt, nsrc = plan.nsrc;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (kk < K) {
        const float4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
    float* sxy_f = reinterpret_cast<float*>(sxy[warp]);
    float* szz_f = reinterpret_cast<float*>(szz[warp]);
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const int nr = (int)(n1 - n0);
    for (int j = lane; j < nr; j += 32) srec[warp][j] = recs[n0 + j];
    __syncwarp();
    const int S = nr ? srec[warp][nr - 1].off + srec[warp][nr - 1].ns : 0;
    const int nfl = S > 0 ? (S + kX2Stage - 1) / kX2Stage : 1;
    const int nvb = (m + VB - 1) / VB;
    const int total = nfl * nvb;
    int epf = 0;
    auto issue = [&](int f) {
        const int vb = f / nfl, base = (f - vb * nfl) * kX2Stage;
        const int v0 = vb * VB, nb = (m - v0) < VB ? (m - v0) : VB;
        const int cnt = (S - base) < kX2Stage ? (S - base) : kX2Stage;
        if (base == 0) epf = 0;
#pragma unroll
        for (int i = 0; i < kX2Stage / 32; ++i) {
            const int k = lane + 32 * i;
            if (k < cnt) {
                const int pos = base + k;
                while (srec[warp][epf].off + srec[warp][epf].ns <= pos) ++epf;
                const int64_t s = srec[warp][epf].s0 + (pos - srec[warp][epf].off);
                cp_async16(&raw[warp][k], spos + s);
#pragma unroll
                for (int b = 0; b < VB; ++b)
                    if (b < nb) cp_async4(&rawq[warp][b][k], sq + (int64_t)(v0 + b) * nsrc + s);
                rawrec[warp][k] = epf;
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    double aphi[VB];
#pragma unroll
    for (int b = 0; b < VB; ++b) aphi[b] = 0.0;
    issue(0);
    for (int f = 0; f < total; ++f) {
        const int vb = f / nfl, base = (f - vb * nfl) * kX2Stage;
        const int v0 = vb * VB, nb = (m - v0) < VB ? (m - v0) : VB;
        const int cnt = (S - base) < kX2Stage ? (S - base) : kX2Stage;
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kX2Stage / 32; ++i) {
            const int k = lane + 32 * i;
            if (k < cnt) {
                const float4 p = raw[warp][k];
                const float4 fr = srec[warp][rawrec[warp][k]].frame;
                const int slot = (k >> 1) * 4 + (k & 1);
                sxy_f[slot] = __fmaf_rn(fr.w, p.x, fr.x);
                sxy_f[slot + 2] = __fmaf_rn(fr.w, p.y, fr.y);
                szz_f[k] = __fmaf_rn(fr.w, p.z, fr.z);
#pragma unroll
                for (int b = 0; b < VB; ++b)
                    if (b < nb) reinterpret_cast<float*>(sqq[warp][b])[k] = rawq[warp][b][k];
            }
        }
        if ((cnt & 1) && lane == 0) {  // odd count: a zero charge completes the last pair
            const int slot = (cnt >> 1) * 4 + 1;
            sxy_f[slot] = 0.f;
            sxy_f[slot + 2] = 0.f;
            szz_f[cnt] = 0.f;
#pragma unroll
            for (int b = 0; b < VB; ++b) reinterpret_cast<float*>(sqq[warp][b])[cnt] = 0.f;
        }
        __syncwarp();
        if (f + 1 < total) issue(f + 1);
        float2 pphi[VB];
#pragma unroll
        for (int b = 0; b < VB; ++b) pphi[b] = f2(0.f, 0.f);
        const int npairs = (cnt + 1) >> 1;
#pragma unroll 2
        for (int i = kk; i < npairs; i += K) {
            const float4 a = sxy[warp][i];
            const float2 zz = szz[warp][i];
            const float2 dx = __fadd2_rn(f2(a.x, a.y), ntx);
            const float2 dy = __fadd2_rn(f2(a.z, a.w), nty);
            const float2 dz = __fadd2_rn(zz, ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float ri0 = fminf(rsqrtf(r2.x), rmax);
            const float ri1 = fminf(rsqrtf(r2.y), rmax);
            const float2 rinv = f2(ri0, ri1);
#pragma unroll
            for (int b = 0; b < VB; ++b)
                if (b < nb) pphi[b] = __fadd2_rn(pphi[b], __fmul2_rn(sqq[warp][b][i], rinv));
        }
#pragma unroll
        for (int b = 0; b < VB; ++b) {
            aphi[b] += (double)pphi[b].x;
            aphi[b] += (double)pphi[b].y;
        }
        __syncwarp();  // the pairs are read before the next map overwrites them
        if (f - vb * nfl != nfl - 1) continue;
        // ---- the last flush of vectors v0 .. v0 + nb: finish their targets ----
        if (K > 1) {
#pragma unroll
            for (int b = 0; b < VB; ++b) red[b][lane] = aphi[b];
            __syncwarp();
            if (valid)
                for (int j = 1; j < K; ++j)
#pragma unroll
                    for (int b = 0; b < VB; ++b) aphi[b] += red[b][ti + ns * j];
            __syncwarp();
        }
        if (valid) {
            if (near)
#pragma unroll
                for (int b = 0; b < VB; ++b)
                    if (b < nb) close_sum_add1(close, (int64_t)(v0 + b) * nt + t, aphi[b]);
#pragma unroll
            for (int b = 0; b < VB; ++b) {
                if (b >= nb) break;
                const int v = v0 + b;
                if (accumulate == 2) {
                    out_phi[(int64_t)v * nt + t] = aphi[b];
                } else if (accumulate) {
                    far_phi[(int64_t)v * nt + t] = far_phi[(int64_t)v * nt + t] + aphi[b];
                } else {
                    const double ph = far_phi[(int64_t)v * nt + t] + aphi[b];
                    out_phi[(int64_t)v * nt + plan.tgt_perm[t]] = ph / phi_scale;
                }
            }
        }
#pragma unroll
        for (int b = 0; b < VB; ++b) aphi[b] = 0.0;
    }
}

// ---------------------------------------------------------------------------------------
// The streamed form.  A near row's source stream (its near entries in row order, each
// source leaf's points in leaf order) is mapped into the target leaf's frame once, at build
// time, with the same f32 fma as the map step above (y = fma(r, u, c), the frame of the
// entry's NearRec), and stored in the staged pair layout: per pair of stream positions
// (2i, 2i + 1) a float4 (x0, x1, y0, y1), a float2 (z0, z1) and the two sources' indices
// (leaf order; an odd stream ends with a padding source at the origin, index -1, whose
// charge is zero, as the map step pads an odd flush).  A flush is then plain copies of
// consecutive pairs plus a gather of the flush's charges by index, double-buffered: the
// staged floats, the pair-steps and every addition are those of p2p_x2_kernel and
// p2p_x2_mv_kernel, so the two forms give the same bits.

struct P2pStream {
    const int64_t* row_pair;  // per leaf (nleaves + 1): the first pair of its row's stream
    const float4* xy;         // per pair: (x0, x1, y0, y1) in the target leaf's frame
    const float2* zz;         // per pair: (z0, z1)
    const int2* idx;          // per pair: the sources' indices in leaf order (-1: padding)
};

// Build time: warp per leaf row, writing that row's pairs.
static __global__ void near_stream_kernel(DevPlan plan, int64_t nleaves, const NearRec* __restrict__ recs,
                                   const float4* __restrict__ spos, const int64_t* __restrict__ row_pair,
                                   float4* __restrict__ xy_out, float2* __restrict__ zz_out,
                                   int2* __restrict__ idx_out) {
    const int64_t leaf = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (leaf >= nleaves) return;
    const int64_t pb = row_pair[leaf];
    float* xy = reinterpret_cast<float*>(xy_out + pb);
    float* zz = reinterpret_cast<float*>(zz_out + pb);
    int* ix = reinterpret_cast<int*>(idx_out + pb);
    int S = 0;
    for (int64_t e = plan.near_row[leaf]; e < plan.near_row[leaf + 1]; ++e) {
        const NearRec r = recs[e];
        for (int k = lane; k < r.ns; k += 32) {
            const int pos = r.off + k;
            const float4 u = spos[r.s0 + k];
            const int slot = (pos >> 1) * 4 + (pos & 1);
            xy[slot] = __fmaf_rn(r.frame.w, u.x, r.frame.x);
            xy[slot + 2] = __fmaf_rn(r.frame.w, u.y, r.frame.y);
            zz[pos] = __fmaf_rn(r.frame.w, u.z, r.frame.z);
            ix[pos] = (int)(r.s0 + k);
        }
        S = r.off + r.ns;
    }
    if ((S & 1) && lane == 0) {
        const int slot = (S >> 1) * 4 + 1;
        xy[slot] = 0.f;
        xy[slot + 2] = 0.f;
        zz[S] = 0.f;
        ix[S] = -1;
    }
}

constexpr int kStPairs = kX2Stage / 2;  // pairs a flush (64)

// NB flush buffers (NB - 1 flushes in flight while one is computed); three measured no
// faster than two at the bench size (P2P 2.046 vs 2.042 ms): the flush latency is hidden.
constexpr int kStBufs = 2;

// The arguments of the streamed P2P launches.
struct P2pStArgs {
    DevPlan plan;
    P2pItems items;
    int m, near;
    float rmax;
    P2pStream st;
    const float* sq;
    const float4* tpos;
    ClosePairs close;
    double *far_phi, *far_g;
    int accumulate;
    double *out_phi, *out_g;
};

// One work item of the streamed P2P, by one warp, with its NB flush buffers sxy / szq.
// V1: one charge vector (m = 1), the vector loop compiled out.  KS: the lanes a target
// splits its pair-steps over when fixed at compile time (items of 32 / KS slots: 1 one
// target a lane, 2, 4 or 8 a strided loop of constant stride), 0 any item.
template <bool GRAD, bool V1, int KS>
__device__ __forceinline__ void p2p_st_item(const P2pStArgs& a, int64_t item, float4 (*sxy)[kStPairs],
                                            float4 (*szq)[kStPairs], int lane) {
    constexpr int NB = kStBufs;
    const DevPlan& plan = a.plan;
    const P2pItems& items = a.items;
    const P2pStream& st = a.st;
    const ClosePairs& close = a.close;
    const float* __restrict__ sq = a.sq;
    const float4* __restrict__ tpos = a.tpos;
    double* __restrict__ far_phi = a.far_phi;
    double* __restrict__ far_g = a.far_g;
    double* __restrict__ out_phi = a.out_phi;
    double* __restrict__ out_g = a.out_g;
    const int near = a.near, accumulate = a.accumulate;
    const float rmax = a.rmax;
    const int m = V1 ? 1 : a.m;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    // the lanes of an item of ni < 32 targets split the pair-steps (p2p_x2_kernel)
    constexpr int NIS = KS ? 32 / KS : 0;  // slots of an item when KS fixes them
    int ni, ns;
    item_shape(items, item, t1, ni, ns);
    if (KS) ns = NIS;
    const int K = KS ? KS : 32 / ns;
    const int kk = KS ? lane / NIS : lane < ns * K ? lane / ns : K;
    const int ti = KS ? lane % NIS : lane < ns * K ? lane % ns : 0;
    const int64_t t = items.t0[item] + ti;
    const bool valid = lane < ni;
    const bool has_target = kk < K && ti < ni;  // lanes of padding slots hold no target
    const int64_t nt = plan.ntgt, nsrc = plan.nsrc;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (has_target) {
        const float4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    const int64_t pb = st.row_pair[leaf];
    const int np_row = near ? (int)(st.row_pair[leaf + 1] - pb) : 0;  // pairs in the row's stream
    const int nfl = np_row > 0 ? (np_row + kStPairs - 1) / kStPairs : 1;  // flushes per vector
    const int total = nfl * m;
    // the issue pointer (vector iv, flush ifl) and the source indices of that flush
    int iv = 0, ifl = 0;
    int2 ix0 = make_int2(-1, -1), ix1 = make_int2(-1, -1);
    auto load_idx = [&]() {
        const int i0 = ifl * kStPairs + lane, i1 = i0 + 32;
        ix0 = i0 < np_row ? st.idx[pb + i0] : make_int2(-1, -1);
        ix1 = i1 < np_row ? st.idx[pb + i1] : make_int2(-1, -1);
    };
    auto issue = [&](int b) {
        const float* qv = sq + (int64_t)iv * nsrc;
        const int64_t base = pb + (int64_t)ifl * kStPairs;
        const int npf = np_row - ifl * kStPairs;
        float* zq = reinterpret_cast<float*>(&szq[b][0]);
        if (lane < npf) {
            cp_async16_cg(&sxy[b][lane], st.xy + base + lane);
            cp_async8(zq + 4 * lane, st.zz + base + lane);
            cp_async4_zf(zq + 4 * lane + 2, qv + (ix0.x < 0 ? 0 : ix0.x), ix0.x < 0 ? 0 : 4);
            cp_async4_zf(zq + 4 * lane + 3, qv + (ix0.y < 0 ? 0 : ix0.y), ix0.y < 0 ? 0 : 4);
        }
        if (lane + 32 < npf) {
            cp_async16_cg(&sxy[b][lane + 32], st.xy + base + lane + 32);
            cp_async8(zq + 4 * (lane + 32), st.zz + base + lane + 32);
            cp_async4_zf(zq + 4 * (lane + 32) + 2, qv + (ix1.x < 0 ? 0 : ix1.x), ix1.x < 0 ? 0 : 4);
            cp_async4_zf(zq + 4 * (lane + 32) + 3, qv + (ix1.y < 0 ? 0 : ix1.y), ix1.y < 0 ? 0 : 4);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        if (V1) {
            if (++ifl < nfl) load_idx();  // lands while the flush being computed runs
        } else {
            if (++ifl == nfl) {
                ifl = 0;
                ++iv;
            }
            if (iv < m) load_idx();
        }
    };
    load_idx();
    for (int f = 0; f < NB - 1; ++f) {  // the first NB - 1 flushes in flight (empty groups past the end)
        if (f < total) issue(f);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    double aphi = 0.0, ag0 = 0.0, ag1 = 0.0, ag2 = 0.0;
    int cv = 0, cfl = 0;  // the flush being computed
    for (int f = 0; f < total; ++f) {
        const int b = f % NB;
        // flush f has landed once at most NB - 2 younger groups are pending
        asm volatile("cp.async.wait_group %0;" ::"n"(NB - 2) : "memory");
        __syncwarp();
        // buffer (f + NB - 1) % NB was last read by flush f - 1; an empty group keeps the count
        if (f + NB - 1 < total) issue((f + NB - 1) % NB);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        const int rem = np_row - cfl * kStPairs;
        const int npairs = rem < kStPairs ? rem : kStPairs;
        float2 pphi = f2(0.f, 0.f), pg0 = f2(0.f, 0.f), pg1 = f2(0.f, 0.f), pg2 = f2(0.f, 0.f);
        auto step = [&](int i) {
            const float4 a = sxy[b][i];
            const float4 c = szq[b][i];
            const float2 dx = __fadd2_rn(f2(a.x, a.y), ntx);
            const float2 dy = __fadd2_rn(f2(a.z, a.w), nty);
            const float2 dz = __fadd2_rn(f2(c.x, c.y), ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float ri0 = fminf(rsqrtf(r2.x), rmax);
            const float ri1 = fminf(rsqrtf(r2.y), rmax);
            const float2 rinv = f2(ri0, ri1);
            const float2 qr = __fmul2_rn(f2(c.z, c.w), rinv);
            pphi = __fadd2_rn(pphi, qr);
            if (GRAD) {
                const float2 qr3 = __fmul2_rn(__fmul2_rn(qr, rinv), rinv);
                pg0 = __ffma2_rn(qr3, dx, pg0);
                pg1 = __ffma2_rn(qr3, dy, pg1);
                pg2 = __ffma2_rn(qr3, dz, pg2);
            }
        };
        if (K == 1) {  // the common item of one target a lane: a unit stride (11 % faster)
#pragma unroll 16
            for (int i = 0; i < npairs; ++i) step(i);
        } else if (KS) {  // a constant stride
#pragma unroll 8
            for (int i = kk; i < npairs; i += KS) step(i);
        } else {
#pragma unroll 2
            for (int i = kk; i < npairs; i += K) step(i);
        }
        aphi += (double)pphi.x;
        aphi += (double)pphi.y;
        if (GRAD) {
            ag0 += (double)pg0.x;
            ag0 += (double)pg0.y;
            ag1 += (double)pg1.x;
            ag1 += (double)pg1.y;
            ag2 += (double)pg2.x;
            ag2 += (double)pg2.y;
        }
        __syncwarp();  // buffer b is read before it is refilled or reused below
        const int v = cv;
        const bool last = cfl == nfl - 1;
        if (++cfl == nfl) {
            cfl = 0;
            ++cv;
        }
        if (!last) continue;
        // ---- the last flush of vector v: finish its targets ----
        if (K > 1) {  // the target's K partial sums, in kk order, through buffer b
            double(*red)[32] = reinterpret_cast<double(*)[32]>(&sxy[b][0]);
            red[0][lane] = aphi;
            red[1][lane] = ag0;
            red[2][lane] = ag1;
            red[3][lane] = ag2;
            __syncwarp();
            if (valid)
                for (int j = 1; j < K; ++j) {
                    aphi += red[0][ti + ns * j];
                    ag0 += red[1][ti + ns * j];
                    ag1 += red[2][ti + ns * j];
                    ag2 += red[3][ti + ns * j];
                }
            __syncwarp();
        }
        if (valid) {
            if (near) close_sum_add<GRAD>(close, (int64_t)v * nt + t, aphi, ag0, ag1, ag2);
            if (accumulate == 2) {
                out_phi[(int64_t)v * nt + t] = aphi;
                if (GRAD) {
                    double* o = out_g + ((int64_t)v * nt + t) * 3;
                    o[0] = ag0;
                    o[1] = ag1;
                    o[2] = ag2;
                }
            } else if (accumulate) {
                far_phi[(int64_t)v * nt + t] = far_phi[(int64_t)v * nt + t] + aphi;
                if (GRAD) {
                    double* fg = far_g + ((int64_t)v * nt + t) * 3;
                    fg[0] = fg[0] + ag0;
                    fg[1] = fg[1] + ag1;
                    fg[2] = fg[2] + ag2;
                }
            } else {
                const double ph = far_phi[(int64_t)v * nt + t] + aphi;
                const int64_t i = plan.tgt_perm[t];
                out_phi[(int64_t)v * nt + i] = ph / phi_scale;
                if (GRAD) {
                    const double* fg = far_g + ((int64_t)v * nt + t) * 3;
                    double* o = out_g + ((int64_t)v * nt + i) * 3;
                    o[0] = (fg[0] + ag0) / g_scale;
                    o[1] = (fg[1] + ag1) / g_scale;
                    o[2] = (fg[2] + ag2) / g_scale;
                }
            }
        }
        aphi = ag0 = ag1 = ag2 = 0.0;
    }
}

// The streamed P2P over a work list of items of 32 / KS slots: W warps a block, a warp an
// item.  (One kernel for every split, each item's taken from its slots, measured slower:
// sphere 4e6 2.32 against 1.94 ms.)
template <bool GRAD, int W, bool V1, int KS>
__global__ void __launch_bounds__(32 * W, 32 / W) p2p_st_kernel(P2pStArgs a) {
    __shared__ float4 sxy[W][kStBufs][kStPairs];  // (x0, x1, y0, y1), NB flushes
    __shared__ float4 szq[W][kStBufs][kStPairs];  // (z0, z1, q0, q1)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * W + warp;
    if (item >= a.items.count) return;
    p2p_st_item<GRAD, V1, KS>(a, item, sxy[warp], szq[warp], lane);
}

// Host: the streamed P2P with gradients over a work list on stream s (p2p_launch.cu, its
// own translation unit: these kernels depend on no expansion order): W = warps a block
// (1, 2 or 4), ks the split of every item (1, 2, 4 or 8; 0 any item).
void launch_p2p_st(const P2pStArgs& a, int warps, int ks, unsigned grid, cudaStream_t s);

// Potentials of several vectors from the stream: p2p_x2_mv_kernel's pair-steps (the pair
// geometry once, q rinv added per vector) on flushes copied from the stream.
template <int W>
__global__ void __launch_bounds__(32 * W, 20 / W) p2p_st_mv_kernel(
    DevPlan plan, P2pItems items, int m, int near, float rmax, P2pStream st, const float* __restrict__ sq,
    const float4* __restrict__ tpos, ClosePairs close, double* __restrict__ far_phi, int accumulate,
    double* __restrict__ out_phi) {
    constexpr int VB = kX2Vb;
    __shared__ float4 sxy[W][2][kStPairs];
    __shared__ float2 szz[W][2][kStPairs];
    __shared__ float2 sqq[W][2][VB][kStPairs];
    static_assert(VB * 32 * sizeof(double) <= sizeof(float4) * kStPairs, "reduction buffer");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * W + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    int ni, ns;
    item_shape(items, item, t1, ni, ns);
    const int K = 32 / ns;
    const int kk = lane < ns * K && lane % ns < ni ? lane / ns : K;
    const int ti = lane < ns * K ? lane % ns : 0;
    const int64_t t = items.t0[item] + ti;
    const bool valid = lane < ni;
    const int64_t nt = plan.ntgt, nsrc = plan.nsrc;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (kk < K) {
        const float4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const int64_t pb = st.row_pair[leaf];
    const int np_row = near ? (int)(st.row_pair[leaf + 1] - pb) : 0;
    const int nfl = np_row > 0 ? (np_row + kStPairs - 1) / kStPairs : 1;
    const int nvb = (m + VB - 1) / VB;
    const int total = nfl * nvb;
    int ivb = 0, ifl = 0;
    int2 ix0 = make_int2(-1, -1), ix1 = make_int2(-1, -1);
    auto load_idx = [&]() {
        const int i0 = ifl * kStPairs + lane, i1 = i0 + 32;
        ix0 = i0 < np_row ? st.idx[pb + i0] : make_int2(-1, -1);
        ix1 = i1 < np_row ? st.idx[pb + i1] : make_int2(-1, -1);
    };
    auto issue = [&](int b) {
        const int v0 = ivb * VB, nb = (m - v0) < VB ? (m - v0) : VB;
        const int64_t base = pb + (int64_t)ifl * kStPairs;
        const int npf = np_row - ifl * kStPairs;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = lane + 32 * h;
            const int2 ix = h ? ix1 : ix0;
            if (i < npf) {
                cp_async16_cg(&sxy[warp][b][i], st.xy + base + i);
                cp_async8(&szz[warp][b][i], st.zz + base + i);
#pragma unroll
                for (int vb = 0; vb < VB; ++vb)
                    if (vb < nb) {
                        const float* qv = sq + (int64_t)(v0 + vb) * nsrc;
                        float* d = reinterpret_cast<float*>(&sqq[warp][b][vb][i]);
                        cp_async4_zf(d, qv + (ix.x < 0 ? 0 : ix.x), ix.x < 0 ? 0 : 4);
                        cp_async4_zf(d + 1, qv + (ix.y < 0 ? 0 : ix.y), ix.y < 0 ? 0 : 4);
                    }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        if (++ifl == nfl) {
            ifl = 0;
            ++ivb;
        }
        if (ivb < nvb) load_idx();
    };
    load_idx();
    issue(0);
    double aphi[VB];
#pragma unroll
    for (int vb = 0; vb < VB; ++vb) aphi[vb] = 0.0;
    int cvb = 0, cfl = 0;
    for (int f = 0; f < total; ++f) {
        const int b = f & 1;
        const int v0 = cvb * VB, nb = (m - v0) < VB ? (m - v0) : VB;
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        if (f + 1 < total) issue(b ^ 1);
        const int rem = np_row - cfl * kStPairs;
        const int npairs = rem < kStPairs ? rem : kStPairs;
        float2 pphi[VB];
#pragma unroll
        for (int vb = 0; vb < VB; ++vb) pphi[vb] = f2(0.f, 0.f);
        auto step = [&](int i) {
            const float4 a = sxy[warp][b][i];
            const float2 zz = szz[warp][b][i];
            const float2 dx = __fadd2_rn(f2(a.x, a.y), ntx);
            const float2 dy = __fadd2_rn(f2(a.z, a.w), nty);
            const float2 dz = __fadd2_rn(zz, ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float ri0 = fminf(rsqrtf(r2.x), rmax);
            const float ri1 = fminf(rsqrtf(r2.y), rmax);
            const float2 rinv = f2(ri0, ri1);
#pragma unroll
            for (int vb = 0; vb < VB; ++vb)
                if (vb < nb) pphi[vb] = __fadd2_rn(pphi[vb], __fmul2_rn(sqq[warp][b][vb][i], rinv));
        };
        if (K == 1) {  // the common item of one target a lane: a unit stride
#pragma unroll 2
            for (int i = 0; i < npairs; ++i) step(i);
        } else {
#pragma unroll 2
            for (int i = kk; i < npairs; i += K) step(i);
        }
#pragma unroll
        for (int vb = 0; vb < VB; ++vb) {
            aphi[vb] += (double)pphi[vb].x;
            aphi[vb] += (double)pphi[vb].y;
        }
        __syncwarp();
        const bool last = cfl == nfl - 1;
        if (++cfl == nfl) {
            cfl = 0;
            ++cvb;
        }
        if (!last) continue;
        if (K > 1) {
            double(*red)[32] = reinterpret_cast<double(*)[32]>(&sxy[warp][b][0]);
#pragma unroll
            for (int vb = 0; vb < VB; ++vb) red[vb][lane] = aphi[vb];
            __syncwarp();
            if (valid)
                for (int j = 1; j < K; ++j)
#pragma unroll
                    for (int vb = 0; vb < VB; ++vb) aphi[vb] += red[vb][ti + ns * j];
            __syncwarp();
        }
        if (valid) {
#pragma unroll
            for (int vb = 0; vb < VB; ++vb) {
                if (vb >= nb) break;
                const int v = v0 + vb;
                if (near) close_sum_add1(close, (int64_t)v * nt + t, aphi[vb]);
                if (accumulate == 2) {
                    out_phi[(int64_t)v * nt + t] = aphi[vb];
                } else if (accumulate) {
                    far_phi[(int64_t)v * nt + t] = far_phi[(int64_t)v * nt + t] + aphi[vb];
                } else {
                    const double ph = far_phi[(int64_t)v * nt + t] + aphi[vb];
                    out_phi[(int64_t)v * nt + plan.tgt_perm[t]] = ph / phi_scale;
                }
            }
        }
#pragma unroll
        for (int vb = 0; vb < VB; ++vb) aphi[vb] = 0.0;
    }
}

}  // namespace fmmb
