// Device kernels of the FMM evaluation passes (one rank, one GPU).
//
// Data in HBM (all level-major, see plan.hpp):
//   multipoles / locals : [box][vector][(p+1)^2]            (T)
//   source points       : xyz as T4 (w unused) + charges [vector][point]  (leaf order)
//   target points       : xyz as T4                                       (leaf order)
//   far-field partials  : phi [vector][target], grad [vector][target][3]  (f64)
//   output              : caller order, phi [vector][target], grad [...][3] (f64)
// Every kernel adds into its output in a fixed order per output value, with no atomics,
// so two evaluations are bit-identical.
#pragma once

#include <cstdint>

#include "harmonics.cuh"
#include "leaf_far_x2.cuh"

namespace fmmb {

template <typename T>
struct Vec4;
template <>
struct Vec4<double> {
    using type = double4;
};
template <>
struct Vec4<float> {
    using type = float4;
};

struct DevPlan {
    int nlevels;
    double side;
    const int32_t* level;      // per box
    const uint32_t* idx;       // 3 per box
    const int32_t* parent;
    const int32_t* child_first;
    const int32_t* box_leaf;
    const int64_t* src_below;
    const int64_t* tgt_below;
    const int32_t* leaf_box;
    const int64_t* src_start;
    const int64_t* tgt_start;
    const int64_t* tgt_perm;
    const int64_t* src_perm;
    const int64_t *near_row, *w_row, *x_row, *v_row;
    const int32_t *near_col, *w_col, *x_col, *v_col, *v_off;
    int64_t nsrc, ntgt;
    const double* box_side;  // forests: the domain side of each box's tree (null: `side`)
};

// 2^e for |e| <= 126, built from the exponent field (exact, no library call)
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }
__device__ __forceinline__ double pow2d(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }
template <typename T>
__device__ __forceinline__ T pow2(int e);
template <>
__device__ __forceinline__ float pow2<float>(int e) { return pow2f(e); }
template <>
__device__ __forceinline__ double pow2<double>(int e) { return pow2d(e); }

// relative frame of box s seen from box t (CONVENTIONS 3.13 "Relative frames"):
// c = (C_L(s) - C_L(t)) 2^(l_t - L), r = 2^(l_t - l_s); exact in f32 and f64 (the
// integer difference has at most 17 bits and the scale is a power of two).
template <typename T>
__device__ __forceinline__ void rel_frame(const DevPlan& P, int s, int t, T c[3], T& r) {
    int ls = P.level[s], lt = P.level[t];
    int L = ls > lt ? ls : lt;
    const T scale = pow2<T>(lt - L);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int Cs = (int)((2u * P.idx[3 * s + k] + 1u) << (L - ls));
        int Ct = (int)((2u * P.idx[3 * t + k] + 1u) << (L - lt));
        c[k] = (T)(Cs - Ct) * scale;
    }
    r = pow2<T>(lt - ls);
}

// ---------------------------------------------------------------------------------
// Charge load: caller-order charges (m per point, point-major) -> leaf order [v][i].
// ---------------------------------------------------------------------------------
// (m vectors of a pass; the caller's array holds `stride` charges per point, the pass's
// first at q_caller[0])
template <typename T>
__global__ void charge_load_kernel(const double* __restrict__ q_caller, const int64_t* __restrict__ perm,
                                   int64_t n, int m, int stride, T* __restrict__ q_leaf, double* __restrict__ q64) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t c = perm[i];
    for (int v = 0; v < m; ++v) {
        double q = q_caller[c * stride + v];
        q_leaf[(int64_t)v * n + i] = (T)q;
        if (q64) q64[(int64_t)v * n + i] = q;  // the mixed form keeps f64 charges for its f64 pairs
    }
}

// ---------------------------------------------------------------------------------
// P2M (rows = leaves, source = the leaf itself, unit frame) and P2L (rows = boxes,
// sources = X-list leaves, frame (c(t|s), r(t|s))): one warp per row.  Each lane forms
// the harmonics of one source and writes conj(X) into shared memory; lanes then sum
// the 32 sources of a chunk per coefficient in source order.
//   multipole: M_n^m += q conj R_n^m(u);  local: L_n^m += q conj I_n^m((u - c)/r)
// ---------------------------------------------------------------------------------
template <int P, typename T, bool IRREG>
__global__ void __launch_bounds__(32) expand_kernel(DevPlan plan, int64_t row_begin, int64_t row_end,
                                                    const int32_t* __restrict__ rows, int m,
                                                    const typename Vec4<T>::type* __restrict__ spos,
                                                    const T* __restrict__ sq, T* __restrict__ out) {
    constexpr int NC = nc_of(P);
    extern __shared__ unsigned char smem_raw[];
    T* S = reinterpret_cast<T*>(smem_raw);  // [NC][32]
    T* Q = S + NC * 32;                     // [m][32]
    const int lane = threadIdx.x;
    const int64_t idx = row_begin + blockIdx.x;  // rows[idx] when a row list is given
    if (idx >= row_end) return;
    const int64_t row = rows ? rows[idx] : idx;
    int box, nent;
    int64_t ent0;
    if (!IRREG) {  // row = leaf
        box = plan.leaf_box[row];
        nent = 1;
        ent0 = 0;
        if (plan.src_below[box] == 0) return;
    } else {  // row = box
        box = (int)row;
        ent0 = plan.x_row[row];
        nent = (int)(plan.x_row[row + 1] - ent0);
        if (nent == 0) return;
    }
    T* outb = out + (int64_t)box * m * ms_of(P);
    bool first = true;
    for (int e = 0; e < nent; ++e) {
        int sleaf = IRREG ? plan.x_col[ent0 + e] : (int)row;
        T fc[3] = {T(0), T(0), T(0)};
        T fr = T(1);
        if (IRREG) rel_frame<T>(plan, box, plan.leaf_box[sleaf], fc, fr);  // (c(t|s), r(t|s))
        T finv = T(1) / fr;
        int64_t s0 = plan.src_start[sleaf], s1 = plan.src_start[sleaf + 1];
        for (int64_t cb = s0; cb < s1; cb += 32) {
            int64_t si = cb + lane;
            bool valid = si < s1;
            T x = T(0), y = T(0), z = T(1);
            if (valid) {
                auto p4 = spos[si];
                x = (p4.x - fc[0]) * finv;
                y = (p4.y - fc[1]) * finv;
                z = (p4.z - fc[2]) * finv;
            }
            for (int v = 0; v < m; ++v) Q[v * 32 + lane] = valid ? sq[(int64_t)v * plan.nsrc + si] : T(0);
            if constexpr (!IRREG && sizeof(T) == 4) {  // f32: the rows on the packed pipe (leaf_far_x2.cuh)
                RegularRows2<P> h;
                h.init((float)x, (float)y, (float)z);
#pragma unroll
                for (int n = 0; n <= P; ++n) {
                    h.step(n);
#pragma unroll
                    for (int mm = 0; mm <= n; ++mm) {
                        S[slot(n, mm) * 32 + lane] = valid ? (T)h.c[mm].x : T(0);
                        if (mm) S[slot(n, -mm) * 32 + lane] = valid ? (T)-h.c[mm].y : T(0);
                    }
                }
            } else if (!IRREG) {
                RegularRows<P, T> h;
                h.init(x, y, z);
#pragma unroll
                for (int n = 0; n <= P; ++n) {
                    h.step(n);
#pragma unroll
                    for (int mm = 0; mm <= n; ++mm) {
                        S[slot(n, mm) * 32 + lane] = valid ? h.cre[mm] : T(0);
                        if (mm) S[slot(n, -mm) * 32 + lane] = valid ? -h.cim[mm] : T(0);
                    }
                }
            } else {
                IrregularRows<P, T> h;
                T r2 = x * x + y * y + z * z;
                h.init(x, y, z, valid ? T(1) / sqrt(r2) : T(0));
#pragma unroll
                for (int n = 0; n <= P; ++n) {
                    h.step(n);
#pragma unroll
                    for (int mm = 0; mm <= n; ++mm) {
                        S[slot(n, mm) * 32 + lane] = valid ? h.cre[mm] : T(0);
                        if (mm) S[slot(n, -mm) * 32 + lane] = valid ? -h.cim[mm] : T(0);
                    }
                }
            }
            __syncwarp();
            int cnt = (int)((s1 - cb) < 32 ? (s1 - cb) : 32);
            for (int v = 0; v < m; ++v)
                for (int c = lane; c < NC; c += 32) {
                    T acc = T(0);
                    for (int j = 0; j < cnt; ++j) acc += Q[v * 32 + j] * S[c * 32 + j];
                    T* o = outb + (int64_t)v * ms_of(P) + c;
                    if (first && !IRREG) *o = acc;
                    else *o += acc;
                }
            first = false;
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------------
// P2M / P2L, f32 single-vector form: one warp per row; lane j takes source points
// j, j+32, ... of every entry and accumulates q conj(X) for all (p+1)^2 slots in
// registers; one butterfly reduce-scatter per row then leaves every lane with
// NCP/32 finished slots (NCP = slots padded to a multiple of 32).  The summation order
// is fixed (per-lane partial sums, then a fixed tree), so results are repeatable.
// ---------------------------------------------------------------------------------
// One X-list entry of the f32 P2L, fixed at build (x_record_kernel): the source leaf's
// frame seen from the target box, (c(t|s), r(t|s)) of rel_frame<float>, and its sources,
// so that an entry costs one load, issued while the entry before it is summed.
struct __align__(16) XRec {
    float4 frame;  // (c0, c1, c2, r)
    long long s0;  // the source leaf's first source (leaf order)
    int ns;        // its sources
    int pad;
};

// Build time: thread per X entry of the boxes of `rows` (x_row order).
static __global__ void x_record_kernel(DevPlan plan, const int32_t* __restrict__ rows, int64_t nrows,
                                       XRec* __restrict__ rec) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const int box = rows[r];
    for (int64_t e = plan.x_row[box]; e < plan.x_row[box + 1]; ++e) {
        const int sleaf = plan.x_col[e];
        float c[3], fr;
        rel_frame<float>(plan, box, plan.leaf_box[sleaf], c, fr);
        XRec x;
        x.frame = make_float4(c[0], c[1], c[2], fr);
        x.s0 = plan.src_start[sleaf];
        x.ns = (int)(plan.src_start[sleaf + 1] - plan.src_start[sleaf]);
        x.pad = 0;
        rec[e] = x;
    }
}

template <int P, bool IRREG, bool MULTI>
__global__ void __launch_bounds__(32) expand_bfly_kernel(DevPlan plan, int64_t row_begin, int64_t row_end,
                                                         const int32_t* __restrict__ rows,
                                                         const float4* __restrict__ spos, int m,
                                                         const float* __restrict__ sq, float* __restrict__ out,
                                                         const XRec* __restrict__ xrec = nullptr, int overwrite = 0) {
    constexpr int NC = nc_of(P);
    constexpr int NCP = ((NC + 31) / 32) * 32;
    const int lane = threadIdx.x;
    const int64_t idx = row_begin + blockIdx.x;  // rows[idx] when a row list is given
    if (idx >= row_end) return;
    const int64_t row = rows ? rows[idx] : idx;
    int box, nent;
    int64_t ent0;
    if (!IRREG) {
        // a leaf without sources keeps its zero multipole; the test reads the leaf's source
        // range, which needs no load of its box first (the box is read beside it)
        box = plan.leaf_box[row];
        nent = 1;
        ent0 = 0;
        if (plan.src_start[row + 1] == plan.src_start[row]) return;
    } else {
        box = (int)row;
        ent0 = plan.x_row[row];
        nent = (int)(plan.x_row[row + 1] - ent0);
        if (nent == 0) return;
    }
    // the charge vectors one after the other (charges [v][point], expansions [box][v]);
    // MULTI = false compiles the one-vector form (m = 1) without the loop's registers
    for (int v = 0; v < (MULTI ? m : 1); ++v) {
    const float* qv = sq + (int64_t)v * plan.nsrc;
    float w[NCP];
#pragma unroll
    for (int c = 0; c < NCP; ++c) w[c] = 0.0f;
    // P2L: the entries' records, the next one loaded while the current one is summed
    XRec xn{};
    if (IRREG) xn = xrec[ent0];
    for (int e = 0; e < nent; ++e) {
        float fc[3] = {0.0f, 0.0f, 0.0f}, fr = 1.0f;  // (c(t|s), r(t|s))
        int64_t s0, s1;
        if (IRREG) {
            const XRec xr = xn;
            if (e + 1 < nent) xn = xrec[ent0 + e + 1];
            fc[0] = xr.frame.x;
            fc[1] = xr.frame.y;
            fc[2] = xr.frame.z;
            fr = xr.frame.w;
            s0 = xr.s0;
            s1 = s0 + xr.ns;
        } else {
            s0 = plan.src_start[row];
            s1 = plan.src_start[row + 1];
        }
        const float finv = 1.0f / fr;
        // the lane's next source is loaded before its current one is summed
        int64_t si = s0 + lane;
        float4 pn = make_float4(0.f, 0.f, 0.f, 0.f);
        float qn = 0.f;
        if (si < s1) {
            pn = spos[si];
            qn = qv[si];
        }
        for (; si < s1; si += 32) {
            const float4 p4 = pn;
            const float q = qn;
            if (si + 32 < s1) {
                pn = spos[si + 32];
                qn = qv[si + 32];
            }
            const float x = (p4.x - fc[0]) * finv, y = (p4.y - fc[1]) * finv, z = (p4.z - fc[2]) * finv;
            // conj(X) q into the slots: (w[slot(n, mm)], w[slot(n, -mm)]) += (q, -q) * X_n^mm,
            // one packed fused multiply-add an order mm > 0 (the rows on the packed pipe,
            // leaf_far_x2.cuh)
            const float2 qq = make_float2(q, -q);
            auto scatter = [&](int n, const float2* cr) {
#pragma unroll
                for (int mm = 0; mm <= n; ++mm) {
                    if (mm == 0) {
                        w[slot(n, 0)] = fmaf(q, cr[0].x, w[slot(n, 0)]);
                    } else {
                        const float2 acc = __ffma2_rn(qq, cr[mm], make_float2(w[slot(n, mm)], w[slot(n, -mm)]));
                        w[slot(n, mm)] = acc.x;
                        w[slot(n, -mm)] = acc.y;
                    }
                }
            };
            if (!IRREG) {
                RegularRows2<P> h;
                h.init(x, y, z);
#pragma unroll
                for (int n = 0; n <= P; ++n) {
                    h.step(n);
                    scatter(n, h.c);
                }
            } else {
                IrregularRows2<P> h;
                h.init(x, y, z, rsqrtf(x * x + y * y + z * z));
#pragma unroll
                for (int n = 0; n <= P; ++n) {
                    h.step(n);
                    scatter(n, h.c);
                }
            }
        }
    }
    // reduce-scatter: after the step with offset s a lane keeps the half of its slots
    // selected by its bit s and adds the partner's copy of that half
#pragma unroll
    for (int s = 16, len = NCP / 2; s >= 1; s >>= 1, len >>= 1) {
        const bool upper = lane & s;
#pragma unroll
        for (int i = 0; i < len; ++i) {
            const float send = upper ? w[i] : w[i + len];
            const float keep = upper ? w[i + len] : w[i];
            w[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    int base = 0;
#pragma unroll
    for (int s = 16, len = NCP / 2; s >= 1; s >>= 1, len >>= 1)
        if (lane & s) base += len;
    float* o = out + ((int64_t)box * m + v) * ms_of(P);
#pragma unroll
    for (int i = 0; i < NCP / 32; ++i) {
        const int c = base + i;
        if (c < NC) {
            if (IRREG && !overwrite) o[c] += w[i];
            else o[c] = w[i];
        }
    }
    }
}

// ---------------------------------------------------------------------------------
// M2M and L2L run as batched GEMMs too (m2l_gemm_kernel with the 8 octant tables): the
// product for child c is written to row c of Yo (M2M: T_o M_c; L2L: T_o L_parent(c)).
// The reduces below then add rows in the reference's order.
// ---------------------------------------------------------------------------------

// M2M reduce for the parents of one level: M_p = sum over octants o (in order) of the
// products of its children that hold a source.  Block per parent, thread per slot.
template <int P, typename T>
__global__ void m2m_reduce_kernel(DevPlan plan, const int32_t* __restrict__ parents, int64_t n, int m,
                                  const T* __restrict__ Yo, T* __restrict__ M) {
    constexpr int NC = nc_of(P), YS = ys_of(P);
    const int64_t j = blockIdx.x;
    if (j >= n) return;
    const int p = parents[j];
    const int c0 = plan.child_first[p];
    for (int v = 0; v < m; ++v)
        for (int i = threadIdx.x; i < NC; i += blockDim.x) {
            T s = T(0);
#pragma unroll
            for (int o = 0; o < 8; ++o)
                if (plan.src_below[c0 + o]) s += Yo[((int64_t)(c0 + o) * m + v) * YS + i];
            M[((int64_t)p * m + v) * ms_of(P) + i] = s;
        }
}

// The locals of one level (>= 2), for every box with a target below it:
//   L = (l >= 3 ? T_o L_parent : 0) + the V row's products in offset-index order
// (the product of V entry e sits at row vpos[e] of Yv, its place in the M2L tile list),
// written once (fmm-plan/src/operator.rs:34-45: L2L, then V by offset; X is added after).
// Block per box, thread per slot; the V loop issues eight (then four) loads before adding them in order.
// The evaluation writes L = Yo + sum_V Y (accumulate = 0); the level calls add into L:
// L2L with with_v = 0, then M2L with with_l2l = 0, which gives the same floats when the
// L2L call comes first (L starts at zero, so 0 + Yo = Yo).
template <int P, typename T>
__global__ void local_reduce_kernel(DevPlan plan, int64_t b0, int64_t b1, int m, int with_l2l, int with_v,
                                    int accumulate, const T* __restrict__ Yo, const T* __restrict__ Yv,
                                    const int64_t* __restrict__ vpos, T* __restrict__ Lc) {
    constexpr int NC = nc_of(P), YS = ys_of(P);
    const int64_t b = b0 + blockIdx.x;
    if (b >= b1 || plan.tgt_below[b] == 0) return;
    const int64_t e0 = plan.v_row[b], e1 = with_v ? plan.v_row[b + 1] : e0;
    for (int v = 0; v < m; ++v)
        for (int i = threadIdx.x; i < NC; i += blockDim.x) {
            T s = accumulate ? Lc[(b * m + v) * ms_of(P) + i] : T(0);
            if (with_l2l) s = accumulate ? s + Yo[(b * m + v) * YS + i] : Yo[(b * m + v) * YS + i];
            int64_t e = e0;
            for (; e + 8 <= e1; e += 8) {  // eight rows in flight, added in row order
                T y[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) y[j] = __ldcs(Yv + (vpos[e + j] * m + v) * YS + i);
#pragma unroll
                for (int j = 0; j < 8; ++j) s += y[j];
            }
            for (; e + 4 <= e1; e += 4) {
                const T y0 = __ldcs(Yv + (vpos[e] * m + v) * YS + i), y1 = __ldcs(Yv + (vpos[e + 1] * m + v) * YS + i);
                const T y2 = __ldcs(Yv + (vpos[e + 2] * m + v) * YS + i), y3 = __ldcs(Yv + (vpos[e + 3] * m + v) * YS + i);
                s += y0;
                s += y1;
                s += y2;
                s += y3;
            }
            for (; e < e1; ++e) s += __ldcs(Yv + (vpos[e] * m + v) * YS + i);
            Lc[(b * m + v) * ms_of(P) + i] = s;
        }
}

// The same reduce for f32 expansions with 16-byte accesses: a warp per box (4 a block).
// A box's m rows (its m vectors) are m NQ consecutive quads in the locals, in Yo and in
// each of its V entries' products (ys_of = ms_of = 4 NQ), so the lanes take quads f, f + 32,
// ... of that run: every lane busy for any m (m = 16 at p = 6: 208 quads, 7 passes), 13 of
// 32 when the lanes held one vector's quads.  Every coefficient adds the same terms in the
// same order as local_reduce_kernel, so the floats are that kernel's.  The last quad of a
// row is read with its padding, which is never written.  Four blocks an SM in the launch
// bound leave room for sixteen 16-byte rows in flight.
__device__ __forceinline__ void add4(float4& s, const float4 y) {
    s.x += y.x;
    s.y += y.y;
    s.z += y.z;
    s.w += y.w;
}

template <int P, bool ONE>  // ONE: m = 1 at compile time
__global__ void __launch_bounds__(128, 4) local_reduce4_kernel(DevPlan plan, int64_t b0, int64_t b1, int m_,
                                                            int with_l2l, int with_v, int accumulate,
                                                            const float* __restrict__ Yo, const float* __restrict__ Yv,
                                                            const int64_t* __restrict__ vpos, float* __restrict__ Lc,
                                                            const float* __restrict__ Lx = nullptr) {
    constexpr int NC = nc_of(P), YS = ys_of(P), MS = ms_of(P), NQ = (NC + 3) / 4;
    static_assert(YS == MS && MS == 4 * NQ, "a box's m rows are m NQ consecutive quads");
    const int m = ONE ? 1 : m_;
    const int64_t b = b0 + (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (b >= b1 || plan.tgt_below[b] == 0) return;
    const int64_t e0 = plan.v_row[b], e1 = with_v ? plan.v_row[b + 1] : e0;
    const int F = m * NQ;  // the box's quads, all vectors
    // P2L computed apart (Lx, the box's X-list sum, written by the P2L kernel beside the
    // upward pass): added last, as the P2L kernel adds it to the stored locals otherwise
    const bool with_x = Lx && plan.x_row[b + 1] > plan.x_row[b];
    for (int f = threadIdx.x & 31; f < F; f += 32) {
        const int q = f % NQ;  // the quad within its vector's row
        float4* out = reinterpret_cast<float4*>(Lc + b * m * MS) + f;
        float4 s = accumulate ? *out : make_float4(0.f, 0.f, 0.f, 0.f);
        if (with_l2l) {
            const float4 y = reinterpret_cast<const float4*>(Yo + b * m * YS)[f];
            if (accumulate)
                add4(s, y);
            else
                s = y;
        }
        auto row = [&](int64_t e) { return __ldcs(reinterpret_cast<const float4*>(Yv + vpos[e] * m * YS) + f); };
        int64_t e = e0;
        for (; e + 16 <= e1; e += 16) {  // sixteen rows in flight, added in row order
            float4 y[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) y[j] = row(e + j);
#pragma unroll
            for (int j = 0; j < 16; ++j) add4(s, y[j]);
        }
        for (; e + 8 <= e1; e += 8) {
            float4 y[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) y[j] = row(e + j);
#pragma unroll
            for (int j = 0; j < 8; ++j) add4(s, y[j]);
        }
        for (; e + 4 <= e1; e += 4) {
            float4 y[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) y[j] = row(e + j);
#pragma unroll
            for (int j = 0; j < 4; ++j) add4(s, y[j]);
        }
        for (; e < e1; ++e) add4(s, row(e));
        if (with_x) add4(s, reinterpret_cast<const float4*>(Lx + b * m * MS)[f]);
        if (4 * q + 3 < NC) {
            *out = s;
        } else {  // the last quad: its coefficients below NC only (NC - 4q of them, 1 to 3)
            float* o = reinterpret_cast<float*>(out);
            o[0] = s.x;
            if (4 * q + 1 < NC) o[1] = s.y;
            if (4 * q + 2 < NC) o[2] = s.z;
        }
    }
}

// ---------------------------------------------------------------------------------
// Dense M2L as batched GEMM, SIMT form (f64 path): the V pairs of every level are
// grouped by offset index d (fmm-kernels/src/translate.rs:61-74 batches them the same
// way); a block takes a tile of up to 64 pairs of one offset, stages A_d (column-major,
// so row k of the staged array holds column k) and the tile's source multipoles in
// shared memory, and writes the products Y[e] = A_d M_s (e = the pair's position in
// the target's V row).  Each thread holds 4 pairs x 6 output slots in registers.
// ---------------------------------------------------------------------------------
constexpr int kGemmPairs = 64;

// one element global -> shared by an asynchronous copy; zero-filled when !valid (the source
// address is then not read)
template <typename T>
__device__ __forceinline__ void gemm_cp_async(T* smem, const T* gmem, bool valid) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t n = valid ? (uint32_t)sizeof(T) : 0u;
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(gmem), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(gmem), "r"(n) : "memory");
}

// Shared memory of the SIMT GEMM: the table (columns as rows, NCP wide) and the tile's
// source rows, KC input slots at a time.  KC = the matrix order (one staging) where both
// fit in 200 KB; at higher degree in f64 the input slots are staged in chunks of KC, the
// accumulators kept in registers across the chunks (the same order of additions).  CPLX:
// the Helmholtz form, a complex expansion as one real vector of 2 (p+1)^2 entries (the
// real plane, then the imaginary plane) and the table a real 2n x 2n matrix.
template <int P, typename T, bool CPLX = false>
struct GemmShape {
    static constexpr int NC = nc_of(P);
    static constexpr int NE = CPLX ? 2 * NC : NC;  // matrix order
    static constexpr int NCP = 96 > NE ? 96 : ((NE + 15) / 16) * 16;
    static constexpr int ROW_BYTES = (NCP + kGemmPairs) * (int)sizeof(T);
    static constexpr int KC_FIT = (200 * 1024) / ROW_BYTES;
    static constexpr int KC = KC_FIT < NE ? KC_FIT : NE;
    static constexpr int SMEM = KC * ROW_BYTES;
};

// Y[pair] = A_d X[source] for a tile of pairs of one matrix d (column-major NE x NE).
// Rows: a box holds MV = m (real) or 2m (CPLX: rows 2v and 2v + 1 the real and imaginary
// planes of vector v) expansion rows of ms_of(P) slots; a product holds MV rows of
// ys_of(P) slots.
template <int P, typename T, bool CPLX = false>
__global__ void __launch_bounds__(256) m2l_gemm_kernel(const int32_t* __restrict__ tile_d,
                                                       const int64_t* __restrict__ tile_begin,
                                                       const int32_t* __restrict__ tile_count,
                                                       const int64_t* __restrict__ pair_e,
                                                       const int32_t* __restrict__ pair_src, int m,
                                                       const T* __restrict__ tab, const T* __restrict__ M,
                                                       T* __restrict__ Y) {
    using S = GemmShape<P, T, CPLX>;
    constexpr int NC = S::NC, NE = S::NE, NCP = S::NCP, KC = S::KC;
    constexpr int JN = NCP / 16;
    constexpr bool kOneStage = KC == NE;
    const int mv = CPLX ? 2 * m : m;  // expansion rows a box
    extern __shared__ unsigned char smem_raw[];
    T* At = reinterpret_cast<T*>(smem_raw);  // [KC][NCP]: At[k][n] = A_d[n][k0 + k]
    T* Xs = At + KC * NCP;                   // [KC][64]:  Xs[k][pair]
    const int tile = blockIdx.x;
    const int d = tile_d[tile];
    const int64_t p0 = tile_begin[tile];
    const int cnt = tile_count[tile];
    const T* A = tab + (int64_t)d * NE * NE;
    // staging by asynchronous copies (every copy of the block in flight at once; padding
    // zero-filled): the table, then each vector's source rows once the tile's sources are
    // known; 256 threads
    __shared__ int32_t srcs[kGemmPairs];
    if (threadIdx.x < kGemmPairs) srcs[threadIdx.x] = threadIdx.x < cnt ? pair_src[p0 + threadIdx.x] : 0;
    auto stage_table = [&](int k0, int kc) {
        for (int t = threadIdx.x; t < kc * NCP; t += 256) {
            const int k = t / NCP, n = t % NCP;
            gemm_cp_async<T>(At + t, A + (int64_t)(k0 + k) * NE + (n < NE ? n : 0), n < NE);
        }
    };
    if (kOneStage) stage_table(0, NE);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    for (int v = 0; v < m; ++v) {
        const int vrow = CPLX ? 2 * v : v;
        T acc[4][JN];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < JN; ++j) acc[i][j] = T(0);
        for (int k0 = 0; k0 < NE; k0 += KC) {
            const int kc = NE - k0 < KC ? NE - k0 : KC;
            __syncthreads();  // srcs written; the previous chunk's or vector's staging read
            if (!kOneStage) stage_table(k0, kc);
            for (int t = threadIdx.x; t < kc * kGemmPairs; t += 256) {
                const int pr = t / kc, kk = k0 + t % kc;
                const int plane = CPLX ? kk / NC : 0, slot_ = CPLX ? kk % NC : kk;
                gemm_cp_async<T>(Xs + (t % kc) * kGemmPairs + pr,
                                 M + ((int64_t)srcs[pr] * mv + vrow + plane) * ms_of(P) + slot_, pr < cnt);
            }
            asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
            __syncthreads();
            if constexpr (sizeof(T) == 4) {
                // f32: two pairs' sums of one slot in one packed fused multiply-add (the
                // same fma a sum as the scalar loop below)
                float2 acc2[2][JN];
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < JN; ++j) acc2[i][j] = make_float2(acc[2 * i][j], acc[2 * i + 1][j]);
#pragma unroll 3
                for (int k = 0; k < kc; ++k) {
                    const float4 xv = *reinterpret_cast<const float4*>(Xs + k * kGemmPairs + ty * 4);
                    float av[JN];
#pragma unroll
                    for (int j = 0; j < JN; ++j) av[j] = At[k * NCP + tx + 16 * j];
#pragma unroll
                    for (int j = 0; j < JN; ++j) {
                        acc2[0][j] = __ffma2_rn(make_float2(av[j], av[j]), make_float2(xv.x, xv.y), acc2[0][j]);
                        acc2[1][j] = __ffma2_rn(make_float2(av[j], av[j]), make_float2(xv.z, xv.w), acc2[1][j]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < JN; ++j) {
                        acc[2 * i][j] = acc2[i][j].x;
                        acc[2 * i + 1][j] = acc2[i][j].y;
                    }
            } else {
#pragma unroll 3
                for (int k = 0; k < kc; ++k) {
                    T xv[4], av[JN];
#pragma unroll
                    for (int i = 0; i < 4; ++i) xv[i] = Xs[k * kGemmPairs + ty * 4 + i];
#pragma unroll
                    for (int j = 0; j < JN; ++j) av[j] = At[k * NCP + tx + 16 * j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < JN; ++j) acc[i][j] += av[j] * xv[i];
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int pr = ty * 4 + i;
            if (pr >= cnt) continue;
            const int64_t e = pair_e ? pair_e[p0 + pr] : p0 + pr;
#pragma unroll
            for (int j = 0; j < JN; ++j) {
                const int n = tx + 16 * j;
                if (n < NE) {
                    const int plane = CPLX ? n / NC : 0, slot_ = CPLX ? n % NC : n;
                    // read once by the reduce: stream past L2
                    __stcs(Y + (e * mv + vrow + plane) * ys_of(P) + slot_, acc[i][j]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// L2P (own local) then M2P (W list, by box index) for every target of a leaf.
// Gradients by the ladder identities, contracted with shifted coefficients:
//   (d/dx - i d/dy) phi = sum L_{k+1}^{mu+1} R_k^mu - conj(sum L_{k+1}^{mu-1} R_k^mu)
//   d/dz phi = sum w_mu Re(L_{k+1}^mu R_k^mu)          (L2P; M2P uses M_{k-1}, sign -)
// Results (phi_hat, g_hat in the leaf's units) go to the f64 far-field partials.
// ---------------------------------------------------------------------------------
// The weight 2 of the orders mu > 0 is applied once at the end: their terms add into
// their own sums (f1, dz1), the mu = 0 terms (real harmonics: no imaginary part) into f0,
// dz0, so a term costs two fused multiply-adds, not a product, a difference and a scaled add.
template <int P, typename T, bool GRAD>
__device__ __forceinline__ void l2p_eval(const T* L, T x, T y, T z, T& phi, T& gx, T& gy, T& gz) {
    RegularRows<P, T> h;
    h.init(x, y, z);
    T f0 = T(0), f1 = T(0), dz0 = T(0), dz1 = T(0), are = T(0), aim = T(0);
#pragma unroll
    for (int k = 0; k <= P; ++k) {
        h.step(k);
#pragma unroll
        for (int mu = 0; mu <= k; ++mu) {
            Cx<T> c = coef_at(L, k, mu);
            if (mu == 0) {
                f0 += c.re * h.cre[0];
            } else {
                f1 += c.re * h.cre[mu];
                f1 -= c.im * h.cim[mu];
            }
            if (GRAD && k < P) {
                Cx<T> c1 = coef_at(L, k + 1, mu);
                if (mu == 0) {
                    dz0 += c1.re * h.cre[0];
                } else {
                    dz1 += c1.re * h.cre[mu];
                    dz1 -= c1.im * h.cim[mu];
                }
                Cx<T> up = coef_at(L, k + 1, mu + 1);
                are += up.re * h.cre[mu] - up.im * h.cim[mu];
                aim += up.re * h.cim[mu] + up.im * h.cre[mu];
                if (mu >= 1) {
                    Cx<T> dn = coef_at(L, k + 1, mu - 1);
                    are -= dn.re * h.cre[mu] - dn.im * h.cim[mu];
                    aim += dn.re * h.cim[mu] + dn.im * h.cre[mu];  // minus conj
                }
            }
        }
    }
    phi = f0 + T(2) * f1;
    gx = are;
    gy = -aim;
    gz = dz0 + T(2) * dz1;
}

template <int P, typename T, bool GRAD>
__device__ __forceinline__ void m2p_eval(const T* M, T x, T y, T z, T& phi, T& gx, T& gy, T& gz) {
    constexpr int KMAX = GRAD ? P + 1 : P;
    IrregularRows<P, T> h;
    T r2 = x * x + y * y + z * z;
    h.init(x, y, z, T(1) / sqrt(r2));
    // the orders mu > 0 into their own sums, weighted 2 at the end (as l2p_eval)
    T f0 = T(0), f1 = T(0), dz0 = T(0), dz1 = T(0), are = T(0), aim = T(0);
#pragma unroll
    for (int k = 0; k <= KMAX; ++k) {
        h.step(k);
#pragma unroll
        for (int mu = 0; mu <= k; ++mu) {
            if (k <= P) {
                Cx<T> c = coef_at(M, k, mu);
                if (mu == 0) {
                    f0 += c.re * h.cre[0];
                } else {
                    f1 += c.re * h.cre[mu];
                    f1 -= c.im * h.cim[mu];
                }
            }
            if (GRAD && k >= 1) {
                Cx<T> c1 = coef_at(M, k - 1, mu);
                if (mu == 0) {
                    dz0 -= c1.re * h.cre[0];
                } else {
                    dz1 -= c1.re * h.cre[mu];
                    dz1 += c1.im * h.cim[mu];
                }
                if (mu <= k - 2) {
                    Cx<T> up = coef_at(M, k - 1, mu + 1);
                    are += up.re * h.cre[mu] - up.im * h.cim[mu];
                    aim += up.re * h.cim[mu] + up.im * h.cre[mu];
                }
                if (mu >= 1) {
                    Cx<T> dn = coef_at(M, k - 1, mu - 1);
                    are -= dn.re * h.cre[mu] - dn.im * h.cim[mu];
                    aim += dn.re * h.cim[mu] + dn.im * h.cre[mu];
                }
            }
        }
    }
    phi = f0 + T(2) * f1;
    gx = are;
    gy = -aim;
    gz = dz0 + T(2) * dz1;
}

// mode: bit 0 L2P, bit 1 M2P, bit 2 add into far_phi / far_g (else overwrite them).
// The evaluation runs mode 3; the level calls run 5 (L2P) then 6 (M2P) on stores that
// start at zero, which gives the same floats.
template <int P, typename T, bool GRAD>
__global__ void __launch_bounds__(128) leaf_far_kernel(DevPlan plan, int64_t leaf0, int mode, int m,
                                                      const typename Vec4<T>::type* __restrict__ tpos,
                                                      const T* __restrict__ M, const T* __restrict__ Lc,
                                                      double* __restrict__ far_phi, double* __restrict__ far_g) {
    constexpr int NC = nc_of(P);
    // f32: the expansions are read straight from global memory (every thread reads the same
    // coefficient at the same time: one broadcast through L1, no block barrier); f64 stages
    // each expansion in shared memory (measured faster for 8-byte coefficients)
    constexpr bool kStage = sizeof(T) == 8;
    extern __shared__ unsigned char smem_raw[];
    T* C = reinterpret_cast<T*>(smem_raw);  // [NC] when staged
    const int64_t leaf = leaf0 + blockIdx.x;
    const int box = plan.leaf_box[leaf];
    const int64_t t0 = plan.tgt_start[leaf], t1 = plan.tgt_start[leaf + 1];
    if (t1 == t0) return;
    const int64_t w0 = plan.w_row[leaf], w1 = (mode & 2) ? plan.w_row[leaf + 1] : plan.w_row[leaf];
    const int64_t nt = plan.ntgt;
    for (int v = 0; v < m; ++v) {
        for (int64_t tb = t0; tb < t1; tb += blockDim.x) {
            int64_t t = tb + threadIdx.x;
            bool valid = t < t1;
            T ux = T(0), uy = T(0), uz = T(0);
            if (valid) {
                auto p4 = tpos[t];
                ux = p4.x;
                uy = p4.y;
                uz = p4.z;
            }
            double fphi = 0.0, fg[3] = {0.0, 0.0, 0.0};
            if ((mode & 4) && valid) {
                fphi = far_phi[(int64_t)v * nt + t];
                if (GRAD)
                    for (int k = 0; k < 3; ++k) fg[k] = far_g[((int64_t)v * nt + t) * 3 + k];
            }
            // L2P, unit frame
            if (mode & 1) {
                const T* Lb = Lc + ((int64_t)box * m + v) * ms_of(P);
                if (kStage) {
                    for (int k = threadIdx.x; k < NC; k += blockDim.x) C[k] = Lb[k];
                    __syncthreads();
                    Lb = C;
                }
                if (valid) {
                    T ph, gx, gy, gz;
                    l2p_eval<P, T, GRAD>(Lb, ux, uy, uz, ph, gx, gy, gz);
                    fphi = (mode & 4) ? fphi + (double)ph : (double)ph;
                    if (GRAD) {
                        fg[0] = (mode & 4) ? fg[0] + (double)gx : (double)gx;
                        fg[1] = (mode & 4) ? fg[1] + (double)gy : (double)gy;
                        fg[2] = (mode & 4) ? fg[2] + (double)gz : (double)gz;
                    }
                }
                if (kStage) __syncthreads();
            }
            // M2P over the W list, frame (c(s|t), r(s|t))
            for (int64_t e = w0; e < w1; ++e) {
                int s = plan.w_col[e];
                const T* Mb = M + ((int64_t)s * m + v) * ms_of(P);
                if (kStage) {
                    for (int k = threadIdx.x; k < NC; k += blockDim.x) C[k] = Mb[k];
                    __syncthreads();
                    Mb = C;
                }
                if (valid) {
                    T c[3], r;
                    rel_frame<T>(plan, s, box, c, r);
                    T rinv = T(1) / r;
                    T ph, gx, gy, gz;
                    m2p_eval<P, T, GRAD>(Mb, (ux - c[0]) * rinv, (uy - c[1]) * rinv, (uz - c[2]) * rinv, ph, gx,
                                         gy, gz);
                    fphi += (double)(ph * rinv);
                    if (GRAD) {
                        T r2inv = rinv * rinv;
                        fg[0] += (double)(gx * r2inv);
                        fg[1] += (double)(gy * r2inv);
                        fg[2] += (double)(gz * r2inv);
                    }
                }
                if (kStage) __syncthreads();
            }
            if (valid) {
                far_phi[(int64_t)v * nt + t] = fphi;
                if (GRAD) {
                    double* g = far_g + ((int64_t)v * nt + t) * 3;
                    g[0] = fg[0];
                    g[1] = fg[1];
                    g[2] = fg[2];
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// L2P + M2P of the potentials for several charge vectors (f32, m > 1): the harmonics of a
// target are formed once per W entry (and once for L2P) and dotted with VB vectors'
// expansions, which are consecutive rows of ms_of(P) floats.  Per vector the terms are
// those of l2p_eval / m2p_eval, with the harmonic rows on the packed f32x2 pipe and each
// order mu > 0 one packed fused multiply-add (real and imaginary products summed apart).
template <int P, int VB>
__device__ __forceinline__ void l2p_eval_mv(const float* L, int nb, float x, float y, float z, float (&f)[VB]) {
    constexpr int MS = ms_of(P);
    RegularRows2<P> h;  // the rows on the packed pipe (leaf_far_x2.cuh)
    h.init(x, y, z);
    float2 f1[VB];  // the orders mu > 0, real and imaginary products apart, weighted 2 at the end
#pragma unroll
    for (int b = 0; b < VB; ++b) {
        f[b] = 0.0f;
        f1[b] = make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int k = 0; k <= P; ++k) {
        h.step(k);
#pragma unroll
        for (int mu = 0; mu <= k; ++mu) {
#pragma unroll
            for (int b = 0; b < VB; ++b)
                if (b < nb) {
                    const Cx<float> c = coef_at(L + b * MS, k, mu);
                    if (mu == 0)
                        f[b] = fmaf(c.re, h.c[0].x, f[b]);
                    else
                        f1[b] = __ffma2_rn(make_float2(c.re, c.im), h.c[mu], f1[b]);
                }
        }
    }
#pragma unroll
    for (int b = 0; b < VB; ++b) f[b] += 2.0f * (f1[b].x - f1[b].y);
}

template <int P, int VB>
__device__ __forceinline__ void m2p_eval_mv(const float* M, int nb, float x, float y, float z, float (&f)[VB]) {
    constexpr int MS = ms_of(P);
    IrregularRows2<P> h;
    const float r2 = x * x + y * y + z * z;
    h.init(x, y, z, 1.0f / sqrt(r2));
    float2 f1[VB];
#pragma unroll
    for (int b = 0; b < VB; ++b) {
        f[b] = 0.0f;
        f1[b] = make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int k = 0; k <= P; ++k) {
        h.step(k);
#pragma unroll
        for (int mu = 0; mu <= k; ++mu) {
#pragma unroll
            for (int b = 0; b < VB; ++b)
                if (b < nb) {
                    const Cx<float> c = coef_at(M + b * MS, k, mu);
                    if (mu == 0)
                        f[b] = fmaf(c.re, h.c[0].x, f[b]);
                    else
                        f1[b] = __ffma2_rn(make_float2(c.re, c.im), h.c[mu], f1[b]);
                }
        }
    }
#pragma unroll
    for (int b = 0; b < VB; ++b) f[b] += 2.0f * (f1[b].x - f1[b].y);
}

// ---------------------------------------------------------------------------------
// P2P + output pass.  One warp per work item = up to 32 targets of one leaf (lane =
// target); the warp walks the leaf's near row (source leaves by leaf index) and stages
// each source leaf's points in its own shared memory, mapped to the target leaf's
// frame: y = fma(r, u_s, c) (CONVENTIONS 3.13 "Device kernels", rule 1), the leaf
// itself unchanged.  Per pair d = u_t - y, r2 by explicit fma (rules 2-3), and the
// pair is skipped by a select before rho meets a charge (rule 4): iff r2 == 0, the
// coincidence rule of the reference.  This is the plain f64 kernel; the mixed form's
// P2P is in p2p_x2.cuh (its near-singular pairs found by close_pairs_kernel below, whose
// f32 r2 is formed with pair_r2).  The per-target sum is added to the far-field partial
// and scaled once, phi = phi_hat/(4 pi r_t) and g = g_hat/((4 pi r_t) r_t)
// (fmm-exec/src/fmm.rs:4750-4778), in caller order.
// ---------------------------------------------------------------------------------
constexpr int kP2pWarps = 4;
constexpr int kP2pStage = 64;

template <typename T>
__device__ __forceinline__ T map_coord(T r, T u, T c);
template <>
__device__ __forceinline__ float map_coord<float>(float r, float u, float c) { return __fmaf_rn(r, u, c); }
template <>
__device__ __forceinline__ double map_coord<double>(double r, double u, double c) { return __fma_rn(r, u, c); }

template <typename T>
__device__ __forceinline__ T pair_r2(T dx, T dy, T dz);
template <>
__device__ __forceinline__ float pair_r2<float>(float dx, float dy, float dz) {
    return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}
template <>
__device__ __forceinline__ double pair_r2<double>(double dx, double dy, double dz) {
    return __fma_rn(dx, dx, __fma_rn(dy, dy, __dmul_rn(dz, dz)));
}
template <typename T>
__device__ __forceinline__ T sub_rn(T a, T b);
template <>
__device__ __forceinline__ float sub_rn<float>(float a, float b) { return __fsub_rn(a, b); }
template <>
__device__ __forceinline__ double sub_rn<double>(double a, double b) { return __dsub_rn(a, b); }

struct P2pItems {
    const int32_t* leaf;  // work item -> target leaf
    const int64_t* t0;    // work item -> first target (leaf order)
    int64_t count;
    // work item -> its targets (1 to 32) | its lane slots << 8 (a power of two >= the
    // targets, 0: the targets); null: up to 32 targets, to the leaf's end, in as many slots
    const int32_t* n = nullptr;
};

// The targets ni of a work item and its slots ns: the lanes are ns targets x K = 32 / ns
// pair-step splits (lane = kk ns + ti), so an item padded to ns > ni slots splits its
// pairs as an item of ns targets would, and lanes with ti >= ni hold no target.
__device__ __forceinline__ void item_shape(const P2pItems& items, int64_t item, int64_t t1, int& ni, int& ns) {
    if (items.n) {
        const int v = items.n[item];
        ni = v & 255;
        ns = (v >> 8) ? (v >> 8) : ni;
        return;
    }
    const int64_t r = t1 - items.t0[item];
    ni = ns = (int)(r < 32 ? r : 32);
}

// L2P + M2P of the f32 form over P2P work items: a warp per item (up to 32 targets of one
// leaf, lane = target), any number of warps a block.  Each target sums the terms of
// leaf_far_kernel<P, float, GRAD> in the same order (the compiler may contract products
// into fmas differently, so the last bits can differ); what changes is the occupancy: a
// block per leaf holds every thread of its block while a leaf of few targets keeps one
// warp busy, a warp per item leaves no idle warp resident.  leaf_far_mv_items_kernel forms
// each target's harmonics once for up to VB vectors (l2p_eval_mv / m2p_eval_mv).
// The gradient form is held to 96 registers up to p = 8 (21 warps an SM, no spills) and to
// 168 above (12 warps an SM; no spills to p = 12).
// With gradients (the mixed form's only use of this kernel) the terms run on the packed
// f32x2 pipe, coefficient by coefficient (l2p_x2 / m2p_x2, leaf_far_x2.cuh).
template <int P, bool GRAD>
__global__ void __launch_bounds__(128, P <= 8 ? 5 : 3) leaf_far_items_kernel(DevPlan plan, P2pItems items, int mode, int m,
                                                             const float4* __restrict__ tpos,
                                                             const float* __restrict__ M, const float* __restrict__ Lc,
                                                             double* __restrict__ far_phi, double* __restrict__ far_g) {
    static_assert(GRAD, "potentials: leaf_far_mv_items_kernel");
    const int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int64_t t = items.t0[item] + (threadIdx.x & 31);
    if (t >= plan.tgt_start[leaf + 1]) return;
    const int box = plan.leaf_box[leaf];
    const int64_t w0 = plan.w_row[leaf], w1 = (mode & 2) ? plan.w_row[leaf + 1] : plan.w_row[leaf];
    const int64_t nt = plan.ntgt;
    const float4 p4 = tpos[t];
    for (int v = 0; v < m; ++v) {
        // an opaque copy of the position each vector: the harmonics are formed per
        // evaluation in registers, never hoisted out of this loop as invariants (which held
        // every row of them live across it and spilled)
        float ux = p4.x, uy = p4.y, uz = p4.z;
        asm volatile("" : "+f"(ux), "+f"(uy), "+f"(uz));
        double fphi = 0.0, fg[3] = {0.0, 0.0, 0.0};
        if (mode & 4) {
            fphi = far_phi[(int64_t)v * nt + t];
            for (int k = 0; k < 3; ++k) fg[k] = far_g[((int64_t)v * nt + t) * 3 + k];
        }
        if (mode & 1) {
            float ph, gx, gy, gz;
            l2p_x2<P>(Lc + ((int64_t)box * m + v) * ms_of(P), ux, uy, uz, ph, gx, gy, gz);
            fphi = (mode & 4) ? fphi + (double)ph : (double)ph;
            fg[0] = (mode & 4) ? fg[0] + (double)gx : (double)gx;
            fg[1] = (mode & 4) ? fg[1] + (double)gy : (double)gy;
            fg[2] = (mode & 4) ? fg[2] + (double)gz : (double)gz;
        }
        for (int64_t e = w0; e < w1; ++e) {
            const int s = plan.w_col[e];
            float c[3], r;
            rel_frame<float>(plan, s, box, c, r);
            const float rinv = 1.0f / r;
            float ph, gx, gy, gz;
            m2p_x2<P>(M + ((int64_t)s * m + v) * ms_of(P), (ux - c[0]) * rinv, (uy - c[1]) * rinv,
                      (uz - c[2]) * rinv, ph, gx, gy, gz);
            fphi += (double)(ph * rinv);
            const float r2inv = rinv * rinv;
            fg[0] += (double)(gx * r2inv);
            fg[1] += (double)(gy * r2inv);
            fg[2] += (double)(gz * r2inv);
        }
        far_phi[(int64_t)v * nt + t] = fphi;
        double* g = far_g + ((int64_t)v * nt + t) * 3;
        g[0] = fg[0];
        g[1] = fg[1];
        g[2] = fg[2];
    }
}

template <int P, int VB>
__global__ void __launch_bounds__(128) leaf_far_mv_items_kernel(DevPlan plan, P2pItems items, int mode, int m,
                                                                const float4* __restrict__ tpos,
                                                                const float* __restrict__ M,
                                                                const float* __restrict__ Lc,
                                                                double* __restrict__ far_phi) {
    constexpr int MS = ms_of(P);
    const int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int64_t t = items.t0[item] + (threadIdx.x & 31);
    if (t >= plan.tgt_start[leaf + 1]) return;
    const int box = plan.leaf_box[leaf];
    const int64_t w0 = plan.w_row[leaf], w1 = (mode & 2) ? plan.w_row[leaf + 1] : plan.w_row[leaf];
    const int64_t nt = plan.ntgt;
    const float4 p4 = tpos[t];
    const float ux = p4.x, uy = p4.y, uz = p4.z;
    for (int v0 = 0; v0 < m; v0 += VB) {
        const int nb = (m - v0) < VB ? (m - v0) : VB;
        double fphi[VB];
#pragma unroll
        for (int b = 0; b < VB; ++b) fphi[b] = (b < nb && (mode & 4)) ? far_phi[(int64_t)(v0 + b) * nt + t] : 0.0;
        if (mode & 1) {
            float ph[VB];
            l2p_eval_mv<P, VB>(Lc + ((int64_t)box * m + v0) * MS, nb, ux, uy, uz, ph);
#pragma unroll
            for (int b = 0; b < VB; ++b) fphi[b] = (mode & 4) ? fphi[b] + (double)ph[b] : (double)ph[b];
        }
        for (int64_t e = w0; e < w1; ++e) {
            const int s = plan.w_col[e];
            float c[3], r;
            rel_frame<float>(plan, s, box, c, r);
            const float rinv = 1.0f / r;
            float ph[VB];
            m2p_eval_mv<P, VB>(M + ((int64_t)s * m + v0) * MS, nb, (ux - c[0]) * rinv, (uy - c[1]) * rinv,
                               (uz - c[2]) * rinv, ph);
#pragma unroll
            for (int b = 0; b < VB; ++b) fphi[b] += (double)(ph[b] * rinv);
        }
#pragma unroll
        for (int b = 0; b < VB; ++b)
            if (b < nb) far_phi[(int64_t)(v0 + b) * nt + t] = fphi[b];
    }
}

struct ClosePairs {  // near-singular pairs of the mixed form, CSR by target (leaf order)
    const int64_t* row;
    const int64_t* src;   // source point (leaf order)
    const int32_t* leaf;  // its source leaf
    const double4* spos;  // f64 leaf-scaled coordinates
    const double4* tpos;
    const double* q;      // f64 charges in leaf order [vector][point]
    const double4* y;     // the source point in the target leaf's frame (f64), per pair
    // mixed Laplace P2P: per target the f64 sum over its pairs of q times the pair's
    // weight (close_sum_kernel), [vector][target], 4 doubles (phi, grad) or 1 (phi)
    const double* acc;
};

// Build time (mixed form): each near-singular pair's source point mapped into its target
// leaf's frame in f64, y = fma(r, u, c) with the exact relative frame (the identity for the
// leaf itself), as the evaluation would form it.  Block per leaf.
static __global__ void close_map_kernel(DevPlan plan, ClosePairs close, double4* __restrict__ y) {
    const int64_t leaf = blockIdx.x;
    const int box = plan.leaf_box[leaf];
    for (int64_t t = plan.tgt_start[leaf] + threadIdx.x; t < plan.tgt_start[leaf + 1]; t += blockDim.x)
        for (int64_t c2 = close.row[t]; c2 < close.row[t + 1]; ++c2) {
            const int sl = close.leaf[c2];
            const double4 ps = close.spos[close.src[c2]];
            const double sw = (double)close.src[c2];  // w: the source's index (exact below 2^53)
            if (sl == leaf) {
                y[c2] = make_double4(ps.x, ps.y, ps.z, sw);
            } else {
                double cc[3], rr;
                rel_frame<double>(plan, plan.leaf_box[sl], box, cc, rr);
                y[c2] = make_double4(__fma_rn(rr, ps.x, cc[0]), __fma_rn(rr, ps.y, cc[1]), __fma_rn(rr, ps.z, cc[2]), sw);
            }
        }
}

template <typename T, bool GRAD>
__global__ void __launch_bounds__(128) p2p_kernel(DevPlan plan, P2pItems items, int m, int near, T theta2,
                                                  const typename Vec4<T>::type* __restrict__ spos,
                                                  const T* __restrict__ sq,
                                                  const typename Vec4<T>::type* __restrict__ tpos, ClosePairs close,
                                                  double* __restrict__ far_phi, double* __restrict__ far_g,
                                                  int accumulate, double* __restrict__ out_phi,
                                                  double* __restrict__ out_g) {
    using T4 = typename Vec4<T>::type;
    __shared__ T4 stage[kP2pWarps][kP2pStage];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * kP2pWarps + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    const int64_t t = items.t0[item] + lane;
    const bool valid = t < t1;
    const int64_t n0 = plan.near_row[leaf], n1 = near ? plan.near_row[leaf + 1] : n0;
    const int64_t nt = plan.ntgt;
    T tx = T(0), ty = T(0), tz = T(0);
    if (valid) {
        T4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    for (int v = 0; v < m; ++v) {
        double aphi = 0.0, ag0 = 0.0, ag1 = 0.0, ag2 = 0.0;
        for (int64_t e = n0; e < n1; ++e) {
            const int sl = plan.near_col[e];
            T c[3] = {T(0), T(0), T(0)}, r = T(1);
            const bool self = sl == leaf;
            if (!self) rel_frame<T>(plan, plan.leaf_box[sl], box, c, r);
            const int64_t s0 = plan.src_start[sl], s1 = plan.src_start[sl + 1];
            for (int64_t sb = s0; sb < s1; sb += kP2pStage) {
                const int cnt = (int)((s1 - sb) < kP2pStage ? (s1 - sb) : kP2pStage);
                for (int j = lane; j < cnt; j += 32) {
                    T4 p4 = spos[sb + j];
                    T4 y;
                    y.x = self ? p4.x : map_coord<T>(r, p4.x, c[0]);
                    y.y = self ? p4.y : map_coord<T>(r, p4.y, c[1]);
                    y.z = self ? p4.z : map_coord<T>(r, p4.z, c[2]);
                    y.w = sq[(int64_t)v * plan.nsrc + sb + j];
                    stage[warp][j] = y;
                }
                __syncwarp();
                T pphi = T(0), pg0 = T(0), pg1 = T(0), pg2 = T(0);
#pragma unroll 4
                for (int s = 0; s < cnt; ++s) {
                    const T4 y = stage[warp][s];
                    const T dx = sub_rn<T>(tx, y.x), dy = sub_rn<T>(ty, y.y), dz = sub_rn<T>(tz, y.z);
                    const T r2 = pair_r2<T>(dx, dy, dz);
                    const bool skip = r2 == T(0);
                    const T rinv = skip ? T(0) : rsqrt(r2);
                    const T qr = y.w * rinv;
                    pphi += qr;
                    if (GRAD) {
                        const T qr3 = qr * rinv * rinv;
                        pg0 -= qr3 * dx;
                        pg1 -= qr3 * dy;
                        pg2 -= qr3 * dz;
                    }
                }
                aphi += (double)pphi;
                if (GRAD) {
                    ag0 += (double)pg0;
                    ag1 += (double)pg1;
                    ag2 += (double)pg2;
                }
                __syncwarp();
            }
        }
        if (!valid) continue;
        if (accumulate == 2) {  // near field alone, leaf order (added to the far field by output_kernel)
            out_phi[(int64_t)v * nt + t] = aphi;
            if (GRAD) {
                double* o = out_g + ((int64_t)v * nt + t) * 3;
                o[0] = ag0;
                o[1] = ag1;
                o[2] = ag2;
            }
            continue;
        }
        const double ph = far_phi[(int64_t)v * nt + t] + aphi;
        if (accumulate) {  // level calls: add into the leaf-order store, scaled by output_kernel
            far_phi[(int64_t)v * nt + t] = ph;
            if (GRAD) {
                double* fg = far_g + ((int64_t)v * nt + t) * 3;
                fg[0] = fg[0] + ag0;
                fg[1] = fg[1] + ag1;
                fg[2] = fg[2] + ag2;
            }
            continue;
        }
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

// Output pass (fmm-kernels/src/movement.rs:411 gather_output with the scaling of
// fmm-exec/src/fmm.rs:4750-4778): phi = phi_hat / (4 pi r_t) and
// g = g_hat / ((4 pi r_t) r_t), leaf order -> caller order, phi_hat = far + near when the
// near field was summed apart (near_phi non-null), else the store as it is (level calls).
// Block per leaf; the same expressions as the P2P kernels' fused output, so all of them
// give the same floats.
static __global__ void output_kernel(DevPlan plan, int m, const double* __restrict__ far_phi,
                              const double* __restrict__ far_g, const double* __restrict__ near_phi,
                              const double* __restrict__ near_g, double* __restrict__ out_phi,
                              double* __restrict__ out_g) {
    const int64_t leaf = blockIdx.x;
    const int box = plan.leaf_box[leaf];
    const double rt = (plan.box_side ? plan.box_side[box] : plan.side) * pow2d(-(plan.level[box] + 1));
    const double phi_scale = 4.0 * 3.141592653589793 * rt;
    const double g_scale = phi_scale * rt;
    const int64_t nt = plan.ntgt;
    for (int v = 0; v < m; ++v)
        for (int64_t t = plan.tgt_start[leaf] + threadIdx.x; t < plan.tgt_start[leaf + 1]; t += blockDim.x) {
            const int64_t i = plan.tgt_perm[t];
            const double ph = near_phi ? far_phi[(int64_t)v * nt + t] + near_phi[(int64_t)v * nt + t]
                                       : far_phi[(int64_t)v * nt + t];
            out_phi[(int64_t)v * nt + i] = ph / phi_scale;
            if (out_g) {
                const double* fg = far_g + ((int64_t)v * nt + t) * 3;
                double* o = out_g + ((int64_t)v * nt + i) * 3;
                if (near_phi) {
                    const double* ng = near_g + ((int64_t)v * nt + t) * 3;
                    o[0] = (fg[0] + ng[0]) / g_scale;
                    o[1] = (fg[1] + ng[1]) / g_scale;
                    o[2] = (fg[2] + ng[2]) / g_scale;
                } else {
                    o[0] = fg[0] / g_scale;
                    o[1] = fg[1] / g_scale;
                    o[2] = fg[2] / g_scale;
                }
            }
        }
}

// Build time (mixed form): every near pair whose f32 r2, formed exactly as p2p_kernel
// forms it, is below theta2.  Appends (target, source point, source leaf); *count may
// exceed cap, in which case the caller enlarges the buffer and runs it again.
template <typename T>
__global__ void __launch_bounds__(128) close_pairs_kernel(DevPlan plan, P2pItems items, T theta2,
                                                          const typename Vec4<T>::type* __restrict__ spos,
                                                          const typename Vec4<T>::type* __restrict__ tpos,
                                                          unsigned long long* count, int64_t cap,
                                                          int64_t* __restrict__ out_t, int64_t* __restrict__ out_s,
                                                          int32_t* __restrict__ out_leaf) {
    using T4 = typename Vec4<T>::type;
    __shared__ T4 stage[kP2pWarps][kP2pStage];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * kP2pWarps + warp;
    if (item >= items.count) return;
    const int leaf = items.leaf[item];
    const int box = plan.leaf_box[leaf];
    const int64_t t1 = plan.tgt_start[leaf + 1];
    const int64_t t = items.t0[item] + lane;
    const bool valid = t < t1;
    T tx = T(0), ty = T(0), tz = T(0);
    if (valid) {
        T4 p4 = tpos[t];
        tx = p4.x;
        ty = p4.y;
        tz = p4.z;
    }
    for (int64_t e = plan.near_row[leaf]; e < plan.near_row[leaf + 1]; ++e) {
        const int sl = plan.near_col[e];
        T c[3] = {T(0), T(0), T(0)}, r = T(1);
        const bool self = sl == leaf;
        if (!self) rel_frame<T>(plan, plan.leaf_box[sl], box, c, r);
        const int64_t s0 = plan.src_start[sl], s1 = plan.src_start[sl + 1];
        for (int64_t sb = s0; sb < s1; sb += kP2pStage) {
            const int cnt = (int)((s1 - sb) < kP2pStage ? (s1 - sb) : kP2pStage);
            for (int j = lane; j < cnt; j += 32) {
                T4 p4 = spos[sb + j];
                T4 y;
                y.x = self ? p4.x : map_coord<T>(r, p4.x, c[0]);
                y.y = self ? p4.y : map_coord<T>(r, p4.y, c[1]);
                y.z = self ? p4.z : map_coord<T>(r, p4.z, c[2]);
                y.w = T(0);
                stage[warp][j] = y;
            }
            __syncwarp();
            if (valid)
                for (int s = 0; s < cnt; ++s) {
                    const T4 y = stage[warp][s];
                    const T dx = sub_rn<T>(tx, y.x), dy = sub_rn<T>(ty, y.y), dz = sub_rn<T>(tz, y.z);
                    if (pair_r2<T>(dx, dy, dz) < theta2) {
                        unsigned long long k = atomicAdd(count, 1ULL);
                        if ((int64_t)k < cap) {
                            out_t[k] = t;
                            out_s[k] = sb + s;
                            out_leaf[k] = sl;
                        }
                    }
                }
            __syncwarp();
        }
    }
}

}  // namespace fmmb
