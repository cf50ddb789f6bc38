// Dense M2L on the tensor cores, fused with the local reduce (mixed form).
//
// The product path of m2l_tc.cuh writes every V pair's product A_d M_s (one row of
// (p+1)^2 f32 per pair and charge vector) to memory, and local_reduce_kernel reads them
// back to add them into the locals in each row's order.  Here the products never reach
// memory: every target box belongs to exactly one CTA, which takes the V pairs of its
// target boxes offset by offset and adds each product straight from tensor memory into
// the target's local, L[t] += A_d M_s.  A target's V row is sorted by offset index
// (fmm-plan/src/lists.rs V lists; the accumulation order of fmm-plan/src/operator.rs:34-45),
// so its products arrive in row order, and with L holding the L2L part first the sums
// are the floats of local_reduce_kernel (L2L, then V in row order), bit for bit.
//
// Work layout.  Per level the target boxes with a V row are cut into chunks of
// consecutive boxes; a chunk's pairs are ordered by (offset, target) and cut into tiles of
// NT / m pairs of one offset, m charge vectors per pair: column c of a tile is pair
// c / m, vector c % m.  A CTA takes a contiguous range of chunks (the tile range
// cta_tiles[c] .. cta_tiles[c + 1]), so no two CTAs touch one local, and its chunks are
// small enough that their locals stay in L2 while the CTA walks the offsets.
// MMA: D[slot][column] = A_d[slot][k] X[column][k], the table A_d in tensor memory
// (M = 128 lanes = output slots, two buffers so the next offset's table is written while
// the current one is read), the gathered multipoles X in shared memory (N = NT columns,
// K-major, 128-byte swizzled, two stages); 3xTF32 as in m2l_tc.cuh.
// Roles (mbarriers only, every wait bounded):
//   warps 12-19 (producers): gather tile k's columns, split hi / lo into stage k & 1
//     once MMA(k-2) released it;
//   warps 8-11 (table loaders, one per lane quarter below (p+1)^2): one thread copies
//     each offset's table image (only its rows below the quarters in use, laid out so
//     a warp's shared-memory reads are conflict-free) into a staging ring with one bulk
//     asynchronous copy, STG - 1 offsets ahead; every loader warp moves its lane quarter
//     from the staging slot into tensor-memory buffer (change & 1) once the MMAs of
//     change - 2 are done;
//   warp 20, one thread (MMA): table full, X full, accumulator free -> 3 x KSTEPS MMAs,
//     commits X empty and accumulator full, and table free after an offset's last tile;
//   warps 0-7 (epilogue, lane quarter w & 3, target parity w >> 2): read the
//     accumulator, release it, and add the columns whose target box has this warp's
//     parity into the locals with red.global.add.f32 (round to nearest, as the reduce's
//     add).  A local (box, vector, slot) is only ever added to by one thread, in tile
//     order, so its additions are applied in that order without any barrier.
#pragma once

#include "m2l_tc.cuh"

namespace fmmb {

constexpr int kFuWarps = 21;
constexpr int kFuEpi = 8;     // warps 0-7
constexpr int kFuTab0 = 8;    // warps 8-11
constexpr int kFuProd0 = 12;  // warps 12-19
constexpr int kFuProd = 8;
constexpr int kFuMma = 20;

template <int P>
struct FuShape {
    static constexpr int NC = nc_of(P);
    static constexpr int KA = (NC + 31) / 32;
    static constexpr int KP = 32 * KA;       // padded K (input slots)
    static constexpr int KSTEPS = KP / 8;
    // columns per tile: what tensor memory leaves after two tables (hi, lo each) and two
    // accumulators, at most 128
    static constexpr int NT_FIT = ((512 - 4 * KP) / 2) / 16 * 16;
    static constexpr int NT = NT_FIT < 128 ? NT_FIT : 128;
    static constexpr int RPW = NT / kFuProd;  // gathered rows per producer warp
    static constexpr int X_BYTES = NT * KP * 4;  // one part (hi or lo) of one stage
    static constexpr int COL_D0 = 4 * KP;        // TMEM columns: tables [2][hi, lo], then D [2][NT]
    static constexpr int IMG_WORDS = 2 * 128 * KP;
    static constexpr int QUARTERS = (NC + 31) / 32;  // lane quarters holding output slots
    static constexpr int ROWS = 32 * QUARTERS;       // table rows moved per offset
    static constexpr int KC = KP / 16;               // 16-column groups of a table part
    static constexpr int TBYTES = 2 * KP * ROWS * 4;  // one offset's image: [part][KC][4][ROWS] uint4
    static constexpr int TWORDS = TBYTES / 4;
    static constexpr int STG = 4 * X_BYTES + 2 * TBYTES + 1024 <= 227 * 1024 ? 2 : 1;  // staging slots
    static constexpr int SMEM = 4 * X_BYTES + STG * TBYTES + 1024;
    static_assert(NC <= 128, "UMMA M = 128 output slots");
    static_assert(NT >= 16 && NT % 16 == 0, "UMMA N");
    static_assert(4 * KP + 2 * NT <= 512, "TMEM budget");
    static_assert(NT % kFuProd == 0 && RPW <= 32, "producer rows");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};


// one bulk copy global -> this CTA's shared memory, completion counted on mbar (both
// addresses 16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

// tile columns (pairs x charge vectors) of the fused kernel at degree p; 0 where it does
// not apply (p > 8: tensor memory holds two tables only up to KP = 96)
inline int fused_tile_columns(int p) {
    switch (p) {
        case 3: return FuShape<3>::NT;
        case 4: return FuShape<4>::NT;
        case 5: return FuShape<5>::NT;
        case 6: return FuShape<6>::NT;
        case 7: return FuShape<7>::NT;
        case 8: return FuShape<8>::NT;
        default: return 0;
    }
}

template <int P>
__global__ void __launch_bounds__(32 * kFuWarps, 1) m2l_fused_kernel(
    const int32_t* __restrict__ tile_d, const int64_t* __restrict__ tile_begin, const int32_t* __restrict__ tile_np,
    const int64_t* __restrict__ cta_tiles, const int32_t* __restrict__ pair_src, const int32_t* __restrict__ pair_tgt,
    int m, const uint32_t* __restrict__ timg, const float* __restrict__ M, float* __restrict__ L,
    int* __restrict__ error) {
    using S = FuShape<P>;
    constexpr int NC = S::NC, NT = S::NT, RPW = S::RPW, STG = S::STG;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* xbuf = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);  // [2 stages][hi, lo]
    unsigned char* sbuf = xbuf + 4 * S::X_BYTES;  // table staging [STG][TBYTES]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __shared__ uint64_t bar_full[2], bar_empty[2], bar_accf[2], bar_acce[2], bar_tfull[2], bar_tfree[2];
    __shared__ uint64_t bar_sfull[2], bar_sempty[2];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const int64_t i0 = cta_tiles[blockIdx.x], i1 = cta_tiles[blockIdx.x + 1];
    if (i0 >= i1) return;
    const int64_t ntile = i1 - i0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bar_full[b]), kFuProd);
            mbar_init(smem_u32(&bar_empty[b]), 1);
            mbar_init(smem_u32(&bar_accf[b]), 1);
            mbar_init(smem_u32(&bar_acce[b]), kFuEpi);
            mbar_init(smem_u32(&bar_tfull[b]), S::QUARTERS);
            mbar_init(smem_u32(&bar_tfree[b]), 1);
            mbar_init(smem_u32(&bar_sfull[b]), 1);
            mbar_init(smem_u32(&bar_sempty[b]), S::QUARTERS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    volatile int* abort = &abort_flag;
    auto give_up = [&]() {
        *abort = 1;
        atomicExch(error, 1);
    };
    auto warp_wait = [&](uint64_t* bar, uint32_t parity) {
        int ok = 0;
        if (lane == 0) ok = mbar_wait_bounded(smem_u32(bar), parity, kTcWait, abort);
        return __shfl_sync(0xffffffffu, ok, 0) != 0;
    };
    auto warp_aborted = [&]() {
        int a = 0;
        if (lane == 0) a = *abort;
        return __shfl_sync(0xffffffffu, a, 0) != 0;
    };

    if (warp >= kFuProd0 && warp < kFuProd0 + kFuProd) {
        // ---------------- producers ----------------
        const int pw = warp - kFuProd0;
        // lane j < RPW holds the multipole row (box * m + vector) of tile row pw + 8 j, or -1
        auto row_src = [&](int64_t it) {
            const int64_t pb = tile_begin[it];
            const int ncol = tile_np[it] * m;
            int64_t s = -1;
            const int r = pw + kFuProd * lane;
            if (lane < RPW && r < ncol) s = (int64_t)pair_src[pb + r / m] * m + r % m;
            return s;
        };
        int64_t nsrc = row_src(i0);
        for (int64_t k = 0; k < ntile && !warp_aborted(); ++k) {
            const int st = (int)(k & 1);
            const int64_t my_src = nsrc;
            unsigned char* xh = xbuf + (size_t)st * 2 * S::X_BYTES;
            unsigned char* xl = xh + S::X_BYTES;
            float x[RPW][S::KA];
#pragma unroll
            for (int j = 0; j < RPW; ++j) {
                const long long sr = __shfl_sync(0xffffffffu, (long long)my_src, j);
                const float* src = M + (sr < 0 ? 0 : sr) * ms_of(P);
#pragma unroll
                for (int a = 0; a < S::KA; ++a) {
                    const int kk = a * 32 + lane;
                    x[j][a] = (sr >= 0 && kk < NC) ? __ldg(src + kk) : 0.0f;
                }
            }
            if (k + 1 < ntile) nsrc = row_src(i0 + k + 1);  // in flight with the loads above
            if (k >= 2 && !warp_wait(&bar_empty[st], (uint32_t)(((k - 2) >> 1) & 1))) {
                if (lane == 0) give_up();
                break;
            }
#pragma unroll
            for (int j = 0; j < RPW; ++j) {
                const int r = pw + kFuProd * j;
#pragma unroll
                for (int a = 0; a < S::KA; ++a) {
                    const int kk = a * 32 + lane;
                    const uint32_t hi = cvt_tf32(x[j][a]);
                    const uint32_t lo = cvt_tf32(x[j][a] - __uint_as_float(hi));
                    const uint32_t off = sw128_offset(r, kk, NT);
                    *reinterpret_cast<uint32_t*>(xh + off) = hi;
                    *reinterpret_cast<uint32_t*>(xl + off) = lo;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_full[st]));
        }
    } else if (warp >= kFuTab0 && warp < kFuTab0 + 4) {
        // ---------------- table loaders ----------------
        const int q = warp & 3;  // lane quarter: output slots 32 q .. 32 q + 31
        if (32 * q < NC) {
            // the copy issuer (quarter 0, lane 0) runs its own cursor over the tiles, STG - 1
            // offset changes ahead of the copies into tensor memory
            int64_t ik = 0, ic = -1;
            int id = -1;
            auto issue_next = [&]() -> bool {  // false only on a timed-out wait
                while (ik < ntile) {
                    const int d = tile_d[i0 + ik++];
                    if (d == id) continue;
                    id = d;
                    ++ic;
                    const int slot = (int)(ic % STG);
                    if (ic >= STG && !mbar_wait_bounded(smem_u32(&bar_sempty[slot]),
                                                        (uint32_t)(((ic - STG) / STG) & 1), kTcWait, abort))
                        return false;
                    mbar_expect_tx(smem_u32(&bar_sfull[slot]), (uint32_t)S::TBYTES);
                    bulk_g2s(smem_u32(sbuf + (size_t)slot * S::TBYTES), timg + (size_t)d * S::TWORDS,
                             (uint32_t)S::TBYTES, smem_u32(&bar_sfull[slot]));
                    return true;
                }
                return true;
            };
            const bool issuer = q == 0;
            int ok = 1;
            if (issuer && lane == 0)
                for (int i = 0; i < STG - 1 && ok; ++i) ok = issue_next();
            int cur_d = -1;
            int64_t c = -1;  // offset changes so far
            for (int64_t k = 0; k < ntile; ++k) {
                const int d = tile_d[i0 + k];
                if (d == cur_d) continue;
                cur_d = d;
                ++c;
                if (issuer && lane == 0 && ok) ok = issue_next();
                if (issuer && !__shfl_sync(0xffffffffu, ok, 0)) {
                    if (lane == 0) give_up();
                    break;
                }
                if (warp_aborted()) break;
                const int slot = (int)(c % STG), b = (int)(c & 1);
                if (!warp_wait(&bar_sfull[slot], (uint32_t)((c / STG) & 1)) ||
                    (c >= 2 && !warp_wait(&bar_tfree[b], (uint32_t)(((c - 2) >> 1) & 1)))) {
                    if (lane == 0) give_up();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint4* stg = reinterpret_cast<const uint4*>(sbuf + (size_t)slot * S::TBYTES);
                const int row = 32 * q + lane;
                const uint32_t col0 = (uint32_t)(b * 2 * S::KP);
#pragma unroll 1
                for (int part = 0; part < 2; ++part)
#pragma unroll 2
                    for (int kc = 0; kc < S::KC; ++kc) {
                        uint32_t r16[16];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const uint4 u = stg[((part * S::KC + kc) * 4 + j) * S::ROWS + row];
                            r16[4 * j] = u.x;
                            r16[4 * j + 1] = u.y;
                            r16[4 * j + 2] = u.z;
                            r16[4 * j + 3] = u.w;
                        }
                        tmem_st16(tmem + ((uint32_t)(32 * q) << 16) + (col0 + (uint32_t)(part * S::KP + 16 * kc)), r16);
                    }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(smem_u32(&bar_sempty[slot]));
                    mbar_arrive(smem_u32(&bar_tfull[b]));
                }
            }
        }
    } else if (warp == kFuMma) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = tf32_idesc_ts<NT>();
            int cur_d = -1;
            int64_t c = -1;
            int64_t issued = 0;
            for (int64_t k = 0; k < ntile && !*abort; ++k) {
                const int64_t it = i0 + k;
                const int st = (int)(k & 1);
                const int d = tile_d[it];
                bool ok = true;
                if (d != cur_d) {
                    ++c;
                    cur_d = d;
                    ok = mbar_wait_bounded(smem_u32(&bar_tfull[c & 1]), (uint32_t)((c >> 1) & 1), kTcWait, abort);
                }
                ok = ok && mbar_wait_bounded(smem_u32(&bar_full[st]), (uint32_t)((k >> 1) & 1), kTcWait, abort);
                ok = ok && (k < 2 || mbar_wait_bounded(smem_u32(&bar_acce[st]), (uint32_t)(((k - 2) >> 1) & 1),
                                                       kTcWait, abort));
                if (!ok) {
                    give_up();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t xh = smem_u32(xbuf + (size_t)st * 2 * S::X_BYTES), xl = xh + S::X_BYTES;
                const uint32_t dcol = tmem + (uint32_t)(S::COL_D0 + st * NT);
                const uint32_t ahi = (uint32_t)((c & 1) * 2 * S::KP), alo = ahi + (uint32_t)S::KP;
                const uint32_t As[3] = {ahi, alo, ahi};
                const uint32_t Bs[3] = {xl, xh, xh};  // A_hi X_lo, A_lo X_hi, then A_hi X_hi
                uint32_t acc = 0;
#pragma unroll
                for (int t = 0; t < 3; ++t)
#pragma unroll
                    for (int s2 = 0; s2 < S::KSTEPS; ++s2) {
                        const uint32_t kb = (uint32_t)((s2 >> 2) * NT * 128 + (s2 & 3) * 32);
                        umma_tf32_ts(dcol, tmem + As[t] + (uint32_t)(8 * s2), sw128_desc(Bs[t] + kb), idesc, acc);
                        acc = 1;
                    }
                umma_commit(smem_u32(&bar_empty[st]));
                umma_commit(smem_u32(&bar_accf[st]));
                if (k + 1 == ntile || tile_d[it + 1] != d) umma_commit(smem_u32(&bar_tfree[c & 1]));
                issued = k + 1;
            }
            if (*abort && issued > 0) {
                const int64_t k = issued - 1;
                mbar_wait_bounded(smem_u32(&bar_empty[k & 1]), (uint32_t)((k >> 1) & 1), kTcWait);
            }
        }
        __syncwarp();
    } else if (warp < kFuEpi) {
        // ---------------- epilogue: add the products into the locals ----------------
        const int q = warp & 3, g = warp >> 2;  // lane quarter (slots), target parity
        const int n = 32 * q + lane;            // this lane's output slot
        const bool active = 32 * q < NC;
        for (int64_t k = 0; k < ntile && !warp_aborted(); ++k) {
            const int64_t it = i0 + k;
            const int st = (int)(k & 1);
            const int64_t pb = tile_begin[it];
            const int ncol = tile_np[it] * m;
            // lane j holds the local row (box * m + vector) * ms_of(P) of columns j, j + 32, j + 64,
            // j + 96, or -1 where the column is empty or its box has the other parity
            long long rb[(NT + 31) / 32];
#pragma unroll
            for (int h = 0; h < (NT + 31) / 32; ++h) {
                const int cc = 32 * h + lane;
                rb[h] = -1;
                if (cc < ncol) {
                    const int t = pair_tgt[pb + cc / m];
                    if ((t & 1) == g) rb[h] = ((long long)t * m + cc % m) * ms_of(P);
                }
            }
            if (!warp_wait(&bar_accf[st], (uint32_t)((k >> 1) & 1))) {
                if (lane == 0) give_up();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (active) {
#pragma unroll
                for (int c0 = 0; c0 < NT; c0 += 16) {
                    if (c0 >= ncol) break;
                    float dv[16];
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(S::COL_D0 + st * NT + c0), dv);
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const long long row = __shfl_sync(0xffffffffu, rb[(c0 + i) >> 5], (c0 + i) & 31);
                        if (row >= 0 && n < NC) atomicAdd(L + row + n, dv[i]);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_acce[st]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// Host: the fused kernel's table images from the tensor-memory images of
// build_tc_table_images (tc: [d][part][128 slots][KP]): per offset only the rows of the
// lane quarters in use, as [part][16-column group][4 words][row][4], so that loader lane
// `row` reads its 16 consecutive words of a group as 4 uint4 at consecutive addresses
// across the warp.
template <int P>
void build_fused_table_images(const std::vector<uint32_t>& tc, std::vector<uint32_t>& img) {
    using S = FuShape<P>;
    constexpr int KP = S::KP, KC = S::KC, ROWS = S::ROWS;
    img.assign((size_t)316 * S::TWORDS, 0u);
    for (int d = 0; d < 316; ++d)
        for (int part = 0; part < 2; ++part)
            for (int kc = 0; kc < KC; ++kc)
                for (int j = 0; j < 4; ++j)
                    for (int row = 0; row < ROWS; ++row)
                        for (int w = 0; w < 4; ++w)
                            img[(size_t)d * S::TWORDS + ((((size_t)part * KC + kc) * 4 + j) * ROWS + row) * 4 + w] =
                                tc[(size_t)d * 2 * 128 * KP + ((size_t)part * 128 + row) * KP + 16 * kc + 4 * j + w];
}

}  // namespace fmmb
