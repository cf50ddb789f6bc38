// Dense M2L on the tensor cores (mixed form): tcgen05.mma kind::tf32 with a 3-term
// split, accumulators in tensor memory.
//
// The V pairs of every level are grouped by offset d (the batches of m2l_gemm_kernel)
// and cut into tiles; for a tile the MMA forms D[slot][column] = A_d[slot][k] X[column][k],
// the table A_d (M = 128 output slots) in tensor memory and X the tile's gathered source
// multipoles (N = the tile's columns, K = the (p+1)^2 input slots padded to KP = 32 * KA)
// in shared memory.  f32 data is split as x = hi + lo with hi = tf32(x),
// lo = tf32(x - hi), and D = A_hi X_lo + A_lo X_hi + A_hi X_hi (the lo*lo term, 2^-22
// relative, is dropped), each product an exact tf32 product summed in f32 in tensor
// memory.  The X operand is K-major in 128-byte-swizzled shared memory: 8-row x 128 B
// atoms, 16 B chunk c of row r stored at chunk c ^ (r % 8); a K-step of 8 tf32 (32 B)
// advances the descriptor start address by 32 B inside an atom, and atoms of 32
// K-elements follow each other.  The table images (hi and lo) are precomputed on the host.
// The persistent, warp-specialised kernel is described above m2l_tc_kernel.
//
// Descriptor fields follow cute/arch/mma_sm100_desc.hpp (CUTLASS 4.5): SmemDescriptor
// (start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48), layout [61,64),
// SWIZZLE_128B = 2) and InstrDescriptor (c_format [4,6), a/b_format [7,10)/[10,13),
// a/b_major [15]/[16], N>>3 [17,23), M>>4 [24,29)).
//
// Waits are bounded: a CTA that gives up sets *error and skips its epilogue.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "harmonics.cuh"

namespace fmmb {

// byte offset of element (row r, column k) in a K-major SW128 operand of `rows` rows
__host__ __device__ __forceinline__ uint32_t sw128_offset(int r, int k, int rows) {
    int atom = k >> 5, kk = k & 31;
    int chunk = (kk >> 2) ^ (r & 7);
    return (uint32_t)(atom * rows * 128 + r * 128 + chunk * 16 + (kk & 3) * 4);
}

__host__ __device__ __forceinline__ uint32_t tf32_round_bits(uint32_t bits) {
    // round to nearest, ties away from zero, to 10 explicit mantissa bits (cvt.rna.tf32.f32)
    return (bits + 0x1000u) & ~0x1FFFu;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                   // LBO (unused by swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;         // SBO: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                   // version (sm_100)
    d |= (uint64_t)2 << 61;                   // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ uint32_t cvt_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// returns true when the barrier's phase `parity` completed within `limit` clock cycles;
// false on timeout or when *abort is set (another role gave up)
// Each try_wait may suspend the thread until the phase completes or kWaitHintNs elapse
// (a hint to the hardware), so a waiting warp takes few issue slots from the working ones;
// the bound and the abort flag are checked between tries.
constexpr uint32_t kWaitHintNs = 20000;
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, long long limit,
                                                  const volatile int* abort = nullptr) {
    const long long start = clock64();
    while (clock64() - start < limit) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity), "r"(kWaitHintNs)
            : "memory");
        if (done) return true;
        if (abort && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile(
        "{\n\t"
        ".reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t"
        "}\n" ::"r"(mbar)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// Persistent, warp-specialised form.  CTA c takes the contiguous range of tiles
// [c T / G, (c + 1) T / G) of the offset-sorted tile list.  The table of the current
// offset lives in tensor memory as the MMA's A operand (M = 128 lanes = output slots,
// K = input slots in columns; hi and lo parts), so the MMA is D[slot][pair] = A_d . X^T
// with the gathered multipoles X as the shared-memory B operand (N = NT pairs,
// K-major, 128-byte swizzled).  Roles, coupled only by mbarriers (no block barrier in
// the loop):
//   warp 17 (gather): for tile k, once the raw stage k % RS is free, the lanes fetch the
//     tile's multipole rows with the copy engine into the raw stage, completion counted
//     on raw_full: with fewer than four vectors each lane fetches four rows with one
//     tile::gather4 (box one row of KP f32, the slots beyond (p+1)^2 filled with zeros);
//     with m >= 4 the m vectors of a pair are m consecutive rows and lane j fetches pair
//     j's with one 2D tile load (box m rows).  The copy engine keeps the whole tile's
//     rows in flight at once, where per-lane loads were limited by the SM's outstanding
//     misses;
//   warps 8-15 (converters): wait raw_full, split the raw rows into X stage k&1
//     (x = hi + lo in tf32, 128-byte swizzled) once MMA(k-2) has released it
//     (empty[k&1]), signal full[k&1] and raw_empty; warps 8-11 also replace the table in
//     tensor memory when the offset changes, after MMA(k-1) has read the old one;
//   warp 16, one thread (MMA): waits full[k&1], the table and the accumulator k&1
//     (acc_empty, released by the epilogue of tile k-2), issues the 3 x KSTEPS MMAs
//     and commits to empty[k&1] and acc_full[k&1];
//   warps 0-7 (epilogue): wait acc_full[k&1], read the accumulator with tcgen05.ld
//     and stream the products past L2 into Y at the pairs' positions in the tile list
//     (a tile's rows consecutive, each ys_of(P) slots: (p+1)^2 rounded up to 4),
//     then release acc_empty[k&1].
// Every wait is bounded; a role that gives up sets the shared abort flag (which ends
// the other roles' waits) and *error, and the CTA frees its tensor memory and returns.
// A tile holds cnt <= NT / m pairs of one offset with all m charge vectors: column
// c is pair c / m, vector c % m, its product row in Y is p0 * m + c (the pair's rows are
// its m vectors in order).
constexpr int kTcWarps = 18;
constexpr int kTcProd = 8;        // converter warps (8..15)
constexpr int kTcMmaWarp = 16;    // the MMA issuer's warp
constexpr int kTcGatherWarp = 17; // the gather issuer's warp
constexpr long long kTcWait = 4000000000LL;  // clock cycles (about 2 s)

// CPLX: the Helmholtz form, a complex table A = A_r + i A_i applied to the real and the
// imaginary plane of a multipole as two columns (its two expansion rows), with the table's
// rows [A_r; A_i] as two halves of 128 output slots (the n = (p+1)^2 rows of each padded):
// the products of a column are A_r x in slots 0..n and A_i x in slots 128..128+n of a
// 256-slot row, which the complex local reduce combines into the local's two planes.
// NTA: the columns of a tile when nonzero (the tuner's alternative), else the default below
template <int P, bool CPLX = false, int NTA = 0>
struct TcTs {
    static constexpr int NC = nc_of(P);
    static constexpr int KA = (NC + 31) / 32;
    static constexpr int KP = 32 * KA;             // padded K (input slots)
    static constexpr int KSTEPS = KP / 8;
    // output slot halves: (p+1)^2 > 128 (p = 11, 12) takes two passes over a tile's
    // columns, each with the table rows of one half (128 slots) in tensor memory
    static constexpr int H = (CPLX || NC > 128) ? 2 : 1;
    static constexpr int YS = CPLX ? 256 : ys_of(P);  // product row stride (floats)
    // columns per tile (UMMA N): 96 at p = 7, 8 (KP = 96), where shared memory then holds
    // two raw stages (measured faster than 64 columns with four); 64 at p = 9, 10
    // (KP = 128), the most beside two X stages and two raw stages; 48 at p = 11, 12
    // (KP = 160, 192: tensor memory then holds the table's 2 KP columns and two 48-column
    // accumulators, shared memory two X stages and two or three raw stages)
    static constexpr int NT = NTA ? NTA : KP > 128 ? 48 : KP > 96 ? 64 : KP > 64 ? 96 : 128;
    static constexpr int X_BYTES = NT * KP * 4;    // one part of one stage (also one raw stage)
    // raw stages: as many as shared memory holds beside the two X stages, at most 4 (the
    // copy engine's loads take several tiles' time to land)
    static constexpr int RS_FIT = (227 * 1024 - 256 - 1024 - 4 * X_BYTES) / X_BYTES;
    static constexpr int RS = RS_FIT < 4 ? RS_FIT : 4;
    static constexpr int SMEM = (4 + RS) * X_BYTES + 1024;  // X [2 stages][hi, lo], raw [RS stages]
    static constexpr int COL_AHI = 0, COL_ALO = KP, COL_D0 = 2 * KP;  // TMEM columns
    static constexpr int TMEM_COLS = 512;
    static constexpr int IMG_WORDS = 2 * 128 * KP;  // table image words per (offset, half) (hi, lo)
    static_assert(NC <= (CPLX ? 128 : 256), "two halves of UMMA M = 128 output slots");
    static_assert(2 * KP + 2 * NT <= TMEM_COLS, "TMEM budget");
    static_assert(NT % 16 == 0 && NT / 4 <= 32, "UMMA N; gather rows: four per lane");
    static_assert(RS >= 2, "raw stages");
    static_assert(SMEM + 256 <= 227 * 1024, "shared memory");
};

template <int NTILE>
__host__ __device__ constexpr uint32_t tf32_idesc_ts() {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NTILE >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile(
        "{\n\t"
        ".reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t"
        "}\n" ::"r"(mbar),
        "r"(bytes)
        : "memory");
}

// four rows (r0..r3) of a 2D tensor map, one box each (KP f32 at x = 0), into dst
// (four consecutive box rows), completion counted on mbar; no multicast
// one box (x = 0, first row y) of a 2D tensor map into dst, completion counted on mbar;
// no multicast
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int y, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap* map, int r0, int r1, int r2, int r3,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(mbar)
        : "memory");
}

template <int P, bool CPLX = false, int NTA = 0>
__global__ void __launch_bounds__(32 * kTcWarps, 1) m2l_tc_kernel(const int32_t* __restrict__ tile_d,
                                                                  const int64_t* __restrict__ tile_begin,
                                                                  const int32_t* __restrict__ tile_count,
                                                                  int64_t ntiles,
                                                                  const int32_t* __restrict__ pair_src, int m,
                                                                  const uint32_t* __restrict__ timg,
                                                                  const __grid_constant__ CUtensorMap mmap,
                                                                  const __grid_constant__ CUtensorMap vmap,
                                                                  float* __restrict__ Y, int* __restrict__ error) {
    using S = TcTs<P, CPLX, NTA>;
    constexpr int NT = S::NT, KP = S::KP, YS = S::YS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* xbuf = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);  // [2 stages][hi, lo]
    unsigned char* rbuf = xbuf + 4 * S::X_BYTES;                                      // raw [RS stages][NT][KP]
    constexpr int RS = S::RS;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __shared__ uint64_t bar_full[2], bar_empty[2], bar_accf[2], bar_acce[2], bar_table, bar_rfull[RS], bar_rempty[RS];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const int64_t i0 = (int64_t)blockIdx.x * ntiles / gridDim.x;
    const int64_t i1 = (int64_t)(blockIdx.x + 1) * ntiles / gridDim.x;
    if (i0 >= i1) return;
    const int64_t ntile = i1 - i0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(S::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bar_full[b]), kTcProd);
            mbar_init(smem_u32(&bar_empty[b]), 1);
            mbar_init(smem_u32(&bar_accf[b]), 1);
            mbar_init(smem_u32(&bar_acce[b]), 8);
        }
        for (int b = 0; b < RS; ++b) {
            mbar_init(smem_u32(&bar_rfull[b]), 1);
            mbar_init(smem_u32(&bar_rempty[b]), kTcProd);
        }
        mbar_init(smem_u32(&bar_table), 4);
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
    // warp-wide roles: lane 0 waits (or reads the abort flag) and the warp takes its answer,
    // so the lanes of a warp never part ways
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

    if (warp == kTcGatherWarp) {
        // ---------------- gather ----------------
        const bool blocks = m >= 4;        // one box of m rows a pair
        const int ppt = NT / m;            // pairs a tile holds
        const uint32_t tx = blocks ? (uint32_t)(ppt * m * KP * 4) : (uint32_t)S::X_BYTES;
        int64_t issued = 0;
        for (int64_t k = 0; k < ntile && !warp_aborted(); ++k) {
            const int64_t it = i0 + k;
            const int rs = (int)(k % RS);
            const int64_t p0 = tile_begin[it];
            const int ncol = tile_count[it] * m;
            // rows past the tile's columns fetch row 0 (their products are never stored)
            int r[4];
            if (blocks) {
                r[0] = (lane < ppt && lane * m < ncol) ? pair_src[p0 + lane] * m : 0;
            } else if (m == 1) {  // the common case without the divisions
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = 4 * lane + j;
                    r[j] = (c < ncol) ? pair_src[p0 + c] : 0;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = 4 * lane + j;
                    r[j] = (c < ncol) ? pair_src[p0 + c / m] * m + c % m : 0;
                }
            }
            if (k >= RS && !warp_wait(&bar_rempty[rs], (uint32_t)(((k - RS) / RS) & 1))) {
                if (lane == 0) give_up();
                break;
            }
            if (lane == 0) mbar_expect_tx(smem_u32(&bar_rfull[rs]), tx);
            __syncwarp();
            unsigned char* dst = rbuf + (size_t)rs * S::X_BYTES;
            if (blocks) {
                if (lane < ppt)
                    tma_load_2d(smem_u32(dst + (size_t)lane * m * KP * 4), &vmap, r[0], smem_u32(&bar_rfull[rs]));
            } else if (4 * lane < NT) {
                tma_gather4(smem_u32(dst + (size_t)4 * lane * KP * 4), &mmap, r[0], r[1], r[2], r[3],
                            smem_u32(&bar_rfull[rs]));
            }
            issued = k + 1;
        }
        // on a give-up, the gathers still in flight land before the shared memory is released
        if (lane == 0 && *abort)
            for (int64_t k = issued > RS ? issued - RS : 0; k < issued; ++k)
                mbar_wait_bounded(smem_u32(&bar_rfull[k % RS]), (uint32_t)((k / RS) & 1), kTcWait);
        __syncwarp();
    } else if (warp >= kTcProd && warp < kTcProd + kTcProd) {
        // ---------------- converters ----------------
        const int pw = warp - kTcProd;
        const int ctid = tid - 32 * kTcProd;  // 0 .. 255
        const uint32_t* img_prev = nullptr;
        for (int64_t k = 0; k < ntile && !warp_aborted(); ++k) {
            const int64_t it = i0 + k;
            const int st = (int)(k & 1);
            unsigned char* xh = xbuf + (size_t)st * 2 * S::X_BYTES;
            unsigned char* xl = xh + S::X_BYTES;
            const int rs = (int)(k % RS);
            const float4* raw = reinterpret_cast<const float4*>(rbuf + (size_t)rs * S::X_BYTES);
            // the raw rows of tile k are in; the stage is written only once MMA(k-2) has read it
            if (!warp_wait(&bar_rfull[rs], (uint32_t)((k / RS) & 1)) ||
                (k >= 2 && !warp_wait(&bar_empty[st], (uint32_t)(((k - 2) >> 1) & 1)))) {
                if (lane == 0) give_up();
                break;
            }
            // raw [NT][KP] -> hi / lo, four consecutive slots (one 16-byte chunk) at a time
#pragma unroll 4
            for (int c = ctid; c < NT * KP / 4; c += 32 * kTcProd) {
                const int row = c / (KP / 4), k4 = 4 * (c % (KP / 4));
                const float4 x = raw[c];
                uint4 hi, lo;
                hi.x = cvt_tf32(x.x);
                hi.y = cvt_tf32(x.y);
                hi.z = cvt_tf32(x.z);
                hi.w = cvt_tf32(x.w);
                lo.x = cvt_tf32(x.x - __uint_as_float(hi.x));
                lo.y = cvt_tf32(x.y - __uint_as_float(hi.y));
                lo.z = cvt_tf32(x.z - __uint_as_float(hi.z));
                lo.w = cvt_tf32(x.w - __uint_as_float(hi.w));
                const uint32_t off = sw128_offset(row, k4, NT);
                *reinterpret_cast<uint4*>(xh + off) = hi;
                *reinterpret_cast<uint4*>(xl + off) = lo;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(smem_u32(&bar_full[st]));
                mbar_arrive(smem_u32(&bar_rempty[rs]));
            }
            // the table of tile k (warps 8-11, one per lane quarter), once MMA(k-1) is done
            const uint32_t* img = timg + (size_t)tile_d[it] * S::IMG_WORDS;
            if (pw < 4 && img != img_prev) {
                if (k >= 1 && !warp_wait(&bar_empty[(k - 1) & 1], (uint32_t)(((k - 1) >> 1) & 1))) {
                    if (lane == 0) give_up();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
                for (int part = 0; part < 2; ++part)
#pragma unroll 1
                    for (int k0 = 0; k0 < S::KP; k0 += 48) {
                        uint4 u[12];
                        const uint4* row =
                            reinterpret_cast<const uint4*>(img + ((size_t)part * 128 + 32 * pw + lane) * S::KP + k0);
#pragma unroll
                        for (int q = 0; q < 12; ++q) u[q] = (k0 + 4 * q < S::KP) ? __ldg(row + q) : make_uint4(0, 0, 0, 0);
#pragma unroll
                        for (int h = 0; h < 3; ++h) {
                            if (k0 + 16 * h >= S::KP) break;
                            uint32_t r16[16];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                r16[4 * q] = u[4 * h + q].x;
                                r16[4 * q + 1] = u[4 * h + q].y;
                                r16[4 * q + 2] = u[4 * h + q].z;
                                r16[4 * q + 3] = u[4 * h + q].w;
                            }
                            tmem_st16(tmem + ((uint32_t)(32 * pw) << 16) +
                                          (uint32_t)((part ? S::COL_ALO : S::COL_AHI) + k0 + 16 * h),
                                      r16);
                        }
                    }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&bar_table));
            }
            img_prev = img;
        }
    } else if (warp == kTcMmaWarp) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = tf32_idesc_ts<NT>();
            int cur_d = -1;
            uint32_t nchg = 0;
            int64_t issued = 0;
            for (int64_t k = 0; k < ntile && !*abort; ++k) {
                const int64_t it = i0 + k;
                const int st = (int)(k & 1);
                const int d = tile_d[it];
                bool ok = true;
                if (d != cur_d) {
                    ok = mbar_wait_bounded(smem_u32(&bar_table), nchg & 1, kTcWait, abort);
                    ++nchg;
                    cur_d = d;
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
                const uint32_t As[3] = {(uint32_t)S::COL_AHI, (uint32_t)S::COL_ALO, (uint32_t)S::COL_AHI};
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
                issued = k + 1;
            }
            // on a give-up, let the MMAs already issued finish before the memory is freed
            if (*abort && issued > 0) {
                const int64_t k = issued - 1;
                mbar_wait_bounded(smem_u32(&bar_empty[k & 1]), (uint32_t)((k >> 1) & 1), kTcWait);
            }
        }
        __syncwarp();
    } else if (warp < 8) {
        // ---------------- epilogue ----------------
        const int q = warp & 3, g = warp >> 2;  // lane quarter, column group (16-column chunks g, g + 2, ...)
        for (int64_t k = 0; k < ntile && !warp_aborted(); ++k) {
            const int64_t it = i0 + k;
            const int st = (int)(k & 1);
            const int64_t p0 = tile_begin[it];
            const int ncol = tile_count[it] * m;
            const int h = S::H == 2 ? (tile_d[it] & 1) : 0;  // slot half of this pass
            const int n = 128 * h + 32 * q + lane;            // output slot of this lane
            if (!warp_wait(&bar_accf[st], (uint32_t)((k >> 1) & 1))) {
                if (lane == 0) give_up();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (128 * h + 32 * q < YS) {
                // products at rows p0 * m + c (a tile's rows are consecutive), the slots
                // below YS (rows >= NC of the table are zero), 16 columns per TMEM load
#pragma unroll 1
                for (int c0 = 16 * g; c0 < NT; c0 += 32) {
                    if (c0 >= ncol) break;
                    float v0[16];
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(S::COL_D0 + st * NT + c0), v0);
                    float* yb = Y + (p0 * m + c0) * YS + n;
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (c0 + i < ncol && n < YS) __stcs(yb + (int64_t)i * YS, v0[i]);
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS));
    }
}

// the autotuner's alternative tile of the real M2L: 80 columns where the default has 96
// (p = 8: three raw stages instead of two), 64 where it has 128, 32 where it has 64 or 48
// (more raw stages in the shared memory freed)
template <int P>
constexpr int tc_alt_columns() {
    return TcTs<P>::NT == 96 ? 80 : TcTs<P>::NT >= 96 ? 64 : 32;
}
static_assert(TcTs<8, false, 80>::RS == 3, "p = 8's alternative tile holds three raw stages");

// columns (pairs x vectors) of a tensor-core M2L tile at degree p (0 to 12)
inline int tc_tile_columns(int p) {
    switch (p) {
        case 0: return TcTs<0>::NT;
        case 1: return TcTs<1>::NT;
        case 2: return TcTs<2>::NT;
        case 3: return TcTs<3>::NT;
        case 4: return TcTs<4>::NT;
        case 5: return TcTs<5>::NT;
        case 6: return TcTs<6>::NT;
        case 7: return TcTs<7>::NT;
        case 8: return TcTs<8>::NT;
        case 9: return TcTs<9>::NT;
        case 10: return TcTs<10>::NT;
        case 11: return TcTs<11>::NT;
        case 12: return TcTs<12>::NT;
        default: return 0;
    }
}

// Host: the tensor map of the multipoles for the gathers: 2D, rows (box * m + vector) of
// ms_of(P) f32 (16-byte multiples), the inner extent (p+1)^2 so that a box of KP slots
// reads zeros past the row's coefficients; boxes of box_rows rows, no swizzle.  The
// driver's encoder is fetched through the runtime (no link against the driver library).
template <int P>
void encode_multipole_map(CUtensorMap* map, const float* M, int64_t rows, int box_rows = 1) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q{};
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            throw std::runtime_error("cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dim[2] = {(cuuint64_t)nc_of(P), (cuuint64_t)(rows > 0 ? rows : 1)};
    const cuuint64_t stride[1] = {(cuuint64_t)ms_of(P) * 4};
    const cuuint32_t box[2] = {(cuuint32_t)TcTs<P>::KP, (cuuint32_t)box_rows};
    const cuuint32_t estride[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(M), dim, stride, box,
                              estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

// Host: the table images for tensor memory, per offset and slot half a hi and a lo part,
// each [128 output slots][KP input slots] of tf32 bits (round to nearest, ties away),
// zero-padded: image[d][h][part][n][k] = A_d[128 h + n][k].
template <int P>
void build_tc_table_images(const std::vector<double>& m2l, std::vector<uint32_t>& img, int count = 316) {
    using S = TcTs<P>;
    constexpr int NC = S::NC;
    img.assign((size_t)count * S::H * S::IMG_WORDS, 0u);
    for (int d = 0; d < count; ++d)
        for (int n = 0; n < NC; ++n)
            for (int k = 0; k < NC; ++k) {
                float a = (float)m2l[(size_t)d * NC * NC + (size_t)k * NC + n];
                uint32_t bits;
                std::memcpy(&bits, &a, 4);
                uint32_t hi = tf32_round_bits(bits);
                float fhi;
                std::memcpy(&fhi, &hi, 4);
                float rem = a - fhi;
                uint32_t rb;
                std::memcpy(&rb, &rem, 4);
                uint32_t lo = tf32_round_bits(rb);
                // image (d, half n / 128): the table index of a tile is d * H + half
                size_t base = ((size_t)d * S::H + n / 128) * S::IMG_WORDS + (size_t)(n % 128) * S::KP + k;
                img[base] = hi;
                img[base + (size_t)128 * S::KP] = lo;
            }
}

// Host: the complex form's images of one level's tables (host layout: per offset a real
// 2n x n matrix, column-major, column j = the local of e_j, real plane over imaginary
// plane), appended to img: per offset d, half 0 holds A_r (rows 0..n), half 1 A_i, each
// [part][128][KP] of tf32 bits; table index (level set * 316 + d) * 2 + half.
template <int P>
void append_tc_complex_images(const std::vector<double>& host, std::vector<uint32_t>& img) {
    using S = TcTs<P, true>;
    constexpr int NC = S::NC;
    const size_t base0 = img.size();
    img.resize(base0 + (size_t)316 * 2 * S::IMG_WORDS, 0u);
    for (int d = 0; d < 316; ++d)
        for (int h = 0; h < 2; ++h)
            for (int n = 0; n < NC; ++n)
                for (int k = 0; k < NC; ++k) {
                    const float a = (float)host[(size_t)d * 2 * NC * NC + (size_t)k * 2 * NC + h * NC + n];
                    uint32_t bits;
                    std::memcpy(&bits, &a, 4);
                    const uint32_t hi = tf32_round_bits(bits);
                    float fhi;
                    std::memcpy(&fhi, &hi, 4);
                    const float rem = a - fhi;
                    uint32_t rb;
                    std::memcpy(&rb, &rem, 4);
                    const size_t at = base0 + ((size_t)d * 2 + h) * S::IMG_WORDS + (size_t)n * S::KP + k;
                    img[at] = hi;
                    img[at + (size_t)128 * S::KP] = tf32_round_bits(rb);
                }
}

}  // namespace fmmb
