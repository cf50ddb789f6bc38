// Dense M2L on the tensor cores (mixed form): tcgen05.mma kind::tf32 with a 3-term
// split, accumulators in tensor memory.
//
// One CTA (4 warps) takes a tile of up to 128 V pairs of one offset d (the batches of
// m2l_gemm_kernel, 128 pairs wide) and forms D = X * A_d^T, X the 128 gathered source
// multipoles (M = 128 rows, K = the (p+1)^2 input slots padded to KP = 32 * KA),
// A_d^T the table (N = the output slots padded to NP).  f32 data is split as
// x = hi + lo with hi = tf32(x), lo = tf32(x - hi), and
//   D = X_lo A_hi^T + X_hi A_lo^T + X_hi A_hi^T
// (the lo*lo term, 2^-22 relative, is dropped), each product an exact tf32 product
// summed in f32 in TMEM.  Operands are K-major in 128-byte-swizzled shared memory:
// 8-row x 128 B atoms, 16 B chunk c of row r stored at chunk c ^ (r % 8); a K-step of 8
// tf32 (32 B) advances the descriptor start address by 32 B inside an atom, and atoms
// of 32 K-elements follow each other.  The table images (hi and lo) are precomputed on
// the host in exactly this layout, so the CTA copies them verbatim.
//
// Descriptor fields follow cute/arch/mma_sm100_desc.hpp (CUTLASS 4.5): SmemDescriptor
// (start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48), layout [61,64),
// SWIZZLE_128B = 2) and InstrDescriptor (c_format [4,6), a/b_format [7,10)/[10,13),
// a/b_major [15]/[16], N>>3 [17,23), M>>4 [24,29)).
//
// Waits are bounded: a CTA that gives up sets *error and skips its epilogue.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include "harmonics.cuh"

namespace fmmb {

constexpr int kTcRows = 128;  // pairs per tile (UMMA M)

template <int P>
struct TcShape {
    static constexpr int NC = nc_of(P);
    static constexpr int KA = (NC + 31) / 32;                   // K atoms of 32 tf32
    static constexpr int KP = 32 * KA;                          // padded K
    static constexpr int NP = ((NC + 15) / 16) * 16;            // padded N (M = 128 needs N % 16 == 0)
    static constexpr int KSTEPS = KP / 8;
    static constexpr int A_BYTES = kTcRows * KP * 4;            // one part (hi or lo)
    static constexpr int B_BYTES = NP * KP * 4;
    static constexpr int TMEM_COLS = NP <= 32 ? 32 : NP <= 64 ? 64 : NP <= 128 ? 128 : 256;
    static constexpr int SMEM = 2 * A_BYTES + 2 * B_BYTES + 1024 + 64;
    static_assert(NP <= 256, "UMMA N must not exceed 256");
};

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

template <int NP>
__host__ __device__ constexpr uint32_t tf32_idesc() {
    return (1u << 4)                 // D f32
           | (2u << 7) | (2u << 10)  // A, B tf32
           | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t cvt_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
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

// returns true when the barrier's phase `parity` completed within `limit` clock cycles
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, long long limit) {
    const long long start = clock64();
    while (clock64() - start < limit) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Persistent form.  CTA c takes the contiguous range of tiles [c T / G, (c + 1) T / G) of
// the offset-sorted tile list.  The table of the current offset lives in tensor memory
// as the MMA's A operand (M = 128 lanes = output slots, K = input slots in columns; hi
// and lo parts), so the MMA is D[slot][pair] = A_d . X^T with the gathered multipoles X
// as the shared-memory B operand (N = 128 pairs, K-major, 128-byte swizzled), double
// buffered.  Per tile i (16 warps):
//   gather + split X(i) into buffer i&1 (its last reader, MMA(i-2), has completed),
//   wait MMA(i-1); if the offset changes, warps 0-3 store the new table into TMEM,
//   thread 0 issues MMA(i) into accumulator i&1 and commits to the barrier,
//   epilogue(i-1): each thread holds one slot of 16 pairs per TMEM load, so the stores
//   of one pair's row are contiguous across the warp's lanes.
// One vector per launch.
constexpr int kTcWarps = 16;

template <int P>
struct TcTs {
    static constexpr int NC = nc_of(P);
    static constexpr int KA = (NC + 31) / 32;
    static constexpr int KP = 32 * KA;             // padded K (input slots)
    static constexpr int KSTEPS = KP / 8;
    static constexpr int NT = kTcRows;             // pairs per tile (UMMA N)
    static constexpr int X_BYTES = NT * KP * 4;    // one part of one buffer
    static constexpr int SMEM = 4 * X_BYTES + 1024 + 64;
    static constexpr int COL_AHI = 0, COL_ALO = KP, COL_D0 = 2 * KP;  // TMEM columns
    static constexpr int TMEM_COLS = 512;
    static constexpr int IMG_WORDS = 2 * 128 * KP;  // table image words per offset (hi, lo)
    static_assert(NC <= 128, "UMMA M = 128 output slots");
    static_assert(2 * KP + 2 * NT <= TMEM_COLS, "TMEM budget");
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

template <int P>
__global__ void __launch_bounds__(32 * kTcWarps, 1) m2l_tc_kernel(const int32_t* __restrict__ tile_d,
                                                                  const int64_t* __restrict__ tile_begin,
                                                                  const int32_t* __restrict__ tile_count,
                                                                  int64_t ntiles, const int64_t* __restrict__ pair_e,
                                                                  const int32_t* __restrict__ pair_src, int m, int v,
                                                                  const uint32_t* __restrict__ timg,
                                                                  const float* __restrict__ M, float* __restrict__ Y,
                                                                  int* __restrict__ error) {
    using S = TcTs<P>;
    constexpr int NC = S::NC;
    constexpr int kGather = kTcWarps / 2;     // warps 8..15 gather, warps 0..7 run the epilogue
    constexpr int RPW = S::NT / kGather;      // gathered rows per gather warp
    extern __shared__ unsigned char smem_raw[];
    unsigned char* xbuf = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);  // [2 bufs][hi, lo]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __shared__ uint64_t mbar[2];  // MMA(k) commits to mbar[k & 1] (k counted from the CTA's first tile)
    __shared__ uint32_t tmem_base;
    // tile k's row indices live from its gather (iteration k-1) to its epilogue
    // (iteration k+1): three slots, slot (k - i0) % 3
    __shared__ int32_t row_src[3][S::NT];
    __shared__ int64_t row_e[3][S::NT];
    __shared__ int32_t row_cnt[3];
    const int64_t i0 = (int64_t)blockIdx.x * ntiles / gridDim.x;
    const int64_t i1 = (int64_t)(blockIdx.x + 1) * ntiles / gridDim.x;
    if (i0 >= i1) return;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(S::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    constexpr uint32_t idesc = tf32_idesc_ts<S::NT>();

    auto rows = [&](int64_t it, int b) {  // threads 0..127: the tile's row indices into meta slot b
        const int64_t p0 = tile_begin[it];
        const int cnt = tile_count[it];
        if (tid < S::NT) {
            row_src[b][tid] = tid < cnt ? pair_src[p0 + tid] : 0;
            row_e[b][tid] = tid < cnt ? pair_e[p0 + tid] : 0;
        }
        if (tid == 0) row_cnt[b] = cnt;
    };
    // gather + split X into buffer xb from meta slot b (gather warps, gw = 0..kGather-1):
    // every load of a warp's rows is issued before any is converted and stored
    auto gather = [&](int xb, int b, int gw) {
        const int cnt = row_cnt[b];
        unsigned char* xh = xbuf + (size_t)xb * 2 * S::X_BYTES;
        unsigned char* xl = xh + S::X_BYTES;
        float x[RPW][S::KA];
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = gw + kGather * j;
            const float* src = M + ((int64_t)row_src[b][r] * m + v) * NC;
#pragma unroll
            for (int a = 0; a < S::KA; ++a) {
                const int k = a * 32 + lane;
                x[j][a] = (r < cnt && k < NC) ? __ldg(src + k) : 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = gw + kGather * j;
#pragma unroll
            for (int a = 0; a < S::KA; ++a) {
                const int k = a * 32 + lane;
                const uint32_t hi = cvt_tf32(x[j][a]);
                const uint32_t lo = cvt_tf32(x[j][a] - __uint_as_float(hi));
                const uint32_t off = sw128_offset(r, k, S::NT);
                *reinterpret_cast<uint32_t*>(xh + off) = hi;
                *reinterpret_cast<uint32_t*>(xl + off) = lo;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    };
    // the table of offset d into TMEM (warps 0..3, one per lane quarter)
    auto load_table = [&](int d) {
        if (warp < 4) {
            const uint32_t* src = timg + (size_t)d * S::IMG_WORDS;
#pragma unroll 1
            for (int part = 0; part < 2; ++part)
#pragma unroll 1
                for (int k0 = 0; k0 < S::KP; k0 += 16) {
                    uint32_t r[16];
                    const uint4* row =
                        reinterpret_cast<const uint4*>(src + ((size_t)part * 128 + 32 * warp + lane) * S::KP + k0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const uint4 u = __ldg(row + q);
                        r[4 * q] = u.x;
                        r[4 * q + 1] = u.y;
                        r[4 * q + 2] = u.z;
                        r[4 * q + 3] = u.w;
                    }
                    tmem_st16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)((part ? S::COL_ALO : S::COL_AHI) + k0),
                              r);
                }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        }
    };
    auto issue = [&](int b) {  // thread 0: MMA of X buffer b into accumulator b, commit to mbar[b]
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t xh = smem_u32(xbuf + (size_t)b * 2 * S::X_BYTES), xl = xh + S::X_BYTES;
        const uint32_t dcol = tmem + (uint32_t)(S::COL_D0 + b * S::NT);
        const uint32_t As[3] = {(uint32_t)S::COL_AHI, (uint32_t)S::COL_ALO, (uint32_t)S::COL_AHI};
        const uint32_t Bs[3] = {xl, xh, xh};  // A_hi X_lo, A_lo X_hi, then A_hi X_hi
        uint32_t acc = 0;
#pragma unroll
        for (int t = 0; t < 3; ++t)
#pragma unroll
            for (int s = 0; s < S::KSTEPS; ++s) {
                const uint32_t kb = (uint32_t)((s >> 2) * S::NT * 128 + (s & 3) * 32);
                umma_tf32_ts(dcol, tmem + As[t] + (uint32_t)(8 * s), sw128_desc(Bs[t] + kb), idesc, acc);
                acc = 1;
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar[b]))
                     : "memory");
    };
    // accumulator db with meta slot b (epilogue warps 0..7): lanes = slots, columns = pairs
    auto epilogue = [&](int db, int b) {
        const int q = warp & 3, g = warp >> 2;  // lane quarter, column group (64 pairs)
        const int n = 32 * q + lane;
        if (32 * q >= NC) return;  // the whole quarter is padding
        const int cnt = row_cnt[b];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int c0 = 64 * g + 16 * h;
            if (c0 >= cnt) break;
            float vals[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(S::COL_D0 + db * S::NT + c0), vals);
            if (n < NC) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i < cnt) __stcs(Y + (row_e[b][c0 + i] * m + v) * NC + n, vals[i]);  // streamed
            }
        }
    };
    // MMA(k) done: all threads wait, the CTA agrees on the outcome
    bool failed = false;
    auto wait_mma = [&](int64_t k) {
        const int b = (int)((k - i0) & 1);
        const uint32_t parity = (uint32_t)(((k - i0) >> 1) & 1);
        const bool ok = mbar_wait_bounded(smem_u32(&mbar[b]), parity, 4000000000LL);
        if (__syncthreads_or(!ok)) {
            failed = true;
            if (tid == 0) atomicExch(error, 1);
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
    };

    auto meta = [&](int64_t k) { return (int)((k - i0) % 3); };
    int cur_d = tile_d[i0];
    rows(i0, 0);
    __syncthreads();
    if (warp >= kGather) gather(0, 0, warp - kGather);
    load_table(cur_d);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (tid == 0) issue(0);
    __syncwarp();
    for (int64_t it = i0; it < i1; ++it) {
        const int b = (int)((it - i0) & 1);
        if (it > i0) {
            wait_mma(it - 1);  // X buffer b^1 and accumulator b^1 are free / readable
            if (failed) break;
        }
        const bool next = it + 1 < i1;
        if (next) rows(it + 1, meta(it + 1));
        __syncthreads();
        if (warp >= kGather) {
            if (next) gather(b ^ 1, meta(it + 1), warp - kGather);
        } else if (it > i0) {
            epilogue(b ^ 1, meta(it - 1));
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (next) {
            const int d = tile_d[it + 1];
            if (d != cur_d) {  // MMA(it) still reads the old table: wait for it first
                wait_mma(it);
                if (failed) break;
                load_table(d);
                cur_d = d;
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncthreads();
            }
            if (tid == 0) issue(b ^ 1);
            __syncwarp();
        }
    }
    if (!failed) {
        wait_mma(i1 - 1);
        if (!failed && warp < kGather) epilogue((int)((i1 - 1 - i0) & 1), meta(i1 - 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS));
    }
}

// Host: the table images for tensor memory, per offset a hi and a lo part, each
// [128 output slots][KP input slots] of tf32 bits (round to nearest, ties away),
// zero-padded: image[d][part][n][k] = A_d[n][k].
template <int P>
void build_tc_table_images(const std::vector<double>& m2l, std::vector<uint32_t>& img) {
    using S = TcTs<P>;
    constexpr int NC = S::NC;
    img.assign((size_t)316 * S::IMG_WORDS, 0u);
    for (int d = 0; d < 316; ++d)
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
                size_t base = (size_t)d * S::IMG_WORDS + (size_t)n * S::KP + k;
                img[base] = hi;
                img[base + (size_t)128 * S::KP] = lo;
            }
}

}  // namespace fmmb
