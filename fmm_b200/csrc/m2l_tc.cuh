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

// Persistent form: CTA c takes the contiguous range of tiles [c T / G, (c + 1) T / G) of
// the offset-sorted tile list, so the table image changes only a few times per CTA.
// 16 warps: all of them gather (loads of a warp's 8 rows issued before use) and convert
// A; thread 0 issues the MMAs; the epilogue of tile i-1 (TMEM buffer (i-1)&1, read by
// the 4 warps of each TMEM lane quarter, 16 columns at a time, staged per warp so that
// stores run along Y rows) overlaps MMA(i) into buffer i&1.  One vector per launch.
constexpr int kTcWarps = 16;

template <int P>
struct TcShape2 : TcShape<P> {
    static constexpr int OUT_BYTES = kTcWarps * 32 * 17 * 4;  // per-warp 32 x 16 epilogue tiles
    static constexpr int SMEM2 = 2 * TcShape<P>::A_BYTES + 2 * TcShape<P>::B_BYTES + OUT_BYTES + 1024 + 64;
};

template <int P>
__global__ void __launch_bounds__(32 * kTcWarps, 1) m2l_tc_kernel(const int32_t* __restrict__ tile_d,
                                                                  const int64_t* __restrict__ tile_begin,
                                                                  const int32_t* __restrict__ tile_count,
                                                                  int64_t ntiles, const int64_t* __restrict__ pair_e,
                                                                  const int32_t* __restrict__ pair_src, int m, int v,
                                                                  const uint4* __restrict__ bimg,
                                                                  const float* __restrict__ M, float* __restrict__ Y,
                                                                  int* __restrict__ error) {
    using S = TcShape2<P>;
    constexpr int NC = S::NC;
    constexpr int RPW = kTcRows / kTcWarps;  // rows per warp in the gather
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    unsigned char* a_hi = base;
    unsigned char* a_lo = a_hi + S::A_BYTES;
    unsigned char* b_hi = a_lo + S::A_BYTES;
    unsigned char* b_lo = b_hi + S::B_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* outw = reinterpret_cast<float*>(b_lo + S::B_BYTES) + warp * 32 * 17;
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int32_t row_src[kTcRows];
    __shared__ int64_t row_e[2][kTcRows];
    const int64_t i0 = (int64_t)blockIdx.x * ntiles / gridDim.x;
    const int64_t i1 = (int64_t)(blockIdx.x + 1) * ntiles / gridDim.x;
    if (i0 >= i1) return;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(2 * S::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = tf32_idesc<S::NP>();
    int cur_d = -1;
    uint32_t phase = 0;
    bool failed = false;
    int prev_cnt = 0;

    auto epilogue = [&](int buf, int cnt) {
        const int quarter = warp & 3;        // TMEM lanes 32 quarter .. + 31
        const int rw = 32 * quarter;
        const int half = lane >> 4, col = lane & 15;
        for (int c0 = 16 * (warp >> 2); c0 < S::NP; c0 += 16 * (kTcWarps / 4)) {
            float vals[16];
            tmem_ld16(tmem + (uint32_t)(buf * S::TMEM_COLS) + ((uint32_t)rw << 16) + (uint32_t)c0, vals);
#pragma unroll
            for (int i = 0; i < 16; ++i) outw[lane * 17 + i] = vals[i];
            __syncwarp();
            if (c0 + col < NC) {
#pragma unroll 4
                for (int rr = half; rr < 32; rr += 2) {
                    const int r = rw + rr;
                    if (r < cnt) Y[(row_e[buf][r] * m + v) * NC + c0 + col] = outw[rr * 17 + col];
                }
            }
            __syncwarp();
        }
    };

    for (int64_t it = i0; it < i1 && !failed; ++it) {
        const int buf = (int)((it - i0) & 1);
        if (it > i0) {  // MMA(it-1) done: A and B may be overwritten
            const bool ok = mbar_wait_bounded(smem_u32(&mbar), phase, 4000000000LL);
            if (__syncthreads_or(!ok)) {  // the CTA leaves together, so no barrier is left waiting
                failed = true;
                if (tid == 0) atomicExch(error, 1);
                break;
            }
            phase ^= 1;
            asm volatile("tcgen05.fence::after_thread_sync;");
        }
        const int d = tile_d[it];
        const int64_t p0 = tile_begin[it];
        const int cnt = tile_count[it];
        if (d != cur_d) {
            const uint4* src = bimg + (size_t)d * (2 * S::B_BYTES / 16);
            uint4* dst = reinterpret_cast<uint4*>(b_hi);
            for (int i = tid; i < 2 * S::B_BYTES / 16; i += 32 * kTcWarps) dst[i] = src[i];
            cur_d = d;
        }
        if (tid < kTcRows) {
            row_src[tid] = tid < cnt ? pair_src[p0 + tid] : 0;
            row_e[buf][tid] = tid < cnt ? pair_e[p0 + tid] : 0;
        }
        __syncthreads();
        // gather + split: warp w holds rows w + 16 j; every load is issued before any use
        float x[RPW][S::KA];
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = warp + kTcWarps * j;
            const float* src = M + ((int64_t)row_src[r] * m + v) * NC;
#pragma unroll
            for (int a = 0; a < S::KA; ++a) {
                const int k = a * 32 + lane;
                x[j][a] = (r < cnt && k < NC) ? __ldg(src + k) : 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = warp + kTcWarps * j;
#pragma unroll
            for (int a = 0; a < S::KA; ++a) {
                const int k = a * 32 + lane;
                const uint32_t hi = cvt_tf32(x[j][a]);
                const uint32_t lo = cvt_tf32(x[j][a] - __uint_as_float(hi));
                const uint32_t off = sw128_offset(r, k, kTcRows);
                *reinterpret_cast<uint32_t*>(a_hi + off) = hi;
                *reinterpret_cast<uint32_t*>(a_lo + off) = lo;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t sa_hi = smem_u32(a_hi), sa_lo = smem_u32(a_lo);
            const uint32_t sb_hi = smem_u32(b_hi), sb_lo = smem_u32(b_lo);
            const uint32_t dcol = tmem + (uint32_t)(buf * S::TMEM_COLS);
            uint32_t acc = 0;
            const uint32_t As[3] = {sa_lo, sa_hi, sa_hi}, Bs[3] = {sb_hi, sb_lo, sb_hi};
#pragma unroll
            for (int t = 0; t < 3; ++t)
#pragma unroll
                for (int s = 0; s < S::KSTEPS; ++s) {
                    const uint32_t ka = (uint32_t)((s >> 2) * kTcRows * 128 + (s & 3) * 32);
                    const uint32_t kb = (uint32_t)((s >> 2) * S::NP * 128 + (s & 3) * 32);
                    umma_tf32(dcol, sw128_desc(As[t] + ka), sw128_desc(Bs[t] + kb), idesc, acc);
                    acc = 1;
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        __syncwarp();
        if (it > i0) epilogue(buf ^ 1, prev_cnt);  // overlaps MMA(it)
        prev_cnt = cnt;
    }
    if (!failed) {
        const bool ok = mbar_wait_bounded(smem_u32(&mbar), phase, 4000000000LL);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(error, 1);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;");
            epilogue((int)((i1 - 1 - i0) & 1), prev_cnt);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * S::TMEM_COLS));
    }
}

// Host: the table images, hi and lo parts per offset, in the SW128 K-major layout with
// B[n][k] = A_d[n][k] (output slot n, input slot k), zero padding.
template <int P>
void build_tc_table_images(const std::vector<double>& m2l, std::vector<uint32_t>& img) {
    using S = TcShape<P>;
    constexpr int NC = S::NC;
    const size_t part = S::B_BYTES / 4;
    img.assign(316 * 2 * part, 0u);
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
                size_t o = sw128_offset(n, k, S::NP) / 4;
                img[(size_t)d * 2 * part + o] = hi;
                img[(size_t)d * 2 * part + part + o] = lo;
            }
}

}  // namespace fmmb
