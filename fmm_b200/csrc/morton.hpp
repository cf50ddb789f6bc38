// Morton keys of the reference's octree (octree/src/morton.rs): the three level-16 index
// bits of each level interleaved, x highest, shifted left 15, the level in the low 15 bits.
// Host and device.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define FMMB_HD __host__ __device__
#else
#define FMMB_HD
#endif

namespace fmmb {

FMMB_HD inline uint64_t morton_spread3(uint64_t x) {
    x &= 0xFFFF;
    x = (x | (x << 32)) & 0x1F00000000FFFFULL;
    x = (x | (x << 16)) & 0x1F0000FF0000FFULL;
    x = (x | (x << 8)) & 0x100F00F00F00F00FULL;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

// the key of the box (i, j, k) of `level` (indices on that level)
FMMB_HD inline uint64_t morton_encode_hd(uint32_t i, uint32_t j, uint32_t k, int level) {
    const int d = 16 - level;
    const uint64_t m = (morton_spread3((uint64_t)i << d) << 2) | (morton_spread3((uint64_t)j << d) << 1) |
                       morton_spread3((uint64_t)k << d);
    return (m << 15) | (uint64_t)level;
}

}  // namespace fmmb
