// expand.cuh -- packed 2-bit BED words into INT8 genotype / non-missing
// operand bytes in shared memory, for the fused Gram forms (the converter
// warps of gram_tc.cu and gram_pair.cu).
#pragma once
#include <cstdint>

namespace ldsc {

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Genotype and non-missing bytes of 16 individuals from their code word
// (count-A1 codes, src/bed.rs:470-521: 00 -> 2, 01 -> missing, 10 -> 1,
// 11 -> 0).  Byte order in the chunk: individuals 0,2,..,14 then 1,3,..,15.
__device__ __forceinline__ void expand_chunk(uint32_t w, uint4& g, uint4& mk) {
    constexpr uint32_t TG = 0x00010002u;           // code c -> byte c of TG
    constexpr uint32_t TM = 0x01010001u;
    const uint32_t se = w & 0x33333333u;           // nibble i: code of individual 2i
    const uint32_t so = (w >> 2) & 0x33333333u;    // nibble i: code of individual 2i + 1
    const uint32_t se2 = se >> 16, so2 = so >> 16;
    g.x = __byte_perm(TG, 0u, se);
    g.y = __byte_perm(TG, 0u, se2);
    g.z = __byte_perm(TG, 0u, so);
    g.w = __byte_perm(TG, 0u, so2);
    mk.x = __byte_perm(TM, 0u, se);
    mk.y = __byte_perm(TM, 0u, se2);
    mk.z = __byte_perm(TM, 0u, so);
    mk.w = __byte_perm(TM, 0u, so2);
}

// Byte offset of 16-byte chunk c of row R in a K-major 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t sw128_off(int R, int c) {
    return (uint32_t)((R >> 3) * 1024 + (R & 7) * 128 + ((c ^ (R & 7)) << 4));
}

}  // namespace ldsc
