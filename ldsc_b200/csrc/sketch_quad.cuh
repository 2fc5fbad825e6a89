// sketch_quad.cuh -- the bit-plane quad of the CountSketch layout.
//
// A permuted row is stored as 16-byte quads of 64 positions.  Each quad holds
// the two bits of every 2-bit BED code in separate planes, 32 positions per
// word:
//     word 0 = low bits (b0) of positions  0..31    word 1 = high bits (b1) of 0..31
//     word 2 = low bits      of positions 32..63    word 3 = high bits      of 32..63
// bit t of a word = position t of its half.  The BED codes (b1 b0) are
// 00 -> genotype 2, 10 -> 1, 11 -> 0, 01 = missing (positions past the used
// individuals are written as missing), so over any span
//     bits    = popc(b0) + popc(b1)           (the code's bit count)
//     missing = popc(b0 & ~b1)
//     sum g   = 2 len - bits - missing,       present = len - missing
//     #2      = len - popc(b1) - missing      (code 00)
// Kept apart from the interleaved 2-bit form, the missing test is one logic
// operation per 32 positions and the genotype-2 count needs no popcount of
// its own.  Host and device share these helpers.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace ldsc {

__host__ __device__ __forceinline__ int32_t popc32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}

// Bits, missing positions and high bits over the whole quad.
__host__ __device__ __forceinline__ void quad_counts(uint4 v, int32_t& bits, int32_t& miss, int32_t& high) {
    high = popc32(v.y) + popc32(v.w);
    bits = popc32(v.x) + popc32(v.z) + high;
    miss = popc32(v.x & ~v.y) + popc32(v.z & ~v.w);
}

// The same, with the bits and missing positions of the first half (0..31).
__host__ __device__ __forceinline__ void quad_counts(uint4 v, int32_t& bits, int32_t& miss, int32_t& high,
                                                     int32_t& bits0, int32_t& miss0) {
    const int32_t cy = popc32(v.y), cw = popc32(v.w);
    bits0 = popc32(v.x) + cy;
    miss0 = popc32(v.x & ~v.y);
    high = cy + cw;
    bits = bits0 + popc32(v.z) + cw;
    miss = miss0 + popc32(v.z & ~v.w);
}

// Bits and missing positions at quad positions [0, j), 0 <= j < 64.
__host__ __device__ __forceinline__ void quad_head(uint4 v, uint32_t j, int32_t& bits, int32_t& miss) {
    const uint32_t m0 = j >= 32 ? 0xFFFFFFFFu : (j ? 0xFFFFFFFFu >> (32 - j) : 0u);
    const uint32_t m1 = j > 32 ? 0xFFFFFFFFu >> (64 - j) : 0u;
    bits = popc32(v.x & m0) + popc32(v.y & m0) + popc32(v.z & m1) + popc32(v.w & m1);
    miss = popc32(v.x & ~v.y & m0) + popc32(v.z & ~v.w & m1);
}

// Bits and missing positions at half positions [0, j), 0 <= j < 32, from the
// half's (low, high) plane words.
__host__ __device__ __forceinline__ void half_head(uint32_t lo, uint32_t hi, uint32_t j, int32_t& bits,
                                                   int32_t& miss) {
    const uint32_t m = j ? 0xFFFFFFFFu >> (32 - j) : 0u;
    bits = popc32(lo & m) + popc32(hi & m);
    miss = popc32(lo & ~hi & m);
}

}  // namespace ldsc
