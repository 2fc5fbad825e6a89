// synth.cu -- seeded synthetic BED panels on the device (benchmark input).
//
// Byte-identical to the numpy generator in ldsc_b200/synth.py: every draw is
// splitmix64(splitmix64(seed + stream*KS + a*KA) + b), uniforms are the top 53
// bits, bounded draws are multiply-shift.  Floating-point steps are written
// with explicit round-to-nearest intrinsics so that no fused multiply-add
// changes a comparison relative to numpy.
#include <cuda_runtime.h>

#include "engine.h"

namespace ldsc {

namespace {

constexpr uint64_t G0 = 0x9E3779B97F4A7C15ull, G1 = 0xBF58476D1CE4E5B9ull,
                   G2 = 0x94D049BB133111EBull, KS = 0xD1B54A32D192ED03ull,
                   KA = 0xAEF17502108EF2D9ull;

__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
    uint64_t z = x + G0;
    z = (z ^ (z >> 30)) * G1;
    z = (z ^ (z >> 27)) * G2;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t draw(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b) {
    return splitmix(splitmix(seed + stream * KS + a * KA) + b);
}

__device__ __forceinline__ double u01(uint64_t h) {
    return __dmul_rn((double)(h >> 11), 1.0 / 9007199254740992.0);
}

__device__ __forceinline__ uint32_t bounded(uint64_t h, uint32_t n) {
    return (uint32_t)(((h >> 32) * (uint64_t)n) >> 32);
}

__global__ void k_founders(uint8_t* table, uint32_t founders, uint64_t n_snp, uint64_t seed) {
    uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_snp) return;
    double p = __dadd_rn(0.01, __dmul_rn(0.49, u01(draw(seed, 6, 0, j))));
    if (draw(seed, 7, 0, j) & 1ull) p = __dsub_rn(1.0, p);
    for (uint32_t f = 0; f < founders; f++)
        table[(uint64_t)f * n_snp + j] = u01(draw(seed, 1, f, j)) < p ? 1 : 0;
}

constexpr int SEG = 1024;

// One thread per (BED byte column = 4 individuals, segment of SEG SNPs).
__global__ void k_synth(uint8_t* rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                        uint32_t founders, double switch_p, double miss, uint64_t seed,
                        const uint8_t* __restrict__ table) {
    const uint64_t bcol = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t bpr = (n_indiv + 3) / 4;
    if (bcol >= bpr) return;
    const uint64_t j0 = (uint64_t)blockIdx.y * SEG;
    if (j0 >= n_snp) return;
    const uint64_t j1 = j0 + SEG < n_snp ? j0 + SEG : n_snp;
    uint32_t state[8];
    // founder state at j0: the last switch at or before j0 (switches start at j = 1)
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const uint64_t h = bcol * 8 + t;
        uint32_t s = bounded(draw(seed, 3, h, ~0ull), founders);
        for (uint64_t jj = j0; jj >= 1; jj--) {
            if (u01(draw(seed, 2, h, jj)) < switch_p) {
                s = bounded(draw(seed, 3, h, jj), founders);
                break;
            }
        }
        state[t] = s;
    }
    for (uint64_t j = j0; j < j1; j++) {
        uint32_t byte = 0;
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const uint64_t h = bcol * 8 + t;
            if (j > j0 && u01(draw(seed, 2, h, j)) < switch_p) state[t] = bounded(draw(seed, 3, h, j), founders);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint64_t i = bcol * 4 + q;
            uint32_t code = 0;
            if (i < n_indiv) {
                const uint32_t g = table[(uint64_t)state[2 * q] * n_snp + j] +
                                   table[(uint64_t)state[2 * q + 1] * n_snp + j];
                code = g == 2 ? 0u : (g == 1 ? 2u : 3u);
                if (u01(draw(seed, 4, i, j)) < miss) code = 1u;
            }
            byte |= code << (2 * q);
        }
        rows[j * pitch + bcol] = (uint8_t)byte;
    }
}

}  // namespace

cudaError_t launch_synth(uint8_t* rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                         uint32_t founders, double switch_p, double miss, uint64_t seed,
                         uint8_t* founder_table, cudaStream_t stream) {
    if (n_snp == 0) return cudaSuccess;
    k_founders<<<(unsigned)((n_snp + 255) / 256), 256, 0, stream>>>(founder_table, founders, n_snp, seed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint64_t bpr = (n_indiv + 3) / 4;
    dim3 grid((unsigned)((bpr + 127) / 128), (unsigned)((n_snp + SEG - 1) / SEG));
    k_synth<<<grid, 128, 0, stream>>>(rows, pitch, n_indiv, n_snp, founders, switch_p, miss, seed,
                                      founder_table);
    return cudaGetLastError();
}

cudaError_t preload_synth() {
    cudaError_t e = preload_kernel(k_founders);
    if (e == cudaSuccess) e = preload_kernel(k_synth);
    return e;
}

}  // namespace ldsc
