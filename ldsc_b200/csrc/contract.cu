// contract.cu -- annotation contraction of banded r2u tiles (K > 1).
//
// The reference contracts each chunk's r2u blocks with the annotation matrix
// in both directions (src/l2/compute.rs:1869-1893, 2259-2314):
//     l2[window] += R_ab * A_chunk,   l2[chunk] += R_ab^T * A_window (+ R_bb A_chunk).
// Here the Gram kernels leave every band tile's masked r2u values in global
// memory (f32) and these passes do the two products per block of rows:
// pass "by right block" owns l2 rows j of one right block, pass "by left
// block" owns l2 rows k of one left block, so no row is written by two CTAs of
// a pass and the summation order is fixed.  Products are f32 over one tile,
// accumulated across tiles in f64.
#include <cuda_runtime.h>

#include "engine.h"

namespace ldsc {

namespace {

constexpr int NT = 128;
constexpr int KC = 16;   // annotation columns per register chunk

template <int TA, int TB, bool BY_RIGHT>
__global__ void __launch_bounds__(NT) k_contract(const float* __restrict__ rtiles, const Tile* __restrict__ tiles,
                                                 const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                 int32_t nblocks, EpilogueArgs ep) {
    extern __shared__ float rs_raw[];
    float (*Rs)[TB + 1] = reinterpret_cast<float (*)[TB + 1]>(rs_raw);
    constexpr int OB = BY_RIGHT ? TB : TA;   // output rows per block
    constexpr int PARTS = NT / OB;           // threads per output row
    const int tid = threadIdx.x;
    const int o = tid % OB, part = tid / OB;
    const int K = ep.K;
    const int64_t m = ep.m;
    const int cbeg = part * K / PARTS, cend = (part + 1) * K / PARTS;
    for (int32_t blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
        const int32_t t0 = ptr[blk], t1 = ptr[blk + 1];
        if (t0 == t1) continue;
        const int64_t row = (int64_t)blk * OB + o;
        // every thread runs the same number of chunks (the block synchronises
        // inside), threads past their column range just skip the products
        const int nch = ((K + PARTS - 1) / PARTS + KC - 1) / KC;
        for (int ci = 0; ci < nch; ci++) {
            const int c0 = cbeg + ci * KC;
            const int nc = cend - c0 < KC ? (cend - c0 > 0 ? cend - c0 : 0) : KC;
            double tot[KC];
#pragma unroll
            for (int c = 0; c < KC; c++) tot[c] = 0.0;
            for (int32_t ti = t0; ti < t1; ti++) {
                const int32_t t = idx[ti];
                const Tile tl = tiles[t];
                const float4* src = reinterpret_cast<const float4*>(rtiles + (size_t)t * TA * TB);
                __syncthreads();
                for (int q = tid; q < TA * TB / 4; q += NT) {
                    const float4 v = __ldg(src + q);
                    const int e = q * 4, r = e / TB, cc = e % TB;
                    Rs[r][cc] = v.x; Rs[r][cc + 1] = v.y; Rs[r][cc + 2] = v.z; Rs[r][cc + 3] = v.w;
                }
                __syncthreads();
                float acc[KC];
#pragma unroll
                for (int c = 0; c < KC; c++) acc[c] = 0.f;
                if (BY_RIGHT) {
                    const int64_t k0 = (int64_t)tl.a_blk * TA;
                    const int kmax = (int)((m - k0) < TA ? (m - k0) : TA);
                    for (int k = 0; k < kmax; k++) {
                        const float r = Rs[k][o];
                        if (r == 0.f) continue;
                        const float* arow = ep.aeff32 + (k0 + k) * K + c0;
#pragma unroll
                        for (int c = 0; c < KC; c++)
                            if (c < nc) acc[c] += r * __ldg(arow + c);
                    }
                } else {
                    const int64_t j0 = (int64_t)tl.b_blk * TB;
                    const int jmax = (int)((m - j0) < TB ? (m - j0) : TB);
                    for (int j = 0; j < jmax; j++) {
                        const float r = Rs[o][j];
                        if (r == 0.f) continue;
                        const float* arow = ep.aeff32 + (j0 + j) * K + c0;
#pragma unroll
                        for (int c = 0; c < KC; c++)
                            if (c < nc) acc[c] += r * __ldg(arow + c);
                    }
                }
#pragma unroll
                for (int c = 0; c < KC; c++) tot[c] += (double)acc[c];
            }
            if (row < m) {
#pragma unroll
                for (int c = 0; c < KC; c++)
                    if (c < nc) ep.l2[row + (int64_t)(c0 + c) * m] += tot[c];
            }
        }
    }
}

}  // namespace

cudaError_t launch_contract(const float* rtiles, int ta, int tb, const Tile* tiles, const int32_t* ptr,
                            const int32_t* idx, int32_t nblocks, bool by_right, const EpilogueArgs& ep,
                            cudaStream_t stream) {
    if (nblocks <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)(nblocks < 148 * 8 ? nblocks : 148 * 8);
    const size_t smem = sizeof(float) * (size_t)ta * (tb + 1);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, NT, smem, stream>>>(rtiles, tiles, ptr, idx, nblocks, ep);
        return cudaGetLastError();
    };
    if (ta == 64 && tb == 128) return by_right ? go(k_contract<64, 128, true>) : go(k_contract<64, 128, false>);
    if (ta == 128 && tb == 128) return by_right ? go(k_contract<128, 128, true>) : go(k_contract<128, 128, false>);
    return cudaErrorInvalidValue;
}

}  // namespace ldsc
