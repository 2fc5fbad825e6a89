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

constexpr int NT = 256;
constexpr int CC = 32;  // annotation columns per CTA

// Grid: (output block, 32-column chunk), chunk fastest so the CTAs of one
// output block run together and share its r2u tiles through L2.  Per tile the
// r2u tile and the 32 annotation columns of the other side are staged in
// shared memory; each thread owns RJ output rows x 4 columns, accumulates the
// tile's products in f32 and the tiles in f64.
//   BY_RIGHT: out rows j of the right block, out[j][c] += sum_k R[k][j] A[k][c]  (RJ = 4)
//   BY_LEFT:  out rows k of the left block,  out[k][c] += sum_j R[k][j] A[j][c]  (RJ = 2)
template <int TA, int TB, bool BY_RIGHT>
__global__ void __launch_bounds__(NT, 3) k_contract(const float* __restrict__ rtiles, const Tile* __restrict__ tiles,
                                                    const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                    int32_t nblocks, EpilogueArgs ep) {
    constexpr int OB = BY_RIGHT ? TB : TA;       // output rows per block
    constexpr int NS = BY_RIGHT ? TA : TB;       // summed index extent per tile
    constexpr int RJ = OB / 32;                  // output rows per thread
    extern __shared__ float sm_raw[];
    float (*Rs)[TB + 1] = reinterpret_cast<float (*)[TB + 1]>(sm_raw);  // [TA][TB + 1]
    float4* As = reinterpret_cast<float4*>(sm_raw + TA * (TB + 1));     // [NS][CC / 4]
    const int tid = threadIdx.x;
    const int og = tid & 31, cg = tid >> 5;      // rows og + 32 i, columns 4 cg .. 4 cg + 3
    const int K = ep.K;
    const int64_t m = ep.m;
    const int nchunks = (K + CC - 1) / CC;
    for (int64_t w = blockIdx.x; w < (int64_t)nblocks * nchunks; w += gridDim.x) {
        const int32_t blk = (int32_t)(w / nchunks);
        const int c0 = (int)(w % nchunks) * CC;
        const int32_t t0 = ptr[blk], t1 = ptr[blk + 1];
        if (t0 == t1) continue;
        double tot[RJ][4];
#pragma unroll
        for (int i = 0; i < RJ; i++)
#pragma unroll
            for (int u = 0; u < 4; u++) tot[i][u] = 0.0;
        for (int32_t ti = t0; ti < t1; ti++) {
            const int32_t t = idx[ti];
            const Tile tl = tiles[t];
            const float4* src = reinterpret_cast<const float4*>(rtiles + (size_t)t * TA * TB);
            // rows of the summed side of this tile
            const int64_t s0 = BY_RIGHT ? (int64_t)tl.a_blk * TA : (int64_t)tl.b_blk * TB;
            __syncthreads();  // the previous tile's stages are no longer read
            for (int q = tid; q < TA * TB / 4; q += NT) {
                const float4 v = __ldg(src + q);
                const int e = q * 4, r = e / TB, cc = e % TB;
                Rs[r][cc] = v.x;
                Rs[r][cc + 1] = v.y;
                Rs[r][cc + 2] = v.z;
                Rs[r][cc + 3] = v.w;
            }
            for (int q = tid; q < NS * CC; q += NT) {
                const int r = q / CC, c = q % CC;
                const int64_t srow = s0 + r;
                const float v = (srow < m && c0 + c < K) ? __ldg(ep.aeff32 + srow * K + c0 + c) : 0.f;
                reinterpret_cast<float*>(As)[r * CC + c] = v;
            }
            __syncthreads();
            float acc[RJ][4];
#pragma unroll
            for (int i = 0; i < RJ; i++)
#pragma unroll
                for (int u = 0; u < 4; u++) acc[i][u] = 0.f;
#pragma unroll 4
            for (int sidx = 0; sidx < NS; sidx++) {
                const float4 a = As[sidx * (CC / 4) + cg];
#pragma unroll
                for (int i = 0; i < RJ; i++) {
                    const float r = BY_RIGHT ? Rs[sidx][og + 32 * i] : Rs[og + 32 * i][sidx];
                    acc[i][0] += r * a.x;
                    acc[i][1] += r * a.y;
                    acc[i][2] += r * a.z;
                    acc[i][3] += r * a.w;
                }
            }
#pragma unroll
            for (int i = 0; i < RJ; i++)
#pragma unroll
                for (int u = 0; u < 4; u++) tot[i][u] += (double)acc[i][u];
        }
#pragma unroll
        for (int i = 0; i < RJ; i++) {
            const int64_t row = (int64_t)blk * OB + og + 32 * i;
            if (row >= m) continue;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int c = c0 + 4 * cg + u;
                if (c < K) ep.l2[row + (int64_t)c * m] += tot[i][u];
            }
        }
    }
}

}  // namespace

cudaError_t launch_contract(const float* rtiles, int ta, int tb, const Tile* tiles, const int32_t* ptr,
                            const int32_t* idx, int32_t nblocks, bool by_right, const EpilogueArgs& ep,
                            cudaStream_t stream) {
    if (nblocks <= 0) return cudaSuccess;
    const int nchunks = (ep.K + CC - 1) / CC;
    const int64_t work = (int64_t)nblocks * nchunks;
    const unsigned grid = (unsigned)(work < 148 * 8 ? work : 148 * 8);
    auto go = [&](auto kern, int ns) {
        const size_t smem = sizeof(float) * ((size_t)ta * (tb + 1) + (size_t)ns * CC);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, NT, smem, stream>>>(rtiles, tiles, ptr, idx, nblocks, ep);
        return cudaGetLastError();
    };
    if (ta == 64 && tb == 128)
        return by_right ? go(k_contract<64, 128, true>, 64) : go(k_contract<64, 128, false>, 128);
    if (ta == 128 && tb == 128)
        return by_right ? go(k_contract<128, 128, true>, 128) : go(k_contract<128, 128, false>, 128);
    return cudaErrorInvalidValue;
}

}  // namespace ldsc
