// contract.cu -- annotation contraction of banded r2u tiles (K > 1), in f64.
//
// The reference contracts each chunk's r2u blocks with the annotation matrix
// in both directions (src/l2/compute.rs:1869-1893, 2259-2314):
//     l2[window] += R_ab * A_chunk,   l2[chunk] += R_ab^T * A_window (+ R_bb A_chunk).
// Here the Gram kernels leave every band tile's masked r2u values in global
// memory (f64, row k of the tile = TB values) and these passes do the two
// products per block of rows: pass "by right block" owns l2 rows j of one
// right block, pass "by left block" owns l2 rows k of one left block, so no
// row is written by two CTAs of a pass and the summation order is fixed.
// Everything is f64 -- the r2u values as the epilogue formed them, the
// effective annotations as given, the products and sums -- so each l2_jC
// carries f64 rounding only, binary and continuous columns alike.
#include <cuda_runtime.h>

#include "engine.h"

namespace ldsc {

namespace {

constexpr int NT = 256;
constexpr int CW = 8;              // annotation columns per warp
constexpr int CC = CW * NT / 32;   // annotation columns per CTA
constexpr int ALD = CC + 2;        // staged annotation row stride (even: 16-byte reads; staging stores 2-way)

// Grid: (output block, CC-column chunk), chunk fastest so the CTAs of one
// output block run together and share its r2u tiles through L2.  Per tile,
// in steps of JS summed records, the step's r2u values (padded row stride:
// the lanes that read one column hit distinct bank pairs) and the CC
// annotation columns of those records are staged in shared memory; thread
// (og, cg) owns output rows og + 32 i (i < RJ) and columns CW cg .. CW cg +
// CW - 1, in f64 registers across all tiles of the block.  Per summed record a
// warp reads its CW annotation values as broadcasts and RJ r2u values, for
// RJ x CW fused multiply-adds.  Warps whose columns lie past K skip the
// products.  The left-block pass stages 64 of a tile's 128 right records at a
// time, which keeps its shared memory at 67 KB (three CTAs per SM).
//   BY_RIGHT: out rows j of the right block, out[j][c] += sum_k R[k][j] A[k][c]  (RJ = TB / 32)
//   BY_LEFT:  out rows k of the left block,  out[k][c] += sum_j R[k][j] A[j][c]  (RJ = TA / 32)
template <int TA, int TB, bool BY_RIGHT>
struct ContractShape {
    static constexpr int OB = BY_RIGHT ? TB : TA;          // output rows per block
    static constexpr int NS = BY_RIGHT ? TA : TB;          // summed records per tile
    static constexpr int JS = BY_RIGHT ? NS : 64;          // summed records per staging step
    static constexpr int RLD = BY_RIGHT ? TB + 1 : JS + 1; // staged r2u row stride (doubles)
    static constexpr int RROWS = BY_RIGHT ? JS : TA;       // staged r2u rows
    static constexpr size_t smem = sizeof(double) * ((size_t)RROWS * RLD + (size_t)JS * ALD);
};

template <int TA, int TB, bool BY_RIGHT>
__global__ void __launch_bounds__(NT) k_contract(const double* __restrict__ rtiles, const Tile* __restrict__ tiles,
                                                 const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                 int32_t nblocks, EpilogueArgs ep) {
    using S = ContractShape<TA, TB, BY_RIGHT>;
    constexpr int OB = S::OB, NS = S::NS, JS = S::JS, RLD = S::RLD, RROWS = S::RROWS;
    constexpr int RJ = OB / 32;                  // output rows per thread
    extern __shared__ double smd[];
    double* Rs = smd;                            // BY_RIGHT: [JS k][TB j]; BY_LEFT: [TA k][JS j]
    double* As = smd + RROWS * RLD;              // [JS][ALD]
    const int tid = threadIdx.x;
    const int og = tid & 31, cg = tid >> 5;
    const int K = ep.K;
    const int64_t m = ep.m;
    const int nchunks = (K + CC - 1) / CC;
    for (int64_t w = blockIdx.x; w < (int64_t)nblocks * nchunks; w += gridDim.x) {
        const int32_t blk = (int32_t)(w / nchunks);
        const int c0 = (int)(w % nchunks) * CC;
        const int32_t t0 = ptr[blk], t1 = ptr[blk + 1];
        if (t0 == t1) continue;
        const bool active = c0 + CW * cg < K;    // warp-uniform
        double acc[RJ][CW];
#pragma unroll
        for (int i = 0; i < RJ; i++)
#pragma unroll
            for (int u = 0; u < CW; u++) acc[i][u] = 0.0;
        for (int32_t ti = t0; ti < t1; ti++) {
            const int32_t t = idx[ti];
            const Tile tl = tiles[t];
            const double* src = rtiles + (size_t)t * TA * TB;
            // records of the summed side of this tile
            const int64_t s0 = BY_RIGHT ? (int64_t)tl.a_blk * TA : (int64_t)tl.b_blk * TB;
            for (int js = 0; js < NS; js += JS) {
                __syncthreads();  // the previous step's stages are no longer read
                if (BY_RIGHT) {
                    // r2u rows k of the step, all TB columns
#pragma unroll 4
                    for (int q = tid; q < JS * TB / 2; q += NT) {
                        const double2 v = __ldg(reinterpret_cast<const double2*>(src + (size_t)js * TB) + q);
                        const int e = q * 2, r = e / TB, cc = e % TB;
                        Rs[r * RLD + cc] = v.x;
                        Rs[r * RLD + cc + 1] = v.y;
                    }
                } else {
                    // all TA rows, columns js .. js + JS of the step
#pragma unroll 4
                    for (int q = tid; q < TA * JS / 2; q += NT) {
                        const int e = q * 2, r = e / JS, cc = e % JS;
                        const double2 v = __ldg(reinterpret_cast<const double2*>(src + (size_t)r * TB + js + cc));
                        Rs[r * RLD + cc] = v.x;
                        Rs[r * RLD + cc + 1] = v.y;
                    }
                }
                // annotation column c of record s0 + js + r at aeff[s0 + js + r + c * m]: consecutive r are coalesced
#pragma unroll 4
                for (int q = tid; q < JS * CC; q += NT) {
                    const int r = q % JS, c = q / JS;
                    const int64_t srow = s0 + js + r;
                    As[r * ALD + c] = (srow < m && c0 + c < K) ? __ldg(ep.aeff + srow + (int64_t)(c0 + c) * m) : 0.0;
                }
                __syncthreads();
                if (!active) continue;
#pragma unroll 2
                for (int sidx = 0; sidx < JS; sidx++) {
                    double a[CW];
#pragma unroll
                    for (int u = 0; u < CW; u += 2) {
                        const double2 v = *reinterpret_cast<const double2*>(As + sidx * ALD + CW * cg + u);
                        a[u] = v.x;
                        a[u + 1] = v.y;
                    }
#pragma unroll
                    for (int i = 0; i < RJ; i++) {
                        const double r = BY_RIGHT ? Rs[sidx * RLD + og + 32 * i] : Rs[(og + 32 * i) * RLD + sidx];
#pragma unroll
                        for (int u = 0; u < CW; u++) acc[i][u] = fma(r, a[u], acc[i][u]);
                    }
                }
            }
        }
        if (!active) continue;
#pragma unroll
        for (int i = 0; i < RJ; i++) {
            const int64_t row = (int64_t)blk * OB + og + 32 * i;
            if (row >= m) continue;
#pragma unroll
            for (int u = 0; u < CW; u++) {
                const int c = c0 + CW * cg + u;
                if (c < K) ep.l2[row + (int64_t)c * m] += acc[i][u];
            }
        }
    }
}

// K = 1: one thread per record, the record's column sums over the tiles of its
// right block, then its row sums over the tiles of its left block, in list
// order (coalesced: consecutive records read consecutive partials of a tile).
__global__ void __launch_bounds__(NT) k_l2_reduce(int64_t m, int ta, int tb, const int32_t* __restrict__ ptr_r,
                                                  const int32_t* __restrict__ idx_r, const int32_t* __restrict__ ptr_l,
                                                  const int32_t* __restrict__ idx_l, const double* __restrict__ prow,
                                                  const double* __restrict__ pcol, double* __restrict__ l2) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    double acc = l2[j];
    const int64_t rb = j / tb, lb = j / ta;
    for (int32_t i = ptr_r[rb]; i < ptr_r[rb + 1]; i++) acc += pcol[(size_t)idx_r[i] * tb + (j - rb * tb)];
    for (int32_t i = ptr_l[lb]; i < ptr_l[lb + 1]; i++) acc += prow[(size_t)idx_l[i] * ta + (j - lb * ta)];
    l2[j] = acc;
}

}  // namespace

cudaError_t launch_l2_reduce(int64_t m, int ta, int tb, const int32_t* ptr_r, const int32_t* idx_r,
                             const int32_t* ptr_l, const int32_t* idx_l, const double* prow, const double* pcol,
                             double* l2, cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    k_l2_reduce<<<(unsigned)((m + NT - 1) / NT), NT, 0, stream>>>(m, ta, tb, ptr_r, idx_r, ptr_l, idx_l, prow, pcol,
                                                                  l2);
    return cudaGetLastError();
}

cudaError_t launch_contract(const double* rtiles, int ta, int tb, const Tile* tiles, const int32_t* ptr,
                            const int32_t* idx, int32_t nblocks, bool by_right, const EpilogueArgs& ep,
                            cudaStream_t stream) {
    if (nblocks <= 0) return cudaSuccess;
    const int nchunks = (ep.K + CC - 1) / CC;
    const int64_t work = (int64_t)nblocks * nchunks;
    const unsigned grid = (unsigned)(work < 148 * 8 ? work : 148 * 8);
    auto go = [&](auto kern, size_t smem) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, NT, smem, stream>>>(rtiles, tiles, ptr, idx, nblocks, ep);
        return cudaGetLastError();
    };
    if (ta == 64 && tb == 128)
        return by_right ? go(k_contract<64, 128, true>, ContractShape<64, 128, true>::smem)
                        : go(k_contract<64, 128, false>, ContractShape<64, 128, false>::smem);
    if (ta == 128 && tb == 128)
        return by_right ? go(k_contract<128, 128, true>, ContractShape<128, 128, true>::smem)
                        : go(k_contract<128, 128, false>, ContractShape<128, 128, false>::smem);
    return cudaErrorInvalidValue;
}

cudaError_t preload_contract() {
    cudaError_t e = preload_kernel(k_contract<64, 128, true>);
    if (e == cudaSuccess) e = preload_kernel(k_contract<64, 128, false>);
    if (e == cudaSuccess) e = preload_kernel(k_contract<128, 128, true>);
    if (e == cudaSuccess) e = preload_kernel(k_contract<128, 128, false>);
    if (e == cudaSuccess) e = preload_kernel(k_l2_reduce);
    return e;
}

}  // namespace ldsc
