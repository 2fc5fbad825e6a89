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
#include "sm100.cuh"

namespace ldsc {

namespace {

constexpr int NT = 256;  // threads of k_l2_reduce

// The contraction on the FP64 tensor path (mma.sync m8n8k4 .f64):
//   BY_RIGHT: out rows j of the right block, out[j][c] += sum_k R[k][j] A[k][c]
//   BY_LEFT:  out rows k of the left block,  out[k][c] += sum_j R[k][j] A[j][c]
// One CTA owns one output block and up to MK = 128 annotation columns (K > 128
// runs column chunks).  The summed records of every tile of the block go by in
// steps of JS_M = 32; a step's r2u values and the annotation values of its 32
// records are staged by cp.async into one of two buffers while the MMAs run
// on the other.  Warp (rg, cg) owns output rows 32 rg .. 32 rg + 31 and
// columns 32 cg .. 32 cg + 31 of the chunk: 4 x 4 fragments of 8 x 8 f64
// accumulators, eight k-steps of four records per staged step.  Fragment
// layouts of m8n8k4 (row.col): A element (lane / 4, lane % 4), B element
// (lane % 4, lane / 4), D elements (lane / 4, 2 (lane % 4) + {0, 1}).  Shared
// rows are padded to a stride of 4 mod 16 doubles, so each half-warp's 16
// 8-byte fragment loads hit 16 distinct bank pairs.
constexpr int MK = 128;        // annotation columns per chunk
constexpr int JS_M = 32;       // summed records per staged step
constexpr int SLD = JS_M + 4;  // staged annotation stride (annotations are [column][record])

template <int TA, int TB, bool BY_RIGHT>
struct MmaShape {
    static constexpr int OB = BY_RIGHT ? TB : TA;          // output rows per block
    static constexpr int NS = BY_RIGHT ? TA : TB;          // summed records per tile
    static constexpr int SPT = NS / JS_M;                  // staged steps per tile
    static constexpr int WARPS = (OB / 32) * (MK / 32);
    static constexpr int THREADS = 32 * WARPS;
    // r2u stage: BY_RIGHT [JS_M k][TB j], BY_LEFT [TA k][JS_M j]
    static constexpr int RLD = BY_RIGHT ? TB + 4 : JS_M + 4;
    static constexpr int RROWS = BY_RIGHT ? JS_M : TA;
    static constexpr int R_ELEMS = RROWS * RLD;
    static constexpr int A_ELEMS = MK * SLD;
    static constexpr int STAGE = R_ELEMS + A_ELEMS;          // doubles per buffer
    static constexpr size_t smem = sizeof(double) * 2 * (size_t)STAGE;
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// 8 bytes, or zeros (nothing read) when !valid
__device__ __forceinline__ void cp_async8_zfill(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int TA, int TB, bool BY_RIGHT>
__global__ void __launch_bounds__(MmaShape<TA, TB, BY_RIGHT>::THREADS)
    k_contract_mma(const double* __restrict__ rtiles, const Tile* __restrict__ tiles,
                   const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int32_t nblocks,
                   EpilogueArgs ep) {
    using S = MmaShape<TA, TB, BY_RIGHT>;
    constexpr int NTH = S::THREADS, SPT = S::SPT, RLD = S::RLD, OB = S::OB;
    extern __shared__ __align__(16) double smm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rg = warp / (MK / 32), cg = warp % (MK / 32);
    const int K = ep.K;
    const int64_t m = ep.m;
    const int nchunks = (K + MK - 1) / MK;
    const int fr = lane >> 2, fc = lane & 3;   // fragment row / column of this lane

    for (int64_t w = blockIdx.x; w < (int64_t)nblocks * nchunks; w += gridDim.x) {
        const int32_t blk = (int32_t)(w / nchunks);
        const int c0 = (int)(w % nchunks) * MK;
        const int32_t t0 = ptr[blk], t1 = ptr[blk + 1];
        const int nsteps = (t1 - t0) * SPT;
        if (nsteps == 0) continue;
        const bool active = c0 + 32 * cg < K;  // warp-uniform: any of this warp's columns in range

        // stage step st into buffer b
        auto issue = [&](int st, int b) {
            const int32_t t = idx[t0 + st / SPT];
            const int js = (st % SPT) * JS_M;
            const Tile tl = tiles[t];
            const double* src = rtiles + (size_t)t * TA * TB;
            double* Rs = smm + b * S::STAGE;
            double* As = Rs + S::R_ELEMS;
            if (BY_RIGHT) {
                // rows k = js .. js + 31 of the tile, all TB values: 16-byte pieces
#pragma unroll
                for (int q = tid; q < JS_M * TB / 2; q += NTH) {
                    const int r = q / (TB / 2), cc = 2 * (q % (TB / 2));
                    cp_async16(Rs + r * RLD + cc, src + (size_t)(js + r) * TB + cc);
                }
            } else {
                // all TA rows, values js .. js + 31
#pragma unroll
                for (int q = tid; q < TA * JS_M / 2; q += NTH) {
                    const int r = q / (JS_M / 2), cc = 2 * (q % (JS_M / 2));
                    cp_async16(Rs + r * RLD + cc, src + (size_t)r * TB + js + cc);
                }
            }
            // annotation column c0 + c of summed record s at aeff[s + (c0 + c) m]; consecutive threads
            // take consecutive records (coalesced), zeros past m or K
            const int64_t s0 = (BY_RIGHT ? (int64_t)tl.a_blk * TA : (int64_t)tl.b_blk * TB) + js;
#pragma unroll
            for (int e = tid; e < MK * JS_M; e += NTH) {
                const int s = e & (JS_M - 1), c = e / JS_M;
                const bool ok = s0 + s < m && c0 + c < K;
                cp_async8_zfill(As + c * SLD + s, ok ? ep.aeff + (s0 + s) + (int64_t)(c0 + c) * m : ep.aeff, ok);
            }
        };

        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

        issue(0, 0);
        cp_async_commit();
        for (int st = 0; st < nsteps; st++) {
            if (st + 1 < nsteps) issue(st + 1, (st + 1) & 1);
            cp_async_commit();
            cp_async_wait1();  // step st's copies (this thread's) have landed
            __syncthreads();   // ... and every thread's
            if (active) {
                const double* Rs = smm + (st & 1) * S::STAGE;
                const double* As = Rs + S::R_ELEMS;
#pragma unroll
                for (int kk = 0; kk < JS_M; kk += 4) {
                    double a[4], b[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int orow = 32 * rg + 8 * i + fr;  // output row of the fragment
                        a[i] = BY_RIGHT ? Rs[(kk + fc) * RLD + orow] : Rs[orow * RLD + kk + fc];
                    }
#pragma unroll
                    for (int j = 0; j < 4; j++) b[j] = As[(32 * cg + 8 * j + fr) * SLD + kk + fc];
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
                }
            }
            __syncthreads();  // buffer st & 1 is refilled by the next iteration's issue
        }
        if (!active) continue;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int64_t row = (int64_t)blk * OB + 32 * rg + 8 * i + fr;
            if (row >= m) continue;
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int c = c0 + 32 * cg + 8 * j + 2 * fc + h;
                    if (c < K) ep.l2[row + (int64_t)c * m] += acc[i][j][h];
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
    const int64_t work = (int64_t)nblocks * ((ep.K + MK - 1) / MK);
    auto go = [&](auto kern, size_t smem, int threads) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        // 512-thread CTAs (141 - 147 KB): one per SM; 256-thread CTAs (111 KB): two
        const int64_t cap = (int64_t)148 * (threads <= 256 ? 2 : 1);
        kern<<<(unsigned)(work < cap ? work : cap), threads, smem, stream>>>(rtiles, tiles, ptr, idx, nblocks, ep);
        return cudaGetLastError();
    };
#define LDSC_CONTRACT(TA_, TB_, BR_) \
    go(k_contract_mma<TA_, TB_, BR_>, MmaShape<TA_, TB_, BR_>::smem, MmaShape<TA_, TB_, BR_>::THREADS)
    if (ta == 64 && tb == 128) return by_right ? LDSC_CONTRACT(64, 128, true) : LDSC_CONTRACT(64, 128, false);
    if (ta == 128 && tb == 128) return by_right ? LDSC_CONTRACT(128, 128, true) : LDSC_CONTRACT(128, 128, false);
#undef LDSC_CONTRACT
    return cudaErrorInvalidValue;
}

cudaError_t preload_contract() {
    cudaError_t e = preload_kernel(k_contract_mma<64, 128, true>);
    if (e == cudaSuccess) e = preload_kernel(k_contract_mma<64, 128, false>);
    if (e == cudaSuccess) e = preload_kernel(k_contract_mma<128, 128, true>);
    if (e == cudaSuccess) e = preload_kernel(k_contract_mma<128, 128, false>);
    if (e == cudaSuccess) e = preload_kernel(k_l2_reduce);
    return e;
}

}  // namespace ldsc
