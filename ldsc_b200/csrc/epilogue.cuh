// epilogue.cuh -- l2 accumulation shared by the band-Gram kernels.
//
// A tile holds unbiased r^2 values R[k][j] for left records k (rows) and
// right records j (columns); pairs outside the band are exactly 0.  The
// reference contracts R with the annotation matrix in both directions
// (src/l2/compute.rs:1869-1893, 2259-2314):
//     l2[k, C] += sum_j R[k][j] * a[j, C]      (the window side)
//     l2[j, C] += sum_k R[k][j] * a[k, C]      (the chunk side)
#pragma once
#include <cstdint>

#include "engine.h"

namespace ldsc {

// Pair (k, j) contributes iff left[j] <= k < j < m.
__device__ __forceinline__ bool pair_in_band(int64_t k, int64_t j, int64_t m,
                                             const int64_t* __restrict__ left) {
    return j < m && k < j && __ldg(left + j) <= k;
}

// K > 1 contraction of an f32 R tile staged in shared memory (row stride ldr).
__device__ inline void contract_tile_smem(const float* __restrict__ Rs, int ldr, int ta, int tb,
                                          int64_t k0, int64_t j0, const EpilogueArgs& ep, int tid,
                                          int nthreads) {
    const int K = ep.K;
    const int64_t m = ep.m;
    for (int idx = tid; idx < ta * K; idx += nthreads) {
        const int k = idx % ta, C = idx / ta;
        if (k0 + k >= m) continue;
        float acc = 0.f;
        const float* rrow = Rs + k * ldr;
        const int jmax = (int)((m - j0) < tb ? (m - j0) : tb);
        for (int j = 0; j < jmax; j++) acc += rrow[j] * __ldg(ep.aeff32 + (j0 + j) * K + C);
        if (acc != 0.f) atomicAdd(ep.l2 + (k0 + k) + (int64_t)C * m, (double)acc);
    }
    for (int idx = tid; idx < tb * K; idx += nthreads) {
        const int j = idx % tb, C = idx / tb;
        if (j0 + j >= m) continue;
        float acc = 0.f;
        const int kmax = (int)((m - k0) < ta ? (m - k0) : ta);
        for (int k = 0; k < kmax; k++) acc += Rs[k * ldr + j] * __ldg(ep.aeff32 + (k0 + k) * K + C);
        if (acc != 0.f) atomicAdd(ep.l2 + (j0 + j) + (int64_t)C * m, (double)acc);
    }
}

}  // namespace ldsc
