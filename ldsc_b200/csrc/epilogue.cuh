// epilogue.cuh -- l2 accumulation shared by the band-Gram kernels.
//
// A tile holds unbiased r^2 values R[k][j] for left records k (rows) and
// right records j (columns); pairs outside the band are exactly 0.  With one
// annotation column (K = 1) the Gram epilogues accumulate l2 directly; with
// K > 1 they store R and contract.cu does the products.
#pragma once
#include <cstdint>

#include "engine.h"

namespace ldsc {

// Pair (k, j) contributes iff left[j] <= k < j < m.
__device__ __forceinline__ bool pair_in_band(int64_t k, int64_t j, int64_t m,
                                             const int64_t* __restrict__ left) {
    return j < m && k < j && __ldg(left + j) <= k;
}

}  // namespace ldsc
