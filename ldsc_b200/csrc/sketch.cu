// sketch.cu -- fused BED decode -> standardise -> CountSketch scatter -> ratio
// renormalisation, one CTA per SNP record.
//
// Reference (src/wasm_simd.rs:1617-1784 via src/l2/compute.rs:601-770): for
// each individual i, out[bucket[i]] += sign[i] * (g_i - mean) * inv_std
// (missing -> 0) in f32, then out *= sqrt(N / sum(out^2)) with the squared
// norm accumulated in f64.
//
// Here the bucket sums are formed exactly in integers and the affine
// standardisation is applied once per bucket:
//     sum_{i in b} sign_i (g_i - mean) inv_std = inv_std * (S1_b - mean * S0_b)
//     S0_b = sum_{i in b, present} sign_i = T_b - Y_b,  Y_b = sum_{i in b, missing} sign_i
//     S1_b = sum_{i in b, present} sign_i g_i
// T_b (all individuals' signs per bucket) is precomputed once per sketch.  When
// the A1 allele is the major one, S1_b = 2 S0_b - sum sign_i (2 - g_i), whose
// terms are non-zero less often.  The only shared-memory atomics left are for
// non-zero terms and missing genotypes.  mean / inv_std are the reference's
// f32-rounded values; the bucket value is rounded to f32 once.
#include <cuda_runtime.h>

#include "engine.h"

namespace ldsc {

namespace {

__device__ __forceinline__ uint32_t codes16(const uint8_t* __restrict__ row, IndivSel sel,
                                            uint64_t i0) {
    if (i0 >= sel.n) return 0x55555555u;
    uint32_t w;
    if (sel.keep == nullptr) {
        w = __ldg(reinterpret_cast<const uint32_t*>(row + (i0 >> 2)));
    } else {
        w = 0;
#pragma unroll
        for (int t = 0; t < 16; t++) {
            uint64_t i = i0 + t;
            uint32_t code = 1u;
            if (i < sel.n) {
                int64_t iid = __ldg(sel.keep + i);
                code = (__ldg(row + (iid >> 2)) >> ((iid & 3) * 2)) & 3u;
            }
            w |= code << (2 * t);
        }
    }
    if (i0 + 16 > sel.n) {
        uint32_t valid = static_cast<uint32_t>(sel.n - i0);
        uint32_t keepm = valid >= 16 ? 0xFFFFFFFFu : ((1u << (2 * valid)) - 1u);
        w = (w & keepm) | (0x55555555u & ~keepm);
    }
    return w;
}

constexpr int NT = 256;

__global__ void __launch_bounds__(NT) k_sketch(PanelView p, const uint64_t* __restrict__ rec_rows,
                                               int64_t m, IndivSel sel,
                                               const uint32_t* __restrict__ packed,
                                               const int32_t* __restrict__ tsum, uint32_t d,
                                               RecStats st, float* __restrict__ out, uint64_t ld) {
    extern __shared__ int32_t sh[];
    int32_t* Z = sh;
    int32_t* Y = sh + d;
    __shared__ double red[NT / 32];
    const double nn = (double)sel.n;
    for (int64_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint8_t* row = p.rows + brow * p.pitch;
        const float mean32 = (float)st.mean[r];
        const float inv32 = (float)st.inv_std[r];
        const bool comp = st.mean[r] > 1.0;
        for (uint32_t b = threadIdx.x; b < 2 * d; b += NT) sh[b] = 0;
        __syncthreads();
        for (uint64_t i0 = (uint64_t)threadIdx.x * 16; i0 < sel.n; i0 += (uint64_t)NT * 16) {
            const uint32_t w = codes16(row, sel, i0);
            const uint4* pk4 = reinterpret_cast<const uint4*>(packed + i0);
            uint32_t pk[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                // packed has at least round_up(n, 16) entries (padding: bucket 0, sign +)
                const uint4 v = __ldg(pk4 + q);
                pk[4 * q] = v.x; pk[4 * q + 1] = v.y; pk[4 * q + 2] = v.z; pk[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int t = 0; t < 16; t++) {
                const uint32_t code = (w >> (2 * t)) & 3u;
                const uint32_t b = pk[t] & 0x7FFFFFFFu;
                const int32_t sg = (pk[t] >> 31) ? -1 : 1;
                if (code == 1u) {
                    if (i0 + t < sel.n) atomicAdd(&Y[b], sg);
                } else {
                    const int32_t g = code == 0u ? 2 : (code == 2u ? 1 : 0);
                    const int32_t h = comp ? 2 - g : g;
                    if (h) atomicAdd(&Z[b], sg * h);
                }
            }
        }
        __syncthreads();
        double part = 0.0;
        float* orow = out + (uint64_t)r * ld;
        for (uint32_t b = threadIdx.x; b < d; b += NT) {
            const int64_t s0 = (int64_t)__ldg(tsum + b) - Y[b];
            const int64_t s1 = comp ? 2 * s0 - Z[b] : Z[b];
            const float o = (float)((double)inv32 * ((double)s1 - (double)mean32 * (double)s0));
            orow[b] = o;
            part += (double)o * (double)o;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        double nrm = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < NT / 32; w2++) nrm += red[w2];
        if (nrm > 0.0) {
            const float scale = (float)sqrt(nn / nrm);
            for (uint32_t b = threadIdx.x; b < d; b += NT) orow[b] *= scale;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_sketch_scatter(const PanelView& p, const uint64_t* rec_rows, int64_t m,
                                  IndivSel sel, const uint32_t* packed, const int32_t* tsum,
                                  uint32_t d, RecStats st, float* out, uint64_t ld,
                                  cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    const size_t smem = sizeof(int32_t) * 2 * (size_t)d;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_sketch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    int64_t grid = m < 148 * 8 ? m : 148 * 8;
    k_sketch<<<(unsigned)grid, NT, smem, stream>>>(p, rec_rows, m, sel, packed, tsum, d, st, out, ld);
    return cudaGetLastError();
}

}  // namespace ldsc
