// decode.cu -- PLINK BED decode kernels (HBM-bound).
//
// One warp per SNP record.  Each lane takes 16 individuals at a time as one
// 32-bit word of 2-bit codes (count-A1 LUT [2, missing, 1, 0], reference
// src/bed.rs:470-521) and turns it into per-slot bit masks:
//     lo = bit 0 of each code, hi = bit 1
//     present = !lo | hi            (code != 01)
//     g == 2  <=> code 00 = !lo & !hi
//     g == 1  <=> code 10 = !lo &  hi
// so the per-SNP integer moments (src/l2/compute.rs:334-512) are popcounts
// and the INT8 operand rows are a bit spread of the same masks.
#include <cuda_runtime.h>

#include "engine.h"

namespace ldsc {

namespace {

constexpr uint32_t kEven = 0x55555555u;

// Code word of individuals [i0, i0 + 16); slots past sel.n read as missing.
__device__ __forceinline__ uint32_t codes16(const uint8_t* __restrict__ row, IndivSel sel,
                                            uint64_t i0) {
    if (i0 >= sel.n) return 0x55555555u;  // all missing: padding columns
    uint32_t w;
    if (sel.keep == nullptr) {
        // i0 is a multiple of 16, rows are 16-byte aligned and padded to a
        // multiple of 16 bytes, so the word load stays inside the row pitch.
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
        uint32_t valid = sel.n > i0 ? static_cast<uint32_t>(sel.n - i0) : 0u;
        uint32_t keepm = valid >= 16 ? 0xFFFFFFFFu : ((1u << (2 * valid)) - 1u);
        w = (w & keepm) | (0x55555555u & ~keepm);
    }
    return w;
}

// bits 0,2,4,6 of x -> bit 0 of bytes 0..3
__device__ __forceinline__ uint32_t spread4(uint32_t x) {
    return (x & 1u) | ((x & 4u) << 6) | ((x & 16u) << 12) | ((x & 64u) << 18);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Expand one 16-individual code word into genotype and mask bytes and
// accumulate the moment counts.
__device__ __forceinline__ void expand16(uint32_t w, uint8_t* grow, uint8_t* mrow, uint64_t i0, uint32_t& cn,
                                         uint32_t& c1, uint32_t& c2) {
    const uint32_t lo = w & kEven;
    const uint32_t hi = (w >> 1) & kEven;
    const uint32_t pres = (~lo | hi) & kEven;
    const uint32_t two = ~lo & ~hi & kEven;
    const uint32_t one = ~lo & hi & kEven;
    cn += __popc(pres);
    c1 += __popc(one);
    c2 += __popc(two);
    if (grow) {
        uint4 g, mk;
        g.x = spread4(one) + 2u * spread4(two);
        g.y = spread4(one >> 8) + 2u * spread4(two >> 8);
        g.z = spread4(one >> 16) + 2u * spread4(two >> 16);
        g.w = spread4(one >> 24) + 2u * spread4(two >> 24);
        mk.x = spread4(pres);
        mk.y = spread4(pres >> 8);
        mk.z = spread4(pres >> 16);
        mk.w = spread4(pres >> 24);
        // a warp stores 512 contiguous bytes; streaming stores: the operand
        // rows are re-read by the Gram from HBM, not from L2
        __stcs(reinterpret_cast<uint4*>(grow + i0), g);
        __stcs(reinterpret_cast<uint4*>(mrow + i0), mk);
    }
}

// A warp decodes 2,048 individuals per step: lane l takes words l, l+32,
// l+64, l+96 of the step (loads issued together, stores coalesced).
__global__ void __launch_bounds__(256) k_decode_i8(PanelView p, const uint64_t* __restrict__ rec_rows,
                                                   int64_t m, IndivSel sel, uint8_t* __restrict__ ops,
                                                   uint64_t ld, RecStats st, int want_moments) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t span = ops ? ld : ((sel.n + 15) & ~uint64_t(15));
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < m; r += warps) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint8_t* row = p.rows + brow * p.pitch;
        uint32_t cn = 0, c1 = 0, c2 = 0;
        uint8_t* grow = ops ? ops + (uint64_t)(2 * r) * ld : nullptr;
        uint8_t* mrow = ops ? grow + ld : nullptr;
        for (uint64_t s0 = 0; s0 < span; s0 += 2048) {
            uint32_t w[4];
#pragma unroll
            for (int u = 0; u < 4; u++) w[u] = codes16(row, sel, s0 + 512 * u + 16 * lane);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint64_t i0 = s0 + 512 * u + 16 * lane;
                if (i0 < span) expand16(w[u], grow, mrow, i0, cn, c1, c2);
            }
        }
        const uint32_t cs = c1 + 2 * c2, cq = c1 + 4 * c2, c3 = c1 + 8 * c2, c4 = c1 + 16 * c2;
        const uint32_t tn = warp_sum(cn), ts = warp_sum(cs), tq = warp_sum(cq);
        const uint32_t t3 = want_moments ? warp_sum(c3) : 0u, t4 = want_moments ? warp_sum(c4) : 0u;
        if (lane == 0) {
            st.n[r] = (int32_t)tn;
            st.s[r] = (int32_t)ts;
            st.q[r] = (int32_t)tq;
            if (want_moments && st.q3) {
                st.q3[r] = (int32_t)t3;
                st.q4[r] = (int32_t)t4;
            }
        }
    }
}

// Per-record finalisation (src/l2/normalize.rs:71-110 for mean / inv_std /
// MAF; per_snp_kappa src/l2/compute.rs:525-538; pq scaling
// src/l2/compute.rs:1406-1412,1595-1603).  Also seeds l2 with the diagonal
// term r2u_jj * a_j = a_j.
__global__ void k_finalize(int64_t m, uint64_t n_indiv, RecStats st, const double* __restrict__ annot,
                           uint64_t annot_ld, int32_t K, int has_pq, double pq_exp, double* __restrict__ aeff,
                           double* __restrict__ l2_init) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const int64_t n = st.n[r], s = st.s[r], q = st.q[r];
    const double N = (double)n_indiv;
    const double mean = n > 0 ? (double)s / (double)n : 0.0;
    double freq = mean / 2.0;
    freq = freq < 0.0 ? 0.0 : (freq > 1.0 ? 1.0 : freq);
    const double maf = freq < 1.0 - freq ? freq : 1.0 - freq;
    const double css = (double)q - (double)n * mean * mean;
    const double var = css / N;
    const double sd = sqrt(var);
    const double inv = sd > 0.0 ? 1.0 / sd : 0.0;
    const int64_t V = n * q - s * s;  // n * css, exact
    const double qinv = (inv > 0.0 && V > 0) ? 1.0 / sqrt((double)n * (double)V) : 0.0;
    st.maf[r] = maf;
    st.mean[r] = mean;
    st.inv_std[r] = inv;
    st.qinv[r] = qinv;
    double pq = 1.0;
    if (has_pq) {
        pq = pow(maf * (1.0 - maf), pq_exp);
        if (st.pq) st.pq[r] = pq;
    }
    if (st.kappa) {
        double kap = 0.0;
        if (st.q3 && n > 0) {
            const double cf = (double)n;
            const double mu = (double)s / cf;
            const double m4 = (double)st.q4[r] - 4.0 * mu * (double)st.q3[r] +
                              6.0 * mu * mu * (double)q - 3.0 * mu * mu * mu * mu * cf;
            const double c2 = (double)q - cf * mu * mu;
            kap = c2 > 0.0 ? m4 / (c2 * c2) : 0.0;
        }
        st.kappa[r] = kap;
    }
    for (int32_t c = 0; c < K; c++) {
        double a = annot ? annot[r + c * annot_ld] : 1.0;
        a *= pq;
        aeff[r + (int64_t)c * m] = a;
        l2_init[r + (int64_t)c * m] = a;
    }
}

// Standardised f64 columns (normalize_col_f64_with_stats,
// src/l2/normalize.rs:71-110): x = (g - mean) * inv_std, missing -> 0.
__global__ void __launch_bounds__(256) k_decode_f64(PanelView p, const uint64_t* __restrict__ rec_rows,
                                                    int64_t m, IndivSel sel, RecStats st,
                                                    double* __restrict__ x, uint64_t ld) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < m; r += warps) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint8_t* row = p.rows + brow * p.pitch;
        const double mean = st.mean[r];
        const double inv = st.inv_std[r];
        const double v2 = (2.0 - mean) * inv, v1 = (1.0 - mean) * inv, v0 = (0.0 - mean) * inv;
        double* xr = x + (uint64_t)r * ld;
        for (uint64_t i0 = (uint64_t)lane * 16; i0 < ld; i0 += 512) {
            const uint32_t w = codes16(row, sel, i0);
            double v[16];
#pragma unroll
            for (int t = 0; t < 16; t++) {
                const uint32_t c = (w >> (2 * t)) & 3u;
                v[t] = c == 0 ? v2 : (c == 2 ? v1 : (c == 3 ? v0 : 0.0));
            }
#pragma unroll
            for (int t = 0; t < 16; t += 2) {
                *reinterpret_cast<double2*>(xr + i0 + t) = make_double2(v[t], v[t + 1]);
            }
        }
    }
}

// One thread per 4-byte word of the pitched rows; the source is the file's
// unpadded rows, read byte-wise (their starts are not word aligned).
__global__ void __launch_bounds__(256) k_repitch(const uint8_t* __restrict__ src, uint64_t bpr,
                                                 uint8_t* __restrict__ dst, uint64_t pitch, uint64_t r0,
                                                 uint64_t r1) {
    const uint64_t wpr = pitch >> 2;
    const uint64_t total = (r1 - r0) * wpr;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint64_t r = r0 + t / wpr;
        const uint64_t x = (t % wpr) * 4;
        const uint8_t* srow = src + r * bpr;
        uint32_t w = 0;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if (x + b < bpr) w |= (uint32_t)__ldg(srow + x + b) << (8 * b);
        *reinterpret_cast<uint32_t*>(dst + r * pitch + x) = w;
    }
}

int decode_grid(int64_t m) {
    int64_t blocks = (m + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    return (int)blocks;
}

}  // namespace

cudaError_t launch_decode_i8(const PanelView& p, const uint64_t* rec_rows, int64_t m, IndivSel sel,
                             uint8_t* ops, uint64_t ld, RecStats st, int want_moments,
                             cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    k_decode_i8<<<decode_grid(m), 256, 0, stream>>>(p, rec_rows, m, sel, ops, ld, st, want_moments);
    return cudaGetLastError();
}

cudaError_t launch_repitch(const uint8_t* src, uint64_t bpr, uint8_t* dst, uint64_t pitch, uint64_t r0,
                           uint64_t r1, cudaStream_t stream) {
    if (r1 <= r0) return cudaSuccess;
    const uint64_t words = (r1 - r0) * (pitch >> 2);
    uint64_t blocks = (words + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_repitch<<<(unsigned)blocks, 256, 0, stream>>>(src, bpr, dst, pitch, r0, r1);
    return cudaGetLastError();
}

cudaError_t launch_finalize_stats(int64_t m, uint64_t n_indiv, RecStats st, const double* annot,
                                  int32_t K, int has_pq, double pq_exp, double* aeff,
                                  double* l2_init, cudaStream_t stream, uint64_t annot_ld) {
    if (m <= 0) return cudaSuccess;
    k_finalize<<<(unsigned)((m + 255) / 256), 256, 0, stream>>>(m, n_indiv, st, annot,
                                                              annot_ld ? annot_ld : (uint64_t)m, K, has_pq,
                                                              pq_exp, aeff, l2_init);
    return cudaGetLastError();
}

cudaError_t launch_decode_f64(const PanelView& p, const uint64_t* rec_rows, int64_t m, IndivSel sel,
                              RecStats st, double* x, uint64_t ld, cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    k_decode_f64<<<decode_grid(m), 256, 0, stream>>>(p, rec_rows, m, sel, st, x, ld);
    return cudaGetLastError();
}

cudaError_t preload_decode() {
    cudaError_t e = preload_kernel(k_decode_i8);
    if (e == cudaSuccess) e = preload_kernel(k_finalize);
    if (e == cudaSuccess) e = preload_kernel(k_decode_f64);
    if (e == cudaSuccess) e = preload_kernel(k_repitch);
    return e;
}

}  // namespace ldsc
