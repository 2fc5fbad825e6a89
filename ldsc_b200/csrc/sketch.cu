// sketch.cu -- CountSketch projection of BED rows (HBM-bound).
//
// Reference (src/wasm_simd.rs:1617-1784 via src/l2/compute.rs:601-770): per
// SNP, out[bucket[i]] += sign[i] * (g_i - mean) * inv_std over individuals i
// (missing -> 0), in f32, then out *= sqrt(N / sum(out^2)) with the squared
// norm accumulated in f64.
//
// Linearity gives, per bucket b,
//     out_b = inv_std * (S1_b - mean * S0_b)
//     S1_b  = sum_{i in b, present} sign_i g_i,   S0_b = sum_{i in b, present} sign_i,
// two integer sums.  The bucket/sign map is the same for every SNP, so the
// individuals are put once into bucket-major order (bucket, then sign):
// k_sketch_permute rewrites every panel row in that order (2-bit codes, 16 per
// word), after which each (bucket, sign) group is a contiguous run of
// positions.  k_sketch_seg then streams a permuted row once and forms the
// bucket sums with popcounts on 32-bit words (16 genotypes at a time); the
// same popcounts give the per-SNP moments.
//
// mean / inv_std are the reference's f32-rounded values; each bucket value is
// formed exactly and rounded to f32 once (the reference accumulates f32 in
// individual order; the two agree to f32 rounding).  The per-SNP moments
// (n, s, q, and the 3rd/4th for the MAF-aware correction) are permutation
// invariant and are produced by the same pass.
#include <cuda_runtime.h>

#include "engine.h"
#include "sm100.cuh"

namespace ldsc {

namespace {

constexpr uint32_t kEven = 0x55555555u;
constexpr int NT = 256;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Rewrite panel rows in bucket-major individual order.  perm[p] = FAM index
// of the individual at permuted position p (p < n_used); positions past n_used
// read as missing.  One CTA per row, the row staged in shared memory when it
// fits (smem_row != 0).
__global__ void __launch_bounds__(NT) k_sketch_permute(PanelView p, const int32_t* __restrict__ perm,
                                                       uint64_t n_used, uint32_t* __restrict__ out,
                                                       uint64_t out_pitch_words, int smem_row) {
    extern __shared__ uint32_t srow32[];
    const uint8_t* srow = reinterpret_cast<const uint8_t*>(srow32);
    const uint64_t words = (n_used + 15) / 16;
    for (uint64_t r = blockIdx.x; r < p.n_snp; r += gridDim.x) {
        const uint8_t* row = p.rows + r * p.pitch;
        if (smem_row) {
            const uint4* src = reinterpret_cast<const uint4*>(row);
            uint4* dst = reinterpret_cast<uint4*>(srow32);
            for (uint64_t q = threadIdx.x; q < p.pitch / 16; q += NT) dst[q] = __ldg(src + q);
            __syncthreads();
        }
        const uint8_t* from = smem_row ? srow : row;
        uint32_t* orow = out + r * out_pitch_words;
        for (uint64_t w = threadIdx.x; w < out_pitch_words; w += NT) {
            uint32_t word = 0x55555555u;
            if (w < words) {
                word = 0;
#pragma unroll 4
                for (int t = 0; t < 16; t++) {
                    const uint64_t pos = w * 16 + t;
                    uint32_t code = 1u;
                    if (pos < n_used) {
                        const int32_t iid = __ldg(perm + pos);
                        code = (from[iid >> 2] >> ((iid & 3) * 2)) & 3u;
                    }
                    word |= code << (2 * t);
                }
            }
            orow[w] = word;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t span_mask(uint32_t a, uint32_t b) {  // even bits of positions [a, b)
    const uint32_t hi = b >= 16 ? 0xFFFFFFFFu : ((1u << (2 * b)) - 1u);
    const uint32_t lo = (1u << (2 * a)) - 1u;
    return hi & ~lo & kEven;
}

// One CTA per record, one pass over the permuted row: per-SNP moments and
// per-bucket sums S1 (sum sign * g) and S0 (sum sign * present), then the
// standardised, renormalised bucket values.  Each thread takes a contiguous
// range of words (loaded QB x 16 bytes at a time into registers); a bucket
// that lies wholly inside one thread's range is written with a plain store,
// only the two buckets at the ends of a range use shared-memory atomics.
// Output row r: `ld` floats (zero padded past d), or with split the hi/lo
// tensor-core rows 2r / 2r+1.
__global__ void __launch_bounds__(NT, 4) k_sketch_seg(const uint32_t* __restrict__ pp, uint64_t pp_pitch_words,
                                                   const uint64_t* __restrict__ rec_rows, int64_t m, uint64_t n_used,
                                                   const int32_t* __restrict__ seg_off,
                                                   const int32_t* __restrict__ word_seg, uint32_t d, RecStats st,
                                                   int want_moments, int split, float* __restrict__ out,
                                                   uint64_t ld) {
    extern __shared__ int32_t sh[];
    int32_t* Z = sh;       // S1 per bucket
    int32_t* P = sh + d;   // S0 per bucket
    __shared__ int64_t red[5][NT / 32];
    __shared__ double dred[NT / 32];
    __shared__ double s_mean, s_inv;
    const uint64_t words = (n_used + 15) / 16;
    const uint32_t nseg = 2 * d;
    const uint64_t quads = (words + 3) / 4;
    const uint64_t q0 = quads * threadIdx.x / NT, q1 = quads * (threadIdx.x + 1) / NT;
    for (int64_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint4* row = reinterpret_cast<const uint4*>(pp + brow * pp_pitch_words);
        for (uint32_t b = threadIdx.x; b < 2 * d; b += NT) sh[b] = 0;
        __syncthreads();
        // counts over the row: present, genotype 1, genotype 2 (sum g^k = #1 + 2^k #2)
        uint32_t cn = 0, c1 = 0, c2 = 0;
        if (q0 < q1) {
            uint32_t k = (uint32_t)__ldg(word_seg + q0 * 4);
            int32_t cut = __ldg(seg_off + k + 1);
            int32_t sg = (k & 1u) ? -1 : 1;
            const uint32_t first_b = k >> 1;
            uint32_t cur_b = first_b;
            uint32_t zr = 0, pr = 0;       // sums over the current run
            int32_t zacc = 0, pacc = 0;    // signed sums over the current bucket
            int32_t base = (int32_t)(q0 * 64);
            uint4 nxt = __ldg(row + q0);
            for (uint64_t q = q0; q < q1; q++) {
                const uint4 v = nxt;
                if (q + 1 < q1) nxt = __ldg(row + q + 1);
                const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int t = 0; t < 4; t++, base += 16) {
                    const uint32_t x = wv[t];
                    const uint32_t lo = x & kEven, hi = (x >> 1) & kEven;
                    const uint32_t one = hi & ~lo, two = ~(lo | hi) & kEven, pres = (~lo | hi) & kEven;
                    const uint32_t p1 = __popc(one), p2 = __popc(two), pn = __popc(pres);
                    cn += pn;
                    c1 += p1;
                    c2 += p2;
                    if (cut > base + 16) {  // the whole word lies in run k (or past the last run)
                        zr += p1 + 2 * p2;
                        pr += pn;
                        continue;
                    }
                    uint32_t a = 0;
                    while (true) {
                        const uint32_t b = cut < base + 16 ? (uint32_t)(cut - base) : 16u;
                        const uint32_t msk = span_mask(a, b);
                        zr += __popc(one & msk) + 2 * __popc(two & msk);
                        pr += __popc(pres & msk);
                        // run k ends at position base + b
                        zacc += sg * (int32_t)zr;
                        pacc += sg * (int32_t)pr;
                        zr = pr = 0;
                        k++;
                        if ((k >> 1) != cur_b || k >= nseg) {
                            if (cur_b == first_b) {
                                if (zacc) atomicAdd(&Z[cur_b], zacc);
                                if (pacc) atomicAdd(&P[cur_b], pacc);
                            } else {
                                Z[cur_b] = zacc;
                                P[cur_b] = pacc;
                            }
                            zacc = pacc = 0;
                            cur_b = k >> 1;
                        }
                        if (k >= nseg) {
                            cut = 0x7FFFFFFF;
                            break;
                        }
                        cut = __ldg(seg_off + k + 1);
                        sg = (k & 1u) ? -1 : 1;
                        a = b;
                        if (a >= 16) break;
                        if (cut > base + 16) {  // the new run covers the rest of the word
                            const uint32_t rest = span_mask(a, 16);
                            zr += __popc(one & rest) + 2 * __popc(two & rest);
                            pr += __popc(pres & rest);
                            break;
                        }
                    }
                }
            }
            if (k < nseg) {  // bucket continuing past this thread's range
                zacc += sg * (int32_t)zr;
                pacc += sg * (int32_t)pr;
                if (zacc) atomicAdd(&Z[cur_b], zacc);
                if (pacc) atomicAdd(&P[cur_b], pacc);
            }
        }
        const uint32_t cs = c1 + 2 * c2, cq = c1 + 4 * c2, c3 = c1 + 8 * c2, c4 = c1 + 16 * c2;
        int64_t mom[5] = {warp_sum(cn), warp_sum(cs), warp_sum(cq), warp_sum(c3), warp_sum(c4)};
        if ((threadIdx.x & 31) == 0)
            for (int i = 0; i < 5; i++) red[i][threadIdx.x >> 5] = mom[i];
        __syncthreads();
        if (threadIdx.x < 32) {
            int64_t t[5];
#pragma unroll
            for (int i = 0; i < 5; i++) t[i] = warp_sum(threadIdx.x < NT / 32 ? red[i][threadIdx.x] : (int64_t)0);
            if (threadIdx.x == 0) {
                const int64_t n = t[0], s = t[1], q = t[2];
                st.n[r] = (int32_t)n;
                st.s[r] = (int32_t)s;
                st.q[r] = (int32_t)q;
                if (want_moments && st.q3) {
                    st.q3[r] = (int32_t)t[3];
                    st.q4[r] = (int32_t)t[4];
                }
                // normalize_col_f32_with_stats constants (src/l2/normalize.rs:115-154)
                const double mean = n > 0 ? (double)s / (double)n : 0.0;
                const double css = (double)q - (double)n * mean * mean;
                const double sd = sqrt(css / (double)n_used);
                s_mean = (double)(float)mean;
                s_inv = sd > 0.0 ? (double)(float)(1.0 / sd) : 0.0;
            }
        }
        __syncthreads();
        const double mean = s_mean, inv = s_inv;
        double part = 0.0;
        float* ov = reinterpret_cast<float*>(Z);  // bucket values replace S1 in shared memory
        for (uint32_t b = threadIdx.x; b < d; b += NT) {
            const float o = (float)(inv * ((double)Z[b] - mean * (double)P[b]));
            ov[b] = o;
            part += (double)o * (double)o;
        }
        part = warp_sum(part);
        if ((threadIdx.x & 31) == 0) dred[threadIdx.x >> 5] = part;
        __syncthreads();
        double nrm = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++) nrm += dred[w];
        const float scale = nrm > 0.0 ? (float)sqrt((double)n_used / nrm) : 1.0f;
        float* orow = out + (uint64_t)r * (split ? 2 : 1) * ld;
        if (split) {
            // tensor-core operand rows: 2r = tf32(v), 2r+1 = tf32(v - tf32(v))
            float* lrow = orow + ld;
            for (uint64_t b = threadIdx.x; b < ld; b += NT) {
                float hi = 0.f, lo = 0.f;
                if (b < d) {
                    const float v = nrm > 0.0 ? ov[b] * scale : ov[b];
                    hi = to_tf32(v);
                    lo = to_tf32(v - hi);
                }
                orow[b] = hi;
                lrow[b] = lo;
            }
        } else {
            for (uint64_t b = threadIdx.x; b < ld; b += NT)
                orow[b] = b < d ? (nrm > 0.0 ? ov[b] * scale : ov[b]) : 0.f;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_sketch_permute(const PanelView& p, const int32_t* perm, uint64_t n_used, uint32_t* out,
                                  uint64_t out_pitch_words, cudaStream_t stream) {
    if (p.n_snp == 0) return cudaSuccess;
    int smem_row = p.pitch <= 160 * 1024 ? 1 : 0;
    size_t smem = smem_row ? p.pitch : 0;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_sketch_permute, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    uint64_t grid = p.n_snp < 148 * 16 ? p.n_snp : 148 * 16;
    k_sketch_permute<<<(unsigned)grid, NT, smem, stream>>>(p, perm, n_used, out, out_pitch_words, smem_row);
    return cudaGetLastError();
}

cudaError_t launch_sketch_seg(const uint32_t* pp, uint64_t pp_pitch_words, const uint64_t* rec_rows, int64_t m,
                              uint64_t n_used, const int32_t* seg_off, const int32_t* word_seg, uint32_t d,
                              RecStats st, int want_moments, int split, float* out, uint64_t ld,
                              cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    const size_t smem = sizeof(int32_t) * 2 * (size_t)d;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_sketch_seg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int64_t grid = m < 148 * 8 ? m : 148 * 8;
    k_sketch_seg<<<(unsigned)grid, NT, smem, stream>>>(pp, pp_pitch_words, rec_rows, m, n_used, seg_off, word_seg, d,
                                                       st, want_moments, split, out, ld);
    return cudaGetLastError();
}

}  // namespace ldsc
