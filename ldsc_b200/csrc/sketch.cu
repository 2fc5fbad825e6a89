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
// k_sketch_permute rewrites every panel row in that order (bit-plane quads of
// 64 positions, sketch_quad.cuh), after which each (bucket, sign) group is a
// contiguous run of positions.  k_sketch_seg then streams a permuted row once
// and forms the bucket sums from popcount prefix sums at the run boundaries;
// the same popcounts give the per-SNP moments.
//
// mean / inv_std are the reference's f32-rounded values; each bucket value is
// formed exactly and rounded to f32 once (the reference accumulates f32 in
// individual order; the two agree to f32 rounding).  The per-SNP moments
// (n, s, q, and the 3rd/4th for the MAF-aware correction) are permutation
// invariant and are produced by the same pass.
#include <cuda_runtime.h>

#include "engine.h"
#include "sketch_quad.cuh"
#include "sm100.cuh"

namespace ldsc {

namespace {

constexpr int NT = 256;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Rewrite panel rows in bucket-major individual order, as bit-plane quads
// (sketch_quad.cuh).  perm[p] = FAM index of the individual at permuted
// position p (p < n_used); positions past n_used read as missing.  One CTA per
// row, the row staged in shared memory when it fits (smem_row != 0).  A warp
// forms 32 halves (32 positions each) per step: for half h lane l reads the
// code at position 32 h + l (coalesced perm loads, eight halves' loads in
// flight), two ballots give the half's low-plane and high-plane words, and
// lane t keeps half t's pair, so the step ends in one coalesced 256-byte store.
__global__ void __launch_bounds__(NT) k_sketch_permute(PanelView p, const int32_t* __restrict__ perm,
                                                       uint64_t n_used, uint32_t* __restrict__ out,
                                                       uint64_t out_pitch_words, int smem_row) {
    extern __shared__ uint32_t srow32[];
    const uint8_t* srow = reinterpret_cast<const uint8_t*>(srow32);
    const uint64_t halves = out_pitch_words / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    for (uint64_t r = blockIdx.x; r < p.n_snp; r += gridDim.x) {
        const uint8_t* row = p.rows + r * p.pitch;
        if (smem_row) {
            const uint4* src = reinterpret_cast<const uint4*>(row);
            uint4* dst = reinterpret_cast<uint4*>(srow32);
            for (uint64_t q = threadIdx.x; q < p.pitch / 16; q += NT) dst[q] = __ldg(src + q);
            __syncthreads();
        }
        const uint8_t* from = smem_row ? srow : row;
        uint2* orow = reinterpret_cast<uint2*>(out + r * out_pitch_words);
        for (uint64_t g0 = (uint64_t)warp * 32; g0 < halves; g0 += NW * 32) {
            uint32_t my_lo = 0, my_hi = 0;
#pragma unroll 8
            for (int t = 0; t < 32; t++) {
                const uint64_t h = g0 + t;  // the same in every lane
                if (h >= halves) break;
                const uint64_t pos = h * 32 + lane;
                uint32_t code = 1u;  // missing
                if (pos < n_used) {
                    const int32_t iid = __ldg(perm + pos);
                    code = (from[iid >> 2] >> ((iid & 3) * 2)) & 3u;
                }
                const uint32_t lo = __ballot_sync(0xFFFFFFFFu, code & 1u);
                const uint32_t hi = __ballot_sync(0xFFFFFFFFu, code >> 1);
                if (lane == t) {
                    my_lo = lo;
                    my_hi = hi;
                }
            }
            if (g0 + lane < halves) orow[g0 + lane] = make_uint2(my_lo, my_hi);
        }
        __syncthreads();
    }
}

// Bucket sums from prefix sums.  Over any span of positions (quad counts in
// sketch_quad.cuh)  sum g = 2 len - bits - missing  and  present = len -
// missing.  With the prefix (sum g, present) at every run boundary k, bucket
// b is
//     S1_b = (PF[2b+1] - PF[2b]) - (PF[2b+2] - PF[2b+1])   (g sums; S0_b with present)
// and row moments come from the totals:
//     n = present, s = sum g, q = s + 2 #2, q3 = s + 6 #2, q4 = s + 14 #2
// (#2 = number of genotype-2 codes = len - high bits - missing).
//
// Two phases per record.  (1) Streaming: each warp owns a contiguous block of
// the row's 16-byte quads and walks it 64 quads at a time, two adjacent quads
// per lane (coalesced loads, branch-free popcounts); one warp scan of the
// packed (bits, missing) counts gives the prefix at the start of every quad,
// kept in shared memory.  (2) Boundaries: after a block scan over the warps,
// thread t takes the buckets [d t / SNT, d (t+1) / SNT) and walks their
// boundaries in order; each prefix is the quad prefix, plus the offset of the
// warp that streamed the quad, plus popcounts inside the quad (re-read from
// L1/L2).  Thread t's boundary positions come from a thread-major table built
// once per layout (entry i * SNT + t = its i-th boundary, with the owning warp
// in the top bits), so their loads are coalesced.  Each bucket's value is
// formed on the spot.  No atomics, and nothing needs clearing between
// records.
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

constexpr int SNT = 128;       // threads of the sketch kernel
constexpr int SNW = SNT / 32;  // warps
constexpr int CHUNK_Q = 64;    // quads per warp step (2 per lane)

__host__ __device__ inline uint64_t sketch_quads(uint64_t n_used) { return ((n_used + 15) / 16 + 3) / 4; }

// Thread t of a T-thread CTA takes buckets [seg_b(d, t), seg_b(d, t + 1)):
// 2 (b1 - b0) + 1 boundaries; seg_rows bounds that count over t.
template <int T>
__host__ __device__ inline uint32_t seg_b(uint32_t d, uint32_t t) { return (uint32_t)((uint64_t)d * t / T); }
template <int T>
__host__ __device__ inline uint32_t seg_count(uint32_t d, uint32_t t) {
    const uint32_t b0 = seg_b<T>(d, t), b1 = seg_b<T>(d, t + 1);
    return b0 < b1 ? 2 * (b1 - b0) + 1 : 0;
}
template <int T>
__host__ __device__ inline uint32_t seg_rows(uint32_t d) { return 2 * ((d + T - 1) / T) + 1; }

// Boundary table entry of the streaming-form kernel: position | owning warp << 28.
constexpr int SEG_POS_BITS = 28;
constexpr int32_t SEG_POS_MASK = (1 << SEG_POS_BITS) - 1;

// Dynamic shared memory of the sketch kernel: per-quad prefixes (an even
// count, so the bucket values start on 16 bytes) and the d bucket values
// (+16 bytes read past d by the vector output loop).
__host__ __device__ inline size_t sketch_smem(uint64_t n_used, uint32_t d) {
    return 8 * ((sketch_quads(n_used) + 1) & ~1ull) + 4 * (size_t)d + 16;
}

// Record r's output from the bucket values ob (16-byte aligned): `ld` floats
// (zero padded past d), or with split the tensor-core operand rows
// 2r = tf32(v) and 2r+1 = tf32(v - tf32(v)), stored four at a time (ld is a
// multiple of 32 there).
template <int T>
__device__ __forceinline__ void write_sketch_row(const float* ob, uint32_t d, double nrm, float scale, int split,
                                                 float* orow, uint64_t ld) {
    if (split) {
        float4* h4 = reinterpret_cast<float4*>(orow);
        float4* l4 = reinterpret_cast<float4*>(orow + ld);
        const float4* o4 = reinterpret_cast<const float4*>(ob);
        for (uint32_t v = threadIdx.x; v < (uint32_t)(ld / 4); v += T) {
            const float4 x = 4 * v < d ? o4[v] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float e[4] = {x.x, x.y, x.z, x.w};
            float hi[4], lo[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float val = nrm > 0.0 ? e[k] * scale : e[k];
                hi[k] = 4 * v + k < d ? to_tf32(val) : 0.f;
                lo[k] = 4 * v + k < d ? to_tf32(val - hi[k]) : 0.f;
            }
            h4[v] = make_float4(hi[0], hi[1], hi[2], hi[3]);
            l4[v] = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
    } else {
        for (uint64_t b = threadIdx.x; b < ld; b += T) orow[b] = b < d ? (nrm > 0.0 ? ob[b] * scale : ob[b]) : 0.f;
    }
}

// One CTA per record (grid-stride over records).  Output row r: `ld` floats
// (zero padded past d), or with split the hi/lo tensor-core rows 2r / 2r+1.
__global__ void __launch_bounds__(SNT, 8) k_sketch_seg(const uint32_t* __restrict__ pp, uint64_t pp_pitch_words,
                                                    const uint64_t* __restrict__ rec_rows, int64_t m, uint64_t n_used,
                                                    const int32_t* __restrict__ segt, uint32_t d, RecStats st,
                                                    int want_moments, int split, float* __restrict__ out,
                                                    uint64_t ld) {
    extern __shared__ __align__(16) int32_t sh[];
    const uint32_t quads = (uint32_t)sketch_quads(n_used);  // the permuted pitch is 4 quads' worth of words, padded
    int2* Pq = reinterpret_cast<int2*>(sh);                  // (popc, missing) before each quad, warp-relative
    float* ob = reinterpret_cast<float*>(sh + 2 * ((quads + 1) & ~1u));  // bucket values
    __shared__ int32_t wa[SNW], wm[SNW], wt[SNW];
    __shared__ int2 woff[SNW];  // (bits, missing) before each warp's block
    __shared__ double dred[SNW], rconst[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t wq0 = (uint32_t)((uint64_t)quads * warp / SNW), wq1 = (uint32_t)((uint64_t)quads * (warp + 1) / SNW);
    const uint32_t b0 = seg_b<SNT>(d, threadIdx.x), nbd = seg_count<SNT>(d, threadIdx.x);
    const int32_t row_len = (int32_t)(64 * quads);
    for (int64_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint4* row = reinterpret_cast<const uint4*>(pp + brow * pp_pitch_words);
        // ---- phase 1: stream the warp's quads ----
        int32_t carryA = 0, carryM = 0, HT = 0;
        uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
        if (wq0 + 2 * lane < wq1) n0 = __ldg(row + wq0 + 2 * lane);
        if (wq0 + 2 * lane + 1 < wq1) n1 = __ldg(row + wq0 + 2 * lane + 1);
        for (uint32_t c0 = wq0; c0 < wq1; c0 += CHUNK_Q) {
            const uint32_t qa = c0 + 2 * lane;
            const bool l0 = qa < wq1, l1 = qa + 1 < wq1;
            const uint4 v0 = n0, v1 = n1;
            if (qa + CHUNK_Q < wq1) n0 = __ldg(row + qa + CHUNK_Q);
            if (qa + CHUNK_Q + 1 < wq1) n1 = __ldg(row + qa + CHUNK_Q + 1);
            int32_t a0, m0, h0, a1, m1, h1;
            quad_counts(v0, a0, m0, h0);
            quad_counts(v1, a1, m1, h1);
            const int32_t la = (l0 ? a0 : 0) + (l1 ? a1 : 0), lm = (l0 ? m0 : 0) + (l1 ? m1 : 0);
            HT += (l0 ? h0 : 0) + (l1 ? h1 : 0);
            // (bits, missing) packed in 16-bit halves: a chunk holds at most
            // 64 quads x 128 bits = 8,192, so the halves cannot carry
            const int32_t lp = la | (lm << 16);
            const int32_t ip = warp_incl_scan(lp, lane);
            const int32_t ia = ip & 0xFFFF, im = ip >> 16;
            const int32_t ea = carryA + ia - la, em = carryM + im - lm;
            if (l0) Pq[qa] = make_int2(ea, em);
            if (l1) Pq[qa + 1] = make_int2(ea + a0, em + m0);
            const int32_t tp = __shfl_sync(0xFFFFFFFFu, ip, 31);
            carryA += tp & 0xFFFF;
            carryM += tp >> 16;
        }
        const int32_t htw = warp_sum(HT);
        if (lane == 0) {
            wa[warp] = carryA;
            wm[warp] = carryM;
            wt[warp] = htw;
        }
        __syncthreads();
        // ---- block scan over the warps: offsets and row totals ----
        int32_t A = 0, MS = 0, H = 0;
#pragma unroll
        for (int w = 0; w < SNW; w++) {
            A += wa[w];
            MS += wm[w];
            H += wt[w];
        }
        // padding positions are missing: no effect on G and N, and TT = #2
        const int32_t G = 2 * row_len - A - MS, N = row_len - MS, TT = row_len - H - MS;
        if (threadIdx.x == 0) {
            st.n[r] = N;
            st.s[r] = G;
            st.q[r] = G + 2 * TT;
            if (want_moments && st.q3) {
                st.q3[r] = G + 6 * TT;
                st.q4[r] = G + 14 * TT;
            }
        }
        // normalize_col_f32_with_stats constants (src/l2/normalize.rs:115-154),
        // formed once and read by every thread after the barrier below
        if (threadIdx.x == 0) {
            const double dmean = N > 0 ? (double)G / (double)N : 0.0;
            const double css = (double)(G + 2 * TT) - (double)N * dmean * dmean;
            const double sd = sqrt(css / (double)n_used);
            rconst[0] = (double)(float)dmean;
            rconst[1] = sd > 0.0 ? (double)(float)(1.0 / sd) : 0.0;
        }
        if (threadIdx.x < SNW) {
            int32_t oa = 0, om = 0;
#pragma unroll
            for (int w = 0; w < SNW - 1; w++)
                if (w < (int)threadIdx.x) {
                    oa += wa[w];
                    om += wm[w];
                }
            woff[threadIdx.x] = make_int2(oa, om);
        }
        __syncthreads();
        const double mean = rconst[0], inv = rconst[1];
        // ---- phase 2: this thread's buckets ----
        // Boundaries in groups of four: the group's table entries are loaded
        // one group ahead and its four quads are loaded together.
        double part = 0.0;
        if (nbd) {
            int32_t pn[4];
#pragma unroll
            for (int u = 0; u < 4; u++) pn[u] = (uint32_t)u < nbd ? __ldg(segt + u * SNT + threadIdx.x) : row_len;
            int32_t g1 = 0, n1w = 0, g2 = 0, n2w = 0;  // prefixes at the previous two boundaries
            for (uint32_t i = 0; i < nbd; i += 4) {
                int32_t pc[4];
                uint4 qv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    pc[u] = pn[u];
                    pn[u] = i + 4 + u < nbd ? __ldg(segt + (i + 4 + u) * SNT + threadIdx.x) : row_len;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int32_t p = pc[u] & SEG_POS_MASK;
                    qv[u] = p < row_len ? __ldg(row + (p >> 6)) : make_uint4(0, 0, 0, 0);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (i + u >= nbd) break;
                    const int32_t p = pc[u] & SEG_POS_MASK;
                    int32_t pg = G, pnr = N;  // at or past the row end: the totals
                    if (p < row_len) {
                        // quad prefix + offset of the warp that streamed the quad + inside the quad
                        const int2 pq = Pq[p >> 6], of = woff[(uint32_t)pc[u] >> SEG_POS_BITS];
                        int32_t ha, hm;
                        quad_head(qv[u], (uint32_t)p & 63u, ha, hm);
                        const int32_t pa = pq.x + of.x + ha, pm = pq.y + of.y + hm;
                        pg = 2 * p - pa - pm;
                        pnr = p - pm;
                    }
                    const uint32_t idx = i + u;
                    if (idx >= 2 && !(idx & 1)) {  // bucket b0 + idx/2 - 1 is complete
                        const int32_t s1 = (g1 - g2) - (pg - g1), s0 = (n1w - n2w) - (pnr - n1w);
                        const float o = (float)(inv * ((double)s1 - mean * (double)s0));
                        ob[b0 + idx / 2 - 1] = o;
                        part += (double)o * (double)o;
                    }
                    g2 = g1;
                    n2w = n1w;
                    g1 = pg;
                    n1w = pnr;
                }
            }
        }
        part = warp_sum(part);
        if (lane == 0) dred[warp] = part;
        __syncthreads();
        double nrm = 0.0;
#pragma unroll
        for (int w = 0; w < SNW; w++) nrm += dred[w];
        const float scale = nrm > 0.0 ? (float)sqrt((double)n_used / nrm) : 1.0f;
        write_sketch_row<SNT>(ob, d, nrm, scale, split, out + (uint64_t)r * (split ? 2 : 1) * ld, ld);
        __syncthreads();  // Pq, ob, wa and dred are rewritten by the next record
    }
}

// ---- large d: quads in shared memory, thread-major boundary positions ----
//
// With many buckets the boundary phase dominates and its quad re-reads go to
// L2.  This form keeps the row's quads in shared memory and, per quad, the
// prefix before it (made block-absolute by a fix-up pass) and the counts of
// its first half; thread t's boundary positions come from a thread-major
// table (entry i * S6T + t = i-th boundary of thread t, built once per
// layout), so their loads are coalesced, and each boundary prefix costs two
// shared-memory loads (the quad's prefix entry and its half's two plane
// words) and three popcounts.  256 threads per
// CTA: its shared memory (32 B per 64 individuals + 4 B per bucket) allows
// few CTAs per SM, so each CTA brings more warps.  Same arithmetic as the
// kernel above; results are bit-identical.
constexpr int S6T = 256;
constexpr int S6W = S6T / 32;

__host__ __device__ inline size_t sketch6_smem(uint64_t n_used, uint32_t d) {
    return 32 * sketch_quads(n_used) + 4 * (size_t)d + 16;
}

// Thread-major boundary table for a T-thread kernel: entry i * T + t = the
// i-th boundary position of thread t (0x7FFFFFFF past its count); with
// owners, the streaming-form entry (position | owning warp << 28, the warp
// of SNW whose block holds the position's quad).
template <int T, bool OWNERS>
__global__ void k_sketch_segt(const int32_t* __restrict__ seg_off, uint32_t d, uint32_t rows, uint32_t quads,
                              int32_t* __restrict__ segt) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * T; e += gridDim.x * blockDim.x) {
        const uint32_t i = e / T, t = e % T;
        int32_t v = 0x7FFFFFFF;
        if (i < seg_count<T>(d, t)) {
            v = seg_off[2 * seg_b<T>(d, t) + i];
            if (OWNERS) {
                const uint64_t q = (uint64_t)v >> 6;
                int32_t w = 0;
                for (int o = 1; o < SNW; o++)
                    if (q >= (uint64_t)quads * o / SNW) w = o;
                v |= w << SEG_POS_BITS;
            }
        }
        segt[e] = v;
    }
}

__global__ void __launch_bounds__(S6T, 3) k_sketch_seg6(const uint32_t* __restrict__ pp, uint64_t pp_pitch_words,
                                                      const uint64_t* __restrict__ rec_rows, int64_t m,
                                                      uint64_t n_used, const int32_t* __restrict__ segt, uint32_t d,
                                                      RecStats st, int want_moments, int split,
                                                      float* __restrict__ out, uint64_t ld) {
    extern __shared__ __align__(16) uint4 sh6[];
    const uint32_t quads = (uint32_t)sketch_quads(n_used);
    uint4* PQ = sh6;          // (bits, missing) before the quad, then in its first half
    uint4* Rs = sh6 + quads;  // the quads
    float* ob = reinterpret_cast<float*>(sh6 + 2 * (size_t)quads);
    __shared__ int32_t wa[S6W], wm[S6W], wt[S6W];
    __shared__ double dred[S6W], rconst[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t wq0 = (uint32_t)((uint64_t)quads * warp / S6W), wq1 = (uint32_t)((uint64_t)quads * (warp + 1) / S6W);
    const uint32_t b0 = seg_b<S6T>(d, threadIdx.x), nbd = seg_count<S6T>(d, threadIdx.x);
    const int32_t row_len = (int32_t)(64 * quads);
    for (int64_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint64_t brow = rec_rows ? rec_rows[r] : (uint64_t)r;
        const uint4* row = reinterpret_cast<const uint4*>(pp + brow * pp_pitch_words);
        // ---- phase 1 ----
        int32_t carryA = 0, carryM = 0, HT = 0;
        uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
        if (wq0 + 2 * lane < wq1) n0 = __ldg(row + wq0 + 2 * lane);
        if (wq0 + 2 * lane + 1 < wq1) n1 = __ldg(row + wq0 + 2 * lane + 1);
        for (uint32_t c0 = wq0; c0 < wq1; c0 += CHUNK_Q) {
            const uint32_t qa = c0 + 2 * lane;
            const bool l0 = qa < wq1, l1 = qa + 1 < wq1;
            const uint4 v0 = n0, v1 = n1;
            if (qa + CHUNK_Q < wq1) n0 = __ldg(row + qa + CHUNK_Q);
            if (qa + CHUNK_Q + 1 < wq1) n1 = __ldg(row + qa + CHUNK_Q + 1);
            int32_t a0, m0, h0, fa0, fm0, a1, m1, h1, fa1, fm1;
            quad_counts(v0, a0, m0, h0, fa0, fm0);
            quad_counts(v1, a1, m1, h1, fa1, fm1);
            const int32_t la = (l0 ? a0 : 0) + (l1 ? a1 : 0), lm = (l0 ? m0 : 0) + (l1 ? m1 : 0);
            HT += (l0 ? h0 : 0) + (l1 ? h1 : 0);
            const int32_t lp = la | (lm << 16);  // at most 8,192 bits per chunk: no carry
            const int32_t ip = warp_incl_scan(lp, lane);
            const int32_t ia = ip & 0xFFFF, im = ip >> 16;
            const int32_t ea = carryA + ia - la, em = carryM + im - lm;
            if (l0) {
                PQ[qa] = make_uint4((uint32_t)ea, (uint32_t)em, (uint32_t)fa0, (uint32_t)fm0);
                Rs[qa] = v0;
            }
            if (l1) {
                PQ[qa + 1] = make_uint4((uint32_t)(ea + a0), (uint32_t)(em + m0), (uint32_t)fa1, (uint32_t)fm1);
                Rs[qa + 1] = v1;
            }
            const int32_t tp = __shfl_sync(0xFFFFFFFFu, ip, 31);
            carryA += tp & 0xFFFF;
            carryM += tp >> 16;
        }
        const int32_t htw = warp_sum(HT);
        if (lane == 0) {
            wa[warp] = carryA;
            wm[warp] = carryM;
            wt[warp] = htw;
        }
        __syncthreads();
        int32_t A = 0, MS = 0, H = 0, offA = 0, offM = 0;
#pragma unroll
        for (int w = 0; w < S6W; w++) {
            if (w < warp) {
                offA += wa[w];
                offM += wm[w];
            }
            A += wa[w];
            MS += wm[w];
            H += wt[w];
        }
        const int32_t G = 2 * row_len - A - MS, N = row_len - MS, TT = row_len - H - MS;
        if (threadIdx.x == 0) {
            st.n[r] = N;
            st.s[r] = G;
            st.q[r] = G + 2 * TT;
            if (want_moments && st.q3) {
                st.q3[r] = G + 6 * TT;
                st.q4[r] = G + 14 * TT;
            }
        }
        if (threadIdx.x == 0) {  // the record's constants, read after the barrier below
            const double dmean = N > 0 ? (double)G / (double)N : 0.0;
            const double css = (double)(G + 2 * TT) - (double)N * dmean * dmean;
            const double sd = sqrt(css / (double)n_used);
            rconst[0] = (double)(float)dmean;
            rconst[1] = sd > 0.0 ? (double)(float)(1.0 / sd) : 0.0;
        }
        // block-absolute quad prefixes
        if (offA | offM)
            for (uint32_t q = wq0 + lane; q < wq1; q += 32) {
                uint2* e = reinterpret_cast<uint2*>(PQ + q);
                const uint2 v = *e;
                *e = make_uint2(v.x + (uint32_t)offA, v.y + (uint32_t)offM);
            }
        __syncthreads();
        const double mean = rconst[0], inv = rconst[1];
        // ---- phase 2 ----
        double part = 0.0;
        if (nbd) {
            const uint2* rh = reinterpret_cast<const uint2*>(Rs);  // (low, high) plane words of each half
            int32_t pn[4];
#pragma unroll
            for (int u = 0; u < 4; u++) pn[u] = (uint32_t)u < nbd ? __ldg(segt + u * S6T + threadIdx.x) : row_len;
            int32_t g1 = 0, n1w = 0, g2 = 0, n2w = 0;
            for (uint32_t i = 0; i < nbd; i += 4) {
                int32_t pc[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    pc[u] = pn[u];
                    pn[u] = i + 4 + u < nbd ? __ldg(segt + (i + 4 + u) * S6T + threadIdx.x) : row_len;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (i + u >= nbd) break;
                    const int32_t p = pc[u];
                    int32_t pg = G, pnr = N;  // at the row end: the totals
                    if (p < row_len) {
                        const uint32_t q = (uint32_t)p >> 6, hf = ((uint32_t)p >> 5) & 1u;
                        const uint4 e = PQ[q];
                        const uint2 lh = rh[2 * q + hf];
                        int32_t ha, hm;
                        half_head(lh.x, lh.y, (uint32_t)p & 31u, ha, hm);
                        const int32_t pa = (int32_t)e.x + (hf ? (int32_t)e.z : 0) + ha;
                        const int32_t pm = (int32_t)e.y + (hf ? (int32_t)e.w : 0) + hm;
                        pg = 2 * p - pa - pm;
                        pnr = p - pm;
                    }
                    const uint32_t idx = i + u;
                    if (idx >= 2 && !(idx & 1)) {  // bucket b0 + idx/2 - 1 is complete
                        const int32_t s1 = (g1 - g2) - (pg - g1), s0 = (n1w - n2w) - (pnr - n1w);
                        const float o = (float)(inv * ((double)s1 - mean * (double)s0));
                        ob[b0 + idx / 2 - 1] = o;
                        part += (double)o * (double)o;
                    }
                    g2 = g1;
                    n2w = n1w;
                    g1 = pg;
                    n1w = pnr;
                }
            }
        }
        part = warp_sum(part);
        if (lane == 0) dred[warp] = part;
        __syncthreads();
        double nrm = 0.0;
#pragma unroll
        for (int w = 0; w < S6W; w++) nrm += dred[w];
        const float scale = nrm > 0.0 ? (float)sqrt((double)n_used / nrm) : 1.0f;
        write_sketch_row<S6T>(ob, d, nrm, scale, split, out + (uint64_t)r * (split ? 2 : 1) * ld, ld);
        __syncthreads();  // PQ, Rs, ob, wa and dred are rewritten by the next record
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
                              uint64_t n_used, const int32_t* segt, uint32_t d, RecStats st, int want_moments,
                              int split, float* out, uint64_t ld, cudaStream_t stream) {
    if (m <= 0) return cudaSuccess;
    const int64_t grid = m < 148 * 16 ? m : 148 * 16;
    if (sketch_large_d(n_used, d)) {
        const size_t smem6 = sketch6_smem(n_used, d);
        cudaError_t e = cudaFuncSetAttribute(k_sketch_seg6, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem6);
        if (e != cudaSuccess) return e;
        // three 256-thread CTAs per SM: their rows and prefixes need the
        // largest shared-memory carveout
        e = cudaFuncSetAttribute(k_sketch_seg6, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        k_sketch_seg6<<<(unsigned)grid, S6T, smem6, stream>>>(pp, pp_pitch_words, rec_rows, m, n_used, segt, d, st,
                                                               want_moments, split, out, ld);
        return cudaGetLastError();
    }
    const size_t smem = sketch_smem(n_used, d);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;  // rejected by the caller first (ldsc_sketch_supported)
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_sketch_seg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_sketch_seg<<<(unsigned)grid, SNT, smem, stream>>>(pp, pp_pitch_words, rec_rows, m, n_used, segt, d, st,
                                                       want_moments, split, out, ld);
    return cudaGetLastError();
}

bool sketch_supported(uint64_t n_used, uint32_t d) { return sketch_smem(n_used, d) <= 200 * 1024; }

// Measured at N = 100,000: the streaming form is faster up to d ~ 2,600, the
// shared-memory-row form above (d = 2,500: 0.50 vs 0.52 ms per 20,000 rows;
// d = 3,000: 0.63 vs 0.57 ms).
bool sketch_large_d(uint64_t n_used, uint32_t d) { return d >= 2560 && sketch6_smem(n_used, d) <= 200 * 1024; }

uint64_t sketch_segt_count(uint64_t n_used, uint32_t d) {
    return sketch_large_d(n_used, d) ? (uint64_t)seg_rows<S6T>(d) * S6T : (uint64_t)seg_rows<SNT>(d) * SNT;
}

cudaError_t launch_sketch_segt(const int32_t* seg_off, uint64_t n_used, uint32_t d, int32_t* segt,
                               cudaStream_t stream) {
    const uint32_t quads = (uint32_t)sketch_quads(n_used);
    if (sketch_large_d(n_used, d))
        k_sketch_segt<S6T, false><<<64, 256, 0, stream>>>(seg_off, d, seg_rows<S6T>(d), quads, segt);
    else
        k_sketch_segt<SNT, true><<<64, 256, 0, stream>>>(seg_off, d, seg_rows<SNT>(d), quads, segt);
    return cudaGetLastError();
}

cudaError_t preload_sketch() {
    cudaError_t e = preload_kernel(k_sketch_permute);
    if (e == cudaSuccess) e = preload_kernel(k_sketch_seg);
    if (e == cudaSuccess) e = preload_kernel(k_sketch_seg6);
    if (e == cudaSuccess) e = preload_kernel(k_sketch_segt<SNT, true>);
    if (e == cudaSuccess) e = preload_kernel(k_sketch_segt<S6T, false>);
    return e;
}

}  // namespace ldsc
