// gram_tc.cu -- band Gram on the 5th-generation tensor cores (tcgen05), in
// two operand kinds that share one tile structure:
//   * INT8-exact form (kind::i8): genotype / mask rows, exact epilogue;
//   * CountSketch form (kind::tf32): each sketched f32 value v is split as
//     v = hi + lo with hi = tf32(v), lo = tf32(v - hi), stored as rows 2r (hi)
//     and 2r+1 (lo); one UMMA then yields hi.hi, hi.lo, lo.hi, lo.lo for every
//     pair, whose sum is the f32-accurate dot product (the reference's f32
//     GEMM, src/l2/compute.rs:1897-2079), followed by the quadratic bias
//     inversion (src/l2/compute.rs:947-998) in f64.
//
// INT8-exact form:
// Operands: for record r, row 2r holds its genotypes G (0/1/2, 0 at missing)
// and row 2r+1 its non-missing mask M (0/1), one byte per individual, rows of
// `ld` bytes (a multiple of 128).  One UMMA tile multiplies 128 A rows
// (64 left records k) by 256 B rows (128 right records j) over K = individuals
// with INT32 accumulation in TMEM, which yields for every record pair the
// four integer products
//     GG = sum G_k G_j,  GM = sum G_k M_j,  MG = sum M_k G_j,  MM = sum M_k M_j.
// With n, s, q the per-record non-missing count, genotype sum and sum of
// squares, the reference's standardised dot product (normalize.rs:71-110
// followed by the A^T B GEMM, compute.rs:1897-2236) is recovered exactly:
//     X   = n_k n_j GG - n_k s_j GM - s_k n_j MG + s_k s_j MM   (int64, exact)
//     r   = X / sqrt(n_k V_k n_j V_j),  V = n q - s^2            (f64)
//     r2u = r^2 (1 + 1/(N-2)) - 1/(N-2)                           (f64)
// N cancels from r; a monomorphic record (V = 0) gives r = 0 and
// r2u = -1/(N-2), as the reference's zero inv_std does.
//
// Kernel structure (persistent, one CTA per SM, 6 warps):
//   warp 0     TMA producer: A 128x128 B + B 256x128 B per stage, 128-byte swizzle
//   warp 1     TMEM allocator (512 columns = two 256-column accumulators) and
//              UMMA issuer (tcgen05.mma kind::i8, M=128 N=256 K=32, four per stage)
//   warps 2-5  epilogue: tcgen05.ld of the accumulator, exact r^2, band mask,
//              l2 accumulation; accumulator double-buffering overlaps the
//              epilogue of tile t with the MMAs of tile t+1.  Where the
//              epilogue outweighs the MMAs -- INT8 rows of fewer than 32,768
//              individuals, and the sketch forms (short K, a heavier per-pair
//              correction) -- warps 2-9 (2-17) do it: two (four) warps per
//              TMEM lane quarter, each on a share of the columns.  With K > 1
//              annotation columns the epilogue stores each tile's masked r2u
//              values (f64) for the contraction passes of contract.cu.
// Fused INT8 form (the operand rows are never written to HBM): warp 0 stages
// the packed 2-bit BED rows themselves by TMA -- 32 bytes per record per 128
// individuals, 6 KB per stage for the 64 + 128 records of a tile instead of
// 48 KB of operand rows -- and four or eight converter warps expand each packed stage
// in shared memory into the 128-byte-swizzled G / M operand tiles the MMA warp
// reads, with a proxy fence before they hand the stage over.  The K order of
// individuals inside a 16-byte chunk is permuted (evens, then odds) the same
// way in every row, which leaves every product sum unchanged; individuals past
// N read as missing.
//
// Every mbarrier wait is bounded; on timeout the kernel records an error word,
// drains its own in-flight copies / MMAs (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include "engine.h"
#include "epilogue.cuh"
#include "expand.cuh"
#include "sm100.cuh"

namespace ldsc {

namespace {

constexpr int TA = 64;             // left records per tile (A rows = 128)
constexpr int TB = 128;            // right records per tile (B rows = 256)
constexpr int A_BYTES = 128 * 128; // one stage of A
constexpr int B_BYTES = 256 * 128; // one stage of B
// fused form: packed ring of 2-bit rows, 128 individuals (32 bytes) per record per stage
constexpr int P_STAGES = 4;
constexpr int PA_BYTES = TA * 32;
constexpr int P_BYTES = (TA + TB) * 32;
// converter warps: 8 beside 4 epilogue warps (fused Gram 21.1 -> 20.1 ms at
// 50,000 individuals x 100,000 SNPs), 4 beside 8 (448 threads either way;
// 8 + 8 would be 576 threads, capping registers at 113 and spilling)
constexpr int CONV_WARPS = 4;
constexpr int CONV_WARPS_NARROW = 8;
// threads per CTA: TMA and MMA warps + ew epilogue warps (4, 8 or 16) + cw converter warps
__host__ __device__ constexpr int gram_threads(int ew, int cw) { return 64 + 32 * ew + 32 * cw; }
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ int64_t shfl_xor_i64(int64_t v, int mask) {
    int lo = (int)(v & 0xFFFFFFFF), hi = (int)(v >> 32);
    lo = __shfl_xor_sync(0xFFFFFFFFu, lo, mask);
    hi = __shfl_xor_sync(0xFFFFFFFFu, hi, mask);
    return ((int64_t)hi << 32) | (uint32_t)lo;
}

// MODE 0: INT8 exact r^2; 1: TF32 sketch, quadratic correction; 2: same, MAF-aware.
template <int MODE>
__device__ __forceinline__ double sketch_r2u(float val, int64_t k, int64_t j, const EpilogueArgs& ep) {
    const double v = (double)val;
    const double kap = MODE == 2 ? __ldg(ep.kappa + k) + __ldg(ep.kappa + j) : 0.0;
    const double tilde = v * v * ep.n_inv_sq;
    const double dm3 = ep.sketch_d - 3.0 - 2.0 * kap;
    const double disc = dm3 * dm3 + 8.0 * (ep.sketch_d * tilde - 1.0);
    const double r2 = disc >= 0.0 ? (-dm3 + sqrt(disc)) * 0.25 : 0.0;
    return r2 * ep.r2u_a + ep.r2u_b;
}

// Sketch constants in f32 for sketch_r2u_f32.
struct SketchF {
    float n_inv_sq, d, r2u_a, r2u_b;
};

// sketch_r2u in f32, for d >= 8 (then dm3 > 2 - 2 kappa > 0 and the
// discriminant is positive): the root (-dm3 + sqrt(disc)) / 4 is taken in the
// cancellation-free form 2 q / (sqrt(disc) + dm3), q = d tilde - 1 (the same
// value: disc - dm3^2 = 8 q).  Its absolute error is about ulp(d tilde) / dm3,
// 3e-10 at d = 200, against the reference's f64 evaluation; l2 sums of a
// thousand such terms move by ~1e-7 relative, far inside the sketch's own
// f32 dot-product error.  Each pair's value depends on that pair alone, so
// runs over different tile grids (slices, shards) still agree to f64
// rounding of the sums.
template <int MODE>
__device__ __forceinline__ float sketch_r2u_f32(float val, int64_t k, int64_t j, const EpilogueArgs& ep,
                                                const SketchF& cf) {
    const float kap = MODE == 2 ? (float)(__ldg(ep.kappa + k) + __ldg(ep.kappa + j)) : 0.f;
    const float tilde = val * val * cf.n_inv_sq;
    const float dm3 = cf.d - 3.f - 2.f * kap;
    const float q = fmaf(cf.d, tilde, -1.f);
    const float disc = fmaf(dm3, dm3, 8.f * q);
    const float r2 = disc >= 0.f ? 2.f * q / (sqrtf(disc) + dm3) : 0.f;
    return fmaf(r2, cf.r2u_a, cf.r2u_b);
}

// CW = 0: A / B operand rows staged by TMA.  CW > 0 (INT8 only): packed 2-bit
// rows staged by TMA (tmA / tmB map the BED rows, boxes of 32 bytes x 64 / 128
// rows) and expanded by CW converter warps; n_indiv masks the last stage.
template <int STAGES, int MODE, int EW, int CW>
__global__ void __launch_bounds__(gram_threads(EW, CW), 1)
    k_gram_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              int num_kb, const Tile* __restrict__ tiles, int64_t n_tiles, EpilogueArgs ep,
              int32_t* __restrict__ dbg, uint64_t n_indiv) {
    static_assert(CW == 0 || MODE == 0, "the fused form is INT8 only");
    // elements per 128-byte stage row: 128 (INT8) or 32 (TF32); TMA x is in elements
    constexpr int KSTEP = MODE == 0 ? 128 : 32;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    uint8_t* smem = smem_raw + pad;
    uint8_t* sA = smem;
    uint8_t* sB = sA + STAGES * A_BYTES;
    uint8_t* sP = sB + STAGES * B_BYTES;   // fused form: packed ring
    uint64_t* full = reinterpret_cast<uint64_t*>(sP + (CW > 0 ? P_STAGES * P_BYTES : 0));
    uint64_t* empty = full + STAGES;
    uint64_t* pfull = empty + STAGES;   // [P_STAGES], fused form
    uint64_t* pempty = pfull + P_STAGES;
    uint64_t* tfull = pempty + P_STAGES;   // [2]
    uint64_t* tempty = tfull + 2;       // [2]
    uint64_t* drain = tempty + 2;       // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    double* cpart = reinterpret_cast<double*>(drain + 2);  // [4][TB]
    double* rpart = cpart + 4 * TB;                         // [4][TA]: row sums per column group

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], CW > 0 ? CW : 1);   // TMA transaction, or one arrival per converter warp
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < P_STAGES; s++) {
            mbar_init(&pfull[s], 1);
            mbar_init(&pempty[s], CW > 0 ? CW : 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 32 * EW);
        }
        mbar_init(drain, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (elect_one_sync()) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            uint32_t armed = 0;        // bit s: stage s has a load in flight we may need to drain
            uint32_t armed_par = 0;    // bit s: parity of that load's phase
            // the ring this warp fills: operand stages, or packed stages in the fused form
            constexpr int RING = CW > 0 ? P_STAGES : STAGES;
            uint64_t* rfull = CW > 0 ? pfull : full;
            uint64_t* rempty = CW > 0 ? pempty : empty;
            for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                const Tile tl = tiles[t];
                // operand rows: two per record; packed rows: one per record
                const int32_t ya = (int32_t)tl.a_blk * (CW > 0 ? TA : 2 * TA);
                const int32_t yb = (int32_t)tl.b_blk * (CW > 0 ? TB : 2 * TB);
                for (int kb = 0; kb < num_kb; kb++) {
                    if (!mbar_wait(&rempty[stage], phase ^ 1, WAIT_LIMIT_NS)) {
                        ok = false;
                        break;
                    }
                    if constexpr (CW > 0) {
                        mbar_arrive_expect_tx(&rfull[stage], P_BYTES);
                        tma_load_2d(sP + stage * P_BYTES, &tmA, &rfull[stage], kb * 32, ya);
                        tma_load_2d(sP + stage * P_BYTES + PA_BYTES, &tmB, &rfull[stage], kb * 32, yb);
                    } else {
                        mbar_arrive_expect_tx(&rfull[stage], A_BYTES + B_BYTES);
                        tma_load_2d(sA + stage * A_BYTES, &tmA, &rfull[stage], kb * KSTEP, ya);
                        tma_load_2d(sB + stage * B_BYTES, &tmB, &rfull[stage], kb * KSTEP, yb);
                    }
                    armed |= 1u << stage;
                    armed_par = (armed_par & ~(1u << stage)) | (phase << stage);
                    if (++stage == RING) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (!ok) {
                atomicOr(ep.err, 1u);
                // our copies in flight must land before the CTA's smem is released
                for (int s = 0; s < RING; s++)
                    if (armed & (1u << s)) mbar_wait(&rfull[s], (armed_par >> s) & 1u, WAIT_LIMIT_NS);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ UMMA issuer
        if (elect_one_sync()) {
            const uint32_t idesc = MODE == 0 ? idesc_i8(128, 256) : idesc_tf32(128, 256);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t aphase = 0;
            bool ok = true;
            bool issued = false;
            for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                if (!mbar_wait(&tempty[acc], aphase ^ 1, WAIT_LIMIT_NS)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)acc * 256u;
                for (int kb = 0; kb < num_kb; kb++) {
                    if (!mbar_wait(&full[stage], phase, WAIT_LIMIT_NS)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(sA + stage * A_BYTES);
                    const uint32_t b_addr = smem_u32(sB + stage * B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        if (MODE == 0)
                            umma_i8(d_tmem, sdesc_k_sw128(a_addr + kk * 32), sdesc_k_sw128(b_addr + kk * 32),
                                    idesc, (kb | kk) != 0 ? 1u : 0u);
                        else
                            umma_tf32(d_tmem, sdesc_k_sw128(a_addr + kk * 32), sdesc_k_sw128(b_addr + kk * 32),
                                      idesc, (kb | kk) != 0 ? 1u : 0u);
                    }
                    issued = true;
                    umma_commit(&empty[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                umma_commit(&tfull[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aphase ^= 1;
                }
            }
            if (!ok) atomicOr(ep.err, 2u);
            if (issued) {
                // all of this thread's MMAs complete before TMEM is freed
                umma_commit(drain);
                mbar_wait(drain, 0, WAIT_LIMIT_NS);
            }
        }
    } else if (CW > 0 && warp >= 2 + EW) {
        // ------------------------------------------------ converters (fused form)
        // Thread ct takes 16-individual word wd of the stage's packed rows for
        // records ct / 8 + RPP * i: the warp reads 128 contiguous packed bytes
        // per pass, and each 8-thread phase of a 16-byte store fills one whole
        // 128-byte operand row (no bank conflicts).
        constexpr int RPP = 32 * (CW > 0 ? CW : 1) / 8;   // records per pass
        constexpr int NPASS = (TA + TB) / RPP;
        constexpr int APASS = TA / RPP;              // passes that fill the A tile
        static_assert((TA + TB) % RPP == 0 && TA % RPP == 0, "converter passes");
        const int ct = threadIdx.x - (64 + 32 * EW);
        const int wd = ct & 7;
        uint32_t offP[NPASS], offG[NPASS], offM[NPASS];
#pragma unroll
        for (int i = 0; i < NPASS; i++) {
            const int rr = (ct >> 3) + RPP * i;        // record slot: A 0..63, B 64..191
            const int r = i < APASS ? rr : rr - TA;
            offP[i] = (uint32_t)(rr * 32 + wd * 4);
            offG[i] = sw128_off(2 * r, wd);
            offM[i] = sw128_off(2 * r + 1, wd);
        }
        int os = 0, ps = 0;
        uint32_t oph = 0, pph = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
            // records past the last one read as missing (the map's zero fill would read as genotype 2)
            const Tile tl = tiles[t];
            uint32_t live = 0;
#pragma unroll
            for (int i = 0; i < NPASS; i++) {
                const int rr = (ct >> 3) + RPP * i;
                const int64_t rec = i < APASS ? (int64_t)tl.a_blk * TA + rr : (int64_t)tl.b_blk * TB + (rr - TA);
                live |= (rec < ep.m ? 1u : 0u) << i;
            }
            for (int kb = 0; kb < num_kb; kb++) {
                // every lane waits (TMA data visible to each reader); the warp agrees on the outcome
                const bool got = mbar_wait(&pfull[ps], pph, WAIT_LIMIT_NS) &&
                                 mbar_wait(&empty[os], oph ^ 1, WAIT_LIMIT_NS);
                if (!__all_sync(0xFFFFFFFFu, got)) {
                    if (lane == 0) atomicOr(ep.err, 8u);
                    ok = false;
                    break;
                }
                const uint8_t* pk = sP + ps * P_BYTES;
                uint8_t* oa = sA + os * A_BYTES;
                uint8_t* ob = sB + os * B_BYTES;
                uint32_t w[NPASS];
#pragma unroll
                for (int i = 0; i < NPASS; i++)
                    w[i] = (live >> i) & 1u ? *reinterpret_cast<const uint32_t*>(pk + offP[i]) : 0x55555555u;
                const uint64_t i0 = (uint64_t)kb * 128 + (uint64_t)wd * 16;
                if (i0 + 16 > n_indiv) {
                    // individuals past N (and the zero fill past the row) read as missing
                    const uint32_t valid = n_indiv > i0 ? (uint32_t)(n_indiv - i0) : 0u;
                    const uint32_t keepm = (1u << (2 * valid)) - 1u;   // valid < 16 here
#pragma unroll
                    for (int i = 0; i < NPASS; i++) w[i] = (w[i] & keepm) | (0x55555555u & ~keepm);
                }
#pragma unroll
                for (int i = 0; i < NPASS; i++) {
                    uint4 g, mk;
                    expand_chunk(w[i], g, mk);
                    uint8_t* base = i < APASS ? oa : ob;
                    *reinterpret_cast<uint4*>(base + offG[i]) = g;
                    *reinterpret_cast<uint4*>(base + offM[i]) = mk;
                }
                // the generic-proxy stores must be visible to the tensor core's async proxy
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&full[os]);
                    mbar_arrive(&pempty[ps]);
                }
                if (++os == STAGES) {
                    os = 0;
                    oph ^= 1;
                }
                if (++ps == P_STAGES) {
                    ps = 0;
                    pph ^= 1;
                }
            }
        }
    } else {
        // ------------------------------------------------ epilogue
        constexpr int EPI_T = 32 * EW;                  // epilogue threads
        constexpr int CPW = 4 / (EPI_T / 128);          // 64-column chunks per warp
        const int et = threadIdx.x - 64;         // 0..EPI_T-1
        const int ew = et >> 5;                  // epilogue warp
        const int quarter = warp & 3;            // TMEM lanes this warp may access
        const int c_lo = (ew >> 2) * CPW;        // this warp's first column chunk
        // column partials: one slot per warp with four epilogue warps, per lane quarter with eight
        const int cslot = EPI_T == 128 ? ew : quarter;
        const int row = quarter * 32 + lane;     // accumulator row = A row
        const bool grow = (row & 1) == 0;        // genotype row (else mask row)
        const int64_t m = ep.m;
        int acc = 0;
        uint32_t aphase = 0;
        for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
            const Tile tl = tiles[t];
            const int64_t k0 = (int64_t)tl.a_blk * TA, j0 = (int64_t)tl.b_blk * TB;
            const int64_t k = k0 + (row >> 1);
            const bool kval = k < m;
            const int64_t nk = (MODE == 0 && kval) ? __ldg(ep.n + k) : 0;
            const int64_t sk = (MODE == 0 && kval) ? __ldg(ep.s + k) : 0;
            const double qk = (MODE == 0 && kval) ? __ldg(ep.qinv + k) : 0.0;
            const double ak = (kval && ep.K == 1) ? __ldg(ep.aeff + k) : 0.0;

            // One thread does the bounded wait; the decision is made uniform for
            // all 128 epilogue threads through shared memory before anyone
            // continues, so no thread can be left waiting at a named barrier.
            volatile uint32_t* go = tmem_slot + 1;
            if (et == 0) *go = mbar_wait(&tfull[acc], aphase, WAIT_LIMIT_NS) ? 1u : 0u;
            named_bar_sync(2, EPI_T);
            if (*go == 0u) {
                if (et == 0) atomicOr(ep.err, 4u);
                break;
            }
            tc_fence_after();
            double rsum = 0.0;
            const SketchF cf{(float)ep.n_inv_sq, (float)ep.sketch_d, (float)ep.r2u_a, (float)ep.r2u_b};
            const bool f32_corr = MODE != 0 && ep.sketch_d >= 8.0;
            for (int c = c_lo; c < c_lo + CPW; c++) {
                uint32_t v[64];
                tmem_ld_32x32b_x64(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)acc * 256u +
                                       (uint32_t)c * 64u,
                                   v);
                tmem_ld_wait();
                if (c == c_lo + CPW - 1) {
                    // this thread's part of the accumulator read: hand it back to the MMA warp
                    tc_fence_before();
                    mbar_arrive(&tempty[acc]);
                }
                if (dbg != nullptr && t == 0) {
#pragma unroll
                    for (int q = 0; q < 64; q++) dbg[row * 256 + c * 64 + q] = (int32_t)v[q];
                }
#pragma unroll
                for (int p = 0; p < 32; p += 2) {
                    const int64_t ja = j0 + c * 32 + p, jb = ja + 1;
                    int64_t j;
                    bool valid;
                    double r2u = 0.0;
                    if (MODE == 0) {
                        const int64_t nja = ja < m ? __ldg(ep.n + ja) : 0, sja = ja < m ? __ldg(ep.s + ja) : 0;
                        const int64_t njb = jb < m ? __ldg(ep.n + jb) : 0, sjb = jb < m ? __ldg(ep.s + jb) : 0;
                        const int64_t ga = (int32_t)v[2 * p], ma = (int32_t)v[2 * p + 1];
                        const int64_t gb = (int32_t)v[2 * p + 2], mb = (int32_t)v[2 * p + 3];
                        int64_t Pa, Pb;
                        if (grow) {
                            Pa = nk * (nja * ga - sja * ma);   // n_k n_j GG - n_k s_j GM
                            Pb = nk * (njb * gb - sjb * mb);
                        } else {
                            Pa = sk * (sja * ma - nja * ga);   // s_k s_j MM - s_k n_j MG
                            Pb = sk * (sjb * mb - njb * gb);
                        }
                        const int64_t send = grow ? Pb : Pa;
                        const int64_t recv = shfl_xor_i64(send, 1);
                        const int64_t X = (grow ? Pa : Pb) + recv;
                        j = grow ? ja : jb;
                        valid = kval && pair_in_band(k, j, m, ep.left);
                        if (valid) {
                            const double r = (double)X * qk * __ldg(ep.qinv + j);
                            r2u = r * r * ep.r2u_a + ep.r2u_b;
                        }
                    } else {
                        // this row's (hi or lo)_k times (hi_j + lo_j); the partner lane holds the other half
                        const float pa = __uint_as_float(v[2 * p]) + __uint_as_float(v[2 * p + 1]);
                        const float pb = __uint_as_float(v[2 * p + 2]) + __uint_as_float(v[2 * p + 3]);
                        const float send = grow ? pb : pa;
                        const float recv = __shfl_xor_sync(0xFFFFFFFFu, send, 1);
                        const float val = (grow ? pa : pb) + recv;
                        j = grow ? ja : jb;
                        valid = kval && pair_in_band(k, j, m, ep.left);
                        if (valid)
                            r2u = f32_corr ? (double)sketch_r2u_f32<MODE>(val, k, j, ep, cf)
                                           : sketch_r2u<MODE>(val, k, j, ep);
                    }
                    if (ep.K == 1) {
                        if (valid) rsum += r2u * __ldg(ep.aeff + j);
                        // column j: sum over the 16 same-parity lanes of this warp
                        double cv = r2u * ak;
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 2);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 4);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 8);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 16);
                        if (lane < 2) cpart[cslot * TB + c * 32 + p + lane] = cv;
                    } else {
                        // K > 1: the masked r2u value goes to the tile's f64 slot in
                        // global memory (record k's row of TB values) for the banded
                        // annotation contraction (contract.cu); lane pairs write
                        // adjacent values
                        ep.rtiles[(size_t)t * TA * TB + (size_t)(row >> 1) * TB + c * 32 + p + (grow ? 0 : 1)] = r2u;
                    }
                }
            }
            if (ep.K == 1) {
                rsum += __shfl_xor_sync(0xFFFFFFFFu, rsum, 1);
                if (ep.prow) {
                    // per-tile sums in fixed order; launch_l2_reduce adds them to l2
                    constexpr int G = EPI_T / 128;   // warps per TMEM lane quarter (column groups)
                    if (grow) rpart[(ew >> 2) * TA + (row >> 1)] = rsum;
                    named_bar_sync(1, EPI_T);
                    if (et < TA) {
                        double rs = 0.0;
#pragma unroll
                        for (int g = 0; g < G; g++) rs += rpart[g * TA + et];
                        ep.prow[(size_t)t * TA + et] = rs;
                    }
                    if (et < TB)
                        ep.pcol[(size_t)t * TB + et] = cpart[et] + cpart[TB + et] + cpart[2 * TB + et] + cpart[3 * TB + et];
                } else {
                    if (grow && kval && rsum != 0.0) atomicAdd(ep.l2 + k, rsum);
                    named_bar_sync(1, EPI_T);
                    if (et < TB) {
                        const int64_t j = j0 + et;
                        const double cs = cpart[et] + cpart[TB + et] + cpart[2 * TB + et] + cpart[3 * TB + et];
                        if (j < m && cs != 0.0) atomicAdd(ep.l2 + j, cs);
                    }
                }
                named_bar_sync(1, EPI_T);
            } else {
                // every thread has read this tile's wait decision before the next one is written
                named_bar_sync(1, EPI_T);
            }
            if (++acc == 2) {
                acc = 0;
                aphase ^= 1;
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem_base, 512);
}

}  // namespace

static uint64_t round_up_128(uint64_t x) { return (x + 127) / 128 * 128; }

using PFN_encodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                     const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                     const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                     CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled>(p);
    }
    return fn;
}

static bool make_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, uint64_t ld_elems,
                     uint64_t elem_bytes, uint64_t rows, uint32_t box_rows) {
    PFN_encodeTiled enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {ld_elems, rows};
    cuuint64_t strides[1] = {ld_elems * elem_bytes};
    cuuint32_t box[2] = {(cuuint32_t)(128 / elem_bytes), box_rows};  // 128-byte rows
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int STAGES, int MODE, int EW, int CW = 0>
static cudaError_t run_tc(const CUtensorMap& tmA, const CUtensorMap& tmB, int num_kb, const Tile* tiles,
                          int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg, size_t smem, int64_t grid,
                          cudaStream_t stream, uint64_t n_indiv = 0) {
    cudaError_t e = cudaFuncSetAttribute(k_gram_tc<STAGES, MODE, EW, CW>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_gram_tc<STAGES, MODE, EW, CW><<<(unsigned)grid, gram_threads(EW, CW), smem, stream>>>(
        tmA, tmB, num_kb, tiles, dbg ? 1 : n_tiles, ep, dbg, n_indiv);
    return cudaGetLastError();
}

// barriers (operand ring, packed ring, accumulators, drain) + TMEM slot words
static constexpr size_t ctrl_bytes(int stages) { return 8 * (2 * stages + 2 * P_STAGES + 2 + 2 + 1 + 1); }

template <int MODE>
static cudaError_t launch_tc(const void* ops, CUtensorMapDataType dt, uint64_t elem_bytes, uint64_t ld_elems,
                             int64_t m, const Tile* tiles, int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg,
                             int sms, cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    if ((ld_elems * elem_bytes) % 128 != 0 || (reinterpret_cast<uintptr_t>(ops) & 15) != 0)
        return cudaErrorInvalidValue;
    CUtensorMap tmA, tmB;
    const uint64_t rows = (uint64_t)(2 * m);
    if (!make_map(&tmA, ops, dt, ld_elems, elem_bytes, rows, 2 * TA) ||
        !make_map(&tmB, ops, dt, ld_elems, elem_bytes, rows, 2 * TB))
        return cudaErrorInvalidValue;
    const int num_kb = (int)(ld_elems * elem_bytes / 128);
    const size_t ctrl = ctrl_bytes(4);  // upper bound over the stage counts used
    const size_t cbytes = sizeof(double) * 4 * (TB + TA);   // column and row partials
    int64_t grid = n_tiles < sms ? n_tiles : sms;
    if (dbg) grid = 1;
    // more epilogue warps where the epilogue outweighs the MMAs: sixteen for
    // the sketch forms (the f64 quadratic correction per pair), eight for
    // INT8 rows under 32,768 individuals
    const bool wide = MODE != 0 || ld_elems * elem_bytes < 32768;
    const size_t smem = 1024 + 4 * (size_t)(A_BYTES + B_BYTES) + ctrl + cbytes;
    if constexpr (MODE != 0) {
        return run_tc<4, MODE, 16>(tmA, tmB, num_kb, tiles, n_tiles, ep, dbg, smem, grid, stream);
    } else {
        if (wide) return run_tc<4, MODE, 8>(tmA, tmB, num_kb, tiles, n_tiles, ep, dbg, smem, grid, stream);
        return run_tc<4, MODE, 4>(tmA, tmB, num_kb, tiles, n_tiles, ep, dbg, smem, grid, stream);
    }
}

cudaError_t launch_gram_i8(const uint8_t* ops, uint64_t ld, int64_t m, const Tile* tiles, int64_t n_tiles,
                           const EpilogueArgs& ep, int32_t* dbg, int sms, cudaStream_t stream) {
    return launch_tc<0>(ops, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ld, m, tiles, n_tiles, ep, dbg, sms, stream);
}

// Map of the packed BED rows (record r at rows + r * pitch): boxes of 32 bytes
// (128 individuals) x box_rows records, no swizzle (the converters read it
// with plain shared loads).  Bytes past the pitch read as zero.
static bool make_packed_map(CUtensorMap* map, const uint8_t* rows, uint64_t pitch, uint64_t m, uint32_t box_rows) {
    PFN_encodeTiled enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {pitch, m};
    cuuint64_t strides[1] = {pitch};
    cuuint32_t box[2] = {32, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(rows), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

cudaError_t launch_gram_i8_packed(const uint8_t* rows, uint64_t pitch, uint64_t n_indiv, int64_t m, const Tile* tiles,
                                  int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg, int sms,
                                  cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    if (pitch % 16 != 0 || pitch < (n_indiv + 3) / 4 || n_indiv == 0 ||
        (reinterpret_cast<uintptr_t>(rows) & 15) != 0)
        return cudaErrorInvalidValue;
    CUtensorMap tmA, tmB;
    if (!make_packed_map(&tmA, rows, pitch, (uint64_t)m, TA) || !make_packed_map(&tmB, rows, pitch, (uint64_t)m, TB))
        return cudaErrorInvalidValue;
    const int num_kb = (int)((n_indiv + 127) / 128);
    const size_t cbytes = sizeof(double) * 4 * (TB + TA);   // column and row partials
    const size_t pbytes = (size_t)P_STAGES * P_BYTES;
    int64_t grid = n_tiles < sms ? n_tiles : sms;
    if (dbg) grid = 1;
    const bool wide = round_up_128(n_indiv) < 32768;
    const size_t smem = 1024 + 4 * (size_t)(A_BYTES + B_BYTES) + pbytes + ctrl_bytes(4) + cbytes;
    if (wide)
        return run_tc<4, 0, 8, CONV_WARPS>(tmA, tmB, num_kb, tiles, n_tiles, ep, dbg, smem, grid, stream, n_indiv);
    return run_tc<4, 0, 4, CONV_WARPS_NARROW>(tmA, tmB, num_kb, tiles, n_tiles, ep, dbg, smem, grid, stream,
                                              n_indiv);
}

cudaError_t launch_gram_tf32(const float* ops, uint64_t ld, int64_t m, const Tile* tiles, int64_t n_tiles,
                             const EpilogueArgs& ep, int maf_aware, int32_t* dbg, int sms, cudaStream_t stream) {
    if (maf_aware)
        return launch_tc<2>(ops, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ld, m, tiles, n_tiles, ep, dbg, sms, stream);
    return launch_tc<1>(ops, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ld, m, tiles, n_tiles, ep, dbg, sms, stream);
}

cudaError_t preload_gram_tc() {
    cudaError_t e = preload_kernel(k_gram_tc<4, 0, 4, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_tc<4, 0, 8, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_tc<4, 1, 16, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_tc<4, 2, 16, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_tc<4, 0, 4, CONV_WARPS_NARROW>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_tc<4, 0, 8, CONV_WARPS>);
    return e;
}

}  // namespace ldsc
