// gram_pair.cu -- the INT8-exact band Gram on SM pairs (tcgen05 cta_group::2).
//
// Same arithmetic, operand rows and epilogue as the single-SM form in
// gram_tc.cu (genotype row 2r and non-missing row 2r+1 per record, INT32
// products GG / GM / MG / MM, exact r^2 from integer moments), but a tile is
// 128 left records x 128 right records computed by a cluster of two CTAs on
// two SMs with one 256 x 256 MMA per K-step:
//   * each CTA stages its own half of A (64 left records = 128 rows) and its
//     own half of B (64 right records = 128 rows) by TMA: 32 KB per K-stage
//     instead of the single-SM form's 48 KB, with the leader CTA's barrier
//     counting both CTAs' bytes;
//   * the leader CTA issues tcgen05.mma.cta_group::2 (M = 256 over the pair,
//     N = 256): the B operand is read once for both SMs, so each SM's shared
//     memory serves a third fewer bytes per multiply -- the single-SM Gram is
//     bound by shared-memory bandwidth, not by its tensor pipe;
//   * commits are multicast to both CTAs (stage release, accumulator ready);
//     both CTAs' epilogues release the accumulator on the leader's barrier;
//   * each CTA's epilogue reads its own TMEM half: its 64 left records against
//     all 128 right records, i.e. the single-SM epilogue on the 64 x 128
//     sub-tile 2 t + rank, which keeps the per-tile sums, r2u tiles,
//     reduction and contraction passes of the single-SM form unchanged.
// Every wait is bounded (2 s); on timeout a CTA records an error word, drains
// its own copies / MMAs, and the pair meets at a bounded end-of-kernel
// handshake before TMEM is freed.
#include <cuda.h>
#include <cuda_runtime.h>

#include "engine.h"
#include "epilogue.cuh"
#include "expand.cuh"
#include "sm100.cuh"

namespace ldsc {

namespace {

constexpr int TA = 64;              // left records per CTA (sub-tile rows / 2)
constexpr int TB = 128;             // right records per tile (all of them in each CTA's accumulator)
constexpr int STAGE_A = 128 * 128;  // this CTA's A half: 128 rows x 128 B
constexpr int STAGE_B = 128 * 128;  // this CTA's B half: 128 rows x 128 B
constexpr int STAGES = 6;
// fused form: packed ring of 2-bit rows, 128 individuals (32 bytes) per record per stage
constexpr int P_STAGES = 4;
constexpr int PA_BYTES = TA * 32;          // this CTA's 64 left records
constexpr int P_BYTES = 2 * TA * 32;       // + its 64 right records
constexpr int CONV_WARPS = 4;
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;

// threads per CTA: TMA and MMA warps + ew epilogue warps + cw converter warps
__host__ __device__ constexpr int pair_threads(int ew, int cw) { return 64 + 32 * ew + 32 * cw; }

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ void remote_arrive(uint32_t cluster_bar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}

// Bounded wait with cluster-scope acquire: the arrivals it waits for come from the other CTA.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t"
            ".reg .pred P;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// 2D tiled load into this CTA's shared memory whose completion bytes count on
// the leader CTA's barrier (a shared::cluster address).
__device__ __forceinline__ void tma_load_2d_pair(void* smem_dst, const void* tmap, uint32_t leader_bar, int32_t x,
                                                 int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(leader_bar)
        : "memory");
}

__device__ __forceinline__ void umma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive once on `bar` (same offset) in both CTAs when this thread's MMAs complete.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
    const uint16_t mask = 3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(mask)
        : "memory");
}

__device__ __forceinline__ int64_t shfl_xor_i64(int64_t v, int mask) {
    int lo = (int)(v & 0xFFFFFFFF), hi = (int)(v >> 32);
    lo = __shfl_xor_sync(0xFFFFFFFFu, lo, mask);
    hi = __shfl_xor_sync(0xFFFFFFFFu, hi, mask);
    return ((int64_t)hi << 32) | (uint32_t)lo;
}

// Warps: 0 TMA producer (both CTAs), 1 TMEM allocator (both) and MMA issuer
// (leader), 2 .. 2 + EW - 1 epilogue (both), then CW converter warps (both,
// fused form).  tiles: 128 x 128 band tiles (a_blk in units of 128 left
// records).
// Staged form (CW = 0): warp 0 loads this CTA's operand-row halves by TMA,
// the bytes counted on the leader's full barrier.
// Fused form (CW > 0): warp 0 loads this CTA's 64 + 64 packed 2-bit rows
// (4 KB per stage) into a local ring; the converter warps expand them into
// this CTA's operand halves (as in gram_tc.cu's fused form) and arrive on the
// leader's full barrier, 2 CW arrivals per stage over the pair.
template <int EW, int CW>
__global__ void __launch_bounds__(pair_threads(EW, CW), 1)
    k_gram_pair(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int num_kb,
                const Tile* __restrict__ tiles, int64_t n_tiles, EpilogueArgs ep, int32_t* __restrict__ dbg,
                uint64_t n_indiv) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    uint8_t* smem = smem_raw + pad;
    uint8_t* sA = smem;
    uint8_t* sB = sA + STAGES * STAGE_A;
    uint8_t* sP = sB + STAGES * STAGE_B;                                       // fused: packed ring
    uint64_t* full = reinterpret_cast<uint64_t*>(sP + (CW > 0 ? P_STAGES * P_BYTES : 0));  // leader's count both CTAs
    uint64_t* empty = full + STAGES;                                      // [STAGES], one multicast commit each
    uint64_t* pfull = empty + STAGES;                                     // [P_STAGES], fused only
    uint64_t* pempty = pfull + P_STAGES;                                  // [P_STAGES], fused only
    uint64_t* tfull = pempty + P_STAGES;                                  // [2]
    uint64_t* tempty = tfull + 2;                                         // [2], leader's: both epilogues
    uint64_t* drain = tempty + 2;                                         // [1]
    uint64_t* done = drain + 1;                                           // [1], end-of-kernel handshake
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);          // [0] TMEM base, [1] wait decision
    double* cpart = reinterpret_cast<double*>(done + 2);                  // [4][TB]
    double* rpart = cpart + 4 * TB;                                       // [4][TA]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int64_t npairs = gridDim.x / 2;
    const int64_t pair_id = blockIdx.x / 2;
    constexpr int EPI_T = 32 * EW;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], CW > 0 ? 2 * CW : 1);   // TMA bytes of both CTAs, or both CTAs' converter warps
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < P_STAGES; s++) {
            mbar_init(&pfull[s], 1);
            mbar_init(&pempty[s], CW > 0 ? CW : 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * EPI_T);
        }
        mbar_init(drain, 1);
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    // both CTAs' barriers are initialised before either touches the other's
    cluster_sync_all();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t leader_full0 = peer_addr(&full[0], 0);

    if (warp == 0) {
        // ------------------------------------------------ TMA producer (both CTAs)
        if (elect_one_sync()) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            uint32_t armed = 0;        // fused: bit s = packed stage s has a load in flight
            uint32_t armed_par = 0;    // fused: parity of that load's phase
            constexpr int RING = CW > 0 ? P_STAGES : STAGES;
            uint64_t* rempty = CW > 0 ? pempty : empty;
            for (int64_t t = pair_id; t < n_tiles && ok; t += npairs) {
                const Tile tl = tiles[t];
                // this CTA's 64 left and 64 right records: 128 operand rows, or 64 packed rows, each
                const int32_t ra = ((int32_t)tl.a_blk * 2 + (int32_t)rank) * TA;
                const int32_t rb = (int32_t)tl.b_blk * TB + (int32_t)rank * TA;
                for (int kb = 0; kb < num_kb; kb++) {
                    if (!mbar_wait(&rempty[stage], phase ^ 1, WAIT_LIMIT_NS)) {
                        ok = false;
                        break;
                    }
                    if constexpr (CW > 0) {
                        mbar_arrive_expect_tx(&pfull[stage], P_BYTES);
                        tma_load_2d(sP + stage * P_BYTES, &tmA, &pfull[stage], kb * 32, ra);
                        tma_load_2d(sP + stage * P_BYTES + PA_BYTES, &tmB, &pfull[stage], kb * 32, rb);
                        armed |= 1u << stage;
                        armed_par = (armed_par & ~(1u << stage)) | (phase << stage);
                    } else {
                        if (leader) mbar_arrive_expect_tx(&full[stage], 2 * (STAGE_A + STAGE_B));
                        const uint32_t fb = leader_full0 + (uint32_t)stage * 8u;
                        tma_load_2d_pair(sA + stage * STAGE_A, &tmA, fb, kb * 128, 2 * ra);
                        tma_load_2d_pair(sB + stage * STAGE_B, &tmB, fb, kb * 128, 2 * rb);
                    }
                    if (++stage == RING) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (!ok) {
                atomicOr(ep.err, 1u);
                // fused: this CTA's packed copies in flight land before its shared memory is released
                if constexpr (CW > 0)
                    for (int s = 0; s < RING; s++)
                        if (armed & (1u << s)) mbar_wait(&pfull[s], (armed_par >> s) & 1u, WAIT_LIMIT_NS);
            }
            // staged: every operand copy is consumed by an MMA, and the leader's
            // drain of every MMA precedes the end-of-kernel handshake
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer (leader)
        if (leader && elect_one_sync()) {
            const uint32_t idesc = idesc_i8(256, 256);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t aphase = 0;
            bool ok = true;
            bool issued = false;
            for (int64_t t = pair_id; t < n_tiles && ok; t += npairs) {
                if (!mbar_wait_cluster(&tempty[acc], aphase ^ 1, WAIT_LIMIT_NS)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)acc * 256u;
                for (int kb = 0; kb < num_kb; kb++) {
                    if (!mbar_wait_cluster(&full[stage], phase, WAIT_LIMIT_NS)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(sA + stage * STAGE_A);
                    const uint32_t b_addr = smem_u32(sB + stage * STAGE_B);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                        umma_i8_pair(d_tmem, sdesc_k_sw128(a_addr + kk * 32), sdesc_k_sw128(b_addr + kk * 32), idesc,
                                     (kb | kk) != 0 ? 1u : 0u);
                    issued = true;
                    umma_commit_pair(&empty[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                umma_commit_pair(&tfull[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aphase ^= 1;
                }
            }
            if (!ok) atomicOr(ep.err, 2u);
            if (issued) {
                // every MMA of the pair completes before shared memory or TMEM is released
                asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(drain))
                             : "memory");
                if (!mbar_wait(drain, 0, WAIT_LIMIT_NS)) atomicOr(ep.err, 32u);
            }
        }
    } else if (CW > 0 && warp >= 2 + EW) {
        // ------------------------------------------------ converters (fused form, both CTAs)
        // Thread ct takes 16-individual word wd of the stage's packed rows for
        // records ct / 8 + RPP * i (A slots 0..63, B slots 64..127): the warp
        // reads 128 contiguous packed bytes per pass, and each 8-thread phase of
        // a 16-byte store fills one whole 128-byte operand row.
        constexpr int RPP = 32 * (CW > 0 ? CW : 1) / 8;   // records per pass
        constexpr int NPASS = 2 * TA / RPP;
        constexpr int APASS = TA / RPP;
        static_assert(TA % RPP == 0, "converter passes");
        const int ct = threadIdx.x - (64 + 32 * EW);
        const int wd = ct & 7;
        uint32_t offP[NPASS], offG[NPASS], offM[NPASS];
#pragma unroll
        for (int i = 0; i < NPASS; i++) {
            const int rr = (ct >> 3) + RPP * i;
            const int r = i < APASS ? rr : rr - TA;
            offP[i] = (uint32_t)(rr * 32 + wd * 4);
            offG[i] = sw128_off(2 * r, wd);
            offM[i] = sw128_off(2 * r + 1, wd);
        }
        int os = 0, ps = 0;
        uint32_t oph = 0, pph = 0;
        bool ok = true;
        for (int64_t t = pair_id; t < n_tiles && ok; t += npairs) {
            // records past the last one read as missing (the map's zero fill would read as genotype 2)
            const Tile tl = tiles[t];
            const int64_t ra = ((int64_t)tl.a_blk * 2 + rank) * TA, rb = (int64_t)tl.b_blk * TB + (int64_t)rank * TA;
            uint32_t live = 0;
#pragma unroll
            for (int i = 0; i < NPASS; i++) {
                const int rr = (ct >> 3) + RPP * i;
                const int64_t rec = i < APASS ? ra + rr : rb + (rr - TA);
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
                uint8_t* oa = sA + os * STAGE_A;
                uint8_t* ob = sB + os * STAGE_B;
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
                    remote_arrive(leader_full0 + (uint32_t)os * 8u);
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
        // ------------------------------------------------ epilogue (both CTAs)
        constexpr int CPW = 4 / (EPI_T / 128);   // 64-column chunks per warp
        const int et = threadIdx.x - 64;
        const int ew = et >> 5;
        const int quarter = warp & 3;
        const int c_lo = (ew >> 2) * CPW;
        const int cslot = EPI_T == 128 ? ew : quarter;
        const int row = quarter * 32 + lane;     // accumulator row of this CTA's half of A
        const bool grow = (row & 1) == 0;
        const int64_t m = ep.m;
        const uint32_t leader_tempty0 = peer_addr(&tempty[0], 0);
        int acc = 0;
        uint32_t aphase = 0;
        for (int64_t t = pair_id; t < n_tiles; t += npairs) {
            const Tile tl = tiles[t];
            const int64_t sub = 2 * t + rank;    // this CTA's 64 x 128 sub-tile
            const int64_t k0 = ((int64_t)tl.a_blk * 2 + rank) * TA, j0 = (int64_t)tl.b_blk * TB;
            const int64_t k = k0 + (row >> 1);
            const bool kval = k < m;
            const int64_t nk = kval ? __ldg(ep.n + k) : 0;
            const int64_t sk = kval ? __ldg(ep.s + k) : 0;
            const double qk = kval ? __ldg(ep.qinv + k) : 0.0;
            const double ak = (kval && ep.K == 1) ? __ldg(ep.aeff + k) : 0.0;

            volatile uint32_t* go = tmem_slot + 1;
            if (et == 0) *go = mbar_wait(&tfull[acc], aphase, WAIT_LIMIT_NS) ? 1u : 0u;
            named_bar_sync(2, EPI_T);
            if (*go == 0u) {
                if (et == 0) atomicOr(ep.err, 4u);
                break;
            }
            tc_fence_after();
            double rsum = 0.0;
            for (int c = c_lo; c < c_lo + CPW; c++) {
                uint32_t v[64];
                tmem_ld_32x32b_x64(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)acc * 256u +
                                       (uint32_t)c * 64u,
                                   v);
                tmem_ld_wait();
                if (c == c_lo + CPW - 1) {
                    // this thread's part of the accumulator is read: release it on the leader
                    tc_fence_before();
                    remote_arrive(leader_tempty0 + (uint32_t)acc * 8u);
                }
                if (dbg != nullptr && t == 0) {
#pragma unroll
                    for (int q = 0; q < 64; q++) dbg[(size_t)rank * 128 * 256 + row * 256 + c * 64 + q] = (int32_t)v[q];
                }
#pragma unroll
                for (int p = 0; p < 32; p += 2) {
                    const int64_t ja = j0 + c * 32 + p, jb = ja + 1;
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
                    const int64_t j = grow ? ja : jb;
                    const bool valid = kval && pair_in_band(k, j, m, ep.left);
                    double r2u = 0.0;
                    if (valid) {
                        const double r = (double)X * qk * __ldg(ep.qinv + j);
                        r2u = r * r * ep.r2u_a + ep.r2u_b;
                    }
                    if (ep.K == 1) {
                        if (valid) rsum += r2u * __ldg(ep.aeff + j);
                        double cv = r2u * ak;
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 2);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 4);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 8);
                        cv += __shfl_xor_sync(0xFFFFFFFFu, cv, 16);
                        if (lane < 2) cpart[cslot * TB + c * 32 + p + lane] = cv;
                    } else {
                        ep.rtiles[(size_t)sub * TA * TB + (size_t)(row >> 1) * TB + c * 32 + p + (grow ? 0 : 1)] = r2u;
                    }
                }
            }
            if (ep.K == 1) {
                rsum += __shfl_xor_sync(0xFFFFFFFFu, rsum, 1);
                if (ep.prow) {
                    // per-sub-tile sums in fixed order; launch_l2_reduce adds them to l2
                    constexpr int G = EPI_T / 128;
                    if (grow) rpart[(ew >> 2) * TA + (row >> 1)] = rsum;
                    named_bar_sync(1, EPI_T);
                    if (et < TA) {
                        double rs = 0.0;
#pragma unroll
                        for (int g = 0; g < G; g++) rs += rpart[g * TA + et];
                        ep.prow[(size_t)sub * TA + et] = rs;
                    }
                    if (et < TB)
                        ep.pcol[(size_t)sub * TB + et] =
                            cpart[et] + cpart[TB + et] + cpart[2 * TB + et] + cpart[3 * TB + et];
                } else {
                    if (grow && kval && rsum != 0.0) atomicAdd(ep.l2 + k, rsum);
                    named_bar_sync(1, EPI_T);
                    if (et < TB) {
                        const int64_t j = j0 + et;
                        const double cs = cpart[et] + cpart[TB + et] + cpart[2 * TB + et] + cpart[3 * TB + et];
                        if (j < m && cs != 0.0) atomicAdd(ep.l2 + j, cs);
                    }
                }
            }
            // every thread has read this tile's wait decision and partials before they are rewritten
            named_bar_sync(1, EPI_T);
            if (++acc == 2) {
                acc = 0;
                aphase ^= 1;
            }
        }
    }

    // End of kernel: the peer's shared memory and TMEM stay alive until the
    // leader's MMAs have drained (bounded handshake: each CTA arrives on the
    // other's `done` barrier and waits for its own).
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        remote_arrive(peer_addr(done, rank ^ 1u));
        if (!mbar_wait_cluster(done, 0, WAIT_LIMIT_NS)) atomicOr(ep.err, 16u);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512) : "memory");
}

using PFN_encodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                     const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

PFN_encodeTiled get_encode_pair() {
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

// rows of `width` bytes, `stride` apart: boxes of box_w bytes x box_rows rows
bool make_pair_map(CUtensorMap* map, const uint8_t* base, uint64_t width, uint64_t stride, uint64_t rows,
                   uint32_t box_w, uint32_t box_rows, CUtensorMapSwizzle swz) {
    PFN_encodeTiled enc = get_encode_pair();
    if (!enc) return false;
    cuuint64_t dims[2] = {width, rows};
    cuuint64_t strides[1] = {stride};
    cuuint32_t box[2] = {box_w, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int EW, int CW>
cudaError_t run_pair(const CUtensorMap& tmA, const CUtensorMap& tmB, int num_kb, const Tile* tiles, int64_t n_tiles,
                     const EpilogueArgs& ep, int32_t* dbg, int64_t pairs, uint64_t n_indiv, cudaStream_t stream) {
    const size_t ctrl = 8 * (2 * STAGES + 2 * P_STAGES + 2 + 2 + 1 + 1 + 1);
    const size_t smem = 1024 + (size_t)STAGES * (STAGE_A + STAGE_B) + (CW > 0 ? (size_t)P_STAGES * P_BYTES : 0) +
                        ctrl + sizeof(double) * 4 * (TB + TA);
    cudaError_t e = cudaFuncSetAttribute(k_gram_pair<EW, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * pairs), 1, 1);
    cfg.blockDim = dim3(pair_threads(EW, CW), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // persistent: no more pairs than can be resident at once (a GPC with an
    // odd number of free SMs leaves one of them out)
    int resident = 0;
    if (cudaOccupancyMaxActiveClusters(&resident, k_gram_pair<EW, CW>, &cfg) == cudaSuccess && resident > 0 &&
        resident < pairs)
        cfg.gridDim = dim3((unsigned)(2 * resident), 1, 1);
    cudaGetLastError();
    e = cudaLaunchKernelEx(&cfg, k_gram_pair<EW, CW>, tmA, tmB, num_kb, tiles, dbg ? (int64_t)1 : n_tiles, ep, dbg,
                           n_indiv);
    return e != cudaSuccess ? e : cudaGetLastError();
}

int64_t pair_grid(int64_t n_tiles, int sms, int32_t* dbg) {
    if (dbg) return 1;
    return n_tiles < sms / 2 ? n_tiles : sms / 2;
}

}  // namespace

cudaError_t launch_gram_i8_pair(const uint8_t* ops, uint64_t ld, int64_t m, const Tile* tiles, int64_t n_tiles,
                                const EpilogueArgs& ep, int32_t* dbg, int sms, cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    if (ld % 128 != 0 || (reinterpret_cast<uintptr_t>(ops) & 15) != 0) return cudaErrorInvalidValue;
    // operand rows (2 per record, `ld` bytes): boxes of 128 bytes x 128 rows, 128-byte swizzle
    CUtensorMap tm;
    if (!make_pair_map(&tm, ops, ld, ld, (uint64_t)(2 * m), 128, 128, CU_TENSOR_MAP_SWIZZLE_128B))
        return cudaErrorInvalidValue;
    const int num_kb = (int)(ld / 128);
    const int64_t pairs = pair_grid(n_tiles, sms, dbg);
    if (ld < 32768) return run_pair<8, 0>(tm, tm, num_kb, tiles, n_tiles, ep, dbg, pairs, 0, stream);
    return run_pair<4, 0>(tm, tm, num_kb, tiles, n_tiles, ep, dbg, pairs, 0, stream);
}

cudaError_t launch_gram_i8_pair_packed(const uint8_t* rows, uint64_t pitch, uint64_t n_indiv, int64_t m,
                                       const Tile* tiles, int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg,
                                       int sms, cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    if (pitch % 16 != 0 || pitch < (n_indiv + 3) / 4 || n_indiv == 0 ||
        (reinterpret_cast<uintptr_t>(rows) & 15) != 0)
        return cudaErrorInvalidValue;
    // packed rows (one per record): boxes of 32 bytes (128 individuals) x 64 records, no swizzle;
    // bytes past the pitch read as zero
    CUtensorMap tm;
    if (!make_pair_map(&tm, rows, pitch, pitch, (uint64_t)m, 32, TA, CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorInvalidValue;
    const int num_kb = (int)((n_indiv + 127) / 128);
    const int64_t pairs = pair_grid(n_tiles, sms, dbg);
    if ((n_indiv + 127) / 128 * 128 < 32768)
        return run_pair<8, CONV_WARPS>(tm, tm, num_kb, tiles, n_tiles, ep, dbg, pairs, n_indiv, stream);
    return run_pair<4, CONV_WARPS>(tm, tm, num_kb, tiles, n_tiles, ep, dbg, pairs, n_indiv, stream);
}

cudaError_t preload_gram_pair() {
    cudaError_t e = preload_kernel(k_gram_pair<4, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_pair<8, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_pair<4, CONV_WARPS>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_pair<8, CONV_WARPS>);
    return e;
}

}  // namespace ldsc
