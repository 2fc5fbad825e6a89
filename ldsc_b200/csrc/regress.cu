// regress.cu -- batched LD-score regressions (h2 and genetic covariance) on
// device-resident LD scores: weights, two IRWLS re-weightings, block
// jackknife.  Restates the reference's
//   ldsc_weights / aggregate / irwls_ldsc / jackknife_fast   (src/h2.rs:100-458)
//   jackknife_se_cov                                          (src/jackknife.rs:10-59)
//   gencov_weights / run_hsq_ldsc / run_gencov_ldsc           (src/regressions.rs:1612-2052)
// for the one-LD-score-column case (K = 1), many traits at once.
//
// Every per-SNP pass is one kernel over (jackknife block, job): a warp sums
// its block's contributions in f64, and per-job kernels combine the blocks in
// a fixed order, so results do not depend on scheduling.  The weighted least
// squares uses the 2 x 2 normal equations of the reference's weighted design
// (the reference solves the same system by QR); the weights' global scale
// 1/sum(w) cancels in every solve.
#include <cuda_runtime.h>

#include <cmath>

#include "engine.h"
#include "regress.h"

namespace ldsc {

namespace {

constexpr int NT = 256;

__device__ __forceinline__ double job_y(const RegJob& jb, uint64_t i) {
    const double a = jb.ya[i];
    if (jb.ymode == REG_Y_SQUARE) return fmax(a * a, 0.0);
    if (jb.ymode == REG_Y_PRODUCT) return a * jb.yb[i];
    return a;
}

// Per-job constants of the weights, formed once per pass.
struct WeightConsts {
    double inv_nbar;  // 1 / nbar
    double hm;        // REG_HSQ: clamp(hsq, 0, 1) / M
    double h1m, h2m;  // REG_GENCOV: clamp(h1, 0, 1) / M, clamp(h2, 0, 1) / M
    double sm;        // REG_GENCOV: rho_g / M
};

__device__ __forceinline__ WeightConsts weight_consts(const RegState& st, double m) {
    WeightConsts k;
    k.inv_nbar = 1.0 / st.nbar;
    k.hm = fmin(fmax(st.slope, 0.0), 1.0) / m;
    k.h1m = fmin(fmax(st.h1, 0.0), 1.0) / m;
    k.h2m = fmin(fmax(st.h2, 0.0), 1.0) / m;
    k.sm = st.slope / m;
    return k;
}

// Regression weight of SNP i under the job's current parameters (the square
// of the reference's w): ldsc_weights (src/h2.rs:185-206) or gencov_weights
// (src/regressions.rs:1612-1645).  The reference's two reciprocals (of the
// heteroskedasticity term and of the overcounting LD score) are taken as one.
template <int KIND>
__device__ __forceinline__ double job_weight(const RegJob& jb, const RegState& st, const WeightConsts& k,
                                             double ld_raw, double wld_raw, double n1, double n2) {
    const double ocd = fmax(wld_raw, 1.0);
    if (KIND == REG_HSQ) {
        // step 1 of --two-step re-weights with the regressor in place of the LD
        // score (src/h2.rs:347-351: ldsc_weights(x1_col0, ...))
        const double ld = jb.ld_from_x && st.n_updates > 0 ? fmax(n1 * ld_raw * k.inv_nbar, 1.0) : fmax(ld_raw, 1.0);
        const double t = st.intercept + k.hm * n1 * ld;
        return 1.0 / (2.0 * t * t * ocd);
    }
    const double ld = fmax(ld_raw, 1.0);
    const double a = n1 * k.h1m * ld + st.int_h1;
    const double b = n2 * k.h2m * ld + st.int_h2;
    const double c = sqrt(n1 * n2) * k.sm * ld + st.intercept;
    return 1.0 / ((a * b + c * c) * ocd);
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; w++) t += red[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ uint64_t sep(uint64_t n, int nb, int b) {
    // get_separators (src/h2.rs:31-41): floor(b * n / nb), last = n
    if (b >= nb) return n;
    return (uint64_t)floor((double)b * (double)n / (double)nb);
}

// Per (jackknife block, job) sums.  MODE 0: sum y, sum ld*Nx, sum Nx.
// MODE 1: with w = job weight and x0 = Nx*ld/nbar:
//   sum w x0^2, sum w x0, sum w, sum w x0 y, sum w y.
// One warp per (block, job), RJ jobs of the same block per CTA (their LD
// scores are the same rows, read once into L1); each lane sums every 32nd SNP
// of the block, RU loads in flight, then a warp reduction.  No block
// barriers, and the order of the sums depends only on the block's bounds.
constexpr int RJ = 8;  // jobs per CTA
constexpr int RU = 4;  // SNPs per lane whose loads are issued together

template <int MODE, int KIND>
__device__ __forceinline__ void reg_term(const RegJob& jb, const RegState& st, const WeightConsts& k, double y,
                                         double l, double wl, double n1, double n2, double* s) {
    if (MODE == 1 && jb.use_mask && !(y < jb.mask_max)) return;
    // sample size that scales the regressor: N (h2) or sqrt(N1 N2) (gencov)
    const double nx = KIND == REG_HSQ ? n1 : sqrt(n1 * n2);
    if (MODE == 0) {
        s[0] += y;
        s[1] += l * nx;
        s[2] += nx;
    } else {
        const double w = job_weight<KIND>(jb, st, k, l, wl, n1, n2);
        const double x0 = nx * l * k.inv_nbar;
        s[0] += w * x0 * x0;
        s[1] += w * x0;
        s[2] += w;
        s[3] += w * x0 * y;
        s[4] += w * y;
    }
}

// Kind and y of every job of a launch (FORM = REG_FORM_*).
__host__ __device__ constexpr int form_kind(int f) { return f == REG_FORM_GENCOV_PRODUCT ? REG_GENCOV : REG_HSQ; }
__host__ __device__ constexpr int form_ymode(int f) {
    return f == REG_FORM_HSQ_DIRECT ? REG_Y_DIRECT : (f == REG_FORM_HSQ_SQUARE ? REG_Y_SQUARE : REG_Y_PRODUCT);
}

// FORM: the kind and y of every job of the launch (a job of another form gets
// NaN sums).  The job's arrays are offset to its block once, so the per-SNP
// indexing is 32-bit and the y form is fixed at compile time.
template <int MODE, int FORM>
__global__ void __launch_bounds__(RJ * 32, form_kind(FORM) == REG_HSQ ? 3 : 1)
    k_reg_sums(const RegJob* __restrict__ jobs, const RegState* __restrict__ states, const double* __restrict__ ld,
               const double* __restrict__ wld, uint64_t n, int nb, double m, int njobs, double* __restrict__ part) {
    constexpr int KIND = form_kind(FORM), YM = form_ymode(FORM);
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x, j = blockIdx.y * RJ + (threadIdx.x >> 5);
    if (j >= njobs) return;
    const RegJob jb = jobs[j];
    const RegState st = states[j];
    const uint64_t lo = jb.seps ? (uint64_t)jb.seps[b] : sep(n, nb, b);
    const uint64_t hi = jb.seps ? (uint64_t)jb.seps[b + 1] : sep(n, nb, b + 1);
    const uint32_t cnt = (uint32_t)(hi - lo);  // n < 2^31 (checked by the launcher)
    const double* __restrict__ ya = jb.ya + lo;
    const double* __restrict__ yb = YM == REG_Y_PRODUCT ? jb.yb + lo : nullptr;
    const double* __restrict__ n1p = jb.n1 ? jb.n1 + lo : nullptr;
    const double* __restrict__ n2p = (KIND == REG_GENCOV && jb.n2) ? jb.n2 + lo : nullptr;
    const double* __restrict__ lb = ld + lo;
    const double* __restrict__ wb = wld + lo;
    const WeightConsts k = weight_consts(st, m);
    double s[5] = {0, 0, 0, 0, 0};
    // lane l takes SNPs lo + l, lo + l + 32, ... in that order; RU of them per
    // step have their loads in flight together
    for (uint32_t k0 = lane; k0 < cnt; k0 += 32 * RU) {
        double y[RU], l[RU], wl[RU], n1[RU], n2[RU];
#pragma unroll
        for (int u = 0; u < RU; u++) {
            const uint32_t q = k0 + 32 * u;
            const bool v = q < cnt;
            double a = v ? ya[q] : 0.0;
            if (YM == REG_Y_SQUARE) a = fmax(a * a, 0.0);
            if (YM == REG_Y_PRODUCT) a *= v ? yb[q] : 0.0;
            y[u] = a;
            l[u] = v ? lb[q] : 0.0;
            wl[u] = (MODE == 1 && v) ? wb[q] : 1.0;
            n1[u] = (n1p && v) ? n1p[q] : jb.n1s;
            n2[u] = KIND == REG_GENCOV ? ((n2p && v) ? n2p[q] : jb.n2s) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < RU; u++)
            if (k0 + 32 * u < cnt) reg_term<MODE, KIND>(jb, st, k, y[u], l[u], wl[u], n1[u], n2[u], s);
    }
    if (jb.kind != KIND || jb.ymode != YM)
#pragma unroll
        for (int q = 0; q < 5; q++) s[q] = NAN;
    constexpr int NQ = MODE == 0 ? 3 : 5;
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xFFFFFFFFu, s[q], o);
    if (lane == 0) {
        double* out = part + ((size_t)j * nb + b) * 5;
#pragma unroll
        for (int q = 0; q < NQ; q++) out[q] = s[q];
    }
}

// 2 x 2 (or 1 x 1 with a fixed intercept) normal equations from the five sums.
__device__ __forceinline__ void wls_solve(const double* S, const RegJob& jb, double fixed_int, double* coef) {
    if (jb.fixed) {
        coef[0] = (S[3] - fixed_int * S[1]) / S[0];
        coef[1] = fixed_int;
        return;
    }
    const double a = S[0], b = S[1], c = S[2], d = S[3], e = S[4];
    const double det = a * c - b * b;
    coef[0] = (c * d - b * e) / det;
    coef[1] = (a * e - b * d) / det;
}

// MODE 0: initialise from the aggregate pass (src/h2.rs:208-218, :266-268).
// MODE 1: one IRWLS update: solve, then set the weights' parameters.
template <int MODE>
__global__ void k_reg_update(const RegJob* __restrict__ jobs, RegState* __restrict__ states,
                             const RegOut* __restrict__ ref_outs, const double* __restrict__ part, uint64_t n, int nb,
                             double m, int njobs) {
    // one warp per job: lane l sums blocks l, l + 32, ..., then a fixed-order
    // warp reduction
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= njobs) return;
    constexpr int NQ = MODE == 0 ? 3 : 5;
    double S[5] = {0, 0, 0, 0, 0};
    for (int b = lane; b < nb; b += 32)
#pragma unroll
        for (int q = 0; q < NQ; q++) S[q] += part[((size_t)j * nb + b) * 5 + q];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) S[q] += __shfl_xor_sync(0xFFFFFFFFu, S[q], o);
    if (lane) return;
    const RegJob jb = jobs[j];
    RegState st = states[j];
    if (MODE == 0) {
        const double nn = (double)n;
        st.mean_y = S[0] / nn;
        st.nbar = S[2] / nn;
        // --two-step's second fit starts from the unconstrained initial weights
        // (intercept 1) and solves with step 1's intercept held fixed
        const bool from_step1 = jb.int_from >= 0;
        const double int0 = jb.fixed && !from_step1 ? jb.fixed_int : (jb.kind == REG_HSQ ? 1.0 : 0.0);
        st.slope = m * (st.mean_y - int0) / (S[1] / nn);  // aggregate
        st.intercept = int0;
        st.fixed_int = from_step1 ? ref_outs[jb.int_from].est[1] : jb.fixed_int;
        st.n_updates = 0;
        st.c_num = st.c_den = 0.0;
        if (jb.kind == REG_GENCOV) {
            const RegOut& o1 = ref_outs[jb.hsq1];
            const RegOut& o2 = ref_outs[jb.hsq2];
            st.h1 = o1.tot;
            st.h2 = o2.tot;
            st.int_h1 = o1.intercept;
            st.int_h2 = o2.intercept;
        }
    } else {
        if (st.n_updates == 0) {  // the first least squares runs on the initial weights
            st.c_num = S[1];
            st.c_den = S[0];
        }
        double coef[2];
        wls_solve(S, jb, st.fixed_int, coef);
        st.slope = m * coef[0] / st.nbar;
        st.intercept = coef[1];
        st.n_updates++;
    }
    states[j] = st;
}

// Block jackknife (jackknife_fast + jackknife_se_cov) on the final weights'
// per-block sums; one CTA per job, one thread per block.
__global__ void __launch_bounds__(NT) k_reg_jackknife(const RegJob* __restrict__ jobs, const RegState* __restrict__ states,
                                                      RegOut* __restrict__ outs, const double* __restrict__ part,
                                                      int nb, double m, double* __restrict__ tot_delete,
                                                      double* __restrict__ dv) {
    __shared__ double tot[5];
    __shared__ double red[NT / 32];
    const int j = blockIdx.x;
    const RegJob jb = jobs[j];
    const RegState st = states[j];
    const double* P = part + (size_t)j * nb * 5;
    if (threadIdx.x < 5) {
        double t = 0.0;
        for (int b = 0; b < nb; b++) t += P[b * 5 + threadIdx.x];
        tot[threadIdx.x] = t;
    }
    __syncthreads();
    double est[2];
    wls_solve(tot, jb, st.fixed_int, est);
    const int p = jb.fixed ? 1 : 2;
    // delete values and pseudovalues; threads loop over blocks
    double sp0 = 0, sp1 = 0;
    for (int b = threadIdx.x; b < nb; b += NT) {
        double Sd[5], del[2];
        for (int q = 0; q < 5; q++) Sd[q] = tot[q] - P[b * 5 + q];
        wls_solve(Sd, jb, st.fixed_int, del);
        if (tot_delete) tot_delete[(size_t)j * nb + b] = m * del[0] / st.nbar;
        if (dv) {
            dv[((size_t)j * nb + b) * 2] = del[0];
            dv[((size_t)j * nb + b) * 2 + 1] = del[1];
        }
        sp0 += (double)nb * est[0] - (double)(nb - 1) * del[0];
        sp1 += (double)nb * est[1] - (double)(nb - 1) * del[1];
    }
    const double mean0 = block_sum(sp0, red) / nb;
    const double mean1 = block_sum(sp1, red) / nb;
    __shared__ double s_mean[2];
    if (threadIdx.x == 0) {
        s_mean[0] = mean0;
        s_mean[1] = mean1;
    }
    __syncthreads();
    double c00 = 0, c01 = 0, c11 = 0;
    for (int b = threadIdx.x; b < nb; b += NT) {
        double Sd[5], del[2];
        for (int q = 0; q < 5; q++) Sd[q] = tot[q] - P[b * 5 + q];
        wls_solve(Sd, jb, st.fixed_int, del);
        const double d0 = (double)nb * est[0] - (double)(nb - 1) * del[0] - s_mean[0];
        const double d1 = (double)nb * est[1] - (double)(nb - 1) * del[1] - s_mean[1];
        c00 += d0 * d0;
        c01 += d0 * d1;
        c11 += d1 * d1;
    }
    c00 = block_sum(c00, red);
    c01 = block_sum(c01, red);
    c11 = block_sum(c11, red);
    if (threadIdx.x == 0) {
        const double denom = ((double)nb - 1.0) * (double)nb;
        RegOut o;
        o.est[0] = est[0];
        o.est[1] = est[1];
        o.cov[0] = c00 / denom;
        o.cov[1] = c01 / denom;
        o.cov[2] = c11 / denom;
        o.se[0] = sqrt(o.cov[0]);
        o.se[1] = p == 2 ? sqrt(o.cov[2]) : NAN;
        o.nbar = st.nbar;
        o.mean_y = st.mean_y;
        // total_from_jknife (src/regressions.rs:1565-1610), K = 1
        o.tot = m * est[0] / st.nbar;
        o.tot_se = sqrt(fmax(m * m * o.cov[0] / (st.nbar * st.nbar), 0.0));
        o.intercept = jb.fixed ? st.fixed_int : est[1];
        o.intercept_se = jb.fixed ? NAN : o.se[1];
        o.median_y = NAN;
        outs[j] = o;
    }
}

// rg = gencov / sqrt(h1 h2) with the ratio jackknife over delete values
// (src/regressions.rs:1067-1120, 2425-2451).  One CTA per pair.
__global__ void __launch_bounds__(NT) k_rg_finish(const RgPairIdx* __restrict__ pairs, const RegOut* __restrict__ outs,
                                                  const double* __restrict__ tot_delete, int nb,
                                                  RgOut* __restrict__ res) {
    __shared__ double red[NT / 32];
    __shared__ double s_mean;
    const RgPairIdx pi = pairs[blockIdx.x];
    const RegOut& h1 = outs[pi.hsq1];
    const RegOut& h2 = outs[pi.hsq2];
    const RegOut& g = outs[pi.gencov];
    const bool ok = h1.tot > 0.0 && h2.tot > 0.0;
    const double rg = ok ? g.tot / sqrt(h1.tot * h2.tot) : NAN;
    double sp = 0;
    const double* d1 = tot_delete + (size_t)pi.hsq1 * nb;
    const double* d2 = tot_delete + (size_t)pi.hsq2 * nb;
    const double* dg = tot_delete + (size_t)pi.gencov * nb;
    auto pseudo = [&](int b) {
        const double pr = d1[b] * d2[b];
        const double den = (isfinite(pr) && pr >= 0.0) ? sqrt(pr) : NAN;
        return den == 0.0 ? NAN : (double)nb * rg - (double)(nb - 1) * (dg[b] / den);
    };
    for (int b = threadIdx.x; b < nb; b += NT) sp += pseudo(b);
    const double tsum = block_sum(sp, red);
    if (threadIdx.x == 0) s_mean = tsum / nb;
    __syncthreads();
    double cv = 0;
    for (int b = threadIdx.x; b < nb; b += NT) {
        const double dlt = pseudo(b) - s_mean;
        cv += dlt * dlt;
    }
    cv = block_sum(cv, red);
    if (threadIdx.x == 0) {
        RgOut o;
        o.rg = rg;
        const double scale = ((double)nb - 1.0) * (double)nb;
        o.rg_se = ok ? sqrt(fmax(scale > 0 ? cv / scale : cv, 0.0)) : NAN;
        o.gencov = g.tot;
        o.gencov_se = g.tot_se;
        o.gencov_intercept = g.intercept;
        o.gencov_intercept_se = g.intercept_se;
        o.h2_1 = h1.tot;
        o.h2_1_se = h1.tot_se;
        o.h2_2 = h2.tot;
        o.h2_2_se = h2.tot_se;
        o.mean_z1z2 = g.mean_y;
        res[blockIdx.x] = o;
    }
}

// The two middle order statistics of each job's y (ranks ra <= rb, rb - ra
// <= 1), exactly: a radix select over the order-preserving 64-bit keys of the
// doubles, 11 bits per digit, one CTA per job.  Each digit is one sweep over
// the job's y; the sweep histograms the keys that share the prefix fixed so
// far.  Once that prefix holds at most SEL_CAP keys, one more sweep gathers
// them into shared memory and they are ranked there.  If the two ranks fall
// in different buckets of a digit, ra is the largest key of its bucket and rb
// the smallest of its own, found by one more sweep.  On LD-score chi2 values
// two digits (sign and exponent, then the mantissa's top bits) usually leave
// about a hundred keys, so the select reads each y three times.
__device__ __forceinline__ uint64_t okey(double v) {
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_value(uint64_t k) {
    const uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((long long)b);
}

constexpr int SEL_T = 256;
constexpr int SEL_W = SEL_T / 32;
constexpr int SEL_BITS = 11;
constexpr int SEL_BINS = 1 << SEL_BITS;
constexpr int SEL_CAP = 2048;  // keys ranked in shared memory
constexpr int SEL_U = 8;       // loads in flight per thread

// Calls f(key, valid) for every y of the job; the trip count is the same in
// every lane of a warp, so f may use warp-collective operations.
template <class F>
__device__ __forceinline__ void sel_sweep(const RegJob& jb, uint64_t n, F f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t i0 = (uint64_t)warp * 32 * SEL_U; i0 < n; i0 += (uint64_t)SEL_T * SEL_U) {
        uint64_t k[SEL_U];
        bool v[SEL_U];
#pragma unroll
        for (int u = 0; u < SEL_U; u++) {
            const uint64_t i = i0 + (uint64_t)u * 32 + lane;
            v[u] = i < n;
            k[u] = v[u] ? okey(job_y(jb, i)) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < SEL_U; u++) f(k[u], v[u]);
    }
}

__global__ void __launch_bounds__(SEL_T, 8) k_select_mid(const RegJob* __restrict__ jobs, uint64_t n, uint64_t ra,
                                                      uint64_t rb, double* __restrict__ out_a,
                                                      double* __restrict__ out_b) {
    __shared__ uint32_t hist[SEL_BINS];
    __shared__ uint64_t cand[SEL_CAP];
    __shared__ uint32_t wsum[SEL_W];
    __shared__ uint32_t s_da, s_db, s_acc_a, s_acc_b, s_cnt;
    __shared__ unsigned long long s_ka, s_kb;
    const RegJob jb = jobs[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t prefix = 0, pmask = 0, cnt = n;
    uint64_t qa = ra, qb = rb;  // ranks among the keys that match the prefix
    int top = 64;               // bits below the prefix
    for (;;) {
        if (cnt <= SEL_CAP) {
            // gather the prefix's keys and rank them in shared memory
            if (threadIdx.x == 0) s_cnt = 0;
            __syncthreads();
            sel_sweep(jb, n, [&](uint64_t k, bool v) {
                const bool take = v && (k & pmask) == prefix;
                const unsigned m = __ballot_sync(0xFFFFFFFFu, take);
                uint32_t base = 0;
                if (lane == 0 && m) base = atomicAdd(&s_cnt, (uint32_t)__popc(m));
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (take) cand[base + __popc(m & ((1u << lane) - 1u))] = k;
            });
            __syncthreads();
            const uint32_t c = s_cnt;
            for (uint32_t i = threadIdx.x; i < c; i += SEL_T) {
                const uint64_t ki = cand[i];
                uint32_t r = 0;
                for (uint32_t j = 0; j < c; j++) {
                    const uint64_t kj = cand[j];
                    r += (kj < ki || (kj == ki && j < i)) ? 1u : 0u;
                }
                if (r == qa) s_ka = ki;
                if (r == qb) s_kb = ki;
            }
            __syncthreads();
            break;
        }
        if (top == 0) {  // every key left equals the prefix
            if (threadIdx.x == 0) s_ka = s_kb = prefix;
            __syncthreads();
            break;
        }
        const int width = top < SEL_BITS ? top : SEL_BITS;
        const int shift = top - width;
        const uint32_t dmask = (1u << width) - 1u;
        for (int i = threadIdx.x; i < SEL_BINS; i += SEL_T) hist[i] = 0;
        __syncthreads();
        sel_sweep(jb, n, [&](uint64_t k, bool v) {
            const bool take = v && (k & pmask) == prefix;
            const uint32_t bin = take ? (uint32_t)(k >> shift) & dmask : 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
            if (take && lane == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
        });
        __syncthreads();
        // bins of this thread: [PER t, PER t + PER); exclusive block scan of their sums
        constexpr int PER = SEL_BINS / SEL_T;
        uint32_t c[PER], tsum = 0;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            c[q] = hist[threadIdx.x * PER + q];
            tsum += c[q];
        }
        uint32_t incl = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t acc = incl - tsum;
        for (int w = 0; w < warp; w++) acc += wsum[w];
#pragma unroll
        for (int q = 0; q < PER; q++) {
            if (qa >= acc && qa < acc + c[q]) {
                s_da = threadIdx.x * PER + q;
                s_acc_a = acc;
            }
            if (qb >= acc && qb < acc + c[q]) {
                s_db = threadIdx.x * PER + q;
                s_acc_b = acc;
            }
            acc += c[q];
        }
        __syncthreads();
        const uint32_t da = s_da, db = s_db;
        const uint64_t dm = (uint64_t)dmask << shift;
        if (da == db) {
            prefix |= (uint64_t)da << shift;
            pmask |= dm;
            qa -= s_acc_a;
            qb -= s_acc_b;
            cnt = hist[da];
            top = shift;
            __syncthreads();  // hist and the s_ values are rewritten by the next digit
            continue;
        }
        // ra is the largest key of bucket da, rb the smallest of bucket db
        const uint64_t pa = prefix | ((uint64_t)da << shift), pb = prefix | ((uint64_t)db << shift);
        const uint64_t nm = pmask | dm;
        if (threadIdx.x == 0) {
            s_ka = 0ull;
            s_kb = ~0ull;
        }
        __syncthreads();
        sel_sweep(jb, n, [&](uint64_t k, bool v) {
            if (v && (k & nm) == pa) atomicMax(&s_ka, (unsigned long long)k);
            if (v && (k & nm) == pb) atomicMin(&s_kb, (unsigned long long)k);
        });
        __syncthreads();
        break;
    }
    if (threadIdx.x == 0) {
        out_a[blockIdx.x] = okey_value(s_ka);
        out_b[blockIdx.x] = okey_value(s_kb);
    }
}

// ---- --two-step ----
constexpr int TS_CHUNK = 4096;

__global__ void __launch_bounds__(NT) k_ts_count(const RegJob* __restrict__ jobs, uint64_t n, int32_t* __restrict__ cnt) {
    __shared__ int32_t red[NT / 32];
    const RegJob jb = jobs[blockIdx.y];
    const uint64_t lo = (uint64_t)blockIdx.x * TS_CHUNK, hi = lo + TS_CHUNK < n ? lo + TS_CHUNK : n;
    int32_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) c += job_y(jb, i) < jb.mask_max ? 1 : 0;
    c = block_sum(c, red);
    if (threadIdx.x == 0) cnt[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = c;
}

// Each CTA ranks the kept SNPs of its chunk (block scan of 16-element runs)
// and writes seps[b] for the b whose rank floor(b n1 / nb) falls in it.
__global__ void __launch_bounds__(NT) k_ts_seps(const RegJob* __restrict__ jobs, uint64_t n, int nb,
                                               const int32_t* __restrict__ cnt, int32_t* __restrict__ seps,
                                               int32_t* __restrict__ n1_out) {
    constexpr int PER = TS_CHUNK / NT;  // 16 SNPs per thread
    __shared__ int32_t wsum[NT / 32];
    __shared__ int64_t s_base, s_n1;
    const int job = blockIdx.y, nch = gridDim.x;
    const RegJob jb = jobs[job];
    int32_t* sp = seps + (size_t)job * (nb + 1);
    if (threadIdx.x == 0) {
        int64_t base = 0, tot = 0;
        for (int c = 0; c < nch; c++) {
            const int64_t v = cnt[(size_t)job * nch + c];
            if (c < (int)blockIdx.x) base += v;
            tot += v;
        }
        s_base = base;
        s_n1 = tot;
    }
    __syncthreads();
    const int64_t n1 = s_n1;
    if (n1 < nb) {  // reported as an error by the host; plain block starts keep every access in range
        if (blockIdx.x == 0)
            for (int b = threadIdx.x; b <= nb; b += NT) sp[b] = (int32_t)sep(n, nb, b);
        if (blockIdx.x == 0 && threadIdx.x == 0) n1_out[job] = (int32_t)n1;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sp[0] = 0;
        sp[nb] = (int32_t)n;
        n1_out[job] = (int32_t)n1;
    }
    const uint64_t lo = (uint64_t)blockIdx.x * TS_CHUNK + (uint64_t)threadIdx.x * PER;
    uint32_t flags = 0;
    int32_t c = 0;
#pragma unroll
    for (int u = 0; u < PER; u++) {
        const uint64_t i = lo + u;
        if (i < n && job_y(jb, i) < jb.mask_max) {
            flags |= 1u << u;
            c++;
        }
    }
    // exclusive scan of the per-thread counts
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int64_t rank = s_base + incl - c;
    for (int w = 0; w < warp; w++) rank += wsum[w];
    for (int u = 0; u < PER; u++) {
        if (!(flags >> u & 1u)) continue;
        // the b with floor(b n1 / nb) == rank, if any (at most one: n1 >= nb)
        const int64_t b = (rank * nb + n1 - 1) / n1;
        if (b >= 1 && b < nb && (b * n1) / nb == rank) sp[b] = (int32_t)(lo + u);
        rank++;
    }
}

__global__ void __launch_bounds__(NT) k_ts_combine(const RegOut* __restrict__ out1, const RegOut* __restrict__ out2,
                                                  const RegState* __restrict__ st2, const double* __restrict__ dv1,
                                                  const double* __restrict__ dv2, int nb, double m,
                                                  RegOut* __restrict__ outs) {
    __shared__ double red[NT / 32];
    __shared__ double s_mean[2];
    const int t = blockIdx.x;
    const RegOut& a = out1[t];
    const RegOut& b2 = out2[t];
    const RegState st = st2[t];
    const double c = st.c_num / st.c_den;
    const double e0 = b2.est[0], e1 = a.est[1];
    const double* d1 = dv1 + (size_t)t * nb * 2;
    const double* d2 = dv2 + (size_t)t * nb * 2;
    auto del = [&](int k, int p) { return p == 1 ? d1[2 * k + 1] : d2[2 * k] - c * (d1[2 * k + 1] - e1); };
    double sp0 = 0, sp1 = 0;
    for (int k = threadIdx.x; k < nb; k += NT) {
        sp0 += (double)nb * e0 - (double)(nb - 1) * del(k, 0);
        sp1 += (double)nb * e1 - (double)(nb - 1) * del(k, 1);
    }
    const double m0 = block_sum(sp0, red) / nb, m1 = block_sum(sp1, red) / nb;
    if (threadIdx.x == 0) {
        s_mean[0] = m0;
        s_mean[1] = m1;
    }
    __syncthreads();
    double c00 = 0, c01 = 0, c11 = 0;
    for (int k = threadIdx.x; k < nb; k += NT) {
        const double q0 = (double)nb * e0 - (double)(nb - 1) * del(k, 0) - s_mean[0];
        const double q1 = (double)nb * e1 - (double)(nb - 1) * del(k, 1) - s_mean[1];
        c00 += q0 * q0;
        c01 += q0 * q1;
        c11 += q1 * q1;
    }
    c00 = block_sum(c00, red);
    c01 = block_sum(c01, red);
    c11 = block_sum(c11, red);
    if (threadIdx.x == 0) {
        const double denom = ((double)nb - 1.0) * (double)nb;
        RegOut o;
        o.est[0] = e0;
        o.est[1] = e1;
        o.cov[0] = c00 / denom;
        o.cov[1] = c01 / denom;
        o.cov[2] = c11 / denom;
        o.se[0] = sqrt(o.cov[0]);
        o.se[1] = sqrt(o.cov[2]);
        o.nbar = st.nbar;
        o.mean_y = st.mean_y;
        o.tot = m * e0 / st.nbar;
        o.tot_se = sqrt(fmax(m * m * o.cov[0] / (st.nbar * st.nbar), 0.0));
        o.intercept = e1;
        o.intercept_se = o.se[1];
        o.median_y = NAN;
        outs[t] = o;
    }
}

}  // namespace

cudaError_t launch_twostep_seps(const RegJob* jobs, uint64_t n, int nb, int32_t* seps, int32_t* n1, int32_t* cnt,
                                int njobs, cudaStream_t s) {
    if (njobs <= 0 || n == 0) return cudaSuccess;
    const dim3 grid((unsigned)((n + TS_CHUNK - 1) / TS_CHUNK), njobs);
    k_ts_count<<<grid, NT, 0, s>>>(jobs, n, cnt);
    k_ts_seps<<<grid, NT, 0, s>>>(jobs, n, nb, cnt, seps, n1);
    return cudaGetLastError();
}

cudaError_t launch_twostep_combine(const RegOut* out1, const RegOut* out2, const RegState* st2, const double* dv1,
                                   const double* dv2, int nb, double m, RegOut* outs, int ntraits, cudaStream_t s) {
    if (ntraits <= 0) return cudaSuccess;
    k_ts_combine<<<ntraits, NT, 0, s>>>(out1, out2, st2, dv1, dv2, nb, m, outs);
    return cudaGetLastError();
}

cudaError_t launch_regressions(const RegJob* jobs, RegState* states, RegOut* outs, const RegOut* ref_outs,
                               double* part, double* tot_delete, const double* ld, const double* wld, uint64_t n,
                               int nb, double m, int njobs, cudaStream_t s, double* dv, int form) {
    if (njobs <= 0) return cudaSuccess;
    if (form < REG_FORM_HSQ_DIRECT || form > REG_FORM_GENCOV_PRODUCT || n >= (1ull << 31))
        return cudaErrorInvalidValue;
    const dim3 grid(nb, (njobs + RJ - 1) / RJ);
    const int ub = (njobs + 3) / 4;  // k_reg_update: four warps (jobs) per CTA
    auto sums = [&](int mode) {
        if (form == REG_FORM_HSQ_DIRECT) {
            if (mode == 0) k_reg_sums<0, REG_FORM_HSQ_DIRECT><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
            else k_reg_sums<1, REG_FORM_HSQ_DIRECT><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
        } else if (form == REG_FORM_HSQ_SQUARE) {
            if (mode == 0) k_reg_sums<0, REG_FORM_HSQ_SQUARE><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
            else k_reg_sums<1, REG_FORM_HSQ_SQUARE><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
        } else {
            if (mode == 0) k_reg_sums<0, REG_FORM_GENCOV_PRODUCT><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
            else k_reg_sums<1, REG_FORM_GENCOV_PRODUCT><<<grid, RJ * 32, 0, s>>>(jobs, states, ld, wld, n, nb, m, njobs, part);
        }
    };
    sums(0);
    k_reg_update<0><<<ub, 128, 0, s>>>(jobs, states, ref_outs, part, n, nb, m, njobs);
    for (int it = 0; it < 2; it++) {  // irwls_ldsc: two re-weightings
        sums(1);
        k_reg_update<1><<<ub, 128, 0, s>>>(jobs, states, ref_outs, part, n, nb, m, njobs);
    }
    sums(1);
    k_reg_jackknife<<<njobs, NT, 0, s>>>(jobs, states, outs, part, nb, m, tot_delete, dv);
    return cudaGetLastError();
}

cudaError_t launch_rg_finish(const RgPairIdx* pairs, const RegOut* outs, const double* tot_delete, int nb,
                             RgOut* res, int npairs, cudaStream_t s) {
    if (npairs <= 0) return cudaSuccess;
    k_rg_finish<<<npairs, NT, 0, s>>>(pairs, outs, tot_delete, nb, res);
    return cudaGetLastError();
}

cudaError_t launch_select_mid(const RegJob* jobs, uint64_t n, uint64_t ra, uint64_t rb, double* out_a, double* out_b,
                              int njobs, cudaStream_t s) {
    if (njobs <= 0 || n == 0 || ra > rb || rb - ra > 1 || rb >= n) return cudaErrorInvalidValue;
    k_select_mid<<<njobs, SEL_T, 0, s>>>(jobs, n, ra, rb, out_a, out_b);
    return cudaGetLastError();
}

cudaError_t preload_regress() {
    cudaError_t e = preload_kernel(k_reg_sums<0, REG_FORM_HSQ_DIRECT>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<1, REG_FORM_HSQ_DIRECT>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<0, REG_FORM_HSQ_SQUARE>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<1, REG_FORM_HSQ_SQUARE>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<0, REG_FORM_GENCOV_PRODUCT>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<1, REG_FORM_GENCOV_PRODUCT>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_update<0>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_update<1>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_jackknife);
    if (e == cudaSuccess) e = preload_kernel(k_rg_finish);
    if (e == cudaSuccess) e = preload_kernel(k_select_mid);
    if (e == cudaSuccess) e = preload_kernel(k_ts_count);
    if (e == cudaSuccess) e = preload_kernel(k_ts_seps);
    if (e == cudaSuccess) e = preload_kernel(k_ts_combine);
    return e;
}

}  // namespace ldsc
