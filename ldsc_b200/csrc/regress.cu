// regress.cu -- batched LD-score regressions (h2 and genetic covariance) on
// device-resident LD scores: weights, two IRWLS re-weightings, block
// jackknife.  Restates the reference's
//   ldsc_weights / aggregate / irwls_ldsc / jackknife_fast   (src/h2.rs:100-458)
//   jackknife_se_cov                                          (src/jackknife.rs:10-59)
//   gencov_weights / run_hsq_ldsc / run_gencov_ldsc           (src/regressions.rs:1612-2052)
// for the one-LD-score-column case (K = 1), many traits at once.
//
// Every per-SNP pass is one kernel over (jackknife block, job): a CTA sums
// its block's contributions in f64, and per-job kernels combine the blocks in
// block order, so results do not depend on scheduling.  The weighted least
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
__device__ __forceinline__ double job_n1(const RegJob& jb, uint64_t i) { return jb.n1 ? jb.n1[i] : jb.n1s; }
__device__ __forceinline__ double job_n2(const RegJob& jb, uint64_t i) { return jb.n2 ? jb.n2[i] : jb.n2s; }
// sample size that scales the regressor: N (h2) or sqrt(N1 N2) (gencov)
__device__ __forceinline__ double job_nx(const RegJob& jb, uint64_t i) {
    return jb.kind == REG_HSQ ? job_n1(jb, i) : sqrt(job_n1(jb, i) * job_n2(jb, i));
}

// Regression weight of SNP i under the job's current parameters (the square
// of the reference's w): ldsc_weights (src/h2.rs:185-206) or gencov_weights
// (src/regressions.rs:1612-1645).
__device__ __forceinline__ double job_weight(const RegJob& jb, const RegState& st, double ld_raw, double wld_raw,
                                             uint64_t i, double m) {
    const double oc = 1.0 / fmax(wld_raw, 1.0);
    if (jb.kind == REG_HSQ) {
        // step 1 of --two-step re-weights with the regressor in place of the LD
        // score (src/h2.rs:347-351: ldsc_weights(x1_col0, ...))
        const double ld = jb.ld_from_x && st.n_updates > 0 ? fmax(job_n1(jb, i) * ld_raw / st.nbar, 1.0) : fmax(ld_raw, 1.0);
        const double hsq = fmin(fmax(st.slope, 0.0), 1.0);
        const double c = hsq * job_n1(jb, i) / m;
        const double t = st.intercept + c * ld;
        return 1.0 / (2.0 * t * t) * oc;
    }
    const double ld = fmax(ld_raw, 1.0);
    const double h1 = fmin(fmax(st.h1, 0.0), 1.0), h2 = fmin(fmax(st.h2, 0.0), 1.0);
    const double n1 = job_n1(jb, i), n2 = job_n2(jb, i);
    const double a = n1 * h1 * ld / m + st.int_h1;
    const double b = n2 * h2 * ld / m + st.int_h2;
    const double c = sqrt(n1 * n2) * st.slope * ld / m + st.intercept;
    return 1.0 / (a * b + c * c) * oc;
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
template <int MODE>
__global__ void __launch_bounds__(NT) k_reg_sums(const RegJob* __restrict__ jobs, const RegState* __restrict__ states,
                                                 const double* __restrict__ ld, const double* __restrict__ wld,
                                                 uint64_t n, int nb, double m, double* __restrict__ part) {
    __shared__ double red[NT / 32];
    const int b = blockIdx.x, j = blockIdx.y;
    const RegJob jb = jobs[j];
    const RegState st = states[j];
    const uint64_t lo = jb.seps ? (uint64_t)jb.seps[b] : sep(n, nb, b);
    const uint64_t hi = jb.seps ? (uint64_t)jb.seps[b + 1] : sep(n, nb, b + 1);
    double s[5] = {0, 0, 0, 0, 0};
    for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) {
        const double y = job_y(jb, i);
        if (MODE == 1 && jb.use_mask && !(y < jb.mask_max)) continue;
        const double l = ld[i];
        const double nx = job_nx(jb, i);
        if (MODE == 0) {
            s[0] += y;
            s[1] += l * nx;
            s[2] += nx;
        } else {
            const double w = job_weight(jb, st, l, wld[i], i, m);
            const double x0 = nx * l / st.nbar;
            s[0] += w * x0 * x0;
            s[1] += w * x0;
            s[2] += w;
            s[3] += w * x0 * y;
            s[4] += w * y;
        }
    }
    double* out = part + ((size_t)j * nb + b) * 5;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        if (MODE == 0 && q >= 3) break;
        const double t = block_sum(s[q], red);
        if (threadIdx.x == 0) out[q] = t;
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
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const RegJob jb = jobs[j];
    RegState st = states[j];
    double S[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < nb; b++)
        for (int q = 0; q < (MODE == 0 ? 3 : 5); q++) S[q] += part[((size_t)j * nb + b) * 5 + q];
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

// Exact order statistic of each job's y (radix select over the order-
// preserving 64-bit keys of the doubles), 8 bits per pass; one CTA per job.
__device__ __forceinline__ uint64_t okey(double v) {
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_value(uint64_t k) {
    const uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((long long)b);
}

__global__ void __launch_bounds__(NT) k_select(const RegJob* __restrict__ jobs, uint64_t n, uint64_t rank,
                                               double* __restrict__ out) {
    __shared__ uint32_t hist[256];
    __shared__ uint64_t s_prefix, s_rank;
    const RegJob jb = jobs[blockIdx.x];
    uint64_t prefix = 0, r = rank;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += NT) hist[i] = 0;
        __syncthreads();
        const uint64_t pmask = shift == 56 ? 0ull : (~0ull << (shift + 8));
        for (uint64_t i = threadIdx.x; i < n; i += NT) {
            const uint64_t k = okey(job_y(jb, i));
            if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 0xFF], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t acc = 0;
            int d = 0;
            for (; d < 256; d++) {
                if (acc + hist[d] > r) break;
                acc += hist[d];
            }
            s_prefix = prefix | ((uint64_t)d << shift);
            s_rank = r - acc;
        }
        __syncthreads();
        prefix = s_prefix;
        r = s_rank;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = okey_value(prefix);
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
                               int nb, double m, int njobs, cudaStream_t s, double* dv) {
    if (njobs <= 0) return cudaSuccess;
    const dim3 grid(nb, njobs);
    const int ub = (njobs + 127) / 128;
    k_reg_sums<0><<<grid, NT, 0, s>>>(jobs, states, ld, wld, n, nb, m, part);
    k_reg_update<0><<<ub, 128, 0, s>>>(jobs, states, ref_outs, part, n, nb, m, njobs);
    for (int it = 0; it < 2; it++) {  // irwls_ldsc: two re-weightings
        k_reg_sums<1><<<grid, NT, 0, s>>>(jobs, states, ld, wld, n, nb, m, part);
        k_reg_update<1><<<ub, 128, 0, s>>>(jobs, states, ref_outs, part, n, nb, m, njobs);
    }
    k_reg_sums<1><<<grid, NT, 0, s>>>(jobs, states, ld, wld, n, nb, m, part);
    k_reg_jackknife<<<njobs, NT, 0, s>>>(jobs, states, outs, part, nb, m, tot_delete, dv);
    return cudaGetLastError();
}

cudaError_t launch_rg_finish(const RgPairIdx* pairs, const RegOut* outs, const double* tot_delete, int nb,
                             RgOut* res, int npairs, cudaStream_t s) {
    if (npairs <= 0) return cudaSuccess;
    k_rg_finish<<<npairs, NT, 0, s>>>(pairs, outs, tot_delete, nb, res);
    return cudaGetLastError();
}

cudaError_t launch_select(const RegJob* jobs, uint64_t n, uint64_t rank, double* out, int njobs, cudaStream_t s) {
    if (njobs <= 0 || n == 0) return cudaSuccess;
    k_select<<<njobs, NT, 0, s>>>(jobs, n, rank, out);
    return cudaGetLastError();
}

cudaError_t preload_regress() {
    cudaError_t e = preload_kernel(k_reg_sums<0>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_sums<1>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_update<0>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_update<1>);
    if (e == cudaSuccess) e = preload_kernel(k_reg_jackknife);
    if (e == cudaSuccess) e = preload_kernel(k_rg_finish);
    if (e == cudaSuccess) e = preload_kernel(k_select);
    if (e == cudaSuccess) e = preload_kernel(k_ts_count);
    if (e == cudaSuccess) e = preload_kernel(k_ts_seps);
    if (e == cudaSuccess) e = preload_kernel(k_ts_combine);
    return e;
}

}  // namespace ldsc
