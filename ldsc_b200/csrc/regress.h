// regress.h -- device structures of the batched LD-score regressions.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace ldsc {

enum { REG_HSQ = 0, REG_GENCOV = 1 };
enum { REG_Y_DIRECT = 0, REG_Y_SQUARE = 1, REG_Y_PRODUCT = 2 };
// (kind, y) shared by every job of one launch_regressions call: h2 fits on
// chi2, h2 fits on z (y = z^2), genetic-covariance fits (y = z1 z2)
enum { REG_FORM_HSQ_DIRECT = 0, REG_FORM_HSQ_SQUARE = 1, REG_FORM_GENCOV_PRODUCT = 2 };

// One regression: y ~ [x0 = Nx * ld / nbar, 1] with weights of its kind.
struct RegJob {
    const double* ya;   // y source (device)
    const double* yb;   // second factor for REG_Y_PRODUCT
    int32_t ymode;      // y = ya | max(ya^2, 0) | ya * yb
    int32_t kind;       // REG_HSQ or REG_GENCOV
    const double* n1;   // per-SNP sample sizes (device) or null
    const double* n2;
    double n1s, n2s;    // scalar sample sizes when n1 / n2 are null
    int32_t fixed;      // intercept constrained
    double fixed_int;
    int32_t hsq1, hsq2; // REG_GENCOV: job indices of the two h2 fits
    // --two-step (src/h2.rs:319-393)
    const int32_t* seps;  // nb + 1 block starts in SNP index space, or null: floor(b n / nb)
    int32_t use_mask;     // least-squares sums over SNPs with y < mask_max only (step 1)
    double mask_max;
    int32_t ld_from_x;    // re-weighting uses the regressor x0 in place of the LD score (step 1)
    int32_t int_from;     // fixed intercept = est[1] of ref_outs[int_from] (step 2), or -1
};

// Running parameters of a job between passes.
struct RegState {
    double nbar, mean_y;
    double slope;       // hsq (REG_HSQ) or rho_g (REG_GENCOV) used by the weights
    double intercept;
    double h1, h2, int_h1, int_h2;  // REG_GENCOV weight constants
    double fixed_int;               // intercept of the least squares when jb.fixed
    double c_num, c_den;            // sum w0 x0, sum w0 x0^2 under the initial weights
    int32_t n_updates;
};

struct RegOut {
    double est[2], se[2], cov[3];   // coefficient on x0 and intercept; cov = (00, 01, 11)
    double tot, tot_se;             // h2 or genetic covariance: M * est0 / nbar
    double intercept, intercept_se;
    double nbar, mean_y, median_y;
};

struct RgPairIdx {
    int32_t hsq1, hsq2, gencov;
};

struct RgOut {
    double rg, rg_se;
    double gencov, gencov_se, gencov_intercept, gencov_intercept_se;
    double h2_1, h2_1_se, h2_2, h2_2_se;
    double mean_z1z2;
};

// Aggregate pass, two IRWLS updates and the block jackknife for all jobs,
// every one of them of the given form (REG_FORM_*); n < 2^31.
// outs[j] receives job j's result; ref_outs holds the h2 results that
// REG_GENCOV jobs refer to by index.  part: njobs * nb * 5 doubles of
// scratch; tot_delete (optional): njobs * nb; dv (optional): njobs * nb * 2
// delete values.
cudaError_t launch_regressions(const RegJob* jobs, RegState* states, RegOut* outs, const RegOut* ref_outs,
                               double* part, double* tot_delete, const double* ld, const double* wld, uint64_t n,
                               int nb, double m, int njobs, cudaStream_t s, double* dv = nullptr,
                               int form = REG_FORM_HSQ_DIRECT);

// --two-step block starts: for each job, mask = y < mask_max, n1 = its size,
// and seps[b] = index of the kept SNP of rank floor(b n1 / nb) (0 and n at
// the ends): get_separators on the kept SNPs mapped back by update_separators
// (src/h2.rs:31-58).  seps: njobs * (nb + 1); n1: njobs; cnt: scratch of
// njobs * ceil(n / 4096) ints.
cudaError_t launch_twostep_seps(const RegJob* jobs, uint64_t n, int nb, int32_t* seps, int32_t* n1, int32_t* cnt,
                                int njobs, cudaStream_t s);

// combine_twostep (src/h2.rs:220-256) + the h2 result: step 1 jobs s1[t],
// step 2 jobs s2[t] (the fixed-intercept fit on all SNPs), their delete
// values dv1 / dv2 (nb * 2 per job) -> outs[t].
cudaError_t launch_twostep_combine(const RegOut* out1, const RegOut* out2, const RegState* st2, const double* dv1,
                                   const double* dv2, int nb, double m, RegOut* outs, int ntraits, cudaStream_t s);

cudaError_t launch_rg_finish(const RgPairIdx* pairs, const RegOut* outs, const double* tot_delete, int nb,
                             RgOut* res, int npairs, cudaStream_t s);

// The ra-th and rb-th smallest y of each job (exact; ra <= rb <= ra + 1),
// out_a[job] and out_b[job].
cudaError_t launch_select_mid(const RegJob* jobs, uint64_t n, uint64_t ra, uint64_t rb, double* out_a, double* out_b,
                              int njobs, cudaStream_t s);

// ---- partitioned h2 (fit_h2_partitioned, src/regressions.rs:1121-1226) ----

struct PartJob {
    const double* chi2;    // n (device)
    const double* nv;      // per-SNP sample sizes (device) or null
    double ns;             // scalar sample size when nv is null
    const int32_t* seps;   // nb + 1 jackknife block starts in SNP index space
    double mask_max;       // SNPs with chi2 < mask_max are kept
    double n_obs;          // number of kept SNPs
    int32_t fixed;         // intercept constrained to fixed_int
    double fixed_int;
};

struct PartState {
    double nbar, mean_chi2, hsq, agg_int, n_obs;
};

// Parameters: K LD-score coefficients, plus the intercept when it is free.
__host__ __device__ inline int part_params(int k, bool fixed) { return k + (fixed ? 0 : 1); }
// Doubles per job in the result array: est p, cov p x p, delete values
// nb x p, h2 per annotation k, then h2_total, h2_total_se, intercept,
// intercept_se, nbar, mean_chi2, n_obs.
__host__ __device__ inline size_t part_result_len(int nb, int k, int p) { return (size_t)p * (1 + p + nb) + k + 7; }
// Shared memory of one delete-value solve (p x (p + 1) doubles) is capped here.
constexpr int PART_SOLVE_SMEM = 210 * 1024;
// Traits per launch: the block Grams of a launch (traits x nb x q^2 doubles)
// stay within 1 GiB.
inline int part_trait_chunk(int traits, int nb, int q) {
    const double per = 8.0 * nb * (double)q * q;
    int c = (int)((double)(1u << 30) / per);
    if (c < 1) c = 1;
    return c < traits ? c : traits;
}

// x_tot (when want_xtot), aggregate, per-block Grams of the weighted design,
// block totals, nb + 1 LU solves and the jackknife for every job.  Scratch:
// xtot n, part njobs * nb * 3, gram njobs * nb * (p+1)^2, tot njobs *
// (p+1)^2, sol njobs * (nb+1) * p; res njobs * part_result_len; st njobs.
// m_vec: k per-annotation M on the device.
cudaError_t launch_partitioned(const PartJob* jobs, PartState* st, const double* l2, uint64_t ld, int k, bool fixed,
                               const double* wld, uint64_t n, int nb, double m_tot, const double* m_vec, double* xtot,
                               bool want_xtot, double* part, double* gram, double* tot, double* sol, double* res,
                               int njobs, cudaStream_t s);

}  // namespace ldsc
