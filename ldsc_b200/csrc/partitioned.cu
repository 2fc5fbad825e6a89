// partitioned.cu -- partitioned (stratified) h2 on device-resident LD scores:
// one weighted least squares on K annotation LD-score columns plus an
// intercept, with the block jackknife.  Restates fit_h2_partitioned
// (src/regressions.rs:1121-1226): weights from the summed LD score
// (aggregate, ldsc_weights, src/h2.rs:185-218), the weighted design
// (weight_xy, src/h2.rs:60-80), jackknife_fast's per-block X'X / X'y and LU
// solves (src/h2.rs:100-183) and jackknife_se_cov (src/jackknife.rs:10-59).
//
// The design is augmented with y as its last column, Z = [x_1..x_K, 1, y],
// so one symmetric Gram per jackknife block, sum_i w_i z_i z_i', holds X'X,
// X'y and y'y.  Rows are scaled by sqrt(w_i) as in the reference, which also
// divides by sum_j sqrt(w_j): that global factor cancels in every solve.  SNPs dropped by the chi2 cut contribute nothing and the
// jackknife blocks are the reference's blocks over the kept SNPs (block starts
// mapped back to SNP indices).  Block partial sums are combined in block
// order, so results do not depend on scheduling.
#include <cuda_runtime.h>

#include <cmath>

#include "engine.h"
#include "regress.h"

namespace ldsc {

namespace {

constexpr int NT = 256;
constexpr int ROWS = 32;       // SNPs staged per step of the Gram

__device__ __forceinline__ double part_n(const PartJob& jb, uint64_t i) { return jb.nv ? jb.nv[i] : jb.ns; }
__device__ __forceinline__ bool part_kept(const PartJob& jb, uint64_t i) { return jb.chi2[i] < jb.mask_max; }

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

// x_tot[i] = sum_j l2[i, j], columns added in order (src/regressions.rs:1158-1165)
__global__ void __launch_bounds__(NT) k_p_xtot(const double* __restrict__ l2, uint64_t ld, int k, uint64_t n,
                                              double* __restrict__ xtot) {
    for (uint64_t i = (uint64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * NT) {
        double s = 0.0;
        for (int j = 0; j < k; j++) s += l2[(size_t)j * ld + i];
        xtot[i] = s;
    }
}

// Per (jackknife block, job): sum chi2, sum x_tot * N, sum N over kept SNPs.
__global__ void __launch_bounds__(NT) k_p_sums(const PartJob* __restrict__ jobs, const double* __restrict__ xtot,
                                              int nb, double* __restrict__ part) {
    __shared__ double red[NT / 32];
    const int b = blockIdx.x, j = blockIdx.y;
    const PartJob jb = jobs[j];
    const uint64_t lo = (uint64_t)jb.seps[b], hi = (uint64_t)jb.seps[b + 1];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) {
        if (!part_kept(jb, i)) continue;
        const double nn = part_n(jb, i);
        s0 += jb.chi2[i];
        s1 += xtot[i] * nn;
        s2 += nn;
    }
    double* out = part + ((size_t)j * nb + b) * 3;
    s0 = block_sum(s0, red);
    s1 = block_sum(s1, red);
    s2 = block_sum(s2, red);
    if (threadIdx.x == 0) {
        out[0] = s0;
        out[1] = s1;
        out[2] = s2;
    }
}

// nbar, mean chi2 and the aggregate h2 that seeds the weights
// (src/regressions.rs:1189-1191).
__global__ void k_p_aggregate(const PartJob* __restrict__ jobs, const double* __restrict__ part, int nb,
                              double m_tot, PartState* __restrict__ st, int njobs) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int b = 0; b < nb; b++) {
        const double* p = part + ((size_t)j * nb + b) * 3;
        s0 += p[0];
        s1 += p[1];
        s2 += p[2];
    }
    const double nobs = jobs[j].n_obs;
    PartState& o = st[j];
    o.n_obs = nobs;
    o.nbar = s2 / nobs;
    o.mean_chi2 = s0 / nobs;
    o.agg_int = jobs[j].fixed ? jobs[j].fixed_int : 1.0;
    o.hsq = m_tot * (o.mean_chi2 - o.agg_int) / (s1 / nobs);
}

// Gram of the augmented weighted design over one jackknife block:
// G = sum_i w_i z_i z_i' with z_i = [N_i l2_i1 / nbar, ..., N_i l2_iK / nbar,
// 1 (free intercept only), chi2_i - fixed intercept] and w_i the reference's
// weight (its weighted design scales rows by sqrt(w_i) / sum_j sqrt(w_j),
// src/h2.rs:60-80; the global factor cancels in every solve).  The upper
// triangle is cut into 16 x 16 micro-tiles, 16 per CTA (4 x 4 outputs per
// thread).  Rows are staged 32 at a time, double-buffered: the raw LD scores
// of the next 32 rows arrive by cp.async while the current ones are
// multiplied.  A row is staged as v_i = z_i / s_i with s_i = N_i / nbar (the
// LD-score columns are then the raw values, the intercept 1 / s_i, the chi2
// column y_i / s_i) and enters as (w_i s_i^2) v_i v_i'; a row with N_i = 0
// is staged as z_i with factor w_i.
constexpr int MT = 16;                                  // micro-tile edge
__host__ __device__ inline int part_qp(int q) { return (q + MT - 1) / MT * MT; }
__host__ __device__ inline int part_ustride(int q) { return part_qp(q) + 2; }  // doubles per staged row
__host__ __device__ inline size_t part_gram_smem(int q) { return 2 * (size_t)ROWS * part_ustride(q) * sizeof(double); }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(NT, 3) k_p_gram(const PartJob* __restrict__ jobs, const PartState* __restrict__ st,
                                                 const double* __restrict__ l2, uint64_t ld, int k,
                                                 const double* __restrict__ xtot, const double* __restrict__ wld,
                                                 double m_tot, int nb, int q, double* __restrict__ gram) {
    extern __shared__ __align__(16) double U[];  // 2 x ROWS x ustride
    __shared__ double rf[2][ROWS];               // row factors w_i s_i^2 (0: row not kept)
    __shared__ double rsc[2][ROWS];              // s_i, or 0 when the row is staged as z_i
    const int b = blockIdx.x, j = blockIdx.z;
    const int qp = part_qp(q), us = part_ustride(q), nm = qp / MT;
    const int count = nm * (nm + 1) / 2;
    // this thread's micro-tile (row-major over the upper triangle) and 4 x 4 block in it
    const int g = blockIdx.y * (NT / MT) + threadIdx.x / MT;
    const bool active = g < count;
    int mi = 0, rem = active ? g : 0;
    while (rem >= nm - mi) {
        rem -= nm - mi;
        mi++;
    }
    const int mj = mi + rem;
    const int r0c = mi * MT + ((threadIdx.x % MT) / 4) * 4, c0c = mj * MT + (threadIdx.x % 4) * 4;
    const PartJob jb = jobs[j];
    const PartState s = st[j];
    const bool free_int = !jb.fixed;
    const double yoff = jb.fixed ? jb.fixed_int : 0.0;
    const double hsq = fmin(fmax(s.hsq, 0.0), 1.0);
    const uint64_t lo = (uint64_t)jb.seps[b], hi = (uint64_t)jb.seps[b + 1];
    const int nchunks = (int)((hi - lo + ROWS - 1) / ROWS);
    // padding columns [q, qp) stay zero in both buffers
    for (int e = threadIdx.x; e < 2 * ROWS * (qp - q); e += NT) {
        const int bb = e / (ROWS * (qp - q)), r = (e / (qp - q)) % ROWS, c = q + e % (qp - q);
        U[(size_t)bb * ROWS * us + r * us + c] = 0.0;
    }
    // stage rows [lo + c ROWS, ...) into buffer c & 1: factors and the special
    // columns by one thread per row, then the LD scores (barrier between)
    auto stage_meta = [&](int c) {
        if (threadIdx.x < ROWS) {
            const int bb = c & 1;
            const uint64_t i = lo + (uint64_t)c * ROWS + threadIdx.x;
            double* row = U + (size_t)bb * ROWS * us + threadIdx.x * us;
            double f = 0.0, sc = 0.0, vi = 0.0, vy = 0.0;
            if (i < hi && part_kept(jb, i)) {
                // ldsc_weights (src/h2.rs:185-206) on x_tot with M = sum(M_k)
                const double nn = part_n(jb, i);
                const double cc = hsq * nn / m_tot;
                const double t = s.agg_int + cc * fmax(xtot[i], 1.0);
                const double w = 1.0 / (2.0 * t * t) / fmax(wld[i], 1.0);
                sc = nn / s.nbar;
                const double y = jb.chi2[i] - yoff;
                if (sc != 0.0) {
                    f = w * sc * sc;
                    vi = 1.0 / sc;
                    vy = y / sc;
                } else {
                    f = w;
                    vi = 1.0;
                    vy = y;
                }
            }
            if (free_int) row[k] = vi;
            row[q - 1] = vy;
            rf[bb][threadIdx.x] = f;
            rsc[bb][threadIdx.x] = sc;
        }
    };
    auto stage_ld = [&](int c) {
        const int bb = c & 1;
        const uint64_t r0 = lo + (uint64_t)c * ROWS;
        double* buf = U + (size_t)bb * ROWS * us;
        for (int e = threadIdx.x; e < ROWS * k; e += NT) {
            const int col = e / ROWS, r = e % ROWS;
            const uint64_t i = r0 + r;
            if (rf[bb][r] != 0.0 && rsc[bb][r] != 0.0)
                cp_async8(buf + r * us + col, l2 + (size_t)col * ld + i);
            else
                buf[r * us + col] = 0.0;   // row not kept (or N = 0: its LD-score columns are 0)
        }
        cp_async_commit();
    };
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = 0.0;
    if (nchunks > 0) {
        stage_meta(0);
        __syncthreads();
        stage_ld(0);
    }
    for (int c = 0; c < nchunks; c++) {
        const bool next = c + 1 < nchunks;
        if (next) stage_meta(c + 1);   // buffer (c + 1) & 1 was released by the previous iteration's barrier
        __syncthreads();
        if (next) {
            stage_ld(c + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (active) {
            const int bb = c & 1;
            const double* buf = U + (size_t)bb * ROWS * us;
            const uint64_t r0 = lo + (uint64_t)c * ROWS;
            const int nr = (int)(hi - r0 < (uint64_t)ROWS ? hi - r0 : (uint64_t)ROWS);
            for (int r = 0; r < nr; r++) {
                const double f = rf[bb][r];
                const double2 a01 = *reinterpret_cast<const double2*>(&buf[r * us + r0c]);
                const double2 a23 = *reinterpret_cast<const double2*>(&buf[r * us + r0c + 2]);
                const double2 b01 = *reinterpret_cast<const double2*>(&buf[r * us + c0c]);
                const double2 b23 = *reinterpret_cast<const double2*>(&buf[r * us + c0c + 2]);
                const double av[4] = {a01.x * f, a01.y * f, a23.x * f, a23.y * f};
                const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
            }
        }
        __syncthreads();
    }
    if (!active) return;
    // write row <= col and its mirror, so the stored matrix is exactly symmetric
    double* G = gram + ((size_t)j * nb + b) * (size_t)q * q;
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int rr = r0c + u, cc = c0c + v;
            if (rr < q && cc < q && rr <= cc) {
                G[(size_t)rr * q + cc] = acc[u][v];
                G[(size_t)cc * q + rr] = acc[u][v];
            }
        }
}

// tot[j] = sum over blocks in order of the block Grams.
__global__ void __launch_bounds__(NT) k_p_total(const double* __restrict__ gram, int nb, int qq,
                                               double* __restrict__ tot) {
    const int j = blockIdx.y;
    const int e = blockIdx.x * NT + threadIdx.x;
    if (e >= qq) return;
    const double* g = gram + (size_t)j * nb * qq + e;
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += g[(size_t)b * qq];
    tot[(size_t)j * qq + e] = s;
}

// One solve per CTA: (X'X_tot - X'X_b) beta = X'y_tot - X'y_b for b < nb
// (the delete values), the total system for b == nb.  Gaussian elimination
// with partial pivoting (largest |pivot|, first on ties) on the augmented
// p x (p+1) system in shared memory, then back substitution.
__global__ void __launch_bounds__(NT) k_p_solve(const double* __restrict__ gram, const double* __restrict__ tot,
                                               int nb, int q, double* __restrict__ sol) {
    extern __shared__ __align__(16) double M[];  // p x (p + 1), row-major
    __shared__ double rv[NT / 32];
    __shared__ int ri[NT / 32];
    __shared__ int piv;
    const int b = blockIdx.x, j = blockIdx.y;
    const int p = q - 1, w = p + 1;
    const size_t qq = (size_t)q * q;
    const double* T = tot + (size_t)j * qq;
    const double* G = b < nb ? gram + ((size_t)j * nb + b) * qq : nullptr;
    for (int e = threadIdx.x; e < p * w; e += NT) {
        const int r = e / w, c = e % w;
        const int src = r * q + (c < p ? c : q - 1);  // last column: X'y
        M[e] = G ? T[src] - G[src] : T[src];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < p; c++) {
        // pivot row: largest |M[r][c]|, r >= c, first index on ties
        double best = -1.0;
        int bi = p;
        for (int r = c + threadIdx.x; r < p; r += NT) {
            const double v = fabs(M[r * w + c]);
            if (v > best) {
                best = v;
                bi = r;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xFFFFFFFFu, best, o);
            const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            rv[warp] = best;
            ri[warp] = bi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bv = rv[0];
            int bidx = ri[0];
            for (int x = 1; x < NT / 32; x++)
                if (rv[x] > bv || (rv[x] == bv && ri[x] < bidx)) {
                    bv = rv[x];
                    bidx = ri[x];
                }
            piv = bidx < p ? bidx : c;  // NaN column: keep the row
        }
        __syncthreads();
        const int pr = piv;
        if (pr != c)
            for (int x = c + threadIdx.x; x < w; x += NT) {
                const double t = M[c * w + x];
                M[c * w + x] = M[pr * w + x];
                M[pr * w + x] = t;
            }
        __syncthreads();
        // multipliers, then the trailing update
        const double d = M[c * w + c];
        for (int r = c + 1 + threadIdx.x; r < p; r += NT) M[r * w + c] = M[r * w + c] / d;
        __syncthreads();
        // trailing update: warps over rows, lanes over columns
        for (int r = c + 1 + warp; r < p; r += NT / 32) {
            const double mr = M[r * w + c];
            for (int x = c + 1 + lane; x < w; x += 32) M[r * w + x] = fma(-mr, M[c * w + x], M[r * w + x]);
        }
        __syncthreads();
    }
    // back substitution into the last column
    for (int c = p - 1; c >= 0; c--) {
        if (threadIdx.x == 0) M[c * w + p] = M[c * w + p] / M[c * w + c];
        __syncthreads();
        const double xc = M[c * w + p];
        for (int r = threadIdx.x; r < c; r += NT) M[r * w + p] = fma(-M[r * w + c], xc, M[r * w + p]);
        __syncthreads();
    }
    double* out = sol + ((size_t)j * (nb + 1) + b) * p;
    for (int r = threadIdx.x; r < p; r += NT) out[r] = M[r * w + p];
}

// Estimates, delete values, jackknife covariance and the h2 figures of each
// job.  res[j]: [est p][cov p x p][delete values nb x p][h2 per annotation k]
// [h2_total, h2_total_se, intercept, intercept_se, nbar, mean_chi2, n_obs].
__global__ void __launch_bounds__(NT) k_p_finish(const PartJob* __restrict__ jobs, const PartState* __restrict__ st,
                                                const double* __restrict__ sol, const double* __restrict__ m_vec,
                                                int nb, int k, int p, double* __restrict__ res) {
    extern __shared__ double mean[];  // p pseudo-value means
    __shared__ double red[NT / 32];
    const int j = blockIdx.x;
    const PartJob jb = jobs[j];
    const PartState s = st[j];
    const double* S = sol + (size_t)j * (nb + 1) * p;
    const double* est = S + (size_t)nb * p;
    double* R = res + (size_t)j * part_result_len(nb, k, p);
    double* o_est = R;
    double* o_cov = o_est + p;
    double* o_dv = o_cov + (size_t)p * p;
    double* o_h2 = o_dv + (size_t)nb * p;
    double* o_sc = o_h2 + k;
    const double fnb = (double)nb;
    for (int c = threadIdx.x; c < p; c += NT) {
        o_est[c] = est[c];
        double sm = 0.0;
        for (int b = 0; b < nb; b++) sm += fnb * est[c] - (fnb - 1.0) * S[(size_t)b * p + c];
        mean[c] = sm / fnb;
    }
    for (size_t e = threadIdx.x; e < (size_t)nb * p; e += NT) o_dv[e] = S[e];
    __syncthreads();
    // jackknife_se_cov: centred pseudo-values, cov = C'C / ((nb - 1) nb)
    const double scale = (fnb - 1.0) * fnb;
    for (int e = threadIdx.x; e < p * p; e += NT) {
        const int r = e / p, c = e % p;
        if (r > c) continue;
        double acc = 0.0;
        for (int b = 0; b < nb; b++) {
            const double pr = fnb * est[r] - (fnb - 1.0) * S[(size_t)b * p + r] - mean[r];
            const double pc = fnb * est[c] - (fnb - 1.0) * S[(size_t)b * p + c] - mean[c];
            acc = fma(pr, pc, acc);
        }
        const double v = scale > 0.0 ? acc / scale : acc;
        o_cov[(size_t)r * p + c] = v;
        o_cov[(size_t)c * p + r] = v;
    }
    __syncthreads();
    // total h2 and its SE (total_from_jknife, src/regressions.rs:1565-1610)
    double tv = 0.0;
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int r = e / k, c = e % k;
        tv += m_vec[r] * m_vec[c] * (o_cov[(size_t)r * p + c] / (s.nbar * s.nbar));
    }
    tv = block_sum(tv, red);
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int c = 0; c < k; c++) {
            const double h = est[c] / s.nbar * m_vec[c];
            o_h2[c] = h;
            tot += h;
        }
        o_sc[0] = tot;
        o_sc[1] = sqrt(fmax(tv, 0.0));
        o_sc[2] = jb.fixed ? jb.fixed_int : est[k];
        o_sc[3] = jb.fixed ? NAN : sqrt(fmax(o_cov[(size_t)k * p + k], 0.0));
        o_sc[4] = s.nbar;
        o_sc[5] = s.mean_chi2;
        o_sc[6] = s.n_obs;
    }
}

}  // namespace

cudaError_t launch_partitioned(const PartJob* jobs, PartState* st, const double* l2, uint64_t ld, int k, bool fixed,
                               const double* wld, uint64_t n, int nb, double m_tot, const double* m_vec, double* xtot,
                               bool want_xtot, double* part, double* gram, double* tot, double* sol, double* res,
                               int njobs, cudaStream_t s) {
    const int p = part_params(k, fixed), q = p + 1;
    const int nm = part_qp(q) / MT, gram_ctas = (nm * (nm + 1) / 2 + NT / MT - 1) / (NT / MT);
    const size_t gram_smem = part_gram_smem(q);
    const size_t solve_smem = (size_t)p * (p + 1) * sizeof(double);
    if (solve_smem > (size_t)PART_SOLVE_SMEM) return cudaErrorInvalidValue;
    if (want_xtot) {
        const uint64_t g = (n + NT - 1) / NT;
        k_p_xtot<<<(unsigned)(g < 148 * 8 ? g : 148 * 8), NT, 0, s>>>(l2, ld, k, n, xtot);
    }
    k_p_sums<<<dim3(nb, njobs), NT, 0, s>>>(jobs, xtot, nb, part);
    k_p_aggregate<<<(njobs + 127) / 128, 128, 0, s>>>(jobs, part, nb, m_tot, st, njobs);
    if (gram_smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_p_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem);
        if (e != cudaSuccess) return e;
    }
    k_p_gram<<<dim3(nb, gram_ctas, njobs), NT, gram_smem, s>>>(jobs, st, l2, ld, k, xtot, wld, m_tot, nb, q, gram);
    k_p_total<<<dim3((q * q + NT - 1) / NT, njobs), NT, 0, s>>>(gram, nb, q * q, tot);
    cudaError_t e = cudaFuncSetAttribute(k_p_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem);
    if (e != cudaSuccess) return e;
    k_p_solve<<<dim3(nb + 1, njobs), NT, solve_smem, s>>>(gram, tot, nb, q, sol);
    k_p_finish<<<njobs, NT, (size_t)p * sizeof(double), s>>>(jobs, st, sol, m_vec, nb, k, p, res);
    return cudaGetLastError();
}

cudaError_t preload_partitioned() {
    cudaError_t e = preload_kernel(k_p_xtot);
    if (e == cudaSuccess) e = preload_kernel(k_p_sums);
    if (e == cudaSuccess) e = preload_kernel(k_p_aggregate);
    if (e == cudaSuccess) e = preload_kernel(k_p_gram);
    if (e == cudaSuccess) e = preload_kernel(k_p_total);
    if (e == cudaSuccess) e = preload_kernel(k_p_solve);
    if (e == cudaSuccess) e = preload_kernel(k_p_finish);
    return e;
}

}  // namespace ldsc
