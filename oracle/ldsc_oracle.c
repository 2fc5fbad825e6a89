/*
 * ldsc_oracle.c -- CPU restatement of ldsc-rs's `l2` LD-score path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * library in ldsc_b200/csrc.  Only the test suite, the smoke check and the
 * benchmark's CPU-baseline / reference arm may load it, and only as the
 * checker or as the timed CPU baseline -- never as the product path.
 *
 * It restates, in plain C with OpenMP, the algorithm of the reference's
 * `compute_ldscore_global` (src/l2/compute.rs:1009-2447) and of the pieces
 * it calls:
 *   - BED 2-bit decode, count-A1 LUT [2, missing, 1, 0]   src/bed.rs:470-521
 *   - per-SNP stats and standardisation                     src/l2/normalize.rs:71-154
 *   - per-chromosome window boundaries                      src/l2/window.rs:15-90
 *   - chunk window selection and ring buffer                src/l2/compute.rs:1164-1184,1288-1299
 *   - unbiased r^2 constants                                src/l2/compute.rs:1067-1077
 *   - B^T B / A^T B + r2u fill, diagonal forced to 1        src/l2/compute.rs:1636-1851,1897-2236
 *   - SNP-level masking                                     src/l2/compute.rs:1855-1867,2244-2257
 *   - annotation contraction, pq scaling, all-zero skips    src/l2/compute.rs:1594-1631,1869-1893,1908-1947,2259-2314
 *   - CountSketch bucket/sign stream (fastrand 2.3.0 WyRand, seed 42)
 *                                                           src/l2/compute.rs:178-192,1146-1147
 *   - fused decode->normalise->scatter + ratio renorm       src/l2/compute.rs:601-916, src/wasm_simd.rs:1544-1784
 *   - quadratic sketch-bias inversion (+ MAF-aware)         src/l2/compute.rs:947-998, :514-538
 *   - per-chromosome fan-out vs --global-pass               src/l2/mod.rs:439-575
 *
 * Parity status of the pieces:
 *   - exact f64 / f32 modes: restated from the reference source; pinned by
 *     the reference's known-answer micro BED (src/l2/mod.rs:1191-1225) and
 *     by closed-form checks in tests/.
 *   - CountSketch bucket/sign stream: fastrand 2.3.0 is a third-party crate
 *     (Cargo.lock pins 2.3.0) whose source is not vendored in the reference.
 *     The generator below restates its published WyRand algorithm; no
 *     reference test vector exists for it, so sketch bit-parity with the
 *     reference's `--sketch` output is UNPINNED.
 *   - GEMM summation order follows no particular library (the reference
 *     uses faer 0.24); results agree to rounding, not bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR -1

static void set_err(char *err, int errlen, const char *msg) {
    if (err && errlen > 0) {
        snprintf(err, (size_t)errlen, "%s", msg);
    }
}

/* ------------------------------------------------------------------ */
/* fastrand 2.3.0 WyRand restatement (Rng::with_seed, u32(..d), bool) */
/* ------------------------------------------------------------------ */

typedef struct {
    uint64_t s;
} wyrand_t;

static uint64_t wy_next(wyrand_t *r) {
    r->s += 0x2d358dccaa6c78a5ULL;
    __uint128_t t = (__uint128_t)r->s * (__uint128_t)(r->s ^ 0x8bb84b93962eacc9ULL);
    return (uint64_t)t ^ (uint64_t)(t >> 64);
}

/* Lemire multiply-shift bounded draw with rejection (fastrand gen_mod_u32). */
static uint32_t wy_mod_u32(wyrand_t *r, uint32_t n) {
    uint32_t x = (uint32_t)wy_next(r);
    uint64_t mprod = (uint64_t)x * (uint64_t)n;
    uint32_t lo = (uint32_t)mprod;
    if (lo < n) {
        uint32_t t = (uint32_t)(0u - n) % n;
        while (lo < t) {
            x = (uint32_t)wy_next(r);
            mprod = (uint64_t)x * (uint64_t)n;
            lo = (uint32_t)mprod;
        }
    }
    return (uint32_t)(mprod >> 32);
}

/* fastrand bool(): u8(..) % 2 == 0, u8(..) = low byte of a 32-bit draw. */
static int wy_bool(wyrand_t *r) { return (((uint8_t)(uint32_t)wy_next(r)) & 1u) == 0; }

/* CountSketchProj::new(n_indiv, d, seed): all buckets first, then signs.
 * src/l2/compute.rs:179-184 */
void oracle_countsketch_hash(int64_t n_indiv, uint32_t d, uint64_t seed, uint32_t *bucket,
                             float *sign) {
    wyrand_t r = {seed};
    for (int64_t i = 0; i < n_indiv; i++) bucket[i] = wy_mod_u32(&r, d);
    for (int64_t i = 0; i < n_indiv; i++) sign[i] = wy_bool(&r) ? 1.0f : -1.0f;
}

/* Raw WyRand stream, exposed so tests can check the generator itself. */
void oracle_wyrand_stream(uint64_t seed, int64_t count, uint64_t *out) {
    wyrand_t r = {seed};
    for (int64_t i = 0; i < count; i++) out[i] = wy_next(&r);
}

/* ------------------------------------------------------------------ */
/* Window boundaries (src/l2/window.rs:15-90)                          */
/* ------------------------------------------------------------------ */

/* mode: 0 = cM, 1 = kb (bp/1000), 2 = SNP count. Returns any_full_chr_window. */
int oracle_block_lefts(int64_t m, const uint8_t *chr, const double *cm, const uint32_t *bp,
                       int mode, double wind, int64_t half, int64_t *bl) {
    int any_full = 0;
    int64_t start = 0;
    while (start < m) {
        uint8_t c = chr[start];
        int64_t end = start + 1;
        while (end < m && chr[end] == c) end++;
        int64_t len = end - start;
        if (mode == 2) {
            if (half >= (len > 0 ? len - 1 : 0)) any_full = 1;
            for (int64_t i = 0; i < len; i++) bl[start + i] = start + (i > half ? i - half : 0);
        } else {
            int64_t j = 0;
            for (int64_t i = 0; i < len; i++) {
                double ci = mode == 0 ? cm[start + i] : (double)bp[start + i] / 1000.0;
                for (;;) {
                    if (j >= len) break;
                    double cj = mode == 0 ? cm[start + j] : (double)bp[start + j] / 1000.0;
                    if (fabs(ci - cj) > wind) {
                        j++;
                    } else {
                        break;
                    }
                }
                bl[start + i] = start + j;
            }
            if (len > 0 && bl[end - 1] == start) any_full = 1;
        }
        start = end;
    }
    return any_full;
}

/* ------------------------------------------------------------------ */
/* Decode + per-SNP stats                                              */
/* ------------------------------------------------------------------ */

/* count-A1 code -> genotype; -1 for missing (src/bed.rs:470-476) */
static inline int code_geno(int code) {
    static const int lut[4] = {2, -1, 1, 0};
    return lut[code & 3];
}

static inline int geno_at(const uint8_t *row, int64_t iid) {
    return code_geno((row[iid >> 2] >> ((iid & 3) * 2)) & 3);
}

/* Integer sums of the non-missing genotypes of one SNP row over the kept
 * individuals: sum, count, sum of squares, sum of cubes, sum of 4th powers
 * (src/l2/compute.rs:334-512). */
static void snp_moments(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv, int64_t *s,
                        int64_t *n, int64_t *q, int64_t *q3, int64_t *q4) {
    int64_t ss = 0, nn = 0, qq = 0, c3 = 0, c4 = 0;
    for (int64_t i = 0; i < n_indiv; i++) {
        int g = geno_at(row, iid_idx ? iid_idx[i] : i);
        if (g < 0) continue;
        ss += g;
        nn += 1;
        qq += g * g;
        c3 += g * g * g;
        c4 += g * g * g * g;
    }
    *s = ss;
    *n = nn;
    *q = qq;
    if (q3) *q3 = c3;
    if (q4) *q4 = c4;
}

/* per_snp_kappa (src/l2/compute.rs:525-538) */
static double per_snp_kappa(int64_t sum, int64_t count, int64_t sum_sq, int64_t sum_cube,
                            int64_t sum_4th) {
    if (count == 0) return 0.0;
    double count_f = (double)count;
    double mean = (double)sum / count_f;
    double m4 = (double)sum_4th - 4.0 * mean * (double)sum_cube +
                6.0 * mean * mean * (double)sum_sq - 3.0 * pow(mean, 4) * count_f;
    double css = (double)sum_sq - count_f * mean * mean;
    if (css <= 0.0) return 0.0;
    return m4 / (css * css);
}

/* per_snp_kappa_from_col_f32 (src/l2/compute.rs:547-560), raw genotypes */
static double per_snp_kappa_from_col(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv,
                                     double mean, double css) {
    if (css <= 0.0) return 0.0;
    double m4 = 0.0;
    for (int64_t i = 0; i < n_indiv; i++) {
        int g = geno_at(row, iid_idx ? iid_idx[i] : i);
        if (g < 0) continue;
        double d = (double)g - mean;
        double d2 = d * d;
        m4 += d2 * d2;
    }
    return m4 / (css * css);
}

/* Standardise one SNP into an f64 column (normalize_col_f64_with_stats,
 * src/l2/normalize.rs:71-110).  Returns MAF. */
static double standardize_f64(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv,
                              double *col) {
    int64_t s, n, q;
    snp_moments(row, iid_idx, n_indiv, &s, &n, &q, NULL, NULL);
    double avg = n > 0 ? (double)s / (double)n : 0.0;
    double freq = avg / 2.0;
    if (freq < 0.0) freq = 0.0;
    if (freq > 1.0) freq = 1.0;
    double maf = freq < 1.0 - freq ? freq : 1.0 - freq;
    double css = (double)q - (double)n * avg * avg;
    double var = css / (double)n_indiv;
    double sd = sqrt(var);
    double inv = sd > 0.0 ? 1.0 / sd : 0.0;
    for (int64_t i = 0; i < n_indiv; i++) {
        int g = geno_at(row, iid_idx ? iid_idx[i] : i);
        col[i] = g < 0 ? 0.0 : ((double)g - avg) * inv;
    }
    return maf;
}

/* normalize_col_f32_with_stats (src/l2/normalize.rs:115-154).  Returns the
 * MAF rounded through f32, as the reference's f32 path does. */
static double standardize_f32(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv,
                              float *col) {
    int64_t s, n, q;
    snp_moments(row, iid_idx, n_indiv, &s, &n, &q, NULL, NULL);
    double avg = n > 0 ? (double)s / (double)n : 0.0;
    double freq = avg / 2.0;
    if (freq < 0.0) freq = 0.0;
    if (freq > 1.0) freq = 1.0;
    double maf = freq < 1.0 - freq ? freq : 1.0 - freq;
    double css = (double)q - (double)n * avg * avg;
    double var = css / (double)n_indiv;
    double sd = sqrt(var);
    float inv = sd > 0.0 ? (float)(1.0 / sd) : 0.0f;
    float avg32 = (float)avg;
    for (int64_t i = 0; i < n_indiv; i++) {
        int g = geno_at(row, iid_idx ? iid_idx[i] : i);
        col[i] = g < 0 ? 0.0f : ((float)g - avg32) * inv;
    }
    return (double)(float)maf;
}

/* ------------------------------------------------------------------ */
/* CountSketch scatter (src/wasm_simd.rs:1544-1784, compute.rs:601-916) */
/* ------------------------------------------------------------------ */

/* One column, f32 path: LUT value (code - mean) * inv_std in f32, missing
 * -> 0, scatter-add in individual order, then rescale so ||col||^2 = n_norm
 * with the squared norm accumulated in f64. */
void oracle_scatter_column_f32(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv,
                               const uint32_t *bucket, const float *sign, float mean,
                               float inv_std, double n_norm, int64_t d, float *out) {
    float code_vals[4] = {(2.0f - mean) * inv_std, 0.0f, (1.0f - mean) * inv_std,
                          -mean * inv_std};
    for (int64_t b = 0; b < d; b++) out[b] = 0.0f;
    for (int64_t i = 0; i < n_indiv; i++) {
        int64_t iid = iid_idx ? iid_idx[i] : i;
        int code = (row[iid >> 2] >> ((iid & 3) * 2)) & 3;
        out[bucket[i]] += sign[i] * code_vals[code];
    }
    double nrm = 0.0;
    for (int64_t b = 0; b < d; b++) nrm += (double)out[b] * (double)out[b];
    if (nrm > 0.0) {
        float scale = (float)sqrt(n_norm / nrm);
        for (int64_t b = 0; b < d; b++) out[b] *= scale;
    }
}

static void scatter_column_f64(const uint8_t *row, const int64_t *iid_idx, int64_t n_indiv,
                               const uint32_t *bucket, const double *sign, double mean,
                               double inv_std, double n_norm, int64_t d, double *out) {
    double code_vals[4] = {(2.0 - mean) * inv_std, 0.0, (1.0 - mean) * inv_std,
                           -mean * inv_std};
    for (int64_t b = 0; b < d; b++) out[b] = 0.0;
    for (int64_t i = 0; i < n_indiv; i++) {
        int64_t iid = iid_idx ? iid_idx[i] : i;
        int code = (row[iid >> 2] >> ((iid & 3) * 2)) & 3;
        out[bucket[i]] += sign[i] * code_vals[code];
    }
    double nrm = 0.0;
    for (int64_t b = 0; b < d; b++) nrm += out[b] * out[b];
    if (nrm > 0.0) {
        double scale = sqrt(n_norm / nrm);
        for (int64_t b = 0; b < d; b++) out[b] *= scale;
    }
}

/* quadratic_sketch_correction[_maf_aware] (src/l2/compute.rs:947-998) */
static inline double quad_corr(double val, double n_inv_sq, double d_f, double a, double b,
                               double kj, double kk) {
    double tilde = val * val * n_inv_sq;
    double dm3 = d_f - 3.0 - 2.0 * (kj + kk);
    double disc = dm3 * dm3 + 8.0 * (d_f * tilde - 1.0);
    double r2 = disc >= 0.0 ? (-dm3 + sqrt(disc)) * 0.25 : 0.0;
    return r2 * a + b;
}

/* ------------------------------------------------------------------ */
/* Column Gram kernels: out[w x c] = A^T B over gemm_n rows             */
/* ------------------------------------------------------------------ */

typedef double v4d __attribute__((vector_size(32)));
typedef float v8f __attribute__((vector_size(32)));

static inline v4d ld4d(const double *p) {
    v4d v;
    memcpy(&v, p, sizeof(v));
    return v;
}
static inline v8f ld8f(const float *p) {
    v8f v;
    memcpy(&v, p, sizeof(v));
    return v;
}

/* Cache-blocked column Gram.  Each thread owns a macro tile of GB_W A columns
 * x GB_C B columns and walks the individual axis in chunks of GB_K: a chunk
 * of the macro tile's columns (GB_W + GB_C columns x 2 KB) stays in the
 * core's L2 while every register block of the tile reads it, so a column is
 * fetched from memory once per chunk instead of once per register block.
 * With AVX2 the register blocks are 3 x 4 dot products vectorised along the
 * individual axis (scalar tails); with AVX-512 the A chunk is packed and a
 * 16 x 8 outer-product micro kernel runs over it (gram_f64_packed).
 * Summation order differs from faer's, as any blocked GEMM's would. */
#ifndef GB_W
#define GB_W 64
#endif
#ifndef GB_C
#define GB_C 64
#endif
#ifndef GB_K
#define GB_K 256
#endif

/* 8-double vectors for hosts with AVX-512 (chosen at run time). */
typedef double v8d __attribute__((vector_size(64)));

/* Packed form for hosts with AVX-512: per macro tile and chunk of GB_K
 * individuals, the tile's A columns are packed into 16-row panels (for each
 * individual, 16 consecutive output rows contiguous), and a 16 x 8 micro
 * kernel keeps 16 accumulators: per individual two panel loads, eight
 * broadcasts of B and sixteen vector FMAs, with no horizontal sums.  Output
 * rows past the tile are zero-padded in the panels and not stored. */
#define PK_R 16
#define PK_C 8
__attribute__((target("avx512f"))) static void gram_f64_packed(int64_t n, int64_t w, int64_t c,
                                                               double *const *acol, double *const *bcol,
                                                               double *out) {
    const int64_t nwt = (w + GB_W - 1) / GB_W, nct = (c + GB_C - 1) / GB_C;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int64_t ct = 0; ct < nct; ct++) {
        for (int64_t wt = 0; wt < nwt; wt++) {
            const int64_t i0 = wt * GB_W, i1 = i0 + GB_W < w ? i0 + GB_W : w;
            const int64_t j0 = ct * GB_C, j1 = j0 + GB_C < c ? j0 + GB_C : c;
            const int64_t nr = i1 - i0, np = (nr + PK_R - 1) / PK_R;
            double tile[GB_W * GB_C];
            memset(tile, 0, sizeof(tile));
            static __thread double pa[GB_W * GB_K] __attribute__((aligned(64)));
            for (int64_t k0 = 0; k0 < n; k0 += GB_K) {
                const int64_t kc = (k0 + GB_K < n ? k0 + GB_K : n) - k0;
                /* pack: panel p, individual kk, row r at pa[(p * GB_K + kk) * PK_R + r] */
                for (int64_t p = 0; p < np; p++)
                    for (int64_t r = 0; r < PK_R; r++) {
                        const int64_t i = i0 + p * PK_R + r;
                        double *dst = pa + (p * GB_K) * PK_R + r;
                        if (i < i1) {
                            const double *src = acol[i] + k0;
                            for (int64_t kk = 0; kk < kc; kk++) dst[kk * PK_R] = src[kk];
                        } else {
                            for (int64_t kk = 0; kk < kc; kk++) dst[kk * PK_R] = 0.0;
                        }
                    }
                for (int64_t jb = j0; jb < j1; jb += PK_C) {
                    const int64_t je = jb + PK_C < j1 ? jb + PK_C : j1;
                    const double *bp[PK_C];
                    for (int t = 0; t < PK_C; t++) bp[t] = bcol[jb + t < je ? jb + t : jb] + k0;
                    for (int64_t p = 0; p < np; p++) {
                        const double *ap = pa + (p * GB_K) * PK_R;
                        v8d acc0[PK_C], acc1[PK_C];
                        memset(acc0, 0, sizeof(acc0));
                        memset(acc1, 0, sizeof(acc1));
                        for (int64_t kk = 0; kk < kc; kk++) {
                            v8d a0, a1;
                            memcpy(&a0, ap + kk * PK_R, sizeof(v8d));
                            memcpy(&a1, ap + kk * PK_R + 8, sizeof(v8d));
                            for (int t = 0; t < PK_C; t++) {
                                const double bv = bp[t][kk];
                                const v8d b = {bv, bv, bv, bv, bv, bv, bv, bv};
                                acc0[t] += a0 * b;
                                acc1[t] += a1 * b;
                            }
                        }
                        for (int64_t j = jb; j < je; j++) {
                            double *trow = tile + (j - j0) * GB_W + p * PK_R;
                            const int64_t rmax = nr - p * PK_R < PK_R ? nr - p * PK_R : PK_R;
                            for (int64_t r = 0; r < rmax; r++)
                                trow[r] += r < 8 ? acc0[j - jb][r] : acc1[j - jb][r - 8];
                        }
                    }
                }
            }
            for (int64_t j = j0; j < j1; j++)
                for (int64_t i = i0; i < i1; i++) out[i + j * w] = tile[(i - i0) + (j - j0) * GB_W];
        }
    }
}

static void gram_f64(int64_t n, int64_t w, int64_t c, double *const *acol, double *const *bcol,
                     double *out) {
    if (__builtin_cpu_supports("avx512f")) {
        gram_f64_packed(n, w, c, acol, bcol, out);
        return;
    }
    const int64_t nwt = (w + GB_W - 1) / GB_W, nct = (c + GB_C - 1) / GB_C;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int64_t ct = 0; ct < nct; ct++) {
        for (int64_t wt = 0; wt < nwt; wt++) {
            const int64_t i0 = wt * GB_W, i1 = i0 + GB_W < w ? i0 + GB_W : w;
            const int64_t j0 = ct * GB_C, j1 = j0 + GB_C < c ? j0 + GB_C : c;
            double tile[GB_W * GB_C];
            memset(tile, 0, sizeof(tile));
            for (int64_t k0 = 0; k0 < n; k0 += GB_K) {
                const int64_t k1 = k0 + GB_K < n ? k0 + GB_K : n;
                const int64_t kv = k0 + ((k1 - k0) & ~(int64_t)3);
                for (int64_t jb = j0; jb < j1; jb += 4) {
                    for (int64_t ib = i0; ib < i1; ib += 3) {
                        /* 3 x 4 register block: 12 accumulators, 3 A vectors, 1 B vector */
                        const int64_t ie = ib + 3 < i1 ? ib + 3 : i1;
                        const int64_t je = jb + 4 < j1 ? jb + 4 : j1;
                        const double *ap[3], *bp[4];
                        for (int t = 0; t < 3; t++) ap[t] = acol[ib + t < ie ? ib + t : ib];
                        for (int t = 0; t < 4; t++) bp[t] = bcol[jb + t < je ? jb + t : jb];
                        v4d acc[3][4];
                        memset(acc, 0, sizeof(acc));
                        for (int64_t k = k0; k < kv; k += 4) {
                            const v4d a0 = ld4d(ap[0] + k), a1 = ld4d(ap[1] + k), a2 = ld4d(ap[2] + k);
                            v4d b = ld4d(bp[0] + k);
                            acc[0][0] += a0 * b; acc[1][0] += a1 * b; acc[2][0] += a2 * b;
                            b = ld4d(bp[1] + k);
                            acc[0][1] += a0 * b; acc[1][1] += a1 * b; acc[2][1] += a2 * b;
                            b = ld4d(bp[2] + k);
                            acc[0][2] += a0 * b; acc[1][2] += a1 * b; acc[2][2] += a2 * b;
                            b = ld4d(bp[3] + k);
                            acc[0][3] += a0 * b; acc[1][3] += a1 * b; acc[2][3] += a2 * b;
                        }
                        for (int64_t i = ib; i < ie; i++)
                            for (int64_t j = jb; j < je; j++) {
                                v4d v = acc[i - ib][j - jb];
                                double s = (v[0] + v[1]) + (v[2] + v[3]);
                                for (int64_t k = kv; k < k1; k++) s += ap[i - ib][k] * bp[j - jb][k];
                                tile[(i - i0) + (j - j0) * GB_W] += s;
                            }
                    }
                }
            }
            for (int64_t j = j0; j < j1; j++)
                for (int64_t i = i0; i < i1; i++) out[i + j * w] = tile[(i - i0) + (j - j0) * GB_W];
        }
    }
}

static void gram_f32(int64_t n, int64_t w, int64_t c, float *const *acol, float *const *bcol,
                     float *out) {
    int64_t nv = n & ~(int64_t)7;
#pragma omp parallel for collapse(2) schedule(dynamic, 2)
    for (int64_t jb = 0; jb < c; jb += 4) {
        for (int64_t ib = 0; ib < w; ib += 2) {
            int64_t ie = ib + 2 < w ? ib + 2 : w;
            int64_t je = jb + 4 < c ? jb + 4 : c;
            const float *ap[2], *bp[4];
            for (int t = 0; t < 2; t++) ap[t] = acol[ib + t < ie ? ib + t : ib];
            for (int t = 0; t < 4; t++) bp[t] = bcol[jb + t < je ? jb + t : jb];
            v8f acc[2][4];
            memset(acc, 0, sizeof(acc));
            for (int64_t k = 0; k < nv; k += 8) {
                v8f a0 = ld8f(ap[0] + k), a1 = ld8f(ap[1] + k);
                v8f b0 = ld8f(bp[0] + k), b1 = ld8f(bp[1] + k);
                v8f b2 = ld8f(bp[2] + k), b3 = ld8f(bp[3] + k);
                acc[0][0] += a0 * b0; acc[0][1] += a0 * b1; acc[0][2] += a0 * b2; acc[0][3] += a0 * b3;
                acc[1][0] += a1 * b0; acc[1][1] += a1 * b1; acc[1][2] += a1 * b2; acc[1][3] += a1 * b3;
            }
            for (int64_t i = ib; i < ie; i++)
                for (int64_t j = jb; j < je; j++) {
                    v8f v = acc[i - ib][j - jb];
                    float s = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
                    for (int64_t k = nv; k < n; k++) s += ap[i - ib][k] * bp[j - jb][k];
                    out[i + j * w] = s;
                }
        }
    }
}

/* ------------------------------------------------------------------ */
/* compute_ldscore_global restatement                                  */
/* ------------------------------------------------------------------ */

typedef struct {
    const uint8_t *bed;      /* BED body (no magic), SNP-major */
    int64_t bpr;             /* bytes per SNP row = ceil(n_file_indiv / 4) */
    int64_t n_file_indiv;    /* individuals in the .fam */
    const int64_t *iid_idx;  /* kept individuals (--keep), NULL = all */
    int64_t n_indiv;         /* number of kept individuals */
    int64_t m;               /* SNP records */
    const int64_t *bed_idx;  /* BED row of each record */
    const uint8_t *chr;
    const double *cm;
    const uint32_t *bp;
    int mode;                /* 0 cM, 1 kb, 2 SNP */
    double wind;
    int64_t wind_snp;
    int64_t chunk_c;
    const double *annot;     /* m x K column-major, NULL = all ones (K = 1) */
    int64_t K;
    int has_pq;
    double pq_exp;
    int use_f32;
    int64_t sketch_d;        /* 0 = exact */
    int sketch_maf_aware;
    int masking;             /* --snp-level-masking */
    int per_chr;             /* 1 = per-chromosome fan-out, 0 = --global-pass */
    int n_threads;           /* 0 = OpenMP default */
} oracle_l2_args;

typedef struct {
    int64_t n_pairs;         /* off-diagonal pairs contributing to l2 in this mode */
    int any_full_chr_window;
    int64_t n_dots;          /* column dot products the chunk Grams computed (w x c + c x c per chunk) */
    double gemm_secs;        /* wall time inside the chunk Grams */
} oracle_l2_info;

/* Work and time of the chunk Grams of the current oracle_l2 call (the chunk
 * loop calls them one at a time; each Gram is parallel inside). */
static int64_t g_dots;
static double g_gemm_secs;

static double wall_secs(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* One compute_ldscore_global call over records [r0, r0 + m). */
static int compute_global(const oracle_l2_args *a, int64_t r0, int64_t m, double *l2, int64_t ldl,
                          double *maf_out, int64_t *pairs, int *any_full, char *err, int errlen) {
    int64_t chunk_c = a->chunk_c;
    int64_t n_indiv = a->n_indiv;
    int64_t K = a->annot ? a->K : 1;
    if (m == 0) return OR_OK;

    int64_t *bl = (int64_t *)malloc(sizeof(int64_t) * m);
    int full = oracle_block_lefts(m, a->chr + r0, a->cm ? a->cm + r0 : NULL,
                                  a->bp ? a->bp + r0 : NULL, a->mode, a->wind, a->wind_snp, bl);
    if (full) *any_full = 1;

    double n = (double)n_indiv;
    double n_inv = 1.0 / n;
    double r2u_denom = n_indiv > 2 ? n - 2.0 : n;
    double r2u_denom_inv = 1.0 / r2u_denom;
    double r2u_a = 1.0 + r2u_denom_inv;
    double r2u_b = -r2u_denom_inv;
    double n_inv_sq_r2u_a = n_inv * n_inv * r2u_a;
    double n_inv_sq = n_inv * n_inv;

    int64_t d = a->sketch_d;
    if (d > 0 && !(d >= 3 && d < n_indiv)) {
        free(bl);
        set_err(err, errlen, "--sketch is out of bounds (must be 3 <= d < n_indiv)");
        return OR_ERR;
    }
    int64_t gemm_n = d > 0 ? d : n_indiv;
    double quad_d_f = (double)d;
    int use_f32 = a->use_f32;
    int maf_aware = a->sketch_maf_aware && d > 0;

    uint32_t *bucket = NULL;
    float *sign32 = NULL;
    double *sign64 = NULL;
    if (d > 0) {
        bucket = (uint32_t *)malloc(sizeof(uint32_t) * n_indiv);
        sign32 = (float *)malloc(sizeof(float) * n_indiv);
        sign64 = (double *)malloc(sizeof(double) * n_indiv);
        oracle_countsketch_hash(n_indiv, (uint32_t)d, 42, bucket, sign32);
        for (int64_t i = 0; i < n_indiv; i++) sign64[i] = (double)sign32[i];
    }

    /* block sizes / ring (src/l2/compute.rs:1164-1181) */
    int64_t max_window = 0;
    int64_t *block_sizes = (int64_t *)malloc(sizeof(int64_t) * m);
    for (int64_t i = 0; i < m; i++) {
        int64_t dist = i - bl[i];
        block_sizes[i] = dist == 0 ? 0 : ((dist + chunk_c - 1) / chunk_c) * chunk_c;
        if (block_sizes[i] > max_window) max_window = block_sizes[i];
    }
    int64_t ring_size = max_window + 8 * chunk_c;
    if (ring_size < 1) ring_size = 1;
    ring_size = ((ring_size + chunk_c - 1) / chunk_c) * chunk_c;

    size_t esz = use_f32 ? sizeof(float) : sizeof(double);
    char *ring = (char *)calloc((size_t)gemm_n * (size_t)ring_size, esz);
    double *kurt = maf_aware ? (double *)calloc((size_t)m, sizeof(double)) : NULL;
    double *pq = a->has_pq ? (double *)malloc(sizeof(double) * m) : NULL;
    if (pq)
        for (int64_t i = 0; i < m; i++) pq[i] = 1.0;
    double *r2u_bb = (double *)malloc(sizeof(double) * chunk_c * chunk_c);
    double *r2u_ab = (double *)malloc(sizeof(double) * (max_window > 0 ? max_window : 1) * chunk_c);
    void *gbuf = malloc(esz * (size_t)(max_window > chunk_c ? max_window : chunk_c) * chunk_c);
    double *ann_c = (double *)malloc(sizeof(double) * chunk_c * K);
    double *ann_w = (double *)malloc(sizeof(double) * (max_window > 0 ? max_window : 1) * K);
    void **acol = (void **)malloc(sizeof(void *) * (max_window > 0 ? max_window : 1));
    void **bcol = (void **)malloc(sizeof(void *) * chunk_c);
    /* non-fused sketch path needs an N x 1 staging column per SNP */
    float *stage32 = (d > 0 && use_f32) ? (float *)malloc(sizeof(float) * n_indiv * chunk_c) : NULL;
    double *stage64 = (d > 0 && !use_f32) ? (double *)malloc(sizeof(double) * n_indiv * chunk_c) : NULL;

    int64_t npairs = 0;
    for (int64_t cs = 0; cs < m; cs += chunk_c) {
        int64_t ce = cs + chunk_c < m ? cs + chunk_c : m;
        int64_t c = ce - cs;
        int64_t b = block_sizes[cs];
        if (b > cs) b = cs;
        int64_t a_left = cs - b;
        int64_t w = cs - a_left;

        /* pair count for the r^2-pairs/sec numerator */
        if (a->masking) {
            for (int64_t j = cs; j < ce; j++) npairs += j - bl[j];
        } else {
            npairs += w * c + c * (c - 1) / 2;
        }

        /* contiguous-BED test for the fused sketch path (compute.rs:1308-1318) */
        int contiguous = a->bed_idx[r0 + ce - 1] == a->bed_idx[r0 + cs] + c - 1;

        /* ---- decode + normalise (+ sketch) the chunk into ring slots ---- */
        for (int64_t j = 0; j < c; j++) {
            int64_t slot = (cs + j) % ring_size;
            bcol[j] = ring + (size_t)slot * (size_t)gemm_n * esz;
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t j = 0; j < c; j++) {
            int64_t rec = r0 + cs + j;
            const uint8_t *row = a->bed + (size_t)a->bed_idx[rec] * (size_t)a->bpr;
            if (d == 0) {
                if (use_f32)
                    maf_out[cs + j] = standardize_f32(row, a->iid_idx, n_indiv, (float *)bcol[j]);
                else
                    maf_out[cs + j] = standardize_f64(row, a->iid_idx, n_indiv, (double *)bcol[j]);
                continue;
            }
            int64_t s, nn, q, q3, q4;
            snp_moments(row, a->iid_idx, n_indiv, &s, &nn, &q, &q3, &q4);
            double mean = nn > 0 ? (double)s / (double)nn : 0.0;
            double freq = mean / 2.0;
            if (freq < 0.0) freq = 0.0;
            if (freq > 1.0) freq = 1.0;
            double maf = freq < 1.0 - freq ? freq : 1.0 - freq;
            double css = (double)q - (double)nn * mean * mean;
            double var = css / (double)n_indiv;
            double sd = sqrt(var);
            if (contiguous) {
                /* fused path: MAF in f64, kappa from byte moments */
                maf_out[cs + j] = maf;
                if (maf_aware) kurt[cs + j] = per_snp_kappa(s, nn, q, q3, q4);
                if (use_f32) {
                    float inv = sd > 0.0 ? (float)(1.0 / sd) : 0.0f;
                    oracle_scatter_column_f32(row, a->iid_idx, n_indiv, bucket, sign32,
                                              (float)mean, inv, n, d, (float *)bcol[j]);
                } else {
                    double inv = sd > 0.0 ? 1.0 / sd : 0.0;
                    scatter_column_f64(row, a->iid_idx, n_indiv, bucket, sign64, mean, inv, n, d,
                                       (double *)bcol[j]);
                }
            } else {
                /* standard path: normalise into a full column, then project.  The
                 * f32 normalise returns its MAF through f32. */
                if (maf_aware) kurt[cs + j] = per_snp_kappa_from_col(row, a->iid_idx, n_indiv, mean, css);
                if (use_f32) {
                    float *col = stage32 + (size_t)j * n_indiv;
                    maf_out[cs + j] = standardize_f32(row, a->iid_idx, n_indiv, col);
                    float *dst = (float *)bcol[j];
                    for (int64_t bb = 0; bb < d; bb++) dst[bb] = 0.0f;
                    for (int64_t i = 0; i < n_indiv; i++) dst[bucket[i]] += sign32[i] * col[i];
                    double nrm = 0.0;
                    for (int64_t bb = 0; bb < d; bb++) nrm += (double)dst[bb] * (double)dst[bb];
                    if (nrm > 0.0) {
                        float scale = (float)sqrt(n / nrm);
                        for (int64_t bb = 0; bb < d; bb++) dst[bb] *= scale;
                    }
                } else {
                    double *col = stage64 + (size_t)j * n_indiv;
                    maf_out[cs + j] = standardize_f64(row, a->iid_idx, n_indiv, col);
                    double *dst = (double *)bcol[j];
                    for (int64_t bb = 0; bb < d; bb++) dst[bb] = 0.0;
                    for (int64_t i = 0; i < n_indiv; i++) dst[bucket[i]] += sign64[i] * col[i];
                    double nrm = 0.0;
                    for (int64_t bb = 0; bb < d; bb++) nrm += dst[bb] * dst[bb];
                    if (nrm > 0.0) {
                        double scale = sqrt(n / nrm);
                        for (int64_t bb = 0; bb < d; bb++) dst[bb] *= scale;
                    }
                }
            }
        }
        if (pq) {
            for (int64_t j = 0; j < c; j++) {
                double mf = maf_out[cs + j];
                pq[cs + j] = pow(mf * (1.0 - mf), a->pq_exp);
            }
        }

        /* ---- effective annotation for chunk ---- */
        int chunk_all_zero = 1;
        for (int64_t k = 0; k < K; k++)
            for (int64_t j = 0; j < c; j++) {
                double v = a->annot ? a->annot[(r0 + cs + j) + k * a->m] : 1.0;
                if (pq) v *= pq[cs + j];
                ann_c[j + k * c] = v;
                if (v != 0.0) chunk_all_zero = 0;
            }

        /* ---- B x B (compute.rs:1636-1895) ---- */
        if (!chunk_all_zero) {
            if (use_f32) {
                float *bb = (float *)gbuf;
                gram_f32(gemm_n, c, c, (float *const *)bcol, (float *const *)bcol, bb);
                for (int64_t x = 0; x < c * c; x++) r2u_bb[x] = (double)bb[x];
            } else {
                double *bb = (double *)gbuf;
                const double t0 = wall_secs();
                gram_f64(gemm_n, c, c, (double *const *)bcol, (double *const *)bcol, bb);
                g_gemm_secs += wall_secs() - t0;
                g_dots += c * c;
                for (int64_t x = 0; x < c * c; x++) r2u_bb[x] = bb[x];
            }
            /* fill: diagonal 1, off-diagonal from the (k, j) entry, symmetric */
            for (int64_t j = 0; j < c; j++) {
                for (int64_t k = 0; k < j; k++) {
                    double val = r2u_bb[k + j * c];
                    double r;
                    if (d > 0) {
                        double kj = maf_aware ? kurt[cs + j] : 0.0;
                        double kk = maf_aware ? kurt[cs + k] : 0.0;
                        r = quad_corr(val, n_inv_sq, quad_d_f, r2u_a, r2u_b, kj, kk);
                    } else {
                        r = val * val * n_inv_sq_r2u_a + r2u_b;
                    }
                    r2u_bb[j + k * c] = r;
                }
            }
            for (int64_t j = 0; j < c; j++) {
                r2u_bb[j + j * c] = 1.0;
                for (int64_t k = 0; k < j; k++) r2u_bb[k + j * c] = r2u_bb[j + k * c];
            }
            if (a->masking) {
                for (int64_t j = 1; j < c; j++) {
                    int64_t bl_j = bl[cs + j];
                    if (bl_j <= cs) continue;
                    int64_t cutoff = bl_j - cs;
                    int64_t lim = cutoff < j ? cutoff : j;
                    for (int64_t k = 0; k < lim; k++) {
                        r2u_bb[j + k * c] = 0.0;
                        r2u_bb[k + j * c] = 0.0;
                    }
                }
            }
            /* l2[chunk] += R_bb * A_chunk */
            for (int64_t kk = 0; kk < K; kk++)
                for (int64_t j = 0; j < c; j++) {
                    double acc = 0.0;
                    for (int64_t t = 0; t < c; t++) acc += r2u_bb[j + t * c] * ann_c[t + kk * c];
                    l2[(cs + j) + kk * ldl] += acc;
                }
        }

        /* ---- A x B (compute.rs:1897-2318) ---- */
        if (w > 0) {
            int window_all_zero = 1;
            for (int64_t k = 0; k < K; k++)
                for (int64_t i = 0; i < w; i++) {
                    int64_t g = a_left + i;
                    double v = a->annot ? a->annot[(r0 + g) + k * a->m] : 1.0;
                    if (pq) v *= pq[g];
                    ann_w[i + k * w] = v;
                    if (v != 0.0) window_all_zero = 0;
                }
            if (!(chunk_all_zero && window_all_zero)) {
                for (int64_t i = 0; i < w; i++) {
                    int64_t slot = (a_left + i) % ring_size;
                    acol[i] = ring + (size_t)slot * (size_t)gemm_n * esz;
                }
                if (use_f32) {
                    float *ab = (float *)gbuf;
                    gram_f32(gemm_n, w, c, (float *const *)acol, (float *const *)bcol, ab);
                    for (int64_t x = 0; x < w * c; x++) r2u_ab[x] = (double)ab[x];
                } else {
                    double *ab = (double *)gbuf;
                    const double t0 = wall_secs();
                    gram_f64(gemm_n, w, c, (double *const *)acol, (double *const *)bcol, ab);
                    g_gemm_secs += wall_secs() - t0;
                    g_dots += w * c;
                    for (int64_t x = 0; x < w * c; x++) r2u_ab[x] = ab[x];
                }
                for (int64_t j = 0; j < c; j++)
                    for (int64_t i = 0; i < w; i++) {
                        double val = r2u_ab[i + j * w];
                        if (d > 0) {
                            double ka = maf_aware ? kurt[a_left + i] : 0.0;
                            double kb = maf_aware ? kurt[cs + j] : 0.0;
                            r2u_ab[i + j * w] = quad_corr(val, n_inv_sq, quad_d_f, r2u_a, r2u_b, ka, kb);
                        } else {
                            r2u_ab[i + j * w] = val * val * n_inv_sq_r2u_a + r2u_b;
                        }
                    }
                if (a->masking) {
                    int64_t cutoff_row = 0;
                    for (int64_t j = 0; j < c; j++) {
                        int64_t bl_j = bl[cs + j];
                        while (cutoff_row < w && a_left + cutoff_row < bl_j) cutoff_row++;
                        for (int64_t i = 0; i < cutoff_row; i++) r2u_ab[i + j * w] = 0.0;
                    }
                }
                if (!chunk_all_zero) {
                    /* l2[window] += R_ab * A_chunk */
                    for (int64_t kk = 0; kk < K; kk++)
                        for (int64_t i = 0; i < w; i++) {
                            double acc = 0.0;
                            for (int64_t j = 0; j < c; j++) acc += r2u_ab[i + j * w] * ann_c[j + kk * c];
                            l2[(a_left + i) + kk * ldl] += acc;
                        }
                }
                if (!window_all_zero) {
                    /* l2[chunk] += R_ab^T * A_window */
                    for (int64_t kk = 0; kk < K; kk++)
                        for (int64_t j = 0; j < c; j++) {
                            double acc = 0.0;
                            for (int64_t i = 0; i < w; i++) acc += r2u_ab[i + j * w] * ann_w[i + kk * w];
                            l2[(cs + j) + kk * ldl] += acc;
                        }
                }
            }
        }
    }
    *pairs += npairs;

    free(bl);
    free(block_sizes);
    free(ring);
    free(kurt);
    free(pq);
    free(r2u_bb);
    free(r2u_ab);
    free(gbuf);
    free(ann_c);
    free(ann_w);
    free(acol);
    free(bcol);
    free(stage32);
    free(stage64);
    free(bucket);
    free(sign32);
    free(sign64);
    return OR_OK;
}

/* Full l2 pass: per-chromosome fan-out (default) or one global pass.
 * l2_out is m x K column-major (K = 1 when annot is NULL). */
int oracle_l2(const oracle_l2_args *a, double *l2_out, double *maf_out, oracle_l2_info *info,
              char *err, int errlen) {
    if (a->chunk_c < 1) {
        set_err(err, errlen, "compute_ldscore_global: chunk_size must be >= 1");
        return OR_ERR;
    }
    if (a->n_indiv < 1) {
        set_err(err, errlen, "n_indiv must be >= 1");
        return OR_ERR;
    }
#ifdef _OPENMP
    if (a->n_threads > 0) omp_set_num_threads(a->n_threads);
#endif
    int64_t K = a->annot ? a->K : 1;
    memset(l2_out, 0, sizeof(double) * (size_t)(a->m * K));
    int64_t pairs = 0;
    int any_full = 0;
    g_dots = 0;
    g_gemm_secs = 0.0;
    if (!a->per_chr) {
        int rc = compute_global(a, 0, a->m, l2_out, a->m, maf_out, &pairs, &any_full, err, errlen);
        if (rc) return rc;
    } else {
        int64_t start = 0;
        while (start < a->m) {
            int64_t end = start + 1;
            while (end < a->m && a->chr[end] == a->chr[start]) end++;
            int rc = compute_global(a, start, end - start, l2_out + start, a->m, maf_out + start,
                                    &pairs, &any_full, err, errlen);
            if (rc) return rc;
            start = end;
        }
    }
    if (info) {
        info->n_pairs = pairs;
        info->any_full_chr_window = any_full;
        info->n_dots = g_dots;
        info->gemm_secs = g_gemm_secs;
    }
    return OR_OK;
}

/* Thread count OpenMP will use (for reporting the CPU baseline). */
int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
