/*
 * ldsc_b200.h -- C ABI of the B200 LD-score engine (libldsc_b200.so).
 *
 * Plain C types only: pointers, sizes, status codes.  Every entry point
 * returns an `int` status (LDSC_OK = 0, negative on error); the message of the
 * last failure on a context is available from ldsc_last_error().
 *
 * The engine replaces the compute core of ldsc-rs's `l2` subcommand:
 *
 *   compute_ldscore_global(all_snps, bed, mmap_bed, n_indiv, mode, chunk_c,
 *       annot, iid_indices, pq_exp, yes_really, [gpu_ctx, gpu_config],
 *       use_f32, verbose_timing, sketch, sketch_maf_aware,
 *       snp_level_masking, on_progress) -> (l2 M x K, maf, L2Perf)
 *   (reference: src/l2/compute.rs:1009-1028)
 *
 * and the per-chromosome / --global-pass fan-out around it in `l2::run`
 * (src/l2/mod.rs:439-575).  One call of ldsc_l2_run() computes every
 * chromosome of the record list; in the default per-chromosome mode each
 * chromosome is chunked from its own first SNP exactly as the reference's
 * per-chromosome rayon tasks do.
 *
 * Thread safety: a context serialises its calls with an internal mutex, so
 * the reference's concurrent per-chromosome callers (src/l2/mod.rs:502-553)
 * may share one context.  There is no CPU fallback: every compute entry point
 * fails with LDSC_E_CUDA when no usable GPU is present.
 */
#ifndef LDSC_B200_H
#define LDSC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDSC_B200_ABI_VERSION 1

typedef struct ldsc_ctx ldsc_ctx;
typedef struct ldsc_panel ldsc_panel;

/* Status codes. */
enum {
    LDSC_OK = 0,
    LDSC_E_INVALID = -1,      /* malformed arguments (anyhow::ensure! failures in the reference) */
    LDSC_E_NOMEM = -2,        /* device allocation failed */
    LDSC_E_CUDA = -3,         /* CUDA runtime / driver error, or no GPU */
    LDSC_E_TIMEOUT = -4,      /* a device wait exceeded its bound and the kernel gave up */
    LDSC_E_UNSUPPORTED = -5,  /* valid request outside what this build implements */
    LDSC_E_BED = -6           /* BED header / length validation failed (src/bed.rs:73-110) */
};

/* Window definition, WindowMode (src/l2/window.rs:5-12). */
enum { LDSC_WINDOW_CM = 0, LDSC_WINDOW_KB = 1, LDSC_WINDOW_SNP = 2 };

/* Arithmetic form of the exact window Gram. */
enum {
    LDSC_PRECISION_FP64 = 0,  /* plain form: standardised f64 columns, f64 Gram (the reference method) */
    LDSC_PRECISION_INT8 = 1   /* genotype/mask INT8 tcgen05 Gram, INT32 accumulation, exact epilogue */
};

/* Per-chunk progress, L2Progress (src/l2/mod.rs:22-39).  The engine reports
 * progress per Gram launch rather than per 200-SNP chunk. */
typedef struct {
    uint64_t chunks_done;
    uint64_t chunks_total;
    uint64_t snps_done;
    uint64_t snps_total;
    double chunk_wall_ms;
} ldsc_progress;

typedef void (*ldsc_progress_fn)(const ldsc_progress *progress, void *user);

/* Per-phase timing, L2Perf (src/l2/mod.rs:1016-1034), plus device detail.
 * Phase times are device (CUDA event) times of this call's kernels. */
typedef struct {
    uint64_t m;                 /* SNP records of the call */
    uint64_t n_indiv;           /* individuals used (after --keep) */
    double bed_read_secs;       /* host->device upload of BED bytes done by this call */
    double norm_secs;           /* decode + per-SNP stats + standardisation */
    double sketch_secs;         /* CountSketch projection; negative when not sketching */
    double bb_dot_secs;         /* 0: the within-chunk block is part of the band Gram */
    double ab_dot_secs;         /* band Gram + r^2 epilogue + l2 accumulation */
    double ring_store_secs;     /* 0: the panel is resident, there is no ring buffer */
    uint64_t n_pairs;           /* off-diagonal (j,k) pairs contributing to l2 in this mode */
    uint64_t n_tiles;           /* Gram tiles launched */
    uint32_t kernel_launches;   /* kernels launched by this call */
    uint32_t gram_kind;         /* 0 fp64, 1 int8 tcgen05, 2 fp32 sketch */
    double device_ms;           /* whole call, device time */
    double contract_secs;       /* K > 1: the annotation contraction passes (inside ab_dot_secs) */
    double layout_secs;         /* --sketch: wall time spent building the CountSketch layout (hash,
                                   bucket-major order, panel rows rewritten in it); 0 when this call
                                   reused a layout built earlier */
} ldsc_perf;

/* Arguments of one l2 computation.  Record i of the call is BED row
 * bed_idx[i] of the panel (the reference's BimRecord.bed_idx). */
typedef struct {
    uint64_t n_snp;               /* number of SNP records */
    const uint64_t *bed_idx;      /* BED row per record; NULL = records are rows 0..n_snp-1 */
    const uint8_t *chr;           /* chromosome code per record (BimRecord.chr) */
    const double *cm;             /* genetic position (cM) per record */
    const uint32_t *bp;           /* physical position per record */
    int32_t window_mode;          /* LDSC_WINDOW_* */
    double window_size;           /* cM or kb */
    uint64_t window_snps;         /* half-window in SNPs for LDSC_WINDOW_SNP */
    uint32_t chunk_size;          /* --chunk-size (default 200) */
    int32_t global_pass;          /* 1 = --global-pass; 0 = per-chromosome (default) */
    int32_t snp_level_masking;    /* --snp-level-masking */
    int32_t precision;            /* LDSC_PRECISION_* for exact mode */
    int32_t use_f32;              /* --fast-f32: accepted; exact modes keep their own arithmetic */
    uint32_t sketch_d;            /* --sketch d; 0 = exact */
    int32_t sketch_maf_aware;     /* --sketch-maf-aware */
    const int64_t *keep_iids;     /* --keep: FAM indices of kept individuals; NULL = all */
    uint64_t n_keep;
    const double *annot;          /* M x K column-major annotation; NULL = single all-ones column */
    uint32_t n_annot;             /* K */
    int32_t has_pq_exp;           /* --pq-exp / --per-allele applied inside the compute */
    double pq_exp;
    int32_t yes_really;           /* --yes-really: silence the whole-chromosome window warning */
    ldsc_progress_fn on_progress; /* optional */
    void *progress_user;
    /* Extensions for a resident panel (no reference counterpart; zero = off). */
    uint64_t row_begin;           /* with bed_idx NULL: record i is row row_begin + i */
    int32_t annot_on_device;      /* annot points to device memory (read in place) */
    uint64_t annot_ld;            /* rows between annot columns; 0 = n_snp */
    int32_t out_on_device;        /* l2_out / maf_out are device pointers */
} ldsc_l2_args;

/* Synthetic panel description (seeded founder mosaic; see ldsc_b200/synth.py). */
typedef struct {
    uint64_t n_indiv;
    uint64_t n_snp;
    uint32_t founders;
    double switch_p;
    double miss;
    uint64_t seed;
} ldsc_synth_spec;

/* ---- library / context ------------------------------------------------ */

int ldsc_abi_version(void);

/* Create a context on CUDA device `device` (the reference creates one
 * GpuContext per run and shares it across chromosomes: src/l2/mod.rs:410-436).
 * flags: 0, or LDSC_CTX_FUSED_OPERANDS. */
int ldsc_ctx_create(int device, uint32_t flags, ldsc_ctx **out);

/* Context flag: run the INT8-exact form as one fused Gram that stages the
 * packed 2-bit BED rows and expands them into operand tiles in shared memory,
 * instead of the default two passes (decode the panel into INT8 genotype /
 * mask operand rows in device memory, 2 bytes per individual per SNP, then the
 * band Gram over them).  Results are bit-identical; the fused form needs no
 * operand buffer (10 GB for 50,000 individuals x 100,000 SNPs) but its Gram
 * is slower (shared-memory bandwidth: the expansion writes the same operand
 * bytes the two-pass form's TMA copies write, on top of the packed rows).
 * Runs with --keep, or whose records are not consecutive panel rows, always
 * take the two-pass form. */
#define LDSC_CTX_FUSED_OPERANDS 1u
int ldsc_ctx_destroy(ldsc_ctx *ctx);

/* Launch this context's work on an existing cudaStream_t (NULL = the
 * context's own stream). */
int ldsc_ctx_set_stream(ldsc_ctx *ctx, void *cuda_stream);

/* Copy the last error message of the context into buf (always terminated). */
int ldsc_last_error(const ldsc_ctx *ctx, char *buf, size_t len);

/* Number of kernels this context has launched since creation. */
uint64_t ldsc_ctx_kernel_count(const ldsc_ctx *ctx);

/* Number of cached CUDA-graph replays (regression pipelines) of this context. */
uint64_t ldsc_ctx_graph_launches(const ldsc_ctx *ctx);

/* Free the context's device workspace and cached graphs (they grow back on
 * demand).  Waits for the context's work. */
int ldsc_ctx_trim(ldsc_ctx *ctx);

/* ---- BED validation and resident panels -------------------------------- */

/* Bed::from_bytes header/length validation (src/bed.rs:53-128) on a whole
 * .bed image (magic + body).  Host only; no GPU needed.  Returns LDSC_E_BED
 * with the reference's message ("invalid magic bytes", "not SNP-major",
 * "invalid length") in err. */
int ldsc_bed_validate(const uint8_t *bed_file, uint64_t len, uint64_t n_indiv, uint64_t n_snp,
                      char *err, size_t errlen);

/* Upload a BED body (SNP-major, ceil(n_indiv/4) bytes per SNP, no magic)
 * into device memory, where it stays resident until ldsc_panel_destroy. */
int ldsc_panel_upload(ldsc_ctx *ctx, const uint8_t *bed_body, uint64_t body_bytes,
                      uint64_t n_indiv, uint64_t n_snp, ldsc_panel **out);

/* Generate a synthetic panel directly in device memory. */
int ldsc_panel_synth(ldsc_ctx *ctx, const ldsc_synth_spec *spec, ldsc_panel **out);

/* Copy BED rows [snp_begin, snp_end) of a panel to host (ceil(n_indiv/4)
 * bytes per row, no magic). */
int ldsc_panel_download(ldsc_ctx *ctx, const ldsc_panel *panel, uint64_t snp_begin,
                        uint64_t snp_end, uint8_t *out);

int ldsc_panel_destroy(ldsc_panel *panel);

/* Individuals and SNP rows of a panel. */
int ldsc_panel_shape(const ldsc_panel *panel, uint64_t *n_indiv, uint64_t *n_snp);

/* ---- the l2 computation ------------------------------------------------ */

/* compute_ldscore_global on a resident panel.  l2_out: n_snp x K column-major
 * (K = n_annot, or 1 without annotation); maf_out: n_snp.  Host pointers. */
int ldsc_l2_run(ldsc_ctx *ctx, const ldsc_panel *panel, const ldsc_l2_args *args, double *l2_out,
                double *maf_out, ldsc_perf *perf);

/* compute_l2_from_bytes / compute_l2_from_bed (src/l2/mod.rs:1049-1169) on a
 * whole .bed image in host memory: validate, upload, compute, return. */
int ldsc_l2_from_bed(ldsc_ctx *ctx, const uint8_t *bed_file, uint64_t len, uint64_t n_indiv,
                     const ldsc_l2_args *args, double *l2_out, double *maf_out, ldsc_perf *perf);

/* compute_snp_stats (src/l2/snp_stats.rs:5-195), the --maf / --pq-exp
 * prefilter: per record of `args` (n_snp, bed_idx or row_begin, keep_iids),
 * MAF = min(f, 1 - f) with f = sum / (2 count), and het_miss_ok = 1 when
 * het + missing < n (0 for an all-het-or-missing SNP).  One decode pass. */
int ldsc_snp_stats(ldsc_ctx *ctx, const ldsc_panel *panel, const ldsc_l2_args *args, double *maf_out,
                   uint8_t *het_miss_ok_out);

/* Number of off-diagonal pairs the call would accumulate (host only). */
int ldsc_l2_pair_count(const ldsc_l2_args *args, uint64_t *n_pairs);

/* Device workspace (bytes) ldsc_l2_run would hold for these arguments on a
 * panel of n_indiv individuals, not counting the panel and its shared
 * CountSketch layout (host only). */
int ldsc_l2_workspace_bytes(const ldsc_l2_args *args, uint64_t n_indiv, uint64_t *bytes);

/* Per-record left window limit L[i] (host only): record i pairs with every
 * record k, L[i] <= k < i.  Masked mode: the per-SNP block_left
 * (src/l2/window.rs:32-90); chunked mode: the chunk's ring-window start
 * (src/l2/compute.rs:1164-1184,1288-1299). */
int ldsc_l2_left_limits(const ldsc_l2_args *args, int64_t *left_out);

/* ---- CountSketch ------------------------------------------------------- */

/* CountSketchProj::new(n_indiv, d, seed) bucket/sign stream
 * (src/l2/compute.rs:178-192; fastrand 2.3.0 WyRand).  Host only. */
int ldsc_countsketch_hash(uint64_t n_indiv, uint32_t d, uint64_t seed, uint32_t *bucket,
                          float *sign);

/* Fused decode -> standardise -> CountSketch scatter -> ratio renorm of BED
 * rows [snp_begin, snp_end) with explicit bucket/sign arrays
 * (scatter_one_column_f32, src/wasm_simd.rs:1617-1784).  out: rows x d f32,
 * row-major (one sketched SNP per row).  keep_iids may be NULL. */
int ldsc_sketch_project(ldsc_ctx *ctx, const ldsc_panel *panel, uint64_t snp_begin,
                        uint64_t snp_end, const int64_t *keep_iids, uint64_t n_keep,
                        const uint32_t *bucket, const float *sign, uint32_t d, float *out);

/* ---- LD-score regressions (h2 / rg) ------------------------------------ */

/* Batched h2 regressions against one LD-score column (K = 1): weights
 * (ldsc_weights, src/h2.rs:185-206), two IRWLS re-weightings (irwls_ldsc,
 * src/h2.rs:435-458) and the block jackknife (jackknife_fast,
 * src/h2.rs:100-183; jackknife_se_cov, src/jackknife.rs:10-59), as in
 * run_h2_ldsc / run_hsq_ldsc (src/h2.rs:258-433, src/regressions.rs:1648-1825),
 * with --two-step when asked.  One regression per trait; all traits share the
 * SNPs, ref_l2 and w_l2. */
typedef struct {
    uint64_t n_snp;
    uint32_t n_traits;
    uint32_t n_blocks;            /* --n-blocks (200); must be <= n_snp */
    const double *chi2;           /* n_traits x n_snp, row-major */
    const double *n_per_snp;      /* n_traits x n_snp sample sizes, or NULL */
    const double *n_scalar;       /* n_traits sample sizes (when n_per_snp is NULL) */
    const double *ref_l2;         /* n_snp LD scores */
    const double *w_l2;           /* n_snp regression-weight LD scores */
    double m_snps;                /* M */
    int32_t fixed_intercept;      /* --intercept-h2 */
    double intercept;
    int32_t want_lambda_gc;       /* median(chi2) / 0.4549 (exact order statistics) */
    int32_t device_pointers;      /* 1: the arrays above are device pointers */
    int32_t two_step;             /* --two-step: fit the intercept on chi2 < two_step_cutoff first */
    double two_step_cutoff;
} ldsc_h2_args;

typedef struct {
    double h2, h2_se, intercept, intercept_se;
    double mean_chi2, lambda_gc, ratio, ratio_se;  /* ratio: NaN when mean_chi2 <= 1 or fixed */
    double coef, coef_se;                          /* slope per unit of N * l2 */
} ldsc_h2_result;

int ldsc_h2_batch(ldsc_ctx *ctx, const ldsc_h2_args *args, ldsc_h2_result *results);

/* Batched genetic correlations (run_rg, src/regressions.rs:2113-2460): per
 * pair, two h2 fits on z^2, the genetic-covariance fit on z1 * z2
 * (gencov_weights, run_gencov_ldsc, src/regressions.rs:1612-1645,1828-2052),
 * rg = gencov / sqrt(h2_1 h2_2) and its ratio-jackknife SE
 * (ratio_jackknife, src/regressions.rs:1067-1120).  Free intercepts, no
 * --two-step. */
typedef struct {
    uint64_t n_snp;
    uint32_t n_pairs;
    uint32_t n_blocks;
    const double *z1;             /* n_pairs x n_snp signed z-scores of trait 1 */
    const double *z2;             /* n_pairs x n_snp of trait 2 */
    const double *n1;             /* n_pairs scalar sample sizes */
    const double *n2;
    const double *ref_l2;
    const double *w_l2;
    double m_snps;
    int32_t device_pointers;
} ldsc_rg_args;

typedef struct {
    double rg, rg_se, z, p;
    double gencov, gencov_se, gencov_intercept, gencov_intercept_se;
    double h2_1, h2_1_se, h2_2, h2_2_se;
    double mean_z1z2;
} ldsc_rg_result;

int ldsc_rg_batch(ldsc_ctx *ctx, const ldsc_rg_args *args, ldsc_rg_result *results);

/* Partitioned h2 (fit_h2_partitioned, src/regressions.rs:1121-1226; the
 * K > 1 branch of run_h2, src/regressions.rs:561-630): one weighted least
 * squares of chi2 on K LD-score columns scaled by N / nbar, plus an intercept
 * unless constrained, with weights ldsc_weights(sum of the K columns, w_l2,
 * N, sum(M), aggregate h2) and the block jackknife over min(kept SNPs,
 * n_blocks) blocks.  SNPs whose chi2 is not below the trait's chisq_max (NaN
 * included) are dropped first; run_h2's default for K > 1 is
 * max(0.001 max(N), 80), N over the SNPs with a chi2.
 * One regression per trait; traits share ref_l2, w_l2 and m_vec.
 * P = K + 1 with a free intercept, K with a fixed one; P <= 160. */
typedef struct {
    uint64_t n_snp;
    uint32_t n_traits;
    uint32_t n_annot;             /* K */
    uint32_t n_blocks;            /* --n-blocks (200) */
    const double *chi2;           /* n_traits x n_snp, row-major */
    const double *n_per_snp;      /* n_traits x n_snp sample sizes, or NULL */
    const double *n_scalar;       /* n_traits sample sizes (when n_per_snp is NULL) */
    const double *ref_l2;         /* n_snp x K LD scores, column-major, column stride ref_ld */
    uint64_t ref_ld;              /* 0: n_snp */
    const double *w_l2;           /* n_snp regression-weight LD scores */
    const double *m_vec;          /* K per-annotation M (host) */
    int32_t fixed_intercept;      /* --intercept-h2 (or --no-intercept: 1.0) */
    double intercept;
    const double *chisq_max;      /* n_traits cut-offs (host); INFINITY keeps every finite chi2 */
    int32_t device_pointers;      /* 1: chi2, n_per_snp, n_scalar, ref_l2, w_l2 are device pointers */
    double *est;                  /* out, host, may be NULL: n_traits x P jackknife estimates
                                     (coefficient x nbar per annotation, then the intercept) */
    double *cov;                  /* out, host, may be NULL: n_traits x P x P jackknife covariance */
    double *delete_values;        /* out, host, may be NULL: n_traits x n_blocks x P (NaN past
                                     a trait's block count) */
    double *h2_annot;             /* out, host, may be NULL: n_traits x K, coefficient x M_k */
} ldsc_h2p_args;

typedef struct {
    double h2_total, h2_total_se;    /* sum of h2_annot; SE from the coefficients' covariance
                                        (total_from_jknife, src/regressions.rs:1565-1610) */
    double intercept, intercept_se;  /* intercept_se NaN when fixed */
    double n_mean, mean_chi2;        /* over the kept SNPs */
    uint64_t n_obs;                  /* kept SNPs */
    uint32_t n_blocks;               /* jackknife blocks used */
} ldsc_h2p_result;

int ldsc_h2_partitioned(ldsc_ctx *ctx, const ldsc_h2p_args *args, ldsc_h2p_result *results);

/* ---- serving: continuous batching over resident panels ------------------ */

/* No counterpart in the reference (one computation per process there).  A
 * server owns n_slots engine contexts, each with its own stream, workspace
 * and worker thread.  Queued jobs are admitted in arrival order as a slot
 * and device memory free up: a job fits when its workspace fits in the
 * slot's, or when growing the slot keeps all slots' workspace within
 * device_budget (0 = free memory at creation minus 4 GiB).  A later job may
 * pass an older one that does not fit yet; idle slots give their workspace
 * back when the oldest job needs it.  Admitted jobs run concurrently and
 * their kernels overlap on the device; the h2 and rg pipelines replay as
 * cached CUDA graphs (partitioned h2 reads its kept-SNP counts on the host
 * part-way and runs as plain launches).  A job's result does not depend on
 * what else runs. */
typedef struct ldsc_server ldsc_server;

enum { LDSC_JOB_L2 = 0, LDSC_JOB_H2 = 1, LDSC_JOB_RG = 2, LDSC_JOB_H2P = 3 };

typedef struct {
    int32_t kind;                 /* LDSC_JOB_* */
    const ldsc_panel *panel;      /* L2: resident panel */
    ldsc_l2_args l2;              /* L2 arguments (copied; the arrays they point to must stay valid
                                     until the job completes) */
    double *l2_out;               /* L2: n_snp x K column-major, host */
    double *maf_out;              /* L2: n_snp, host, may be NULL */
    ldsc_h2_args h2;              /* H2 */
    ldsc_h2_result *h2_out;       /* H2: n_traits results */
    ldsc_rg_args rg;              /* RG */
    ldsc_rg_result *rg_out;       /* RG: n_pairs results */
    uint64_t device_bytes;        /* workspace the job needs; 0 = estimated by the server */
    ldsc_h2p_args h2p;            /* H2P: partitioned h2 (its est / cov / delete_values / h2_annot
                                     outputs are written when the job completes) */
    ldsc_h2p_result *h2p_out;     /* H2P: n_traits results */
} ldsc_job;

typedef struct {
    int32_t status;               /* LDSC_OK or an error code */
    uint32_t slot;                /* slot that ran the job */
    double queue_ms;              /* submit -> start */
    double run_ms;                /* start -> end */
    double latency_ms;            /* submit -> end */
    ldsc_perf perf;               /* L2 jobs */
    char error[256];
} ldsc_job_result;

typedef struct {
    uint64_t submitted, completed, running, queued;
    uint64_t budget_bytes;        /* device workspace budget */
    uint64_t reserved_bytes;      /* workspace the slots may hold now */
    uint64_t graph_launches;      /* cached-graph replays over all slots */
    uint64_t kernels;             /* kernels launched over all slots */
} ldsc_server_stats;

int ldsc_server_create(int device, uint32_t n_slots, uint64_t device_budget, ldsc_server **out);
/* Queue a job; returns at once with its ticket.  LDSC_E_NOMEM if the job's
 * workspace exceeds the whole budget. */
int ldsc_server_submit(ldsc_server *srv, const ldsc_job *job, uint64_t *ticket);
/* Block until the job ends; returns its status and releases the ticket. */
int ldsc_server_wait(ldsc_server *srv, uint64_t ticket, ldsc_job_result *result);
/* Run `job` once on every slot, one slot after another, and return when the
 * last has finished (no reference counterpart).  Each slot's workspace then
 * holds what that job needs, so later jobs no larger than it start without
 * allocating device memory: growing the device's memory pool while other
 * slots run measured 0.1 - 0.9 s per allocation here, with the other slots'
 * work held up meanwhile.  Prewarm with the largest job of each kind before
 * serving.  The job's outputs are written once per slot. */
int ldsc_server_prewarm(ldsc_server *srv, const ldsc_job *job);
int ldsc_server_stats_get(ldsc_server *srv, ldsc_server_stats *stats);
/* Finish running jobs, fail queued ones, free the slots. */
int ldsc_server_destroy(ldsc_server *srv);

/* ---- allocation-free entry point ---------------------------------------- */

/* No counterpart in the reference: this entry point exists for callers that
 * cannot allocate device memory -- a host that owns all device memory through
 * its own arena (an allocation behind its back breaks its accounting), or a
 * latency-critical request loop in which an allocation or free would
 * synchronise the device.
 *
 * It runs the INT8-exact l2 pass (all-ones annotation, K = 1) on device
 * buffers the caller owns and allocates nothing: all scratch lives in one
 * static device array of LDSC_NOALLOC_SCRATCH_BYTES bytes inside the library,
 * which every GPU that loads the library holds until the process exits.
 *   d_rows   device BED rows, n_snp rows of `pitch` bytes (pitch a multiple of
 *            16, >= ceil(n_indiv/4); 16-byte aligned)
 *   left     HOST array of n_snp window limits (ldsc_l2_left_limits)
 *   d_l2     device output, n_snp doubles;  d_maf  device output, n_snp doubles
 *   stream   cudaStream_t to run on (NULL = the legacy default stream)
 * Requests whose scratch exceeds the array are rejected with LDSC_E_INVALID.
 * The scratch is 2 * n_snp * round_up(n_indiv, 128) bytes of operands, 52
 * bytes per SNP of statistics and limits, 8 bytes per band tile (64 x 128
 * records) and a 16-byte error word, each of its 11 parts starting on a
 * 256-byte boundary.  All calls share the array, which keeps the last call's
 * contents; calls that overlap on the GPU race.  The call runs on the current
 * device, to which d_rows, d_l2, d_maf and the stream must belong.  The first
 * call on a device looks up the array's address, keeps it for the life of the
 * process, and should come before any stream capture; after a device reset
 * the library must be reloaded.  The call waits for its own work before
 * returning.  Messages: ldsc_noalloc_last_error(). */
#define LDSC_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)

int ldsc_l2_int8_noalloc(const uint8_t *d_rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                         const int64_t *left, double *d_l2, double *d_maf, void *stream);

/* Last error message of ldsc_l2_int8_noalloc (process-wide). */
int ldsc_noalloc_last_error(char *buf, size_t len);

/* ---- diagnostics ------------------------------------------------------- */

/* Raw INT32 accumulators of the INT8 tcgen05 Gram for one tile: A side =
 * records [k0, k0+64) (genotype row, mask row interleaved: 128 rows), B side =
 * records [j0, j0+128) (256 rows).  out: 128 x 256 int32 row-major.  Used to
 * check the tensor-core Gram bit-exactly against an integer recompute. */
int ldsc_debug_gram_i8_tile(ldsc_ctx *ctx, const ldsc_panel *panel, uint64_t k0, uint64_t j0,
                            int32_t *out);

#ifdef __cplusplus
}
#endif

#endif /* LDSC_B200_H */
