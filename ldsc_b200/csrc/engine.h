// engine.h -- internal interfaces between the host runtime (engine.cpp) and
// the CUDA kernels of libldsc_b200.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace ldsc {

// Device view of a resident BED panel: n_snp rows of `pitch` bytes, the first
// bpr = ceil(n_indiv / 4) of which are the BED row (count-A1 2-bit codes,
// individual i in byte i/4 at bit 2*(i%4)); the padding bytes are zero.
struct PanelView {
    const uint8_t* rows;
    uint64_t n_snp;
    uint64_t n_indiv;
    uint64_t bpr;
    uint64_t pitch;
};

// Which individuals a run uses: all (keep == nullptr) or FAM indices keep[i].
struct IndivSel {
    const int64_t* keep;  // device pointer or nullptr
    uint64_t n;           // individuals used
};

// Per-record statistics produced by the decode kernels (device SoA arrays).
struct RecStats {
    int32_t* n;        // non-missing count
    int32_t* s;        // sum of genotypes
    int32_t* q;        // sum of squared genotypes
    int32_t* q3;       // sum of cubes (MAF-aware sketch only, may be null)
    int32_t* q4;       // sum of 4th powers (MAF-aware sketch only, may be null)
    double* maf;       // minor allele frequency
    double* mean;      // mean over non-missing
    double* inv_std;   // 1 / sqrt(css / N), 0 when css <= 0
    double* qinv;      // 1 / sqrt(n * (n q - s^2)), 0 when the SNP is monomorphic
    double* kappa;     // per-SNP kurtosis term (MAF-aware sketch), may be null
    double* pq;        // (maf (1 - maf))^pq_exp, may be null
};

// Band tile: A block (k side, left SNPs) x B block (j side, right SNPs).
struct Tile {
    uint32_t a_blk;
    uint32_t b_blk;
};

// Everything the Gram epilogues need.
struct EpilogueArgs {
    const int64_t* left;      // L[j]: pair (k, j) counts iff left[j] <= k < j
    const int32_t* n;         // INT8 form: per-record counts
    const int32_t* s;
    const double* qinv;
    const double* kappa;      // sketch MAF-aware, else null
    const double* aeff;       // M x K column-major effective annotation (f64)
    double* l2;               // M x K column-major output accumulator
    int64_t m;                // records
    int32_t K;                // annotation columns
    double r2u_a;             // 1 + 1/(N-2)
    double r2u_b;             // -1/(N-2)
    double n_inv_sq_r2u_a;    // r2u_a / N^2   (FP64 form)
    double n_inv_sq;          // 1 / N^2       (sketch form)
    double sketch_d;          // d as double   (sketch form)
    unsigned int* err;        // device error word (non-zero = a bounded wait gave up)
    double* rtiles;           // K > 1: tile t's masked r2u values, ta rows (k) x tb (j) f64 at t * ta * tb
    // K = 1: tile t's row sums (ta values at prow + t * ta: sum_j r2u a_j for
    // each left record k) and column sums (tb values at pcol + t * tb), added
    // to l2 in a fixed order by launch_l2_reduce; null = atomics into l2
    double* prow;
    double* pcol;
};

// ---- kernels (launchers return cudaError_t of the launch) ----

// Decode + stats (+ optional INT8 genotype/mask operand rows, interleaved:
// row 2r = genotype, row 2r+1 = non-missing mask, `ld` bytes per row).
cudaError_t launch_decode_i8(const PanelView& p, const uint64_t* rec_rows, int64_t m,
                             IndivSel sel, uint8_t* ops, uint64_t ld, RecStats st,
                             int want_moments, cudaStream_t stream);

// Finalise per-record stats: maf, mean, inv_std, qinv, pq, kappa, aeff.
cudaError_t launch_finalize_stats(int64_t m, uint64_t n_indiv, RecStats st,
                                  const double* annot, int32_t K, int has_pq, double pq_exp,
                                  double* aeff, double* l2_init,
                                  cudaStream_t stream, uint64_t annot_ld = 0);

// Standardised f64 columns, row r of `x` = record r, `ld` doubles per row.
// Rows [r0, r1) of a packed BED body (bpr bytes per row, as in the file) to
// the pitched panel layout; pad bytes are zeroed.
cudaError_t launch_repitch(const uint8_t* src, uint64_t bpr, uint8_t* dst, uint64_t pitch, uint64_t r0,
                           uint64_t r1, cudaStream_t stream);

cudaError_t launch_decode_f64(const PanelView& p, const uint64_t* rec_rows, int64_t m,
                              IndivSel sel, RecStats st, double* x, uint64_t ld,
                              cudaStream_t stream);

// FP64 band Gram + unbiased-r^2 epilogue (TA = TB = 128 records per tile).
cudaError_t launch_gram_f64(const double* x, uint64_t ld, uint64_t kdim, const Tile* tiles,
                            int64_t n_tiles, const EpilogueArgs& ep, int sms,
                            cudaStream_t stream);

// INT8 tcgen05 band Gram + exact epilogue (TA = 64, TB = 128 records per tile).
// ops: 2*m rows of `ld` bytes.  dbg (optional) receives the raw accumulators
// of the first tile (128 x 256 int32).
cudaError_t launch_gram_i8(const uint8_t* ops, uint64_t ld, int64_t m, const Tile* tiles,
                           int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg, int sms,
                           cudaStream_t stream);

// Fused INT8 band Gram over the packed BED rows themselves (record r at
// rows + r * pitch, all n_indiv individuals): the kernel stages 2-bit rows by
// TMA and expands them into the G / M operand tiles in shared memory, so no
// operand rows exist in device memory.  Same tiles, epilogue and results as
// launch_gram_i8; the per-record n / s / qinv come from a moments-only decode.
cudaError_t launch_gram_i8_packed(const uint8_t* rows, uint64_t pitch, uint64_t n_indiv, int64_t m, const Tile* tiles,
                                  int64_t n_tiles, const EpilogueArgs& ep, int32_t* dbg, int sms,
                                  cudaStream_t stream);

// CountSketch, step 1 (once per panel, sketch dimension and individual set):
// rewrite every panel row in bucket-major individual order, perm[p] = FAM
// index of the individual at permuted position p.  out: n_snp rows of
// out_pitch_words 32-bit words, bit-plane quads of 64 positions.
cudaError_t launch_sketch_permute(const PanelView& p, const int32_t* perm, uint64_t n_used, uint32_t* out,
                                  uint64_t out_pitch_words, cudaStream_t stream);

// CountSketch, step 2 (per call): per record, run sums over the permuted row,
// per-SNP moments into st.n/s/q (and q3/q4 when want_moments), standardised
// and renormalised bucket values.  segt: the layout's thread-major boundary
// table (launch_sketch_segt) for this n_used and d; large d (sketch_large_d)
// runs the shared-memory-row form.
// out: m rows of `ld` floats, or with split = 1 the tensor-core operand form:
// rows 2r = tf32(v) and 2r+1 = tf32(v - tf32(v)), `ld` floats each.
cudaError_t launch_sketch_seg(const uint32_t* pp, uint64_t pp_pitch_words, const uint64_t* rec_rows, int64_t m,
                              uint64_t n_used, const int32_t* segt, uint32_t d, RecStats st, int want_moments,
                              int split, float* out, uint64_t ld, cudaStream_t stream);
// Whether d and n_used take the large-d form (d >= 2560 and its shared memory fits).
bool sketch_large_d(uint64_t n_used, uint32_t d);
// Entries of the thread-major boundary table, and its construction (once per
// layout) from seg_off, the 2d + 1 run starts (run k = bucket k/2, sign + for
// even k).
uint64_t sketch_segt_count(uint64_t n_used, uint32_t d);
cudaError_t launch_sketch_segt(const int32_t* seg_off, uint64_t n_used, uint32_t d, int32_t* segt,
                               cudaStream_t stream);
// Whether the sketch kernel's shared memory holds n_used individuals and d buckets.
bool sketch_supported(uint64_t n_used, uint32_t d);

// CountSketch band Gram on tcgen05 kind::tf32 over split rows (hi/lo
// interleaved, `ld` floats per row, ld*4 a multiple of 128) + quadratic
// bias-correction epilogue (TA = 64, TB = 128 records per tile).
cudaError_t launch_gram_tf32(const float* ops, uint64_t ld, int64_t m, const Tile* tiles, int64_t n_tiles,
                             const EpilogueArgs& ep, int maf_aware, int32_t* dbg, int sms, cudaStream_t stream);

// FP32 band Gram of sketched rows + quadratic bias correction epilogue.
cudaError_t launch_gram_f32(const float* x, uint64_t ld, uint64_t kdim, const Tile* tiles,
                            int64_t n_tiles, const EpilogueArgs& ep, int maf_aware, int sms,
                            cudaStream_t stream);

// K > 1 annotation contraction from the R tiles a Gram wrote (no atomics, each
// l2 row owned by one CTA per pass):
//   by right block:  l2[j, C] += sum over tiles of block, sum_k R[k][j] a[k, C]
//   by left block:   l2[k, C] += sum over tiles of block, sum_j R[k][j] a[j, C]
// ptr/idx: CSR lists of tile indices per right block (by_right) or per left block.
cudaError_t launch_contract(const double* rtiles, int ta, int tb, const Tile* tiles, const int32_t* ptr,
                            const int32_t* idx, int32_t nblocks, bool by_right, const EpilogueArgs& ep,
                            cudaStream_t stream);

// Load a kernel's code on the current device now.  With lazy module loading
// (the CUDA 12 default) a kernel is loaded at its first launch, which can
// stall work already running on the device; contexts load every kernel of the
// library when they are created (preload_* below, one per source file).
template <typename F>
cudaError_t preload_kernel(F* kernel) {
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(kernel));
}
cudaError_t preload_gram_tc();
cudaError_t preload_gram_simt();
cudaError_t preload_decode();
cudaError_t preload_sketch();
cudaError_t preload_contract();
cudaError_t preload_synth();
cudaError_t preload_regress();
cudaError_t preload_partitioned();

// K = 1: l2[j] += the column sums of the tiles of j's right block, then the
// row sums of the tiles of j's left block, in list order (deterministic).
// ptr/idx: the CSR tile lists of launch_contract.
cudaError_t launch_l2_reduce(int64_t m, int ta, int tb, const int32_t* ptr_r, const int32_t* idx_r,
                             const int32_t* ptr_l, const int32_t* idx_l, const double* prow, const double* pcol,
                             double* l2, cudaStream_t stream);

// Synthetic panel generator (founder mosaic, counter-based RNG).
cudaError_t launch_synth(uint8_t* rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                         uint32_t founders, double switch_p, double miss, uint64_t seed,
                         uint8_t* founder_table, cudaStream_t stream);

}  // namespace ldsc
