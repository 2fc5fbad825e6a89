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
    const float* aeff32;      // M x K row-major effective annotation (f32, K > 1 path)
    double* l2;               // M x K column-major output accumulator
    int64_t m;                // records
    int32_t K;                // annotation columns
    double r2u_a;             // 1 + 1/(N-2)
    double r2u_b;             // -1/(N-2)
    double n_inv_sq_r2u_a;    // r2u_a / N^2   (FP64 form)
    double n_inv_sq;          // 1 / N^2       (sketch form)
    double sketch_d;          // d as double   (sketch form)
    unsigned int* err;        // device error word (non-zero = a bounded wait gave up)
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
                                  double* aeff, float* aeff32, double* l2_init,
                                  cudaStream_t stream);

// Standardised f64 columns, row r of `x` = record r, `ld` doubles per row.
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

// CountSketch: per record, scatter into d buckets and ratio-renormalise.
// `packed` holds bucket | (sign < 0) << 31 per individual; tsum[b] = sum of
// signs of bucket b over all used individuals.  out: m rows of `ld` floats.
cudaError_t launch_sketch_scatter(const PanelView& p, const uint64_t* rec_rows, int64_t m,
                                  IndivSel sel, const uint32_t* packed, const int32_t* tsum,
                                  uint32_t d, RecStats st, float* out, uint64_t ld,
                                  cudaStream_t stream);

// FP32 band Gram of sketched rows + quadratic bias correction epilogue.
cudaError_t launch_gram_f32(const float* x, uint64_t ld, uint64_t kdim, const Tile* tiles,
                            int64_t n_tiles, const EpilogueArgs& ep, int maf_aware, int sms,
                            cudaStream_t stream);

// Synthetic panel generator (founder mosaic, counter-based RNG).
cudaError_t launch_synth(uint8_t* rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                         uint32_t founders, double switch_p, double miss, uint64_t seed,
                         uint8_t* founder_table, cudaStream_t stream);

}  // namespace ldsc
