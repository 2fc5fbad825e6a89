// plan.h -- host-side planning of an l2 run: window limits, pair counts and
// the band tile list.  Pure host code (no CUDA), shared by the C ABI and the
// CPU tests through ldsc_l2_left_limits / ldsc_l2_pair_count.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace ldsc {

// get_block_lefts_by_chr (src/l2/window.rs:32-90) over records [0, m):
// bl[i] = first record on i's chromosome within the window.  Returns
// any_full_chr_window.
bool block_lefts(int64_t m, const uint8_t* chr, const double* cm, const uint32_t* bp, int mode,
                 double wind, uint64_t half, int64_t* bl);

// Left limit of each record's pairs.  Pair (k, j), k < j, contributes to l2
// iff left[j] <= k.
//   masked  : left[j] = bl[j]                          (compute.rs:1855-1867, 2244-2257)
//   chunked : left[j] = start of the ring window of j's chunk, i.e.
//             cs - ceil((cs - bl[cs]) / c) * c with cs the chunk's first
//             record (compute.rs:1164-1184, 1288-1299); chunks start at each
//             chromosome in per-chromosome mode, at record 0 for --global-pass.
// A LeftLimits reused across calls keeps its storage (no fresh pages per call).
struct LeftLimits {
    std::vector<int64_t> left;
    std::vector<int64_t> bl;  // block lefts (scratch)
    uint64_t n_pairs = 0;
    uint64_t chunks = 0;
    bool any_full = false;
};
bool left_limits(int64_t m, const uint8_t* chr, const double* cm, const uint32_t* bp, int mode,
                 double wind, uint64_t half, uint32_t chunk, bool masking, bool global_pass,
                 LeftLimits* out, std::string* err);

// Band tiles of ta x tb records covering every pair left[j] <= k < j; the
// second form refills *out, keeping its storage.
std::vector<Tile> band_tiles(const std::vector<int64_t>& left, int ta, int tb);
void band_tiles(const std::vector<int64_t>& left, int ta, int tb, std::vector<Tile>* out);

// fastrand 2.3.0 WyRand stream as used by CountSketchProj::new
// (src/l2/compute.rs:179-184): n bucket draws u32(..d), then n bool draws.
void countsketch_hash(uint64_t n, uint32_t d, uint64_t seed, uint32_t* bucket, float* sign);

// Bucket-major order of the used individuals for the permuted-panel sketch:
// runs k = 2*bucket + (sign < 0), stable in individual order.
struct SketchOrder {
    std::vector<int32_t> perm;      // FAM index at each permuted position
    std::vector<int32_t> seg_off;   // 2d + 1 run starts
};
SketchOrder sketch_order(uint64_t n_used, uint32_t d, const uint32_t* bucket, const float* sign,
                         const int64_t* keep);

}  // namespace ldsc
