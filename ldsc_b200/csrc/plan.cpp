// plan.cpp -- see plan.h.
#include "plan.h"

#include <cmath>

namespace ldsc {

namespace {

// bl over one chromosome's records [start, start + len) by the reference's
// two-pointer walk: for each i, j moves forward while |x_i - x_j| > wind.
template <typename Coord>
void lefts_walk(int64_t start, int64_t len, double wind, Coord coord, int64_t* bl) {
    int64_t j = 0;
    for (int64_t i = 0; i < len; i++) {
        const double ci = coord(start + i);
        while (j < len && std::fabs(ci - coord(start + j)) > wind) j++;
        bl[start + i] = start + j;
    }
}

// The same result when the coordinates are non-decreasing and wind >= 0.
// Then x_i - x_j >= 0 for j <= i, the walk never passes i, and "x_i - x_j >
// wind" holds for a prefix of j (rounding is monotone), so walk i's j is the
// first j where it fails: a binary search gives it at any i.  The range is
// cut into WALKERS segments, each started by that search and then walked as
// in lefts_walk; the segments' walks are interleaved in one loop, so their
// dependent compare-and-advance chains overlap in the core.
template <typename Coord>
void lefts_sorted(int64_t start, int64_t len, double wind, Coord coord, int64_t* bl) {
    constexpr int WALKERS = 8;
    int64_t wi[WALKERS], wj[WALKERS], we[WALKERS];
    for (int w = 0; w < WALKERS; w++) {
        const int64_t i0 = len * w / WALKERS, i1 = len * (w + 1) / WALKERS;
        wi[w] = i0;
        we[w] = i1;
        int64_t lo = 0, hi = i0;  // first j in [0, i0] with !(x_i0 - x_j > wind)
        if (i0 < i1) {
            const double ci = coord(start + i0);
            while (lo < hi) {
                const int64_t mid = lo + (hi - lo) / 2;
                if (ci - coord(start + mid) > wind)
                    lo = mid + 1;
                else
                    hi = mid;
            }
        }
        wj[w] = lo;
    }
    for (;;) {
        bool busy = false;
#pragma GCC unroll 8
        for (int w = 0; w < WALKERS; w++) {
            if (wi[w] < we[w]) {
                busy = true;
                const bool adv = coord(start + wi[w]) - coord(start + wj[w]) > wind;
                bl[start + wi[w]] = start + wj[w];
                wj[w] += adv;
                wi[w] += !adv;
            }
        }
        if (!busy) break;
    }
}

}  // namespace

bool block_lefts(int64_t m, const uint8_t* chr, const double* cm, const uint32_t* bp, int mode,
                 double wind, uint64_t half, int64_t* bl) {
    bool any_full = false;
    int64_t start = 0;
    while (start < m) {
        const uint8_t c = chr[start];
        int64_t end = start + 1;
        while (end < m && chr[end] == c) end++;
        const int64_t len = end - start;
        if (mode == 2) {
            if ((int64_t)half >= (len > 0 ? len - 1 : 0)) any_full = true;
            for (int64_t i = 0; i < len; i++)
                bl[start + i] = start + (i > (int64_t)half ? i - (int64_t)half : 0);
        } else {
            auto run = [&](auto coord) {
                bool sorted = wind >= 0.0;  // NaN coordinates or window fail the comparisons
                for (int64_t r = start + 1; r < end; r++) sorted &= coord(r) >= coord(r - 1);
                if (sorted && len >= 64)
                    lefts_sorted(start, len, wind, coord, bl);
                else
                    lefts_walk(start, len, wind, coord, bl);
            };
            if (mode == 0)
                run([cm](int64_t r) { return cm[r]; });
            else
                run([bp](int64_t r) { return (double)bp[r] / 1000.0; });
            if (len > 0 && bl[end - 1] == start) any_full = true;
        }
        start = end;
    }
    return any_full;
}

bool left_limits(int64_t m, const uint8_t* chr, const double* cm, const uint32_t* bp, int mode,
                 double wind, uint64_t half, uint32_t chunk, bool masking, bool global_pass,
                 LeftLimits* out, std::string* err) {
    if (chunk < 1) {
        *err = "compute_ldscore_global: chunk_size must be >= 1, got 0";
        return false;
    }
    if (mode < 0 || mode > 2) {
        *err = "invalid window mode";
        return false;
    }
    if ((mode == 0 && !cm) || (mode == 1 && !bp) || (m > 0 && !chr)) {
        *err = "missing chr / cm / bp arrays for the window mode";
        return false;
    }
    out->left.resize((size_t)m);
    out->bl.resize((size_t)m);
    out->n_pairs = 0;
    out->chunks = 0;
    std::vector<int64_t>& bl = out->bl;
    out->any_full = block_lefts(m, chr, cm, bp, mode, wind, half, bl.data());
    // chunking groups: each chromosome (per-chromosome mode) or everything
    int64_t g0 = 0;
    while (g0 < m) {
        int64_t g1 = m;
        if (!global_pass) {
            g1 = g0 + 1;
            while (g1 < m && chr[g1] == chr[g0]) g1++;
        }
        const int64_t c = chunk;
        // locals, so the loop below does not go through *out on every record
        int64_t* left = out->left.data();
        const int64_t* blp = bl.data();
        uint64_t pairs = 0, chunks = 0;
        for (int64_t cs = g0; cs < g1; cs += c) {
            const int64_t ce = cs + c < g1 ? cs + c : g1;
            chunks++;
            // block_sizes[cs] within the group (compute.rs:1164-1173, 1288-1292)
            const int64_t dist = cs - blp[cs];
            int64_t b = dist == 0 ? 0 : ((dist + c - 1) / c) * c;
            if (b > cs - g0) b = cs - g0;
            const int64_t a_left = cs - b;
            for (int64_t j = cs; j < ce; j++) {
                const int64_t L = masking ? blp[j] : a_left;
                left[j] = L;
                pairs += (uint64_t)(j - L);
            }
        }
        out->n_pairs += pairs;
        out->chunks += chunks;
        g0 = g1;
    }
    return true;
}

std::vector<Tile> band_tiles(const std::vector<int64_t>& left, int ta, int tb) {
    std::vector<Tile> tiles;
    band_tiles(left, ta, tb, &tiles);
    return tiles;
}

void band_tiles(const std::vector<int64_t>& left, int ta, int tb, std::vector<Tile>* out) {
    std::vector<Tile>& tiles = *out;
    tiles.clear();
    const int64_t m = (int64_t)left.size();
    for (int64_t j0 = 0; j0 < m; j0 += tb) {
        const int64_t j1 = j0 + tb < m ? j0 + tb : m;
        // left is non-decreasing, so the block's smallest limit is left[j0]
        int64_t kmin = left[j0];
        for (int64_t j = j0 + 1; j < j1; j++) kmin = left[j] < kmin ? left[j] : kmin;
        const int64_t kmax = j1 - 2;  // largest k with k < j for some j in the block
        if (kmax < kmin) continue;
        // skip A blocks that contain no in-band pair
        for (int64_t a = kmin / ta; a <= kmax / ta; a++) {
            const int64_t ka0 = a * ta, ka1 = ka0 + ta - 1;
            bool any = false;
            for (int64_t j = j0; j < j1 && !any; j++) {
                const int64_t lo = left[j] > ka0 ? left[j] : ka0;
                const int64_t hi = (j - 1) < ka1 ? (j - 1) : ka1;
                any = lo <= hi;
            }
            if (any) tiles.push_back(Tile{(uint32_t)a, (uint32_t)(j0 / tb)});
        }
    }
}

// ---- fastrand 2.3.0 WyRand (independent restatement of the published
// algorithm; the crate is not vendored with the reference) ----
namespace {
struct WyRand {
    uint64_t s;
    uint64_t next() {
        s += 0x2d358dccaa6c78a5ull;
        const unsigned __int128 t = (unsigned __int128)s * (unsigned __int128)(s ^ 0x8bb84b93962eacc9ull);
        return (uint64_t)t ^ (uint64_t)(t >> 64);
    }
    // u32(..n): multiply-shift with rejection of the biased low products
    uint32_t below(uint32_t n) {
        uint32_t x = (uint32_t)next();
        uint64_t prod = (uint64_t)x * n;
        uint32_t lo = (uint32_t)prod;
        if (lo < n) {
            const uint32_t thresh = (uint32_t)(0u - n) % n;
            while (lo < thresh) {
                x = (uint32_t)next();
                prod = (uint64_t)x * n;
                lo = (uint32_t)prod;
            }
        }
        return (uint32_t)(prod >> 32);
    }
    // bool(): u8(..) % 2 == 0
    bool coin() { return ((uint8_t)(uint32_t)next() % 2) == 0; }
};
}  // namespace

void countsketch_hash(uint64_t n, uint32_t d, uint64_t seed, uint32_t* bucket, float* sign) {
    WyRand r{seed};
    for (uint64_t i = 0; i < n; i++) bucket[i] = r.below(d);
    for (uint64_t i = 0; i < n; i++) sign[i] = r.coin() ? 1.0f : -1.0f;
}

SketchOrder sketch_order(uint64_t n_used, uint32_t d, const uint32_t* bucket, const float* sign,
                         const int64_t* keep) {
    SketchOrder o;
    const uint32_t nseg = 2 * d;
    o.seg_off.assign(nseg + 1, 0);
    for (uint64_t i = 0; i < n_used; i++) o.seg_off[2 * bucket[i] + (sign[i] < 0 ? 1 : 0) + 1]++;
    for (uint32_t k = 0; k < nseg; k++) o.seg_off[k + 1] += o.seg_off[k];
    std::vector<int32_t> fill(o.seg_off.begin(), o.seg_off.end() - 1);
    o.perm.assign(n_used, 0);
    for (uint64_t i = 0; i < n_used; i++) {
        const uint32_t k = 2 * bucket[i] + (sign[i] < 0 ? 1 : 0);
        o.perm[fill[k]++] = (int32_t)(keep ? keep[i] : (int64_t)i);
    }
    return o;
}

}  // namespace ldsc
