// Global Gotoh scores and decisions over a proven band of diagonals (reference band_groups.mojo: a band
// each pair's own score proves, leftovers swept whole).
#pragma once

#include "affine.cuh"

namespace dinara {

// The band a pair is swept over: 64 diagonals, 4 lanes of 16, from its lowest diagonal `low`.
constexpr int kBandLanes = 4;
constexpr int kBandColumns = 16;
constexpr int kBandWidth = kBandLanes * kBandColumns;

// The lowest diagonal (column less row) of a pair's band: the main diagonal, the end diagonal and those
// between, the slack shared either side. INT32_MIN when the band cannot hold both ends.
__host__ __device__ inline int32_t band_low_for(int64_t rows, int64_t columns) {
    const int64_t delta = columns - rows;
    const int64_t span = delta < 0 ? -delta : delta;
    if (span + 1 > kBandWidth) return INT32_MIN;
    const int64_t slack = (kBandWidth - 1 - span) / 2;
    return int32_t((delta < 0 ? delta : 0) - slack);
}

// Whether a pair can be swept over the band at all: both sides non-empty and both ends' diagonals in it.
__host__ __device__ inline bool band_eligible(uint32_t rows, uint32_t columns) {
    return rows > 0 && columns > 0 && band_low_for(rows, columns) != INT32_MIN;
}

// Whether a band score proves itself (the bound of band_groups.mojo:235-248, restated for a table's
// best entry `best` and gaps in the kernels' terms): any path visiting a diagonal outside [low, high]
// takes at least two gap runs and g gap letters, g from the nearest diagonal outside, so scores at most
// best * (rows + columns - g) / 2 + 2 open + (g - 2) extend; the band's score is the optimum, and every
// optimal path lies inside it, when both sides' bounds fall strictly below it.
__host__ __device__ inline bool band_proves(int64_t score, int64_t rows, int64_t columns, int64_t low, int64_t best,
                                            int64_t open, int64_t extend) {
    if (2 * extend - best > 0) return false;  // a gap letter beats half a best pair: no bound
    const int64_t delta = columns - rows;
    const int64_t high = low + kBandWidth - 1;
    const int64_t twice = 2 * score;
    // 2 x the bound for g gap letters.
    auto bound = [&](int64_t g) { return best * (rows + columns) + g * (2 * extend - best) + 4 * (open - extend); };
    if (high + 1 <= columns) {
        const int64_t g = 2 * (high + 1) - delta;
        if (!(twice > bound(g))) return false;
    }
    if (low - 1 >= -rows) {
        const int64_t g = delta - 2 * (low - 1);
        if (!(twice > bound(g))) return false;
    }
    return true;
}

// band_proves for a band of `width` diagonals from `low`: the same bound, the nearest diagonals outside
// being low - 1 and low + width.
__host__ __device__ inline bool band_proves_width(int64_t score, int64_t rows, int64_t columns, int64_t low,
                                                  int64_t width, int64_t best, int64_t open, int64_t extend) {
    if (2 * extend - best > 0) return false;
    const int64_t delta = columns - rows;
    const int64_t high = low + width - 1;
    const int64_t twice = 2 * score;
    auto bound = [&](int64_t g) { return best * (rows + columns) + g * (2 * extend - best) + 4 * (open - extend); };
    if (high + 1 <= columns && !(twice > bound(2 * (high + 1) - delta))) return false;
    if (low - 1 >= -rows && !(twice > bound(delta - 2 * (low - 1)))) return false;
    return true;
}

// The 16-bit pair sweep (banded_pairs_kernel) holds every value a pair's band takes as a 16-bit half of a
// register: real cells plus kPairBias, cells no path reaches from kPairUnreached up. With K the largest
// step a cell takes from its neighbour (the largest shifted table entry, or a gap's opening), a real
// value lies within (rows + columns + 2) K of the bias; the sweep also runs a few columns right of a
// pair's end and rows below it (to its group's last row), so a batch's pairs may take it when rows +
// columns + 130 <= kPairReach / K. Then real values lie in [bias - reach, bias + reach], unreached ones
// in [unreached, unreached + reach], the two stay apart by more than K, and every value and every
// value plus one step lies in [0, 0x8000): no half overflows and no half borrows from the other.
constexpr int32_t kPairBias = 16384;
constexpr int32_t kPairUnreached = 1024;
constexpr int32_t kPairReach = 7400;

// The largest rows + columns a pair of the 16-bit sweep may have under a table whose largest step is
// `step` (0 when the table's entries do not fit a byte or the step is past 512).
__host__ __device__ inline int32_t band_pair_limit(int32_t step, bool bytes_fit) {
    if (!bytes_fit || step <= 0 || step > 512) return 0;
    const int32_t limit = kPairReach / step - 130;
    return limit > 0 ? limit : 0;
}

struct BandedBatch {
    const uint32_t *tape;
    const PairShape *shapes;
    const uint32_t *order;  // pairs to sweep
    int64_t count;
    int32_t open, extend, best;
    uint2 rows16[4];        // the shifted table, 16 bits an entry
    uint32_t rows8[4];      // the shifted table, a byte an entry (the 16-bit pair sweep)
    int32_t *scores;        // by pair
    uint8_t *proven;        // by pair, when given: 1 when the band proved its score
    uint32_t *leftovers;    // pairs the band did not prove
    unsigned int *leftover_count;
    // Recording: 64-bit words, kBandLanes x rows_pad a pair, from decision_offsets[pair - first_pair].
    uint64_t *decisions;
    const int64_t *decision_offsets;
    int64_t first_pair;
    // Recording, when given: each pair's layout (by pair - first_pair), set to 4 where the narrow band
    // proved the pair. Counting, when given: the band cells the launch swept (rows x band width a pair).
    uint8_t *layouts;
    unsigned long long *band_cells;
};

// Launches the banded sweep (scores, or with `record` scores and decisions) over `batch.count` pairs; with
// `pairs_of_16` the 16-bit pair sweep, two pairs a lane group (every pair within band_pair_limit), over a
// band of `lanes` x 16 diagonals (2: the narrow first pass; 4: the full band).
void banded_launch(dinara_gpu *gpu, const BandedBatch &batch, bool record, bool pairs_of_16 = false,
                   int lanes = kBandLanes);

}  // namespace dinara
