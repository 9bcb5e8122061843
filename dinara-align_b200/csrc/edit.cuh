// Unit-cost global edit distance on the GPU: banded Myers/Hyyro bit-vectors with band doubling
// (reference dinara_align/device_edit.mojo for the bit-vector step, band.mojo:526-657 for doubling).
#pragma once

#include "internal.cuh"

namespace dinara {

// A pair as the band kernels read it: the pattern (the shorter side, the query on a tie, as
// api.mojo:1286-1293 picks it) down the rows, the text across the columns, both as offsets into the
// device ASCII tape.
struct EditPair {
    int64_t pattern;
    int64_t text;
    int32_t n;      // pattern letters
    int32_t m;      // text letters
    int32_t dna;    // 1 when both sides hold only A, C, G, T: the kernel reads precomputed match planes
    int32_t words;  // ceil(n / 64)
};

// Window shapes: G lanes x K 64-bit words a lane, a lane one column behind the one above it and its K
// words updated one after another as each word's carry feeds the next. Shapes 0-35 are every G of 1, 2,
// 4, 8, 16, 32 with every K of 1 to 6 (shape 6 log2(G) + K - 1), so nearly every window height has a
// shape that holds it with no word to spare; shapes 36-38 are 32 lanes of 8, 12 and 16 words for the
// widest bands.
constexpr int kBandShapes = DINARA_BAND_SHAPES;
constexpr int kWidestShape = kBandShapes - 1;
static_assert(kBandShapes <= BandTuning::kShapes, "a word cost for every shape");
__host__ __device__ inline int band_lanes(int shape) { return shape < 36 ? 1 << (shape / 6) : 32; }
__host__ __device__ inline int band_words_per_lane(int shape) {
    return shape < 36 ? shape % 6 + 1 : (shape == 36 ? 8 : shape == 37 ? 12 : 16);
}
__host__ __device__ inline int64_t band_capacity(int shape) {
    return int64_t(band_lanes(shape)) * band_words_per_lane(shape);
}

// The words a window needs to hold the band of threshold t at every column: every cell of diagonal d with
// |d| + |d - delta| <= t lies within delta + 2e + 1 rows of a column, e = (t - delta) / 2, and a window
// that slides a word at a time needs one word more than those rows fill. At most the pattern's words.
__host__ __device__ inline int64_t band_words_needed(int64_t n, int64_t m, int64_t t) {
    const int64_t delta = m - n;
    const int64_t e = t > delta ? (t - delta) / 2 : 0;
    const int64_t needed = (delta + 2 * e + 1 + 63) / 64 + 1;
    const int64_t words = (n + 63) / 64;
    return needed < words ? needed : words;
}

// The widest band a window of `window` words holds: e at most (64 (window - 1) - delta - 1) / 2, the
// inverse of band_words_needed. Sweeping that band costs what sweeping a narrower one in the same window
// costs, and settles every pair whose distance lies within delta + 2e + 1.
__host__ __device__ inline int64_t band_reach(int64_t n, int64_t m, int64_t window) {
    const int64_t delta = m - n;
    const int64_t room = 64 * (window - 1) - delta - 1;
    return room < 0 ? -1 : room / 2;
}

// The shape for a pair's band of threshold t. Among shapes holding the band, within a quarter of the
// smallest that does: the cheapest a column (its words times its word cost) whose chain of word steps,
// m x K, stays within the tuning's chain_words; failing that, the same within the tuning's reach (up to
// twice the smallest: a long pair takes a wider window of fewer words a lane rather than hold its lanes
// for a long chain); failing that, the shortest chain. For a round of few pairs (`latency`: the GPU has lanes to spare and the round
// lasts as long as its longest chain), the fewest words a lane within twice the smallest window. A band
// past the widest shape takes the widest. The tuning's figures are BandTuning's (internal.cuh).
__host__ __device__ inline int band_shape_for(int64_t n, int64_t m, int64_t t, bool latency,
                                              const BandTuning &tuning) {
    const int64_t needed = band_words_needed(n, m, t);
    int64_t smallest = INT64_MAX;
    for (int s = 0; s < kBandShapes; ++s) {
        const int64_t c = band_capacity(s);
        if (c >= needed && c < smallest) smallest = c;
    }
    if (smallest == INT64_MAX) return kWidestShape;
    if (latency) {
        int best = -1;
        int64_t best_k = INT64_MAX, best_capacity = INT64_MAX;
        for (int s = 0; s < kBandShapes; ++s) {
            const int64_t c = band_capacity(s), k = band_words_per_lane(s);
            if (c < needed || c > 2 * smallest) continue;
            if (best < 0 || k < best_k || (k == best_k && c < best_capacity)) {
                best = s;
                best_k = k;
                best_capacity = c;
            }
        }
        return best;
    }
    // The cheapest shape whose chain fits, among those within a quarter of the smallest, then within the
    // tuning's reach.
    for (int reach = 5; reach <= tuning.reach; reach = reach < tuning.reach ? tuning.reach : reach + 1) {
        int best = -1;
        float best_cost = 0.f;
        for (int s = 0; s < kBandShapes; ++s) {
            const int64_t c = band_capacity(s);
            if (c < needed || 4 * c > reach * smallest) continue;
            if (m * band_words_per_lane(s) > tuning.chain_words) continue;
            const float cost = float(c) * tuning.word_cost[s];
            if (best < 0 || cost < best_cost) {
                best = s;
                best_cost = cost;
            }
        }
        if (best >= 0) return best;
    }
    // No chain fits: the shortest, then the cheapest, within the reach.
    int best = -1;
    int64_t best_chain = INT64_MAX;
    float best_cost = 0.f;
    for (int s = 0; s < kBandShapes; ++s) {
        const int64_t c = band_capacity(s);
        if (c < needed || 4 * c > (tuning.reach > 5 ? tuning.reach : 5) * smallest) continue;
        const int64_t chain = m * band_words_per_lane(s);
        const float cost = float(c) * tuning.word_cost[s];
        if (best < 0 || chain < best_chain || (chain == best_chain && cost < best_cost)) {
            best = s;
            best_chain = chain;
            best_cost = cost;
        }
    }
    return best;
}

// The tuning a context starts with: a word step costs its 40 operations plus a lane's work a column besides
// its words (about 18 operations) shared by its K words, and chains of up to 40,000 word steps whatever the
// round.
inline BandTuning default_band_tuning() {
    BandTuning t{};
    t.chain_words = 40000;
    for (int s = 0; s < BandTuning::kShapes; ++s)
        t.word_cost[s] = s < kBandShapes ? 40.f + 18.f / float(band_words_per_lane(s)) : 1e30f;
    t.chain_share = 0.f;
    t.reach = 5;
    t.tuned = 0;
    t.full_grids = 0;
    return t;
}

// A batch's pairs as the band kernels read them: shapes, DNA match planes, refusal flags (device).
struct PreparedPairs {
    EditPair *info;
    uint64_t *planes;
    int64_t *plane_offsets;
    uint8_t *status;
};
PreparedPairs prepare_pairs(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                            int64_t *results);

// The autotuner's probe: one launch of window shape `shape` over every prepared pair, on the context's
// stream; returns the words it swept per millisecond. `scratch` holds 2 x pairs int64 (device).
double band_shape_rate(dinara_gpu *gpu, int shape, int64_t pairs, const uint8_t *letters, const PreparedPairs &p,
                       int64_t *scratch);
// Resident blocks of 128 lanes a shape's kernel keeps on an SM.
int band_shape_blocks(dinara_gpu *gpu, int shape);

// The band autotuner (tune.cu): each shape's sweep rate and the chain bound, measured on the device and
// set on the context; and the tuning read back or installed (`set`).
void band_autotune(dinara_gpu *gpu, const dinara_band_tune_options &options, dinara_band_tune_report &report);
void band_tuning_access(dinara_gpu *gpu, bool set, dinara_band_tuning *values);

// Runs band doubling over a batch whose ASCII letters and offsets are on the device already; writes
// every pair's distance (or its code) to `results` (device) and fills `report`. `letters` starts on a
// 16-byte boundary and keeps 16 bytes of room past its last letter (the kernels read whole chunks).
void band_doubling(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                   const int64_t *first_thresholds_device, int64_t default_start, int64_t *results,
                   dinara_band_report *report);

// The learned band's first thresholds for a batch on the device (learned.cu): the predictor's cost
// times its margin, per pair (device array, valid until the next call).
const int64_t *predict_thresholds(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets);

}  // namespace dinara
