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

constexpr int kThroughputShapes = 18;
constexpr int kBandShapes = 23;
// Window shapes (lanes x 64-bit words a lane). Shapes 0-17, narrowest first from 1 to 512 words, each at
// most half again the last, so a tight first threshold gets a tight window; a lane holds up to 16 words,
// updated one after another as each word's carry feeds the next. Shapes 18-22 hold one word a lane (2 to
// 32 lanes): for a round of few pairs, where the GPU has lanes to spare and a pair's sweep waits on its
// longest chain of words, not on the issue rate.
__host__ __device__ inline int band_lanes(int shape) {
    const int lanes[kBandShapes] = {1, 1, 1, 1, 2, 4, 4, 8, 8, 16, 16, 32, 32, 32, 32, 32, 32, 32, 2, 4, 8, 16, 32};
    return lanes[shape];
}
__host__ __device__ inline int band_words_per_lane(int shape) {
    const int words[kBandShapes] = {1, 2, 3, 4, 3, 2, 3, 2, 3, 2, 3, 2, 3, 4, 6, 8, 12, 16, 1, 1, 1, 1, 1};
    return words[shape];
}

// The window that covers the band of threshold t: every cell of diagonal d with |d| + |d - delta| <= t,
// at most delta + 2e + 1 rows a column, e = (t - delta) / 2. The narrowest of shapes 0-17; or, for a
// round of few pairs (`latency`), the fewest words a lane: one word a lane up to 32 words, else 32
// lanes and the fewest words each.
__host__ __device__ inline int band_shape_for(int64_t n, int64_t m, int64_t t, bool latency = false) {
    const int64_t delta = m - n;
    const int64_t e = t > delta ? (t - delta) / 2 : 0;
    int64_t needed = (delta + 2 * e + 1 + 63) / 64 + 1;
    const int64_t words = (n + 63) / 64;
    if (needed > words) needed = words;
    if (latency) {
        if (needed <= 1) return 0;
        for (int s = kThroughputShapes; s < kBandShapes; ++s)
            if (band_lanes(s) >= needed) return s;
        for (int s = 11; s < kThroughputShapes; ++s)
            if (band_lanes(s) * band_words_per_lane(s) >= needed) return s;
        return kThroughputShapes - 1;
    }
    for (int s = 0; s < kThroughputShapes; ++s)
        if (band_lanes(s) * band_words_per_lane(s) >= needed) return s;
    return kThroughputShapes - 1;
}

// Runs band doubling over a batch whose ASCII letters and offsets are on the device already; writes
// every pair's distance (or its code) to `results` (device) and fills `report`.
void band_doubling(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                   const int64_t *first_thresholds_device, int64_t default_start, int64_t *results,
                   dinara_band_report *report);

// The learned band's first thresholds for a batch on the device (learned.cu): the predictor's cost
// times its margin, per pair (device array, valid until the next call).
const int64_t *predict_thresholds(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets);

}  // namespace dinara
