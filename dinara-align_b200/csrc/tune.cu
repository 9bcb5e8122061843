// The band autotuner: measures on the device how fast each unit-cost window shape sweeps, and which bound
// on a pair's chain of word steps gives the shortest band doubling, and sets both on the context, where
// every later round's shape choice reads them (band_shape_for, edit.cuh). North of this file nothing
// about an answer depends on it: a shape only decides how a band is swept, never which band.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "edit.cuh"
#include "learned.cuh"

namespace dinara {
namespace {

constexpr int64_t kChainCandidates[] = {12000, 24000, 48000, 96000};
constexpr int kChainCount = int(sizeof(kChainCandidates) / sizeof(kChainCandidates[0]));
static_assert(2 * kChainCount <= 8, "the report holds every candidate");

// Each shape's words a millisecond, timed on pairs at least `length` letters long and at least eight words
// taller than the shape's window (so every lane sweeps words inside the pattern), at least two full waves
// of the shape's lane groups.
void measure_shapes(dinara_gpu *gpu, uint64_t seed, int64_t length, double rate, double *rates) {
    int64_t done = 0;  // shapes are timed in rounds of one probe length
    while (done < kBandShapes) {
        int64_t probe = 0;
        for (int s = 0; s < kBandShapes; ++s) {
            if (rates[s] > 0) continue;
            const int64_t wanted = std::max<int64_t>(length, 64 * (band_capacity(s) + 8));
            if (probe == 0 || wanted < probe) probe = wanted;
        }
        // This probe length's shapes: those it is long enough for and no shorter probe served.
        int64_t most = 0;
        for (int s = 0; s < kBandShapes; ++s) {
            if (rates[s] > 0 || std::max<int64_t>(length, 64 * (band_capacity(s) + 8)) > probe) continue;
            most = std::max<int64_t>(most, int64_t(band_shape_blocks(gpu, s)) * gpu->multiprocessors *
                                               (128 / band_lanes(s)));
        }
        const int64_t pairs = 2 * most;
        const GeneratedPairs generated = generate_pairs(gpu, seed, pairs, double(probe), double(probe), rate, rate);
        int64_t *results = gpu->distances.ensure<int64_t>(size_t(pairs));
        const PreparedPairs prepared = prepare_pairs(gpu, pairs, generated.letters, generated.offsets, results);
        int64_t *scratch = gpu->predictions.ensure<int64_t>(2 * size_t(pairs));
        for (int s = 0; s < kBandShapes; ++s) {
            if (rates[s] > 0 || std::max<int64_t>(length, 64 * (band_capacity(s) + 8)) > probe) continue;
            // Two waves of this shape's groups; a short first launch warms it.
            const int64_t groups = int64_t(band_shape_blocks(gpu, s)) * gpu->multiprocessors * (128 / band_lanes(s));
            const int64_t count = std::min(pairs, 2 * groups);
            band_shape_rate(gpu, s, std::min<int64_t>(count, 256), generated.letters, prepared, scratch);
            rates[s] = std::max(band_shape_rate(gpu, s, count, generated.letters, prepared, scratch), 1e-9);
            ++done;
        }
    }
}

}  // namespace


void band_autotune(dinara_gpu *gpu, const dinara_band_tune_options &options, dinara_band_tune_report &out) {
    const auto began = std::chrono::steady_clock::now();
    dinara_band_tune_options o = options;
    if (o.seed == 0) o.seed = 77;
    if (o.pairs <= 0) o.pairs = 50000;
    if (o.length_low <= 0) o.length_low = 100;
    if (o.length_high <= 0) o.length_high = 20000;
    if (o.rate_high <= 0) {
        o.rate_low = 0.005;
        o.rate_high = 0.15;
    }
    if (o.probe_length <= 0) o.probe_length = 4096;
    if (o.pairs > (int64_t(1) << 24) || o.length_low > o.length_high || o.length_high > 1e6 || o.rate_low < 0 ||
        o.rate_high > 0.5 || o.rate_low > o.rate_high || o.probe_length > 65536)
        throw Failure(DINARA_INVALID_LENGTH, "autotune options out of range");
    if (gpu->band_tuning.chain_words == 0) gpu->band_tuning = default_band_tuning();
    BandTuning tuning = gpu->band_tuning;
    std::memset(&out, 0, sizeof out);
    // 1. Each shape's sweep rate, on pairs of one length at the distribution's middle error rate.
    if (o.measure_shapes) {
        double rates[kBandShapes] = {0.0};
        measure_shapes(gpu, o.seed, o.probe_length, 0.5 * (o.rate_low + o.rate_high), rates);
        double fastest = 0.0;
        for (int s = 0; s < kBandShapes; ++s) fastest = std::max(fastest, rates[s]);
        for (int s = 0; s < kBandShapes; ++s) {
            out.words_per_ms[s] = rates[s];
            // Relative time a word: the fastest shape's 40 operations, the rest in proportion.
            tuning.word_cost[s] = rates[s] > 0 ? float(40.0 * fastest / rates[s]) : 1e30f;
        }
        out.shapes = kBandShapes;
    }
    // 2. The chain bound and the launches' grids: plain band doubling over pairs of the distribution, twice
    // a candidate.
    const GeneratedPairs generated =
        generate_pairs(gpu, o.seed + 1, o.pairs, o.length_low, o.length_high, o.rate_low, o.rate_high);
    int64_t *results = gpu->features.ensure<int64_t>(size_t(o.pairs));
    double best_ms = 0.0;
    int64_t best_chain = tuning.chain_words;
    int32_t best_grids = tuning.full_grids;
    for (int c = 0; c < 2 * kChainCount; ++c) {
        tuning.chain_words = kChainCandidates[c % kChainCount];
        tuning.full_grids = c / kChainCount;
        gpu->band_tuning = tuning;
        double fastest_run = 0.0;
        for (int repeat = 0; repeat < 2; ++repeat) {
            dinara_band_report band;
            std::memset(&band, 0, sizeof band);
            band_doubling(gpu, o.pairs, generated.letters, generated.offsets, nullptr, 0, results, &band);
            if (repeat == 0 || band.kernel_ms < fastest_run) fastest_run = band.kernel_ms;
        }
        out.chain_words_tried[c] = tuning.full_grids ? -tuning.chain_words : tuning.chain_words;
        out.chain_ms[c] = fastest_run;
        if (c == 0 || fastest_run < best_ms) {
            best_ms = fastest_run;
            best_chain = tuning.chain_words;
            best_grids = tuning.full_grids;
        }
    }
    out.chain_tried = 2 * kChainCount;
    out.full_grids = best_grids;
    tuning.chain_words = best_chain;
    tuning.full_grids = best_grids;
    tuning.tuned = 1;
    gpu->band_tuning = tuning;
    out.chain_words = best_chain;
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - began).count();
}

void band_tuning_access(dinara_gpu *gpu, bool set, int64_t *chain_words, int64_t *full_grids, float *word_costs) {
    if (gpu->band_tuning.chain_words == 0) gpu->band_tuning = default_band_tuning();
    if (set) {
        if (*chain_words < 1) throw Failure(DINARA_INVALID_LENGTH, "a chain bound below one word step");
        for (int s = 0; s < kBandShapes; ++s)
            if (!(word_costs[s] > 0.f) || !std::isfinite(word_costs[s]))
                throw Failure(DINARA_INVALID_LENGTH, "a word cost that is not a positive number");
        gpu->band_tuning.chain_words = *chain_words;
        gpu->band_tuning.full_grids = *full_grids ? 1 : 0;
        for (int s = 0; s < kBandShapes; ++s) gpu->band_tuning.word_cost[s] = word_costs[s];
        gpu->band_tuning.tuned = 1;
        return;
    }
    *chain_words = gpu->band_tuning.chain_words;
    *full_grids = gpu->band_tuning.full_grids;
    for (int s = 0; s < kBandShapes; ++s) word_costs[s] = gpu->band_tuning.word_cost[s];
}

}  // namespace dinara
