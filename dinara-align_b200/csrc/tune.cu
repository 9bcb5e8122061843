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

// Chain bounds tried: a floor in word steps, a share of the round's work per lane above it (0: none) and
// the reach in quarters of the smallest window.
constexpr int64_t kFloorCandidates[] = {24000, 48000, 96000, 12000, 24000, 48000, 24000, 48000};
constexpr double kShareCandidates[] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0};
constexpr int32_t kReachCandidates[] = {5, 5, 5, 8, 8, 8, 8, 8};
constexpr int kChainCount = int(sizeof(kShareCandidates) / sizeof(kShareCandidates[0]));
static_assert(kChainCount <= 8, "the report holds every candidate");

// First thresholds a tenth above each pair's distance: the rounds a learned start gives, for tuning.
__global__ void near_starts_kernel(const int64_t *__restrict__ distances, int64_t pairs, int64_t *__restrict__ starts) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < pairs) starts[k] = distances[k] >= 0 ? distances[k] + distances[k] / 10 + 8 : 1;
}

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
    // 2. The chain bound: band doubling over pairs of the distribution under each candidate, from the plain
    // start and from starts a tenth above each pair's distance (the one large round a learned start
    // gives), their device times summed, the fastest of two runs each.
    const GeneratedPairs generated =
        generate_pairs(gpu, o.seed + 1, o.pairs, o.length_low, o.length_high, o.rate_low, o.rate_high);
    int64_t *results = gpu->features.ensure<int64_t>(2 * size_t(o.pairs));
    int64_t *starts = results + o.pairs;
    gpu->band_tuning = tuning;
    band_doubling(gpu, o.pairs, generated.letters, generated.offsets, nullptr, 0, results, nullptr);
    near_starts_kernel<<<unsigned((o.pairs + 255) / 256), 256, 0, gpu->stream>>>(results, o.pairs, starts);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    double best_ms = 0.0;
    int best = 0;
    for (int c = 0; c < kChainCount; ++c) {
        tuning.chain_words = kFloorCandidates[c];
        tuning.chain_share = float(kShareCandidates[c]);
        tuning.reach = kReachCandidates[c];
        tuning.full_grids = 0;
        gpu->band_tuning = tuning;
        double total = 0.0;
        for (int start = 0; start < 2; ++start) {
            double fastest_run = 0.0;
            for (int repeat = 0; repeat < 2; ++repeat) {
                dinara_band_report band;
                std::memset(&band, 0, sizeof band);
                band_doubling(gpu, o.pairs, generated.letters, generated.offsets, start ? starts : nullptr, 0, results,
                              &band);
                if (repeat == 0 || band.kernel_ms < fastest_run) fastest_run = band.kernel_ms;
            }
            total += fastest_run;
            if (start) out.chain_ms_near[c] = fastest_run;
        }
        out.chain_words_tried[c] = kFloorCandidates[c];
        out.chain_share_tried[c] = kShareCandidates[c];
        out.reach_tried[c] = kReachCandidates[c];
        out.chain_ms[c] = total;
        if (c == 0 || total < best_ms) {
            best_ms = total;
            best = c;
        }
    }
    out.chain_tried = kChainCount;
    tuning.chain_words = kFloorCandidates[best];
    tuning.chain_share = float(kShareCandidates[best]);
    tuning.reach = kReachCandidates[best];
    tuning.full_grids = 0;
    tuning.tuned = 1;
    gpu->band_tuning = tuning;
    out.chain_words = tuning.chain_words;
    out.chain_share = tuning.chain_share;
    out.reach = tuning.reach;
    out.full_grids = 0;
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - began).count();
}

void band_tuning_access(dinara_gpu *gpu, bool set, dinara_band_tuning *values) {
    if (gpu->band_tuning.chain_words == 0) gpu->band_tuning = default_band_tuning();
    if (set) {
        if (values->chain_words < 1) throw Failure(DINARA_INVALID_LENGTH, "a chain bound below one word step");
        if (!(values->chain_share >= 0.0) || !std::isfinite(values->chain_share))
            throw Failure(DINARA_INVALID_LENGTH, "a chain share that is not a number at or above zero");
        for (int s = 0; s < kBandShapes; ++s)
            if (!(values->word_costs[s] > 0.f) || !std::isfinite(values->word_costs[s]))
                throw Failure(DINARA_INVALID_LENGTH, "a word cost that is not a positive number");
        gpu->band_tuning.chain_words = values->chain_words;
        gpu->band_tuning.chain_share = float(values->chain_share);
        if (values->reach < 5 || values->reach > 8) throw Failure(DINARA_INVALID_LENGTH, "a reach outside 5-8 quarters");
        gpu->band_tuning.reach = int32_t(values->reach);
        gpu->band_tuning.full_grids = values->full_grids ? 1 : 0;
        for (int s = 0; s < kBandShapes; ++s) gpu->band_tuning.word_cost[s] = values->word_costs[s];
        gpu->band_tuning.tuned = 1;
        return;
    }
    std::memset(values, 0, sizeof *values);
    values->chain_words = gpu->band_tuning.chain_words;
    values->chain_share = gpu->band_tuning.chain_share;
    values->reach = gpu->band_tuning.reach;
    values->full_grids = gpu->band_tuning.full_grids;
    for (int s = 0; s < kBandShapes; ++s) values->word_costs[s] = gpu->band_tuning.word_cost[s];
}

}  // namespace dinara
