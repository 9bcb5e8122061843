// The learned band predictor's shapes and the entry points capi.cu calls (learned.cu).
#pragma once

#include "internal.cuh"

namespace dinara {

// 256 4-mer count differences, the length ratio and the 6-mer squared count differences' sum.
constexpr int kPredictorInputs = 258;
constexpr int kPredictorHidden = 64;
// w1 [258][64], b1 [64], w2 [64][64], b2 [64], w3 [64], b3 [1], flat in that order.
constexpr int kPredictorParameters =
    kPredictorInputs * kPredictorHidden + kPredictorHidden + kPredictorHidden * kPredictorHidden + kPredictorHidden +
    kPredictorHidden + 1;

// Features of pairs on the device into a feature-major matrix (feature f of pair p at f * pairs + p).
void predictor_features(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets, float *features);

// One batch's gradients of the summed squared error over the mean, for the context's parameters: the
// features feature-major ([258][batch]), targets, gradients and the squared error's sum on the device.
void predictor_gradients(dinara_gpu *gpu, int batch, const float *features, const float *targets, float *grads,
                         float *loss);

// Pairs drawn on the device from the uneven distribution (reference lengths log-uniform in [length_low,
// length_high], an error rate uniform in [rate_low, rate_high] split 50/25/25), into the context's letters
// and offsets buffers (valid until their next use).
struct GeneratedPairs {
    int64_t *offsets;
    uint8_t *letters;
    int64_t letters_total;
};
GeneratedPairs generate_pairs(dinara_gpu *gpu, uint64_t seed, int64_t pairs, double length_low, double length_high,
                              double rate_low, double rate_high);

// Trains the context's predictor on device-generated pairs and sets its margin.
void predictor_train(dinara_gpu *gpu, const dinara_train_options &options, dinara_train_report &report);

}  // namespace dinara
