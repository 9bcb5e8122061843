// The learned band predictor (placeholder until its kernels land).
#include "edit.cuh"

namespace dinara {

const int64_t *predict_thresholds(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets) {
    (void)pairs;
    (void)letters;
    (void)offsets;
    throw Failure(DINARA_INVALID_MODE, "no trained band predictor on this context");
    return gpu ? nullptr : nullptr;
}

}  // namespace dinara
