// Packing the caller's letters on the device, and the longest-first schedule of a batch.
#pragma once

#include "internal.cuh"

namespace dinara {

// Packs pairs of the device ASCII tape (offsets: 2 pairs + 1 entries) into `tape`, each letter through
// `codes` (256 entries, 255 for a byte outside the alphabet), `bits` a letter; writes each pair's shape
// and flags a pair holding an unknown byte.
void pack_pairs(dinara_gpu *gpu, const uint8_t *letters_device, const int64_t *offsets_device, int64_t pairs,
                const uint8_t *codes_device, int bits, uint32_t *tape, PairShape *shapes, uint8_t *unknown);

// A batch's sweep order: pairs by class (the whole-matrix shape classes 0-4, affine_shape_for with
// `record`; with `band` the proven band, kBandClass, and of those the pairs whose rows and columns sum to
// at most `pair_limit`, kBandPairsClass, for the 16-bit pair sweep), classes in descending order, then
// strips and rows descending. `order` is valid on the device until the next call.
constexpr int kClasses = 7;
constexpr int kBandClass = 5;
constexpr int kBandPairsClass = 6;
struct Schedule {
    const uint32_t *order;
    int64_t counts[kClasses];
};

// The order of pairs [first, first + count), or of the `count` pairs listed in `list` (device) when given.
Schedule schedule(dinara_gpu *gpu, const PairShape *shapes, const uint32_t *list, int64_t first, int64_t count,
                  bool record, bool band, int32_t pair_limit = 0);

}  // namespace dinara
