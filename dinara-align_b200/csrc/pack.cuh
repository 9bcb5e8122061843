// Packing the caller's letters on the device, and the longest-first schedule of a batch.
#pragma once

#include "internal.cuh"

namespace dinara {

// Packs pairs of the device ASCII tape (offsets: 2 pairs + 1 entries) into `tape`, each letter through
// `codes` (256 entries, 255 for a byte outside the alphabet), `bits` a letter; writes each pair's shape
// and flags a pair holding an unknown byte.
void pack_pairs(dinara_gpu *gpu, const uint8_t *letters_device, const int64_t *offsets_device, int64_t pairs,
                const uint8_t *codes_device, int bits, uint32_t *tape, PairShape *shapes, uint8_t *unknown);

// The order pairs [first, first + count) are swept in: by shape class (affine_shape_for with
// `record`), descending, then strips and rows, descending (device; valid until the next call).
const uint32_t *schedule(dinara_gpu *gpu, const PairShape *shapes, int64_t first, int64_t count, bool record);

}  // namespace dinara
