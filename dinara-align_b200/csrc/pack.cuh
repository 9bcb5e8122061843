// Packing the caller's letters on the device, and the longest-first schedule of a batch.
#pragma once

#include "internal.cuh"

namespace dinara {

// Packs pairs [first_pair, first_pair + count) of the device ASCII tape (offsets: 2 entries a pair and
// one more, from the batch's first letter) into their places on the batch's `tape`, each letter through
// `codes` (256 entries, 255 for a byte outside the alphabet), `bits` a letter; writes each pair's shape
// and flags a pair holding an unknown byte. Packing a batch a range at a time gives the tape, shapes and
// flags packing it whole gives.
void pack_pairs(dinara_gpu *gpu, const uint8_t *letters_device, const int64_t *offsets_device, int64_t first_pair,
                int64_t count, const uint8_t *codes_device, int bits, uint32_t *tape, PairShape *shapes,
                uint8_t *unknown);

// A batch's sweep order: pairs by class, classes in descending order, then strips and rows descending.
// Classes: the whole-matrix shape classes 0-4 (affine_shape_for with `record`); with `band` the proven
// band, kBandClass, and of those the pairs whose rows and columns sum to at most `limits.band`,
// kBandPairsClass, for the 16-bit pair band sweep; the whole-matrix pairs the 16-bit pair score sweep
// takes, kWholePairsClass plus the shape class; long pairs one block sweeps, kWideClass; and, recording,
// pairs whose widening band proved a width (`limits.band_widths`), kBandRecordClass. `order` is valid on
// the device until the next call.
constexpr int kClasses = 14;
constexpr int kBandClass = 5;
constexpr int kBandPairsClass = 6;
constexpr int kWholePairsClass = 7;
constexpr int kWideClass = 12;
constexpr int kBandRecordClass = 13;
// A pair a whole block sweeps (kWideClass), scoring without a CIGAR: at least this tall and this wide.
constexpr uint32_t kWideRows = 4096, kWideColumns = 2048;
struct Schedule {
    const uint32_t *order;
    int64_t counts[kClasses];
};

// Which pairs the 16-bit pair sweeps take: band pairs whose rows and columns sum to at most `band`; and,
// scoring without a CIGAR, non-empty whole-matrix pairs with best x swept columns + rows x row_step at
// most `whole` (local) or whose rows and swept columns are each at most half of it (global). Zero takes none. With `wide`,
// scoring without a CIGAR, whole-matrix pairs of at least kWideRows x kWideColumns go to kWideClass.
struct PairLimits {
    int32_t band = 0;
    int32_t whole = 0;
    int32_t local = 0;
    int32_t wide = 0;
    // Local: a pair fits when best x swept columns + rows x row_step is at most `whole`.
    int32_t best = 1;
    int32_t row_step = 0;
    // Recording: each pair's proven band width by pair - band_first (0: none), when given; a pair with one
    // goes to kBandRecordClass.
    const int32_t *band_widths = nullptr;
    int64_t band_first = 0;
};

// The order of pairs [first, first + count), or of the `count` pairs listed in `list` (device) when given.
Schedule schedule(dinara_gpu *gpu, const PairShape *shapes, const uint32_t *list, int64_t first, int64_t count,
                  bool record, bool band, PairLimits limits = PairLimits());

}  // namespace dinara
