// Gotoh scoring under a substitution table on the GPU: scores, recorded decisions, the walk back and
// the CIGAR, for global and local alignments (reference dinara_align/device_align.mojo,
// score_groups.mojo, gotoh.mojo).
#pragma once

#include "internal.cuh"

namespace dinara {

constexpr int kAffineShapes = 5;
// Lanes a pair and columns a lane of each compiled shape; a pair takes the narrowest shape spanning its
// columns, the widest in strips of 512 columns (shape 3 is a score-only width: 16 lanes of 20 columns).
__host__ __device__ inline int affine_lanes(int shape) {
    return shape == 0 ? 4 : shape == 1 ? 8 : shape == 2 ? 16 : shape == 3 ? 16 : 32;
}
__host__ __device__ inline int affine_columns(int shape) { return shape == 3 ? 20 : 16; }
__host__ __device__ inline int affine_shape_for(uint32_t columns, bool record) {
    if (columns <= 64) return 0;
    if (columns <= 128) return 1;
    if (columns <= 256) return 2;
    if (!record && columns <= 320) return 3;
    return 4;
}

// Lanes a pair's recording sweep takes: its shape class's, or 32 for the shared-memory table path,
// which sweeps every pair with one shape. The decisions' layout, their sizes and the walk all follow it.
__host__ __device__ inline int record_lanes(uint32_t columns, bool uniform) {
    return uniform ? 32 : affine_lanes(affine_shape_for(columns, true));
}

// The substitution table a launch reads, with the gaps in the kernels' terms: `open` a gap's first
// letter, `extend` each further one (scoring.mojo:202-215 gap_scores).
struct AffineTable {
    int32_t size;       // letters in the alphabet
    int32_t open, extend;
    int32_t entries[32 * 32];
    bool packed16;      // size <= 4 and every shifted entry fits 16 bits: the PRMT lookup serves
};

struct AffineBatch {
    int64_t pairs;
    int bits;            // 2 (alphabet of up to 4 letters) or 8 bits a letter on the packed tape
    bool local;
    const uint32_t *tape;
    const PairShape *shapes;
    uint32_t max_rows, max_columns;
    // Per-pair flags (the packing's unknown-letter flags): a walk that finds its path leaving the proven
    // band sets its pair's to kWalkFailed, which the host reports as DINARA_DEVICE_FAILURE. May be null.
    uint8_t *flags = nullptr;
    // Global scores with free ends (scored.mojo:69-240): letters at the reference's start and end and the
    // query's start and end that may go unaligned for nothing (at most INT32_MAX; a pair reads at most
    // its own length). `free_ends` is set when any is nonzero.
    bool free_ends = false;
    int32_t free_reference_start = 0, free_reference_end = 0, free_query_start = 0, free_query_end = 0;
    // An extension's stop (scoring.mojo:673-688 extension_span): from the origin, or with `from_end` from
    // both sequences' ends (read backwards), to the best cell anywhere; `free_ends` is then set too, with no
    // letters free. A Z-drop of `zdrop` (0 or more; negative: none) ends the sweep early
    // (scored.mojo:272-300); an `end_bonus` above zero takes the alignment reaching the query's far end when
    // its score plus the bonus passes the stop's and the sweep was not ended early (scoring.mojo:704-710).
    bool extension = false, from_end = false;
    int64_t zdrop = -1, end_bonus = -1;
};

// The flag value a failed walk leaves (1 is a letter outside the alphabet).
constexpr uint8_t kWalkFailed = 2;

// Whether a batch's global pairs may be swept over proven bands (a 2-bit alphabet, the 16-bit table and
// a bound that holds for its table): pairs the band does not prove are swept whole.
bool band_serves(const AffineBatch &batch, const AffineTable &table);

// Scores of pairs [first, first + count) of a packed batch into `scores` (device, indexed by pair): the
// proven band where it serves, every other pair over its whole matrix, longest first. With free ends and
// `spans` (device, 4 a pair of the range), each pair's span as the reference places it: the reference's
// first and last letter places, then the query's.
void affine_scores(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, int32_t *scores,
                   int64_t first, int64_t count, int64_t *spans = nullptr);

// Alignments of pairs [first_pair, first_pair + count): scores into `scores` (indexed by pair), spans (4
// per pair of the range: first row, last row, first column, last column of the walk) into `spans`, and
// each pair's CIGAR; returns the CIGAR bytes' total and leaves their offsets (count + 1, device) in
// gpu->cigar_offsets and the bytes in gpu->cigar_bytes.
int64_t affine_alignments(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, bool eqx,
                          int32_t *scores, int64_t *spans, int64_t first_pair, int64_t count);

}  // namespace dinara
