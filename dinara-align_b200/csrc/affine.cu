// Gotoh scores and alignments under a substitution table on the B200.
//
// A group of G lanes sweeps one pair, several pairs a warp: lane `m` of a group holds C consecutive
// columns in registers and runs one row behind lane m-1, whose last column's score and insertion layer
// arrive by one shuffle a row (the layout of the reference's score_groups.mojo:78-236 and
// device_align.mojo:216-263 strip_row). A pair wider than a group's G*C columns is swept in strips,
// the column left of each strip carried through global memory.
//
// Global cells are held shifted by (row + column) * extend (score_groups.mojo:114-120), so the three
// layers take one fused add-and-max each (the DPX `viaddmax`), and the insertion layer's dependency
// along a row collapses to a running maximum of the cells before it: five instructions a cell, one of
// them on the row's dependent chain. The substitution comes from a 4 x 4 table of 16-bit entries held
// in two registers a row letter, picked by one PRMT whose selector is fixed per column.
//
// Recording (for the CIGAR) writes each cell's 4-bit decision exactly as gotoh.mojo:173-186 `decide`
// gives it, 16 columns to a 64-bit word, four rows buffered in registers and stored as one 32-byte
// sector; a thread a pair then walks them back by gotoh.mojo:189-200 `advance`.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "affine.cuh"
#include "affine_kernel.cuh"
#include "banded.cuh"
#include "pack.cuh"

namespace dinara {

namespace {

using namespace sweep;

// ------------------------------------------------------------------------------------------------
// The walk back and the CIGAR
// ------------------------------------------------------------------------------------------------

struct WalkArgs {
    const uint32_t *tape;
    const PairShape *shapes;
    const uint64_t *decisions;
    const uint64_t *decisions_extra;  // the band's leftovers, swept whole afterwards
    // Per pair: 0 whole matrix, 1 band, 2 whole matrix in decisions_extra, 3 and 4 the 16-bit pair band's
    // planes over 64 and 32 diagonals, 5 a band-recorded pair's strips over its proven width (widths[k]).
    const uint8_t *layouts;
    const int32_t *widths;
    const int64_t *decision_offsets;
    const int64_t *ends;
    const int64_t *slot_offsets;  // per pair: its CIGAR slot, a 32-bit run word a letter of the pair and 8 bytes
    char *slots;
    int64_t *lengths;             // per pair: the CIGAR's bytes
    int64_t *run_counts;          // per pair: the CIGAR's runs, left in its slot back to front
    const uint32_t *order;        // the pairs in the sweep's order, when given
    uint8_t *failed;              // per pair of the batch: set to kWalkFailed when a path leaves its band
    int64_t *spans;               // per pair: first row, last row, first column, last column
    int64_t first_pair, count;
    int bits;
    bool local, eqx, uniform;
};

// A run of the CIGAR as the walk leaves it, one 32-bit word: the op in the top two bits (kRunD a letter
// of the reference alone, kRunI of the query alone, kRunM an aligned pair (a match with eqx), kRunX a
// mismatch with eqx) and its length in the low 30 (a pair's letters stay far below 2^30: ScoreReach).
constexpr uint32_t kRunD = 0, kRunI = 1, kRunM = 2, kRunX = 3;
constexpr uint32_t kRunLength = (1u << 30) - 1;

__device__ __forceinline__ int decimal_digits(uint32_t n) {
    return 1 + (n >= 10u) + (n >= 100u) + (n >= 1000u) + (n >= 10000u) + (n >= 100000u) + (n >= 1000000u) +
           (n >= 10000000u) + (n >= 100000000u) + (n >= 1000000000u);
}

// One thread a pair walks its decisions back from its end (gotoh.mojo:189-200 `advance`), taking the pairs
// in the sweep's order (a class at a time, longest first), so a warp's walks are alike in layout and end
// together. Each step is one dependent read of a decision word and selects; the CIGAR leaves as runs
// (back to front), their text's length counted, for cigar_text_kernel to spell.
template <int BITS>
__global__ void walk_kernel(WalkArgs a) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const int64_t k = a.order ? int64_t(a.order[i]) - a.first_pair : i;
    const int64_t pair = a.first_pair + k;
    const PairShape sh = a.shapes[pair];
    const int rows = int(sh.rows), cols = int(sh.columns);
    uint32_t *runs = reinterpret_cast<uint32_t *>(a.slots + a.slot_offsets[k]);
    int64_t run_count = 0, text = 0;
    int row, column;
    if (a.local) {
        const int64_t end = a.ends[k];
        row = int(end >> 32);
        column = int(end & 0xffffffff);
    } else {
        row = rows;
        column = cols;
    }
    const int end_row = row, end_col = column;
    uint32_t run = kRunD, length = 0;
    // `n` more letters of op `op`: a new run when the op changes, the last one left as a word.
    auto add = [&](uint32_t op, uint32_t n) {
        if (op != run) {
            if (length > 0) {
                runs[run_count++] = (run << 30) | length;
                text += 1 + decimal_digits(length);
            }
            run = op;
            length = 0;
        }
        length += n;
    };
    if (rows > 0 && cols > 0) {
        const int layout = a.layouts[k];
        const uint64_t *decisions = layout == 2 ? a.decisions_extra : a.decisions;
        const int G = record_lanes(uint32_t(cols), a.uniform);
        const int lane_shift = __ffs(G * 16) - 1;  // a strip is G lanes of 16 columns
        const bool banded = layout == 1 || layout == 3 || layout == 4;
        const bool planes = layout == 3 || layout == 4;
        const int width = layout == 4 ? kBandWidth / 2 : kBandWidth;  // layout 4: the narrow band's 32
        const int rows_pad = banded ? ((rows + 3) & ~3) : (((rows + 2) | 3) + 1);
        const int low = banded ? band_low_for_width(rows, cols, width) : 0;
        const int64_t base = a.decision_offsets[k];
        // Layout 5: the strip under the walk, its swept rows and its first word (past the earlier strips').
        int strip = 0, strip_first = 1, strip_last = 0, strip_pad = 0, band_low = 0, band_high = 0;
        int64_t strip_at = 0;
        if (layout == 5) {
            const int proven = a.widths[k];
            band_low = band_low_for_width(rows, cols, proven);
            band_high = band_low + proven - 1;
            strip = (cols - 1) / kRecordStrip;
            for (int s = 0; s < strip; ++s)
                strip_at += 32 * int64_t(band_strip_pad(band_strip_first_row(s, band_high),
                                                        band_strip_last_row(s, rows, cols, band_low)));
            strip_first = band_strip_first_row(strip, band_high);
            strip_last = band_strip_last_row(strip, rows, cols, band_low);
            strip_pad = band_strip_pad(strip_first, strip_last);
        }
        int state = 0;  // 0 aligning, 1 deleting, 2 inserting
        // The decision sector under the walk (four words, 32 bytes, from a multiple of four: every layout's
        // lane blocks start there and run up by rows) and the tape words under its letters, kept in registers:
        // a step reads memory only when it leaves them, about one step in four.
        int64_t sector = -1;
        uint64_t held0 = 0, held1 = 0, held2 = 0, held3 = 0;
        constexpr uint32_t per_word = 32 / BITS;
        uint32_t row_word_at = ~0u, column_word_at = ~0u, row_word = 0, column_word = 0;
        while (row > 0 && column > 0) {
            int64_t at;
            int slot_in;
            if (layout == 5) {
                // Strips are left behind right to left: step back over each one the column has passed.
                while (strip > (column - 1) / kRecordStrip) {
                    --strip;
                    strip_first = band_strip_first_row(strip, band_high);
                    strip_last = band_strip_last_row(strip, rows, cols, band_low);
                    strip_pad = band_strip_pad(strip_first, strip_last);
                    strip_at -= 32 * int64_t(strip_pad);
                }
                // The proof keeps every optimal path inside the band, which the swept rows hold; a row
                // outside them would read another strip's decisions, so the walk stops and flags the pair.
                if (row < strip_first || row > strip_last) {
                    if (a.failed) a.failed[pair] = kWalkFailed;
                    break;
                }
                const int within = (column - 1) % kRecordStrip;
                const int member = within / 16;
                slot_in = within % 16;
                at = base + strip_at + int64_t(member) * strip_pad + (row - strip_first + (member & 3));
            } else {
                // The band's layout: place o = column - row - low, a lane of 16 places a block of rows. The
                // proof keeps every optimal path inside the band; a place outside it would read another
                // pair's decisions, so the walk stops there instead and flags the pair, whose CIGAR the host
                // then reports as a device failure rather than a result.
                const int place = column - row - low;
                if (banded && unsigned(place) >= unsigned(width)) {
                    if (a.failed) a.failed[pair] = kWalkFailed;
                    break;
                }
                // The whole matrix's: strips of G lanes, each lane's rows skewed by its place in a sector.
                const int off = column - 1;
                const int member = (off & ((1 << lane_shift) - 1)) >> 4;
                const int64_t whole_at =
                    base + int64_t((off >> lane_shift) * G + member) * rows_pad + (row - 1 + (member & 3));
                const int64_t band_at = base + int64_t(place >> 4) * rows_pad + (row - 1);
                at = banded ? band_at : whole_at;
                slot_in = (banded ? place : off) & 15;
            }
            if ((at & ~int64_t(3)) != sector) {
                sector = at & ~int64_t(3);
                const uint4 low_words = *reinterpret_cast<const uint4 *>(decisions + sector);
                const uint4 high_words = *reinterpret_cast<const uint4 *>(decisions + sector + 2);
                held0 = uint64_t(low_words.x) | (uint64_t(low_words.y) << 32);
                held1 = uint64_t(low_words.z) | (uint64_t(low_words.w) << 32);
                held2 = uint64_t(high_words.x) | (uint64_t(high_words.y) << 32);
                held3 = uint64_t(high_words.z) | (uint64_t(high_words.w) << 32);
            }
            const int within_sector = int(at & 3);
            const uint64_t word = within_sector == 0   ? held0
                                  : within_sector == 1 ? held1
                                  : within_sector == 2 ? held2
                                                       : held3;
            // The 16-bit pair band's planes: bit `slot_in` of deleting, inserting, deletion extending and
            // insertion extending, 16 bits each; inserting wins over deleting as decide() orders them.
            // Otherwise a nibble a place.
            const uint32_t deleting = uint32_t(word >> slot_in) & 1u, inserting = uint32_t(word >> (16 + slot_in)) & 1u;
            const uint32_t from_planes = (inserting ? 2u : deleting) | ((uint32_t(word >> (32 + slot_in)) & 1u) << 2) |
                                         ((uint32_t(word >> (48 + slot_in)) & 1u) << 3);
            const uint32_t nibble = planes ? from_planes : uint32_t(word >> (4 * slot_in)) & 15u;
            if (a.local && state == 0 && (nibble & 3u) == 3u) break;
            const int moving = state == 0 ? int(nibble & 3u) : state;
            uint32_t op = moving == 1 ? kRunD : moving == 2 ? kRunI : kRunM;
            if (a.eqx && op == kRunM) {
                const uint32_t x_at = uint32_t(row - 1), y_at = uint32_t(column - 1);
                if (x_at / per_word != row_word_at) {
                    row_word_at = x_at / per_word;
                    row_word = __ldg(a.tape + sh.first_word + row_word_at);
                }
                if (y_at / per_word != column_word_at) {
                    column_word_at = y_at / per_word;
                    column_word = __ldg(a.tape + sh.second_word + column_word_at);
                }
                constexpr uint32_t mask = BITS == 8 ? 0xFFu : (1u << BITS) - 1u;
                const uint32_t x = (row_word >> (BITS * (x_at % per_word))) & mask;
                const uint32_t y = (column_word >> (BITS * (y_at % per_word))) & mask;
                op = x == y ? kRunM : kRunX;
            }
            add(op, 1);
            state = moving == 1 ? int((nibble >> 2) & 1u) : moving == 2 ? 2 * int((nibble >> 3) & 1u) : 0;
            row -= moving != 2;
            column -= moving != 1;
        }
    }
    if (!a.local) {
        // gotoh.mojo:440-447: a global walk's rest is gaps against the letters left, rows first.
        if (row > 0) add(kRunD, uint32_t(row));
        if (column > 0) add(kRunI, uint32_t(column));
        row = column = 0;
    }
    if (length > 0) {
        runs[run_count++] = (run << 30) | length;
        text += 1 + decimal_digits(length);
    }
    a.lengths[k] = text;
    a.run_counts[k] = run_count;
    int64_t *span = a.spans + 4 * k;
    span[0] = row;
    span[1] = end_row;
    span[2] = column;
    span[3] = end_col;
}

// Each pair's CIGAR text from its runs, which the walk left back to front: a warp a pair, 32 runs at a time
// in the CIGAR's order, each lane's place in the text by a prefix sum of the runs' lengths in letters.
__global__ void cigar_text_kernel(const char *__restrict__ slots, const int64_t *__restrict__ slot_offsets,
                                  const int64_t *__restrict__ run_counts, const int64_t *__restrict__ offsets, bool eqx,
                                  char *__restrict__ out, int64_t count) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;
    const uint32_t *runs = reinterpret_cast<const uint32_t *>(slots + slot_offsets[warp]);
    const int64_t n = run_counts[warp];
    char *to = out + offsets[warp];
    // The ops' letters by run op, a byte each.
    const uint32_t ops = uint32_t('D') | (uint32_t('I') << 8) | (uint32_t(eqx ? '=' : 'M') << 16) | (uint32_t('X') << 24);
    int64_t at = 0;
    for (int64_t first = 0; first < n; first += 32) {
        const int64_t j = first + lane;
        uint32_t word = 0;
        int letters = 0;
        if (j < n) {
            word = runs[n - 1 - j];
            letters = 1 + decimal_digits(word & kRunLength);
        }
        int through = letters;  // inclusive prefix sum over the warp's runs
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int before = __shfl_up_sync(kFull, through, d);
            if (lane >= d) through += before;
        }
        if (j < n) {
            // The count's digits, then the op, ending at the run's last letter.
            char *p = to + at + through - 1;
            *p-- = char((ops >> (8 * (word >> 30))) & 0xFFu);
            uint32_t value = word & kRunLength;
            do {
                *p-- = char('0' + value % 10u);
                value /= 10u;
            } while (value > 0);
        }
        at += __shfl_sync(kFull, through, 31);
    }
}

__global__ void slot_sizes_kernel(const PairShape *__restrict__ shapes, int64_t first_pair, int64_t count, bool uniform,
                                  int32_t band_pair_limit, bool band, const int32_t *__restrict__ widths,
                                  int64_t *__restrict__ decision_words, int64_t *__restrict__ slot_bytes,
                                  uint8_t *__restrict__ layouts) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[first_pair + k];
    int64_t words = 0;
    uint8_t layout = 0;
    if (widths && widths[k] > 0) {
        // A long pair whose widening band proved a width: its strips' swept rows (layout 5).
        layout = 5;
        words = band_record_words(int(sh.rows), int(sh.columns), widths[k]);
    } else if (band && band_eligible(sh.rows, sh.columns)) {
        // The 16-bit pair band (its pairs' rows and columns within the limit) records planes (layout 3).
        layout = int64_t(sh.rows) + sh.columns <= band_pair_limit ? 3 : 1;
        words = int64_t(kBandLanes) * ((int64_t(sh.rows) + 3) & ~int64_t(3));
    } else if (sh.rows > 0 && sh.columns > 0) {
        const int G = record_lanes(sh.columns, uniform);
        const int W = G * 16;
        const int64_t strips = (sh.columns + W - 1) / W;
        const int64_t rows_pad = ((int64_t(sh.rows) + 2) | 3) + 1;
        words = strips * G * rows_pad;
    }
    decision_words[k] = words;
    slot_bytes[k] = 4 * (int64_t(sh.rows) + sh.columns) + 8;
    layouts[k] = layout;
}

// Cells a batch's sweeps update: 64 a row for a banded pair (out[0]); the whole matrix for the rest and
// again for each leftover of the band, and a band-recorded pair's strips (widths, when given) (out[1]).
__global__ void swept_cells_kernel(const PairShape *__restrict__ shapes, int64_t first, int64_t count, bool band,
                                   const uint32_t *__restrict__ leftovers, int64_t left,
                                   const int32_t *__restrict__ widths, unsigned long long *__restrict__ out) {
    unsigned long long banded = 0, whole = 0;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < count + left;
         k += int64_t(gridDim.x) * blockDim.x) {
        const PairShape sh = k < count ? shapes[first + k] : shapes[leftovers[k - count]];
        if (k < count && widths && widths[k] > 0)
            whole += (unsigned long long)band_record_cells(int(sh.rows), int(sh.columns), widths[k]);
        else if (k < count && band && band_eligible(sh.rows, sh.columns))
            banded += (unsigned long long)sh.rows * kBandWidth;
        else
            whole += (unsigned long long)sh.rows * sh.columns;
    }
#pragma unroll
    for (int span = 16; span > 0; span >>= 1) {
        banded += __shfl_xor_sync(0xffffffffu, banded, span);
        whole += __shfl_xor_sync(0xffffffffu, whole, span);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, banded);
        atomicAdd(out + 1, whole);
    }
}

// The whole-matrix words of each leftover pair of the band.
__global__ void leftover_words_kernel(const PairShape *__restrict__ shapes, const uint32_t *__restrict__ leftovers,
                                      int64_t count, bool uniform, int64_t *__restrict__ words) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[leftovers[k]];
    const int G = record_lanes(sh.columns, uniform);
    const int W = G * 16;
    words[k] = (int64_t(sh.columns) + W - 1) / W * G * (((int64_t(sh.rows) + 2) | 3) + 1);
}

// The pairs of [first, first + count) a block sweeps when scoring (kWideRows x kWideColumns or more), listed.
__global__ void long_pairs_kernel(const PairShape *__restrict__ shapes, int64_t first, int64_t count,
                                  uint32_t *__restrict__ list, unsigned int *__restrict__ listed) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[first + k];
    if (sh.rows >= kWideRows && sh.columns >= kWideColumns) list[atomicAdd(listed, 1u)] = uint32_t(first + k);
}

// Points each leftover's decisions at its place in the extra buffer and marks its layout.
__global__ void leftover_places_kernel(const uint32_t *__restrict__ leftovers, int64_t count, int64_t first_pair,
                                       const int64_t *__restrict__ offsets, int64_t *__restrict__ decision_offsets,
                                       uint8_t *__restrict__ layouts) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t pair = int64_t(leftovers[k]) - first_pair;
    decision_offsets[pair] = offsets[k];
    layouts[pair] = 2;
}

// ------------------------------------------------------------------------------------------------
// Launching
// ------------------------------------------------------------------------------------------------

using KernelFn = void (*)(KernelArgs, TableArgs, const int32_t *);

template <int G, int C, bool LOCAL, bool RECORD, int BITS, bool SMEM>
KernelFn kernel_of() {
    return &affine_kernel<G, C, LOCAL, RECORD, BITS, SMEM>;
}

// The kernel for a shape class; record kernels exist for the 16-column shapes only.
KernelFn pick_kernel(int cls, bool local, bool record, int bits, bool smem) {
    if (smem || bits == 8) {
        // The general path: any alphabet of up to 32 letters, the table in shared memory, one shape.
        if (bits == 8) {
            if (local) return record ? kernel_of<32, 16, true, true, 8, true>() : kernel_of<32, 16, true, false, 8, true>();
            return record ? kernel_of<32, 16, false, true, 8, true>() : kernel_of<32, 16, false, false, 8, true>();
        }
        if (local) return record ? kernel_of<32, 16, true, true, 2, true>() : kernel_of<32, 16, true, false, 2, true>();
        return record ? kernel_of<32, 16, false, true, 2, true>() : kernel_of<32, 16, false, false, 2, true>();
    }
#define DINARA_SHAPE(G, C)                                                                                       \
    if (local)                                                                                                   \
        return record ? kernel_of<G, C, true, true, 2, false>() : kernel_of<G, C, true, false, 2, false>();      \
    return record ? kernel_of<G, C, false, true, 2, false>() : kernel_of<G, C, false, false, 2, false>();
    switch (cls) {
        case 0: {
            DINARA_SHAPE(4, 16)
        }
        case 1: {
            DINARA_SHAPE(8, 16)
        }
        case 2: {
            DINARA_SHAPE(16, 16)
        }
        case 3: {
            if (local) return kernel_of<16, 20, true, false, 2, false>();
            return kernel_of<16, 20, false, false, 2, false>();
        }
        default: {
            DINARA_SHAPE(32, 16)
        }
    }
#undef DINARA_SHAPE
}

// The 16-bit pair score sweep for a whole-matrix shape class.
KernelFn pick_pairs_kernel(int cls, bool local) {
    switch (cls) {
        case 0: return local ? &affine_pairs_kernel<4, 16, true> : &affine_pairs_kernel<4, 16, false>;
        case 1: return local ? &affine_pairs_kernel<8, 16, true> : &affine_pairs_kernel<8, 16, false>;
        case 2: return local ? &affine_pairs_kernel<16, 16, true> : &affine_pairs_kernel<16, 16, false>;
        case 3: return local ? &affine_pairs_kernel<16, 20, true> : &affine_pairs_kernel<16, 20, false>;
        default: return local ? &affine_pairs_kernel<32, 16, true> : &affine_pairs_kernel<32, 16, false>;
    }
}

int persistent_blocks(dinara_gpu *gpu, KernelFn fn) {
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    if (per_sm < 1) per_sm = 1;
    return per_sm * gpu->multiprocessors;
}

TableArgs table_args(const AffineTable &table, bool local) {
    TableArgs t;
    std::memset(&t, 0, sizeof t);
    t.size = table.size;
    if (table.packed16) {
        for (int r = 0; r < 4; ++r) {
            uint16_t e[4] = {0, 0, 0, 0};
            for (int c = 0; c < 4; ++c) {
                int32_t v = 0;
                if (r < table.size && c < table.size) {
                    v = table.entries[r * 32 + c];
                    if (!local) v -= 2 * table.extend;
                }
                e[c] = uint16_t(int16_t(v));
            }
            t.rows16[r].x = uint32_t(e[0]) | (uint32_t(e[1]) << 16);
            t.rows16[r].y = uint32_t(e[2]) | (uint32_t(e[3]) << 16);
            // The byte table of the 16-bit pair sweeps, local entries less extend as that sweep holds local
            // cells (entries past a byte never reach them: the schedule keeps such tables off it).
            t.rows8[r] = 0;
            for (int c = 0; c < 4; ++c) {
                const int32_t v = int32_t(int16_t(e[c])) - (local && r < table.size && c < table.size ? table.extend : 0);
                t.rows8[r] |= uint32_t(uint8_t(int8_t(v))) << (8 * c);
            }
        }
    }
    return t;
}

// The table for the shared-memory path: 32 rows of 33 entries, entry 32 of each (a padding column)
// far below any score, so a padded cell never beats a real one.
void upload_table32(dinara_gpu *gpu, const AffineTable &table, bool local, int32_t **out) {
    std::vector<int32_t> host(32 * 33, 0);
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 33; ++c) {
            int32_t v = (r < table.size && c < table.size) ? table.entries[r * 32 + c] : 0;
            if (c == 32) v = -(1 << 20);
            else if (!local) v -= 2 * table.extend;
            host[r * 33 + c] = v;
        }
    // The device copy is kept while the table stays the same: a batch's units each sweep with it, and a
    // copy queued behind the batch's letters would wait for all of them.
    if (gpu->table32_host != host || !gpu->table32.ptr) {
        int32_t *dev = gpu->table32.ensure<int32_t>(host.size());
        DINARA_CUDA(
            cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(int32_t), cudaMemcpyHostToDevice, gpu->stream));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        gpu->table32_host = host;
    }
    *out = gpu->table32.as<int32_t>();
}

// The sorted order's range of each class: classes in descending order (the whole-matrix 16-bit pair
// classes, then the band's two, then the whole-matrix classes 4 to 0).
struct Buckets {
    int64_t begin[kClasses];
    int64_t end[kClasses];
};

Buckets buckets_of(const Schedule &schedule) {
    Buckets b;
    int64_t at = 0;
    for (int cls = kClasses - 1; cls >= 0; --cls) {
        b.begin[cls] = at;
        at += schedule.counts[cls];
        b.end[cls] = at;
    }
    return b;
}

// Device time of a sweep phase, added to the context's tally while it times.
struct PhaseTimer {
    dinara_gpu *gpu;
    double *into;
    explicit PhaseTimer(dinara_gpu *g, double *target) : gpu(g), into(target) {
        if (gpu->timing) DINARA_CUDA(cudaEventRecord(gpu->start, gpu->stream));
    }
    void stop() {
        if (!gpu->timing) return;
        DINARA_CUDA(cudaEventRecord(gpu->stop, gpu->stream));
        DINARA_CUDA(cudaEventSynchronize(gpu->stop));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
        *into += ms;
    }
};

// A widening band round's routing. A pair swept over its band of `swept[k]` diagonals keeps its score
// when the band proves it (band_proves_width), or when the band could not hold both ends (the sweep was
// then whole). Otherwise the band's score, a real alignment's, says how wide a band would prove a score
// that good: g gap letters outside it must cost more than the score, g > (4 (open - extend) + best (rows +
// columns) - 2 score) / (best - 2 extend). The pair goes round again at that width (at least twice the
// last, rounded up to 1,024 diagonals) unless this is the `last` round or that band's strips of
// `strip_columns` would sweep three fifths of its rows or more: then to the whole-matrix list. With `swept`
// null, every pair is routed to `first_width`. With `proven`, a pair whose band proves its score leaves the
// width there (by pair - proven_first).
__global__ void wide_route_kernel(const PairShape *__restrict__ shapes, const uint32_t *__restrict__ pending,
                                  const int32_t *__restrict__ swept, int64_t count, int32_t first_width, bool last,
                                  const int32_t *__restrict__ scores, int32_t best, int32_t open, int32_t extend,
                                  uint32_t *__restrict__ next, int32_t *__restrict__ next_width,
                                  unsigned int *__restrict__ next_count, uint32_t *__restrict__ whole,
                                  unsigned int *__restrict__ whole_count, int32_t *__restrict__ proven,
                                  int64_t proven_first, int32_t strip_columns) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t pair = pending[k];
    const PairShape sh = shapes[pair];
    const int64_t rows = sh.rows, columns = sh.columns;
    int64_t width = first_width;
    if (swept) {
        const int64_t done = swept[k];
        const int32_t low = band_low_for_width(rows, columns, done);
        if (low == INT32_MIN) return;
        const int64_t score = scores[pair];
        if (band_proves_width(score, rows, columns, low, done, best, open, extend)) {
            if (proven) proven[pair - proven_first] = int32_t(done);
            return;
        }
        const int64_t per_letter = int64_t(best) - 2 * int64_t(extend);
        if (per_letter <= 0) {  // no band proves anything narrower than the matrix
            whole[atomicAdd(whole_count, 1u)] = pair;
            return;
        }
        const int64_t g = (4 * (int64_t(open) - extend) + int64_t(best) * (rows + columns) - 2 * score) / per_letter + 2;
        const int64_t delta = columns > rows ? columns - rows : rows - columns;
        width = max(2 * done, g + delta + 2);
        width = (width + 1023) / 1024 * 1024;
    }
    const bool banded = !last && width < (int64_t(1) << 30) && band_low_for_width(rows, columns, width) != INT32_MIN &&
                        10 * (strip_columns + width) < 6 * rows;
    if (banded) {
        const unsigned at = atomicAdd(next_count, 1u);
        next[at] = pair;
        next_width[at] = int32_t(width);
    } else {
        whole[atomicAdd(whole_count, 1u)] = pair;
    }
}

// Scores of long global pairs (the block-a-pair class) by a widening band: a first round sweeps each pair
// over 2,048 diagonals; a pair its band does not prove goes round once more at the width its band score
// says would prove it, or is swept whole when that band would cover most of its matrix (or its second
// band proves nothing either). Every score is the whole matrix's. With `proven`, each pair whose band
// proved its score leaves that band's width there (by pair - proven_first; the rest are left as they were),
// and the pairs left to the whole matrix are not swept here: their recording gives their scores; a band
// is then worth its rounds when the recording's strips (kRecordStrip columns) would sweep few of a pair's
// rows, where the scores' own strips are a block's 4,096 columns.
void widening_band(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, const uint32_t *order,
                   int64_t count, KernelArgs args, int32_t *proven = nullptr, int64_t proven_first = 0) {
    if (count <= 0) return;
    const TableArgs targs = table_args(table, false);
    int32_t best = -128;
    for (int r = 0; r < table.size; ++r)
        for (int c = 0; c < table.size; ++c) best = std::max(best, table.entries[r * 32 + c]);
    uint32_t *lists = gpu->wide_pending.ensure<uint32_t>(5 * size_t(count));
    uint32_t *whole = lists + 2 * count;
    int32_t *widths = reinterpret_cast<int32_t *>(lists + 3 * count);
    unsigned int *counts = gpu->class_counts.ensure<unsigned int>(20) + 9;  // [0] next, [1] whole
    DINARA_CUDA(cudaMemsetAsync(counts + 1, 0, sizeof(unsigned int), gpu->stream));
    constexpr int32_t kFirstWidth = 2048;
    constexpr int kBandRounds = 2;
    const uint32_t *pending = order;
    const int32_t *swept = nullptr;
    int64_t left = count;
    for (int round = 0; round <= kBandRounds && left > 0; ++round) {
        uint32_t *next = lists + (round & 1) * count;
        int32_t *next_widths = widths + (round & 1) * count;
        DINARA_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned int), gpu->stream));
        wide_route_kernel<<<unsigned((left + 255) / 256), 256, 0, gpu->stream>>>(
            batch.shapes, pending, swept, left, kFirstWidth, round == kBandRounds, args.scores, best, table.open,
            table.extend, next, next_widths, counts, whole, counts + 1, proven, proven_first,
            proven ? kRecordStrip : 16 * kBlock);
        DINARA_CUDA(cudaGetLastError());
        gpu->launches += 1;
        unsigned int routed = 0;
        read_back(gpu, &routed, counts, sizeof routed);
        left = routed;
        if (left == 0) break;
        int64_t blocks = persistent_blocks(gpu, &affine_wide_kernel<false, true>);
        blocks = std::max<int64_t>(1, std::min(blocks, left));
        args.carry_stride = int64_t(batch.max_rows) + 1;
        args.carry = gpu->carry.ensure<int2>(size_t(blocks * args.carry_stride));
        args.order = next;
        args.band_widths = next_widths;
        args.begin = 0;
        args.end = uint32_t(left);
        ClockSpan clock(gpu, kClassWhole, gpu->stream);
        affine_wide_kernel<false, true><<<unsigned(blocks), kBlock, 0, gpu->stream>>>(args, targs, nullptr);
        DINARA_CUDA(cudaGetLastError());
        clock.stop();
        gpu->launches += 1;
        pending = next;
        swept = next_widths;
    }
    unsigned int swept_whole = 0;
    if (!proven) read_back(gpu, &swept_whole, counts + 1, sizeof swept_whole);
    if (swept_whole > 0) {
        int64_t blocks = persistent_blocks(gpu, &affine_wide_kernel<false, false>);
        blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, swept_whole));
        args.carry_stride = int64_t(batch.max_rows) + 1;
        args.carry = gpu->carry.ensure<int2>(size_t(blocks * args.carry_stride));
        args.order = whole;
        args.band_widths = nullptr;
        args.begin = 0;
        args.end = swept_whole;
        ClockSpan clock(gpu, kClassWhole, gpu->stream);
        affine_wide_kernel<false, false><<<unsigned(blocks), kBlock, 0, gpu->stream>>>(args, targs, nullptr);
        DINARA_CUDA(cudaGetLastError());
        clock.stop();
        gpu->launches += 1;
    }
}

void affine_launch_all(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, const Schedule &schedule,
                       bool record, KernelArgs args) {
    const bool smem = !table.packed16 || batch.bits == 8;
    const TableArgs targs = table_args(table, batch.local);
    int32_t *table32 = nullptr;
    if (smem) upload_table32(gpu, table, batch.local, &table32);
    const Buckets b = buckets_of(schedule);
    args.order = schedule.order;
    for (int bucket = kClasses - 1; bucket >= 0; --bucket) {
        if (bucket == kBandClass || bucket == kBandPairsClass) continue;
        if (b.end[bucket] <= b.begin[bucket]) continue;
        const bool wide = bucket == kWideClass;
        // Recording, a long global pair whose widening band proved a width: its strips over that band.
        const bool band_record = bucket == kBandRecordClass;
        const bool pairs16 = !wide && !band_record && bucket >= kWholePairsClass;
        const int cls = pairs16 ? bucket - kWholePairsClass : wide || band_record ? 4 : bucket;
        if (wide && !batch.local && !record && band_serves(batch, table)) {
            // Long global pairs take the widening band first.
            widening_band(gpu, batch, table, schedule.order + b.begin[bucket], b.end[bucket] - b.begin[bucket], args);
            continue;
        }
        KernelFn fn = band_record ? &affine_kernel<32, 16, false, true, 2, false, false, true>
                      : wide      ? (batch.local ? &affine_wide_kernel<true, false> : &affine_wide_kernel<false, false>)
                      : pairs16   ? pick_pairs_kernel(cls, batch.local)
                                  : pick_kernel(cls, batch.local, record, batch.bits, smem);
        const int G = wide ? kBlock : (smem && !pairs16) || band_record ? 32 : affine_lanes(cls);
        const int groups_per_block = (pairs16 ? 2 : 1) * kBlock / G;
        int64_t blocks = persistent_blocks(gpu, fn);
        const int64_t needed = (b.end[bucket] - b.begin[bucket] + groups_per_block - 1) / groups_per_block;
        if (blocks > needed) blocks = needed;
        if (blocks < 1) blocks = 1;
        // Carry slots, one a group, each as long as the tallest pair: only a launch whose pairs may be
        // wider than one strip reads them.
        const int width = wide ? 16 * kBlock : (smem && !pairs16) || band_record ? 512 : affine_lanes(cls) * affine_columns(cls);
        args.carry = nullptr;
        args.carry_stride = 0;
        if (batch.max_columns > uint32_t(width)) {
            const int64_t slots = blocks * (kBlock / G);
            args.carry_stride = int64_t(batch.max_rows) + 1;
            args.carry = gpu->carry.ensure<int2>(size_t(slots * args.carry_stride));
        }
        args.begin = uint32_t(b.begin[bucket]);
        args.end = uint32_t(b.end[bucket]);
        ClockSpan clock(gpu, kClassWhole, gpu->stream);
        fn<<<dim3(unsigned(blocks)), kBlock, 0, gpu->stream>>>(args, targs, table32);
        DINARA_CUDA(cudaGetLastError());
        clock.stop();
        gpu->launches += 1;
    }
}

// The largest rows + columns of a pair the 16-bit pair sweep takes under a table (band_pair_limit): the
// largest step a shifted cell takes is a shifted entry or a gap's opening.
int32_t pair_limit_of(const AffineTable &table) {
    int32_t step = std::abs(table.open - table.extend);
    bool bytes_fit = true;
    for (int r = 0; r < table.size; ++r)
        for (int c = 0; c < table.size; ++c) {
            const int32_t v = table.entries[r * 32 + c] - 2 * table.extend;
            step = std::max(step, std::abs(v));
            bytes_fit = bytes_fit && v >= -128 && v <= 127;
        }
    return band_pair_limit(step, bytes_fit);
}

// Which whole-matrix pairs the 16-bit pair score sweep takes (a table of up to four letters on the 2-bit
// tape): locally, a cell held less row x extend reaches at most the best entry times the columns swept
// plus the rows times -extend and falls no lower than a gap's first letter, so that sum is held to half of
// 30,000 less the gaps;
// globally, a shifted cell moves at most the largest step a cell, so rows and swept columns are each held
// to half of 30,000 over it, every value within 30,000 of zero. Entries must fit a byte (shifted, globally).
PairLimits whole_limits_of(const AffineBatch &batch, const AffineTable &table) {
    PairLimits limits;
    if (batch.bits != 2 || !table.packed16) return limits;
    limits.wide = 1;
    const int32_t gaps = std::abs(table.open) + std::abs(table.extend);
    if (gaps > 8000) return limits;
    if (batch.local) {
        int32_t best = 1;
        for (int r = 0; r < table.size; ++r)
            for (int c = 0; c < table.size; ++c) {
                best = std::max(best, table.entries[r * 32 + c]);
                const int32_t shifted = table.entries[r * 32 + c] - table.extend;
                if (shifted < -128 || shifted > 127) return limits;
            }
        limits.local = 1;
        // Half of it a pair: a lane group sweeps its two pairs to the larger one's rows and strips, so the
        // cells past a pair's end reach at most the sum of the two pairs' terms.
        limits.whole = (30000 - gaps) / 2;
        limits.best = best;
        limits.row_step = -table.extend;
        return limits;
    }
    int32_t step = std::abs(table.open - table.extend);
    for (int r = 0; r < table.size; ++r)
        for (int c = 0; c < table.size; ++c) {
            const int32_t v = table.entries[r * 32 + c] - 2 * table.extend;
            if (v < -128 || v > 127) return limits;
            step = std::max(step, std::abs(v));
        }
    limits.whole = 30000 / std::max(step, 1) - 4;
    return limits;
}

// The band's shifted table and best entry for a banded launch: the band's pairs of the 16-bit pair sweep
// (`pairs_of_16`) or the rest, each class's range of the order.
BandedBatch banded_batch(const AffineBatch &batch, const AffineTable &table, const Schedule &schedule, int32_t *scores,
                         uint8_t *proven, uint32_t *leftovers, unsigned int *leftover_count, bool pairs_of_16) {
    BandedBatch band;
    std::memset(&band, 0, sizeof band);
    const TableArgs targs = table_args(table, false);
    for (int r = 0; r < 4; ++r) band.rows16[r] = targs.rows16[r];
    for (int r = 0; r < 4; ++r) {
        uint32_t row = 0;
        for (int c = 0; c < 4; ++c) {
            const int32_t v = r < table.size && c < table.size ? table.entries[r * 32 + c] - 2 * table.extend : 0;
            row |= uint32_t(uint8_t(int8_t(v))) << (8 * c);
        }
        band.rows8[r] = row;
    }
    int32_t best = -128;
    for (int r = 0; r < table.size; ++r)
        for (int c = 0; c < table.size; ++c) best = std::max(best, table.entries[r * 32 + c]);
    band.tape = batch.tape;
    band.shapes = batch.shapes;
    const Buckets buckets = buckets_of(schedule);
    const int cls = pairs_of_16 ? kBandPairsClass : kBandClass;
    band.order = schedule.order + buckets.begin[cls];
    band.count = schedule.counts[cls];
    band.open = table.open;
    band.extend = table.extend;
    band.best = best;
    band.scores = scores;
    band.proven = proven;
    band.leftovers = leftovers;
    band.leftover_count = leftover_count;
    return band;
}

// The band cells a call's band launches count while the context times (null otherwise): zeroed here, read
// by tally_swept.
unsigned long long *band_counter(dinara_gpu *gpu) {
    if (!gpu->timing) return nullptr;
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(gpu->class_counts.ensure<unsigned int>(20) + 16);
    DINARA_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), gpu->stream));
    return counter;
}

// Adds the cells a batch's sweeps updated to the context's tally (only while it times): the whole matrices
// from their shapes, the bands' cells as their launches counted them (a narrow pass and a wide one where
// both ran), band-recorded pairs' strips from their widths (when given).
void tally_swept(dinara_gpu *gpu, const PairShape *shapes, int64_t first, int64_t count, bool band,
                 const uint32_t *leftovers, int64_t left, const int32_t *widths = nullptr) {
    if (!gpu->timing) return;
    unsigned long long *out = reinterpret_cast<unsigned long long *>(gpu->class_counts.ensure<unsigned int>(20) + 12);
    DINARA_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), gpu->stream));
    swept_cells_kernel<<<256, 256, 0, gpu->stream>>>(shapes, first, count, band, leftovers, left, widths, out);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    unsigned long long host[2] = {0, 0};
    read_back(gpu, host, out, sizeof host);
    if (band) read_back(gpu, &host[0], gpu->class_counts.ensure<unsigned int>(20) + 16, sizeof host[0]);
    gpu->swept_cells += int64_t(host[0] + host[1]);
    gpu->band_cells += int64_t(host[0]);
    gpu->whole_cells += int64_t(host[1]);
}

}  // namespace

namespace {

// The proven band's pairs of a schedule: the 16-bit pair sweep's and the rest.
int64_t band_pairs(const Schedule &schedule) {
    return schedule.counts[kBandPairsClass] + schedule.counts[kBandClass];
}

// Sweeps the band's pairs, the 16-bit pair sweep's first, every unproven pair onto one leftover list.
void launch_bands(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, const Schedule &schedule,
                  int32_t *scores, uint32_t *leftovers, unsigned int *leftover_count, bool record, uint64_t *decisions,
                  const int64_t *decision_offsets, int64_t first_pair, uint8_t *layouts,
                  unsigned long long *band_cells) {
    for (int pass = 0; pass < 2; ++pass) {
        const bool pairs_of_16 = pass == 0;
        BandedBatch b = banded_batch(batch, table, schedule, scores, nullptr, leftovers, leftover_count, pairs_of_16);
        if (b.count == 0) continue;
        b.decisions = decisions;
        b.decision_offsets = decision_offsets;
        b.first_pair = first_pair;
        b.band_cells = band_cells;
        if (!pairs_of_16) {
            banded_launch(gpu, b, record, false);
            continue;
        }
        // The 16-bit pair band in two passes: every pair over 32 diagonals first (most short pairs' scores
        // prove there, for half the cells), then the pairs it did not prove, or could not hold, over 64.
        uint32_t *narrow_left = gpu->narrow_leftovers.ensure<uint32_t>(size_t(b.count));
        unsigned int *narrow_count = gpu->class_counts.ensure<unsigned int>(20) + 11;
        DINARA_CUDA(cudaMemsetAsync(narrow_count, 0, sizeof(unsigned int), gpu->stream));
        BandedBatch narrow = b;
        narrow.leftovers = narrow_left;
        narrow.leftover_count = narrow_count;
        narrow.layouts = record ? layouts : nullptr;
        banded_launch(gpu, narrow, record, true, 2);
        unsigned int again = 0;
        read_back(gpu, &again, narrow_count, sizeof again);
        if (again > 0) {
            BandedBatch wide = b;
            wide.order = narrow_left;
            wide.count = again;
            banded_launch(gpu, wide, record, true, kBandLanes);
        }
    }
}

}  // namespace

namespace {

// Each pair's span with free ends from its best end and the start found back from it: the reference's
// letters from end row less the back sweep's row to the end row, then the query's likewise.
__global__ void free_spans_kernel(const int64_t *__restrict__ ends, const int64_t *__restrict__ found, int64_t count,
                                  int64_t *__restrict__ spans) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t end_row = ends[k] >> 32, end_column = ends[k] & 0xffffffff;
    const int64_t back_row = found[k] >> 32, back_column = found[k] & 0xffffffff;
    int64_t *span = spans + 4 * k;
    span[0] = end_row - back_row;
    span[1] = end_row;
    span[2] = end_column - back_column;
    span[3] = end_column;
}

// Each pair's whole extent (rows << 32 | columns), for an extension swept from the ends.
__global__ void extents_kernel(const PairShape *__restrict__ shapes, int64_t first, int64_t count,
                               int64_t *__restrict__ extents) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[first + k];
    extents[k] = (int64_t(sh.rows) << 32) | int64_t(sh.columns);
}

// Each pair's anti-diagonals kept for an extension's Z-drop: rows + columns + 1 (none for an empty side).
__global__ void diagonal_counts_kernel(const PairShape *__restrict__ shapes, int64_t first, int64_t count,
                                       int64_t *__restrict__ counts) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[first + k];
    counts[k] = sh.rows > 0 && sh.columns > 0 ? int64_t(sh.rows) + sh.columns + 1 : 0;
}

// An extension's result from its sweep, one thread a pair. With a Z-drop (`diagonals`), the stop is read
// from the anti-diagonals' bests in order as scored.mojo:272-300 reads them: a best above zero at or
// above the best so far is the new stop (later anti-diagonals win ties); one below it ends the sweep when
// it lies more than `zdrop` plus `slack` a diagonal between them (each's reference less query letters)
// below it. Otherwise the sweep's best cell is the stop. The span runs from the origin to the stop, or
// (swept from the ends) from the stop counted back to the ends. With an end bonus and no early end, the
// alignment reaching the query's far end wins when its score plus the bonus passes the stop's
// (scoring.mojo:704-710), compared without the sum: the bonus may be near 2^63.
__global__ void extension_finish_kernel(const PairShape *__restrict__ shapes, int64_t first, int64_t count,
                                        bool from_end, const int64_t *__restrict__ stops,
                                        const unsigned long long *__restrict__ diagonals,
                                        const int64_t *__restrict__ diagonal_offsets, int64_t zdrop, int64_t slack,
                                        int64_t end_bonus, const int32_t *__restrict__ reach_scores,
                                        const int64_t *__restrict__ reach_spans, int32_t *__restrict__ scores,
                                        int64_t *__restrict__ spans) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t pair = first + k;
    const PairShape sh = shapes[pair];
    const int64_t rows = sh.rows, columns = sh.columns;
    int64_t best = scores[pair], row = stops[k] >> 32, column = stops[k] & 0xffffffff;
    bool dropped = false;
    if (diagonals && rows > 0 && columns > 0) {
        const unsigned long long *kept = diagonals + diagonal_offsets[k];
        int64_t best_row = 0, best_diagonal = 0;
        best = 0;
        for (int64_t d = 2; d <= rows + columns; ++d) {
            const unsigned long long key = kept[d];
            const int64_t most = int64_t(int32_t(uint32_t(key >> 32) ^ 0x80000000u));
            const int64_t furthest = int64_t(key & 0xffffffffu);
            if (most > 0 && most >= best) {
                best = most;
                best_row = furthest;
                best_diagonal = d;
            } else if (most < best) {
                const int64_t lean = 2 * furthest - d, best_lean = 2 * best_row - best_diagonal;
                const int64_t apart = lean > best_lean ? lean - best_lean : best_lean - lean;
                if (best - most > zdrop + slack * apart) {
                    dropped = true;
                    break;
                }
            }
        }
        row = best_row;
        column = best_diagonal - best_row;
    }
    int64_t span[4] = {from_end ? rows - row : 0, from_end ? rows : row, from_end ? columns - column : 0,
                       from_end ? columns : column};
    if (end_bonus > 0 && !dropped && end_bonus > best - int64_t(reach_scores[pair])) {
        best = reach_scores[pair];
        for (int j = 0; j < 4; ++j) span[j] = reach_spans[4 * k + j];
    }
    scores[pair] = int32_t(best);
    if (spans)
        for (int j = 0; j < 4; ++j) spans[4 * k + j] = span[j];
}

// Global scores with free ends: every pair over its whole matrix in 32 bits, one shape (32 lanes of 16
// columns, strips of 512) with the table in shared memory, the free-end form of the sweep. With `spans`
// (4 a pair of the range, by pair - first), each pair's span as the reference places it
// (scoring.mojo:690-722 mode_span, scored.mojo:616-633 started_span): its end, of equal best ends the one
// furthest along the reference less the query; then a sweep back over both prefixes to that end, read
// backwards, with the letters free at the start free at its end, whose best end nearest the other way
// (the least along the reference less the query, reversed) is the start. An extension (batch.extension)
// takes one launch of the same form with no letters free and every cell a candidate stop (ORIGIN), from
// the origin or, read backwards, from the ends; its span runs from its anchor to the stop.
void free_end_scores(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, int32_t *scores,
                     int64_t first, int64_t count, int64_t *spans) {
    // A Z-drop keeps rows + columns + 1 words a pair: a range whose words pass the budget goes in halves.
    constexpr int64_t kDiagonalBudget = int64_t(1) << 28;  // 2 GiB of 8-byte words
    int64_t *diagonal_counts = nullptr, *diagonal_offsets = nullptr;
    if (batch.extension && batch.zdrop >= 0) {
        diagonal_counts = gpu->diagonal_offsets.ensure<int64_t>(2 * (size_t(count) + 1));
        diagonal_offsets = diagonal_counts + (count + 1);
        diagonal_counts_kernel<<<unsigned((count + 255) / 256), 256, 0, gpu->stream>>>(batch.shapes, first, count,
                                                                                     diagonal_counts);
        DINARA_CUDA(cudaGetLastError());
        gpu->launches += 1;
        DINARA_CUDA(cudaMemsetAsync(diagonal_counts + count, 0, sizeof(int64_t), gpu->stream));
        size_t scratch = 0;
        DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, diagonal_counts, diagonal_offsets, int(count + 1),
                                                  gpu->stream));
        void *space = gpu->sort_scratch.ensure<uint8_t>(scratch + 256);
        DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, diagonal_counts, diagonal_offsets, int(count + 1),
                                                  gpu->stream));
        int64_t kept = 0;
        read_back(gpu, &kept, diagonal_offsets + count, sizeof kept);
        if (kept > kDiagonalBudget && count > 1) {
            const int64_t half = count / 2;
            free_end_scores(gpu, batch, table, scores, first, half, spans);
            free_end_scores(gpu, batch, table, scores, first + half, count - half, spans ? spans + 4 * half : nullptr);
            return;
        }
    }
    // An extension's end bonus weighs the alignment reaching the query's far end (from the same anchor, the
    // whole query against the reference, whose far end is free): its score and span first.
    int32_t *reach_scores = nullptr;
    int64_t *reach_spans = nullptr;
    if (batch.extension && batch.end_bonus > 0) {
        AffineBatch reaching = batch;
        reaching.extension = false;
        reaching.free_reference_start = batch.from_end ? INT32_MAX : 0;
        reaching.free_reference_end = batch.from_end ? 0 : INT32_MAX;
        reaching.free_query_start = reaching.free_query_end = 0;
        reach_scores = gpu->reach_scores.ensure<int32_t>(size_t(batch.pairs));
        reach_spans = gpu->reach_spans.ensure<int64_t>(4 * size_t(count));
        free_end_scores(gpu, reaching, table, reach_scores, first, count, reach_spans);
    }
    const Schedule order = dinara::schedule(gpu, batch.shapes, nullptr, first, count, false, false, PairLimits());
    int32_t *table32 = nullptr;
    upload_table32(gpu, table, false, &table32);
    const TableArgs targs = table_args(table, false);
    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.order = order.order;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    args.first_pair = first;
    args.free_reference_start = batch.free_reference_start;
    args.free_reference_end = batch.free_reference_end;
    args.free_query_start = batch.free_query_start;
    args.free_query_end = batch.free_query_end;
    int64_t *ends = nullptr;
    if (spans || batch.extension) {
        ends = gpu->free_spans.ensure<int64_t>(2 * size_t(count));
        args.free_ends_out = ends;
        args.free_highest = 1;
    }
    KernelFn fn = batch.bits == 8 ? static_cast<KernelFn>(&affine_kernel<32, 16, false, false, 8, true, true>)
                                  : static_cast<KernelFn>(&affine_kernel<32, 16, false, false, 2, true, true>);
    if (batch.extension) {
        // An extension's stop: the free-end form with no letters free, every cell a candidate; from the
        // ends, each pair whole and read backwards.
        fn = batch.bits == 8 ? static_cast<KernelFn>(&affine_kernel<32, 16, false, false, 8, true, true, false, true>)
                             : static_cast<KernelFn>(&affine_kernel<32, 16, false, false, 2, true, true, false, true>);
        args.free_reference_start = args.free_reference_end = args.free_query_start = args.free_query_end = 0;
        if (batch.from_end) {
            int64_t *extents = ends + count;
            extents_kernel<<<unsigned((count + 255) / 256), 256, 0, gpu->stream>>>(batch.shapes, first, count,
                                                                                 extents);
            DINARA_CUDA(cudaGetLastError());
            gpu->launches += 1;
            args.extents = extents;
        }
        if (batch.zdrop >= 0) {
            // Room for every pair's anti-diagonals (their offsets scanned above), zeroed: below every key.
            const int64_t kept = [&] {
                int64_t total = 0;
                read_back(gpu, &total, diagonal_offsets + count, sizeof total);
                return total;
            }();
            unsigned long long *diagonals = gpu->diagonals.ensure<unsigned long long>(size_t(kept) + 1);
            DINARA_CUDA(cudaMemsetAsync(diagonals, 0, (size_t(kept) + 1) * sizeof(unsigned long long), gpu->stream));
            args.diagonals = diagonals;
            args.diagonal_offsets = diagonal_offsets;
        }
    }
    int64_t total = 0;
    for (int cls = 0; cls < kClasses; ++cls) total += order.counts[cls];
    int64_t blocks = persistent_blocks(gpu, fn);
    blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, (total + kBlock / 32 - 1) / (kBlock / 32)));
    if (batch.max_columns > 512u) {
        args.carry_stride = int64_t(batch.max_rows) + 1;
        args.carry = gpu->carry.ensure<int2>(size_t(blocks * (kBlock / 32) * args.carry_stride));
    }
    args.begin = 0;
    args.end = uint32_t(total);
    PhaseTimer timer(gpu, &gpu->kernel_ms);
    ClockSpan clock(gpu, kClassWhole, gpu->stream);
    fn<<<dim3(unsigned(blocks)), kBlock, 0, gpu->stream>>>(args, targs, table32);
    DINARA_CUDA(cudaGetLastError());
    clock.stop();
    gpu->launches += 1;
    if (batch.extension) {
        extension_finish_kernel<<<unsigned((count + 255) / 256), 256, 0, gpu->stream>>>(
            batch.shapes, first, count, batch.from_end, ends, args.diagonals, args.diagonal_offsets, batch.zdrop,
            -int64_t(table.extend), batch.end_bonus, reach_scores, reach_spans, scores, spans);
        DINARA_CUDA(cudaGetLastError());
        gpu->launches += 1;
    } else if (spans) {
        // The sweep back: each pair's prefixes to its end, backwards, the start's free letters free at the
        // (backward) end and none at its start; its scores, the same, go to scratch.
        KernelArgs back = args;
        back.scores = gpu->free_scores.ensure<int32_t>(size_t(batch.pairs));
        back.extents = ends;
        back.free_ends_out = ends + count;
        back.free_highest = 0;
        back.free_reference_start = 0;
        back.free_reference_end = batch.free_reference_start;
        back.free_query_start = 0;
        back.free_query_end = batch.free_query_start;
        ClockSpan back_clock(gpu, kClassWhole, gpu->stream);
        fn<<<dim3(unsigned(blocks)), kBlock, 0, gpu->stream>>>(back, targs, table32);
        DINARA_CUDA(cudaGetLastError());
        back_clock.stop();
        free_spans_kernel<<<unsigned((count + 255) / 256), 256, 0, gpu->stream>>>(ends, ends + count, count, spans);
        DINARA_CUDA(cudaGetLastError());
        gpu->launches += 2;
    }
    timer.stop();
}

// Long global pairs of an alignment batch: their scores by the widening band, and each pair's proven width
// (by pair - first_pair; 0 for a pair its band left to the whole matrix), so that its recording sweeps its
// band's rows alone. Null when the range holds no long pair.
int32_t *proven_band_widths(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, int32_t *scores,
                            int64_t first_pair, int64_t count) {
    uint32_t *list = gpu->long_pairs.ensure<uint32_t>(size_t(count));
    unsigned int *listed = gpu->class_counts.ensure<unsigned int>(20) + 18;
    DINARA_CUDA(cudaMemsetAsync(listed, 0, sizeof(unsigned int), gpu->stream));
    long_pairs_kernel<<<unsigned((count + 255) / 256), 256, 0, gpu->stream>>>(batch.shapes, first_pair, count, list,
                                                                             listed);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    unsigned int found = 0;
    read_back(gpu, &found, listed, sizeof found);
    if (found == 0) return nullptr;
    int32_t *widths = gpu->record_widths.ensure<int32_t>(size_t(count));
    DINARA_CUDA(cudaMemsetAsync(widths, 0, sizeof(int32_t) * size_t(count), gpu->stream));
    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    PhaseTimer timer(gpu, &gpu->record_ms);
    widening_band(gpu, batch, table, list, found, args, widths, first_pair);
    timer.stop();
    return widths;
}

}  // namespace

bool band_serves(const AffineBatch &batch, const AffineTable &table) {
    if (batch.local || batch.bits != 2 || !table.packed16) return false;
    int32_t best = -128;
    for (int r = 0; r < table.size; ++r)
        for (int c = 0; c < table.size; ++c) best = std::max(best, table.entries[r * 32 + c]);
    return 2 * int64_t(table.extend) - best <= 0;
}

void affine_scores(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, int32_t *scores,
                   int64_t first, int64_t count, int64_t *spans) {
    if (count <= 0) return;
    if (batch.free_ends) {
        free_end_scores(gpu, batch, table, scores, first, count, spans);
        return;
    }
    const bool band = band_serves(batch, table);
    PairLimits limits = whole_limits_of(batch, table);
    limits.band = band ? pair_limit_of(table) : 0;
    const Schedule schedule_all = dinara::schedule(gpu, batch.shapes, nullptr, first, count, false, band, limits);
    PhaseTimer timer(gpu, &gpu->kernel_ms);
    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    unsigned int *counters = gpu->class_counts.ensure<unsigned int>(20);
    unsigned int *leftover_count = counters + 8;
    uint32_t *leftovers = nullptr;
    if (band_pairs(schedule_all) > 0) {
        leftovers = gpu->leftovers.ensure<uint32_t>(size_t(band_pairs(schedule_all)));
        DINARA_CUDA(cudaMemsetAsync(leftover_count, 0, sizeof(unsigned int), gpu->stream));
        launch_bands(gpu, batch, table, schedule_all, scores, leftovers, leftover_count, false, nullptr, nullptr, 0,
                     nullptr, band_counter(gpu));
    }
    affine_launch_all(gpu, batch, table, schedule_all, false, args);
    unsigned int left = 0;
    if (band_pairs(schedule_all) > 0) {
        read_back(gpu, &left, leftover_count, sizeof left);
        if (left > 0) {
            const Schedule again = dinara::schedule(gpu, batch.shapes, leftovers, 0, left, false, false,
                                                    whole_limits_of(batch, table));
            affine_launch_all(gpu, batch, table, again, false, args);
        }
    }
    timer.stop();
    tally_swept(gpu, batch.shapes, first, count, band, leftovers, left);
}

int64_t affine_alignments(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, bool eqx,
                          int32_t *scores, int64_t *spans, int64_t first_pair, int64_t count) {
    const bool band = band_serves(batch, table);
    const bool uniform = !table.packed16 || batch.bits == 8;
    // Per pair: its decisions' words, its layout and its CIGAR slot, then the offsets by exclusive scans.
    int64_t *words = gpu->decision_offsets.ensure<int64_t>(2 * (count + 1) + 2);
    int64_t *word_offsets = words + (count + 1);
    int64_t *slot_bytes = gpu->cigar_slots.ensure<int64_t>(2 * (count + 1) + 2);
    int64_t *slot_offsets = slot_bytes + (count + 1);
    uint8_t *layouts = gpu->layouts.ensure<uint8_t>(size_t(count) + 1);
    const int threads = 256;
    const unsigned blocks = unsigned((count + threads - 1) / threads);
    const int32_t band_pair_limit = band ? pair_limit_of(table) : 0;
    // Long global pairs take the widening band's scores first, then record over their proven bands.
    const int32_t *widths = band && !batch.local && batch.max_rows >= kWideRows && batch.max_columns >= kWideColumns
                                ? proven_band_widths(gpu, batch, table, scores, first_pair, count)
                                : nullptr;
    slot_sizes_kernel<<<blocks, threads, 0, gpu->stream>>>(batch.shapes, first_pair, count, uniform, band_pair_limit,
                                                           band, widths, words, slot_bytes, layouts);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, words, word_offsets, int(count + 1), gpu->stream));
    size_t scratch2 = 0;
    DINARA_CUDA(
        cub::DeviceScan::ExclusiveSum(nullptr, scratch2, slot_bytes, slot_offsets, int(count + 1), gpu->stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(std::max(scratch, scratch2) + 256);
    // The counts' last entries are zero, so each scan's last output is its total.
    DINARA_CUDA(cudaMemsetAsync(words + count, 0, sizeof(int64_t), gpu->stream));
    DINARA_CUDA(cudaMemsetAsync(slot_bytes + count, 0, sizeof(int64_t), gpu->stream));
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, words, word_offsets, int(count + 1), gpu->stream));
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch2, slot_bytes, slot_offsets, int(count + 1), gpu->stream));
    int64_t totals[2];
    read_back(gpu, &totals[0], word_offsets + count, sizeof(int64_t));
    read_back(gpu, &totals[1], slot_offsets + count, sizeof(int64_t));
    uint64_t *decisions = gpu->decisions.ensure<uint64_t>(size_t(totals[0]) + 8);
    char *slots = gpu->walk_out.ensure<char>(size_t(totals[1]) + 8);
    int64_t *ends = gpu->spans.ensure<int64_t>(size_t(count) + 1);
    int64_t *lengths = gpu->cigar_lengths.ensure<int64_t>(2 * (size_t(count) + 1));
    int64_t *run_counts = lengths + (count + 1);
    PairLimits limits;
    limits.band = band ? pair_limit_of(table) : 0;
    limits.band_widths = widths;
    limits.band_first = first_pair;
    const Schedule schedule_all = dinara::schedule(gpu, batch.shapes, nullptr, first_pair, count, true, band, limits);
    // The walk takes the pairs in this order; a later schedule (the band's leftovers) reuses its buffer.
    uint32_t *walk_order = gpu->walk_order.ensure<uint32_t>(size_t(count));
    DINARA_CUDA(cudaMemcpyAsync(walk_order, schedule_all.order, size_t(count) * sizeof(uint32_t),
                                cudaMemcpyDeviceToDevice, gpu->stream));

    PhaseTimer timer(gpu, &gpu->record_ms);
    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    args.decisions = decisions;
    args.decision_offsets = word_offsets;
    args.ends = ends;
    args.first_pair = first_pair;
    args.band_widths = widths;
    unsigned int *counters = gpu->class_counts.ensure<unsigned int>(20);
    unsigned int *leftover_count = counters + 8;
    uint32_t *leftovers = nullptr;
    uint64_t *extra = nullptr;
    if (band_pairs(schedule_all) > 0) {
        leftovers = gpu->leftovers.ensure<uint32_t>(size_t(band_pairs(schedule_all)));
        DINARA_CUDA(cudaMemsetAsync(leftover_count, 0, sizeof(unsigned int), gpu->stream));
        launch_bands(gpu, batch, table, schedule_all, scores, leftovers, leftover_count, true, decisions, word_offsets,
                     first_pair, layouts, band_counter(gpu));
    }
    affine_launch_all(gpu, batch, table, schedule_all, true, args);
    unsigned int left = 0;
    if (band_pairs(schedule_all) > 0) {
        read_back(gpu, &left, leftover_count, sizeof left);
        if (left > 0) {
            // The band's leftovers, swept whole: their decisions in the extra buffer.
            int64_t *left_words = gpu->thresholds.ensure<int64_t>(2 * (size_t(left) + 1) + 2);
            int64_t *left_offsets = left_words + (left + 1);
            const unsigned left_blocks = unsigned((left + threads - 1) / threads);
            leftover_words_kernel<<<left_blocks, threads, 0, gpu->stream>>>(batch.shapes, leftovers, left, uniform,
                                                                            left_words);
            gpu->launches += 1;
            DINARA_CUDA(cudaGetLastError());
            DINARA_CUDA(cudaMemsetAsync(left_words + left, 0, sizeof(int64_t), gpu->stream));
            size_t bytes = 0;
            DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, left_words, left_offsets, int(left + 1), gpu->stream));
            space = gpu->sort_scratch.ensure<uint8_t>(bytes + 256);
            DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, bytes, left_words, left_offsets, int(left + 1), gpu->stream));
            int64_t extra_total = 0;
            read_back(gpu, &extra_total, left_offsets + left, sizeof(int64_t));
            extra = gpu->decisions_extra.ensure<uint64_t>(size_t(extra_total) + 8);
            leftover_places_kernel<<<left_blocks, threads, 0, gpu->stream>>>(leftovers, left, first_pair, left_offsets,
                                                                             word_offsets, layouts);
            gpu->launches += 1;
            DINARA_CUDA(cudaGetLastError());
            const Schedule again = dinara::schedule(gpu, batch.shapes, leftovers, 0, left, true, false);
            KernelArgs extra_args = args;
            extra_args.decisions = extra;
            affine_launch_all(gpu, batch, table, again, true, extra_args);
        }
    }

    WalkArgs w;
    std::memset(&w, 0, sizeof w);
    w.tape = batch.tape;
    w.shapes = batch.shapes;
    w.decisions = decisions;
    w.decisions_extra = extra ? extra : decisions;
    w.layouts = layouts;
    w.widths = widths;
    w.decision_offsets = word_offsets;
    w.ends = ends;
    w.slot_offsets = slot_offsets;
    w.slots = slots;
    w.lengths = lengths;
    w.run_counts = run_counts;
    w.order = walk_order;
    w.failed = batch.flags;
    w.spans = spans;
    w.first_pair = first_pair;
    w.count = count;
    w.bits = batch.bits;
    w.local = batch.local;
    w.eqx = eqx;
    w.uniform = uniform;
    ClockSpan walk_clock(gpu, kClassWalk, gpu->stream);
    // Blocks of 128: the walk's registers leave room for 28 warps an SM, which 256-thread blocks would cut
    // to 24.
    const unsigned walk_blocks = unsigned((count + 127) / 128);
    if (batch.bits == 8)
        walk_kernel<8><<<walk_blocks, 128, 0, gpu->stream>>>(w);
    else
        walk_kernel<2><<<walk_blocks, 128, 0, gpu->stream>>>(w);
    DINARA_CUDA(cudaGetLastError());
    walk_clock.stop();
    gpu->launches += 1;
    timer.stop();
    tally_swept(gpu, batch.shapes, first_pair, count, band, leftovers, left, widths);

    // The CIGARs' offsets, then each spelled from its runs.
    int64_t *offsets = gpu->cigar_offsets.ensure<int64_t>(size_t(count) + 2);
    DINARA_CUDA(cudaMemsetAsync(lengths + count, 0, sizeof(int64_t), gpu->stream));
    size_t scratch3 = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch3, lengths, offsets, int(count + 1), gpu->stream));
    space = gpu->sort_scratch.ensure<uint8_t>(scratch3 + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch3, lengths, offsets, int(count + 1), gpu->stream));
    int64_t total = 0;
    read_back(gpu, &total, offsets + count, sizeof(int64_t));
    char *out = gpu->cigar_bytes.ensure<char>(size_t(total) + 8);
    const unsigned gather_blocks = unsigned((count * 32 + threads - 1) / threads);
    cigar_text_kernel<<<gather_blocks, threads, 0, gpu->stream>>>(slots, slot_offsets, run_counts, offsets, eqx, out,
                                                                  count);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    return total;
}

}  // namespace dinara
