// The gap-affine sweep kernel shared by the library's launches (affine.cu) and its allocation-free
// entry point (noalloc.cu); see affine.cu for how it sweeps.
#pragma once

#include "affine.cuh"

namespace dinara {
namespace sweep {

constexpr int kBlock = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kPadSelector = 0x9999u;  // every byte the sign of entry 0's high byte: 0 or -1

__device__ __forceinline__ int32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(s));
    return int32_t(d);
}

// The selector that reads letter `x`'s 16-bit entry from a row's two registers, sign-extended.
__device__ __forceinline__ uint32_t selector_of(uint32_t x) {
    const uint32_t lo = 2 * x, hi = 2 * x + 1;
    return lo | (hi << 4) | ((hi | 8u) << 8) | ((hi | 8u) << 12);
}

template <int BITS>
__device__ __forceinline__ uint32_t letter_at(const uint32_t *__restrict__ tape, uint32_t word, uint32_t index) {
    constexpr uint32_t per_word = 32 / BITS;
    constexpr uint32_t mask = BITS == 8 ? 0xFFu : ((1u << BITS) - 1u);
    return (__ldg(tape + word + index / per_word) >> (BITS * (index % per_word))) & mask;
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int span = 16; span > 0; span >>= 1) v = max(v, __shfl_xor_sync(kFull, v, span));
    return v;
}

struct KernelArgs {
    const uint32_t *tape;
    const PairShape *shapes;
    const uint32_t *order;
    uint32_t begin, end;
    int32_t open, extend;
    int32_t *scores;
    int2 *carry;
    int64_t carry_stride;
    // Recording.
    uint64_t *decisions;
    const int64_t *decision_offsets;
    int64_t *ends;  // local: (row << 32) | column of the best cell
    int64_t first_pair;
    // Free ends (affine_kernel<..., FREE>): letters at the reference's start and end and the query's start
    // and end that may go unaligned for nothing, each at most its sequence's length once a pair reads it.
    int32_t free_reference_start, free_reference_end, free_query_start, free_query_end;
    // The widening band (affine_wide_kernel<false, true>): the pair at order[item] is swept over
    // band_widths[item] diagonals from band_low_for_width; the pairs whose band proves nothing are redone
    // wider or whole. A band-recorded pair (affine_kernel<..., BANDED>) reads its proven width at
    // band_widths[pair - first_pair].
    const int32_t *band_widths;
    // Free ends' places (affine_kernel<..., FREE>): with `free_ends_out`, each pair's best end there (row << 32
    // | column, by pair - first_pair), of equal ends the one furthest along the reference less the query
    // with `free_highest`, else the least so (scored.mojo:69-100); with `extents`, each pair is its
    // prefixes of extents[pair - first_pair] (row << 32 | column) letters, both read backwards (the sweep
    // back from an end for its start, scored.mojo:616-633).
    int64_t *free_ends_out;
    const int64_t *extents;
    int32_t free_highest;
    // An extension's Z-drop (affine_kernel<..., ORIGIN>): each anti-diagonal's best cell, its true score
    // (offset by 2^31) in the high 32 bits and its row in the low, kept by atomic maximum at
    // diagonals[diagonal_offsets[pair - first_pair] + row + column].
    unsigned long long *diagonals;
    const int64_t *diagonal_offsets;
};

// The lowest diagonal (column less row) of a band of `width` diagonals holding a pair's main and end
// diagonals, the slack shared either side; INT32_MIN when the band cannot hold both.
__host__ __device__ inline int32_t band_low_for_width(int64_t rows, int64_t columns, int64_t width) {
    const int64_t delta = columns - rows;
    const int64_t span = delta < 0 ? -delta : delta;
    if (span + 1 > width) return INT32_MIN;
    const int64_t slack = (width - 1 - span) / 2;
    return int32_t((delta < 0 ? delta : 0) - slack);
}

// A band-recorded pair (affine_kernel<..., BANDED>): 32 lanes of 16 columns, strips of kRecordStrip
// columns, strip s sweeping only the rows its columns share with the pair's band [low, high] of
// diagonals (column less row) and keeping decisions for those rows alone.
constexpr int kRecordStrip = 512;
__host__ __device__ inline int band_strip_first_row(int s, int high) {
    const int r = s * kRecordStrip + 1 - high;
    return r > 1 ? r : 1;
}
__host__ __device__ inline int band_strip_last_row(int s, int rows, int columns, int low) {
    const int end = (s + 1) * kRecordStrip < columns ? (s + 1) * kRecordStrip : columns;
    return end - low < rows ? end - low : rows;
}
// Words a strip's lane keeps: its rows, the lane's skew of up to 3 and a whole last sector of 4.
__host__ __device__ inline int band_strip_pad(int first_row, int last_row) {
    return ((last_row - first_row + 1 + 2) | 3) + 1;
}
// A band-recorded pair's decision words: 32 lanes a strip.
__host__ __device__ inline int64_t band_record_words(int rows, int columns, int width) {
    const int low = band_low_for_width(rows, columns, width);
    const int high = low + width - 1;
    int64_t words = 0;
    for (int s = 0; s * kRecordStrip < columns; ++s)
        words += 32 * int64_t(band_strip_pad(band_strip_first_row(s, high), band_strip_last_row(s, rows, columns, low)));
    return words;
}
// The cells a band-recorded pair's strips sweep: each strip's rows by its columns.
__host__ __device__ inline int64_t band_record_cells(int rows, int columns, int width) {
    const int low = band_low_for_width(rows, columns, width);
    const int high = low + width - 1;
    int64_t cells = 0;
    for (int s = 0; s * kRecordStrip < columns; ++s) {
        const int strip_columns = columns - s * kRecordStrip < kRecordStrip ? columns - s * kRecordStrip : kRecordStrip;
        cells += int64_t(band_strip_last_row(s, rows, columns, low) - band_strip_first_row(s, high) + 1) * strip_columns;
    }
    return cells;
}

struct TableArgs {
    uint2 rows16[4];       // packed 16-bit entries, letter x at bytes 2x..2x+1
    uint32_t rows8[4];     // byte entries, letter x at byte x (the 16-bit pair sweep)
    int32_t size;
};

// A border cell's true score with free letters (scored.mojo edge): `letters` in from the origin along a side
// whose first `free` letters go unaligned for nothing, a gap from where they end past them.
__device__ __forceinline__ int32_t free_edge(int letters, int free, int32_t open, int32_t extend) {
    return letters <= free ? 0 : open + (letters - free - 1) * extend;
}

// One pair per group of G lanes; see the file's notes. Persistent: each warp takes its next GPW pairs of
// the bucket until the bucket ends. With FREE (global scores, no recording) the letters p.free_* name at
// each end go unaligned for nothing (scored.mojo:69-240 FROM_EDGE): the first row's and first column's
// cells hold free_edge, and the score is the best end on the last row within free_query_end letters of
// the last column or on the last column within free_reference_end letters of the last row.
//
// With BANDED (global recording, 32 lanes of 16 columns) a pair's strip sweeps only the rows its columns
// share with a band of diagonals whose score a sweep over it has proven (band_proves_width), and every
// cell around those rows is unreached (kOut). Each cell's value is then a real path's score within the
// swept rows, and every optimal path of the whole matrix lies in the band, so along such a path each
// decision's terms are the whole matrix's (a term an optimal path reaches equals it; one no optimal path
// reaches is below the cell's value either way), and the walk takes the whole matrix's CIGAR. Decisions
// are kept strip by strip for the swept rows only (band_strip_pad words a lane).
//
// With ORIGIN (and FREE with no free letters: a global sweep from the origin) the result is an extension's
// stop (scored.mojo:69-100 and 272-300, FROM_ORIGIN): the best cell anywhere above zero, of equal ones the
// furthest along both sequences together, then along the reference; none above zero stops at the origin,
// scoring 0.
template <int G, int C, bool LOCAL, bool RECORD, int BITS, bool SMEM_TABLE, bool FREE = false, bool BANDED = false,
          bool ORIGIN = false>
__global__ void __launch_bounds__(kBlock) affine_kernel(KernelArgs p, TableArgs t, const int32_t *__restrict__ table32) {
    static_assert(!FREE || (!LOCAL && !RECORD), "free ends are for global scores");
    static_assert(!BANDED || (!LOCAL && RECORD && !FREE && G == 32 && G * C == kRecordStrip),
                  "a band-recorded pair is global, recorded, and swept in strips of kRecordStrip columns");
    static_assert(!ORIGIN || FREE, "an extension's stop is found by the free-end form");
    constexpr int32_t kOut = -(1 << 28);  // unreached: below every score ScoreReach lets a pair hold
    constexpr int W = G * C;
    constexpr int GPW = 32 / G;
    __shared__ uint2 rows16[4];
    __shared__ int32_t big[SMEM_TABLE ? 32 * 33 : 1];
    if (threadIdx.x < 4) rows16[threadIdx.x] = t.rows16[threadIdx.x];
    if (SMEM_TABLE) {
        for (int i = threadIdx.x; i < 32 * 33; i += kBlock) big[i] = table32[i];
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int member = lane % G;
    const int group = lane / G;
    const int warp = int((int64_t(blockIdx.x) * kBlock + threadIdx.x) >> 5);
    const int warps = int((int64_t(gridDim.x) * kBlock) >> 5);
    const int32_t open = p.open, extend = p.extend;
    const int32_t opening = open - extend;  // a shifted cell's gap step
    const int32_t first_gap = open + extend;
    const int64_t slot = int64_t(warp) * GPW + group;

    for (uint32_t base = p.begin + uint32_t(warp) * GPW; base < p.end; base += uint32_t(warps) * GPW) {
        const uint32_t item = base + group;
        const bool live = item < p.end;
        uint32_t pair = 0;
        PairShape sh{0, 0, 0, 0};
        if (live) {
            pair = p.order[item];
            sh = p.shapes[pair];
        }
        int rows = int(sh.rows), cols = int(sh.columns);
        // FREE with extents: the pair's prefixes, read backwards.
        const bool backwards = FREE && p.extents != nullptr;
        if (backwards && live) {
            const int64_t extent = p.extents[pair - p.first_pair];
            rows = int(extent >> 32);
            cols = int(extent & 0xffffffff);
        }
        const bool work = live && rows > 0 && cols > 0;
        const int strips = work ? (cols + W - 1) / W : 0;
        const int warp_strips = warp_max(strips);
        int32_t reported = 0;
        int32_t best = 0;
        int64_t best_place = 0;
        // Free ends: each side's free letters, and this lane's best end so far (a true score).
        const int free_rs = FREE ? min(p.free_reference_start, rows) : 0;
        const int free_re = FREE ? min(p.free_reference_end, rows) : 0;
        const int free_qs = FREE ? min(p.free_query_start, cols) : 0;
        const int free_qe = FREE ? min(p.free_query_end, cols) : 0;
        int32_t free_best = -(1 << 30);
        int free_key = 0;      // the best end's rows less columns
        int64_t free_at = 0;   // and its place, row << 32 | column
        const bool highest = FREE && p.free_highest != 0;
        if (ORIGIN) free_best = 0;  // an extension's stop beats the origin's 0 only above it
        // An end of `value` at (r, c) against the best so far: higher, or as high on the favoured side
        // (ORIGIN: above zero, and as high further along both, then along the reference).
        auto offer = [&](int32_t value, int r, int c) {
            bool better;
            if (ORIGIN) {
                const int along = r + c, best_along = int(free_at >> 32) + int(free_at & 0xffffffff);
                better = value > 0 && (value > free_best ||
                                       (value == free_best && (along > best_along ||
                                                               (along == best_along && r > int(free_at >> 32)))));
            } else {
                const int key = r - c;
                better = value > free_best || (value == free_best && (highest ? key > free_key : key < free_key));
            }
            if (better) {
                free_best = value;
                free_key = r - c;
                free_at = (int64_t(r) << 32) | int64_t(c);
            }
        };
        int64_t dec_base = 0;
        const int rows_pad = ((rows + 2) | 3) + 1;
        if (RECORD && work) dec_base = p.decision_offsets[pair - p.first_pair];
        // BANDED: the band's diagonals [low, high], the strip's first decision word past the pair's earlier
        // strips', and the previous strip's last swept row.
        int low = 0, high = 0;
        if (BANDED && work) {
            const int width = p.band_widths[pair - p.first_pair];
            low = band_low_for_width(rows, cols, width);
            high = low + width - 1;
        }
        int64_t strip_base = 0;
        int previous_last = rows;
        const int64_t diagonal_base = ORIGIN && p.diagonals && work ? p.diagonal_offsets[pair - p.first_pair] : -1;

        for (int s = 0; s < warp_strips; ++s) {
            const bool strip_live = s < strips;
            const int first_col = s * W + member * C;
            const int owned = min(max(cols - first_col, 0), C);
            // The strip's rows (BANDED: those its columns share with the band) and its lanes' words.
            const int first_row = BANDED ? band_strip_first_row(s, high) : 1;
            const int last_row = BANDED ? band_strip_last_row(s, rows, cols, low) : rows;
            const int strip_pad = BANDED ? band_strip_pad(first_row, last_row) : rows_pad;
            const bool from_top = !BANDED || first_row == 1;
            uint32_t sel[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                const int col = first_col + k;
                if (strip_live && col < cols) {
                    const uint32_t x = letter_at<BITS>(p.tape, sh.second_word, uint32_t(backwards ? cols - 1 - col : col));
                    sel[k] = SMEM_TABLE ? x : selector_of(x);
                } else {
                    sel[k] = SMEM_TABLE ? 32u : kPadSelector;
                }
            }
            const int32_t top = LOCAL ? 0 : opening;
            int32_t H[C], D[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                // The first row, held shifted: with free ends a column's true border less column x extend;
                // BANDED, a strip starting lower has only unreached cells above it.
                H[k] = FREE ? free_edge(first_col + k + 1, free_qs, open, extend) - (first_col + k + 1) * extend : top;
                D[k] = H[k] + first_gap;
                if (!from_top) H[k] = D[k] = kOut;
            }
            int32_t edgeH = FREE ? free_edge(first_col + C, free_qs, open, extend) - (first_col + C) * extend : top;
            int32_t edgeI = edgeH + first_gap;
            int32_t above_left = LOCAL ? 0 : (first_col == 0 ? 0 : opening);
            if (FREE) above_left = free_edge(first_col, free_qs, open, extend) - first_col * extend;
            if (!from_top) {
                // Above and left of the first row: the previous strip's last column for lane 0, else unreached.
                edgeH = edgeI = kOut;
                above_left = member == 0 && s > 0 && strip_live ? p.carry[slot * p.carry_stride + (first_row - 1)].x
                                                                 : kOut;
            }
            const int steps = strip_live ? last_row - first_row + 1 + G : 0;
            const int warp_steps = warp_max(steps);
            uint64_t buffered[4] = {0, 0, 0, 0};
            uint64_t *lane_block = nullptr;
            if (RECORD)
                lane_block = p.decisions + dec_base +
                             (BANDED ? strip_base + int64_t(member) * strip_pad : int64_t(s * G + member) * rows_pad);

            for (int step0 = 1; step0 <= warp_steps; step0 += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int step = step0 + u;
                    if (step <= warp_steps) {
                        const int row = first_row - 1 + step - member;
                        int32_t leftH = __shfl_up_sync(kFull, edgeH, 1, G);
                        int32_t leftI = __shfl_up_sync(kFull, edgeI, 1, G);
                        if (member == 0) {
                            if (s == 0) {
                                leftH = LOCAL ? 0 : opening;
                                // The first column with free ends: the row's true border less row x extend.
                                if (FREE) leftH = free_edge(row, free_rs, open, extend) - row * extend;
                                leftI = leftH + first_gap;
                            } else if (BANDED && row > previous_last) {
                                leftH = leftI = kOut;  // left of the previous strip's swept rows: unreached
                            } else {
                                const int r = min(max(row, 0), rows);
                                const int2 c = p.carry[slot * p.carry_stride + r];
                                leftH = c.x;
                                leftI = c.y;
                            }
                        }
                        int32_t diag = above_left;
                        above_left = leftH;
                        if (strip_live && row >= first_row && row <= last_row) {
                            const uint32_t rl =
                                letter_at<BITS>(p.tape, sh.first_word, uint32_t(backwards ? rows - row : row - 1));
                            uint2 tr = make_uint2(0, 0);
                            const int32_t *trow = nullptr;
                            if (SMEM_TABLE)
                                trow = big + rl * 33;
                            else
                                tr = rows16[rl];
                            int32_t I = 0, Xprev = 0, Hprev = leftH, Iprev = leftI;
                            uint32_t word_lo = 0, word_hi = 0;
                            const int64_t row_place = int64_t(row) * (cols + 1) + first_col + 1;
#pragma unroll
                            for (int k = 0; k < C; ++k) {
                                const int32_t sub = SMEM_TABLE ? trow[sel[k]] : prmt(tr.x, tr.y, sel[k]);
                                const int32_t Hup = H[k], Dup = D[k];
                                int32_t Dn, X, Hn, Xd = 0;
                                if (LOCAL) {
                                    Dn = __viaddmax_s32(Hup, open, Dup + extend);
                                } else {
                                    Dn = __viaddmax_s32(Hup, opening, Dup);
                                }
                                if (RECORD) {
                                    Xd = diag + sub;
                                    X = max(Xd, Dn);
                                } else {
                                    X = __viaddmax_s32(diag, sub, Dn);
                                }
                                if (k == 0) {
                                    I = LOCAL ? max(leftH + open, leftI + extend) : __viaddmax_s32(leftH, opening, leftI);
                                } else {
                                    I = LOCAL ? __viaddmax_s32(I, extend, Xprev) : __viaddmax_s32(Xprev, opening, I);
                                }
                                Hn = LOCAL ? __vimax_s32_relu(X, I) : max(X, I);
                                if (RECORD) {
                                    uint32_t source, dext, iext;
                                    if (LOCAL) {
                                        dext = Dup + extend > Hup + open;
                                        iext = Iprev + extend > Hprev + open;
                                        source = Hn <= 0 ? 3u : (Hn == Xd ? 0u : (Hn == Dn ? 1u : 2u));
                                    } else {
                                        dext = Dup > Hup + opening;
                                        iext = Iprev > Hprev + opening;
                                        source = Hn == Xd ? 0u : (Hn == Dn ? 1u : 2u);
                                    }
                                    const uint32_t nibble = source | (dext << 2) | (iext << 3);
                                    if (k < 8)
                                        word_lo |= nibble << (4 * k);
                                    else
                                        word_hi |= nibble << (4 * (k - 8));
                                    // beats(), gotoh.mojo:122-127, as strips visit rows out of order.
                                    if (LOCAL && k < owned &&
                                        (Hn > best || (Hn == best && Hn != 0 && row_place + k < best_place))) {
                                        best = Hn;
                                        best_place = row_place + k;
                                    }
                                } else if (LOCAL) {
                                    best = max(best, Hn);
                                }
                                // Local: the next cell's insertion reads max(X, 0) + open, kept as Xprev.
                                Xprev = LOCAL ? __viaddmax_s32(X, open, open) : X;
                                Hprev = Hn;
                                Iprev = I;
                                diag = Hup;
                                H[k] = Hn;
                                D[k] = Dn;
                            }
                            edgeH = H[C - 1];
                            edgeI = I;
                            if (member == G - 1 && s + 1 < strips) {
                                p.carry[slot * p.carry_stride + row] = make_int2(H[C - 1], I);
                            }
                            if (!LOCAL && !FREE && row == rows && owned > 0 && first_col + owned == cols) {
                                // The corner by masks, not by an index into H (which would put H in memory).
#pragma unroll
                                for (int k = 0; k < C; ++k) {
                                    const int32_t hit = -int32_t(k == owned - 1);
                                    reported = (reported & ~hit) | (H[k] & hit);
                                }
                            }
                            if (ORIGIN) {
                                // An extension may stop at any cell, as a true score; with a Z-drop each
                                // anti-diagonal's best is kept too, for the stop to be read in their order.
#pragma unroll
                                for (int k = 0; k < C; ++k)
                                    if (k < owned) {
                                        const int column = first_col + k + 1;
                                        const int32_t value = H[k] + (row + column) * extend;
                                        offer(value, row, column);
                                        if (diagonal_base >= 0)
                                            atomicMax(p.diagonals + diagonal_base + row + column,
                                                      (static_cast<unsigned long long>(uint32_t(value) ^ 0x80000000u)
                                                       << 32) | uint32_t(row));
                                    }
                            } else if (FREE) {
                                // Ends on the last row within free_qe letters of the last column, and on the
                                // last column within free_re letters of the last row, as true scores.
                                if (row == rows) {
#pragma unroll
                                    for (int k = 0; k < C; ++k) {
                                        const int column = first_col + k + 1;
                                        if (k < owned && column >= cols - free_qe)
                                            offer(H[k] + (rows + column) * extend, rows, column);
                                    }
                                }
                                if (owned > 0 && first_col + owned == cols && rows - row <= free_re) {
                                    int32_t last = 0;
#pragma unroll
                                    for (int k = 0; k < C; ++k) {
                                        const int32_t hit = -int32_t(k == owned - 1);
                                        last = (last & ~hit) | (H[k] & hit);
                                    }
                                    offer(last + (row + cols) * extend, row, cols);
                                }
                            }
                            if (RECORD) {
                                buffered[u] = (uint64_t(word_hi) << 32) | word_lo;
                                if (u == 3 || row == last_row) {
                                    uint64_t *at = lane_block + ((row - first_row + (member & 3)) & ~3);
                                    reinterpret_cast<uint4 *>(at)[0] = make_uint4(
                                        uint32_t(buffered[0]), uint32_t(buffered[0] >> 32), uint32_t(buffered[1]),
                                        uint32_t(buffered[1] >> 32));
                                    reinterpret_cast<uint4 *>(at)[1] = make_uint4(
                                        uint32_t(buffered[2]), uint32_t(buffered[2] >> 32), uint32_t(buffered[3]),
                                        uint32_t(buffered[3] >> 32));
                                }
                            }
                        }
                    }
                }
            }
            __syncwarp();
            if (BANDED) {
                strip_base += int64_t(G) * strip_pad;
                previous_last = last_row;
            }
        }

        // Results: a global score is the corner shifted back; a local one the group's best.
        if (LOCAL) {
#pragma unroll
            for (int span = 1; span < G; span <<= 1) {
                const int32_t theirs = __shfl_xor_sync(kFull, best, span, G);
                if (RECORD) {
                    const int64_t their_place = __shfl_xor_sync(kFull, best_place, span, G);
                    // beats(), gotoh.mojo:122-127: higher, or equal above zero at an earlier place.
                    if (theirs > best || (theirs == best && theirs != 0 && their_place < best_place)) {
                        best = theirs;
                        best_place = their_place;
                    }
                } else {
                    best = max(best, theirs);
                }
            }
            if (live && member == 0) {
                p.scores[pair] = best;
                if (RECORD) {
                    int64_t end = 0;
                    if (best > 0) {
                        const int64_t stride = cols + 1;
                        end = ((best_place / stride) << 32) | (best_place % stride);
                    }
                    p.ends[pair - p.first_pair] = end;
                }
            }
        } else if (FREE) {
            // The best end of the group's lanes, then the first row's and first column's own ends (a free
            // end reaching the border), or an empty side's run along the other's edge.
#pragma unroll
            for (int span = 1; span < G; span <<= 1) {
                const int32_t their_value = __shfl_xor_sync(kFull, free_best, span, G);
                const int64_t their_at = __shfl_xor_sync(kFull, free_at, span, G);
                offer(their_value, int(their_at >> 32), int(their_at & 0xffffffff));
            }
            if (live && member == 0) {
                if (ORIGIN) {
                    // An extension's stop: the group's best above zero, or the origin.
                } else if (!work) {
                    if (rows == 0 && cols == 0) {
                        free_best = 0;
                        free_at = 0;
                    } else {
                        // scored.mojo:155-176: the run along the other side's edge, ending within its free
                        // letters at the end. Of equal ends, the furthest when the run goes along the
                        // reference and the highest end is favoured (or along the query and the lowest),
                        // else the nearest; free_edge never rises with the letters, so the equal ones run
                        // from the nearest allowed to the last that still scores as it does.
                        const bool along_reference = rows > 0;
                        const int length = along_reference ? rows : cols;
                        const int start_free = along_reference ? free_rs : free_qs;
                        const int lo = max(length - (along_reference ? free_re : free_qe), 0);
                        const int32_t top = free_edge(lo, start_free, open, extend);
                        int reach = lo, beyond = length;
                        if (along_reference == highest) {
                            while (reach < beyond) {
                                const int mid = beyond - (beyond - reach) / 2;
                                if (free_edge(mid, start_free, open, extend) == top)
                                    reach = mid;
                                else
                                    beyond = mid - 1;
                            }
                        }
                        free_best = top;
                        free_at = along_reference ? int64_t(reach) << 32 : int64_t(reach);
                    }
                } else {
                    if (cols <= free_qe) offer(free_edge(rows, free_rs, open, extend), rows, 0);
                    if (rows <= free_re) offer(free_edge(cols, free_qs, open, extend), 0, cols);
                }
                p.scores[pair] = free_best;
                if (p.free_ends_out) p.free_ends_out[pair - p.first_pair] = free_at;
            }
        } else if (live) {
            const int total = rows + cols;
            if (!work) {
                if (member == 0) p.scores[pair] = total == 0 ? 0 : open + (total - 1) * extend;
            } else {
                const int owner_first = ((cols - 1) % W) / C * C;
                if (member == ((cols - 1) % W) / C) {
                    (void)owner_first;
                    p.scores[pair] = reported + total * extend;
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Scores of two pairs a lane group, pair A in every register's low 16 bits and pair B in its high 16 bits:
// the sweep above, cell for cell, each DPX instruction on 16-bit pairs (full rate on this part, as the
// 32-bit ones) moving a cell of each pair. The schedule gives it only pairs whose every value, and every
// value of the cells it sweeps past their ends, stays inside 16 bits: a local cell, held less row x
// extend, is at most the best entry times the columns swept plus the rows times -extend and never below
// a gap's opening; a global cell held shifted moves at most the largest shifted entry or opening a step. Cells past a pair's last row read a row of zero
// entries and cells past its last column a padding of 0 or -1, so neither beats the pair's real cells
// (a local best) nor feeds them (a global corner).
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t halves(int32_t low, int32_t high) {
    return (uint32_t(low) & 0xFFFFu) | (uint32_t(high) << 16);
}
__device__ __forceinline__ int32_t low_of(uint32_t v) { return int32_t(int16_t(uint16_t(v & 0xFFFFu))); }
__device__ __forceinline__ int32_t high_of(uint32_t v) { return int32_t(int16_t(uint16_t(v >> 16))); }

// A column's selector for both pairs: bytes 0-1 pick pair A's entry (sign-extended) from its row's
// register, bytes 2-3 pair B's from the other; kPadHalf reads 0 or -1 (a sign of a byte, replicated).
constexpr uint32_t kPadHalf = 0x99u;
__device__ __forceinline__ uint32_t pair_selector(uint32_t a, uint32_t b) { return a | (b << 8); }
__device__ __forceinline__ uint32_t half_selector_a(uint32_t y) { return 17u * y + 128u; }
__device__ __forceinline__ uint32_t half_selector_b(uint32_t y) { return 17u * y + 196u; }

template <int G, int C, bool LOCAL>
__global__ void __launch_bounds__(kBlock) affine_pairs_kernel(KernelArgs p, TableArgs t, const int32_t *__restrict__) {
    constexpr int W = G * C;
    constexpr int GPW = 32 / G;
    __shared__ uint32_t rows8[4];
    if (threadIdx.x < 4) rows8[threadIdx.x] = t.rows8[threadIdx.x];
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int member = lane % G;
    const int group = lane / G;
    const int warp = int((int64_t(blockIdx.x) * kBlock + threadIdx.x) >> 5);
    const int warps = int((int64_t(gridDim.x) * kBlock) >> 5);
    const int32_t open = p.open, extend = p.extend;
    const int32_t opening = open - extend;
    const int32_t first_gap = open + extend;
    const int64_t slot = int64_t(warp) * GPW + group;
    const uint32_t open2 = halves(open, open), extend2 = halves(extend, extend), opening2 = halves(opening, opening);
    const uint32_t floor2 = halves(-32768, -32768);
    const int32_t top = LOCAL ? 0 : opening;
    const uint32_t top2 = halves(top, top), top_gap2 = halves(top + first_gap, top + first_gap);
    // Local cells are held less row x extend (the table less extend too): a deletion run then climbs by
    // a constant, the zero floor becomes row-dependent, and the best is shifted back a row at a time.
    const uint32_t open_less_extend2 = halves(open - extend, open - extend);

    for (uint32_t base = p.begin + uint32_t(warp) * 2 * GPW; base < p.end; base += uint32_t(warps) * 2 * GPW) {
        const uint32_t item = base + 2 * group;
        bool live[2];
        uint32_t pair[2] = {0, 0};
        PairShape sh[2] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        int rows[2], cols[2], strips[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            live[h] = item + h < p.end;
            if (live[h]) {
                pair[h] = p.order[item + h];
                sh[h] = p.shapes[pair[h]];
            }
            rows[h] = int(sh[h].rows);
            cols[h] = int(sh[h].columns);
            strips[h] = live[h] && rows[h] > 0 && cols[h] > 0 ? (cols[h] + W - 1) / W : 0;
        }
        const int warp_strips = warp_max(max(strips[0], strips[1]));
        uint32_t best2 = 0;
        int32_t reported[2] = {0, 0};

        for (int s = 0; s < warp_strips; ++s) {
            bool strip_live[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) strip_live[h] = s < strips[h];
            const int first_col = s * W + member * C;
            uint32_t sel[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                const int col = first_col + k;
                const uint32_t a = strip_live[0] && col < cols[0]
                                       ? half_selector_a(letter_at<2>(p.tape, sh[0].second_word, uint32_t(col)))
                                       : kPadHalf;
                const uint32_t b = strip_live[1] && col < cols[1]
                                       ? half_selector_b(letter_at<2>(p.tape, sh[1].second_word, uint32_t(col)))
                                       : kPadHalf;
                sel[k] = pair_selector(a, b);
            }
            uint32_t H[C], D[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                H[k] = top2;
                D[k] = top_gap2;
            }
            uint32_t edgeH = top2, edgeI = top_gap2;
            const int32_t corner = LOCAL ? 0 : (first_col == 0 ? 0 : opening);
            uint32_t above_left = halves(corner, corner);
            int group_rows = 0;
#pragma unroll
            for (int h = 0; h < 2; ++h) group_rows = max(group_rows, strip_live[h] ? rows[h] : 0);
            const int steps = group_rows > 0 ? group_rows + G : 0;
            const int warp_steps = warp_max(steps);

            for (int step = 1; step <= warp_steps; ++step) {
                const int row = step - member;
                // Local: this row's lift (row x -extend, at least 0), the floor of its held cells.
                const int32_t lift = LOCAL ? -max(row, 0) * extend : 0;
                const uint32_t floor_h2 = halves(lift, lift), floor_i2 = halves(open + lift, open + lift);
                uint32_t leftH = __shfl_up_sync(kFull, edgeH, 1, G);
                uint32_t leftI = __shfl_up_sync(kFull, edgeI, 1, G);
                if (member == 0) {
                    if (s == 0) {
                        leftH = LOCAL ? floor_h2 : top2;
                        leftI = LOCAL ? halves(lift + first_gap, lift + first_gap) : top_gap2;
                    } else {
                        const int r = min(max(row, 0), group_rows);
                        const int2 c = p.carry[slot * p.carry_stride + r];
                        leftH = uint32_t(c.x);
                        leftI = uint32_t(c.y);
                    }
                }
                uint32_t diag = above_left;
                above_left = leftH;
                if (row >= 1 && row <= group_rows) {
                    uint32_t tr[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        tr[h] = strip_live[h] && row <= rows[h]
                                    ? rows8[letter_at<2>(p.tape, sh[h].first_word, uint32_t(row - 1))]
                                    : 0u;
                    uint32_t I = 0, Xprev = 0;
#pragma unroll
                    for (int k = 0; k < C; ++k) {
                        const uint32_t sub = uint32_t(prmt(tr[0], tr[1], sel[k]));
                        const uint32_t Hup = H[k], Dup = D[k];
                        uint32_t Dn, X, Hn;
                        Dn = __viaddmax_s16x2(Hup, LOCAL ? open_less_extend2 : opening2, Dup);
                        X = __viaddmax_s16x2(diag, sub, Dn);
                        if (k == 0) {
                            I = LOCAL ? __viaddmax_s16x2(leftH, open2, __viaddmax_s16x2(leftI, extend2, floor2))
                                      : __viaddmax_s16x2(leftH, opening2, leftI);
                        } else {
                            I = LOCAL ? __viaddmax_s16x2(I, extend2, Xprev) : __viaddmax_s16x2(Xprev, opening2, I);
                        }
                        if (LOCAL) {
                            Hn = __vimax3_s16x2(X, I, floor_h2);
                            // The next cell's insertion reads the floored X plus an opening.
                            Xprev = __viaddmax_s16x2(X, open2, floor_i2);
                        } else {
                            Hn = __vimax3_s16x2(X, I, X);
                            Xprev = X;
                        }
                        diag = Hup;
                        H[k] = Hn;
                        D[k] = Dn;
                    }
                    edgeH = H[C - 1];
                    edgeI = I;
                    if (LOCAL) {
                        // The row's best, shifted back by its lift, into the running best.
                        uint32_t row_best = H[0];
#pragma unroll
                        for (int k = 1; k + 1 < C; k += 2) row_best = __vimax3_s16x2(row_best, H[k], H[k + 1]);
                        if (C % 2 == 0) row_best = __vimax3_s16x2(row_best, H[C - 1], H[C - 1]);
                        best2 = __viaddmax_s16x2(row_best, halves(-lift, -lift), best2);
                    }
                    if (member == G - 1 && s + 1 < warp_strips)
                        p.carry[slot * p.carry_stride + row] = make_int2(int32_t(H[C - 1]), int32_t(I));
                    if (!LOCAL) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int owned = min(max(cols[h] - first_col, 0), C);
                            if (strip_live[h] && row == rows[h] && owned > 0 && first_col + owned == cols[h]) {
                                // The corner by masks, not by an index into H (which would put H in memory).
                                uint32_t corner = 0;
#pragma unroll
                                for (int k = 0; k < C; ++k) {
                                    const uint32_t hit = 0u - uint32_t(k == owned - 1);
                                    corner |= H[k] & hit;
                                }
                                reported[h] = h == 0 ? low_of(corner) : high_of(corner);
                            }
                        }
                    }
                }
            }
            __syncwarp();
        }

        // Results: a local score is the group's best, a global one the corner (one lane holds it) shifted back.
        if (LOCAL) {
#pragma unroll
            for (int span = 1; span < G; span <<= 1) best2 = __vimax_s16x2_relu(best2, __shfl_xor_sync(kFull, best2, span, G));
            if (member == 0) {
                if (live[0]) p.scores[pair[0]] = low_of(best2);
                if (live[1]) p.scores[pair[1]] = high_of(best2);
            }
        } else {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int32_t value = reported[h];
#pragma unroll
                for (int span = 1; span < G; span <<= 1) value += __shfl_xor_sync(kFull, value, span, G);
                if (live[h] && member == 0) p.scores[pair[h]] = value + (rows[h] + cols[h]) * extend;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Scores of one long pair a block: the sweep above with the whole block of 256 lanes as one group, a
// strip 4,096 columns wide, so a pair of tens of thousands of letters runs on an SM's eight warps
// instead of one. Lane m runs one row behind lane m-1 as before; across a warp boundary the left
// neighbour's edge comes through shared memory, written by the previous warp's last lane in the step
// before and read after the block's barrier that ends it (two buffers by step parity). Every step ends
// with that barrier, so no warp waits on another in any other way.
// ------------------------------------------------------------------------------------------------

// One long pair a block of kBlock lanes, strips of kBlock x 16 columns; see the file's notes. With BANDED
// (global only) a strip sweeps only the rows its columns share with the pair's band of band_widths[item]
// diagonals [low, high]: rows from its first column less high to its last column less low. The cells it
// sweeps outside the band are real cells, and every cell around the swept rows is unreached, so the
// score is the best over paths within the swept rows: at least the band's best, and the whole matrix's
// when the band proves it (band_proves_width).
template <bool LOCAL, bool BANDED>
__global__ void __launch_bounds__(kBlock) affine_wide_kernel(KernelArgs p, TableArgs t, const int32_t *__restrict__) {
    constexpr int C = 16;
    constexpr int W = kBlock * C;
    constexpr int kWarps = kBlock / 32;
    constexpr int32_t kOut = -(1 << 28);  // unreached: below every score ScoreReach lets a pair hold
    static_assert(!(LOCAL && BANDED), "the band proof is for global alignments");
    __shared__ uint2 rows16[4];
    __shared__ int2 handoff[2][kWarps];
    __shared__ int32_t block_best[kWarps];
    if (threadIdx.x < 4) rows16[threadIdx.x] = t.rows16[threadIdx.x];
    __syncthreads();

    const int member = threadIdx.x;
    const int lane = member & 31;
    const int warp = member >> 5;
    const int32_t open = p.open, extend = p.extend;
    const int32_t opening = open - extend;
    const int32_t first_gap = open + extend;
    const int64_t slot = blockIdx.x;

    for (uint32_t item = p.begin + blockIdx.x; item < p.end; item += gridDim.x) {
        const uint32_t pair = p.order[item];
        const PairShape sh = p.shapes[pair];
        const int rows = int(sh.rows), cols = int(sh.columns);
        const int strips = (cols + W - 1) / W;
        int32_t best = 0;
        // The band's diagonals; a pair whose band cannot hold both ends is swept whole.
        int low = -rows, high = cols;
        if (BANDED) {
            const int32_t width = p.band_widths[item];
            const int32_t from = band_low_for_width(rows, cols, width);
            if (from != INT32_MIN) {
                low = from;
                high = from + width - 1;
            }
        }
        int previous_last = rows;  // the previous strip's last swept row

        for (int s = 0; s < strips; ++s) {
            const int first_col = s * W + member * C;
            const int owned = min(max(cols - first_col, 0), C);
            // The strip's rows: those its columns share with the band (all of them when not banded).
            const int first_row = BANDED ? max(1, s * W - high) : 1;
            const int last_row = BANDED ? min(rows, s * W + W - low) : rows;
            uint32_t sel[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                const int col = first_col + k;
                sel[k] = col < cols ? selector_of(letter_at<2>(p.tape, sh.second_word, uint32_t(col))) : kPadSelector;
            }
            // The row above the strip's first: the matrix's top border, or (a strip starting lower, whose
            // cells above lie outside the band) unreached.
            const bool from_top = first_row == 1;
            const int32_t top = from_top ? (LOCAL ? 0 : opening) : kOut;
            int32_t H[C], D[C];
#pragma unroll
            for (int k = 0; k < C; ++k) {
                H[k] = top;
                D[k] = from_top ? top + first_gap : kOut;
            }
            int32_t edgeH = top, edgeI = from_top ? top + first_gap : kOut;
            int32_t above_left = LOCAL ? 0 : (first_col == 0 ? 0 : opening);
            if (BANDED && !from_top) {
                // The cell above and left of the first row: the previous strip's last column (in the band)
                // for lane 0, else outside the band.
                above_left = kOut;
                if (member == 0 && s > 0) above_left = p.carry[slot * p.carry_stride + (first_row - 1)].x;
            }
            const int steps = last_row - first_row + 1 + kBlock;

            for (int step = 1; step <= steps; ++step) {
                const int row = first_row - 1 + step - member;
                int32_t leftH = __shfl_up_sync(kFull, edgeH, 1);
                int32_t leftI = __shfl_up_sync(kFull, edgeI, 1);
                if (lane == 0) {
                    if (member == 0) {
                        if (s == 0) {
                            leftH = LOCAL ? 0 : opening;
                            leftI = leftH + first_gap;
                        } else if (BANDED && row > previous_last) {
                            leftH = kOut;  // left of the previous strip's swept rows: outside the band
                            leftI = kOut;
                        } else {
                            const int r = min(max(row, 0), rows);
                            const int2 c = p.carry[slot * p.carry_stride + r];
                            leftH = c.x;
                            leftI = c.y;
                        }
                    } else {
                        const int2 c = handoff[(step - 1) & 1][warp - 1];
                        leftH = c.x;
                        leftI = c.y;
                    }
                }
                int32_t diag = above_left;
                above_left = leftH;
                if (row >= first_row && row <= last_row) {
                    const uint32_t rl = letter_at<2>(p.tape, sh.first_word, uint32_t(row - 1));
                    const uint2 tr = rows16[rl];
                    int32_t I = 0, Xprev = 0;
#pragma unroll
                    for (int k = 0; k < C; ++k) {
                        const int32_t sub = prmt(tr.x, tr.y, sel[k]);
                        const int32_t Hup = H[k], Dup = D[k];
                        int32_t Dn, X, Hn;
                        if (LOCAL) {
                            Dn = __viaddmax_s32(Hup, open, Dup + extend);
                        } else {
                            Dn = __viaddmax_s32(Hup, opening, Dup);
                        }
                        X = __viaddmax_s32(diag, sub, Dn);
                        if (k == 0) {
                            I = LOCAL ? max(leftH + open, leftI + extend) : __viaddmax_s32(leftH, opening, leftI);
                        } else {
                            I = LOCAL ? __viaddmax_s32(I, extend, Xprev) : __viaddmax_s32(Xprev, opening, I);
                        }
                        Hn = LOCAL ? __vimax_s32_relu(X, I) : max(X, I);
                        if (LOCAL) best = max(best, Hn);
                        Xprev = LOCAL ? __viaddmax_s32(X, open, open) : X;
                        diag = Hup;
                        H[k] = Hn;
                        D[k] = Dn;
                    }
                    edgeH = H[C - 1];
                    edgeI = I;
                    if (member == kBlock - 1 && s + 1 < strips) p.carry[slot * p.carry_stride + row] = make_int2(edgeH, I);
                    if (!LOCAL && row == rows && owned > 0 && first_col + owned == cols) {
                        // The corner by masks, not by an index into H (which would put H in memory).
                        int32_t corner = 0;
#pragma unroll
                        for (int k = 0; k < C; ++k) {
                            const int32_t hit = -int32_t(k == owned - 1);
                            corner = (corner & ~hit) | (H[k] & hit);
                        }
                        p.scores[pair] = corner + (rows + cols) * extend;
                    }
                }
                if (lane == 31) handoff[step & 1][warp] = make_int2(edgeH, edgeI);
                __syncthreads();
            }
            previous_last = last_row;
        }
        if (LOCAL) {
            const int32_t mine = warp_max(best);
            if (lane == 0) block_best[warp] = mine;
            __syncthreads();
            if (member == 0) {
                int32_t all = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) all = max(all, block_best[w]);
                p.scores[pair] = all;
            }
            __syncthreads();
        }
    }
}

}  // namespace sweep
}  // namespace dinara
