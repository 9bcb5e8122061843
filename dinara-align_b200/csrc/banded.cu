// Global Gotoh over a band of 64 diagonals a pair, proven by the pair's own score.
//
// Four lanes hold a pair's band, 16 diagonals each, and sweep its rows together: a cell at band place o
// on row r is column r + low + o, so the cell diagonally before it sits at the same place a row up, the
// one above at place o + 1 (the next lane's first, by shuffle, at a lane's edge), and the one to its
// left at o - 1 on the same row. The insertion layer along a row is a running maximum (cells shifted by
// (row + column) * extend, as score_groups.mojo:114-120 holds them), so the four lanes take it as a
// prefix maximum: each lane's own, then a two-step shuffle scan across the four. Cells left of column 0
// start below every score and stay there; the first column's cells come out of the recurrence as the
// border the reference sets; cells right of the last column are never read by a real one. So no cell is
// masked.
//
// The query's letters move one place along the band each row: a lane keeps the selectors of 32
// consecutive letters and reads them at a place that advances with the row, the rows unrolled sixteen at
// a time so every place is a constant, and refills the 32 every sixteen rows from three packed words.
//
// The band's score is accepted when every path leaving the band provably scores below it
// (band_proves); then every optimal path lies inside it, so the band's cells on those paths hold the
// whole matrix's values and its recorded decisions walk back the same CIGAR as the whole matrix's.
// Pairs the band does not prove go on a leftover list for the whole-matrix sweep.
#include "affine_kernel.cuh"
#include "banded.cuh"

namespace dinara {
namespace {

using namespace sweep;

constexpr int32_t kUnreached = -(1 << 28);  // below every score a sweep can hold (ScoreReach bounds them)

// The 2-bit codes of the 32 letters of a pair's sequence (`length` letters from packed word `first_word`)
// from letter index `start` on, letter j of the run at bits 2(j % 16) of out[j / 16]; letters before the
// sequence or past its end read as code 0. Three aligned words, shifted into place and masked: no word
// outside the sequence's own is read.
__device__ __forceinline__ void run_of_letters(const uint32_t *__restrict__ tape, uint32_t first_word, int length,
                                               int start, uint32_t out[2]) {
    out[0] = out[1] = 0;
    if (length <= 0) return;
    const int word = start >> 4;  // arithmetic shift: the floor for starts before the sequence
    const int last = (length - 1) >> 4;
    uint32_t words[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) words[i] = __ldg(tape + first_word + min(max(word + i, 0), last));
    const uint32_t shift = uint32_t(start & 15) * 2u;
    out[0] = __funnelshift_r(words[0], words[1], shift);
    out[1] = __funnelshift_r(words[1], words[2], shift);
    // Keep letters j with 0 <= start + j < length (any word clamped above holds none of them).
    const int first = max(-start, 0), final = min(length - 1 - start, 31);
    if (final < first) {
        out[0] = out[1] = 0;
        return;
    }
    const uint64_t upto = final == 31 ? ~0ull : ((1ull << (2 * (final + 1))) - 1ull);
    const uint64_t keep = upto & ~((1ull << (2 * first)) - 1ull);
    out[0] &= uint32_t(keep);
    out[1] &= uint32_t(keep >> 32);
}

template <bool RECORD>
__global__ void __launch_bounds__(kBlock) banded_kernel(BandedBatch b) {
    constexpr int G = kBandLanes, C = kBandColumns;
    constexpr int GPW = 32 / G;
    __shared__ uint2 rows16[4];
    if (threadIdx.x < 4) rows16[threadIdx.x] = b.rows16[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int member = lane % G;
    const int group = lane / G;
    const int warp = int((int64_t(blockIdx.x) * kBlock + threadIdx.x) >> 5);
    const int warps = int((int64_t(gridDim.x) * kBlock) >> 5);
    const int32_t open = b.open, extend = b.extend;
    const int32_t opening = open - extend;

    for (int64_t base = int64_t(warp) * GPW; base < b.count; base += int64_t(warps) * GPW) {
        const int64_t item = base + group;
        const bool live = item < b.count;
        uint32_t pair = 0;
        PairShape sh{0, 0, 0, 0};
        if (live) {
            pair = b.order[item];
            sh = b.shapes[pair];
        }
        const int rows = int(sh.rows), cols = int(sh.columns);
        const int low = live ? band_low_for(rows, cols) : 0;
        const int first_place = member * C;  // this lane's first place in the band
        int warp_rows = live ? rows : 0;
#pragma unroll
        for (int span = 16; span > 0; span >>= 1) warp_rows = max(warp_rows, __shfl_xor_sync(kFull, warp_rows, span));

        // Row 0: the origin 0, the first row's shifted border `opening`, left of the matrix unreached.
        int32_t H[C], D[C];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = low + first_place + k;
            H[k] = c < 0 ? kUnreached : (c == 0 ? 0 : opening);
            D[k] = kUnreached;
        }
        const int end_place = cols - rows - low;  // the corner's place in the band
        int32_t reported = kUnreached;
        int64_t dec_base = 0;
        const int rows_pad = (rows + 3) & ~3;
        if (RECORD && live) dec_base = b.decision_offsets[pair - b.first_pair] + int64_t(member) * rows_pad;
        uint64_t buffered[4] = {0, 0, 0, 0};

        for (int r0 = 1; r0 <= warp_rows; r0 += 16) {
            // Selectors of the 32 letters from column r0 + low + first_place on (letter index one less);
            // columns outside the pair read letter 0, which no real cell's value depends on.
            uint32_t codes[2];
            run_of_letters(b.tape, sh.second_word, live ? cols : 0, r0 + low + first_place - 1, codes);
            uint32_t window[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) window[j] = selector_of((codes[j >> 4] >> (2 * (j & 15))) & 3u);
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int row = r0 + u;
                if (row <= warp_rows) {
                    const bool active = live && row <= rows;
                    // The row above's cell at the next place: this lane's next, or the next lane's first.
                    const int32_t nextH = __shfl_down_sync(kFull, H[0], 1, G);
                    const int32_t nextD = __shfl_down_sync(kFull, D[0], 1, G);
                    uint2 tr = make_uint2(0, 0);
                    if (active) tr = rows16[letter_at<2>(b.tape, sh.first_word, uint32_t(row - 1))];
                    int32_t X[C];
                    int32_t S = kUnreached;  // running max of X + opening along this lane's places
                    uint32_t word_lo = 0, word_hi = 0;
                    // Pass 1: the deletion layer and the best of the diagonal and deletion moves. Only D[k] is
                    // rewritten here, after place k-1 has read it, so every read is of the row above.
#pragma unroll
                    for (int k = 0; k < C; ++k) {
                        const int32_t Hup = k + 1 < C ? H[k + 1] : (member == G - 1 ? kUnreached : nextH);
                        const int32_t Dup = k + 1 < C ? D[k + 1] : (member == G - 1 ? kUnreached : nextD);
                        const int32_t sub = prmt(tr.x, tr.y, window[k + u]);
                        if (RECORD) {
                            const int32_t opened = Hup + opening;
                            const int32_t dn = max(opened, Dup);
                            const int32_t xd = H[k] + sub;
                            const int32_t x = max(xd, dn);
                            // gotoh.mojo:173-186 decide: a deletion run extends only where extending beats
                            // opening; the source is the diagonal unless the deletion beats it.
                            const uint32_t bits = (x != xd ? 1u : 0u) | (Dup > opened ? 4u : 0u);
                            if (k < 8)
                                word_lo |= bits << (4 * k);
                            else
                                word_hi |= bits << (4 * (k - 8));
                            D[k] = dn;
                            X[k] = x;
                        } else {
                            D[k] = __viaddmax_s32(Hup, opening, Dup);
                            X[k] = __viaddmax_s32(H[k], sub, D[k]);
                        }
                        S = __viaddmax_s32(X[k], opening, S);
                    }
                    // Exclusive prefix maximum of the four lanes' running maxima.
                    int32_t reach = __shfl_up_sync(kFull, S, 1, G);
                    if (member == 0) reach = kUnreached;
                    {
                        const int32_t further = __shfl_up_sync(kFull, reach, 1, G);
                        if (member >= 1) reach = max(reach, further);
                        const int32_t further2 = __shfl_up_sync(kFull, reach, 2, G);
                        if (member >= 2) reach = max(reach, further2);
                    }
                    // Pass 2: the insertion layer (the best earlier X plus an opening) and the scores.
                    int32_t S2 = reach;
                    uint32_t ins_lo = 0, ins_hi = 0;
#pragma unroll
                    for (int k = 0; k < C; ++k) {
                        const int32_t I = S2;
                        S2 = __viaddmax_s32(X[k], opening, S2);
                        if (RECORD) {
                            const int32_t Hn = max(X[k], I);
                            // The insertion beats both: the source is inserting (ties go to the diagonal,
                            // then the deletion, as decide() orders them).
                            if (k < 8)
                                ins_lo |= (I > X[k] ? 2u : 0u) << (4 * k);
                            else
                                ins_hi |= (I > X[k] ? 2u : 0u) << (4 * (k - 8));
                            H[k] = Hn;
                            X[k] = I;
                        } else {
                            H[k] = max(X[k], I);
                        }
                    }
                    if (RECORD) {
                        word_lo = (word_lo & ~(ins_lo >> 1)) | ins_lo;
                        word_hi = (word_hi & ~(ins_hi >> 1)) | ins_hi;
                        // Pass 3: an insertion run extends where the left cell's insertion layer beats its
                        // score plus an opening; the left of place 0 is the previous lane's last place.
                        int32_t leftH = __shfl_up_sync(kFull, H[C - 1], 1, G);
                        int32_t leftI = __shfl_up_sync(kFull, X[C - 1], 1, G);
                        if (member == 0) {
                            leftH = kUnreached;
                            leftI = kUnreached;
                        }
#pragma unroll
                        for (int k = 0; k < C; ++k) {
                            const int32_t lh = k == 0 ? leftH : H[k - 1];
                            const int32_t li = k == 0 ? leftI : X[k - 1];
                            const uint32_t bit = li > lh + opening ? 8u : 0u;
                            if (k < 8)
                                word_lo |= bit << (4 * k);
                            else
                                word_hi |= bit << (4 * (k - 8));
                        }
                        buffered[u & 3] = (uint64_t(word_hi) << 32) | word_lo;
                        if (active && ((u & 3) == 3 || row == rows)) {
                            uint4 *at = reinterpret_cast<uint4 *>(b.decisions + dec_base + ((row - 1) & ~3));
                            at[0] = make_uint4(uint32_t(buffered[0]), uint32_t(buffered[0] >> 32),
                                               uint32_t(buffered[1]), uint32_t(buffered[1] >> 32));
                            at[1] = make_uint4(uint32_t(buffered[2]), uint32_t(buffered[2] >> 32),
                                               uint32_t(buffered[3]), uint32_t(buffered[3] >> 32));
                        }
                    }
                    if (active && row == rows) {
#pragma unroll
                        for (int k = 0; k < C; ++k)
                            if (first_place + k == end_place) reported = H[k];
                    }
                }
            }
        }
        // The corner's lane reports; the band's score is accepted when the band proves it.
        const bool holder = live && end_place >= first_place && end_place < first_place + C;
        if (holder) {
            const int64_t score = (rows == 0 && cols == 0) ? 0 : int64_t(reported) + int64_t(rows + cols) * extend;
            const bool proven = band_proves(score, rows, cols, low, b.best, open, extend);
            b.scores[pair] = int32_t(score);
            if (b.proven) b.proven[pair] = proven ? 1 : 0;
            if (!proven) b.leftovers[atomicAdd(b.leftover_count, 1u)] = pair;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// The 16-bit pair sweep: two pairs a lane group, pair A in every register's low half and pair B in its
// high half, so each DPX instruction on 16-bit pairs (full rate on this part, as the 32-bit ones) moves
// two cells. The layout and the recurrence are the 32-bit sweep's; values are held as kPairBias plus the
// shifted cell (unreached cells from kPairUnreached), all within [0, 0x8000) by band_pair_limit, so a
// half never overflows and an add across the whole register never carries from one half to the other.
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t pack2(int32_t low, int32_t high) {
    return (uint32_t(low) & 0xFFFFu) | (uint32_t(high) << 16);
}
__device__ __forceinline__ int32_t low_half(uint32_t v) { return int32_t(int16_t(uint16_t(v & 0xFFFFu))); }
__device__ __forceinline__ int32_t high_half(uint32_t v) { return int32_t(int16_t(uint16_t(v >> 16))); }

// The halves' maximum: the DPX maximum floored at zero, which every value here already is at or above.
__device__ __forceinline__ uint32_t max2(uint32_t a, uint32_t b) { return __vimax_s16x2_relu(a, b); }

// Adds to a plane `acc` (pair A's 16 places in the low half, pair B's in the high) place k's flags: set
// where a half of `v` has bit 15 clear. `v` = b - a + 0x8000 in each half (halves in [0, 0x8000), so
// nothing crosses between them) has bit 15 set exactly where b >= a, so a clear bit records a > b. The
// flags move from bits 15 and 31 down to k and 16 + k by the high word of a product, added in the same
// instruction (the FMA pipe's, leaving the ALU to the cells).
__device__ __forceinline__ uint32_t gather_flag(uint32_t acc, uint32_t v, int k) {
    const uint32_t flags = ~v & 0x80008000u;
    return k == 15 ? acc + flags : __umulhi(flags, 1u << (17 + k)) + acc;
}

// b - a + c (the halves' sums in [0, 0x10000), so none crosses into the other) by two multiply-adds,
// which the multiply-add pipe takes, leaving the ALU pipe, the recording sweep's bound, to the cells.
__device__ __forceinline__ uint32_t difference_mad(uint32_t b, uint32_t a, uint32_t c) {
    uint32_t biased, out;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(biased) : "r"(b), "r"(1u), "r"(c));
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(out) : "r"(a), "r"(0xFFFFFFFFu), "r"(biased));
    return out;
}

// LANES lanes of 16 places a lane group: a band of 32 diagonals (2 lanes, the narrow first pass) or 64
// (4 lanes). In the narrow pass a pair whose band cannot hold both its ends goes straight to the leftover
// list, which the wide pass takes; a pair the narrow band proves is marked as its layout 4.
template <bool RECORD, int LANES>
__global__ void __launch_bounds__(kBlock, 2) banded_pairs_kernel(BandedBatch b) {
    constexpr int G = LANES, C = kBandColumns;
    constexpr int kWidth = G * C;
    constexpr int GPW = 32 / G;      // lane groups a warp
    constexpr int PPW = 2 * GPW;     // pairs a warp
    // Rows a selector window serves: few enough that the unrolled body stays in the instruction cache
    // (fewer when recording, whose body is longer); a refill costs a few instructions a column.
    constexpr int U = RECORD ? 4 : 8;
    constexpr int WIN = C + U;
    __shared__ uint32_t rows8[4];
    if (threadIdx.x < 4) rows8[threadIdx.x] = b.rows8[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int member = lane % G;
    const int group = lane / G;
    const int warp = int((int64_t(blockIdx.x) * kBlock + threadIdx.x) >> 5);
    const int warps = int((int64_t(gridDim.x) * kBlock) >> 5);
    const int32_t opening = b.open - b.extend;
    const uint32_t opening2 = pack2(opening, opening);
    const uint32_t unreached2 = pack2(kPairUnreached, kPairUnreached);
    const uint32_t at_least = 0x80008000u;                             // b - a + this: bit 15 where b >= a
    const uint32_t at_least_open = pack2(0x8000 + opening, 0x8000 + opening);  // b + opening >= a

    for (int64_t base = int64_t(warp) * PPW; base < b.count; base += int64_t(warps) * PPW) {
        const int64_t item = base + 2 * group;
        bool live[2];
        uint32_t pair[2] = {0, 0};
        PairShape sh[2] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        int rows[2], cols[2], low[2], end_place[2], rows_pad[2];
        int64_t dec_base[2] = {0, 0};
        int group_rows = 0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            live[h] = item + h < b.count;
            if (live[h]) {
                pair[h] = b.order[item + h];
                sh[h] = b.shapes[pair[h]];
            }
            rows[h] = int(sh[h].rows);
            cols[h] = int(sh[h].columns);
            low[h] = live[h] ? band_low_for_width(rows[h], cols[h], kWidth) : 0;
            if (live[h] && low[h] == INT32_MIN) {
                // Too narrow a band for this pair: the wide pass takes it (one lane records it once).
                if (member == 0) b.leftovers[atomicAdd(b.leftover_count, 1u)] = pair[h];
                live[h] = false;
                sh[h] = PairShape{0, 0, 0, 0};
                rows[h] = cols[h] = 0;
                low[h] = 0;
            }
            end_place[h] = cols[h] - rows[h] - low[h];
            rows_pad[h] = (rows[h] + 3) & ~3;
            if (RECORD && live[h])
                dec_base[h] = b.decision_offsets[pair[h] - b.first_pair] + int64_t(member) * rows_pad[h];
            group_rows = max(group_rows, live[h] ? rows[h] : 0);
        }
        const int first_place = member * C;
        int warp_rows = group_rows;
#pragma unroll
        for (int span = 16; span > 0; span >>= 1) warp_rows = max(warp_rows, __shfl_xor_sync(kFull, warp_rows, span));

        // Row 0: the origin, the first row's shifted border `opening`, left of the matrix unreached.
        uint32_t H[C], D[C];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            int32_t v[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = low[h] + first_place + k;
                v[h] = c < 0 ? kPairUnreached : (c == 0 ? kPairBias : kPairBias + opening);
            }
            H[k] = pack2(v[0], v[1]);
            D[k] = unreached2;
        }
        int32_t reported[2] = {0, 0};
        uint2 buffered[2][2];  // [pair][row of two]: the rows' 64-bit words, low and high 32 bits

        for (int r0 = 1; r0 <= warp_rows; r0 += U) {
            // Selectors of WIN consecutive columns from r0 + low + first_place, both pairs in one: bytes 0-1
            // pick pair A's entry (sign-extended to 16 bits) from its row, bytes 2-3 pair B's.
            uint32_t codes[2][2];
#pragma unroll
            for (int h = 0; h < 2; ++h)
                run_of_letters(b.tape, sh[h].second_word, live[h] ? cols[h] : 0, r0 + low[h] + first_place - 1,
                               codes[h]);
            uint32_t window[WIN];
#pragma unroll
            for (int j = 0; j < WIN; ++j) {
                const uint32_t a = (codes[0][j >> 4] >> (2 * (j & 15))) & 3u;
                const uint32_t c = (codes[1][j >> 4] >> (2 * (j & 15))) & 3u;
                window[j] = (17u * a + 128u) | ((17u * c + 196u) << 8);
            }
            // The window's rows' reference letters, read before the rows are swept so no global load waits
            // inside a row (rows past a pair's end read letter 0, which no real cell uses).
            uint32_t row_codes[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t run[2];
                run_of_letters(b.tape, sh[h].first_word, live[h] ? rows[h] : 0, r0 - 1, run);
                row_codes[h] = run[0];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int row = r0 + u;
                if (row <= warp_rows) {
                    const uint32_t nextH = __shfl_down_sync(kFull, H[0], 1, G);
                    const uint32_t nextD = __shfl_down_sync(kFull, D[0], 1, G);
                    const uint32_t trA = rows8[(row_codes[0] >> (2 * u)) & 3u];
                    const uint32_t trB = rows8[(row_codes[1] >> (2 * u)) & 3u];
                    uint32_t X[C];
                    uint32_t S = unreached2;  // running max of X + opening along this lane's places
                    // Decision planes, each a bit a place for both pairs (see gather_flag).
                    uint32_t deleting = 0, inserting = 0, deletion_runs = 0, insertion_runs = 0;
                    // Pass 1: the deletion layer, the best of the diagonal and deletion moves, and (scores)
                    // each place's best insertion from this lane's earlier places.
#pragma unroll
                    for (int k = 0; k < C; ++k) {
                        const uint32_t Hup = k + 1 < C ? H[k + 1] : (member == G - 1 ? unreached2 : nextH);
                        const uint32_t Dup = k + 1 < C ? D[k + 1] : (member == G - 1 ? unreached2 : nextD);
                        const uint32_t sub = uint32_t(prmt(trA, trB, window[k + u]));
                        const uint32_t dn = __viaddmax_s16x2(Hup, opening2, Dup);
                        if (RECORD) {
                            const uint32_t xd = __viaddmax_s16x2(H[k], sub, 0u);  // H + sub: never below 0
                            X[k] = max2(xd, dn);
                            // gotoh.mojo:173-186 decide: the source leaves the diagonal only where the
                            // deletion beats it; a deletion run extends only where extending beats opening.
                            deleting = gather_flag(deleting, difference_mad(xd, dn, at_least), k);               // dn > xd
                            deletion_runs = gather_flag(deletion_runs, difference_mad(Hup, Dup, at_least_open), k);  // Dup > Hup + opening
                            S = __viaddmax_s16x2(X[k], opening2, S);
                        } else {
                            const uint32_t x = __viaddmax_s16x2(H[k], sub, dn);
                            X[k] = S;  // the insertion from this lane's earlier places
                            S = __viaddmax_s16x2(x, opening2, S);
                            H[k] = x;
                        }
                        D[k] = dn;
                    }
                    // Exclusive prefix maximum of the lanes' running maxima (two or four lanes).
                    uint32_t reach = __shfl_up_sync(kFull, S, 1, G);
                    if (member == 0) reach = unreached2;
                    if (G > 2) {
                        const uint32_t further = __shfl_up_sync(kFull, reach, 1, G);
                        if (member >= 1) reach = max2(reach, further);
                        const uint32_t further2 = __shfl_up_sync(kFull, reach, 2, G);
                        if (member >= 2) reach = max2(reach, further2);
                    }
                    if (RECORD) {
                        // Pass 2: the insertion layer (the best earlier X plus an opening), the scores, and the
                        // insertion decisions: the source is inserting where the insertion beats both moves (ties
                        // go to the diagonal, then the deletion), and an insertion run extends where the left
                        // cell's insertion beats its score plus an opening.
                        uint32_t S2 = reach;
                        uint32_t prevH = 0, prevI = 0;
#pragma unroll
                        for (int k = 0; k < C; ++k) {
                            const uint32_t I = S2;
                            S2 = __viaddmax_s16x2(X[k], opening2, S2);
                            H[k] = max2(X[k], I);
                            inserting = gather_flag(inserting, difference_mad(X[k], I, at_least), k);  // I > X
                            // The left cell's insertion beats its score plus an opening: the run extends.
                            if (k > 0) insertion_runs = gather_flag(insertion_runs, difference_mad(prevH, prevI, at_least_open), k);
                            prevH = H[k];
                            prevI = I;
                        }
                        // Place 0's insertion-run bit: the left cell is the previous lane's last place.
                        uint32_t leftH = __shfl_up_sync(kFull, prevH, 1, G);
                        uint32_t leftI = __shfl_up_sync(kFull, prevI, 1, G);
                        if (member == 0) {
                            leftH = unreached2;
                            leftI = unreached2;
                        }
                        insertion_runs = gather_flag(insertion_runs, leftH - leftI + at_least_open, 0);
                        // Each pair's 64-bit word of the row: its deleting, inserting, deletion-run and
                        // insertion-run planes, 16 bits each (the walk's layout 3).
                        const int slot = u & 1;
                        buffered[0][slot] = make_uint2(uint32_t(prmt(deleting, inserting, 0x5410u)),
                                                       uint32_t(prmt(deletion_runs, insertion_runs, 0x5410u)));
                        buffered[1][slot] = make_uint2(uint32_t(prmt(deleting, inserting, 0x7632u)),
                                                       uint32_t(prmt(deletion_runs, insertion_runs, 0x7632u)));
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            if (live[h] && row <= rows[h] && (slot == 1 || row == rows[h])) {
                                uint4 *at = reinterpret_cast<uint4 *>(b.decisions + dec_base[h] + ((row - 1) & ~1));
                                *at = make_uint4(buffered[h][0].x, buffered[h][0].y, buffered[h][1].x,
                                                 buffered[h][1].y);
                            }
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < C; ++k) H[k] = __vimax3_s16x2(H[k], X[k], reach);
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (live[h] && row == rows[h]) {
#pragma unroll
                            for (int k = 0; k < C; ++k)
                                if (first_place + k == end_place[h])
                                    reported[h] = (h == 0 ? low_half(H[k]) : high_half(H[k])) - kPairBias;
                        }
                    }
                }
            }
        }
        // The corner's lane reports each pair; the band's score is accepted when the band proves it.
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const bool holder = live[h] && end_place[h] >= first_place && end_place[h] < first_place + C;
            if (holder) {
                const int64_t score = int64_t(reported[h]) + int64_t(rows[h] + cols[h]) * b.extend;
                const bool proven = band_proves_width(score, rows[h], cols[h], low[h], kWidth, b.best, b.open, b.extend);
                b.scores[pair[h]] = int32_t(score);
                if (b.proven) b.proven[pair[h]] = proven ? 1 : 0;
                if (!proven) b.leftovers[atomicAdd(b.leftover_count, 1u)] = pair[h];
                // The narrow band's proven pairs walk its two lanes' decisions (layout 4).
                if (RECORD && proven && kWidth < kBandWidth && b.layouts) b.layouts[pair[h] - b.first_pair] = 4;
                if (b.band_cells) atomicAdd(b.band_cells, (unsigned long long)rows[h] * kWidth);
            }
        }
    }
}

}  // namespace

void banded_launch(dinara_gpu *gpu, const BandedBatch &batch, bool record, bool pairs_of_16, int lanes) {
    if (batch.count <= 0) return;
    const bool narrow = pairs_of_16 && lanes == 2;
    auto fn = pairs_of_16 ? (narrow ? (record ? &banded_pairs_kernel<true, 2> : &banded_pairs_kernel<false, 2>)
                                    : (record ? &banded_pairs_kernel<true, kBandLanes>
                                              : &banded_pairs_kernel<false, kBandLanes>))
                          : (record ? &banded_kernel<true> : &banded_kernel<false>);
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    const int64_t pairs_per_block = (pairs_of_16 ? 2 : 1) * kBlock / (narrow ? 2 : kBandLanes);
    int64_t blocks = int64_t(std::max(per_sm, 1)) * gpu->multiprocessors;
    const int64_t needed = (batch.count + pairs_per_block - 1) / pairs_per_block;
    if (blocks > needed) blocks = needed;
    ClockSpan clock(gpu, record ? kClassBandRecord : kClassBandScore, gpu->stream);
    fn<<<unsigned(blocks), kBlock, 0, gpu->stream>>>(batch);
    DINARA_CUDA(cudaGetLastError());
    clock.stop();
    gpu->launches += 1;
}

}  // namespace dinara
