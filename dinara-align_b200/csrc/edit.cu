// Unit-cost global edit distance by banded bit-vectors with band doubling, on the B200.
//
// The reference's GPU engine runs Myers/Hyyro over the whole matrix, a thread a pair, with patterns of at
// most 4,096 letters (device_edit.mojo:29-77); its band doubling exists only on the host
// (band.mojo:526-657). Here a pair is swept over the Ukkonen band of a threshold t: every alignment
// costing at most t stays on diagonals d with |d| + |d - delta| <= t, so a window of 64-row words that
// covers those rows at every column, the cells outside it standing for real paths (a run straight down
// from the window's last word, or along the row above its first), yields the cost of some alignment, and
// the distance itself whenever that cost is within t. A result above t doubles t (band.mojo:617) and the
// pair goes round again.
//
// A group of G lanes holds a pair's window, K words a lane, lane m one column behind lane m-1: the step
// out of a lane's last word reaches the next lane by one shuffle. The window slides down one word at
// a time as the band does; where it slides, each lane stalls one step, takes its lower neighbour's first
// word by shuffle, and lane 0 folds the word it drops into the score of the row above the window.
// Nothing waits on anything but the warp's own steps, so no wait can hang.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <utility>
#include <vector>

#include "edit.cuh"

namespace dinara {

namespace {

constexpr int kBlock = 128;
constexpr unsigned kFull = 0xffffffffu;

// A DNA letter's code, the same for planes and text: bits 1-2 of its ASCII byte (A 0, C 1, T 2, G 3).
__device__ __forceinline__ uint32_t dna_code(uint32_t byte) { return (byte >> 1) & 3u; }

// The Myers/Hyyro step of one word (device_edit.mojo:56-75): `carry` is the step into the word's top
// (-1, 0, +1); returns the step out of its bottom bit.
__device__ __forceinline__ int myers_word(uint64_t equal, uint64_t &positive, uint64_t &negative, int carry) {
    const uint64_t vp = positive, vm = negative;
    const uint64_t carry_negative = carry < 0 ? 1ull : 0ull, carry_positive = carry > 0 ? 1ull : 0ull;
    const uint64_t crossing = equal | vm;
    equal |= carry_negative;
    const uint64_t horizontal = (((equal & vp) + vp) ^ vp) | equal;
    uint64_t plus = vm | ~(horizontal | vp);
    uint64_t minus = vp & horizontal;
    const int out = int((plus >> 63) & 1ull) - int((minus >> 63) & 1ull);
    plus = (plus << 1) | carry_positive;
    minus = (minus << 1) | carry_negative;
    positive = minus | ~(crossing | plus);
    negative = plus & crossing;
    return out;
}

__device__ __forceinline__ uint64_t shfl_down64(uint64_t v, int width) {
    const uint32_t lo = __shfl_down_sync(kFull, uint32_t(v), 1, width);
    const uint32_t hi = __shfl_down_sync(kFull, uint32_t(v >> 32), 1, width);
    return (uint64_t(hi) << 32) | lo;
}

struct BandArgs {
    const uint8_t *letters;
    const EditPair *pairs;
    const uint64_t *planes;
    const int64_t *plane_offsets;
    const uint32_t *order;  // pending pairs, sorted
    uint32_t begin, end;
    unsigned *queue;         // the launch's next item, from 0
    const int64_t *thresholds;
    int64_t *banded;         // the round's result per pair
    unsigned long long *swept;
};

template <int G, int K>
__global__ void __launch_bounds__(kBlock) band_kernel(BandArgs a) {
    constexpr int GPW = 32 / G;
    constexpr int W = G * K;
    const int lane = threadIdx.x & 31;
    const int member = lane % G;
    const int group = lane / G;
    const uint32_t count = a.end - a.begin;

    // Each warp takes its next GPW pairs from the launch's queue when it is done with the last ones. The
    // pairs come longest first, so the longest chains start first and the short ones fill in after them.
    for (;;) {
        unsigned first = 0;
        if (lane == 0) first = atomicAdd(a.queue, unsigned(GPW));
        first = __shfl_sync(kFull, first, 0);
        if (first >= count) break;
        const uint32_t item = a.begin + first + uint32_t(group);
        const bool live = item < a.end;
        uint32_t pair = 0;
        EditPair info{0, 0, 0, 0, 0, 0};
        int64_t t = 0;
        if (live) {
            pair = a.order[item];
            info = a.pairs[pair];
            t = a.thresholds[pair];
        }
        const int n = info.n, m = info.m;
        const int words = info.words;
        const int delta = m - n;
        if (t < delta) t = delta;
        // The window sweeps the widest band it holds (band_reach), which costs no more than the band of t
        // and settles every distance within it.
        int64_t half = (t - delta) / 2;
        if (W < words) half = max(half, band_reach(n, m, W));
        const int e = int(half < int64_t(n) + m ? half : int64_t(n) + m);
        const int last = words > W ? words - W : 0;
        // The window's first word at column c is min(max(c - delta - e - 1, 0) / 64, last): it slides at
        // columns delta + e + 1 + 64 k, k = 1 .. last, known in advance.
        const int final_base = live ? min(max(m - delta - e - 1, 0) >> 6, last) : 0;
        // Lane m takes column c at step c + m + base(c): one stall for each word the window slides.
        const int steps = live ? m + G - 1 + final_base : 0;
        int warp_steps = steps;
#pragma unroll
        for (int span = 16; span > 0; span >>= 1) warp_steps = max(warp_steps, __shfl_xor_sync(kFull, warp_steps, span));

        const uint8_t *text = a.letters + info.text;
        const uint8_t *pattern = a.letters + info.pattern;
        const bool dna = info.dna != 0;
        // This lane's words: base + member * K + i; `mine` points at the first one's four planes.
        const uint64_t *mine = dna && live ? a.planes + a.plane_offsets[pair] + 4 * int64_t(member * K) : nullptr;
        int held = words - member * K;  // words of this lane's K that lie inside the pattern
        uint64_t P[K], M[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            P[i] = ~0ull;
            M[i] = 0ull;
        }
        int above = 0;  // lane 0: the score of the row above the window
        int base = 0;   // the window's first word at this lane's last column
        int next_slide = last > 0 ? delta + e + 1 + 64 : INT_MAX;
        int next_col = 1;
        int next_time = 1 + member + (next_slide == 1 ? 1 : 0);
        uint32_t letter = live && m > 0 ? __ldg(text) : 0u;
        int hout = 0;
        for (int step = 1; step <= warp_steps; ++step) {
            const int from_above = G > 1 ? __shfl_up_sync(kFull, hout, 1, G) : 0;
            const bool due = live && next_col <= m && step == next_time;
            const bool slides = due && next_col == next_slide;
            uint64_t belowP = 0, belowM = 0;
            if (G > 1 && __any_sync(kFull, slides)) {
                belowP = shfl_down64(P[0], G);
                belowM = shfl_down64(M[0], G);
            }
            if (due) {
                const int c = next_col;
                if (slides) {
                    if (member == 0) above += __popcll(P[0]) - __popcll(M[0]);
#pragma unroll
                    for (int i = 0; i + 1 < K; ++i) {
                        P[i] = P[i + 1];
                        M[i] = M[i + 1];
                    }
                    if (member == G - 1) {
                        P[K - 1] = ~0ull;
                        M[K - 1] = 0ull;
                    } else {
                        P[K - 1] = belowP;
                        M[K - 1] = belowM;
                    }
                    base += 1;
                    held -= 1;
                    mine += 4;
                    next_slide = base < last ? next_slide + 64 : INT_MAX;
                }
                const uint32_t here = letter;
                if (c < m) letter = __ldg(text + c);  // the next column's letter, early
                int carry = member == 0 ? 1 : from_above;
                const uint32_t code = dna_code(here);
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (i < held) {
                        uint64_t eq;
                        if (dna) {
                            eq = __ldg(mine + 4 * i + code);
                        } else {
                            eq = 0;
                            const int first_row = (base + member * K + i) * 64;
                            const int rows = min(64, n - first_row);
                            for (int j = 0; j < rows; ++j) eq |= uint64_t(pattern[first_row + j] == here) << j;
                        }
                        carry = myers_word(eq, P[i], M[i], carry);
                    }
                }
                hout = carry;
                if (member == 0) above += 1;
                next_col = c + 1;
                next_time = step + 1 + (next_col == next_slide ? 1 : 0);
            }
        }
        // The distance: the row above the window plus every vertical step down to the pattern's last row.
        int64_t sum = member == 0 ? int64_t(above) : 0;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int w = base + member * K + i;
            if (live && w < words) {
                uint64_t mask = ~0ull;
                if (w == words - 1 && (n & 63)) mask = (1ull << (n & 63)) - 1ull;
                sum += __popcll(P[i] & mask) - __popcll(M[i] & mask);
            }
        }
#pragma unroll
        for (int span = 1; span < G; span <<= 1) sum += __shfl_xor_sync(kFull, sum, span, G);
        if (live && member == 0) {
            a.banded[pair] = sum;
            atomicAdd(a.swept, (unsigned long long)(int64_t(m) * min(W, words)));
        }
    }
}

// Four bytes at once: whether each is A, C, G or T (their codes rebuilt into letters by a byte permute
// must give the bytes back), and whether any is 0xFE or 0xFF (the bytes with their low bit set have a byte
// 0xFF exactly there, a zero byte of the complement).
__device__ __forceinline__ bool four_dna(uint32_t word) {
    const uint32_t c = ((word >> 1) & 0x03030303u) ^ ((word >> 2) & 0x01010101u);  // A 0, C 1, G 2, T 3
    const uint32_t t = c | (c >> 4);
    return __byte_perm(0x54474341u, 0u, (t & 0xFFu) | ((t >> 8) & 0xFF00u)) == word;
}
__device__ __forceinline__ bool four_refused(uint32_t word) {
    const uint32_t complement = ~(word | 0x01010101u);
    return ((complement - 0x01010101u) & ~complement & 0x80808080u) != 0u;
}

// A warp a pair: the pattern (the shorter side; the query on a tie, api.mojo:1286-1293), whether both
// sides are DNA, and a refusal for a 0xFE or 0xFF byte (c/dinara.h:15-17). Both sides lie together on the
// tape, read as aligned 16-byte chunks a lane (device letter buffers keep 16 bytes of room past the
// last letter); bytes of a chunk outside the pair count as an A.
__global__ void prepare_kernel(const uint8_t *__restrict__ letters, const int64_t *__restrict__ offsets, int64_t pairs,
                               EditPair *__restrict__ out, int64_t *__restrict__ plane_words,
                               int64_t *__restrict__ results, uint8_t *__restrict__ status) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= pairs) return;
    const int64_t r0 = offsets[2 * warp], q0 = offsets[2 * warp + 1], q1 = offsets[2 * warp + 2];
    const int64_t rlen = q0 - r0, qlen = q1 - q0;
    bool dna = true, refused = false;
    const int64_t first_chunk = r0 >> 4, end_chunk = (q1 + 15) >> 4;
    for (int64_t chunk = first_chunk + lane; chunk < end_chunk; chunk += 32) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(letters) + chunk);
        const uint32_t words[4] = {v.x, v.y, v.z, v.w};
        const int64_t at = chunk << 4;
        const bool inside = at >= r0 && at + 16 <= q1;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t word = words[j];
            if (!inside) {
                uint32_t keep = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int64_t place = at + 4 * j + b;
                    if (place >= r0 && place < q1) keep |= 0xFFu << (8 * b);
                }
                word = (word & keep) | (0x41414141u & ~keep);
            }
            dna = dna && four_dna(word);
            refused = refused || four_refused(word);
        }
    }
    dna = __all_sync(kFull, dna);
    refused = __any_sync(kFull, refused);
    if (lane != 0) return;
    const bool query_pattern = qlen <= rlen;
    EditPair e;
    e.pattern = query_pattern ? q0 : r0;
    e.text = query_pattern ? r0 : q0;
    e.n = int32_t(query_pattern ? qlen : rlen);
    e.m = int32_t(query_pattern ? rlen : qlen);
    e.dna = dna ? 1 : 0;
    e.words = (e.n + 63) / 64;
    out[warp] = e;
    plane_words[warp] = dna ? 4 * int64_t(e.words) : 0;
    status[warp] = refused ? 1 : 0;
    if (refused)
        results[warp] = DINARA_UNSUPPORTED_SYMBOLS;
    else if (e.n == 0)
        results[warp] = e.m;  // api.mojo:1287-1288: an empty side costs the other's letters
    else
        results[warp] = -1000;  // not yet known
}

// A warp a DNA pair: its pattern's four match planes, a word per 64 letters, 256 letters (four words) a
// pass. Lane l takes letters 8l .. 8l + 7 of the pass as one 8-byte value (two aligned loads, shifted
// into place; device letter buffers keep 16 bytes of room past the last letter), and forms a byte of each
// plane from them; a word's byte i of plane x is then lane 8w + i's byte x, gathered by eight shuffles, and
// lanes 0-15 store the pass's 16 words together. Letters past the pattern match no plane.
__global__ void planes_kernel(const uint8_t *__restrict__ letters, const EditPair *__restrict__ pairs, int64_t count,
                              const int64_t *__restrict__ plane_offsets, uint64_t *__restrict__ planes) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;
    const EditPair e = pairs[warp];
    if (!e.dna || e.n == 0) return;
    uint64_t *out = planes + plane_offsets[warp];
    const uintptr_t origin = reinterpret_cast<uintptr_t>(letters + e.pattern);
    const uint32_t shift = uint32_t(origin & 7u) * 8u;
    const uint64_t *aligned = reinterpret_cast<const uint64_t *>(origin & ~uintptr_t(7));
    for (int pass = 0; 256 * pass < e.n; ++pass) {
        const int first = 256 * pass + 8 * lane;  // this lane's first letter in the pattern
        uint32_t packed = 0;                      // byte x: plane x's 8 bits for this lane's letters
        if (first < e.n) {
            const int64_t word = (256 * int64_t(pass) + 8 * lane) >> 3;
            const uint64_t low = __ldg(aligned + word), high = __ldg(aligned + word + 1);
            const uint64_t eight = shift ? (low >> shift) | (high << (64u - shift)) : low;
            const int valid = min(8, e.n - first);
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const uint32_t code = dna_code(uint32_t(eight >> (8 * b)) & 0xFFu);
                if (b < valid) packed |= 1u << (8 * code + b);
            }
        }
        // Lane j < 16 gathers word j / 4's plane j % 4 from lanes 8 (j / 4) .. 8 (j / 4) + 7.
        const int gathered_word = (lane >> 2) & 3, plane = lane & 3;
        uint64_t bits = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t from = __shfl_sync(kFull, packed, 8 * gathered_word + i);
            bits |= uint64_t((from >> (8 * plane)) & 0xFFu) << (8 * i);
        }
        const int64_t w = 4 * int64_t(pass) + gathered_word;
        if (lane < 16 && w < e.words) out[4 * w + plane] = bits;
    }
}

// The first round's pending list and thresholds.
__global__ void start_kernel(const EditPair *__restrict__ pairs, int64_t count, const int64_t *__restrict__ given,
                             int64_t default_start, const uint8_t *__restrict__ status, int64_t *__restrict__ thresholds,
                             int64_t *__restrict__ firsts, uint32_t *__restrict__ pending,
                             unsigned int *__restrict__ pending_count) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const EditPair e = pairs[k];
    if (status[k] || e.n == 0) return;
    const int64_t delta = int64_t(e.m) - e.n;
    int64_t t = given ? given[k] : delta + default_start;
    if (t < delta) t = delta;
    if (t < 1) t = 1;
    thresholds[k] = t;
    firsts[k] = t;
    pending[atomicAdd(pending_count, 1u)] = uint32_t(k);
}

// The counters a band doubling run keeps on the device. The first two fields and the shape counts and
// work come back to the host together, in one read of the context's readback words.
struct BandCounters {
    unsigned pending, next;
    unsigned shape_counts[kBandShapes + 1];
    unsigned long long shape_work[kBandShapes + 1];  // words x text letters, per shape
    unsigned queues[kBandShapes + 1];                // each shape's launch's next item
    unsigned long long swept;
    unsigned long long tallies[4];
    unsigned long long round_work;
};
constexpr size_t kCountsBytes = offsetof(BandCounters, queues);
static_assert(kCountsBytes <= kReadbackBytes, "a round's counts fit the readback words");

// Keys for the pending pairs: band shape in the top bits, then the text length, longest first; each
// shape's pairs and its work (the words its launch sweeps), summed in the block first.
__global__ void band_keys_kernel(const EditPair *__restrict__ pairs, const uint32_t *__restrict__ pending,
                                 const unsigned int *__restrict__ pending_count, const int64_t *__restrict__ thresholds,
                                 bool latency, BandTuning tuning, uint32_t *__restrict__ keys,
                                 BandCounters *__restrict__ counters) {
    __shared__ unsigned block_counts[kBandShapes];
    __shared__ unsigned long long block_work[kBandShapes];
    for (int s = threadIdx.x; s < kBandShapes; s += blockDim.x) {
        block_counts[s] = 0;
        block_work[s] = 0;
    }
    __syncthreads();
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < *pending_count) {
        const uint32_t pair = pending[k];
        const EditPair e = pairs[pair];
        const int shape = band_shape_for(e.n, e.m, thresholds[pair], latency, tuning);
        uint32_t length = uint32_t(e.m) >> 2;
        if (length > 0xFFFFFFu) length = 0xFFFFFFu;
        keys[k] = (uint32_t(shape) << 24) | length;
        atomicAdd(&block_counts[shape], 1u);
        const int64_t window = band_capacity(shape);
        atomicAdd(&block_work[shape], (unsigned long long)(int64_t(e.m) * (window < e.words ? window : e.words)));
    }
    __syncthreads();
    for (int s = threadIdx.x; s < kBandShapes; s += blockDim.x) {
        if (block_counts[s]) {
            atomicAdd(&counters->shape_counts[s], block_counts[s]);
            atomicAdd(&counters->shape_work[s], block_work[s]);
        }
    }
}

// A round's work in its smallest windows: every pending pair's text letters times the words of the
// smallest shape holding its band (at most its pattern's), summed in the block first.
__global__ void round_work_kernel(const EditPair *__restrict__ pairs, const uint32_t *__restrict__ pending,
                                  const unsigned int *__restrict__ pending_count, const int64_t *__restrict__ thresholds,
                                  unsigned long long *__restrict__ work) {
    __shared__ unsigned long long block_work;
    if (threadIdx.x == 0) block_work = 0;
    __syncthreads();
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < *pending_count) {
        const EditPair e = pairs[pending[k]];
        const int64_t needed = band_words_needed(e.n, e.m, thresholds[pending[k]]);
        int64_t smallest = INT64_MAX;
        for (int s = 0; s < kBandShapes; ++s) {
            const int64_t c = band_capacity(s);
            if (c >= needed && c < smallest) smallest = c;
        }
        if (smallest > e.words) smallest = e.words;
        atomicAdd(&block_work, (unsigned long long)(int64_t(e.m) * smallest));
    }
    __syncthreads();
    if (threadIdx.x == 0 && block_work) atomicAdd(work, block_work);
}

// After a round: a result within the band the pair's window swept (band_reach), or from a window as tall
// as the pattern, is the distance; the rest go round again with the threshold doubled, capped by the
// cheapest alignment any round found for the pair (band.mojo:619-657: a round's result is a real
// alignment's cost, so a threshold at it reaches the distance).
__global__ void settle_kernel(const EditPair *__restrict__ pairs, const uint32_t *__restrict__ pending,
                              const unsigned int *__restrict__ pending_count, int64_t *__restrict__ thresholds,
                              int64_t *__restrict__ cheapest, const int64_t *__restrict__ banded,
                              int64_t *__restrict__ results, int64_t *__restrict__ rounds, bool latency,
                              BandTuning tuning, uint32_t *__restrict__ next, unsigned int *__restrict__ next_count) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= *pending_count) return;
    const uint32_t pair = pending[k];
    const EditPair e = pairs[pair];
    const int64_t t = thresholds[pair];
    const int64_t found = banded[pair];
    rounds[pair] += 1;
    const int shape = band_shape_for(e.n, e.m, t, latency, tuning);
    const int64_t window = band_capacity(shape);
    const bool whole = window >= e.words;  // the window holds every word: the whole matrix
    // The proof needs the window to cover the band; the widest window (512 words) falls short only for
    // patterns past 32,768 letters with bands wider than it, refused here (device memory, as the
    // reference refuses what its device cannot hold, common.mojo:211-218).
    const int64_t delta = int64_t(e.m) - e.n;
    const bool covered = whole || window >= band_words_needed(e.n, e.m, t);
    // The band the window swept: diagonals within delta + 2 reach + 1 of one another, reach at least t's.
    const int64_t half = t > delta ? (t - delta) / 2 : 0;
    const int64_t reach = band_reach(e.n, e.m, window);
    const int64_t swept_threshold = delta + 2 * (reach > half ? reach : half) + 1;
    if (covered && (found <= (t > swept_threshold ? t : swept_threshold) || whole)) {
        results[pair] = found;
    } else if (!covered && t >= int64_t(e.n) + e.m) {
        results[pair] = DINARA_OUT_OF_MEMORY;
    } else {
        // A window short of its band proves nothing at the cap, so only a covered round caps the next.
        const int64_t best = found < cheapest[pair] ? found : cheapest[pair];
        cheapest[pair] = best;
        thresholds[pair] = covered && best < 2 * t ? best : 2 * t;
        next[atomicAdd(next_count, 1u)] = pair;
    }
}

using BandFn = void (*)(BandArgs);

template <int S>
constexpr BandFn band_of() {
    return &band_kernel<(S < 36 ? (1 << (S / 6)) : 32), (S < 36 ? S % 6 + 1 : (S == 36 ? 8 : S == 37 ? 12 : 16))>;
}

template <int... S>
BandFn pick_from(int shape, std::integer_sequence<int, S...>) {
    static const BandFn table[] = {band_of<S>()...};
    return table[shape];
}

BandFn pick_band(int shape) { return pick_from(shape, std::make_integer_sequence<int, kBandShapes>{}); }

// The autotuner's order and thresholds: every pair in batch order, at its length difference.
__global__ void identity_kernel(const EditPair *__restrict__ pairs, int64_t count, uint32_t *__restrict__ order,
                                int64_t *__restrict__ thresholds) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    order[k] = uint32_t(k);
    thresholds[k] = int64_t(pairs[k].m) - pairs[k].n;
}

// The report's per-pair tallies: rounds taken, first-round hits and how the first threshold stood
// against the distance.
__global__ void tally_kernel(const EditPair *__restrict__ pairs, int64_t count, const uint8_t *__restrict__ status,
                             const int64_t *__restrict__ firsts, const int64_t *__restrict__ rounds,
                             const int64_t *__restrict__ results, unsigned long long *__restrict__ tallies) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const EditPair e = pairs[k];
    if (status[k] || e.n == 0 || results[k] < 0) return;
    const int64_t d = results[k];
    atomicAdd(&tallies[0], (unsigned long long)rounds[k]);
    if (rounds[k] == 1) atomicAdd(&tallies[1], 1ull);
    if (firsts[k] >= 2 * (d > 0 ? d : 1)) atomicAdd(&tallies[2], 1ull);
    if (firsts[k] < d) atomicAdd(&tallies[3], 1ull);
}

}  // namespace

PreparedPairs prepare_pairs(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                            int64_t *results) {
    cudaStream_t stream = gpu->stream;
    PreparedPairs p;
    p.info = gpu->shapes.ensure<EditPair>(size_t(pairs));
    int64_t *plane_words = gpu->plane_offsets.ensure<int64_t>(2 * size_t(pairs + 1) + 2);
    p.plane_offsets = plane_words + (pairs + 1);
    p.status = gpu->flags.ensure<uint8_t>(size_t(pairs));
    const int threads = 256;
    const unsigned warp_blocks = unsigned((pairs * 32 + threads - 1) / threads);
    prepare_kernel<<<warp_blocks, threads, 0, stream>>>(letters, offsets, pairs, p.info, plane_words, results,
                                                        p.status);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    DINARA_CUDA(cudaMemsetAsync(plane_words + pairs, 0, sizeof(int64_t), stream));
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, plane_words, p.plane_offsets, int(pairs + 1), stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(scratch + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, plane_words, p.plane_offsets, int(pairs + 1), stream));
    int64_t plane_total = 0;
    read_back(gpu, &plane_total, p.plane_offsets + pairs, sizeof(int64_t));
    p.planes = gpu->planes.ensure<uint64_t>(size_t(plane_total) + 4);
    planes_kernel<<<warp_blocks, threads, 0, stream>>>(letters, p.info, pairs, p.plane_offsets, p.planes);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    return p;
}

double band_shape_rate(dinara_gpu *gpu, int shape, int64_t pairs, const uint8_t *letters, const PreparedPairs &p,
                       int64_t *scratch) {
    cudaStream_t stream = gpu->stream;
    // Every pair once, in batch order, at its length difference: the sweep's work is the window's words
    // at every column whatever the threshold.
    uint32_t *order = gpu->order_sorted.ensure<uint32_t>(size_t(pairs));
    int64_t *thresholds = scratch;
    int64_t *banded = scratch + pairs;
    const int threads = 256;
    identity_kernel<<<unsigned((pairs + threads - 1) / threads), threads, 0, stream>>>(p.info, pairs, order,
                                                                                       thresholds);
    DINARA_CUDA(cudaGetLastError());
    BandCounters *counters = reinterpret_cast<BandCounters *>(
        gpu->counters.ensure<unsigned int>((sizeof(BandCounters) + 3) / 4));
    DINARA_CUDA(cudaMemsetAsync(counters, 0, sizeof(BandCounters), stream));
    BandArgs args;
    args.letters = letters;
    args.pairs = p.info;
    args.planes = p.planes;
    args.plane_offsets = p.plane_offsets;
    args.order = order;
    args.begin = 0;
    args.end = uint32_t(pairs);
    args.queue = &counters->queues[0];
    args.thresholds = thresholds;
    args.banded = banded;
    args.swept = &counters->swept;
    BandFn fn = pick_band(shape);
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    const int64_t groups_per_block = kBlock / band_lanes(shape);
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>(int64_t(std::max(per_sm, 1)) * gpu->multiprocessors, (pairs + groups_per_block - 1) / groups_per_block));
    DINARA_CUDA(cudaEventRecord(gpu->start, stream));
    fn<<<unsigned(grid), kBlock, 0, stream>>>(args);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    DINARA_CUDA(cudaEventRecord(gpu->stop, stream));
    unsigned long long words = 0;
    read_back(gpu, &words, &counters->swept, sizeof words);
    float ms = 0.f;
    DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
    return ms > 0.f ? double(words) / double(ms) : 0.0;
}

int band_shape_blocks(dinara_gpu *gpu, int shape) {
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_band(shape), kBlock, 0));
    return std::max(per_sm, 1);
}

void band_doubling(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                   const int64_t *first_thresholds_device, int64_t default_start, int64_t *results,
                   dinara_band_report *report) {
    cudaStream_t stream = gpu->stream;
    const int threads = 256;
    const unsigned thread_blocks = unsigned((pairs + threads - 1) / threads);
    const PreparedPairs prepared = prepare_pairs(gpu, pairs, letters, offsets, results);
    EditPair *info = prepared.info;
    const int64_t *plane_offsets = prepared.plane_offsets;
    const uint64_t *planes = prepared.planes;
    const uint8_t *status = prepared.status;
    void *space = nullptr;

    int64_t *thresholds = gpu->thresholds.ensure<int64_t>(4 * size_t(pairs));
    int64_t *firsts = thresholds + pairs;
    int64_t *rounds = thresholds + 2 * pairs;
    int64_t *cheapest = thresholds + 3 * pairs;
    int64_t *banded = gpu->distances.ensure<int64_t>(size_t(pairs));
    uint32_t *pending = gpu->pending.ensure<uint32_t>(size_t(pairs));
    uint32_t *next = gpu->pending_next.ensure<uint32_t>(size_t(pairs));
    BandCounters *counters = reinterpret_cast<BandCounters *>(
        gpu->counters.ensure<unsigned int>((sizeof(BandCounters) + 3) / 4));
    unsigned long long *swept = &counters->swept;
    DINARA_CUDA(cudaMemsetAsync(counters, 0, sizeof(BandCounters), stream));
    DINARA_CUDA(cudaMemsetAsync(rounds, 0, size_t(pairs) * sizeof(int64_t), stream));
    DINARA_CUDA(cudaMemsetAsync(cheapest, 0x7f, size_t(pairs) * sizeof(int64_t), stream));  // above any cost
    start_kernel<<<thread_blocks, threads, 0, stream>>>(info, pairs, first_thresholds_device,
                                                        default_start > 0 ? default_start : 256, status, thresholds,
                                                        firsts, pending, &counters->pending);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    uint32_t *keys = gpu->keys.ensure<uint32_t>(size_t(pairs));
    uint32_t *keys_sorted = gpu->keys_sorted.ensure<uint32_t>(size_t(pairs));
    uint32_t *order_sorted = gpu->order_sorted.ensure<uint32_t>(size_t(pairs));
    if (gpu->band_tuning.chain_words == 0) gpu->band_tuning = default_band_tuning();
    const BandTuning tuned = gpu->band_tuning;
    alignas(8) unsigned char host_bytes[kCountsBytes];
    const BandCounters *host = reinterpret_cast<const BandCounters *>(host_bytes);
    read_back(gpu, host_bytes, counters, sizeof(unsigned int));
    int64_t count = host->pending;
    int64_t launches = 0;
    float kernel_ms = 0.f;
    int64_t round = 0;
    int64_t round_pairs[16] = {0}, round_launches[16] = {0};
    double round_ms[16] = {0.0};
    while (count > 0) {
        const int64_t launches_before = launches;
        const int64_t round_count = count;
        // Order the round's pairs: by band shape, longest text first.
        DINARA_CUDA(cudaMemsetAsync(&counters->next, 0, offsetof(BandCounters, swept) - offsetof(BandCounters, next),
                                    stream));
        const unsigned blocks = unsigned((count + threads - 1) / threads);
        // A round of few pairs takes the one-word-a-lane windows: lanes to spare, and the sweep's time is
        // its longest pair's chain of steps.
        const bool latency = count <= int64_t(gpu->multiprocessors) * 32;
        // The round's chain bound from its work over the GPU's lanes (1,024 an SM).
        BandTuning tuning = tuned;
        if (tuned.chain_share > 0.f && !latency) {
            DINARA_CUDA(cudaMemsetAsync(&counters->round_work, 0, sizeof(unsigned long long), stream));
            round_work_kernel<<<blocks, threads, 0, stream>>>(info, pending, &counters->pending, thresholds,
                                                              &counters->round_work);
            gpu->launches += 1;
            DINARA_CUDA(cudaGetLastError());
            unsigned long long work = 0;
            read_back(gpu, &work, &counters->round_work, sizeof work);
            const double per_lane = double(work) / (double(gpu->multiprocessors) * 1024.0);
            tuning.chain_words = std::max<int64_t>(tuned.chain_words, int64_t(tuned.chain_share * per_lane));
        }
        band_keys_kernel<<<blocks, threads, 0, stream>>>(info, pending, &counters->pending, thresholds, latency,
                                                         tuning, keys, counters);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        size_t sort_bytes = 0;
        DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, keys, keys_sorted, pending,
                                                              order_sorted, int(count), 0, 32, stream));
        space = gpu->sort_scratch.ensure<uint8_t>(sort_bytes + 256);
        DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(space, sort_bytes, keys, keys_sorted, pending,
                                                              order_sorted, int(count), 0, 32, stream));
        read_back(gpu, host_bytes, counters, kCountsBytes);
        DINARA_CUDA(cudaEventRecord(gpu->start, stream));
        ClockSpan clock(gpu, kClassUnitBand, stream);
        // Each shape's launch on a side stream, all forked from and joined back to the context's stream,
        // so they run at once. Each takes a share of the GPU's lanes in proportion to its share of the
        // round's work, so that they end together; the longest chains start first within each.
        DINARA_CUDA(cudaEventRecord(gpu->fork, stream));
        bool used[dinara_gpu::kSideStreams] = {false};
        // A shape's share of the round's time: its words at its measured cost a word.
        double total_work = 0.0;
        for (int shape = 0; shape < kBandShapes; ++shape)
            total_work += double(host->shape_work[shape]) * tuning.word_cost[shape];
        // Shapes in descending order, as the keys sort them.
        int64_t at = 0;
        for (int shape = kBandShapes - 1; shape >= 0; --shape) {
            const int64_t n_shape = host->shape_counts[shape];
            if (n_shape == 0) continue;
            BandArgs args;
            args.letters = letters;
            args.pairs = info;
            args.planes = planes;
            args.plane_offsets = plane_offsets;
            args.order = order_sorted;
            args.begin = uint32_t(at);
            args.end = uint32_t(at + n_shape);
            args.queue = &counters->queues[shape];
            args.thresholds = thresholds;
            args.banded = banded;
            args.swept = swept;
            const int G = band_lanes(shape);
            const int groups_per_block = kBlock / G;
            BandFn fn = pick_band(shape);
            int per_sm = 0;
            DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
            const double share = tuning.full_grids || total_work <= 0
                                     ? 1.0
                                     : double(host->shape_work[shape]) * tuning.word_cost[shape] / total_work;
            int64_t grid = int64_t(std::ceil(share * std::max(per_sm, 1) * gpu->multiprocessors));
            const int64_t needed = (n_shape + groups_per_block - 1) / groups_per_block;
            grid = std::max<int64_t>(1, std::min(grid, needed));
            const int side = shape % dinara_gpu::kSideStreams;
            if (!used[side]) DINARA_CUDA(cudaStreamWaitEvent(gpu->side[side], gpu->fork, 0));
            used[side] = true;
            fn<<<unsigned(grid), kBlock, 0, gpu->side[side]>>>(args);
            gpu->launches += 1;
            DINARA_CUDA(cudaGetLastError());
            at += n_shape;
            ++launches;
        }
        for (int side = 0; side < dinara_gpu::kSideStreams; ++side) {
            if (!used[side]) continue;
            DINARA_CUDA(cudaEventRecord(gpu->joins[side], gpu->side[side]));
            DINARA_CUDA(cudaStreamWaitEvent(stream, gpu->joins[side], 0));
        }
        DINARA_CUDA(cudaEventRecord(gpu->stop, stream));
        clock.stop();
        DINARA_CUDA(cudaMemsetAsync(&counters->next, 0, sizeof(unsigned int), stream));
        settle_kernel<<<blocks, threads, 0, stream>>>(info, order_sorted, &counters->pending, thresholds, cheapest,
                                                      banded, results, rounds, latency, tuning, next, &counters->next);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        DINARA_CUDA(cudaMemcpyAsync(&counters->pending, &counters->next, sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                    stream));
        read_back(gpu, host_bytes, counters, sizeof(unsigned int));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
        kernel_ms += ms;
        if (round < 16) {
            round_pairs[round] = round_count;
            round_launches[round] = launches - launches_before;
            round_ms[round] = ms;
        }
        ++round;
        count = host->pending;
        std::swap(pending, next);
    }
    if (report) {
        unsigned long long *tallies = counters->tallies;
        DINARA_CUDA(cudaMemsetAsync(tallies, 0, 4 * sizeof(unsigned long long), stream));
        tally_kernel<<<thread_blocks, threads, 0, stream>>>(info, pairs, status, firsts, rounds, results, tallies);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        unsigned long long totals[5] = {0, 0, 0, 0, 0};
        read_back(gpu, totals, swept, sizeof(totals));
        report->rounds = launches;
        report->words_swept = int64_t(totals[0]);
        report->pair_rounds = int64_t(totals[1]);
        report->first_round_hits = int64_t(totals[2]);
        report->overshoot = int64_t(totals[3]);
        report->undershoot = int64_t(totals[4]);
        report->kernel_ms = kernel_ms;
        for (int k = 0; k < 16; ++k) {
            report->round_pairs[k] = round_pairs[k];
            report->round_launches[k] = round_launches[k];
            report->round_ms[k] = round_ms[k];
        }
    }
}

}  // namespace dinara
