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
#include <vector>

#include "edit.cuh"

namespace dinara {

namespace {

constexpr int kBlock = 128;
constexpr unsigned kFull = 0xffffffffu;

// A DNA letter's code, the same for planes and text: bits 1-2 of its ASCII byte (A 0, C 1, T 2, G 3).
__device__ __forceinline__ uint32_t dna_code(uint32_t byte) { return (byte >> 1) & 3u; }

__device__ __forceinline__ bool is_dna(uint32_t byte) {
    return byte == 'A' || byte == 'C' || byte == 'G' || byte == 'T';
}

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
    const int warp = int((int64_t(blockIdx.x) * kBlock + threadIdx.x) >> 5);
    const int warps = int((int64_t(gridDim.x) * kBlock) >> 5);

    for (uint32_t base_item = a.begin + uint32_t(warp) * GPW; base_item < a.end; base_item += uint32_t(warps) * GPW) {
        const uint32_t item = base_item + group;
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
        const int64_t half = (t - delta) / 2;
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
            const int from_above = __shfl_up_sync(kFull, hout, 1, G);
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
                            const int first = (base + member * K + i) * 64;
                            const int count = min(64, n - first);
                            for (int j = 0; j < count; ++j) eq |= uint64_t(pattern[first + j] == here) << j;
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

// A warp a pair: the pattern (the shorter side; the query on a tie, api.mojo:1286-1293), whether both
// sides are DNA, and a refusal for a 0xFE or 0xFF byte (c/dinara.h:15-17).
__global__ void prepare_kernel(const uint8_t *__restrict__ letters, const int64_t *__restrict__ offsets, int64_t pairs,
                               EditPair *__restrict__ out, int64_t *__restrict__ plane_words,
                               int64_t *__restrict__ results, uint8_t *__restrict__ status) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= pairs) return;
    const int64_t r0 = offsets[2 * warp], q0 = offsets[2 * warp + 1], q1 = offsets[2 * warp + 2];
    const int64_t rlen = q0 - r0, qlen = q1 - q0;
    bool dna = true, refused = false;
    for (int64_t i = lane; i < rlen + qlen; i += 32) {
        const uint32_t byte = letters[r0 + i];
        dna = dna && is_dna(byte);
        refused = refused || byte >= 0xFE;
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

// A warp a DNA pair: its pattern's four match planes, a word per 64 letters. The warp reads a word's 64
// letters two to a lane (coalesced) and takes each plane's 64 bits as two ballots.
__global__ void planes_kernel(const uint8_t *__restrict__ letters, const EditPair *__restrict__ pairs, int64_t count,
                              const int64_t *__restrict__ plane_offsets, uint64_t *__restrict__ planes) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;
    const EditPair e = pairs[warp];
    if (!e.dna || e.n == 0) return;
    uint64_t *out = planes + plane_offsets[warp];
    const uint8_t *pattern = letters + e.pattern;
    for (int w = 0; w < e.words; ++w) {
        const int first = 64 * w + lane, second = first + 32;
        // Letters past the pattern match no plane.
        const uint32_t low_code = first < e.n ? dna_code(__ldg(pattern + first)) : 4u;
        const uint32_t high_code = second < e.n ? dna_code(__ldg(pattern + second)) : 4u;
#pragma unroll
        for (uint32_t x = 0; x < 4; ++x) {
            const uint32_t low = __ballot_sync(kFull, low_code == x);
            const uint32_t high = __ballot_sync(kFull, high_code == x);
            if (lane == int(x)) out[4 * int64_t(w) + x] = (uint64_t(high) << 32) | low;
        }
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

// Keys for the pending pairs: band shape in the top bits, then the text length, longest first.
__global__ void band_keys_kernel(const EditPair *__restrict__ pairs, const uint32_t *__restrict__ pending,
                                 const unsigned int *__restrict__ pending_count, const int64_t *__restrict__ thresholds,
                                 bool latency, uint32_t *__restrict__ keys, unsigned int *__restrict__ shape_counts) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= *pending_count) return;
    const uint32_t pair = pending[k];
    const EditPair e = pairs[pair];
    const int shape = band_shape_for(e.n, e.m, thresholds[pair], latency);
    uint32_t length = uint32_t(e.m) >> 2;
    if (length > 0xFFFFFFu) length = 0xFFFFFFu;
    keys[k] = (uint32_t(shape) << 24) | length;
    atomicAdd(&shape_counts[shape], 1u);
}

// After a round: a result within its threshold, or from a band as wide as the matrix, is the distance;
// the rest go round again with the threshold doubled, capped by the cheapest alignment any round found
// for the pair (band.mojo:619-657: a round's result is a real alignment's cost, so a threshold at it
// reaches the distance).
__global__ void settle_kernel(const EditPair *__restrict__ pairs, const uint32_t *__restrict__ pending,
                              const unsigned int *__restrict__ pending_count, int64_t *__restrict__ thresholds,
                              int64_t *__restrict__ cheapest, const int64_t *__restrict__ banded,
                              int64_t *__restrict__ results, int64_t *__restrict__ rounds, bool latency,
                              uint32_t *__restrict__ next, unsigned int *__restrict__ next_count) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= *pending_count) return;
    const uint32_t pair = pending[k];
    const EditPair e = pairs[pair];
    const int64_t t = thresholds[pair];
    const int64_t found = banded[pair];
    rounds[pair] += 1;
    const int shape = band_shape_for(e.n, e.m, t, latency);
    const int64_t window = int64_t(band_lanes(shape)) * band_words_per_lane(shape);
    const bool whole = window >= e.words;  // the window holds every word: the whole matrix
    // The proof needs the window to cover the band; the widest window (512 words) falls short only for
    // patterns past 32,768 letters with bands wider than it, refused here (device memory, as the
    // reference refuses what its device cannot hold, common.mojo:211-218).
    const int64_t delta = int64_t(e.m) - e.n;
    const int64_t half = t > delta ? (t - delta) / 2 : 0;
    const bool covered = whole || window >= (delta + 2 * half + 1 + 63) / 64 + 1;
    if (covered && (found <= t || whole)) {
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

BandFn pick_band(int shape) {
    switch (shape) {
        case 0: return &band_kernel<1, 1>;
        case 1: return &band_kernel<1, 2>;
        case 2: return &band_kernel<1, 3>;
        case 3: return &band_kernel<1, 4>;
        case 4: return &band_kernel<2, 3>;
        case 5: return &band_kernel<4, 2>;
        case 6: return &band_kernel<4, 3>;
        case 7: return &band_kernel<8, 2>;
        case 8: return &band_kernel<8, 3>;
        case 9: return &band_kernel<16, 2>;
        case 10: return &band_kernel<16, 3>;
        case 11: return &band_kernel<32, 2>;
        case 12: return &band_kernel<32, 3>;
        case 13: return &band_kernel<32, 4>;
        case 14: return &band_kernel<32, 6>;
        case 15: return &band_kernel<32, 8>;
        case 16: return &band_kernel<32, 12>;
        case 17: return &band_kernel<32, 16>;
        case 18: return &band_kernel<2, 1>;
        case 19: return &band_kernel<4, 1>;
        case 20: return &band_kernel<8, 1>;
        case 21: return &band_kernel<16, 1>;
        default: return &band_kernel<32, 1>;
    }
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

void band_doubling(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                   const int64_t *first_thresholds_device, int64_t default_start, int64_t *results,
                   dinara_band_report *report) {
    cudaStream_t stream = gpu->stream;
    EditPair *info = gpu->shapes.ensure<EditPair>(size_t(pairs));
    int64_t *plane_words = gpu->plane_offsets.ensure<int64_t>(2 * size_t(pairs + 1) + 2);
    int64_t *plane_offsets = plane_words + (pairs + 1);
    uint8_t *status = gpu->flags.ensure<uint8_t>(size_t(pairs));
    const int threads = 256;
    const unsigned warp_blocks = unsigned((pairs * 32 + threads - 1) / threads);
    const unsigned thread_blocks = unsigned((pairs + threads - 1) / threads);
    prepare_kernel<<<warp_blocks, threads, 0, stream>>>(letters, offsets, pairs, info, plane_words, results, status);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    DINARA_CUDA(cudaMemsetAsync(plane_words + pairs, 0, sizeof(int64_t), stream));
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, plane_words, plane_offsets, int(pairs + 1), stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(scratch + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, plane_words, plane_offsets, int(pairs + 1), stream));
    int64_t plane_total = 0;
    read_back(gpu, &plane_total, plane_offsets + pairs, sizeof(int64_t));
    uint64_t *planes = gpu->planes.ensure<uint64_t>(size_t(plane_total) + 4);
    planes_kernel<<<warp_blocks, threads, 0, stream>>>(letters, info, pairs, plane_offsets, planes);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());

    int64_t *thresholds = gpu->thresholds.ensure<int64_t>(4 * size_t(pairs));
    int64_t *firsts = thresholds + pairs;
    int64_t *rounds = thresholds + 2 * pairs;
    int64_t *cheapest = thresholds + 3 * pairs;
    int64_t *banded = gpu->distances.ensure<int64_t>(size_t(pairs));
    uint32_t *pending = gpu->pending.ensure<uint32_t>(size_t(pairs));
    uint32_t *next = gpu->pending_next.ensure<uint32_t>(size_t(pairs));
    // counters: [0] pending, [1] next, [2..2+shapes) shape counts, then the swept words (64-bit).
    unsigned int *counters = gpu->counters.ensure<unsigned int>(64);
    unsigned long long *swept = reinterpret_cast<unsigned long long *>(counters + 32);
    DINARA_CUDA(cudaMemsetAsync(counters, 0, 64 * sizeof(unsigned int), stream));
    DINARA_CUDA(cudaMemsetAsync(rounds, 0, size_t(pairs) * sizeof(int64_t), stream));
    DINARA_CUDA(cudaMemsetAsync(cheapest, 0x7f, size_t(pairs) * sizeof(int64_t), stream));  // above any cost
    start_kernel<<<thread_blocks, threads, 0, stream>>>(info, pairs, first_thresholds_device,
                                                        default_start > 0 ? default_start : 256, status, thresholds,
                                                        firsts, pending, counters);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
    uint32_t *keys = gpu->keys.ensure<uint32_t>(size_t(pairs));
    uint32_t *keys_sorted = gpu->keys_sorted.ensure<uint32_t>(size_t(pairs));
    uint32_t *order_sorted = gpu->order_sorted.ensure<uint32_t>(size_t(pairs));
    unsigned int host_counts[2 + kBandShapes];
    read_back(gpu, host_counts, counters, sizeof(unsigned int));
    int64_t count = host_counts[0];
    int64_t launches = 0;
    float kernel_ms = 0.f;
    int64_t round = 0;
    int64_t round_pairs[16] = {0}, round_launches[16] = {0};
    double round_ms[16] = {0.0};
    while (count > 0) {
        const int64_t launches_before = launches;
        const int64_t round_count = count;
        // Order the round's pairs: by band shape, longest text first.
        DINARA_CUDA(cudaMemsetAsync(counters + 1, 0, (1 + kBandShapes) * sizeof(unsigned int), stream));
        const unsigned blocks = unsigned((count + threads - 1) / threads);
        // A round of few pairs takes the one-word-a-lane windows: lanes to spare, and the sweep's time is
        // its longest pair's chain of steps.
        const bool latency = count <= int64_t(gpu->multiprocessors) * 32;
        band_keys_kernel<<<blocks, threads, 0, stream>>>(info, pending, counters, thresholds, latency, keys,
                                                         counters + 2);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        size_t sort_bytes = 0;
        DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, keys, keys_sorted, pending,
                                                              order_sorted, int(count), 0, 32, stream));
        space = gpu->sort_scratch.ensure<uint8_t>(sort_bytes + 256);
        DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(space, sort_bytes, keys, keys_sorted, pending,
                                                              order_sorted, int(count), 0, 32, stream));
        read_back(gpu, host_counts, counters, (2 + kBandShapes) * sizeof(unsigned int));
        DINARA_CUDA(cudaEventRecord(gpu->start, stream));
        ClockSpan clock(gpu, kClassUnitBand, stream);
        // Each shape's launch on a side stream, all forked from and joined back to the context's stream:
        // a launch lasts as long as its longest pair, so running the shapes at once overlaps those tails.
        DINARA_CUDA(cudaEventRecord(gpu->fork, stream));
        bool used[dinara_gpu::kSideStreams] = {false};
        int next_side = 0;
        // Shapes in descending order, as the keys sort them.
        int64_t at = 0;
        for (int shape = kBandShapes - 1; shape >= 0; --shape) {
            const int64_t n_shape = host_counts[2 + shape];
            if (n_shape == 0) continue;
            BandArgs args;
            args.letters = letters;
            args.pairs = info;
            args.planes = planes;
            args.plane_offsets = plane_offsets;
            args.order = order_sorted;
            args.begin = uint32_t(at);
            args.end = uint32_t(at + n_shape);
            args.thresholds = thresholds;
            args.banded = banded;
            args.swept = swept;
            const int G = band_lanes(shape);
            const int groups_per_block = kBlock / G;
            BandFn fn = pick_band(shape);
            int per_sm = 0;
            DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
            int64_t grid = int64_t(std::max(per_sm, 1)) * gpu->multiprocessors;
            const int64_t needed = (n_shape + groups_per_block - 1) / groups_per_block;
            if (grid > needed) grid = needed;
            const int side = next_side;
            next_side = (next_side + 1) % dinara_gpu::kSideStreams;
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
        DINARA_CUDA(cudaMemsetAsync(counters + 1, 0, sizeof(unsigned int), stream));
        settle_kernel<<<blocks, threads, 0, stream>>>(info, order_sorted, counters, thresholds, cheapest, banded,
                                                      results, rounds, latency, next, counters + 1);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        DINARA_CUDA(cudaMemcpyAsync(counters, counters + 1, sizeof(unsigned int), cudaMemcpyDeviceToDevice, stream));
        read_back(gpu, host_counts, counters + 1, sizeof(unsigned int));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
        kernel_ms += ms;
        if (round < 16) {
            round_pairs[round] = round_count;
            round_launches[round] = launches - launches_before;
            round_ms[round] = ms;
        }
        ++round;
        count = host_counts[0];
        std::swap(pending, next);
    }
    if (report) {
        unsigned long long *tallies = swept + 1;
        DINARA_CUDA(cudaMemsetAsync(tallies, 0, 4 * sizeof(unsigned long long), stream));
        tally_kernel<<<thread_blocks, threads, 0, stream>>>(info, pairs, status, firsts, rounds, results, tallies);
        gpu->launches += 1;
        DINARA_CUDA(cudaGetLastError());
        unsigned long long host[5] = {0, 0, 0, 0, 0};
        read_back(gpu, host, swept, sizeof(host));
        report->rounds = launches;
        report->words_swept = int64_t(host[0]);
        report->pair_rounds = int64_t(host[1]);
        report->first_round_hits = int64_t(host[2]);
        report->overshoot = int64_t(host[3]);
        report->undershoot = int64_t(host[4]);
        report->kernel_ms = kernel_ms;
        for (int k = 0; k < 16; ++k) {
            report->round_pairs[k] = round_pairs[k];
            report->round_launches[k] = round_launches[k];
            report->round_ms[k] = round_ms[k];
        }
    }
}

}  // namespace dinara
