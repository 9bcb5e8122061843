// The learned band: a small network that reads a pair's k-mer sketch and predicts its edit distance, so
// band doubling starts near the answer instead of at the default threshold (band.mojo:521 starts an
// untrusted band 256 past what it knows). The network is 258 -> 64 -> 64 -> 1, fp32, ReLU: its input the
// 256 counts of each 4-mer in the reference less those in the query (squared, over the pair's mean
// length), the length ratio, and the 6-mer count differences' squares summed over the mean length; its
// output the distance over the mean length. Nothing about the answer depends on
// it: a low guess costs extra doublings, a high one a wider band, and the doubling that follows is the
// reference's.
//
// Everything runs on the device and is written here: a generator of training pairs (the benchmark's
// uneven distribution, from a counter-based hash so the lengths pass and the letters pass agree), their
// exact distances by the band kernels, the sketch, the training step (tiled fp32 products forward and
// back, Adam), and inference inside the scheduling kernel that sets each pair's first threshold.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "edit.cuh"
#include "learned.cuh"

namespace dinara {

namespace {

constexpr int kIn = kPredictorInputs, kH = kPredictorHidden;
// The parameters' room in the inference kernel's shared memory, rounded up to 4 floats.
constexpr int kParamsRoom = (kPredictorParameters + 3) & ~3;

// ------------------------------------------------------------------------------------------------
// Counter-based randomness
// ------------------------------------------------------------------------------------------------

__host__ __device__ inline uint64_t mix64(uint64_t x) {
    // SplitMix64's finalizer (Steele, Lea and Flood, 2014).
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__host__ __device__ inline uint64_t draw(uint64_t seed, uint64_t pair, uint64_t index) {
    return mix64(seed ^ mix64(pair * 0x9e3779b97f4a7c15ull + index * 0xd1b54a32d192ed03ull + 0x632be59bd9b4e019ull));
}

__host__ __device__ inline double unit(uint64_t h) { return double(h >> 11) * (1.0 / 9007199254740992.0); }

struct PairDraw {
    int64_t length;
    double rate;
};

// A pair's reference length (log-uniform) and error rate (uniform).
__device__ inline PairDraw pair_draw(uint64_t seed, uint64_t pair, double low, double high, double rate_low,
                                     double rate_high) {
    const double u = unit(draw(seed, pair, 0));
    const double v = unit(draw(seed, pair, 1));
    PairDraw d;
    d.length = int64_t(llround(exp(log(low) + u * (log(high) - log(low)))));
    d.rate = rate_low + v * (rate_high - rate_low);
    return d;
}

// Letter i's fate: 0 kept, 1 substituted, 2 deleted, 3 kept with a letter inserted after it (50/25/25).
__device__ inline int fate(uint64_t h, double rate) {
    const double roll = unit(h);
    if (roll < rate * 0.5) return 1;
    if (roll < rate * 0.75) return 2;
    if (roll < rate) return 3;
    return 0;
}

__global__ void generate_lengths_kernel(uint64_t seed, int64_t pairs, double low, double high, double rate_low,
                                        double rate_high, int64_t *lengths) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= pairs) return;
    const PairDraw d = pair_draw(seed, uint64_t(p), low, high, rate_low, rate_high);
    int64_t b = 0;
    for (int64_t i = 0; i < d.length; ++i) {
        const int f = fate(draw(seed, uint64_t(p), uint64_t(i) + 16), d.rate);
        b += f == 2 ? 0 : (f == 3 ? 2 : 1);
    }
    lengths[2 * p] = d.length;
    lengths[2 * p + 1] = b;
}

__global__ void generate_letters_kernel(uint64_t seed, int64_t pairs, double low, double high, double rate_low,
                                        double rate_high, const int64_t *offsets, uint8_t *letters) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= pairs) return;
    const PairDraw d = pair_draw(seed, uint64_t(p), low, high, rate_low, rate_high);
    const char *acgt = "ACGT";
    uint8_t *a = letters + offsets[2 * p];
    uint8_t *b = letters + offsets[2 * p + 1];
    int64_t at = 0;
    for (int64_t i = 0; i < d.length; ++i) {
        const uint64_t h = draw(seed, uint64_t(p), uint64_t(i) + 16);
        const uint32_t letter = uint32_t(h) & 3u;
        a[i] = uint8_t(acgt[letter]);
        const int f = fate(h, d.rate);
        if (f == 1) {
            b[at++] = uint8_t(acgt[(letter + 1 + (uint32_t(h >> 2) % 3u)) & 3u]);
        } else if (f == 0) {
            b[at++] = uint8_t(acgt[letter]);
        } else if (f == 3) {
            b[at++] = uint8_t(acgt[letter]);
            b[at++] = uint8_t(acgt[uint32_t(h >> 4) & 3u]);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// The sketch
// ------------------------------------------------------------------------------------------------

// A letter's 2-bit code (A 0, C 1, G 2, T 3), or -1 for any byte but those four: bits 1, 3, 7 and 20 of
// the mask stand for A, C, G and T (0x41, 0x43, 0x47, 0x54 less 0x40).
__device__ __forceinline__ int code_of(uint32_t byte) {
    const bool dna = (byte & 0xE0u) == 0x40u && ((0x0010008Au >> (byte & 31u)) & 1u);
    return dna ? int(((byte >> 1) & 3u) ^ ((byte >> 2) & 1u)) : -1;
}

// A 4-mer's count index: its letters' 2-bit codes, the first letter in the lowest bits.
// `reversed_kmer` maps between that and the features' order, the first letter in the highest bits.
__device__ __forceinline__ uint32_t reversed_kmer(uint32_t k) {
    return ((k & 3u) << 6) | (((k >> 2) & 3u) << 4) | (((k >> 4) & 3u) << 2) | ((k >> 6) & 3u);
}

// A warp's 6-mer counts of one sequence into `sixes` (shared, 4096 ints, a 6-mer's letters' 2-bit codes
// with the first letter in the lowest bits), `sign` +1 or -1; a 6-mer holding another letter is skipped.
// The 4-mer counts follow from them (a 4-mer is the first four letters of the 6-mer starting with it),
// save where a 4-mer starts no valid 6-mer (the sequence's last two 4-mers, or one whose fifth or sixth
// letter is another letter): those go into `fours` (256 ints, the same order) directly.
// Adds `sign` to 6-mer bin `bin`.
template <bool WIDE>
__device__ __forceinline__ void add_six(unsigned *sixes, uint32_t bin, int sign) {
    if (WIDE) {
        atomicAdd(&sixes[bin], unsigned(sign));
        return;
    }
    // Two 16-bit bins a word, each held as 32,768 plus its count difference. Neither sequence has more
    // than kNarrowLimit letters, so in whatever order they are added no half passes 65,535 or falls below
    // zero, and no add reaches the other half.
    atomicAdd(&sixes[bin >> 1], unsigned(sign) << (16 * (bin & 1u)));
}

template <bool WIDE>
__device__ __forceinline__ int six_at(const unsigned *sixes, uint32_t bin) {
    if (WIDE) return int(sixes[bin]);
    return int((sixes[bin >> 1] >> (16 * (bin & 1u))) & 0xFFFFu) - 32768;
}

// The seven aligned words holding a slot's 16 letters and the five after them (a word may reach three
// bytes past the sequence's end: device letter buffers keep 16 bytes of room there); loaded apart from
// their use so that a lane keeps two slots' loads in flight.
__device__ __forceinline__ void load_slot(const uint8_t *sequence, int64_t length, int64_t slot, uint32_t w[7]) {
    const uintptr_t origin = reinterpret_cast<uintptr_t>(sequence);
    const uintptr_t end = origin + uintptr_t(length);
    const uintptr_t aligned = (origin + uintptr_t(16 * slot)) & ~uintptr_t(3);
    const uint32_t *words = reinterpret_cast<const uint32_t *>(aligned);
#pragma unroll
    for (int i = 0; i < 7; ++i) w[i] = aligned + 4 * uintptr_t(i) < end ? __ldg(words + i) : 0u;
}

// One slot of 16 letters: the 6-mers starting at letters 16 slot .. 16 slot + 15, from its loaded words.
template <bool WIDE>
__device__ void count_kmers(const uint8_t *sequence, int64_t length, int sign, unsigned *sixes, int *fours,
                            int64_t slot, const uint32_t w[7]) {
    {
        const int64_t first = 16 * slot;
        const uintptr_t address = reinterpret_cast<uintptr_t>(sequence) + uintptr_t(first);
        const uint32_t shift = uint32_t(address & 3u) * 8u;
        uint32_t a[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) a[i] = __funnelshift_r(w[i], w[i + 1], shift);
        if (first + 21 <= length) {
            // The lane's 21 letters, four a word at once: each byte's 2-bit code, the letters rebuilt from
            // the codes (A, C, G, T by a byte permute) to check that every byte was one of the four, and
            // the codes packed two bits a letter, the first letter lowest.
            bool valid = true;
            uint64_t packed = 0;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const uint32_t c = ((a[q] >> 1) & 0x03030303u) ^ ((a[q] >> 2) & 0x01010101u);
                const uint32_t t = c | (c >> 4);
                const uint32_t rebuilt = __byte_perm(0x54474341u, 0u, (t & 0xFFu) | ((t >> 8) & 0xFF00u));
                const uint32_t used = q < 5 ? 0xFFFFFFFFu : 0x000000FFu;  // 16 + 5 letters
                valid = valid && ((rebuilt ^ a[q]) & used) == 0u;
                const uint32_t x = c | (c >> 6);
                packed |= uint64_t((x & 0xFu) | ((x >> 12) & 0xF0u)) << (8 * q);
            }
            if (valid) {
#pragma unroll
                for (int j = 0; j < 16; ++j) add_six<WIDE>(sixes, uint32_t(packed >> (2 * j)) & 0xFFFu, sign);
                return;
            }
        }
        // Near the sequence's end or another letter in reach (rare): start by start, letter by letter, in a
        // loop kept rolled so the kernel's body stays in the instruction cache. The 6-mer starting at each
        // of the slot's places, or failing it the 4-mer.
#pragma unroll 1
        for (int j = 0; j < 16; ++j) {
            const int64_t place = first + j;
            if (place + 4 > length) break;
            uint32_t kmer = 0;
            int valid = 0;
#pragma unroll 1
            for (int q = 0; q < 6 && place + q < length; ++q) {
                const int c = code_of(__ldg(sequence + place + q));
                if (c < 0) break;
                kmer |= uint32_t(c) << (2 * q);
                ++valid;
            }
            if (valid == 6)
                add_six<WIDE>(sixes, kmer, sign);
            else if (valid >= 4)
                atomicAdd(&fours[kmer & 0xFFu], sign);
        }
    }
}

// Writes a pair's 258 features, scaled as the network reads them. The first 256: each 4-mer count
// difference squared, times 32 over the mean length, since an error moves a handful of 4-mers between
// bins and the squares of the differences then sum to about eight times the errors whether a bin holds
// one move or many of either sign, so their sum over the length tracks the error rate. Then the length
// ratio. Then the 6-mer count differences' squares summed over their 4,096 bins, over the mean length:
// the same measure with sixteen times the bins, whose noise from moves sharing a bin is a quarter of
// the 4-mers' (about 3.6% against 11% of a 4 kbp pair's distance).
//
// One pass over the counts does it all, and leaves them cleared for the warp's next pair: a lane reads
// the words lane, lane + 32, ... of the 6-mer bins, whose 4-mers (a bin's low eight bits) are eight fixed
// ones per lane, so the 4-mer counts build up in eight registers while the squares are summed.
template <bool WIDE>
__device__ void features_of(unsigned *sixes, int *fours, int64_t reference, int64_t query, float *out, int stride) {
    const int lane = threadIdx.x & 31;
    const float mean = 0.5f * float(reference + query);
    const float scale = 32.0f / (mean > 1.0f ? mean : 1.0f);
    int sums[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long squares = 0;
    if (WIDE) {
        // Word w is bin w; bin lane + 32 i has 4-mer lane + 32 (i mod 8).
#pragma unroll 8
        for (int i = 0; i < 128; ++i) {
            const int v = int(sixes[lane + 32 * i]);
            sixes[lane + 32 * i] = 0u;
            squares += (long long)v * v;
            sums[i & 7] += v;
        }
    } else {
        // Word w holds bins 2w and 2w + 1; for w = lane + 32 i their 4-mers are 2 lane + 64 (i mod 4) and
        // one more.
#pragma unroll 4
        for (int i = 0; i < 64; ++i) {
            const unsigned word = sixes[lane + 32 * i];
            sixes[lane + 32 * i] = 0x80008000u;
            const int low = int(word & 0xFFFFu) - 32768, high = int(word >> 16) - 32768;
            squares += (long long)low * low + (long long)high * high;
            sums[2 * (i & 3)] += low;
            sums[2 * (i & 3) + 1] += high;
        }
    }
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const uint32_t four = WIDE ? uint32_t(lane + 32 * s) : uint32_t(2 * lane + (s & 1) + 64 * (s >> 1));
        const float difference = float(sums[s] + fours[four]);
        fours[four] = 0;
        // Feature k's 4-mer has its first letter in the highest bits; the counts, in the lowest.
        out[int64_t(reversed_kmer(four)) * stride] = difference * difference * scale;
    }
#pragma unroll
    for (int span = 16; span > 0; span >>= 1) squares += __shfl_xor_sync(0xffffffffu, squares, span);
    if (lane == 0) {
        const int64_t low = min(reference, query), high = max(reference, query);
        out[int64_t(256) * stride] = high > 0 ? float(low) / float(high) : 1.0f;
        out[int64_t(257) * stride] = float(double(squares) / double(mean > 1.0f ? mean : 1.0f));
    }
}

// The sketch kernel's warps each take one pair at a time from a queue, its counts in the warp's own
// shared memory: 4,096 6-mer bins (two 16-bit bins a word, or a word each for pairs with a side past
// kNarrowLimit letters) and 256 4-mer ints. No warp waits for another, so a long pair holds up nothing.
constexpr int kSketchWarps = 4;
constexpr int kSketchNarrowWords = 2048 + 256;
constexpr int kSketchWideWords = 4096 + 256;
constexpr int64_t kNarrowLimit = 32000;

template <bool WIDE>
constexpr size_t sketch_shared_bytes() {
    return size_t(kSketchWarps) * size_t(WIDE ? kSketchWideWords : kSketchNarrowWords) * sizeof(unsigned);
}

// Persistent warps, each taking its next pair from a queue: pair `order[item]` (or pair item itself with
// no order). The features into a matrix, feature f of pair p at f * pairs + p (feature-major, as training
// reads them) or at p * kIn + f (pair-major, as prediction does). The narrow form skips pairs with a side
// past kNarrowLimit letters, which the wide form takes.
template <bool WIDE>
__global__ void __launch_bounds__(32 * kSketchWarps) features_kernel(const uint8_t *letters, const int64_t *offsets,
                                                                      int64_t pairs, const uint32_t *order,
                                                                      int64_t count, unsigned *queue, float *features,
                                                                      bool pair_major) {
    extern __shared__ unsigned sketch_counts[];
    constexpr int kWords = WIDE ? kSketchWideWords : kSketchNarrowWords;
    const int lane = threadIdx.x & 31;
    unsigned *sixes = sketch_counts + (threadIdx.x >> 5) * kWords;
    int *fours = reinterpret_cast<int *>(sixes + (WIDE ? 4096 : 2048));
    // Cleared once here; each pair's features clear what its counts used.
    for (int k = lane; k < kWords; k += 32) sixes[k] = (WIDE || k >= 2048) ? 0u : 0x80008000u;
    __syncwarp();
    for (;;) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= count) return;
        const int64_t pair = order ? int64_t(order[item]) : int64_t(item);
        const int64_t r0 = offsets[2 * pair], q0 = offsets[2 * pair + 1], q1 = offsets[2 * pair + 2];
        const int64_t reference = q0 - r0, query = q1 - q0;
        if (!WIDE && (reference > kNarrowLimit || query > kNarrowLimit)) continue;  // the wide form's
        // Both sequences' 16-letter slots in one run, the reference's (+1) then the query's (-1), two slots
        // a lane at a time: both slots' words are loaded before either is counted.
        const int64_t reference_slots = (reference + 15) / 16, slots = reference_slots + (query + 15) / 16;
        for (int64_t slot = lane; slot < slots; slot += 64) {
            const int64_t other = slot + 32;
            const bool first_ref = slot < reference_slots, other_ref = other < reference_slots;
            uint32_t w0[7], w1[7];
            load_slot(first_ref ? letters + r0 : letters + q0, first_ref ? reference : query,
                      first_ref ? slot : slot - reference_slots, w0);
            if (other < slots)
                load_slot(other_ref ? letters + r0 : letters + q0, other_ref ? reference : query,
                          other_ref ? other : other - reference_slots, w1);
            count_kmers<WIDE>(first_ref ? letters + r0 : letters + q0, first_ref ? reference : query, first_ref ? 1 : -1,
                              sixes, fours, first_ref ? slot : slot - reference_slots, w0);
            if (other < slots)
                count_kmers<WIDE>(other_ref ? letters + r0 : letters + q0, other_ref ? reference : query,
                                  other_ref ? 1 : -1, sixes, fours, other_ref ? other : other - reference_slots, w1);
        }
        __syncwarp();
        features_of<WIDE>(sixes, fours, reference, query, pair_major ? features + pair * kIn : features + pair,
                          pair_major ? 1 : int(pairs));
        __syncwarp();
    }
}

// The pairs with a side past kNarrowLimit letters, for the wide form.
__global__ void wide_pairs_kernel(const int64_t *offsets, int64_t pairs, uint32_t *wide, unsigned *count) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= pairs) return;
    if (offsets[2 * p + 1] - offsets[2 * p] > kNarrowLimit || offsets[2 * p + 2] - offsets[2 * p + 1] > kNarrowLimit)
        wide[atomicAdd(count, 1u)] = uint32_t(p);
}

void launch_features(dinara_gpu *gpu, const uint8_t *letters, const int64_t *offsets, int64_t pairs, float *features,
                     bool pair_major) {
    cudaStream_t stream = gpu->stream;
    unsigned *counts = reinterpret_cast<unsigned *>(gpu->counters.ensure<unsigned int>(64) + 56);  // [0] wide, [1..2] queues
    DINARA_CUDA(cudaMemsetAsync(counts, 0, 3 * sizeof(unsigned), stream));
    int per_sm = 0;
    DINARA_CUDA(cudaFuncSetAttribute(features_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(sketch_shared_bytes<false>())));
    DINARA_CUDA(cudaFuncSetAttribute(features_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(sketch_shared_bytes<true>())));
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, features_kernel<false>, 32 * kSketchWarps,
                                                              sketch_shared_bytes<false>()));
    int64_t blocks = std::min<int64_t>(int64_t(std::max(per_sm, 1)) * gpu->multiprocessors,
                                       (pairs + kSketchWarps - 1) / kSketchWarps);
    features_kernel<false><<<unsigned(std::max<int64_t>(blocks, 1)), 32 * kSketchWarps, sketch_shared_bytes<false>(),
                             stream>>>(letters, offsets, pairs, nullptr, pairs, counts + 1, features, pair_major);
    DINARA_CUDA(cudaGetLastError());
    // The few pairs past the narrow bins' reach, again with a word a bin.
    uint32_t *wide = gpu->keys.ensure<uint32_t>(size_t(pairs) + 1);
    wide_pairs_kernel<<<unsigned((pairs + 255) / 256), 256, 0, stream>>>(offsets, pairs, wide, counts);
    DINARA_CUDA(cudaGetLastError());
    unsigned wide_count = 0;
    read_back(gpu, &wide_count, counts, sizeof wide_count);
    if (wide_count > 0) {
        DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, features_kernel<true>, 32 * kSketchWarps,
                                                                  sketch_shared_bytes<true>()));
        blocks = std::min<int64_t>(int64_t(std::max(per_sm, 1)) * gpu->multiprocessors,
                                   (int64_t(wide_count) + kSketchWarps - 1) / kSketchWarps);
        features_kernel<true><<<unsigned(std::max<int64_t>(blocks, 1)), 32 * kSketchWarps, sketch_shared_bytes<true>(),
                                stream>>>(letters, offsets, pairs, wide, wide_count, counts + 2, features, pair_major);
        DINARA_CUDA(cudaGetLastError());
    }
}

// ------------------------------------------------------------------------------------------------
// Training: tiled fp32 products
// ------------------------------------------------------------------------------------------------

// C[m x n] (+)= op(A)[m x k] * op(B)[k x n], all row-major with leading dimensions; op transposes when
// asked. A 64 x 64 tile a block of 256 threads, 4 x 4 outputs a thread, k in steps of 16 through shared
// memory. `accumulate` adds to C; `bias` (length m) and `relu` finish the tile when given.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) product_kernel(int m, int n, int k, const float *A, int lda, const float *B,
                                                      int ldb, float *C, int ldc, const float *bias, bool relu,
                                                      bool accumulate) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int row0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
    float acc[4][4] = {{0.f}};
    for (int kk = 0; kk < k; kk += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int kq = e / 64, i = e % 64;
            const int r = row0 + i, kc = kk + kq;
            float a = 0.f;
            if (r < m && kc < k) a = TA ? A[int64_t(kc) * lda + r] : A[int64_t(r) * lda + kc];
            As[kq][i] = a;
            const int c = col0 + i;
            float bv = 0.f;
            if (c < n && kc < k) bv = TB ? B[int64_t(c) * ldb + kc] : B[int64_t(kc) * ldb + c];
            Bs[kq][i] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[q][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[q][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty * 4 + i;
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx * 4 + j;
            if (c >= n) continue;
            float v = acc[i][j];
            if (accumulate) v += C[int64_t(r) * ldc + c];
            if (bias) v += bias[r];
            if (relu) v = fmaxf(v, 0.f);
            C[int64_t(r) * ldc + c] = v;
        }
    }
}

template <bool TA, bool TB>
void product(cudaStream_t stream, int m, int n, int k, const float *A, int lda, const float *B, int ldb, float *C,
             int ldc, const float *bias = nullptr, bool relu = false, bool accumulate = false) {
    dim3 grid(unsigned((n + 63) / 64), unsigned((m + 63) / 64));
    product_kernel<TA, TB><<<grid, 256, 0, stream>>>(m, n, k, A, lda, B, ldb, C, ldc, bias, relu, accumulate);
    DINARA_CUDA(cudaGetLastError());
}

// The output layer and the loss: y = w3 . h2 + b3 for each sample; dy = 2 (y - target) / batch, and
// the summed squared error into `loss`.
__global__ void output_kernel(const float *h2, int batch, const float *w3, const float *b3, const float *targets,
                              float *y, float *dy, float *loss) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= batch) return;
    float v = b3[0];
    for (int j = 0; j < kH; ++j) v = fmaf(w3[j], h2[int64_t(j) * batch + s], v);
    y[s] = v;
    if (targets) {
        const float e = v - targets[s];
        dy[s] = 2.f * e / float(batch);
        atomicAdd(loss, e * e);
    }
}

// dH2 = w3 dy masked by h2 > 0; db3 = sum dy; dw3 = sum dy h2.
__global__ void output_backward_kernel(const float *h2, const float *dy, int batch, const float *w3, float *dh2,
                                       float *dw3, float *db3) {
    const int j = blockIdx.x;  // a hidden unit a block
    float sum = 0.f, dsum = 0.f;
    for (int s = threadIdx.x; s < batch; s += blockDim.x) {
        const float h = h2[int64_t(j) * batch + s];
        dh2[int64_t(j) * batch + s] = h > 0.f ? w3[j] * dy[s] : 0.f;
        sum += dy[s] * h;
        if (j == 0) dsum += dy[s];
    }
    __shared__ float part[2][256];
    part[0][threadIdx.x] = sum;
    part[1][threadIdx.x] = dsum;
    __syncthreads();
    for (int span = blockDim.x / 2; span > 0; span >>= 1) {
        if (threadIdx.x < span) {
            part[0][threadIdx.x] += part[0][threadIdx.x + span];
            part[1][threadIdx.x] += part[1][threadIdx.x + span];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        dw3[j] = part[0][0];
        if (j == 0) db3[0] = part[1][0];
    }
}

// Masks dH by H > 0 in place, and sums each row into `dbias`.
__global__ void relu_backward_kernel(const float *h, float *dh, int batch, float *dbias) {
    const int j = blockIdx.x;
    float sum = 0.f;
    for (int s = threadIdx.x; s < batch; s += blockDim.x) {
        const int64_t at = int64_t(j) * batch + s;
        const float g = h[at] > 0.f ? dh[at] : 0.f;
        dh[at] = g;
        sum += g;
    }
    __shared__ float part[256];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int span = blockDim.x / 2; span > 0; span >>= 1) {
        if (threadIdx.x < span) part[threadIdx.x] += part[threadIdx.x + span];
        __syncthreads();
    }
    if (threadIdx.x == 0) dbias[j] = part[0];
}

// Adam (Kingma and Ba, 2015) over every parameter.
__global__ void adam_kernel(float *params, const float *grads, float *m, float *v, int count, float rate, float beta1,
                            float beta2, float eps, float correction1, float correction2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= rate * (mi / correction1) / (sqrtf(vi / correction2) + eps);
}

// ------------------------------------------------------------------------------------------------
// Inference inside the scheduling kernel
// ------------------------------------------------------------------------------------------------

// A warp a pair: the sketch, the network with every weight in shared memory, and the first threshold:
// the predicted distance widened by the margin and the slack, never below the length difference.
struct Margins {
    float by_length[4];  // mean length < 300, < 1000, < 4096, longer
};

__device__ __host__ inline int length_class(double mean) { return mean < 300 ? 0 : mean < 1000 ? 1 : mean < 4096 ? 2 : 3; }

// Pairs a warp takes at once: each weight it reads from shared memory serves all of them.
constexpr int kPredictPairs = 4;

__global__ void __launch_bounds__(256) predict_kernel(const float *features, const int64_t *offsets, int64_t pairs,
                                                      const float *params, Margins margins, float slack,
                                                      int64_t *thresholds, float *predicted) {
    extern __shared__ float shared[];
    float *w1 = shared;                 // [kIn][kH]
    float *b1 = w1 + kIn * kH;
    float *w2 = b1 + kH;                // [kH][kH]
    float *b2 = w2 + kH * kH;
    float *w3 = b2 + kH;
    float *b3 = w3 + kH;
    // Each warp's inputs, kPredictPairs rows of 260 (kIn and padding), then its first layer's outputs.
    float *inputs = shared + kParamsRoom;
    for (int i = threadIdx.x; i < kPredictorParameters; i += blockDim.x) shared[i] = params[i];
    const int warp_in_block = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *x = inputs + warp_in_block * kPredictPairs * (260 + kH);
    float *hidden = x + kPredictPairs * 260;
    __syncthreads();
    const int64_t stride = int64_t(gridDim.x) * 8 * kPredictPairs;
    for (int64_t first = (int64_t(blockIdx.x) * 8 + warp_in_block) * kPredictPairs; first < pairs; first += stride) {
        const int count = int(pairs - first < kPredictPairs ? pairs - first : kPredictPairs);
        for (int q = 0; q < kPredictPairs; ++q)
            for (int i = lane; i < kIn; i += 32) x[q * 260 + i] = q < count ? __ldg(features + (first + q) * kIn + i) : 0.f;
        __syncwarp();
        // Hidden layers: lane j computes units j and j + 32 of every pair.
        float h[kPredictPairs][2];
#pragma unroll
        for (int q = 0; q < kPredictPairs; ++q) {
            h[q][0] = b1[lane];
            h[q][1] = b1[lane + 32];
        }
        for (int i = 0; i < kIn; ++i) {
            const float wa = w1[i * kH + lane], wb = w1[i * kH + lane + 32];
#pragma unroll
            for (int q = 0; q < kPredictPairs; ++q) {
                const float xi = x[q * 260 + i];
                h[q][0] = fmaf(xi, wa, h[q][0]);
                h[q][1] = fmaf(xi, wb, h[q][1]);
            }
        }
#pragma unroll
        for (int q = 0; q < kPredictPairs; ++q) {
            hidden[q * kH + lane] = fmaxf(h[q][0], 0.f);
            hidden[q * kH + lane + 32] = fmaxf(h[q][1], 0.f);
        }
        __syncwarp();
        float g[kPredictPairs][2];
#pragma unroll
        for (int q = 0; q < kPredictPairs; ++q) {
            g[q][0] = b2[lane];
            g[q][1] = b2[lane + 32];
        }
        for (int i = 0; i < kH; ++i) {
            const float wa = w2[i * kH + lane], wb = w2[i * kH + lane + 32];
#pragma unroll
            for (int q = 0; q < kPredictPairs; ++q) {
                const float hi = hidden[q * kH + i];
                g[q][0] = fmaf(hi, wa, g[q][0]);
                g[q][1] = fmaf(hi, wb, g[q][1]);
            }
        }
#pragma unroll
        for (int q = 0; q < kPredictPairs; ++q) {
            float y = fmaxf(g[q][0], 0.f) * w3[lane] + fmaxf(g[q][1], 0.f) * w3[lane + 32];
#pragma unroll
            for (int span = 16; span > 0; span >>= 1) y += __shfl_xor_sync(0xffffffffu, y, span);
            y += b3[0];
            if (lane == 0 && q < count) {
                const int64_t pair = first + q;
                const int64_t r0 = offsets[2 * pair], q0 = offsets[2 * pair + 1], q1 = offsets[2 * pair + 2];
                const int64_t n = q0 - r0, m = q1 - q0;
                const double mean = 0.5 * double(n + m);
                const double guess = fmax(0.0, double(y)) * mean;
                const int64_t delta = n > m ? n - m : m - n;
                const double margin = double(margins.by_length[length_class(mean)]);
                int64_t t = int64_t(ceil(guess * margin + double(slack)));
                if (t < delta) t = delta;
                if (t < 1) t = 1;
                thresholds[pair] = t;
                if (predicted) predicted[pair] = float(guess);
            }
        }
        __syncwarp();
    }
}

size_t predict_shared_bytes() { return size_t(kParamsRoom + 8 * kPredictPairs * (260 + kH)) * sizeof(float); }

// Parameter offsets in the flat vector: w1 [kIn][kH], b1, w2 [kH][kH], b2, w3, b3.
constexpr int kW1 = 0, kB1 = kW1 + kIn * kH, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH, kB3 = kW3 + kH;

// One training step's forward and backward over `batch` samples whose features are the columns of X
// (feature-major, leading dimension ldx): gradients into `grads` (flat, like the parameters), the
// squared error summed into `loss`.
void forward_backward(cudaStream_t stream, const float *params, const float *X, int ldx, const float *targets,
                      int batch, float *work, float *grads, float *loss) {
    float *h1 = work, *h2 = h1 + int64_t(kH) * batch, *y = h2 + int64_t(kH) * batch, *dy = y + batch;
    float *dh2 = dy + batch, *dh1 = dh2 + int64_t(kH) * batch;
    // h1 = relu(W1^T X + b1): [kH x batch]; W1 is [kIn x kH] row-major, so op(A) = W1^T.
    product<true, false>(stream, kH, batch, kIn, params + kW1, kH, X, ldx, h1, batch, params + kB1, true);
    product<true, false>(stream, kH, batch, kH, params + kW2, kH, h1, batch, h2, batch, params + kB2, true);
    output_kernel<<<(batch + 255) / 256, 256, 0, stream>>>(h2, batch, params + kW3, params + kB3, targets, y, dy, loss);
    DINARA_CUDA(cudaGetLastError());
    output_backward_kernel<<<kH, 256, 0, stream>>>(h2, dy, batch, params + kW3, dh2, grads + kW3, grads + kB3);
    DINARA_CUDA(cudaGetLastError());
    // dW2[i][j] = sum_s h1[i][s] dh2[j][s]: [kH x kH] = h1 [kH x batch] * dh2^T.
    product<false, true>(stream, kH, kH, batch, h1, batch, dh2, batch, grads + kW2, kH);
    // db2: the rows of dh2.
    relu_backward_kernel<<<kH, 256, 0, stream>>>(h2, dh2, batch, grads + kB2);
    DINARA_CUDA(cudaGetLastError());
    // dh1 = W2 dh2: [kH x batch] = W2 [kH x kH] * dh2, then masked by h1 > 0 with db1 its row sums.
    product<false, false>(stream, kH, batch, kH, params + kW2, kH, dh2, batch, dh1, batch);
    relu_backward_kernel<<<kH, 256, 0, stream>>>(h1, dh1, batch, grads + kB1);
    DINARA_CUDA(cudaGetLastError());
    // dW1[i][j] = sum_s X[i][s] dh1[j][s]: [kIn x kH].
    product<false, true>(stream, kIn, kH, batch, X, ldx, dh1, batch, grads + kW1, kH);
}

size_t work_floats(int batch) { return size_t(batch) * (4 * kH + 2) + 64; }

}  // namespace

// ------------------------------------------------------------------------------------------------
// Entry points used by capi.cu
// ------------------------------------------------------------------------------------------------

void predictor_features(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                        float *features) {
    launch_features(gpu, letters, offsets, pairs, features, false);
    gpu->launches += 2;
}

void predictor_gradients(dinara_gpu *gpu, int batch, const float *features, const float *targets, float *grads,
                         float *loss) {
    float *params = gpu->weights.as<float>();
    float *work = gpu->activations.ensure<float>(work_floats(batch));
    DINARA_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), gpu->stream));
    forward_backward(gpu->stream, params, features, batch, targets, batch, work, grads, loss);
}

const int64_t *predict_thresholds(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets) {
    if (!gpu->predictor_ready) throw Failure(DINARA_INVALID_MODE, "no trained band predictor on this context");
    int64_t *thresholds = gpu->predictions.ensure<int64_t>(size_t(pairs));
    float *predicted = gpu->targets.ensure<float>(size_t(pairs));
    const size_t shared = predict_shared_bytes();
    DINARA_CUDA(cudaFuncSetAttribute(predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shared)));
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, predict_kernel, 256, shared));
    int64_t blocks = int64_t(std::max(per_sm, 1)) * gpu->multiprocessors;
    blocks = std::min<int64_t>(blocks, (pairs + 8 * kPredictPairs - 1) / (8 * kPredictPairs));
    Margins margins;
    for (int k = 0; k < 4; ++k) margins.by_length[k] = float(gpu->predictor_margins[k]);
    // The sketches first, a warp a pair at full occupancy (reading the letters is the slow part), then the
    // network from them with its weights in shared memory.
    float *sketches = gpu->sketches.ensure<float>(size_t(pairs) * kIn);
    launch_features(gpu, letters, offsets, pairs, sketches, true);
    gpu->launches += 2;
    predict_kernel<<<unsigned(std::max<int64_t>(blocks, 1)), 256, shared, gpu->stream>>>(
        sketches, offsets, pairs, gpu->weights.as<float>(), margins, float(gpu->predictor_slack), thresholds, predicted);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    return thresholds;
}

GeneratedPairs generate_pairs(dinara_gpu *gpu, uint64_t seed, int64_t pairs, double length_low, double length_high,
                              double rate_low, double rate_high) {
    cudaStream_t stream = gpu->stream;
    // Lengths first (each pair's letters' fates decide the query's), then offsets, then the letters.
    int64_t *lengths = gpu->thresholds.ensure<int64_t>(size_t(2 * pairs + 1));
    const int threads = 256;
    const unsigned pair_blocks = unsigned((pairs + threads - 1) / threads);
    generate_lengths_kernel<<<pair_blocks, threads, 0, stream>>>(seed, pairs, length_low, length_high, rate_low,
                                                                 rate_high, lengths);
    DINARA_CUDA(cudaGetLastError());
    GeneratedPairs out;
    out.offsets = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
    DINARA_CUDA(cudaMemsetAsync(lengths + 2 * pairs, 0, sizeof(int64_t), stream));
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, lengths, out.offsets, int(2 * pairs + 1), stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(scratch + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, lengths, out.offsets, int(2 * pairs + 1), stream));
    read_back(gpu, &out.letters_total, out.offsets + 2 * pairs, sizeof(int64_t));
    out.letters = gpu->letters.ensure<uint8_t>(size_t(out.letters_total) + 16);
    generate_letters_kernel<<<pair_blocks, threads, 0, stream>>>(seed, pairs, length_low, length_high, rate_low,
                                                                 rate_high, out.offsets, out.letters);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 2;
    return out;
}

void predictor_train(dinara_gpu *gpu, const dinara_train_options &options, dinara_train_report &report) {
    cudaStream_t stream = gpu->stream;
    const int64_t pairs = options.pairs;
    // The training pairs: lengths, offsets, letters, all on the device.
    const GeneratedPairs generated = generate_pairs(gpu, options.seed, pairs, options.length_low, options.length_high,
                                                    options.rate_low, options.rate_high);
    int64_t *offsets = generated.offsets;
    uint8_t *letters = generated.letters;
    // Their exact distances: the method's own, plain band doubling.
    int64_t *distances = gpu->features.ensure<int64_t>(size_t(pairs));
    band_doubling(gpu, pairs, letters, offsets, nullptr, 0, distances, nullptr);
    // Targets (distance over mean length) and features.
    std::vector<int64_t> host_distances(static_cast<size_t>(pairs)), host_offsets(size_t(2 * pairs + 1));
    DINARA_CUDA(cudaMemcpyAsync(host_distances.data(), distances, size_t(pairs) * sizeof(int64_t),
                                cudaMemcpyDeviceToHost, stream));
    DINARA_CUDA(cudaMemcpyAsync(host_offsets.data(), offsets, host_offsets.size() * sizeof(int64_t),
                                cudaMemcpyDeviceToHost, stream));
    DINARA_CUDA(cudaStreamSynchronize(stream));
    std::vector<float> host_targets(static_cast<size_t>(pairs));
    for (int64_t p = 0; p < pairs; ++p) {
        const double mean = 0.5 * double(host_offsets[size_t(2 * p + 2)] - host_offsets[size_t(2 * p)]);
        host_targets[size_t(p)] = mean > 0 ? float(double(host_distances[size_t(p)]) / mean) : 0.f;
    }
    float *targets = gpu->targets.ensure<float>(size_t(pairs));
    DINARA_CUDA(cudaMemcpyAsync(targets, host_targets.data(), size_t(pairs) * sizeof(float), cudaMemcpyHostToDevice,
                                stream));
    // The features, feature-major, into gpu->gradients' room after the parameters' gradients.
    float *features = gpu->planes.ensure<float>(size_t(pairs) * kIn);
    predictor_features(gpu, pairs, letters, offsets, features);

    // Parameters: He initialisation from the seed, biases zero; Adam's moments zero.
    std::vector<float> init(kPredictorParameters, 0.f);
    uint64_t state = options.seed ^ 0x5bd1e995u;
    auto gaussian = [&]() {
        const double u1 = std::max(1e-12, unit(mix64(++state)));
        const double u2 = unit(mix64(++state));
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (int i = 0; i < kIn * kH; ++i) init[size_t(kW1 + i)] = float(gaussian() * std::sqrt(2.0 / kIn));
    for (int i = 0; i < kH * kH; ++i) init[size_t(kW2 + i)] = float(gaussian() * std::sqrt(2.0 / kH));
    for (int i = 0; i < kH; ++i) init[size_t(kW3 + i)] = float(gaussian() * std::sqrt(1.0 / kH));
    float *params = gpu->weights.ensure<float>(kPredictorParameters);
    float *grads = gpu->gradients.ensure<float>(kPredictorParameters);
    float *moments = gpu->optimizer.ensure<float>(2 * kPredictorParameters);
    DINARA_CUDA(cudaMemcpyAsync(params, init.data(), init.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
    DINARA_CUDA(cudaMemsetAsync(moments, 0, 2 * kPredictorParameters * sizeof(float), stream));
    const int batch = int(options.batch);
    float *work = gpu->activations.ensure<float>(work_floats(batch));
    float *loss = work + work_floats(batch) - 8;
    // The last tenth of the pairs is held out for validation.
    const int64_t held = std::max<int64_t>(pairs / 10, 1);
    const int64_t trained = pairs - held;
    int64_t step = 0;
    double last_loss = 0.0;
    for (int64_t epoch = 0; epoch < options.epochs; ++epoch) {
        double epoch_loss = 0.0;
        int64_t batches = 0;
        for (int64_t first = 0; first + batch <= trained; first += batch) {
            DINARA_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), stream));
            forward_backward(stream, params, features + first, int(pairs), targets + first, batch, work, grads, loss);
            ++step;
            const float beta1 = 0.9f, beta2 = 0.999f;
            adam_kernel<<<(kPredictorParameters + 255) / 256, 256, 0, stream>>>(
                params, grads, moments, moments + kPredictorParameters, kPredictorParameters, float(options.learning_rate),
                beta1, beta2, 1e-8f, 1.f - std::pow(beta1, float(step)), 1.f - std::pow(beta2, float(step)));
            DINARA_CUDA(cudaGetLastError());
            if ((batches & 63) == 63 || first + 2 * batch > trained) {
                float host_loss = 0.f;
                DINARA_CUDA(cudaMemcpyAsync(&host_loss, loss, sizeof host_loss, cudaMemcpyDeviceToHost, stream));
                DINARA_CUDA(cudaStreamSynchronize(stream));
                epoch_loss = host_loss / batch;
            }
            ++batches;
        }
        last_loss = epoch_loss;
    }
    report.steps = step;
    report.train_loss = last_loss;
    // Validation: predicted distances on the held-out pairs, and the margin that covers the asked share
    // of them (a first threshold at or above the distance).
    gpu->predictor_ready = true;
    for (int k = 0; k < 4; ++k) gpu->predictor_margins[k] = 1.0;
    gpu->predictor_slack = 0.0;
    int64_t *held_offsets = gpu->pending.ensure<int64_t>(size_t(2 * held + 1));
    std::vector<int64_t> rebased(size_t(2 * held + 1));
    for (int64_t k = 0; k <= 2 * held; ++k) rebased[size_t(k)] = host_offsets[size_t(2 * trained + k)];
    DINARA_CUDA(cudaMemcpyAsync(held_offsets, rebased.data(), rebased.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                stream));
    predict_thresholds(gpu, held, letters, held_offsets);
    std::vector<float> guesses(static_cast<size_t>(held));
    DINARA_CUDA(cudaMemcpyAsync(guesses.data(), gpu->targets.as<float>(), size_t(held) * sizeof(float),
                                cudaMemcpyDeviceToHost, stream));
    DINARA_CUDA(cudaStreamSynchronize(stream));
    // A class's margin is the least that settles a share of its held-out pairs in their first round: a
    // pair settles when its distance lies within the band its first window sweeps (band_reach: a window
    // holds a wider band than the threshold needs, for nothing), with the window the first round would
    // give it under the context's tuning. A pair that misses sweeps again, and the round it adds lasts as
    // long as its longest pair's chain of word steps, so the longer classes are held to a higher share: of
    // the asked coverage's misses, all for pairs under 300 letters, half under 1,000, 3% under 4,096 and
    // 0.3% longer (97%, 98.5%, 99.91% and 99.991% at the default 97%).
    struct HeldPair {
        int64_t n, m, d;
        double guess;
    };
    std::vector<HeldPair> classes[4];
    double squared = 0.0;
    for (int64_t k = 0; k < held; ++k) {
        const int64_t p = trained + k;
        const int64_t reference = host_offsets[size_t(2 * p + 1)] - host_offsets[size_t(2 * p)];
        const int64_t query = host_offsets[size_t(2 * p + 2)] - host_offsets[size_t(2 * p + 1)];
        const double d = double(host_distances[size_t(p)]);
        const double g = double(guesses[size_t(k)]);
        const double mean = 0.5 * double(reference + query);
        classes[length_class(mean)].push_back({std::min(reference, query), std::max(reference, query),
                                               host_distances[size_t(p)], g});
        const double e = (mean > 0 ? d / mean : 0.0) - (mean > 0 ? g / mean : 0.0);
        squared += e * e;
    }
    if (gpu->band_tuning.chain_words == 0) gpu->band_tuning = default_band_tuning();
    // The first round a batch runs is its largest: where a round's chain bound grows with its work, take it
    // as unbounded.
    BandTuning tuning = gpu->band_tuning;
    if (tuning.chain_share > 0.f) tuning.chain_words = INT64_MAX / 4;
    const double slack = options.slack;
    // Whether a pair settles in its first round at margin `margin` (predict_kernel's threshold).
    auto settles = [&](const HeldPair &h, double margin) {
        const int64_t delta = h.m - h.n;
        int64_t t = int64_t(std::ceil(h.guess * margin + slack));
        t = std::max<int64_t>(std::max<int64_t>(t, delta), 1);
        const int64_t window = band_capacity(band_shape_for(h.n, h.m, t, false, tuning));
        const int64_t words = (h.n + 63) / 64;
        if (window >= words) return true;
        if (window < band_words_needed(h.n, h.m, t)) return false;
        const int64_t half = (t - delta) / 2, reach = band_reach(h.n, h.m, window);
        return h.d <= delta + 2 * std::max(half, reach) + 1;
    };
    const double coverage = std::min(std::max(options.coverage, 0.5), 0.999);
    const double misses[4] = {1.0, 0.5, 0.03, 0.003};
    double widest = 0.0;
    for (int c = 0; c < 4; ++c) {
        double margin = 1.0;
        if (!classes[c].empty()) {
            const double share = 1.0 - (1.0 - coverage) * misses[c];
            const int64_t wanted = int64_t(std::ceil(share * double(classes[c].size())));
            auto enough = [&](double mu) {
                int64_t settled = 0;
                for (const HeldPair &h : classes[c]) settled += settles(h, mu) ? 1 : 0;
                return settled >= wanted;
            };
            // The least margin in [0.5, 4] reaching the share, to 1/1000 (settling grows with the margin).
            double low = 0.5, high = 4.0;
            if (enough(low)) {
                high = low;
            } else {
                while (high - low > 1e-3) {
                    const double mid = 0.5 * (low + high);
                    if (enough(mid))
                        high = mid;
                    else
                        low = mid;
                }
            }
            margin = high;
        }
        gpu->predictor_margins[c] = margin;
        widest = std::max(widest, margin);
    }
    gpu->predictor_margin = widest;
    gpu->predictor_slack = options.slack;
    const double margin = widest;
    report.validation_loss = squared / double(held);
    report.margin = margin;
    report.slack = options.slack;
    report.held_out = held;
}

}  // namespace dinara
