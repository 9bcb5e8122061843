// Letters to the packed tape on the device: the caller's ASCII tape is copied over as it is and packed
// here, two bits a letter for an alphabet of up to four letters, else a byte, each sequence from its own
// 16-byte boundary (the reference packs on host threads into page-locked memory instead,
// score_groups.mojo:499-537 `packed_into`; its README found that packing dominated its GPU time).
#include <cub/cub.cuh>

#include "affine.cuh"
#include "banded.cuh"
#include "pack.cuh"

namespace dinara {

// A warp a pair: each lane packs 16-byte chunks of the pair's two sequences, translating each byte by
// `codes` (255 for a byte outside the alphabet, which flags the pair), and writes the pair's shape and
// its scheduling key (shape class, strips, rows; sorted descending so the longest go first).
__global__ void pack_pairs_kernel(const uint8_t *__restrict__ letters, const int64_t *__restrict__ offsets,
                                  int64_t first_pair, int64_t count, const uint8_t *__restrict__ codes, int bits,
                                  uint32_t *__restrict__ tape, PairShape *__restrict__ shapes,
                                  uint8_t *__restrict__ unknown) {
    __shared__ uint8_t code_of[256];
    code_of[threadIdx.x & 255] = codes[threadIdx.x & 255];
    __syncthreads();
    const int64_t nth = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (nth >= count) return;
    const int64_t warp = first_pair + nth;
    const int per_word = 32 / bits;
    const int per_chunk = 4 * per_word;
    const uint32_t mask = bits == 8 ? 0xFFu : ((1u << bits) - 1u);
    bool bad = false;
    uint32_t starts[2], lengths[2];
    for (int side = 0; side < 2; ++side) {
        const int64_t k = 2 * warp + side;
        const int64_t start = offsets[k];
        const int64_t length = offsets[k + 1] - start;
        const uint64_t word0 = packed_word_start(start, k, bits);
        starts[side] = uint32_t(word0);
        lengths[side] = uint32_t(length);
        // Lane i packs output words i, i + 32, ... (consecutive lanes, consecutive words: coalesced both
        // ways), each from its letters read through aligned 32-bit words; the sequence's last chunk is
        // zero-filled past its end. No load starts at or past the sequence's end.
        const uintptr_t end = reinterpret_cast<uintptr_t>(letters + start + length);
        const int64_t words = (length + per_chunk - 1) / per_chunk * 4;
        for (int64_t w = lane; w < words; w += 32) {
            const int64_t first = w * per_word;
            uint32_t word = 0;
            if (first < length) {
                const uintptr_t address = reinterpret_cast<uintptr_t>(letters + start + first);
                const uintptr_t aligned = address & ~uintptr_t(3);
                const uint32_t shift = uint32_t(address & 3u) * 8u;
                uint32_t raw[5];
#pragma unroll
                for (int r = 0; r < 5; ++r)
                    raw[r] = (r <= per_word / 4) && aligned + 4 * uintptr_t(r) < end
                                 ? __ldg(reinterpret_cast<const uint32_t *>(aligned) + r)
                                 : 0u;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (q * 4 >= per_word) break;
                    const uint32_t four = __funnelshift_r(raw[q], raw[q + 1], shift);
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int j = 4 * q + b;
                        if (first + j < length) {
                            uint32_t code = code_of[(four >> (8 * b)) & 0xFFu];
                            if (code == 255u) {
                                bad = true;
                                code = 0;
                            }
                            word |= (code & mask) << (bits * j);
                        }
                    }
                }
            }
            tape[word0 + uint64_t(w)] = word;
        }
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
        PairShape shape{starts[0], lengths[0], starts[1], lengths[1]};
        shapes[warp] = shape;
        unknown[warp] = bad ? 1 : 0;
    }
}

// One pair's scheduling key and class (the kernel below).
__device__ void classify_pair(const PairShape *__restrict__ shapes, const uint32_t *__restrict__ list, int64_t first,
                              int64_t k, int record, int band, PairLimits limits, uint32_t *__restrict__ keys,
                              uint32_t *__restrict__ order, unsigned int *block_counts) {
    const uint32_t pair = list ? list[k] : uint32_t(first + k);
    const PairShape shape = shapes[pair];
    const bool empty = shape.rows == 0 || shape.columns == 0;
    int cls;
    uint32_t strips = 0;
    if (limits.band_widths && limits.band_widths[pair - limits.band_first] > 0) {
        cls = kBandRecordClass;
        strips = (shape.columns + 511) / 512;
        if (strips > 255) strips = 255;
    } else if (band && band_eligible(shape.rows, shape.columns)) {
        cls = int64_t(shape.rows) + shape.columns <= limits.band ? kBandPairsClass : kBandClass;
    } else {
        cls = empty ? 0 : affine_shape_for(shape.columns, record != 0);
        if (!record && limits.wide && shape.rows >= kWideRows && shape.columns >= kWideColumns) cls = kWideClass;
        const uint32_t width = cls == kWideClass ? 4096u : uint32_t(affine_lanes(cls) * affine_columns(cls));
        strips = empty ? 0 : (shape.columns + width - 1) / width;
        const int64_t swept = int64_t(strips) * width;
        const bool pairs16 = cls != kWideClass && !record && !empty && limits.whole > 0 &&
                             (limits.local ? swept * limits.best + int64_t(shape.rows) * limits.row_step <= limits.whole
                                           : 2 * swept <= limits.whole && 2 * int64_t(shape.rows) <= limits.whole);
        if (pairs16) cls += kWholePairsClass;
        if (strips > 255) strips = 255;
    }
    uint32_t rows = shape.rows >> 2;
    if (rows > 0xFFFFFu) rows = 0xFFFFFu;
    keys[k] = (uint32_t(cls) << 28) | (strips << 20) | rows;
    order[k] = pair;
    atomicAdd(&block_counts[cls], 1u);
}

// Scheduling keys: the pair's class in the top bits (the whole-matrix shape class, or the proven band,
// the highest), then strips of its width, then rows, so a descending sort puts each class's longest pairs
// first and warps hold pairs of like size. Counts each class.
__global__ void schedule_keys_kernel(const PairShape *__restrict__ shapes, const uint32_t *__restrict__ list,
                                     int64_t first, int64_t count, int record, int band, PairLimits limits,
                                     uint32_t *__restrict__ keys,
                                     uint32_t *__restrict__ order, unsigned int *__restrict__ class_counts) {
    // Each block counts its classes in shared memory first: a million pairs' counts on a dozen global
    // counters would otherwise queue on the same addresses.
    __shared__ unsigned int block_counts[kClasses];
    if (threadIdx.x < kClasses) block_counts[threadIdx.x] = 0;
    __syncthreads();
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < count) classify_pair(shapes, list, first, k, record, band, limits, keys, order, block_counts);
    __syncthreads();
    if (threadIdx.x < kClasses && block_counts[threadIdx.x] > 0)
        atomicAdd(&class_counts[threadIdx.x], block_counts[threadIdx.x]);
}


void pack_pairs(dinara_gpu *gpu, const uint8_t *letters_device, const int64_t *offsets_device, int64_t first_pair,
                int64_t count, const uint8_t *codes_device, int bits, uint32_t *tape, PairShape *shapes,
                uint8_t *unknown) {
    if (count <= 0) return;
    const int threads = 256;
    const int64_t blocks = (count * 32 + threads - 1) / threads;
    pack_pairs_kernel<<<dim3(unsigned(blocks)), threads, 0, gpu->stream>>>(
        letters_device, offsets_device, first_pair, count, codes_device, bits, tape, shapes, unknown);
    gpu->launches += 1;
    DINARA_CUDA(cudaGetLastError());
}

Schedule schedule(dinara_gpu *gpu, const PairShape *shapes, const uint32_t *list, int64_t first, int64_t count,
                   bool record, bool band, PairLimits limits) {
    Schedule out;
    for (int c = 0; c < kClasses; ++c) out.counts[c] = 0;
    out.order = nullptr;
    if (count <= 0) return out;
    uint32_t *keys = gpu->keys.ensure<uint32_t>(count);
    uint32_t *order = gpu->order.ensure<uint32_t>(count);
    uint32_t *keys_out = gpu->keys_sorted.ensure<uint32_t>(count);
    uint32_t *order_out = gpu->order_sorted.ensure<uint32_t>(count);
    unsigned int *class_counts = gpu->class_counts.ensure<unsigned int>(kClasses);
    DINARA_CUDA(cudaMemsetAsync(class_counts, 0, kClasses * sizeof(unsigned int), gpu->stream));
    const int threads = 256;
    schedule_keys_kernel<<<unsigned((count + threads - 1) / threads), threads, 0, gpu->stream>>>(
        shapes, list, first, count, record ? 1 : 0, band ? 1 : 0, limits, keys, order, class_counts);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, scratch, keys, keys_out, order, order_out,
                                                          int(count), 0, 32, gpu->stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(scratch);
    DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(space, scratch, keys, keys_out, order, order_out,
                                                          int(count), 0, 32, gpu->stream));
    unsigned int host_counts[kClasses];
    read_back(gpu, host_counts, class_counts, sizeof host_counts);
    for (int c = 0; c < kClasses; ++c) out.counts[c] = host_counts[c];
    out.order = order_out;
    return out;
}

}  // namespace dinara
