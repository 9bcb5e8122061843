// Shared definitions of the B200 alignment library: the context, device buffers that grow and are
// kept between calls, error plumbing from CUDA calls to the C ABI's codes, and the packed pair layout
// every kernel reads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "dinara_gpu.h"

namespace dinara {

// A failure carrying one of the C ABI's codes and a message for dinara_gpu_last_error.
struct Failure : std::runtime_error {
    int64_t code;
    Failure(int64_t c, const std::string &message) : std::runtime_error(message), code(c) {}
};

inline void check_cuda(cudaError_t status, const char *what, const char *file, int line) {
    if (status != cudaSuccess) {
        throw Failure(status == cudaErrorMemoryAllocation ? DINARA_OUT_OF_MEMORY : DINARA_DEVICE_FAILURE,
                      std::string(what) + ": " + cudaGetErrorString(status) + " (" + file + ":" + std::to_string(line) +
                          ")");
    }
}

#define DINARA_CUDA(call) ::dinara::check_cuda((call), #call, __FILE__, __LINE__)

// The stream the calling thread's context orders its allocations on (set for the length of each entry
// point). Device buffers grow and shrink by stream-ordered allocation from the device's pool: a plain
// cudaMalloc or cudaFree would wait for every kernel on the device, so one context growing a buffer would
// stall the work every other context (a serving slot, say) has in flight.
inline thread_local cudaStream_t allocation_stream = nullptr;

// Sets the allocation stream for a scope and puts the previous one back after it.
struct AllocationScope {
    cudaStream_t previous;
    explicit AllocationScope(cudaStream_t stream) : previous(allocation_stream) { allocation_stream = stream; }
    ~AllocationScope() { allocation_stream = previous; }
};

// A device allocation that grows on demand and is reused by later calls.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    template <class T>
    T *ensure(size_t count) {
        size_t wanted = count * sizeof(T);
        if (wanted == 0) wanted = 256;
        if (wanted > bytes) {
            if (ptr) cudaFreeAsync(ptr, allocation_stream);
            ptr = nullptr;
            bytes = 0;
            size_t grown = wanted + wanted / 4;
            grown = (grown + 255) & ~size_t(255);
            DINARA_CUDA(cudaMallocAsync(&ptr, grown, allocation_stream));
            bytes = grown;
        }
        return static_cast<T *>(ptr);
    }
    template <class T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
    void release() {
        if (ptr) cudaFreeAsync(ptr, allocation_stream);
        ptr = nullptr;
        bytes = 0;
    }
};

// Page-locked host memory, so copies run at the bus's rate and asynchronously.
struct PinnedBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    template <class T>
    T *ensure(size_t count) {
        size_t wanted = count * sizeof(T);
        if (wanted == 0) wanted = 256;
        if (wanted > bytes) {
            if (ptr) cudaFreeHost(ptr);
            ptr = nullptr;
            bytes = 0;
            size_t grown = wanted + wanted / 4;
            DINARA_CUDA(cudaMallocHost(&ptr, grown));
            bytes = grown;
        }
        return static_cast<T *>(ptr);
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// One pair on the packed tape: each sequence starts on a 16-byte boundary, `letters_per_word` codes a
// 32-bit word, lowest bits first; rows are the reference's letters, columns the query's.
struct PairShape {
    uint32_t first_word;
    uint32_t rows;
    uint32_t second_word;
    uint32_t columns;
};

// Where a sequence of the ASCII tape lands on the packed tape, in 32-bit words: every sequence takes a
// 16-byte chunk boundary, and adding one chunk a sequence to its letter offset keeps them apart.
__host__ __device__ inline uint64_t packed_word_start(int64_t letter_offset, int64_t sequence, int bits) {
    const int64_t letters_per_chunk = 4 * (32 / bits);
    return 4ull * uint64_t(letter_offset / letters_per_chunk + sequence);
}

inline uint64_t packed_words_total(int64_t letters, int64_t sequences, int bits) {
    const int64_t letters_per_chunk = 4 * (32 / bits);
    return 4ull * uint64_t(letters / letters_per_chunk + sequences + 2);
}

}  // namespace dinara

namespace dinara {

// How a unit-cost band round picks a pair's window shape among those that hold its band (band_shape_for,
// edit.cuh). `word_cost` is each shape's time a 64-cell word step, relative (lower is faster), and
// `chain_words` bounds a pair's chain of dependent word steps (text letters x words a lane), so that a
// long pair, which holds its lanes for the whole of that chain, takes more lanes and fewer words each.
// The band autotuner (dinara_gpu_band_autotune) measures both on the device; until then they come from
// default_band_tuning (edit.cuh).
struct BandTuning {
    static constexpr int kShapes = 40;
    int64_t chain_words;
    // A round's chain bound grows with its work: at least chain_words, and chain_share times the round's
    // word steps (in its smallest windows) over the GPU's lanes, so a pair's chain stays within a share of
    // the round it runs in.
    float chain_share;
    // How much wider than the smallest window a shape may be taken so that a long pair's chain fits, in
    // quarters of the smallest (5: a quarter wider; 8: twice as wide).
    int32_t reach;
    float word_cost[kShapes];
    int32_t tuned;  // 1 once the autotuner has set them on this context
    // How a round's launches (one a shape, all at once on side streams) share the GPU: 0 each takes the
    // share of its lanes that its share of the round's time asks for; 1 each may fill the GPU, later
    // launches' blocks starting as earlier ones' finish.
    int32_t full_grids;
};

}  // namespace dinara

// The context behind the C ABI's opaque handle.
struct dinara_gpu {
    int device = 0;
    int multiprocessors = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    // Copies of the caller's letters, a piece at a time, alongside the kernels on `stream`.
    cudaStream_t upload = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    // Side streams that let a round's launches of different shapes run at once, joined by events.
    static constexpr int kSideStreams = 39;  // one for each band window shape
    cudaStream_t side[kSideStreams] = {nullptr};
    cudaEvent_t fork = nullptr, joins[kSideStreams] = {nullptr};
    std::string error;
    // Inputs and their packed form.
    dinara::DeviceBuffer letters, offsets, code_table, tape, shapes, flags;
    // Scheduling: bucket keys and the order pairs are taken in.
    dinara::DeviceBuffer keys, keys_sorted, order, order_sorted, sort_scratch, ranges, class_counts, layouts,
        leftovers, decisions_extra;
    // Outputs and per-launch scratch.
    dinara::DeviceBuffer scores, carry, decisions, decision_offsets, walk_out, cigar_slots, cigar_lengths,
        cigar_offsets, cigar_bytes, spans, wide_pending, narrow_leftovers, record_widths, long_pairs, free_spans,
        free_scores, walk_order, reach_scores, reach_spans, diagonals, diagonal_offsets;
    // The host copies of what code_table and table32 hold.
    uint8_t codes_host[256] = {0};
    std::vector<int32_t> table32_host;
    // Unit-cost band state.
    dinara::DeviceBuffer planes, plane_offsets, thresholds, distances, pending, pending_next, counters, table32;
    // Learned band predictor.
    dinara::DeviceBuffer features, weights, gradients, optimizer, predictions, targets, activations, sketches;
    // Alignments under Costs: each warp's arena of kept fronts (ties.cu).
    dinara::DeviceBuffer wavefront;
    dinara::BandTuning band_tuning{};
    bool predictor_ready = false;
    double predictor_margin = 1.25;    // the largest of the classes' margins (reported)
    double predictor_margins[4] = {1.25, 1.25, 1.25, 1.25};  // by mean length: < 300, < 1000, < 4096, more
    double predictor_slack = 0.0;
    dinara::PinnedBuffer pinned_in, pinned_out, pinned_small;
    // Page-locked stages a batch's results come back through, a unit of pairs at a time.
    static constexpr int kStages = 6;
    dinara::PinnedBuffer stages[kStages];
    // Page-locked words the host reads totals and counts into between launches (a read into pageable
    // memory would wait on the driver's staging, which other threads' calls contend for).
    int64_t *readback = nullptr;
    // Device timing of the sweep kernels, accumulated while `timing` is set.
    bool timing = false;
    double kernel_ms = 0.0, record_ms = 0.0;
    // While `timing` is set, a pair of events around each launch of a kernel class (dinara::ClockSpan),
    // summed per class when the call's timer finishes.
    static constexpr int kClockSpans = 512;
    cudaEvent_t clock_events[2 * kClockSpans] = {nullptr};
    int clock_class[kClockSpans] = {0};
    int clock_used = 0;
    int64_t launches = 0;
    int64_t swept_cells = 0;  // cells the sweeps updated (bands, whole matrices, leftovers)
    int64_t band_cells = 0, whole_cells = 0;  // the same, the proven bands' and the whole matrices' apart
    // Another stream with scratch buffers of its own, so that units of a large batch run at once
    // (capi.cu; a chain of them for more than two); set up at its first use.
    dinara_gpu *partner = nullptr;
    // The resident batch (capi.cu), if one is loaded.
    void *resident = nullptr;
    void (*resident_free)(void *) = nullptr;

    // Every device buffer the context holds.
    template <class F>
    void for_each_buffer(F &&visit) {
        dinara::DeviceBuffer *all[] = {
            &letters,   &offsets,      &code_table, &tape,          &shapes,        &flags,         &keys,
            &keys_sorted, &order,      &order_sorted, &sort_scratch, &ranges,       &class_counts,  &layouts,
            &leftovers, &decisions_extra, &scores,  &carry,         &decisions,     &decision_offsets, &walk_out,
            &cigar_slots, &cigar_lengths, &cigar_offsets, &cigar_bytes, &spans,      &wide_pending,  &narrow_leftovers, &record_widths, &long_pairs, &free_spans, &free_scores, &walk_order, &reach_scores, &reach_spans, &diagonals, &diagonal_offsets, &planes,
            &plane_offsets,
            &thresholds, &distances,   &pending,    &pending_next,  &counters,      &table32,       &features,
            &weights,   &gradients,    &optimizer,  &predictions,   &targets,       &activations,   &sketches,
            &wavefront};
        for (dinara::DeviceBuffer *buffer : all) visit(*buffer);
    }
};

namespace dinara {

// Kernel classes a timed call reports apart (dinara_timing.class_ms).
enum KernelClass {
    kClassBandRecord = 0,  // the proven-band sweep, recording decisions
    kClassBandScore = 1,   // the proven-band sweep, scores only
    kClassWhole = 2,       // whole-matrix sweeps (strips, 16-bit pairs, a block a pair)
    kClassWalk = 3,        // the walk back from recorded decisions
    kClassUnitBand = 4,    // unit-cost band rounds (every window shape of a round, first launch to last)
    kClassPredict = 5,     // the learned band's sketch and prediction
    kClassTrace = 6,       // unit-cost CIGARs: the recording band and its trace
    kClassOther = 7,
};

// Device time of one launch (or one round of launches) on `stream`, kept while the context times.
struct ClockSpan {
    dinara_gpu *gpu;
    cudaStream_t stream;
    int slot = -1;
    ClockSpan(dinara_gpu *g, int cls, cudaStream_t s) : gpu(g), stream(s) {
        if (!gpu->timing || gpu->clock_used >= dinara_gpu::kClockSpans) return;
        slot = gpu->clock_used++;
        for (int k = 0; k < 2; ++k)
            if (!gpu->clock_events[2 * slot + k]) DINARA_CUDA(cudaEventCreate(&gpu->clock_events[2 * slot + k]));
        gpu->clock_class[slot] = cls;
        DINARA_CUDA(cudaEventRecord(gpu->clock_events[2 * slot], stream));
    }
    void stop() {
        if (slot < 0) return;
        DINARA_CUDA(cudaEventRecord(gpu->clock_events[2 * slot + 1], stream));
        slot = -1;
    }
    ~ClockSpan() {
        if (slot >= 0) cudaEventRecord(gpu->clock_events[2 * slot + 1], stream);
    }
};

// Bytes the context's page-locked readback words hold.
constexpr size_t kReadbackBytes = 512;

// Copies `bytes` (at most kReadbackBytes) of device memory to `host` once the context's stream reaches
// the copy, through its page-locked readback words, and waits for it.
inline void read_back(dinara_gpu *gpu, void *host, const void *device, size_t bytes) {
    if (bytes > kReadbackBytes) throw Failure(DINARA_DEVICE_FAILURE, "a read back past the readback words");
    DINARA_CUDA(cudaMemcpyAsync(gpu->readback, device, bytes, cudaMemcpyDeviceToHost, gpu->stream));
    DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
    std::memcpy(host, gpu->readback, bytes);
}

}  // namespace dinara
