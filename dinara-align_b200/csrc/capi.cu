// The C ABI (include/dinara_gpu.h): checks what the reference checks, moves the caller's letters to the
// device, packs and schedules them there, runs the kernels and brings the results back.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "affine.cuh"
#include "banded.cuh"
#include "edit.cuh"
#include "internal.cuh"
#include "learned.cuh"
#include "pack.cuh"

using namespace dinara;

namespace {

thread_local std::string new_error;

template <class F>
int64_t guard(dinara_gpu *gpu, F &&body) {
    // Allocations during the call are ordered on the context's stream.
    AllocationScope scope(gpu ? gpu->stream : nullptr);
    try {
        return body();
    } catch (const Failure &failure) {
        if (gpu) gpu->error = failure.what();
        return failure.code;
    } catch (const std::bad_alloc &) {
        if (gpu) gpu->error = "host memory ran out";
        return DINARA_OUT_OF_MEMORY;
    } catch (const std::exception &error) {
        if (gpu) gpu->error = error.what();
        return DINARA_DEVICE_FAILURE;
    }
}

// A Scoring checked as the reference checks one (scoring.mojo:127-215: letter_count, gap_scores,
// AffineGapCosts.checked), in the kernels' terms, with the byte-to-code table of common.mojo:267-275.
struct CheckedScoring {
    AffineTable table;
    uint8_t codes[256];
    int bits;
    int64_t reach_opening, reach_step;  // ScoreReach, scoring.mojo:228-249
};

CheckedScoring check_scoring(const dinara_scoring *scoring, bool local) {
    if (!scoring || !scoring->alphabet || !scoring->table) throw Failure(DINARA_INVALID_COSTS, "no Scoring given");
    const int64_t size = scoring->alphabet_size;
    if (size < 1 || size > 32)
        throw Failure(DINARA_UNSUPPORTED_SYMBOLS, std::to_string(size) + " letters, from 1 to 32");
    CheckedScoring out;
    std::memset(&out, 0, sizeof out);
    std::memset(out.codes, 255, sizeof out.codes);
    for (int64_t i = 0; i < size; ++i) {
        const uint8_t letter = uint8_t(scoring->alphabet[i]);
        if (letter == '-') throw Failure(DINARA_INVALID_COSTS, "'-' names a gap, not a letter");
        out.codes[letter] = uint8_t(i);
    }
    const int64_t opening = scoring->opening, extension = scoring->extension;
    if (opening > 0) throw Failure(DINARA_INVALID_COSTS, "a gap opening of " + std::to_string(opening) + " rewards a gap");
    const int64_t lowest = -int64_t(INT32_MAX);
    if (std::min(opening, extension) < lowest || extension > int64_t(INT32_MAX) || opening + extension < lowest)
        throw Failure(DINARA_INVALID_COSTS, "a gap opening of " + std::to_string(opening) + " and extension of " +
                                                std::to_string(extension));
    const int32_t open = int32_t(opening + extension), extend = int32_t(extension);
    if (open > extend) throw Failure(DINARA_INVALID_COSTS, "a gap's first letter scoring above a further one");
    if (extend > 0) throw Failure(DINARA_INVALID_COSTS, "a gap that earns");
    out.table.size = int32_t(size);
    out.table.open = open;
    out.table.extend = extend;
    int32_t hi = -128, lo = 127;
    bool fits = size <= 4;
    for (int64_t r = 0; r < size; ++r)
        for (int64_t c = 0; c < size; ++c) {
            const int32_t v = scoring->table[r * size + c];
            out.table.entries[r * 32 + c] = v;
            hi = std::max(hi, v);
            lo = std::min(lo, v);
            const int64_t shifted = local ? int64_t(v) : int64_t(v) - 2 * int64_t(extend);
            if (shifted < -32768 || shifted > 32767) fits = false;
        }
    out.table.packed16 = fits;
    out.bits = size <= 4 ? 2 : 8;
    out.reach_opening = 2 * -int64_t(open);
    out.reach_step = std::max<int64_t>(std::max<int64_t>(hi, -int64_t(lo)), -int64_t(extend));
    return out;
}

// GLOBAL (free ends none, no match score) or LOCAL with no match score of its own: what a Scoring
// aligns on the GPU (scoring.mojo:746-757 check_scoring_mode / refuse_span_modes_on_gpu).
bool check_mode(const dinara_mode *mode) {
    if (!mode) return false;
    if (mode->match_score > 0)
        throw Failure(DINARA_INVALID_MODE, "a match score in the mode as well as in the Scoring's table");
    if (mode->kind == DINARA_LOCAL) return true;
    if (mode->kind == DINARA_ENDS_FREE && mode->reference_start == 0 && mode->reference_end == 0 &&
        mode->query_start == 0 && mode->query_end == 0)
        return false;
    throw Failure(DINARA_INVALID_MODE, "a Scoring aligns only globally or locally on the GPU");
}

bool is_pinned(const void *pointer) {
    cudaPointerAttributes attributes;
    if (cudaPointerGetAttributes(&attributes, pointer) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attributes.type == cudaMemoryTypeHost;
}

// Copies `bytes` of host memory to the device on the context's stream, through page-locked staging
// unless the caller's memory is page-locked already.
void to_device(dinara_gpu *gpu, void *device, const void *host, size_t bytes, dinara::PinnedBuffer &staging) {
    if (bytes == 0) return;
    if (is_pinned(host)) {
        DINARA_CUDA(cudaMemcpyAsync(device, host, bytes, cudaMemcpyHostToDevice, gpu->stream));
        return;
    }
    // Staged a slice at a time, each copy overlapping the next slice's memcpy.
    const size_t slice = size_t(64) << 20;
    uint8_t *stage = staging.ensure<uint8_t>(std::min(bytes, 2 * slice));
    const uint8_t *from = static_cast<const uint8_t *>(host);
    uint8_t *to = static_cast<uint8_t *>(device);
    cudaEvent_t done[2];
    DINARA_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
    DINARA_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
    size_t at = 0;
    int half = 0;
    bool used[2] = {false, false};
    while (at < bytes) {
        const size_t n = std::min(slice, bytes - at);
        uint8_t *buffer = stage + (bytes > slice ? half * slice : 0);
        if (used[half]) DINARA_CUDA(cudaEventSynchronize(done[half]));
        std::memcpy(buffer, from + at, n);
        DINARA_CUDA(cudaMemcpyAsync(to + at, buffer, n, cudaMemcpyHostToDevice, gpu->stream));
        DINARA_CUDA(cudaEventRecord(done[half], gpu->stream));
        used[half] = true;
        at += n;
        half ^= 1;
    }
    DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
}

void to_host(dinara_gpu *gpu, void *host, const void *device, size_t bytes) {
    if (bytes == 0) return;
    DINARA_CUDA(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, gpu->stream));
}

// A host copy shared by four threads.
void parallel_copy(uint8_t *to, const uint8_t *from, size_t bytes) {
    constexpr int kThreads = 4;
    if (bytes < (size_t(1) << 20)) {
        std::memcpy(to, from, bytes);
        return;
    }
    const size_t part = (bytes + kThreads - 1) / kThreads;
    std::thread helpers[kThreads - 1];
    for (int t = 1; t < kThreads; ++t) {
        const size_t begin = std::min(bytes, size_t(t) * part), end = std::min(bytes, begin + part);
        helpers[t - 1] = std::thread([=] { std::memcpy(to + begin, from + begin, end - begin); });
    }
    std::memcpy(to, from, std::min(bytes, part));
    for (auto &helper : helpers) helper.join();
}

// Copies `bytes` of device memory to host memory and waits for them. Large copies into pageable memory
// (which the driver moves at a few GB/s) go through the context's page-locked staging a slice at a time,
// each slice's transfer overlapping the host copy of the one before it.
void to_host_now(dinara_gpu *gpu, void *host, const void *device, size_t bytes) {
    if (bytes == 0) return;
    const size_t slice = size_t(32) << 20;
    if (bytes < (size_t(4) << 20) || is_pinned(host)) {
        DINARA_CUDA(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, gpu->stream));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return;
    }
    uint8_t *stage = gpu->pinned_out.ensure<uint8_t>(std::min(bytes, 2 * slice));
    const uint8_t *from = static_cast<const uint8_t *>(device);
    uint8_t *to = static_cast<uint8_t *>(host);
    size_t at = 0;
    int half = 0;
    size_t previous_at = 0, previous_n = 0;
    while (at < bytes) {
        const size_t n = std::min(slice, bytes - at);
        uint8_t *buffer = stage + (bytes > slice ? size_t(half) * slice : 0);
        DINARA_CUDA(cudaMemcpyAsync(buffer, from + at, n, cudaMemcpyDeviceToHost, gpu->stream));
        // The slice before this one, whose transfer the stream finished first, is copied meanwhile.
        if (previous_n > 0) {
            parallel_copy(to + previous_at, stage + (bytes > slice ? size_t(half ^ 1) * slice : 0), previous_n);
        }
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        previous_at = at;
        previous_n = n;
        at += n;
        half ^= 1;
    }
    parallel_copy(to + previous_at, stage + (bytes > slice ? size_t(half ^ 1) * slice : 0), previous_n);
}

// The batch's letters and offsets on the device, packed, with every pair's shape.
struct Packed {
    int64_t pairs = 0;
    uint32_t *tape = nullptr;
    PairShape *shapes = nullptr;
    uint8_t *unknown = nullptr;
    uint32_t max_rows = 0, max_columns = 0;
};

// Runs work(begin, end) over [0, count) on four threads when the count is large, else on this one; each
// share is contiguous and the shares do not overlap.
template <class F>
void split_work(int64_t count, F &&work) {
    constexpr int kThreads = 4;
    if (count < 65536) {
        work(int64_t(0), count);
        return;
    }
    const int64_t part = (count + kThreads - 1) / kThreads;
    std::thread helpers[kThreads - 1];
    for (int t = 1; t < kThreads; ++t)
        helpers[t - 1] = std::thread([&, t] { work(std::min(count, t * part), std::min(count, (t + 1) * part)); });
    work(int64_t(0), std::min(count, part));
    for (auto &helper : helpers) helper.join();
}

void check_offsets(int64_t pairs, const int64_t *offsets) {
    if (pairs < 0) throw Failure(DINARA_INVALID_LENGTH, "a negative pair count");
    if (pairs > 0 && !offsets) throw Failure(DINARA_INVALID_LENGTH, "no offsets");
    std::atomic<bool> falling{false};
    split_work(2 * pairs, [&](int64_t begin, int64_t end) {
        for (int64_t k = begin; k < end; ++k)
            if (offsets[k + 1] < offsets[k]) falling = true;
    });
    if (falling) throw Failure(DINARA_INVALID_LENGTH, "a sequence's length below zero");
    if (pairs > 0 && offsets[0] < 0) throw Failure(DINARA_INVALID_LENGTH, "an offset below zero");
}

Packed pack_batch(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets, const uint8_t codes[256],
                  int bits) {
    Packed out;
    out.pairs = pairs;
    const int64_t first = offsets[0];
    const int64_t total = offsets[2 * pairs] - first;
    // Offsets as the device sees them, from the letters' first byte.
    std::vector<int64_t> relative;
    const int64_t *device_offsets_host = offsets;
    if (first != 0) {
        relative.resize(size_t(2 * pairs + 1));
        for (int64_t k = 0; k <= 2 * pairs; ++k) relative[size_t(k)] = offsets[k] - first;
        device_offsets_host = relative.data();
    }
    for (int64_t p = 0; p < pairs; ++p) {
        out.max_rows = std::max<uint32_t>(out.max_rows, uint32_t(offsets[2 * p + 1] - offsets[2 * p]));
        out.max_columns = std::max<uint32_t>(out.max_columns, uint32_t(offsets[2 * p + 2] - offsets[2 * p + 1]));
    }
    uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
    int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
    uint8_t *codes_device = gpu->code_table.ensure<uint8_t>(256);
    to_device(gpu, letters_device, letters + first, size_t(total), gpu->pinned_in);
    to_device(gpu, offsets_device, device_offsets_host, size_t(2 * pairs + 1) * sizeof(int64_t), gpu->pinned_small);
    DINARA_CUDA(cudaMemcpyAsync(codes_device, codes, 256, cudaMemcpyHostToDevice, gpu->stream));
    const uint64_t words = packed_words_total(total, 2 * pairs, bits);
    out.tape = gpu->tape.ensure<uint32_t>(size_t(words));
    out.shapes = gpu->shapes.ensure<PairShape>(size_t(pairs));
    out.unknown = gpu->flags.ensure<uint8_t>(size_t(pairs));
    pack_pairs(gpu, letters_device, offsets_device, pairs, codes_device, bits, out.tape, out.shapes, out.unknown);
    return out;
}

// Device memory a launch's recorded decisions may take before the batch is cut into chunks.
constexpr int64_t kDecisionBudget = int64_t(8) << 30;

// The 64-bit words a pair's recorded decisions take (the layout affine.cu's record kernels write).
int64_t record_words(int64_t rows, int64_t columns, bool uniform, bool band) {
    if (rows <= 0 || columns <= 0) return 0;
    if (band && band_eligible(uint32_t(rows), uint32_t(columns))) return int64_t(kBandLanes) * ((rows + 3) & ~int64_t(3));
    const int64_t lanes = record_lanes(uint32_t(columns), uniform);
    return (columns + lanes * 16 - 1) / (lanes * 16) * lanes * (((rows + 2) | 3) + 1);
}

// Per-pair statuses: scores that could pass 2^28 (-3), then a letter outside the alphabet (-1).
void statuses_of(const CheckedScoring &checked, bool local, int64_t pairs, const int64_t *offsets,
                 const uint8_t *unknown_host, int64_t *statuses) {
    if (!statuses) return;
    split_work(pairs, [&](int64_t begin, int64_t end) {
        for (int64_t p = begin; p < end; ++p) {
            const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
            const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
            const int64_t letters = local ? std::min(rows, columns) : rows + columns;
            int64_t status = 0;
            if (checked.reach_opening + 2 * (letters + 2) * checked.reach_step >= (int64_t(1) << 28))
                status = DINARA_INVALID_COSTS;
            else if (unknown_host[p])
                status = DINARA_UNSUPPORTED_SYMBOLS;
            statuses[p] = status;
        }
    });
}

// A tape of the caller's pointer arrays, letters end to end (the reference's PairTape layout).
void gather_tape(int64_t pairs, const char *const *references, const int64_t *reference_lengths,
                 const char *const *queries, const int64_t *query_lengths, std::vector<char> &letters,
                 std::vector<int64_t> &offsets) {
    if (pairs < 0) throw Failure(DINARA_INVALID_LENGTH, "a negative pair count");
    offsets.resize(size_t(2 * pairs + 1));
    int64_t at = 0;
    offsets[0] = 0;
    for (int64_t p = 0; p < pairs; ++p) {
        if (reference_lengths[p] < 0 || query_lengths[p] < 0)
            throw Failure(DINARA_INVALID_LENGTH, "a sequence's length below zero");
        at += reference_lengths[p];
        offsets[size_t(2 * p + 1)] = at;
        at += query_lengths[p];
        offsets[size_t(2 * p + 2)] = at;
    }
    letters.resize(size_t(at) + 1);
    for (int64_t p = 0; p < pairs; ++p) {
        if (reference_lengths[p] > 0)
            std::memcpy(&letters[size_t(offsets[size_t(2 * p)])], references[p], size_t(reference_lengths[p]));
        if (query_lengths[p] > 0)
            std::memcpy(&letters[size_t(offsets[size_t(2 * p + 1)])], queries[p], size_t(query_lengths[p]));
    }
}

// as_alignment's placement (scoring.mojo:724-744): a local alignment's letters placed at the last place
// they occur in their sequence; `start`/`end` are where the walk found them.
int64_t last_place(const char *text, int64_t length, int64_t start, int64_t end) {
    const int64_t k = end - start;
    if (k <= 0) return 0;
    for (int64_t at = length - k; at > start; --at)
        if (text[at] == text[start] && std::memcmp(text + at, text + start, size_t(k)) == 0) return at;
    return start;
}

// The resident batch: packed letters kept on the device between calls.
struct Resident {
    int64_t pairs = 0;
    bool scoring = false;
    CheckedScoring checked;
    Packed packed;
    std::vector<int64_t> offsets;
    const uint8_t *letters_device = nullptr;
    const int64_t *offsets_device = nullptr;
    int64_t cells = 0;
    int last = 0;  // 1 scores, 2 distances
};

void free_resident(void *pointer) { delete static_cast<Resident *>(pointer); }

Resident &resident_of(dinara_gpu *gpu) {
    if (!gpu || !gpu->resident) throw Failure(DINARA_INVALID_MODE, "no resident batch loaded");
    return *static_cast<Resident *>(gpu->resident);
}

struct Timer {
    dinara_gpu *gpu;
    cudaEvent_t begin = nullptr, end = nullptr;
    explicit Timer(dinara_gpu *g) : gpu(g) {
        DINARA_CUDA(cudaEventCreate(&begin));
        DINARA_CUDA(cudaEventCreate(&end));
        DINARA_CUDA(cudaEventRecord(begin, gpu->stream));
        gpu->timing = true;
        gpu->kernel_ms = gpu->record_ms = 0.0;
        gpu->launches = 0;
        gpu->swept_cells = 0;
    }
    void finish(dinara_timing *timing, int64_t cells) {
        DINARA_CUDA(cudaEventRecord(end, gpu->stream));
        DINARA_CUDA(cudaEventSynchronize(end));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, begin, end));
        if (timing) {
            timing->total_ms = ms;
            timing->kernel_ms = gpu->kernel_ms;
            timing->record_ms = gpu->record_ms;
            timing->launches = gpu->launches;
            timing->cells = gpu->swept_cells > 0 ? gpu->swept_cells : cells;
        }
    }
    ~Timer() {
        gpu->timing = false;
        if (begin) cudaEventDestroy(begin);
        if (end) cudaEventDestroy(end);
    }
};

// The learned band's first thresholds, with the device time they took.
const int64_t *timed_predictions(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                                 double *ms) {
    DINARA_CUDA(cudaEventRecord(gpu->start, gpu->stream));
    const int64_t *starts = predict_thresholds(gpu, pairs, letters, offsets);
    DINARA_CUDA(cudaEventRecord(gpu->stop, gpu->stream));
    DINARA_CUDA(cudaEventSynchronize(gpu->stop));
    float elapsed = 0.f;
    DINARA_CUDA(cudaEventElapsedTime(&elapsed, gpu->start, gpu->stop));
    *ms = elapsed;
    return starts;
}

}  // namespace

extern "C" {

dinara_gpu *dinara_gpu_new(int64_t device) {
    dinara_gpu *gpu = nullptr;
    try {
        gpu = new dinara_gpu();
        gpu->device = int(device);
        DINARA_CUDA(cudaSetDevice(int(device)));
        cudaDeviceProp properties;
        DINARA_CUDA(cudaGetDeviceProperties(&properties, int(device)));
        gpu->multiprocessors = properties.multiProcessorCount;
        std::snprintf(gpu->name, sizeof gpu->name, "%s", properties.name);
        DINARA_CUDA(cudaStreamCreateWithFlags(&gpu->stream, cudaStreamNonBlocking));
        // The device's pool keeps what contexts free for their next growth instead of handing it back at
        // every synchronisation (this process's pool only; nothing outlives it).
        cudaMemPool_t pool = nullptr;
        DINARA_CUDA(cudaDeviceGetDefaultMemPool(&pool, int(device)));
        uint64_t keep = UINT64_MAX;
        DINARA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        DINARA_CUDA(cudaEventCreate(&gpu->start));
        DINARA_CUDA(cudaEventCreate(&gpu->stop));
        DINARA_CUDA(cudaEventCreateWithFlags(&gpu->fork, cudaEventDisableTiming));
        for (int k = 0; k < dinara_gpu::kSideStreams; ++k) {
            DINARA_CUDA(cudaStreamCreateWithFlags(&gpu->side[k], cudaStreamNonBlocking));
            DINARA_CUDA(cudaEventCreateWithFlags(&gpu->joins[k], cudaEventDisableTiming));
        }
        return gpu;
    } catch (const std::exception &error) {
        new_error = error.what();
        delete gpu;
        return nullptr;
    }
}

void dinara_gpu_free(dinara_gpu *gpu) {
    if (!gpu) return;
    cudaSetDevice(gpu->device);
    AllocationScope scope(gpu->stream);
    if (gpu->stream) cudaStreamSynchronize(gpu->stream);
    if (gpu->resident) gpu->resident_free(gpu->resident);
    gpu->for_each_buffer([](dinara::DeviceBuffer &buffer) { buffer.release(); });
    if (gpu->stream) cudaStreamSynchronize(gpu->stream);
    gpu->pinned_in.release();
    gpu->pinned_out.release();
    gpu->pinned_small.release();
    if (gpu->start) cudaEventDestroy(gpu->start);
    if (gpu->stop) cudaEventDestroy(gpu->stop);
    if (gpu->fork) cudaEventDestroy(gpu->fork);
    for (int k = 0; k < dinara_gpu::kSideStreams; ++k) {
        if (gpu->side[k]) cudaStreamDestroy(gpu->side[k]);
        if (gpu->joins[k]) cudaEventDestroy(gpu->joins[k]);
    }
    if (gpu->stream) cudaStreamDestroy(gpu->stream);
    delete gpu;
}

const char *dinara_gpu_last_error(const dinara_gpu *gpu) { return gpu ? gpu->error.c_str() : new_error.c_str(); }

int64_t dinara_gpu_device_info(dinara_gpu *gpu, char *name, int64_t name_capacity, int64_t *multiprocessors) {
    if (!gpu) return DINARA_INVALID_MODE;
    if (name && name_capacity > 0) std::snprintf(name, size_t(name_capacity), "%s", gpu->name);
    if (multiprocessors) *multiprocessors = gpu->multiprocessors;
    return 0;
}

void dinara_free(char *cigar) { std::free(cigar); }

int64_t dinara_gpu_scores_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                               const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores,
                               int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        const bool local = check_mode(mode);
        const CheckedScoring checked = check_scoring(scoring, local);
        check_offsets(pairs, offsets);
        if (pairs == 0) return 0;
        DINARA_CUDA(cudaSetDevice(gpu->device));
        Packed packed = pack_batch(gpu, pairs, letters, offsets, checked.codes, checked.bits);
        AffineBatch batch{pairs, checked.bits, local, packed.tape, packed.shapes, packed.max_rows, packed.max_columns};
        int32_t *scores_device = gpu->scores.ensure<int32_t>(size_t(pairs));
        affine_scores(gpu, batch, checked.table, scores_device, 0, pairs);
        std::vector<uint8_t> unknown(static_cast<size_t>(pairs));
        to_host_now(gpu, scores, scores_device, size_t(pairs) * sizeof(int32_t));
        to_host_now(gpu, unknown.data(), packed.unknown, size_t(pairs));
        statuses_of(checked, local, pairs, offsets, unknown.data(), statuses);
        return 0;
    });
}

int64_t dinara_gpu_scores(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                          const int64_t *reference_lengths, const char *const *queries, const int64_t *query_lengths,
                          const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores, int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        const bool local = check_mode(mode);
        (void)check_scoring(scoring, local);
        std::vector<char> letters;
        std::vector<int64_t> offsets;
        gather_tape(pairs, references, reference_lengths, queries, query_lengths, letters, offsets);
        const int64_t code =
            dinara_gpu_scores_tape(gpu, pairs, letters.data(), offsets.data(), scoring, mode, scores, statuses);
        if (code != 0) throw Failure(code, gpu ? gpu->error : std::string("failed"));
        return 0;
    });
}

int64_t dinara_gpu_alignments_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                   const dinara_scoring *scoring, const dinara_mode *mode, int64_t eqx,
                                   int32_t *scores, int64_t *spans, int64_t *cigar_offsets, char **cigar_bytes,
                                   int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        const bool local = check_mode(mode);
        const CheckedScoring checked = check_scoring(scoring, local);
        check_offsets(pairs, offsets);
        if (cigar_bytes) *cigar_bytes = nullptr;
        if (pairs == 0) {
            if (cigar_offsets) cigar_offsets[0] = 0;
            if (cigar_bytes) *cigar_bytes = static_cast<char *>(std::calloc(1, 1));
            return 0;
        }
        DINARA_CUDA(cudaSetDevice(gpu->device));
        Packed packed = pack_batch(gpu, pairs, letters, offsets, checked.codes, checked.bits);
        AffineBatch batch{pairs, checked.bits, local, packed.tape, packed.shapes, packed.max_rows, packed.max_columns};
        int32_t *scores_device = gpu->scores.ensure<int32_t>(size_t(pairs));
        // Chunks whose recorded decisions stay within a budget of device memory.
        const int64_t budget_words = kDecisionBudget / 8;
        const bool uniform = !checked.table.packed16 || checked.bits == 8;
        const bool band = band_serves(batch, checked.table);
        // Every chunk's CIGAR bytes go straight into the caller's buffer, grown a chunk at a time.
        char *bytes = nullptr;
        size_t size = 0;
        std::vector<int64_t> walk_spans(local ? size_t(4 * pairs) : 0);
        std::vector<int64_t> ends(size_t(pairs + 1));
        ends[0] = 0;
        int64_t first = 0;
        while (first < pairs) {
            int64_t count = 0, words = 0;
            while (first + count < pairs) {
                const int64_t p = first + count;
                const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
                const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
                const int64_t w = record_words(rows, columns, uniform, band);
                if (count > 0 && words + w > budget_words) break;
                words += w;
                ++count;
            }
            int64_t *spans_device = gpu->ranges.ensure<int64_t>(size_t(4 * count));
            const int64_t total = affine_alignments(gpu, batch, checked.table, eqx != 0, scores_device, spans_device,
                                                    first, count);
            const size_t at = size;
            char *grown = static_cast<char *>(std::realloc(bytes, at + size_t(total) + 1));
            if (!grown) {
                std::free(bytes);
                throw std::bad_alloc();
            }
            bytes = grown;
            size = at + size_t(total);
            std::vector<int64_t> chunk_offsets(size_t(count + 1));
            to_host_now(gpu, bytes + at, gpu->cigar_bytes.as<char>(), size_t(total));
            to_host_now(gpu, chunk_offsets.data(), gpu->cigar_offsets.as<int64_t>(),
                        size_t(count + 1) * sizeof(int64_t));
            // A global walk spans the whole pair, known on the host; only a local one's spans come back.
            if (local)
                to_host_now(gpu, walk_spans.data() + 4 * first, spans_device, size_t(4 * count) * sizeof(int64_t));
            for (int64_t k = 0; k < count; ++k) ends[size_t(first + k + 1)] = int64_t(at) + chunk_offsets[size_t(k + 1)];
            first += count;
        }
        std::vector<uint8_t> unknown(static_cast<size_t>(pairs));
        to_host_now(gpu, scores, scores_device, size_t(pairs) * sizeof(int32_t));
        to_host_now(gpu, unknown.data(), packed.unknown, size_t(pairs));
        statuses_of(checked, local, pairs, offsets, unknown.data(), statuses);
        // Each pair's spans, a share of the pairs a thread.
        auto place_spans = [&](int64_t begin, int64_t end) {
            for (int64_t p = begin; p < end; ++p) {
                const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
                const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
                int64_t *span = spans + 4 * p;
                if (!local) {
                    span[0] = 0;
                    span[1] = rows;
                    span[2] = 0;
                    span[3] = columns;
                } else {
                    const int64_t *w = walk_spans.data() + 4 * p;
                    const char *reference = letters + offsets[2 * p];
                    const char *query = letters + offsets[2 * p + 1];
                    const int64_t r0 = last_place(reference, rows, w[0], w[1]);
                    const int64_t c0 = last_place(query, columns, w[2], w[3]);
                    span[0] = r0;
                    span[1] = r0 + (w[1] - w[0]);
                    span[2] = c0;
                    span[3] = c0 + (w[3] - w[2]);
                }
            }
        };
        split_work(pairs, place_spans);
        if (cigar_offsets) std::memcpy(cigar_offsets, ends.data(), size_t(pairs + 1) * sizeof(int64_t));
        if (!bytes) bytes = static_cast<char *>(std::malloc(1));
        if (!bytes) throw std::bad_alloc();
        bytes[size] = 0;
        if (cigar_bytes)
            *cigar_bytes = bytes;
        else
            std::free(bytes);
        return 0;
    });
}

int64_t dinara_gpu_alignments(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                              const int64_t *reference_lengths, const char *const *queries,
                              const int64_t *query_lengths, const dinara_scoring *scoring, const dinara_mode *mode,
                              int64_t eqx, dinara_alignment *alignments, int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        const bool local = check_mode(mode);
        (void)check_scoring(scoring, local);
        std::vector<char> letters;
        std::vector<int64_t> offsets;
        gather_tape(pairs, references, reference_lengths, queries, query_lengths, letters, offsets);
        std::vector<int32_t> scores(size_t(std::max<int64_t>(pairs, 1)));
        std::vector<int64_t> spans(size_t(4 * std::max<int64_t>(pairs, 1)));
        std::vector<int64_t> cigar_offsets(size_t(pairs + 1));
        std::vector<int64_t> own_statuses(size_t(std::max<int64_t>(pairs, 1)));
        char *bytes = nullptr;
        const int64_t code = dinara_gpu_alignments_tape(gpu, pairs, letters.data(), offsets.data(), scoring, mode, eqx,
                                                        scores.data(), spans.data(), cigar_offsets.data(), &bytes,
                                                        own_statuses.data());
        if (code != 0) throw Failure(code, gpu ? gpu->error : std::string("failed"));
        for (int64_t p = 0; p < pairs; ++p) {
            if (statuses) statuses[p] = own_statuses[size_t(p)];
            dinara_alignment &a = alignments[p];
            std::memset(&a, 0, sizeof a);
            if (own_statuses[size_t(p)] != 0) continue;
            const int64_t length = cigar_offsets[size_t(p + 1)] - cigar_offsets[size_t(p)];
            a.cigar = static_cast<char *>(std::malloc(size_t(length) + 1));
            if (!a.cigar) throw std::bad_alloc();
            std::memcpy(a.cigar, bytes + cigar_offsets[size_t(p)], size_t(length));
            a.cigar[length] = 0;
            a.cigar_length = length;
            a.score = scores[size_t(p)];
            a.cost = -int64_t(scores[size_t(p)]);
            a.reference_start = spans[size_t(4 * p)];
            a.reference_end = spans[size_t(4 * p + 1)];
            a.query_start = spans[size_t(4 * p + 2)];
            a.query_end = spans[size_t(4 * p + 3)];
        }
        std::free(bytes);
        return 0;
    });
}

int64_t dinara_gpu_distances_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                  const dinara_band_plan *plan, int64_t *results, dinara_band_report *report) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        check_offsets(pairs, offsets);
        if (report) std::memset(report, 0, sizeof *report);
        if (pairs == 0) return 0;
        const int64_t policy = plan ? plan->policy : DINARA_BAND_PLAIN;
        if (policy == DINARA_BAND_GIVEN && (!plan || !plan->start_thresholds))
            throw Failure(DINARA_INVALID_MODE, "given thresholds missing");
        if (policy == DINARA_BAND_LEARNED && !gpu->predictor_ready)
            throw Failure(DINARA_INVALID_MODE, "no trained band predictor on this context");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        const int64_t first = offsets[0];
        const int64_t total = offsets[2 * pairs] - first;
        std::vector<int64_t> relative(size_t(2 * pairs + 1));
        for (int64_t k = 0; k <= 2 * pairs; ++k) relative[size_t(k)] = offsets[k] - first;
        uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
        int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
        to_device(gpu, letters_device, letters + first, size_t(total), gpu->pinned_in);
        to_device(gpu, offsets_device, relative.data(), relative.size() * sizeof(int64_t), gpu->pinned_small);
        const int64_t *starts = nullptr;
        double predict_ms = 0.0;
        if (policy == DINARA_BAND_GIVEN) {
            int64_t *device_starts = gpu->predictions.ensure<int64_t>(size_t(pairs));
            to_device(gpu, device_starts, plan->start_thresholds, size_t(pairs) * sizeof(int64_t), gpu->pinned_small);
            starts = device_starts;
        } else if (policy == DINARA_BAND_LEARNED) {
            starts = timed_predictions(gpu, pairs, letters_device, offsets_device, &predict_ms);
        }
        int64_t *results_device = gpu->scores.ensure<int64_t>(size_t(pairs));
        band_doubling(gpu, pairs, letters_device, offsets_device, starts, plan ? plan->default_start : 0, results_device,
                      report);
        if (report) report->predict_ms = predict_ms;
        to_host_now(gpu, results, results_device, size_t(pairs) * sizeof(int64_t));
        if (report) {
            int64_t cells = 0;
            for (int64_t p = 0; p < pairs; ++p)
                cells += (offsets[2 * p + 1] - offsets[2 * p]) * (offsets[2 * p + 2] - offsets[2 * p + 1]);
            report->full_cells = cells;
        }
        return 0;
    });
}

int64_t dinara_gpu_distances(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                             const int64_t *reference_lengths, const char *const *queries, const int64_t *query_lengths,
                             const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options,
                             int64_t *results) {
    return guard(gpu, [&]() -> int64_t {
        // api.mojo:1237-1247: on the GPU, unit costs, globally, with no band; no cap either here.
        int64_t scale = 1;
        if (costs) {
            const bool one_piece = costs->opening2 < 0 && costs->deletion_extension == 0;
            if (!(one_piece && costs->opening == 0 && costs->mismatch == costs->extension && costs->mismatch > 0))
                throw Failure(DINARA_INVALID_MODE, "on the GPU, distances at unit costs, globally, with no band");
            scale = costs->mismatch;
        }
        if (mode && (mode->kind != DINARA_ENDS_FREE || mode->reference_start || mode->reference_end ||
                     mode->query_start || mode->query_end || mode->match_score))
            throw Failure(DINARA_INVALID_MODE, "on the GPU, distances at unit costs, globally, with no band");
        if (options && (options->band_low > INT64_MIN || options->band_high < INT64_MAX || options->max_cost >= 0))
            throw Failure(DINARA_INVALID_MODE, "on the GPU, distances at unit costs, globally, with no band");
        std::vector<char> letters;
        std::vector<int64_t> offsets;
        gather_tape(pairs, references, reference_lengths, queries, query_lengths, letters, offsets);
        const int64_t code = dinara_gpu_distances_tape(gpu, pairs, letters.data(), offsets.data(), nullptr, results, nullptr);
        if (code != 0) throw Failure(code, gpu ? gpu->error : std::string("failed"));
        for (int64_t p = 0; p < pairs; ++p)
            if (results[p] >= 0) results[p] *= scale;
        return 0;
    });
}

int64_t dinara_gpu_resident_load(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                 const dinara_scoring *scoring) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        check_offsets(pairs, offsets);
        DINARA_CUDA(cudaSetDevice(gpu->device));
        if (gpu->resident) {
            gpu->resident_free(gpu->resident);
            gpu->resident = nullptr;
        }
        Resident *r = new Resident();
        gpu->resident = r;
        gpu->resident_free = free_resident;
        r->pairs = pairs;
        r->offsets.assign(offsets, offsets + 2 * pairs + 1);
        for (int64_t k = 0; k <= 2 * pairs; ++k) r->offsets[size_t(k)] -= offsets[0];
        for (int64_t p = 0; p < pairs; ++p)
            r->cells += (r->offsets[size_t(2 * p + 1)] - r->offsets[size_t(2 * p)]) *
                        (r->offsets[size_t(2 * p + 2)] - r->offsets[size_t(2 * p + 1)]);
        if (pairs == 0) return 0;
        if (scoring) {
            r->scoring = true;
            r->checked = check_scoring(scoring, false);
            r->packed = pack_batch(gpu, pairs, letters, offsets, r->checked.codes, r->checked.bits);
        } else {
            const int64_t total = offsets[2 * pairs] - offsets[0];
            uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
            int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
            to_device(gpu, letters_device, letters + offsets[0], size_t(total), gpu->pinned_in);
            to_device(gpu, offsets_device, r->offsets.data(), r->offsets.size() * sizeof(int64_t), gpu->pinned_small);
            r->letters_device = letters_device;
            r->offsets_device = offsets_device;
        }
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return 0;
    });
}

int64_t dinara_gpu_resident_align(dinara_gpu *gpu, const dinara_mode *mode, int64_t cigars, int64_t eqx,
                                  dinara_timing *timing) {
    return guard(gpu, [&]() -> int64_t {
        Resident &r = resident_of(gpu);
        if (!r.scoring) throw Failure(DINARA_INVALID_MODE, "the resident batch was loaded for distances");
        const bool local = check_mode(mode);
        if (r.pairs == 0) return 0;
        DINARA_CUDA(cudaSetDevice(gpu->device));
        Timer timer(gpu);
        AffineBatch batch{r.pairs, r.checked.bits, local, r.packed.tape, r.packed.shapes, r.packed.max_rows,
                          r.packed.max_columns};
        int32_t *scores_device = gpu->scores.ensure<int32_t>(size_t(r.pairs));
        const int64_t *offsets = r.offsets.data();
        if (!cigars) {
            affine_scores(gpu, batch, r.checked.table, scores_device, 0, r.pairs);
        } else {
            const int64_t budget_words = kDecisionBudget / 8;
            const bool uniform = !r.checked.table.packed16 || r.checked.bits == 8;
            const bool band = band_serves(batch, r.checked.table);
            int64_t first = 0;
            while (first < r.pairs) {
                int64_t count = 0, words = 0;
                while (first + count < r.pairs) {
                    const int64_t p = first + count;
                    const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
                    const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
                    const int64_t w = record_words(rows, columns, uniform, band);
                    if (count > 0 && words + w > budget_words) break;
                    words += w;
                    ++count;
                }
                int64_t *spans_device = gpu->ranges.ensure<int64_t>(size_t(4 * count));
                affine_alignments(gpu, batch, r.checked.table, eqx != 0, scores_device, spans_device, first, count);
                first += count;
            }
        }
        r.last = 1;
        timer.finish(timing, r.cells);
        return 0;
    });
}

int64_t dinara_gpu_resident_distances(dinara_gpu *gpu, const dinara_band_plan *plan, dinara_band_report *report,
                                      dinara_timing *timing) {
    return guard(gpu, [&]() -> int64_t {
        Resident &r = resident_of(gpu);
        if (r.scoring) throw Failure(DINARA_INVALID_MODE, "the resident batch was loaded for a Scoring");
        if (report) std::memset(report, 0, sizeof *report);
        if (r.pairs == 0) return 0;
        const int64_t policy = plan ? plan->policy : DINARA_BAND_PLAIN;
        if (policy == DINARA_BAND_GIVEN && (!plan || !plan->start_thresholds))
            throw Failure(DINARA_INVALID_MODE, "given thresholds missing");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        const int64_t *starts = nullptr;
        if (policy == DINARA_BAND_GIVEN) {
            int64_t *device_starts = gpu->predictions.ensure<int64_t>(size_t(r.pairs));
            to_device(gpu, device_starts, plan->start_thresholds, size_t(r.pairs) * sizeof(int64_t), gpu->pinned_small);
            starts = device_starts;
        }
        Timer timer(gpu);
        double predict_ms = 0.0;
        if (policy == DINARA_BAND_LEARNED)
            starts = timed_predictions(gpu, r.pairs, r.letters_device, r.offsets_device, &predict_ms);
        int64_t *results_device = gpu->scores.ensure<int64_t>(size_t(r.pairs));
        band_doubling(gpu, r.pairs, r.letters_device, r.offsets_device, starts, plan ? plan->default_start : 0,
                      results_device, report);
        if (report) report->predict_ms = predict_ms;
        if (report) report->full_cells = r.cells;
        r.last = 2;
        timer.finish(timing, r.cells);
        if (timing && report) timing->kernel_ms = report->kernel_ms;
        return 0;
    });
}

int64_t dinara_gpu_resident_fetch(dinara_gpu *gpu, int32_t *scores, int64_t *distances) {
    return guard(gpu, [&]() -> int64_t {
        Resident &r = resident_of(gpu);
        if (r.pairs == 0) return 0;
        if (r.last == 1 && scores) to_host(gpu, scores, gpu->scores.as<int32_t>(), size_t(r.pairs) * sizeof(int32_t));
        if (r.last == 2 && distances)
            to_host(gpu, distances, gpu->scores.as<int64_t>(), size_t(r.pairs) * sizeof(int64_t));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return 0;
    });
}

namespace {

// A tape's letters and offsets (rebased to its first letter) on the device.
void upload_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets, const uint8_t **letters_out,
                 const int64_t **offsets_out) {
    const int64_t first = offsets[0];
    const int64_t total = offsets[2 * pairs] - first;
    std::vector<int64_t> relative(size_t(2 * pairs + 1));
    for (int64_t k = 0; k <= 2 * pairs; ++k) relative[size_t(k)] = offsets[k] - first;
    uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
    int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
    to_device(gpu, letters_device, letters + first, size_t(total), gpu->pinned_in);
    to_device(gpu, offsets_device, relative.data(), relative.size() * sizeof(int64_t), gpu->pinned_small);
    *letters_out = letters_device;
    *offsets_out = offsets_device;
}

}  // namespace

int64_t dinara_gpu_predictor_train(dinara_gpu *gpu, const dinara_train_options *options, dinara_train_report *report) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !options) throw Failure(DINARA_INVALID_MODE, "no context or options");
        if (options->pairs < 100 || options->batch < 16 || options->batch > 65536 || options->epochs < 1 ||
            options->length_low < 1 || options->length_high < options->length_low || options->rate_low < 0 ||
            options->rate_high < options->rate_low || options->rate_high > 1 || options->learning_rate <= 0)
            throw Failure(DINARA_INVALID_MODE, "training options out of range");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        dinara_train_report local;
        std::memset(&local, 0, sizeof local);
        const auto begin = std::chrono::steady_clock::now();
        predictor_train(gpu, *options, local);
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        local.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
        if (report) *report = local;
        return 0;
    });
}

int64_t dinara_gpu_predictor_set(dinara_gpu *gpu, const float *parameters, double margin, double slack) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !parameters) throw Failure(DINARA_INVALID_MODE, "no context or parameters");
        if (!(margin >= 0.0) || !(slack >= 0.0)) throw Failure(DINARA_INVALID_MODE, "a negative margin or slack");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        float *weights = gpu->weights.ensure<float>(kPredictorParameters);
        DINARA_CUDA(cudaMemcpyAsync(weights, parameters, kPredictorParameters * sizeof(float), cudaMemcpyHostToDevice,
                                    gpu->stream));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        gpu->predictor_margin = margin;
        for (int k = 0; k < 4; ++k) gpu->predictor_margins[k] = margin;
        gpu->predictor_slack = slack;
        gpu->predictor_ready = true;
        return 0;
    });
}

int64_t dinara_gpu_predictor_get(dinara_gpu *gpu, float *parameters, double *margin, double *slack) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !gpu->predictor_ready) throw Failure(DINARA_INVALID_MODE, "no trained band predictor on this context");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        if (parameters) {
            DINARA_CUDA(cudaMemcpyAsync(parameters, gpu->weights.as<float>(), kPredictorParameters * sizeof(float),
                                        cudaMemcpyDeviceToHost, gpu->stream));
            DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        }
        if (margin) *margin = gpu->predictor_margin;
        if (slack) *slack = gpu->predictor_slack;
        return 0;
    });
}

int64_t dinara_gpu_predictor_margins(dinara_gpu *gpu, int64_t set, double *margins) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !margins) throw Failure(DINARA_INVALID_MODE, "no context or margins");
        if (!set) {
            for (int k = 0; k < 4; ++k) margins[k] = gpu->predictor_margins[k];
            return 0;
        }
        for (int k = 0; k < 4; ++k)
            if (!(margins[k] >= 0.0)) throw Failure(DINARA_INVALID_MODE, "a negative margin");
        double widest = 0.0;
        for (int k = 0; k < 4; ++k) {
            gpu->predictor_margins[k] = margins[k];
            widest = std::max(widest, margins[k]);
        }
        gpu->predictor_margin = widest;
        return 0;
    });
}

int64_t dinara_gpu_predictor_features(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                      float *features) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        check_offsets(pairs, offsets);
        if (pairs == 0) return 0;
        DINARA_CUDA(cudaSetDevice(gpu->device));
        const uint8_t *letters_device;
        const int64_t *offsets_device;
        upload_tape(gpu, pairs, letters, offsets, &letters_device, &offsets_device);
        float *matrix = gpu->features.ensure<float>(size_t(pairs) * kPredictorInputs);
        predictor_features(gpu, pairs, letters_device, offsets_device, matrix);
        std::vector<float> host(size_t(pairs) * kPredictorInputs);
        to_host(gpu, host.data(), matrix, host.size() * sizeof(float));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        for (int64_t p = 0; p < pairs; ++p)
            for (int f = 0; f < kPredictorInputs; ++f)
                features[p * kPredictorInputs + f] = host[size_t(int64_t(f) * pairs + p)];
        return 0;
    });
}

int64_t dinara_gpu_predictor_gradients(dinara_gpu *gpu, int64_t batch, const float *features, const float *targets,
                                       float *gradients, double *loss) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !gpu->predictor_ready) throw Failure(DINARA_INVALID_MODE, "no parameters on this context");
        if (batch < 1 || batch > 65536) throw Failure(DINARA_INVALID_LENGTH, "a batch of 1 to 65,536 samples");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        std::vector<float> matrix(size_t(batch) * kPredictorInputs);
        for (int64_t s = 0; s < batch; ++s)
            for (int f = 0; f < kPredictorInputs; ++f)
                matrix[size_t(int64_t(f) * batch + s)] = features[s * kPredictorInputs + f];
        float *x = gpu->features.ensure<float>(matrix.size());
        float *t = gpu->targets.ensure<float>(size_t(batch));
        float *g = gpu->gradients.ensure<float>(kPredictorParameters);
        float *l = gpu->counters.ensure<float>(64) + 60;
        DINARA_CUDA(cudaMemcpyAsync(x, matrix.data(), matrix.size() * sizeof(float), cudaMemcpyHostToDevice, gpu->stream));
        DINARA_CUDA(cudaMemcpyAsync(t, targets, size_t(batch) * sizeof(float), cudaMemcpyHostToDevice, gpu->stream));
        predictor_gradients(gpu, int(batch), x, t, g, l);
        float summed = 0.f;
        to_host(gpu, gradients, g, kPredictorParameters * sizeof(float));
        to_host(gpu, &summed, l, sizeof summed);
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        if (loss) *loss = double(summed) / double(batch);
        return 0;
    });
}

int64_t dinara_gpu_predictor_predict(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                     float *predicted, int64_t *thresholds) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        check_offsets(pairs, offsets);
        if (pairs == 0) return 0;
        DINARA_CUDA(cudaSetDevice(gpu->device));
        const uint8_t *letters_device;
        const int64_t *offsets_device;
        upload_tape(gpu, pairs, letters, offsets, &letters_device, &offsets_device);
        const int64_t *starts = predict_thresholds(gpu, pairs, letters_device, offsets_device);
        if (thresholds) to_host(gpu, thresholds, starts, size_t(pairs) * sizeof(int64_t));
        if (predicted) to_host(gpu, predicted, gpu->targets.as<float>(), size_t(pairs) * sizeof(float));
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return 0;
    });
}

}  // extern "C"
