// The C ABI (include/dinara_gpu.h): checks what the reference checks, moves the caller's letters to the
// device, packs and schedules them there, runs the kernels and brings the results back.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <sys/mman.h>

#include "affine.cuh"
#include "banded.cuh"
#include "edit.cuh"
#include "internal.cuh"
#include "learned.cuh"
#include "pack.cuh"
#include "ties.cuh"

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

// check_mode for scores, which also take free ends on the GPU (scored.mojo:69-240 FROM_EDGE, the
// reference's host path; its GPU refuses them): GLOBAL, ends_free with any counts, or LOCAL. Sets the
// batch's free letters (clamped to INT32_MAX) and returns whether the mode is local.
bool check_scores_mode(const dinara_mode *mode, AffineBatch &batch) {
    batch.free_ends = false;
    batch.extension = false;
    if (mode && mode->kind == DINARA_EXTENSION) {
        // An extension (scoring.mojo:673-688): from the starts or the ends, no match score of the mode's own
        // beside the table's. A Z-drop too large ever to end the sweep (scores stay within 2^28 of zero) is
        // taken as none, which spares reading the anti-diagonals in order.
        if (mode->match_score > 0)
            throw Failure(DINARA_INVALID_MODE, "a match score in the mode as well as in the Scoring's table");
        if (mode->anchor != 0 && mode->anchor != 1) throw Failure(DINARA_INVALID_MODE, "an anchor at neither end");
        batch.free_ends = true;
        batch.extension = true;
        batch.from_end = mode->anchor == 1;
        batch.zdrop = mode->zdrop >= 0 && mode->zdrop < (int64_t(1) << 29) ? mode->zdrop : -1;
        batch.end_bonus = mode->end_bonus;
        batch.free_reference_start = batch.free_reference_end = batch.free_query_start = batch.free_query_end = 0;
        return false;
    }
    if (mode && mode->kind == DINARA_ENDS_FREE && mode->match_score <= 0 &&
        (mode->reference_start | mode->reference_end | mode->query_start | mode->query_end) != 0) {
        if (mode->reference_start < 0 || mode->reference_end < 0 || mode->query_start < 0 || mode->query_end < 0)
            throw Failure(DINARA_INVALID_MODE, "a free end of fewer than no letters");
        auto clamp = [](int64_t v) { return int32_t(std::min<int64_t>(v, INT32_MAX)); };
        batch.free_ends = true;
        batch.free_reference_start = clamp(mode->reference_start);
        batch.free_reference_end = clamp(mode->reference_end);
        batch.free_query_start = clamp(mode->query_start);
        batch.free_query_end = clamp(mode->query_end);
        return false;
    }
    return check_mode(mode);
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

// A host copy shared by `threads` threads (at most 8).
void parallel_copy(uint8_t *to, const uint8_t *from, size_t bytes, int threads = 4) {
    constexpr int kMostThreads = 8;
    threads = std::max(1, std::min(threads, kMostThreads));
    if (bytes < (size_t(1) << 20) || threads == 1) {
        std::memcpy(to, from, bytes);
        return;
    }
    const size_t part = (bytes + threads - 1) / threads;
    std::thread helpers[kMostThreads - 1];
    for (int t = 1; t < threads; ++t) {
        const size_t begin = std::min(bytes, size_t(t) * part), end = std::min(bytes, begin + part);
        helpers[t - 1] = std::thread([=] { std::memcpy(to + begin, from + begin, end - begin); });
    }
    std::memcpy(to, from, std::min(bytes, part));
    for (int t = 1; t < threads; ++t) helpers[t - 1].join();
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

// Runs work(begin, end) over [0, count) on eight threads when the count is large, else on this one; each
// share is contiguous and the shares do not overlap.
template <class F>
void split_work(int64_t count, F &&work) {
    constexpr int kThreads = 8;
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

// The batch's longest reference and longest query.
void shape_maxima(int64_t pairs, const int64_t *offsets, uint32_t *max_rows, uint32_t *max_columns) {
    std::atomic<uint32_t> rows{0}, columns{0};
    split_work(pairs, [&](int64_t begin, int64_t end) {
        uint32_t r = 0, c = 0;
        for (int64_t p = begin; p < end; ++p) {
            r = std::max<uint32_t>(r, uint32_t(offsets[2 * p + 1] - offsets[2 * p]));
            c = std::max<uint32_t>(c, uint32_t(offsets[2 * p + 2] - offsets[2 * p + 1]));
        }
        for (uint32_t seen = rows.load(); seen < r && !rows.compare_exchange_weak(seen, r);) {
        }
        for (uint32_t seen = columns.load(); seen < c && !columns.compare_exchange_weak(seen, c);) {
        }
    });
    *max_rows = rows.load();
    *max_columns = columns.load();
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
    shape_maxima(pairs, offsets, &out.max_rows, &out.max_columns);
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
    pack_pairs(gpu, letters_device, offsets_device, 0, pairs, codes_device, bits, out.tape, out.shapes, out.unknown);
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

// Per-pair statuses of pairs [first, first + count): scores that could pass 2^28 (-3), then a walk that
// left its band (-8), then a letter outside the alphabet (-1); `unknown_host` holds the range's flags.
void statuses_of(const CheckedScoring &checked, bool local, int64_t first, int64_t count, const int64_t *offsets,
                 const uint8_t *unknown_host, int64_t *statuses) {
    if (!statuses) return;
    split_work(count, [&](int64_t begin, int64_t end) {
        for (int64_t p = first + begin; p < first + end; ++p) {
            const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
            const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
            const int64_t letters = local ? std::min(rows, columns) : rows + columns;
            int64_t status = 0;
            if (checked.reach_opening + 2 * (letters + 2) * checked.reach_step >= (int64_t(1) << 28))
                status = DINARA_INVALID_COSTS;
            else if (unknown_host[p - first] == kWalkFailed)
                status = DINARA_DEVICE_FAILURE;  // a walk whose path left its proven band
            else if (unknown_host[p - first])
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

// A large batch runs as units of pairs, each packed, swept and walked while later units' letters are
// still crossing the bus and earlier units' results are being moved into the caller's buffers.

// Letters go to the device in pieces of this size.
constexpr size_t kUploadPiece = size_t(32) << 20;
// A batch runs in at most this many units, each of at least kUnitPairs pairs: fewer and the first
// upload and the last unit's moves stand out; more and the units' fixed costs (schedules, host waits,
// the tails of the sweeps) do.
constexpr int64_t kMaxUnits = 8;
constexpr int64_t kUnitPairs = 32768;
// Units run on this many lanes: the context, its partner, the partner's partner, and so on.
constexpr size_t kLanes = 4;
constexpr size_t kMaxLanes = 4;
// Units (and lanes) of a streamed distance batch.
constexpr int64_t kDistanceUnits = 2;

// The caller's letters copied to the device a piece at a time on the context's upload stream. From
// page-locked memory every piece is queued at once; from pageable memory a helper thread stages each
// piece through page-locked memory (an eight-thread copy) and queues it.
class LetterUpload {
  public:
    LetterUpload(dinara_gpu *gpu, uint8_t *device, const uint8_t *host, size_t bytes)
        : gpu_(gpu), device_(device), host_(host), bytes_(bytes) {
        events_.assign((bytes + kUploadPiece - 1) / kUploadPiece, nullptr);
        DINARA_CUDA(cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming));
        for (cudaEvent_t &event : events_) DINARA_CUDA(cudaEventCreateWithFlags(&event, cudaEventDisableTiming));
        // The copies come after what the context's stream did before: the buffer's allocation and
        // earlier calls' reads of it.
        DINARA_CUDA(cudaEventRecord(ready_, gpu->stream));
        DINARA_CUDA(cudaStreamWaitEvent(gpu->upload, ready_, 0));
        if (events_.empty()) return;
        if (is_pinned(host)) {
            for (size_t piece = 0; piece < events_.size(); ++piece) queue(piece, host + piece * kUploadPiece);
            queued_ = events_.size();
            return;
        }
        stage_ = gpu->pinned_in.ensure<uint8_t>(std::min(bytes, 2 * kUploadPiece));
        helper_ = std::thread([this] { stage_all(); });
    }

    ~LetterUpload() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        if (helper_.joinable()) helper_.join();
        // Later work on the context's stream (the buffer's next growth, the next call's copies) comes
        // after every queued copy.
        if (queued_ > 0) cudaStreamWaitEvent(gpu_->stream, events_[queued_ - 1], 0);
        for (cudaEvent_t event : events_)
            if (event) cudaEventDestroy(event);
        if (ready_) cudaEventDestroy(ready_);
    }

    // Makes `stream` wait until letters [0, end) are on the device.
    void wait_for(size_t end, cudaStream_t stream) {
        if (end == 0 || events_.empty()) return;
        const size_t piece = std::min(events_.size(), (end + kUploadPiece - 1) / kUploadPiece) - 1;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            ready_cv_.wait(lock, [&] { return queued_ > piece || failure_; });
            if (failure_) std::rethrow_exception(failure_);
        }
        DINARA_CUDA(cudaStreamWaitEvent(stream, events_[piece], 0));
    }

  private:
    void queue(size_t piece, const uint8_t *from) {
        const size_t at = piece * kUploadPiece, n = std::min(kUploadPiece, bytes_ - at);
        DINARA_CUDA(cudaMemcpyAsync(device_ + at, from, n, cudaMemcpyHostToDevice, gpu_->upload));
        DINARA_CUDA(cudaEventRecord(events_[piece], gpu_->upload));
    }

    void stage_all() {
        try {
            DINARA_CUDA(cudaSetDevice(gpu_->device));
            for (size_t piece = 0; piece < events_.size(); ++piece) {
                {
                    std::lock_guard<std::mutex> lock(mutex_);
                    if (stop_) return;
                }
                uint8_t *buffer = stage_ + (piece & 1) * kUploadPiece;
                // This half's previous copy has left it.
                if (piece >= 2) DINARA_CUDA(cudaEventSynchronize(events_[piece - 2]));
                const size_t at = piece * kUploadPiece;
                // Eight threads: from pageable memory this copy, not the bus, sets the upload's pace.
                parallel_copy(buffer, host_ + at, std::min(kUploadPiece, bytes_ - at), 8);
                queue(piece, buffer);
                {
                    std::lock_guard<std::mutex> lock(mutex_);
                    queued_ = piece + 1;
                }
                ready_cv_.notify_all();
            }
        } catch (...) {
            std::lock_guard<std::mutex> lock(mutex_);
            failure_ = std::current_exception();
            ready_cv_.notify_all();
        }
    }

    dinara_gpu *gpu_;
    uint8_t *device_;
    const uint8_t *host_;
    size_t bytes_;
    uint8_t *stage_ = nullptr;
    cudaEvent_t ready_ = nullptr;
    std::vector<cudaEvent_t> events_;
    std::mutex mutex_;
    std::condition_variable ready_cv_;
    size_t queued_ = 0;
    bool stop_ = false;
    std::exception_ptr failure_;
    std::thread helper_;
};

// A batch cut into contiguous units by letters (at most kMaxUnits, each of at least kUnitPairs pairs; one
// unit when `split` is false), none of whose recorded decisions pass `budget_words` when `budgeted` (a
// pair's decision words from `words_of`). The first and last units take half the letters of the others:
// the first one's letters arrive sooner, and the last one's results leave sooner. When the whole batch's
// decisions fit the budget, as they mostly do, the cuts are binary searches over the offsets.
template <class W>
std::vector<std::pair<int64_t, int64_t>> plan_units(int64_t pairs, const int64_t *offsets, bool split, W &&words_of,
                                                    bool budgeted, int64_t budget_words,
                                                    int64_t most_units = kMaxUnits) {
    const int64_t letters = offsets[2 * pairs] - offsets[0];
    const int64_t units = split ? std::min(most_units, std::max<int64_t>(1, pairs / kUnitPairs)) : 1;
    // Unit u ends where the share of letters of units 0..u does: halves at both ends.
    auto share_end = [&](int64_t u) {
        if (u >= units) return letters;
        const double whole = double(units - 1), before = 0.5 + double(u - 1);
        return int64_t(double(letters) * before / whole);
    };
    std::vector<std::pair<int64_t, int64_t>> out;
    std::atomic<int64_t> all_words{0};
    if (budgeted)
        split_work(pairs, [&](int64_t begin, int64_t end) {
            int64_t sum = 0;
            for (int64_t p = begin; p < end; ++p) sum += words_of(p);
            all_words += sum;
        });
    if (!budgeted || all_words.load() <= budget_words) {
        int64_t first = 0;
        for (int64_t u = 1; u <= units && first < pairs; ++u) {
            // The unit ends at the first pair starting at or past its share of the letters.
            int64_t low = first + 1, high = pairs;
            const int64_t goal = offsets[0] + share_end(u);
            while (low < high) {
                const int64_t middle = low + (high - low) / 2;
                if (offsets[2 * middle] >= goal)
                    high = middle;
                else
                    low = middle + 1;
            }
            const int64_t end = u == units ? pairs : low;
            out.emplace_back(first, end - first);
            first = end;
        }
        return out;
    }
    const int64_t target = (letters + units - 1) / units;
    int64_t first = 0;
    while (first < pairs) {
        int64_t count = 0, w = 0;
        const int64_t start = offsets[2 * first];
        while (first + count < pairs) {
            const int64_t p = first + count;
            const int64_t wp = words_of(p);
            if (count > 0 && (offsets[2 * p] - start >= target || w + wp > budget_words)) break;
            w += wp;
            ++count;
        }
        out.emplace_back(first, count);
        first += count;
    }
    return out;
}

// Where a unit's results sit in its page-locked stage: CIGAR bytes, their offsets (count + 1), scores,
// unknown-letter flags and, for local alignments, the walk's spans (4 a pair).
struct StageLayout {
    size_t cigars = 0, cigar_offsets = 0, scores = 0, unknown = 0, spans = 0, bytes = 0;
    StageLayout(int64_t count, int64_t total, bool with_spans) {
        auto up = [](size_t n) { return (n + 255) & ~size_t(255); };
        cigar_offsets = up(size_t(total));
        scores = cigar_offsets + up(size_t(count + 1) * sizeof(int64_t));
        unknown = scores + up(size_t(count) * sizeof(int32_t));
        spans = unknown + up(size_t(count));
        bytes = spans + (with_spans ? size_t(4 * count) * sizeof(int64_t) : 0);
    }
};

// A unit whose copies into a stage are queued.
struct StagedUnit {
    int64_t first = 0, count = 0, total = 0;
    const uint8_t *stage = nullptr;
    StageLayout layout{0, 0, false};
};

// Units' results moved from their stages into the caller's buffers in the units' order: by a helper
// thread when the batch has more than one unit, so that work runs alongside later units' sweeps, else
// on the caller's thread. Unit k writes stage k mod kStages, which it may do once unit k - kStages is
// done. Units may be pushed out of order (from two lanes). The events that follow each unit's copies
// are made and destroyed on the caller's thread: a destroy on the helper would wait on the driver
// while the lanes call into it.
class UnitFinisher {
  public:
    using Work = std::function<void(const StagedUnit &)>;
    UnitFinisher(dinara_gpu *gpu, size_t units, Work work)
        : gpu_(gpu), work_(std::move(work)), pending_(units), arrived_(units, false), done_(units, nullptr) {
        for (cudaEvent_t &event : done_) DINARA_CUDA(cudaEventCreateWithFlags(&event, cudaEventDisableTiming));
        if (units > 1) helper_ = std::thread([this] { run(); });
    }

    ~UnitFinisher() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            abandon_ = true;
        }
        cv_.notify_all();
        if (helper_.joinable()) helper_.join();
        for (cudaEvent_t event : done_)
            if (event) cudaEventDestroy(event);
    }

    // The stage unit `index` is to write, once it is free.
    uint8_t *stage_for(int64_t index, size_t bytes) {
        {
            std::unique_lock<std::mutex> lock(mutex_);
            cv_.wait(lock, [&] { return finished_ + dinara_gpu::kStages > index || failure_; });
            if (failure_) std::rethrow_exception(failure_);
        }
        return gpu_->stages[index % dinara_gpu::kStages].ensure<uint8_t>(bytes);
    }

    // Takes unit `index`, whose copies are queued on `stream`.
    void push(int64_t index, const StagedUnit &unit, cudaStream_t stream) {
        DINARA_CUDA(cudaEventRecord(done_[size_t(index)], stream));
        if (!helper_.joinable()) {
            finish_one(size_t(index), unit);
            ++finished_;
            return;
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            pending_[size_t(index)] = unit;
            arrived_[size_t(index)] = true;
        }
        cv_.notify_all();
    }

    // Stops the units' moves after a lane's failure; waiters rethrow it.
    void fail(std::exception_ptr failure) {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            if (!failure_) failure_ = failure;
        }
        cv_.notify_all();
    }

    // Waits until every unit is in the caller's buffers; rethrows a failure.
    void finish() {
        if (helper_.joinable()) helper_.join();
        if (failure_) std::rethrow_exception(failure_);
    }

  private:
    void finish_one(size_t index, const StagedUnit &unit) {
        DINARA_CUDA(cudaEventSynchronize(done_[index]));
        work_(unit);
    }

    void run() {
        try {
            DINARA_CUDA(cudaSetDevice(gpu_->device));
            for (size_t next = 0; next < pending_.size(); ++next) {
                StagedUnit unit;
                {
                    std::unique_lock<std::mutex> lock(mutex_);
                    cv_.wait(lock, [&] { return arrived_[next] || failure_ || abandon_; });
                    if (failure_ || abandon_) return;
                    unit = pending_[next];
                }
                finish_one(next, unit);
                {
                    std::lock_guard<std::mutex> lock(mutex_);
                    ++finished_;
                }
                cv_.notify_all();
            }
        } catch (...) {
            fail(std::current_exception());
        }
    }

    dinara_gpu *gpu_;
    Work work_;
    std::mutex mutex_;
    std::condition_variable cv_;
    std::vector<StagedUnit> pending_;
    std::vector<bool> arrived_;
    std::vector<cudaEvent_t> done_;
    int64_t finished_ = 0;
    bool abandon_ = false;
    std::exception_ptr failure_;
    std::thread helper_;
};

// Room for a batch's CIGARs taken at once, so that they never move as units arrive: `bound` bytes, which
// an allocation this large takes as address space, mapped (with large pages where the system allows)
// as the copies first touch it. Left empty, to grow a unit at a time, when the address space is refused.
void reserve_cigars(std::unique_ptr<char, void (*)(void *)> &bytes, size_t &room, size_t bound) {
    char *reserved = static_cast<char *>(std::malloc(bound));
    if (!reserved) return;
    bytes.reset(reserved);
    room = bound;
    const uintptr_t huge = uintptr_t(2) << 20;
    const uintptr_t begin = (reinterpret_cast<uintptr_t>(reserved) + huge - 1) & ~(huge - 1);
    const uintptr_t end = (reinterpret_cast<uintptr_t>(reserved) + bound) & ~(huge - 1);
    if (end > begin) madvise(reinterpret_cast<void *>(begin), size_t(end - begin), MADV_HUGEPAGE);
}

// A batch whose letters are on their way to the device a piece at a time, with its packed form's buffers:
// pack_unit packs a unit of pairs once its letters are there.
struct StreamedBatch {
    Packed packed;
    int64_t base = 0;  // the batch's first letter in the caller's tape
    int bits = 0;
    const uint8_t *letters_device = nullptr;
    const int64_t *offsets_device = nullptr;
    const uint8_t *codes_device = nullptr;
    int32_t *scores = nullptr;  // every pair's score on the device
    std::unique_ptr<LetterUpload> upload;
    // Follows the buffers' allocations and the offsets' and codes' copies on the batch's context's stream.
    cudaEvent_t inputs_ready = nullptr;

    StreamedBatch() = default;
    StreamedBatch(const StreamedBatch &) = delete;
    StreamedBatch &operator=(const StreamedBatch &) = delete;
    ~StreamedBatch() {
        upload.reset();
        if (inputs_ready) cudaEventDestroy(inputs_ready);
    }

    // Packs a unit on `ctx`'s stream (the batch's context or its partner) once its letters are there.
    void pack_unit(dinara_gpu *ctx, const int64_t *offsets, int64_t first, int64_t count) {
        upload->wait_for(size_t(offsets[2 * (first + count)] - base), ctx->stream);
        pack_pairs(ctx, letters_device, offsets_device, first, count, codes_device, bits, packed.tape, packed.shapes,
                   packed.unknown);
    }
};

void start_batch(StreamedBatch &out, dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                 const uint8_t codes[256], int bits) {
    out.packed.pairs = pairs;
    out.base = offsets[0];
    out.bits = bits;
    const int64_t total = offsets[2 * pairs] - out.base;
    // The code table is copied only when it changes: it comes from pageable memory, a copy the host
    // waits for, behind whatever is queued before it.
    const bool new_codes = !gpu->code_table.ptr || std::memcmp(gpu->codes_host, codes, 256) != 0;
    uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
    int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
    uint8_t *codes_device = gpu->code_table.ensure<uint8_t>(256);
    if (new_codes) {
        DINARA_CUDA(cudaMemcpyAsync(codes_device, codes, 256, cudaMemcpyHostToDevice, gpu->stream));
        std::memcpy(gpu->codes_host, codes, 256);
    }
    out.packed.tape = gpu->tape.ensure<uint32_t>(size_t(packed_words_total(total, 2 * pairs, bits)));
    out.packed.shapes = gpu->shapes.ensure<PairShape>(size_t(pairs));
    out.packed.unknown = gpu->flags.ensure<uint8_t>(size_t(pairs));
    out.scores = gpu->scores.ensure<int32_t>(size_t(pairs));
    out.letters_device = letters_device;
    out.offsets_device = offsets_device;
    out.codes_device = codes_device;
    // The offsets (from the batch's first letter) on the context's stream, then the letters on the upload
    // stream: copies in one direction share the copy engines in the order they are queued, so the small
    // ones go first.
    std::vector<int64_t> relative;
    const int64_t *device_offsets_host = offsets;
    if (out.base != 0) {
        relative.resize(size_t(2 * pairs + 1));
        split_work(2 * pairs + 1, [&](int64_t begin, int64_t end) {
            for (int64_t k = begin; k < end; ++k) relative[size_t(k)] = offsets[k] - out.base;
        });
        device_offsets_host = relative.data();
    }
    to_device(gpu, offsets_device, device_offsets_host, size_t(2 * pairs + 1) * sizeof(int64_t), gpu->pinned_small);
    DINARA_CUDA(cudaEventCreateWithFlags(&out.inputs_ready, cudaEventDisableTiming));
    DINARA_CUDA(cudaEventRecord(out.inputs_ready, gpu->stream));
    out.upload = std::make_unique<LetterUpload>(gpu, letters_device,
                                                reinterpret_cast<const uint8_t *>(letters) + out.base, size_t(total));
    shape_maxima(pairs, offsets, &out.packed.max_rows, &out.packed.max_columns);
}

// The context's partner, set up at its first use and freed with the context.
dinara_gpu *partner_of(dinara_gpu *gpu) {
    if (!gpu->partner) {
        gpu->partner = dinara_gpu_new(gpu->device);
        if (!gpu->partner) throw Failure(DINARA_DEVICE_FAILURE, "a second stream for a batch's units: " + new_error);
    }
    return gpu->partner;
}

// Runs body(ctx, k) for every unit k of a batch. With more than one lane (and unit), units go round the
// context and its chain of partners (each a stream with scratch buffers of its own), each lane driven by
// its own thread, so that one unit's latency-bound phases (the last pairs of a sweep, the walk, copies
// and host waits) overlap other units' sweeps.
template <class F>
void run_units(dinara_gpu *gpu, const StreamedBatch &streamed, size_t units, size_t lanes, UnitFinisher &finisher,
               F &&body) {
    lanes = std::min({lanes, kMaxLanes, std::max<size_t>(units, 1)});
    dinara_gpu *contexts[kMaxLanes] = {gpu};
    for (size_t l = 1; l < lanes; ++l) contexts[l] = partner_of(contexts[l - 1]);
    std::exception_ptr failures[kMaxLanes];
    auto lane = [&](size_t l) {
        try {
            dinara_gpu *ctx = contexts[l];
            AllocationScope scope(ctx->stream);
            DINARA_CUDA(cudaSetDevice(gpu->device));
            if (ctx != gpu) DINARA_CUDA(cudaStreamWaitEvent(ctx->stream, streamed.inputs_ready, 0));
            for (size_t k = l; k < units; k += lanes) body(ctx, k);
        } catch (...) {
            failures[l] = std::current_exception();
            finisher.fail(failures[l]);
        }
    };
    std::thread helpers[kMaxLanes];
    for (size_t l = 1; l < lanes; ++l) helpers[l] = std::thread(lane, l);
    lane(0);
    for (size_t l = 1; l < lanes; ++l) helpers[l].join();
    for (size_t l = 1; l < lanes; ++l) {
        // Later work on the context's stream comes after everything the partners queued.
        cudaEvent_t joined = nullptr;
        if (cudaEventCreateWithFlags(&joined, cudaEventDisableTiming) == cudaSuccess) {
            if (cudaEventRecord(joined, contexts[l]->stream) == cudaSuccess) cudaStreamWaitEvent(gpu->stream, joined, 0);
            cudaEventDestroy(joined);
        } else {
            cudaStreamSynchronize(contexts[l]->stream);
        }
    }
    for (std::exception_ptr &failure : failures)
        if (failure) std::rethrow_exception(failure);
}

// The resident batch: packed letters kept on the device between calls. It owns its buffers (taken over
// from the context once loaded) and its results, so the context's other calls, which reuse the context's
// buffers, leave it as it was.
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
    // The cuts of a recording pass (global, then local), planned at the first one.
    std::vector<std::pair<int64_t, int64_t>> plans[2];
    dinara::DeviceBuffer held_letters, held_offsets, held_tape, held_shapes, held_flags, results;
};

// Frees a resident batch, its buffers ordered on the calling scope's allocation stream.
void free_resident(void *pointer) {
    Resident *r = static_cast<Resident *>(pointer);
    for (dinara::DeviceBuffer *buffer :
         {&r->held_letters, &r->held_offsets, &r->held_tape, &r->held_shapes, &r->held_flags, &r->results})
        buffer->release();
    delete r;
}

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
        gpu->band_cells = gpu->whole_cells = 0;
        gpu->clock_used = 0;
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
            for (int k = 0; k < 8; ++k) {
                timing->class_ms[k] = 0.0;
                timing->class_launches[k] = 0;
            }
            timing->band_cells = gpu->band_cells;
            timing->whole_cells = gpu->whole_cells;
            for (int slot = 0; slot < gpu->clock_used; ++slot) {
                float span = 0.f;
                DINARA_CUDA(cudaEventElapsedTime(&span, gpu->clock_events[2 * slot], gpu->clock_events[2 * slot + 1]));
                timing->class_ms[gpu->clock_class[slot]] += span;
                timing->class_launches[gpu->clock_class[slot]] += 1;
            }
        }
    }
    ~Timer() {
        gpu->timing = false;
        if (begin) cudaEventDestroy(begin);
        if (end) cudaEventDestroy(end);
    }
};

// The learned band's first thresholds, with the device time they took.
// A partner context takes its context's band tuning and trained predictor (the parameters copied on the
// context's stream), so that a unit it runs chooses windows and first thresholds as the context would.
void share_band_state(dinara_gpu *from, dinara_gpu *to) {
    to->band_tuning = from->band_tuning;
    to->predictor_ready = from->predictor_ready;
    for (int k = 0; k < 4; ++k) to->predictor_margins[k] = from->predictor_margins[k];
    to->predictor_margin = from->predictor_margin;
    to->predictor_slack = from->predictor_slack;
    if (from->predictor_ready) {
        float *parameters = to->weights.ensure<float>(size_t(kPredictorParameters));
        DINARA_CUDA(cudaMemcpyAsync(parameters, from->weights.as<float>(), size_t(kPredictorParameters) * sizeof(float),
                                    cudaMemcpyDeviceToDevice, from->stream));
    }
}

// Adds a unit's band report to the batch's.
void add_band_report(dinara_band_report &into, const dinara_band_report &unit) {
    into.rounds += unit.rounds;
    into.pair_rounds += unit.pair_rounds;
    into.words_swept += unit.words_swept;
    into.first_round_hits += unit.first_round_hits;
    into.overshoot += unit.overshoot;
    into.undershoot += unit.undershoot;
    into.kernel_ms += unit.kernel_ms;
    into.predict_ms += unit.predict_ms;
    for (int r = 0; r < 16; ++r) {
        into.round_pairs[r] += unit.round_pairs[r];
        into.round_launches[r] += unit.round_launches[r];
        into.round_ms[r] += unit.round_ms[r];
    }
}

const int64_t *timed_predictions(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                                 double *ms) {
    DINARA_CUDA(cudaEventRecord(gpu->start, gpu->stream));
    ClockSpan clock(gpu, kClassPredict, gpu->stream);
    const int64_t *starts = predict_thresholds(gpu, pairs, letters, offsets);
    clock.stop();
    DINARA_CUDA(cudaEventRecord(gpu->stop, gpu->stream));
    DINARA_CUDA(cudaEventSynchronize(gpu->stop));
    float elapsed = 0.f;
    DINARA_CUDA(cudaEventElapsedTime(&elapsed, gpu->start, gpu->stop));
    *ms = elapsed;
    return starts;
}

// Distances of a batch of several units (kDistanceUnits at most), its letters streamed: the letters go up
// in pieces on the upload stream while the first unit runs, each unit (its first thresholds, then its band
// doubling) starting once its letters are there, on a lane of its own (the context or its partner, each
// with its stream and scratch). A unit's rounds are bound by its longest pairs' chains of word steps, so
// the call takes about the last unit's upload and its chains; on the uneven batch (1.5 GB, 27 ms to
// upload) two units on two lanes measured 65 ms against 78 unstreamed, and more units or lanes no
// better (six lanes 85 ms: their predictions and rounds crowd each other). Every distance is the one band doubling gives the whole batch: a pair's rounds depend on
// that pair alone.
void streamed_distances(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                        const std::vector<int64_t> &relative, const dinara_band_plan *plan,
                        const std::vector<std::pair<int64_t, int64_t>> &units, int64_t *results,
                        dinara_band_report *report) {
    const int64_t policy = plan ? plan->policy : DINARA_BAND_PLAIN;
    const int64_t first_letter = offsets[0];
    const int64_t total = offsets[2 * pairs] - first_letter;
    uint8_t *letters_device = gpu->letters.as<uint8_t>();
    int64_t *offsets_device = gpu->offsets.as<int64_t>();
    int64_t *results_device = gpu->scores.ensure<int64_t>(size_t(pairs));
    to_device(gpu, offsets_device, relative.data(), relative.size() * sizeof(int64_t), gpu->pinned_small);
    int64_t *given = nullptr;
    if (policy == DINARA_BAND_GIVEN) {
        given = gpu->predictions.ensure<int64_t>(size_t(pairs));
        to_device(gpu, given, plan->start_thresholds, size_t(pairs) * sizeof(int64_t), gpu->pinned_small);
    }
    const size_t lanes = std::min(size_t(kDistanceUnits), units.size());
    dinara_gpu *contexts[kDistanceUnits] = {gpu};
    for (size_t l = 1; l < lanes; ++l) {
        contexts[l] = partner_of(contexts[l - 1]);
        share_band_state(gpu, contexts[l]);
    }
    cudaEvent_t inputs_ready = nullptr;
    DINARA_CUDA(cudaEventCreateWithFlags(&inputs_ready, cudaEventDisableTiming));
    DINARA_CUDA(cudaEventRecord(inputs_ready, gpu->stream));
    std::vector<dinara_band_report> unit_reports(units.size());
    for (dinara_band_report &r : unit_reports) std::memset(&r, 0, sizeof r);
    std::exception_ptr failures[kDistanceUnits];
    {
        LetterUpload upload(gpu, letters_device, reinterpret_cast<const uint8_t *>(letters) + first_letter,
                            size_t(total));
        auto lane = [&](size_t l) {
            try {
                dinara_gpu *ctx = contexts[l];
                AllocationScope scope(ctx->stream);
                DINARA_CUDA(cudaSetDevice(gpu->device));
                if (ctx != gpu) DINARA_CUDA(cudaStreamWaitEvent(ctx->stream, inputs_ready, 0));
                for (size_t k = l; k < units.size(); k += lanes) {
                    const int64_t first = units[k].first, count = units[k].second;
                    upload.wait_for(size_t(offsets[2 * (first + count)] - first_letter), ctx->stream);
                    const int64_t *unit_offsets = offsets_device + 2 * first;
                    const int64_t *starts = nullptr;
                    double predict_ms = 0.0;
                    if (policy == DINARA_BAND_GIVEN)
                        starts = given + first;
                    else if (policy == DINARA_BAND_LEARNED)
                        starts = timed_predictions(ctx, count, letters_device, unit_offsets, &predict_ms);
                    band_doubling(ctx, count, letters_device, unit_offsets, starts, plan ? plan->default_start : 0,
                                  results_device + first, report ? &unit_reports[k] : nullptr);
                    unit_reports[k].predict_ms = predict_ms;
                }
            } catch (...) {
                failures[l] = std::current_exception();
            }
        };
        std::thread helpers[kDistanceUnits];
        for (size_t l = 1; l < lanes; ++l) helpers[l] = std::thread(lane, l);
        lane(0);
        for (size_t l = 1; l < lanes; ++l) helpers[l].join();
        for (size_t l = 1; l < lanes; ++l) {
            // The results' copy waits for every partner's units.
            cudaEvent_t joined = nullptr;
            if (cudaEventCreateWithFlags(&joined, cudaEventDisableTiming) == cudaSuccess) {
                if (cudaEventRecord(joined, contexts[l]->stream) == cudaSuccess)
                    cudaStreamWaitEvent(gpu->stream, joined, 0);
                cudaEventDestroy(joined);
            } else {
                cudaStreamSynchronize(contexts[l]->stream);
            }
        }
    }
    cudaEventDestroy(inputs_ready);
    for (std::exception_ptr &failure : failures)
        if (failure) std::rethrow_exception(failure);
    to_host_now(gpu, results, results_device, size_t(pairs) * sizeof(int64_t));
    if (report) {
        for (const dinara_band_report &r : unit_reports) add_band_report(*report, r);
        int64_t cells = 0;
        for (int64_t p = 0; p < pairs; ++p)
            cells += (offsets[2 * p + 1] - offsets[2 * p]) * (offsets[2 * p + 2] - offsets[2 * p + 1]);
        report->full_cells = cells;
    }
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
        DINARA_CUDA(cudaStreamCreateWithFlags(&gpu->upload, cudaStreamNonBlocking));
        DINARA_CUDA(cudaMallocHost(&gpu->readback, dinara::kReadbackBytes));
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
    if (gpu->partner) dinara_gpu_free(gpu->partner);
    gpu->partner = nullptr;
    cudaSetDevice(gpu->device);
    AllocationScope scope(gpu->stream);
    if (gpu->stream) cudaStreamSynchronize(gpu->stream);
    if (gpu->upload) cudaStreamSynchronize(gpu->upload);
    if (gpu->resident) gpu->resident_free(gpu->resident);
    gpu->for_each_buffer([](dinara::DeviceBuffer &buffer) { buffer.release(); });
    if (gpu->stream) cudaStreamSynchronize(gpu->stream);
    gpu->pinned_in.release();
    gpu->pinned_out.release();
    gpu->pinned_small.release();
    for (dinara::PinnedBuffer &stage : gpu->stages) stage.release();
    if (gpu->readback) cudaFreeHost(gpu->readback);
    if (gpu->start) cudaEventDestroy(gpu->start);
    if (gpu->stop) cudaEventDestroy(gpu->stop);
    if (gpu->fork) cudaEventDestroy(gpu->fork);
    for (cudaEvent_t event : gpu->clock_events)
        if (event) cudaEventDestroy(event);
    for (int k = 0; k < dinara_gpu::kSideStreams; ++k) {
        if (gpu->side[k]) cudaStreamDestroy(gpu->side[k]);
        if (gpu->joins[k]) cudaEventDestroy(gpu->joins[k]);
    }
    if (gpu->upload) cudaStreamDestroy(gpu->upload);
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

}  // extern "C"

namespace {

// Scores of a tape's pairs (dinara_gpu_scores_tape's work); with free ends and `spans` (host, 4 a pair),
// also each pair's span as the reference places it (affine_scores).
void run_scores(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores, int64_t *statuses,
                int64_t *spans) {
    if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
    AffineBatch ends;
    const bool local = check_scores_mode(mode, ends);
    const CheckedScoring checked = check_scoring(scoring, local);
    check_offsets(pairs, offsets);
    if (pairs == 0) return;
    if (!ends.free_ends) spans = nullptr;
    DINARA_CUDA(cudaSetDevice(gpu->device));
    StreamedBatch streamed;
    start_batch(streamed, gpu, pairs, letters, offsets, checked.codes, checked.bits);
    const Packed &packed = streamed.packed;
    AffineBatch batch{pairs, checked.bits, local, packed.tape, packed.shapes, packed.max_rows, packed.max_columns};
    batch.free_ends = ends.free_ends;
    batch.free_reference_start = ends.free_reference_start;
    batch.free_reference_end = ends.free_reference_end;
    batch.free_query_start = ends.free_query_start;
    batch.free_query_end = ends.free_query_end;
    batch.extension = ends.extension;
    batch.from_end = ends.from_end;
    batch.zdrop = ends.zdrop;
    batch.end_bonus = ends.end_bonus;
    int32_t *scores_device = streamed.scores;
    const auto units = plan_units(pairs, offsets, true, [](int64_t) { return int64_t(0); }, false, 0);
    UnitFinisher finisher(gpu, units.size(), [&](const StagedUnit &unit) {
        std::memcpy(scores + unit.first, unit.stage + unit.layout.scores, size_t(unit.count) * sizeof(int32_t));
        if (spans)
            std::memcpy(spans + 4 * unit.first, unit.stage + unit.layout.spans,
                        size_t(4 * unit.count) * sizeof(int64_t));
        statuses_of(checked, local, unit.first, unit.count, offsets, unit.stage + unit.layout.unknown, statuses);
    });
    run_units(gpu, streamed, units.size(), kLanes, finisher, [&](dinara_gpu *ctx, size_t k) {
        const int64_t first = units[k].first, count = units[k].second;
        streamed.pack_unit(ctx, offsets, first, count);
        int64_t *spans_device = spans ? ctx->ranges.ensure<int64_t>(size_t(4 * count)) : nullptr;
        affine_scores(ctx, batch, checked.table, scores_device, first, count, spans_device);
        StagedUnit unit;
        unit.first = first;
        unit.count = count;
        unit.layout = StageLayout(count, 0, spans != nullptr);
        uint8_t *stage = finisher.stage_for(int64_t(k), unit.layout.bytes);
        unit.stage = stage;
        DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.scores, scores_device + first,
                                    size_t(count) * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.unknown, packed.unknown + first, size_t(count),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        if (spans)
            DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.spans, spans_device, size_t(4 * count) * sizeof(int64_t),
                                        cudaMemcpyDeviceToHost, ctx->stream));
        finisher.push(int64_t(k), unit, ctx->stream);
    });
    finisher.finish();
}

// Whether a mode asks a Scoring for free ends (ends_free with any letters free, no match score) or for an
// extension: alignments whose span a sweep places before the span's letters are aligned globally.
bool free_end_mode(const dinara_mode *mode) {
    if (mode && mode->kind == DINARA_EXTENSION) return true;
    return mode && mode->kind == DINARA_ENDS_FREE && mode->match_score <= 0 &&
           (mode->reference_start | mode->reference_end | mode->query_start | mode->query_end) != 0;
}

// Alignments with free ends or as extensions under a Scoring, as the reference's host path makes them
// (scoring.mojo:800-813): each pair's score and span from the free-end or extension sweeps (run_scores;
// an extension's Z-drop and end bonus on the device), then the span's letters aligned globally
// (dinara_gpu_alignments_tape), whose CIGAR is the alignment's. A pair whose span's global score differs
// from its free-end score, or whose span is out of its letters, reports a device failure.
void free_end_alignments(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                         const dinara_scoring *scoring, const dinara_mode *mode, int64_t eqx, int32_t *scores,
                         int64_t *spans, int64_t *cigar_offsets, char **cigar_bytes, int64_t *statuses) {
    const size_t room = size_t(std::max<int64_t>(pairs, 1));
    std::vector<int64_t> own_spans(spans ? 0 : 4 * room);
    int64_t *placed = spans ? spans : own_spans.data();
    std::vector<int64_t> first_statuses(room, 0);
    run_scores(gpu, pairs, letters, offsets, scoring, mode, scores, first_statuses.data(), placed);
    // The spans' letters as a tape of their own.
    std::vector<int64_t> inner_offsets(size_t(2 * pairs + 1), 0);
    std::vector<int64_t> failed(room, 0);
    int64_t total = 0;
    for (int64_t p = 0; p < pairs; ++p) {
        int64_t *span = placed + 4 * p;
        const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
        const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
        if (!(0 <= span[0] && span[0] <= span[1] && span[1] <= rows && 0 <= span[2] && span[2] <= span[3] &&
              span[3] <= columns)) {
            failed[size_t(p)] = 1;
            span[0] = span[1] = span[2] = span[3] = 0;
        }
        inner_offsets[size_t(2 * p)] = total;
        total += span[1] - span[0];
        inner_offsets[size_t(2 * p + 1)] = total;
        total += span[3] - span[2];
    }
    inner_offsets[size_t(2 * pairs)] = total;
    std::vector<char> inner(size_t(std::max<int64_t>(total, 1)));
    split_work(pairs, [&](int64_t begin, int64_t end) {
        for (int64_t p = begin; p < end; ++p) {
            const int64_t *span = placed + 4 * p;
            std::memcpy(inner.data() + inner_offsets[size_t(2 * p)], letters + offsets[2 * p] + span[0],
                        size_t(span[1] - span[0]));
            std::memcpy(inner.data() + inner_offsets[size_t(2 * p + 1)], letters + offsets[2 * p + 1] + span[2],
                        size_t(span[3] - span[2]));
        }
    });
    dinara_mode global = *mode;
    global.kind = DINARA_ENDS_FREE;
    global.reference_start = global.reference_end = global.query_start = global.query_end = 0;
    global.match_score = 0;
    std::vector<int32_t> inner_scores(room, 0);
    std::vector<int64_t> inner_spans(4 * room, 0), inner_statuses(room, 0);
    const int64_t code = dinara_gpu_alignments_tape(gpu, pairs, inner.data(), inner_offsets.data(), scoring, &global,
                                                    eqx, inner_scores.data(), inner_spans.data(), cigar_offsets,
                                                    cigar_bytes, inner_statuses.data());
    if (code != 0) throw Failure(code, gpu->error);
    if (!statuses) return;
    for (int64_t p = 0; p < pairs; ++p) {
        int64_t status = first_statuses[size_t(p)] != 0 ? first_statuses[size_t(p)] : inner_statuses[size_t(p)];
        if (status == 0 && (failed[size_t(p)] || inner_scores[size_t(p)] != scores[p])) status = DINARA_DEVICE_FAILURE;
        statuses[p] = status;
    }
}

}  // namespace

extern "C" {

int64_t dinara_gpu_scores_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                               const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores,
                               int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        run_scores(gpu, pairs, letters, offsets, scoring, mode, scores, statuses, nullptr);
        return 0;
    });
}

int64_t dinara_gpu_scores(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                          const int64_t *reference_lengths, const char *const *queries, const int64_t *query_lengths,
                          const dinara_scoring *scoring, const dinara_mode *mode, int32_t *scores, int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        AffineBatch ends;
        const bool local = check_scores_mode(mode, ends);
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
        if (free_end_mode(mode)) {
            free_end_alignments(gpu, pairs, letters, offsets, scoring, mode, eqx, scores, spans, cigar_offsets,
                                cigar_bytes, statuses);
            return 0;
        }
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
        StreamedBatch streamed;
        start_batch(streamed, gpu, pairs, letters, offsets, checked.codes, checked.bits);
        const Packed &packed = streamed.packed;
        AffineBatch batch{pairs, checked.bits, local, packed.tape, packed.shapes, packed.max_rows, packed.max_columns,
                          packed.unknown};
        int32_t *scores_device = streamed.scores;
        // Units whose recorded decisions stay within a budget of device memory.
        const bool uniform = !checked.table.packed16 || checked.bits == 8;
        const bool band = band_serves(batch, checked.table);
        const auto units = plan_units(
            pairs, offsets, true,
            [&](int64_t p) {
                return record_words(offsets[2 * p + 1] - offsets[2 * p], offsets[2 * p + 2] - offsets[2 * p + 1],
                                    uniform, band);
            },
            true, kDecisionBudget / 8);
        // Every unit's CIGAR bytes go straight into the caller's buffer.
        std::unique_ptr<char, void (*)(void *)> bytes(nullptr, std::free);
        size_t room = 0, size = 0;
        reserve_cigars(bytes, room, 2 * size_t(offsets[2 * pairs] - offsets[0]) + 1);
        if (cigar_offsets) cigar_offsets[0] = 0;
        UnitFinisher finisher(gpu, units.size(), [&](const StagedUnit &unit) {
            if (size + size_t(unit.total) + 1 > room) {
                char *grown = static_cast<char *>(std::realloc(bytes.get(), size + size_t(unit.total) + 1));
                if (!grown) throw std::bad_alloc();
                bytes.release();
                bytes.reset(grown);
                room = size + size_t(unit.total) + 1;
            }
            parallel_copy(reinterpret_cast<uint8_t *>(bytes.get()) + size, unit.stage + unit.layout.cigars,
                          size_t(unit.total));
            const int64_t *ends = reinterpret_cast<const int64_t *>(unit.stage + unit.layout.cigar_offsets);
            const int64_t *walked = reinterpret_cast<const int64_t *>(unit.stage + unit.layout.spans);
            std::memcpy(scores + unit.first, unit.stage + unit.layout.scores, size_t(unit.count) * sizeof(int32_t));
            statuses_of(checked, local, unit.first, unit.count, offsets, unit.stage + unit.layout.unknown, statuses);
            const int64_t at = int64_t(size);
            // Each pair's CIGAR end and spans, a share of the unit's pairs a thread.
            split_work(unit.count, [&](int64_t begin, int64_t end) {
                for (int64_t k = begin; k < end; ++k) {
                    const int64_t p = unit.first + k;
                    if (cigar_offsets) cigar_offsets[p + 1] = at + ends[k + 1];
                    const int64_t rows = offsets[2 * p + 1] - offsets[2 * p];
                    const int64_t columns = offsets[2 * p + 2] - offsets[2 * p + 1];
                    int64_t *span = spans + 4 * p;
                    if (!local) {
                        // A global walk spans the whole pair.
                        span[0] = 0;
                        span[1] = rows;
                        span[2] = 0;
                        span[3] = columns;
                    } else {
                        const int64_t *w = walked + 4 * k;
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
            });
            size += size_t(unit.total);
        });
        run_units(gpu, streamed, units.size(), kLanes, finisher, [&](dinara_gpu *ctx, size_t k) {
            const int64_t first = units[k].first, count = units[k].second;
            streamed.pack_unit(ctx, offsets, first, count);
            int64_t *spans_device = ctx->ranges.ensure<int64_t>(size_t(4 * count));
            StagedUnit unit;
            unit.first = first;
            unit.count = count;
            unit.total = affine_alignments(ctx, batch, checked.table, eqx != 0, scores_device, spans_device, first,
                                           count);
            unit.layout = StageLayout(count, unit.total, local);
            uint8_t *stage = finisher.stage_for(int64_t(k), unit.layout.bytes);
            unit.stage = stage;
            DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.cigars, ctx->cigar_bytes.as<char>(), size_t(unit.total),
                                        cudaMemcpyDeviceToHost, ctx->stream));
            DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.cigar_offsets, ctx->cigar_offsets.as<int64_t>(),
                                        size_t(count + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
            DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.scores, scores_device + first,
                                        size_t(count) * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
            DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.unknown, packed.unknown + first, size_t(count),
                                        cudaMemcpyDeviceToHost, ctx->stream));
            // A global walk spans the whole pair, known on the host; only a local one's spans come back.
            if (local)
                DINARA_CUDA(cudaMemcpyAsync(stage + unit.layout.spans, spans_device,
                                            size_t(4 * count) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                            ctx->stream));
            finisher.push(int64_t(k), unit, ctx->stream);
        });
        finisher.finish();
        if (!bytes) bytes.reset(static_cast<char *>(std::malloc(1)));
        if (!bytes) throw std::bad_alloc();
        if (room > size + 1) {
            // The reservation's untouched rest handed back.
            char *shrunk = static_cast<char *>(std::realloc(bytes.get(), size + 1));
            if (shrunk) {
                bytes.release();
                bytes.reset(shrunk);
            }
        }
        bytes.get()[size] = 0;
        if (cigar_bytes) *cigar_bytes = bytes.release();
        return 0;
    });
}

int64_t dinara_gpu_alignments(dinara_gpu *gpu, int64_t pairs, const char *const *references,
                              const int64_t *reference_lengths, const char *const *queries,
                              const int64_t *query_lengths, const dinara_scoring *scoring, const dinara_mode *mode,
                              int64_t eqx, dinara_alignment *alignments, int64_t *statuses) {
    return guard(gpu, [&]() -> int64_t {
        AffineBatch ends;
        const bool local = free_end_mode(mode) ? check_scores_mode(mode, ends) : check_mode(mode);
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
        const auto units =
            plan_units(pairs, offsets, true, [](int64_t) { return int64_t(0); }, false, 0, kDistanceUnits);
        if (units.size() > 1) {
            streamed_distances(gpu, pairs, letters, offsets, relative, plan, units, results, report);
            return 0;
        }
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
            std::swap(r->held_tape, gpu->tape);
            std::swap(r->held_shapes, gpu->shapes);
            std::swap(r->held_flags, gpu->flags);
        } else {
            const int64_t total = offsets[2 * pairs] - offsets[0];
            uint8_t *letters_device = gpu->letters.ensure<uint8_t>(size_t(total) + 16);
            int64_t *offsets_device = gpu->offsets.ensure<int64_t>(size_t(2 * pairs + 1));
            to_device(gpu, letters_device, letters + offsets[0], size_t(total), gpu->pinned_in);
            to_device(gpu, offsets_device, r->offsets.data(), r->offsets.size() * sizeof(int64_t), gpu->pinned_small);
            r->letters_device = letters_device;
            r->offsets_device = offsets_device;
        }
        std::swap(r->held_letters, gpu->letters);
        std::swap(r->held_offsets, gpu->offsets);
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return 0;
    });
}

int64_t dinara_gpu_resident_align(dinara_gpu *gpu, const dinara_mode *mode, int64_t cigars, int64_t eqx,
                                  dinara_timing *timing) {
    return guard(gpu, [&]() -> int64_t {
        Resident &r = resident_of(gpu);
        if (!r.scoring) throw Failure(DINARA_INVALID_MODE, "the resident batch was loaded for distances");
        AffineBatch ends;
        const bool local = cigars ? check_mode(mode) : check_scores_mode(mode, ends);
        if (r.pairs == 0) return 0;
        DINARA_CUDA(cudaSetDevice(gpu->device));
        Timer timer(gpu);
        AffineBatch batch{r.pairs, r.checked.bits, local, r.packed.tape, r.packed.shapes, r.packed.max_rows,
                          r.packed.max_columns, r.packed.unknown};
        batch.free_ends = ends.free_ends;
        batch.free_reference_start = ends.free_reference_start;
        batch.free_reference_end = ends.free_reference_end;
        batch.free_query_start = ends.free_query_start;
        batch.free_query_end = ends.free_query_end;
        batch.extension = ends.extension;
        batch.from_end = ends.from_end;
        batch.zdrop = ends.zdrop;
        batch.end_bonus = ends.end_bonus;
        int32_t *scores_device = r.results.ensure<int32_t>(size_t(r.pairs));
        const int64_t *offsets = r.offsets.data();
        if (!cigars) {
            affine_scores(gpu, batch, r.checked.table, scores_device, 0, r.pairs);
        } else {
            // The whole batch in one launch sequence, cut only where its decisions would pass the budget;
            // the cuts are planned at the first pass.
            const bool uniform = !r.checked.table.packed16 || r.checked.bits == 8;
            const bool band = band_serves(batch, r.checked.table);
            std::vector<std::pair<int64_t, int64_t>> &units = r.plans[local ? 1 : 0];
            if (units.empty())
                units = plan_units(
                    r.pairs, offsets, false,
                    [&](int64_t p) {
                        return record_words(offsets[2 * p + 1] - offsets[2 * p],
                                            offsets[2 * p + 2] - offsets[2 * p + 1], uniform, band);
                    },
                    true, kDecisionBudget / 8);
            for (const auto &unit : units) {
                int64_t *spans_device = gpu->ranges.ensure<int64_t>(size_t(4 * unit.second));
                affine_alignments(gpu, batch, r.checked.table, eqx != 0, scores_device, spans_device, unit.first,
                                  unit.second);
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
        int64_t *results_device = r.results.ensure<int64_t>(size_t(r.pairs));
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
        if (r.last == 1 && scores) to_host(gpu, scores, r.results.as<int32_t>(), size_t(r.pairs) * sizeof(int32_t));
        if (r.last == 2 && distances)
            to_host(gpu, distances, r.results.as<int64_t>(), size_t(r.pairs) * sizeof(int64_t));
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

// A global mode, as the GPU takes Costs: free ends of none, no match score (null is global).
void check_global(const dinara_mode *mode) {
    if (mode && (mode->kind != DINARA_ENDS_FREE || mode->reference_start || mode->reference_end ||
                 mode->query_start || mode->query_end || mode->match_score))
        throw Failure(DINARA_INVALID_MODE, "on the GPU, Costs align globally");
}

// Whether costs and options are unit costs with no band or cap (api.mojo:1240-1246), which band doubling
// serves; *scale is the factor the costs are of unit costs.
bool unit_costs(const dinara_costs *costs, const dinara_options *options, int64_t *scale) {
    *scale = 1;
    if (options && (options->band_low > INT64_MIN || options->band_high < INT64_MAX || options->max_cost >= 0))
        return false;
    if (!costs) return true;
    const bool symmetric = costs->deletion_extension == 0 ||
                           (costs->deletion_opening == costs->opening && costs->deletion_extension == costs->extension);
    if (costs->opening2 >= 0 || costs->opening != 0 || costs->mismatch != costs->extension || costs->mismatch <= 0 ||
        !symmetric)
        return false;
    *scale = costs->mismatch;
    return true;
}

// The process's context for the entry points under the reference's own names, which take none: device
// 0, opened at the first call and kept; calls from several threads take turns on it.
std::mutex default_lock;
dinara_gpu *default_context = nullptr;

dinara_gpu *default_gpu() {
    if (!default_context) {
        default_context = dinara_gpu_new(0);
        if (!default_context) throw Failure(DINARA_DEVICE_FAILURE, "no GPU: " + new_error);
    }
    return default_context;
}

}  // namespace

int64_t dinara_gpu_band_autotune(dinara_gpu *gpu, const dinara_band_tune_options *options,
                                 dinara_band_tune_report *report) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        DINARA_CUDA(cudaSetDevice(gpu->device));
        dinara_band_tune_options given;
        std::memset(&given, 0, sizeof given);
        if (options) given = *options;
        dinara_band_tune_report local;
        band_autotune(gpu, given, local);
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        if (report) *report = local;
        return 0;
    });
}

int64_t dinara_gpu_band_tuning(dinara_gpu *gpu, int64_t set, dinara_band_tuning *tuning) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu || !tuning) throw Failure(DINARA_INVALID_MODE, "no context or tuning");
        band_tuning_access(gpu, set != 0, tuning);
        return 0;
    });
}

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

int64_t dinara_gpu_cost_alignments_tape(dinara_gpu *gpu, int64_t pairs, const char *letters, const int64_t *offsets,
                                        const dinara_costs *costs, const dinara_mode *mode,
                                        const dinara_options *options, int64_t *results, int64_t *cigar_offsets,
                                        char **cigar_bytes) {
    return guard(gpu, [&]() -> int64_t {
        if (!gpu) throw Failure(DINARA_INVALID_MODE, "no context");
        check_global(mode);
        const CostPlan plan = cost_plan(costs, options);
        check_offsets(pairs, offsets);
        const bool eqx = options ? options->eqx != 0 : true;
        const bool right = options ? options->right_ties != 0 : false;
        if (cigar_bytes) *cigar_bytes = nullptr;
        if (pairs == 0) {
            if (cigar_offsets) cigar_offsets[0] = 0;
            if (cigar_bytes) *cigar_bytes = static_cast<char *>(std::calloc(1, 1));
            return 0;
        }
        DINARA_CUDA(cudaSetDevice(gpu->device));
        const uint8_t *letters_device;
        const int64_t *offsets_device;
        upload_tape(gpu, pairs, letters, offsets, &letters_device, &offsets_device);
        int64_t *results_device = gpu->scores.ensure<int64_t>(size_t(pairs));
        const bool trace = cigar_bytes != nullptr;
        const int64_t total = cost_alignments(gpu, pairs, letters_device, offsets_device, plan, right, eqx, trace,
                                              results_device);
        to_host(gpu, results, results_device, size_t(pairs) * sizeof(int64_t));
        if (trace) {
            std::unique_ptr<char, void (*)(void *)> bytes(static_cast<char *>(std::malloc(size_t(total) + 1)), std::free);
            if (!bytes) throw std::bad_alloc();
            if (cigar_offsets)
                to_host(gpu, cigar_offsets, gpu->cigar_offsets.as<int64_t>(), size_t(pairs + 1) * sizeof(int64_t));
            DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
            to_host_now(gpu, bytes.get(), gpu->cigar_bytes.as<char>(), size_t(total));
            bytes.get()[total] = 0;
            *cigar_bytes = bytes.release();
        }
        DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
        return 0;
    });
}

// ------------------------------------------------------------------------------------------------------
// The reference's own C entry points (c/dinara.h:141-228), on the GPU of the process's default context.

int64_t dinara_distances(int64_t pairs, const char *const *references, const int64_t *reference_lengths,
                         const char *const *queries, const int64_t *query_lengths, const dinara_costs *costs,
                         const dinara_mode *mode, const dinara_options *options, int64_t threads, int64_t *results) {
    (void)threads;  // the device's own parallelism; the host does no per-pair work
    std::lock_guard<std::mutex> hold(default_lock);
    dinara_gpu *gpu = nullptr;
    try {
        gpu = default_gpu();
    } catch (const Failure &failure) {
        return failure.code;
    }
    return guard(gpu, [&]() -> int64_t {
        check_global(mode);
        int64_t scale = 1;
        if (unit_costs(costs, options, &scale)) {
            const int64_t code = dinara_gpu_distances(gpu, pairs, references, reference_lengths, queries,
                                                      query_lengths, costs, mode, options, results);
            if (code != 0) throw Failure(code, gpu->error);
            return 0;
        }
        (void)cost_plan(costs, options);
        std::vector<char> letters;
        std::vector<int64_t> offsets;
        gather_tape(pairs, references, reference_lengths, queries, query_lengths, letters, offsets);
        const int64_t code = dinara_gpu_cost_alignments_tape(gpu, pairs, letters.data(), offsets.data(), costs, mode,
                                                             options, results, nullptr, nullptr);
        if (code != 0) throw Failure(code, gpu->error);
        return 0;
    });
}

int64_t dinara_alignments(int64_t pairs, const char *const *references, const int64_t *reference_lengths,
                          const char *const *queries, const int64_t *query_lengths, const dinara_costs *costs,
                          const dinara_mode *mode, const dinara_options *options, int64_t threads,
                          dinara_alignment *alignments, int64_t *statuses) {
    (void)threads;
    std::lock_guard<std::mutex> hold(default_lock);
    dinara_gpu *gpu = nullptr;
    try {
        gpu = default_gpu();
    } catch (const Failure &failure) {
        return failure.code;
    }
    return guard(gpu, [&]() -> int64_t {
        check_global(mode);
        (void)cost_plan(costs, options);
        std::vector<char> letters;
        std::vector<int64_t> offsets;
        gather_tape(pairs, references, reference_lengths, queries, query_lengths, letters, offsets);
        std::vector<int64_t> results(size_t(std::max<int64_t>(pairs, 1)));
        std::vector<int64_t> cigar_offsets(size_t(pairs + 1));
        char *bytes = nullptr;
        const int64_t code = dinara_gpu_cost_alignments_tape(gpu, pairs, letters.data(), offsets.data(), costs, mode,
                                                             options, results.data(), cigar_offsets.data(), &bytes);
        if (code != 0) throw Failure(code, gpu->error);
        std::unique_ptr<char, void (*)(void *)> owned(bytes, std::free);
        for (int64_t p = 0; p < pairs; ++p) {
            dinara_alignment &a = alignments[p];
            std::memset(&a, 0, sizeof a);
            const int64_t cost = results[size_t(p)];
            if (statuses) statuses[p] = cost < 0 ? cost : 0;
            if (cost < 0) continue;
            const int64_t length = cigar_offsets[size_t(p + 1)] - cigar_offsets[size_t(p)];
            a.cigar = static_cast<char *>(std::malloc(size_t(length) + 1));
            if (!a.cigar) throw std::bad_alloc();
            std::memcpy(a.cigar, bytes + cigar_offsets[size_t(p)], size_t(length));
            a.cigar[length] = 0;
            a.cigar_length = length;
            a.cost = cost;
            a.score = -cost;
            a.reference_start = 0;
            a.reference_end = reference_lengths[p];
            a.query_start = 0;
            a.query_end = query_lengths[p];
        }
        return 0;
    });
}

int64_t dinara_distance(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                        const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options) {
    int64_t result = 0;
    const int64_t code = dinara_distances(1, &reference, &reference_length, &query, &query_length, costs, mode,
                                          options, 0, &result);
    return code != 0 ? code : result;
}

int64_t dinara_align(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                     const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options,
                     dinara_alignment *alignment) {
    int64_t status = 0;
    const int64_t code = dinara_alignments(1, &reference, &reference_length, &query, &query_length, costs, mode,
                                           options, 0, alignment, &status);
    return code != 0 ? code : status;
}

int64_t dinara_score(const char *reference, int64_t reference_length, const char *query, int64_t query_length,
                     const dinara_costs *costs, const dinara_mode *mode, const dinara_options *options,
                     int64_t *score) {
    // The options' cap, eqx, ties and memory change nothing (c/dinara.h:172-177).
    dinara_options plain = {INT64_MIN, INT64_MAX, -1, 1, 0, 0};
    if (options) {
        plain.band_low = options->band_low;
        plain.band_high = options->band_high;
    }
    const int64_t cost = dinara_distance(reference, reference_length, query, query_length, costs, mode, &plain);
    if (cost < 0) return cost;
    if (score) *score = -cost;
    return 0;
}

}  // extern "C"
