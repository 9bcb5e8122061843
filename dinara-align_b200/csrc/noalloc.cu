// Gap-affine scores for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside another framework's memory pool, under a
// memory budget that forbids growth, or in a process whose allocator is not this library's. For them
// dinara_gpu_scores_static scores an already packed batch whose inputs and outputs the caller owns,
// and keeps its own working memory (the sweep's carried columns and its pair order) in one fixed,
// file-scope device array instead of allocating any. Every device that loads this library holds that
// array (kStaticBytes, 20 MiB) until the process exits.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "affine_kernel.cuh"

namespace dinara {
namespace {

// The carried columns: one slot of kStaticRows + 1 (score, insertion) entries per pair group of the
// grid. A pair wider than one strip (512 columns) carries a column per row, so it may have at most
// kStaticRows reference letters.
constexpr int kStaticRows = 8191;
constexpr int kStaticBlocks = 32;                  // of 256 threads: 8 groups of 32 lanes each
constexpr int kStaticSlots = kStaticBlocks * 8;    // 256 pair groups at once
constexpr int64_t kStaticOrder = 1 << 20;          // pairs a launch takes; larger batches go in turns
constexpr size_t kOrderBytes = size_t(kStaticOrder) * sizeof(uint32_t);
constexpr size_t kCarryBytes = size_t(kStaticSlots) * (kStaticRows + 1) * sizeof(int2);
constexpr size_t kVerdictBytes = 256;              // the size check's verdict word, then padding
constexpr size_t kStaticBytes = kOrderBytes + kCarryBytes + kVerdictBytes;  // 4 MiB + 16 MiB + 256 B

static __device__ __align__(256) unsigned char static_scratch[kStaticBytes];

// The array's device address on each device, found once with that device current.
std::mutex setup_lock;
void *scratch_address[64] = {nullptr};

// Verdict bits the check kernel sets.
constexpr unsigned kPastCarry = 1u;  // a pair wider than one strip with more than kStaticRows rows
constexpr unsigned kPastReach = 2u;  // a pair whose scores could pass 2^28 (ScoreReach, scoring.mojo:218-249)

// Reads every pair's shape on the device and sets the verdict's bits for pairs the sweep cannot take:
// one past the carried column, or one whose scores could pass 2^28 as the main entry points refuse them
// per pair (letters = rows + columns globally, the shorter side locally).
__global__ void check_kernel(const dinara_packed_pair *__restrict__ shapes, int64_t pairs, bool local,
                             int64_t reach_opening, int64_t reach_step, unsigned *__restrict__ verdict) {
    unsigned bits = 0;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < pairs; k += int64_t(gridDim.x) * blockDim.x) {
        const dinara_packed_pair s = shapes[k];
        if (s.columns > 512 && s.rows > uint32_t(kStaticRows)) bits |= kPastCarry;
        const int64_t letters = local ? int64_t(min(s.rows, s.columns)) : int64_t(s.rows) + s.columns;
        if (reach_opening + 2 * (letters + 2) * reach_step >= (int64_t(1) << 28)) bits |= kPastReach;
    }
    bits = __reduce_or_sync(0xffffffffu, bits);
    if ((threadIdx.x & 31) == 0 && bits) atomicOr(verdict, bits);
}

__global__ void identity_order_kernel(uint32_t *order, int64_t count) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < count) order[k] = uint32_t(k);
}

// Sets the device's array up on first use: its address, and the identity order later launches read.
// A host-side name of a __device__ array is not a device address, so only the address found here is
// ever handed to a kernel.
cudaError_t scratch_on(int device, cudaStream_t stream, void **out) {
    std::lock_guard<std::mutex> hold(setup_lock);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (scratch_address[device]) {
        *out = scratch_address[device];
        return cudaSuccess;
    }
    void *address = nullptr;
    cudaError_t status = cudaGetSymbolAddress(&address, static_scratch);
    if (status != cudaSuccess) return status;
    identity_order_kernel<<<unsigned((kStaticOrder + 255) / 256), 256, 0, stream>>>(static_cast<uint32_t *>(address),
                                                                                    kStaticOrder);
    status = cudaGetLastError();
    if (status != cudaSuccess) return status;
    status = cudaStreamSynchronize(stream);
    if (status != cudaSuccess) return status;
    scratch_address[device] = address;
    *out = address;
    return cudaSuccess;
}

}  // namespace
}  // namespace dinara

extern "C" int64_t dinara_gpu_scores_static(int64_t device, int64_t pairs, const uint32_t *tape,
                                            const dinara_packed_pair *shapes, const dinara_scoring *scoring,
                                            const dinara_mode *mode, int32_t *scores, void *stream) {
    using namespace dinara;
    using namespace dinara::sweep;
    if (pairs < 0) return DINARA_INVALID_LENGTH;
    if (!scoring || !scoring->table || scoring->alphabet_size < 1 || scoring->alphabet_size > 4)
        return DINARA_INVALID_MODE;  // two bits a letter: alphabets of up to four letters
    bool local = false;
    if (mode) {
        if (mode->match_score > 0) return DINARA_INVALID_MODE;
        if (mode->kind == DINARA_LOCAL)
            local = true;
        else if (mode->kind != DINARA_ENDS_FREE || mode->reference_start || mode->reference_end || mode->query_start ||
                 mode->query_end)
            return DINARA_INVALID_MODE;
    }
    // The gap scores as the main entry points check them (scoring.mojo:202-215 gap_scores).
    const int64_t opening = scoring->opening, extension = scoring->extension;
    if (opening > 0 || extension > 0 || opening + extension < -int64_t(INT32_MAX) || extension < -int64_t(INT32_MAX))
        return DINARA_INVALID_COSTS;
    const int32_t open = int32_t(opening + extension), extend = int32_t(extension);
    // The table in two registers a row letter, 16 bits an entry, shifted for a global sweep.
    TableArgs table;
    std::memset(&table, 0, sizeof table);
    const int64_t size = scoring->alphabet_size;
    int64_t highest = -128, lowest = 127;
    for (int r = 0; r < 4; ++r) {
        uint16_t entries[4] = {0, 0, 0, 0};
        for (int c = 0; c < 4; ++c) {
            int64_t v = 0;
            if (r < size && c < size) {
                const int64_t entry = scoring->table[r * size + c];
                highest = std::max(highest, entry);
                lowest = std::min(lowest, entry);
                v = entry - (local ? 0 : 2 * int64_t(extend));
            }
            if (v < -32768 || v > 32767) return DINARA_INVALID_COSTS;
            entries[c] = uint16_t(int16_t(v));
        }
        table.rows16[r] = make_uint2(uint32_t(entries[0]) | (uint32_t(entries[1]) << 16),
                                     uint32_t(entries[2]) | (uint32_t(entries[3]) << 16));
    }
    table.size = int32_t(size);
    // ScoreReach (scoring.mojo:228-249): what a score can move by at an opening and at a letter.
    const int64_t reach_opening = 2 * -int64_t(open);
    const int64_t reach_step = std::max(std::max(highest, -lowest), -int64_t(extend));
    if (pairs == 0) return 0;
    if (!tape || !shapes || !scores) return DINARA_INVALID_LENGTH;
    cudaStream_t on = static_cast<cudaStream_t>(stream);
    int current = 0;
    if (cudaGetDevice(&current) != cudaSuccess) return DINARA_DEVICE_FAILURE;
    if (cudaSetDevice(int(device)) != cudaSuccess) return DINARA_DEVICE_FAILURE;
    void *scratch = nullptr;
    cudaError_t status = scratch_on(int(device), on, &scratch);
    int64_t code = 0;
    unsigned verdict = 0;
    unsigned *verdict_device =
        reinterpret_cast<unsigned *>(static_cast<unsigned char *>(scratch) + kOrderBytes + kCarryBytes);
    if (status == cudaSuccess) {
        // The check runs on the caller's stream, after whatever wrote the shapes there; its one word comes
        // back before any sweep is launched, so a refused batch runs nothing.
        status = cudaMemsetAsync(verdict_device, 0, sizeof(unsigned), on);
        if (status == cudaSuccess) {
            check_kernel<<<kStaticBlocks * 4, 256, 0, on>>>(shapes, pairs, local, reach_opening, reach_step,
                                                           verdict_device);
            status = cudaGetLastError();
        }
        if (status == cudaSuccess)
            status = cudaMemcpyAsync(&verdict, verdict_device, sizeof(unsigned), cudaMemcpyDeviceToHost, on);
        if (status == cudaSuccess) status = cudaStreamSynchronize(on);
    }
    if (status != cudaSuccess) {
        code = DINARA_DEVICE_FAILURE;
    } else if (verdict & kPastReach) {
        code = DINARA_INVALID_COSTS;  // scores that could pass 2^28, refused as ScoreReach refuses them
    } else if (verdict & kPastCarry) {
        code = DINARA_OUT_OF_MEMORY;  // a pair past the fixed scratch: more than 8191 rows and 512 columns
    } else {
        KernelArgs args;
        std::memset(&args, 0, sizeof args);
        args.tape = tape;
        args.order = static_cast<const uint32_t *>(scratch);
        args.open = open;
        args.extend = extend;
        args.carry = reinterpret_cast<int2 *>(static_cast<unsigned char *>(scratch) + kOrderBytes);
        args.carry_stride = kStaticRows + 1;
        auto kernel = local ? &affine_kernel<32, 16, true, false, 2, false> : &affine_kernel<32, 16, false, false, 2, false>;
        for (int64_t first = 0; first < pairs && code == 0; first += kStaticOrder) {
            const int64_t count = std::min<int64_t>(kStaticOrder, pairs - first);
            args.shapes = reinterpret_cast<const PairShape *>(shapes + first);
            args.scores = scores + first;
            args.begin = 0;
            args.end = uint32_t(count);
            kernel<<<kStaticBlocks, kBlock, 0, on>>>(args, table, nullptr);
            if (cudaGetLastError() != cudaSuccess) code = DINARA_DEVICE_FAILURE;
        }
    }
    cudaSetDevice(current);
    return code;
}
