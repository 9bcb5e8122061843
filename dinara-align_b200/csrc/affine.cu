// Gotoh scores and alignments under a substitution table on the B200.
//
// A group of G lanes sweeps one pair, several pairs a warp: lane `m` of a group holds C consecutive
// columns in registers and runs one row behind lane m-1, whose last column's score and insertion layer
// arrive by one shuffle a row (the layout of the reference's score_groups.mojo:78-236 and
// device_align.mojo:216-263 strip_row). A pair wider than a group's G*C columns is swept in strips,
// the column left of each strip carried through global memory.
//
// Global cells are held shifted by (row + column) * extend (score_groups.mojo:114-120), so the three
// layers take one fused add-and-max each (the DPX `viaddmax`), and the insertion layer's dependency
// along a row collapses to a running maximum of the cells before it: five instructions a cell, one of
// them on the row's dependent chain. The substitution comes from a 4 x 4 table of 16-bit entries held
// in two registers a row letter, picked by one PRMT whose selector is fixed per column.
//
// Recording (for the CIGAR) writes each cell's 4-bit decision exactly as gotoh.mojo:173-186 `decide`
// gives it, 16 columns to a 64-bit word, four rows buffered in registers and stored as one 32-byte
// sector; a thread a pair then walks them back by gotoh.mojo:189-200 `advance`.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "affine.cuh"
#include "affine_kernel.cuh"

namespace dinara {

namespace {

using namespace sweep;

// ------------------------------------------------------------------------------------------------
// The walk back and the CIGAR
// ------------------------------------------------------------------------------------------------

struct WalkArgs {
    const uint32_t *tape;
    const PairShape *shapes;
    const uint64_t *decisions;
    const int64_t *decision_offsets;
    const int64_t *ends;
    const int64_t *slot_offsets;  // per pair: its CIGAR slot, 2 (rows + columns) + 1 bytes
    char *slots;
    int64_t *lengths;             // per pair: the CIGAR's bytes
    int64_t *spans;               // per pair: first row, last row, first column, last column
    int64_t first_pair, count;
    int bits;
    bool local, eqx, uniform;
};

__device__ __forceinline__ void emit_run(char *slot, int64_t &written, char op, int64_t count) {
    // Written back to front: the op, then the count's digits from the last.
    slot[written++] = op;
    do {
        slot[written++] = char('0' + count % 10);
        count /= 10;
    } while (count > 0);
}

template <int BITS>
__device__ __forceinline__ uint32_t walk_letter(const uint32_t *tape, uint32_t word, uint32_t index) {
    return letter_at<BITS>(tape, word, index);
}

template <int BITS>
__global__ void walk_kernel(WalkArgs a) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const int64_t pair = a.first_pair + k;
    const PairShape sh = a.shapes[pair];
    const int rows = int(sh.rows), cols = int(sh.columns);
    char *slot = a.slots + a.slot_offsets[k];
    int64_t written = 0;
    int row, column;
    if (a.local) {
        const int64_t end = a.ends[k];
        row = int(end >> 32);
        column = int(end & 0xffffffff);
    } else {
        row = rows;
        column = cols;
    }
    const int end_row = row, end_col = column;
    char run = 0;
    int64_t count = 0;
    auto add = [&](char op) {
        if (op == run) {
            ++count;
        } else {
            if (count > 0) emit_run(slot, written, run, count);
            run = op;
            count = 1;
        }
    };
    if (rows > 0 && cols > 0) {
        const int G = record_lanes(uint32_t(cols), a.uniform);
        const int W = G * 16;
        const int rows_pad = ((rows + 2) | 3) + 1;
        const int64_t base = a.decision_offsets[k];
        int state = 0;  // 0 aligning, 1 deleting, 2 inserting
        while (row > 0 && column > 0) {
            const int off = column - 1;
            const int s = off / W;
            const int within = off % W;
            const int member = within / 16;
            const int slot_in = within % 16;
            const uint64_t word = a.decisions[base + int64_t(s * G + member) * rows_pad + (row - 1 + (member & 3))];
            const uint32_t nibble = uint32_t(word >> (4 * slot_in)) & 15u;
            if (a.local && state == 0 && (nibble & 3u) == 3u) break;
            const int moving = state == 0 ? int(nibble & 3u) : state;
            if (moving == 1) {
                add('D');
                row -= 1;
                state = (nibble >> 2) & 1u ? 1 : 0;
            } else if (moving == 2) {
                add('I');
                column -= 1;
                state = (nibble >> 3) & 1u ? 2 : 0;
            } else {
                char op = 'M';
                if (a.eqx) {
                    const uint32_t x = walk_letter<BITS>(a.tape, sh.first_word, uint32_t(row - 1));
                    const uint32_t y = walk_letter<BITS>(a.tape, sh.second_word, uint32_t(column - 1));
                    op = x == y ? '=' : 'X';
                }
                add(op);
                row -= 1;
                column -= 1;
                state = 0;
            }
        }
    }
    if (!a.local) {
        // gotoh.mojo:440-447: a global walk's rest is gaps against the letters left, rows first.
        for (; row > 0; --row) add('D');
        for (; column > 0; --column) add('I');
    }
    if (count > 0) emit_run(slot, written, run, count);
    a.lengths[k] = written;
    int64_t *span = a.spans + 4 * k;
    span[0] = row;
    span[1] = end_row;
    span[2] = column;
    span[3] = end_col;
}

// Each pair's CIGAR, written back to front in its slot, turned round into the packed output.
__global__ void gather_cigars_kernel(const char *__restrict__ slots, const int64_t *__restrict__ slot_offsets,
                                     const int64_t *__restrict__ lengths, const int64_t *__restrict__ offsets,
                                     char *__restrict__ out, int64_t count) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;
    const char *from = slots + slot_offsets[warp];
    const int64_t n = lengths[warp];
    char *to = out + offsets[warp];
    for (int64_t i = lane; i < n; i += 32) to[i] = from[n - 1 - i];
}

__global__ void slot_sizes_kernel(const PairShape *__restrict__ shapes, int64_t first_pair, int64_t count, bool uniform,
                                  int64_t *__restrict__ decision_words, int64_t *__restrict__ slot_bytes) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const PairShape sh = shapes[first_pair + k];
    int64_t words = 0;
    if (sh.rows > 0 && sh.columns > 0) {
        const int G = record_lanes(sh.columns, uniform);
        const int W = G * 16;
        const int64_t strips = (sh.columns + W - 1) / W;
        const int64_t rows_pad = ((int64_t(sh.rows) + 2) | 3) + 1;
        words = strips * G * rows_pad;
    }
    decision_words[k] = words;
    slot_bytes[k] = 2 * (int64_t(sh.rows) + sh.columns) + 8;
}

// ------------------------------------------------------------------------------------------------
// Launching
// ------------------------------------------------------------------------------------------------

using KernelFn = void (*)(KernelArgs, TableArgs, const int32_t *);

template <int G, int C, bool LOCAL, bool RECORD, int BITS, bool SMEM>
KernelFn kernel_of() {
    return &affine_kernel<G, C, LOCAL, RECORD, BITS, SMEM>;
}

// The kernel for a shape class; record kernels exist for the 16-column shapes only.
KernelFn pick_kernel(int cls, bool local, bool record, int bits, bool smem) {
    if (smem || bits == 8) {
        // The general path: any alphabet of up to 32 letters, the table in shared memory, one shape.
        if (bits == 8) {
            if (local) return record ? kernel_of<32, 16, true, true, 8, true>() : kernel_of<32, 16, true, false, 8, true>();
            return record ? kernel_of<32, 16, false, true, 8, true>() : kernel_of<32, 16, false, false, 8, true>();
        }
        if (local) return record ? kernel_of<32, 16, true, true, 2, true>() : kernel_of<32, 16, true, false, 2, true>();
        return record ? kernel_of<32, 16, false, true, 2, true>() : kernel_of<32, 16, false, false, 2, true>();
    }
#define DINARA_SHAPE(G, C)                                                                                       \
    if (local)                                                                                                   \
        return record ? kernel_of<G, C, true, true, 2, false>() : kernel_of<G, C, true, false, 2, false>();      \
    return record ? kernel_of<G, C, false, true, 2, false>() : kernel_of<G, C, false, false, 2, false>();
    switch (cls) {
        case 0: {
            DINARA_SHAPE(4, 16)
        }
        case 1: {
            DINARA_SHAPE(8, 16)
        }
        case 2: {
            DINARA_SHAPE(16, 16)
        }
        case 3: {
            if (local) return kernel_of<16, 20, true, false, 2, false>();
            return kernel_of<16, 20, false, false, 2, false>();
        }
        default: {
            DINARA_SHAPE(32, 16)
        }
    }
#undef DINARA_SHAPE
}

int persistent_blocks(dinara_gpu *gpu, KernelFn fn) {
    int per_sm = 0;
    DINARA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    if (per_sm < 1) per_sm = 1;
    return per_sm * gpu->multiprocessors;
}

TableArgs table_args(const AffineTable &table, bool local) {
    TableArgs t;
    std::memset(&t, 0, sizeof t);
    t.size = table.size;
    if (table.packed16) {
        for (int r = 0; r < 4; ++r) {
            uint16_t e[4] = {0, 0, 0, 0};
            for (int c = 0; c < 4; ++c) {
                int32_t v = 0;
                if (r < table.size && c < table.size) {
                    v = table.entries[r * 32 + c];
                    if (!local) v -= 2 * table.extend;
                }
                e[c] = uint16_t(int16_t(v));
            }
            t.rows16[r].x = uint32_t(e[0]) | (uint32_t(e[1]) << 16);
            t.rows16[r].y = uint32_t(e[2]) | (uint32_t(e[3]) << 16);
        }
    }
    return t;
}

// The table for the shared-memory path: 32 rows of 33 entries, entry 32 of each (a padding column)
// far below any score, so a padded cell never beats a real one.
void upload_table32(dinara_gpu *gpu, const AffineTable &table, bool local, int32_t **out) {
    std::vector<int32_t> host(32 * 33, 0);
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 33; ++c) {
            int32_t v = (r < table.size && c < table.size) ? table.entries[r * 32 + c] : 0;
            if (c == 32) v = -(1 << 20);
            else if (!local) v -= 2 * table.extend;
            host[r * 33 + c] = v;
        }
    int32_t *dev = gpu->table32.ensure<int32_t>(host.size());
    DINARA_CUDA(cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(int32_t), cudaMemcpyHostToDevice, gpu->stream));
    DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
    *out = dev;
}

struct Buckets {
    int64_t begin[kAffineShapes];
    int64_t end[kAffineShapes];
};

// The sorted order's ranges per shape class: classes in descending order, as the keys put them.
Buckets buckets_of(const int64_t counts[kAffineShapes]) {
    Buckets b;
    int64_t at = 0;
    for (int cls = kAffineShapes - 1; cls >= 0; --cls) {
        b.begin[cls] = at;
        at += counts[cls];
        b.end[cls] = at;
    }
    return b;
}

}  // namespace

namespace {

void affine_launch_all(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, const uint32_t *order,
                       const int64_t counts[kAffineShapes], bool record, KernelArgs args) {
    const bool smem = !table.packed16 || batch.bits == 8;
    const TableArgs targs = table_args(table, batch.local);
    int32_t *table32 = nullptr;
    if (smem) upload_table32(gpu, table, batch.local, &table32);
    const Buckets b = buckets_of(counts);
    args.order = order;
    if (gpu->timing) DINARA_CUDA(cudaEventRecord(gpu->start, gpu->stream));
    for (int cls = kAffineShapes - 1; cls >= 0; --cls) {
        if (b.end[cls] <= b.begin[cls]) continue;
        KernelFn fn = pick_kernel(cls, batch.local, record, batch.bits, smem);
        const int G = smem ? 32 : affine_lanes(cls);
        const int groups_per_block = kBlock / G;
        int64_t blocks = persistent_blocks(gpu, fn);
        const int64_t needed = (b.end[cls] - b.begin[cls] + groups_per_block - 1) / groups_per_block;
        if (blocks > needed) blocks = needed;
        if (blocks < 1) blocks = 1;
        // Carry slots, one a group, each as long as the tallest pair: only a launch whose pairs may be
        // wider than one strip reads them.
        const int width = smem ? 512 : affine_lanes(cls) * affine_columns(cls);
        args.carry = nullptr;
        args.carry_stride = 0;
        if (batch.max_columns > uint32_t(width)) {
            const int64_t slots = blocks * groups_per_block;
            args.carry_stride = int64_t(batch.max_rows) + 1;
            args.carry = gpu->carry.ensure<int2>(size_t(slots * args.carry_stride));
        }
        args.begin = uint32_t(b.begin[cls]);
        args.end = uint32_t(b.end[cls]);
        fn<<<dim3(unsigned(blocks)), kBlock, 0, gpu->stream>>>(args, targs, table32);
        DINARA_CUDA(cudaGetLastError());
        gpu->launches += 1;
    }
    if (gpu->timing) {
        DINARA_CUDA(cudaEventRecord(gpu->stop, gpu->stream));
        DINARA_CUDA(cudaEventSynchronize(gpu->stop));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
        (record ? gpu->record_ms : gpu->kernel_ms) += ms;
    }
}

}  // namespace

void affine_scores(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, int32_t *scores,
                   const uint32_t *order, const int64_t counts[kAffineShapes]) {
    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    affine_launch_all(gpu, batch, table, order, counts, false, args);
}

int64_t affine_alignments(dinara_gpu *gpu, const AffineBatch &batch, const AffineTable &table, bool eqx,
                          int32_t *scores, int64_t *spans, int64_t first_pair, int64_t count, const uint32_t *order,
                          const int64_t counts[kAffineShapes]) {
    // Per pair: its decisions' words and its CIGAR slot, then their offsets by an exclusive scan.
    int64_t *words = gpu->decision_offsets.ensure<int64_t>(2 * (count + 1) + 2);
    int64_t *word_offsets = words + (count + 1);
    int64_t *slot_bytes = gpu->cigar_slots.ensure<int64_t>(2 * (count + 1) + 2);
    int64_t *slot_offsets = slot_bytes + (count + 1);
    const int threads = 256;
    const unsigned blocks = unsigned((count + threads - 1) / threads);
    const bool uniform = !table.packed16 || batch.bits == 8;
    slot_sizes_kernel<<<blocks, threads, 0, gpu->stream>>>(batch.shapes, first_pair, count, uniform, words, slot_bytes);
    DINARA_CUDA(cudaGetLastError());
    size_t scratch = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch, words, word_offsets, int(count + 1), gpu->stream));
    size_t scratch2 = 0;
    DINARA_CUDA(
        cub::DeviceScan::ExclusiveSum(nullptr, scratch2, slot_bytes, slot_offsets, int(count + 1), gpu->stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(std::max(scratch, scratch2) + 256);
    // The counts' last entries are zero, so each scan's last output is its total.
    DINARA_CUDA(cudaMemsetAsync(words + count, 0, sizeof(int64_t), gpu->stream));
    DINARA_CUDA(cudaMemsetAsync(slot_bytes + count, 0, sizeof(int64_t), gpu->stream));
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch, words, word_offsets, int(count + 1), gpu->stream));
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch2, slot_bytes, slot_offsets, int(count + 1), gpu->stream));
    int64_t totals[2];
    DINARA_CUDA(cudaMemcpyAsync(&totals[0], word_offsets + count, sizeof(int64_t), cudaMemcpyDeviceToHost, gpu->stream));
    DINARA_CUDA(cudaMemcpyAsync(&totals[1], slot_offsets + count, sizeof(int64_t), cudaMemcpyDeviceToHost, gpu->stream));
    DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
    uint64_t *decisions = gpu->decisions.ensure<uint64_t>(size_t(totals[0]) + 8);
    char *slots = gpu->walk_out.ensure<char>(size_t(totals[1]) + 8);
    int64_t *ends = gpu->spans.ensure<int64_t>(size_t(count) + 1);
    int64_t *lengths = gpu->cigar_lengths.ensure<int64_t>(size_t(count) + 1);

    KernelArgs args;
    std::memset(&args, 0, sizeof args);
    args.tape = batch.tape;
    args.shapes = batch.shapes;
    args.open = table.open;
    args.extend = table.extend;
    args.scores = scores;
    args.decisions = decisions;
    args.decision_offsets = word_offsets;
    args.ends = ends;
    args.first_pair = first_pair;
    affine_launch_all(gpu, batch, table, order, counts, true, args);

    WalkArgs w;
    std::memset(&w, 0, sizeof w);
    w.tape = batch.tape;
    w.shapes = batch.shapes;
    w.decisions = decisions;
    w.decision_offsets = word_offsets;
    w.ends = ends;
    w.slot_offsets = slot_offsets;
    w.slots = slots;
    w.lengths = lengths;
    w.spans = spans;
    w.first_pair = first_pair;
    w.count = count;
    w.bits = batch.bits;
    w.local = batch.local;
    w.eqx = eqx;
    w.uniform = uniform;
    if (batch.bits == 8)
        walk_kernel<8><<<blocks, threads, 0, gpu->stream>>>(w);
    else
        walk_kernel<2><<<blocks, threads, 0, gpu->stream>>>(w);
    DINARA_CUDA(cudaGetLastError());

    // The CIGARs' offsets, then each turned round into place.
    int64_t *offsets = gpu->cigar_offsets.ensure<int64_t>(size_t(count) + 2);
    DINARA_CUDA(cudaMemsetAsync(lengths + count, 0, sizeof(int64_t), gpu->stream));
    size_t scratch3 = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scratch3, lengths, offsets, int(count + 1), gpu->stream));
    space = gpu->sort_scratch.ensure<uint8_t>(scratch3 + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scratch3, lengths, offsets, int(count + 1), gpu->stream));
    int64_t total = 0;
    DINARA_CUDA(cudaMemcpyAsync(&total, offsets + count, sizeof(int64_t), cudaMemcpyDeviceToHost, gpu->stream));
    DINARA_CUDA(cudaStreamSynchronize(gpu->stream));
    char *out = gpu->cigar_bytes.ensure<char>(size_t(total) + 8);
    const unsigned gather_blocks = unsigned((count * 32 + threads - 1) / threads);
    gather_cigars_kernel<<<gather_blocks, threads, 0, gpu->stream>>>(slots, slot_offsets, lengths, offsets, out, count);
    DINARA_CUDA(cudaGetLastError());
    return total;
}

}  // namespace dinara
