// Global alignments under Costs on the B200, with the CIGAR the reference's Ties rule picks.
//
// Under a `Costs` (a mismatch, and gaps of k letters costing an opening plus k extensions) dinara-align
// returns, of several equally good alignments, the one its Ties rule names (modes.mojo:402-426):
// Ties.RIGHT is WFA2-lib's backtrace run from the far corner of one search from the start, every edit as
// late as it goes; Ties.LEFT is that rule over both sequences reversed, read forward. At unit costs the
// search is diagonal transition and the trace `best_source` (diagonal.mojo:286-316, traceback.mojo:
// 803-900); otherwise it is the gap-affine wavefront with a flag of which source won each front
// (gap_affine.mojo:858-1010) and its trace (gap_affine.mojo:2028-2124). The reference runs these on the
// CPU only. Here one warp takes one pair: its lanes compute a cost's front, diagonals 32 apart, each
// sliding over its matches; every front is kept in the warp's arena of device memory; lane 0 traces back
// through them and writes the CIGAR. Warps take pairs from a queue, longest first. A pair whose fronts
// outgrow its warp's arena goes onto a list that runs again on fewer warps with larger arenas.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "ties.cuh"

namespace dinara {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWaveBlock = 128;
constexpr int32_t kUnreached = -(1 << 30);
// A pair's slot in the cost table and in `results` while it waits for a larger arena.
constexpr int64_t kRetry = INT64_MIN;

// One cost's front in a warp's arena: diagonals lo ..= hi, its arrays from `offset`.
struct CostEntry {
    int32_t lo, hi;
    int64_t offset;
};

struct WaveArgs {
    const uint8_t *letters;
    const int64_t *offsets;  // 2 * pairs + 1, into `letters`
    const uint32_t *order;   // the pairs this launch takes, longest first
    uint32_t count;
    unsigned int *next;      // the queue's head
    int32_t x, od, ed, oi, ei;  // the costs over their common factor; d a deletion's, i an insertion's
    int64_t scale;
    int64_t ceiling;         // the largest cost (over the common factor) a pair may take
    bool reversed;           // Ties.LEFT: both sequences read back to front
    bool eqx;
    bool trace;
    uint8_t *arena;
    int64_t arena_bytes;     // a warp's
    int32_t table_entries;   // cost entries at the start of each arena
    int64_t *results;        // per pair: its cost, or its code
    const int64_t *slot_offsets;
    char *slots;
    int64_t *lengths;        // per pair: the CIGAR's bytes
    uint32_t *retry;
    unsigned int *retry_count;
};

__device__ __forceinline__ uint8_t letter_of(const uint8_t *s, int32_t length, int32_t i, bool reversed) {
    return __ldg(s + (reversed ? length - 1 - i : i));
}

// The furthest column a diagonal's matches take a front from `column` (row column - diagonal).
__device__ __forceinline__ int32_t slide(const uint8_t *first, int32_t columns, const uint8_t *second, int32_t rows,
                                         int32_t column, int32_t diagonal, bool reversed) {
    int32_t row = column - diagonal;
    while (column < columns && row < rows &&
           letter_of(first, columns, column, reversed) == letter_of(second, rows, row, reversed)) {
        ++column;
        ++row;
    }
    return column;
}

// A front's value on a diagonal: unreached outside its diagonals, before cost zero, or where empty.
__device__ __forceinline__ int32_t front_at(const uint8_t *arena, const CostEntry &e, int32_t layer, int32_t k) {
    if (e.lo > e.hi || k < e.lo || k > e.hi) return kUnreached;
    const int32_t width = e.hi - e.lo + 1;
    return reinterpret_cast<const int32_t *>(arena + e.offset)[int64_t(layer) * width + (k - e.lo)];
}

__device__ __forceinline__ CostEntry entry_of(const CostEntry *table, int32_t s) {
    CostEntry e;
    if (s < 0) {
        e.lo = 1;
        e.hi = 0;
        e.offset = 0;
        return e;
    }
    return table[s];
}

// furthest_source (diagonal.mojo:286-303): the furthest column one more edit reaches on `diagonal`
// before its matches, and the edit (0 a substitution, 1 a letter of the first sequence alone, 2 one of
// the second); ties to a substitution, then to the first sequence's letter.
__device__ __forceinline__ int32_t furthest_source(int32_t same, int32_t left, int32_t up, int32_t diagonal,
                                                   int32_t columns, int32_t rows, int &move) {
    int32_t best = -1;
    move = 0;
    if (same >= 0 && same < columns && same - diagonal < rows) best = same + 1;
    if (left >= 0 && left < columns && left + 1 > best) {
        best = left + 1;
        move = 1;
    }
    if (up >= 0 && up - diagonal - 1 < rows && up > best) {
        best = up;
        move = 2;
    }
    return best;
}

// Lane 0's CIGAR writer: runs joined while their letter repeats (cigar.mojo:183-200), written forward,
// or (for a trace that runs right to left) as the text reversed, which the gather turns round.
struct CigarOut {
    char *slot;
    int64_t capacity;  // the slot's bytes; a run that would pass them sets `overflow` and is dropped
    int64_t written = 0;
    char letter = 0;
    int64_t count = 0;
    bool forward;
    bool overflow = false;
    __device__ void flush() {
        if (count <= 0) return;
        int digits = 1;
        for (int64_t v = count; v >= 10; v /= 10) ++digits;
        if (written + digits + 1 > capacity) {
            overflow = true;
            count = 0;
            return;
        }
        if (forward) {
            char digits[20];
            int d = 0;
            int64_t v = count;
            do {
                digits[d++] = char('0' + v % 10);
                v /= 10;
            } while (v > 0);
            while (d > 0) slot[written++] = digits[--d];
            slot[written++] = letter;
        } else {
            slot[written++] = letter;
            int64_t v = count;
            do {
                slot[written++] = char('0' + v % 10);
                v /= 10;
            } while (v > 0);
        }
        count = 0;
    }
    __device__ void add(char op, int64_t length) {
        if (length <= 0) return;
        if (op != letter) {
            flush();
            letter = op;
        }
        count += length;
    }
};

// The trace of diagonal transition (diagonal_cigar, traceback.mojo:803-900): from the corner, each cost
// undoes the matches its front slid over and the edit `furthest_source` names.
__device__ bool trace_edit(const WaveArgs &a, const uint8_t *arena, const CostEntry *table, int32_t distance,
                           int32_t columns, int32_t rows, CigarOut &out) {
    const char matched = a.eqx ? '=' : 'M', substituted = a.eqx ? 'X' : 'M';
    int32_t diagonal = columns - rows, column = columns;
    for (int32_t score = distance; score > 0; --score) {
        const CostEntry back = table[score - 1];
        int move;
        const int32_t best = furthest_source(front_at(arena, back, 0, diagonal), front_at(arena, back, 0, diagonal - 1),
                                             front_at(arena, back, 0, diagonal + 1), diagonal, columns, rows, move);
        if (best < 0 || best > column) return false;
        out.add(matched, column - best);
        if (move == 0) {
            out.add(substituted, 1);
            column = best - 1;
        } else if (move == 1) {
            out.add('D', 1);
            column = best - 1;
            diagonal -= 1;
        } else {
            out.add('I', 1);
            column = best;
            diagonal += 1;
        }
    }
    out.add(matched, column);
    return true;
}

// Layers of a gap-affine front: the alignment front, the first sequence's gap layer, the second's, and
// the flags (a byte each, after the three int32 layers).
constexpr int kAligned = 0, kFirst = 1, kSecond = 2;
constexpr uint8_t kOpenedFirst = 8, kOpenedSecond = 16;

__device__ __forceinline__ uint8_t flag_at(const uint8_t *arena, const CostEntry &e, int32_t k) {
    const int32_t width = e.hi - e.lo + 1;
    return (arena + e.offset + 12 * int64_t(width))[k - e.lo];
}

// The gap-affine trace (gap_affine.mojo:2028-2124): in the alignment layer the source that won the front
// (a substitution from the front `x` back, or a gap layer at the same cost, entered after the matches
// back to its column); in a gap layer a letter of its sequence, then the opening or the extension its
// flag names, an extension on a tie. On the first row or column the rest is a gap along it.
__device__ bool trace_affine(const WaveArgs &a, const uint8_t *arena, const CostEntry *table, int32_t cost,
                             int32_t columns, int32_t rows, CigarOut &out) {
    const char matched = a.eqx ? '=' : 'M', substituted = a.eqx ? 'X' : 'M';
    int32_t spent = cost, k = columns - rows, c = columns;
    int current = kAligned;
    // Every step moves a letter or leaves the alignment layer, so a consistent trace ends well within
    // this; the bound and the index checks keep an inconsistent one from running on or reading astray.
    for (int64_t steps = 4 * (int64_t(columns) + rows) + int64_t(cost) + 16; steps > 0; --steps) {
        if (spent < 0 || spent > cost || c < 0 || c - k < 0) return false;
        {
            const CostEntry here = table[spent];
            if (spent > 0 && (here.lo > here.hi || k < here.lo || k > here.hi)) return false;
        }
        if (current == kAligned) {
            const int32_t row = c - k;
            if (c == 0) {
                out.add('I', row);
                return true;
            }
            if (row == 0) {
                out.add('D', c);
                return true;
            }
            if (spent == 0) {
                const int32_t start = k > 0 ? k : 0;
                out.add(matched, c - start);
                c = start;
                continue;
            }
            const CostEntry e = table[spent];
            const int source = flag_at(arena, e, k) & 7;
            const int32_t entry = source == kAligned ? front_at(arena, entry_of(table, spent - a.x), kAligned, k) + 1
                                                     : front_at(arena, e, source, k);
            if (entry <= c) {
                out.add(matched, c - entry);
                c = entry;
            }
            if (source == kAligned) {
                out.add(substituted, 1);
                c -= 1;
                spent -= a.x;
            } else {
                current = source;
            }
        } else {
            const CostEntry e = table[spent];
            const bool opened = (flag_at(arena, e, k) & (current == kFirst ? kOpenedFirst : kOpenedSecond)) != 0;
            if (current == kFirst) {
                out.add('D', 1);
                c -= 1;
                k -= 1;
                if (c == 0) {
                    out.add('I', -k);
                    return true;
                }
                if (opened) {
                    spent -= a.od + a.ed;
                    current = kAligned;
                } else {
                    spent -= a.ed;
                }
            } else {
                out.add('I', 1);
                k += 1;
                if (c - k == 0) {
                    out.add('D', c);
                    return true;
                }
                if (opened) {
                    spent -= a.oi + a.ei;
                    current = kAligned;
                } else {
                    spent -= a.ei;
                }
            }
        }
    }
    return false;
}

template <bool EDIT>
__global__ void __launch_bounds__(kWaveBlock) wavefront_kernel(WaveArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * kWaveBlock + threadIdx.x) >> 5;
    uint8_t *arena = a.arena + warp * a.arena_bytes;
    CostEntry *table = reinterpret_cast<CostEntry *>(arena);
    const int64_t data_begin = int64_t(a.table_entries) * int64_t(sizeof(CostEntry));
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.next, 1u);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.count) return;
        const uint32_t pair = a.order[item];
        const int64_t p0 = a.offsets[2 * int64_t(pair)], p1 = a.offsets[2 * int64_t(pair) + 1],
                      p2 = a.offsets[2 * int64_t(pair) + 2];
        const uint8_t *first = a.letters + p0;
        const uint8_t *second = a.letters + p1;
        const int32_t columns = int32_t(p1 - p0), rows = int32_t(p2 - p1);
        const int32_t target = columns - rows;
        int64_t used = data_begin;
        bool overflow = false, found = false;
        int32_t s = 0;
        for (;; ++s) {
            if (s > a.ceiling) break;
            if (s >= a.table_entries) {
                overflow = true;
                break;
            }
            // The diagonals any source reaches, within the matrix.
            int32_t lo, hi;
            CostEntry same_e, open_first_e, ext_first_e, open_second_e, ext_second_e;
            if (s == 0) {
                lo = hi = 0;
            } else if (EDIT) {
                same_e = table[s - 1];
                lo = same_e.lo - 1;
                hi = same_e.hi + 1;
            } else {
                same_e = entry_of(table, s - a.x);
                open_first_e = entry_of(table, s - a.od - a.ed);
                ext_first_e = entry_of(table, s - a.ed);
                open_second_e = entry_of(table, s - a.oi - a.ei);
                ext_second_e = entry_of(table, s - a.ei);
                lo = INT_MAX;
                hi = INT_MIN;
                const CostEntry sources[5] = {same_e, open_first_e, ext_first_e, open_second_e, ext_second_e};
                const int32_t shifts[5] = {0, 1, 1, -1, -1};
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    if (sources[q].lo > sources[q].hi) continue;
                    lo = min(lo, sources[q].lo + shifts[q]);
                    hi = max(hi, sources[q].hi + shifts[q]);
                }
            }
            lo = max(lo, -rows);
            hi = min(hi, columns);
            const int32_t width = hi >= lo ? hi - lo + 1 : 0;
            const int64_t bytes = ((EDIT ? 4 * int64_t(width) : 13 * int64_t(width)) + 15) & ~int64_t(15);
            if (used + bytes > a.arena_bytes) {
                overflow = true;
                break;
            }
            if (lane == 0) {
                CostEntry e;
                e.lo = lo;
                e.hi = hi;
                e.offset = used;
                table[s] = e;
            }
            int32_t *aligned = reinterpret_cast<int32_t *>(arena + used);
            bool hit = false;
            for (int32_t k = lo + lane; k <= hi; k += 32) {
                int32_t value;
                if (s == 0) {
                    value = slide(first, columns, second, rows, 0, 0, a.reversed);
                    if (!EDIT) {
                        aligned[width + (k - lo)] = kUnreached;
                        aligned[2 * width + (k - lo)] = kUnreached;
                        (reinterpret_cast<uint8_t *>(aligned + 3 * width))[k - lo] = 0;
                    }
                } else if (EDIT) {
                    int move;
                    const int32_t best = furthest_source(front_at(arena, same_e, 0, k), front_at(arena, same_e, 0, k - 1),
                                                         front_at(arena, same_e, 0, k + 1), k, columns, rows, move);
                    value = best < 0 ? kUnreached : slide(first, columns, second, rows, best, k, a.reversed);
                } else {
                    const int32_t same = front_at(arena, same_e, kAligned, k);
                    const int32_t opened_below = front_at(arena, open_first_e, kAligned, k - 1);
                    const int32_t extended_below = front_at(arena, ext_first_e, kFirst, k - 1);
                    const int32_t opened_above = front_at(arena, open_second_e, kAligned, k + 1);
                    const int32_t extended_above = front_at(arena, ext_second_e, kSecond, k + 1);
                    const int32_t below = max(opened_below, extended_below);
                    const int32_t above = max(opened_above, extended_above);
                    const int32_t first_gap = below >= 0 && below < columns ? below + 1 : kUnreached;
                    const int32_t second_gap = above >= 0 && above - k <= rows ? above : kUnreached;
                    const int32_t substituted =
                        same >= 0 && same < columns && same - k < rows ? same + 1 : kUnreached;
                    const int32_t gapped = max(first_gap, second_gap);
                    // Ties as WFA2-lib's backtrace breaks them (gap_affine.mojo:984-1006): a substitution,
                    // then a letter of the first sequence alone before one of the second, and an extension
                    // before an opening.
                    uint8_t flag = 0;
                    if (opened_below > extended_below) flag |= kOpenedFirst;
                    if (opened_above > extended_above) flag |= kOpenedSecond;
                    if (!(substituted >= gapped)) flag |= first_gap >= second_gap ? kFirst : kSecond;
                    const int32_t start = max(substituted, gapped);
                    value = start >= 0 ? slide(first, columns, second, rows, start, k, a.reversed) : kUnreached;
                    aligned[width + (k - lo)] = first_gap;
                    aligned[2 * width + (k - lo)] = second_gap;
                    (reinterpret_cast<uint8_t *>(aligned + 3 * width))[k - lo] = flag;
                }
                aligned[k - lo] = value;
                if (k == target && value >= columns) hit = true;
            }
            used += bytes;
            // The front's writes and the table entry, seen by every lane before the next cost reads them.
            __syncwarp();
            if (__any_sync(kFull, hit)) {
                found = true;
                break;
            }
        }
        if (lane == 0) {
            int64_t length = 0;
            if (overflow) {
                a.results[pair] = kRetry;
                a.retry[atomicAdd(a.retry_count, 1u)] = pair;
            } else if (!found) {
                a.results[pair] = DINARA_ABOVE_MAX;
            } else {
                a.results[pair] = int64_t(s) * a.scale;
                if (a.trace) {
                    // The trace runs right to left over the sequences it searched: over the reversed pair
                    // (Ties.LEFT) that is the CIGAR's own order.
                    CigarOut out;
                    out.slot = a.slots + a.slot_offsets[pair];
                    out.capacity = 2 * (int64_t(columns) + rows) + 8;
                    out.forward = a.reversed;
                    const bool traced = EDIT ? trace_edit(a, arena, table, s, columns, rows, out)
                                             : trace_affine(a, arena, table, s, columns, rows, out);
                    out.flush();
                    length = out.written;
                    if (!traced || out.overflow) {
                        // A trace that does not reach the origin within its fronts is a failure, reported
                        // as the pair's code rather than as a CIGAR.
                        a.results[pair] = DINARA_DEVICE_FAILURE;
                        length = 0;
                    }
                }
            }
            if (a.lengths) a.lengths[pair] = length;
        }
        __syncwarp();
    }
}

// Per pair: its sort key (letters, longest first), its CIGAR slot's bytes, and a refusal for a 0xFE or
// 0xFF byte (c/dinara.h:15-17), one warp a pair.
__global__ void wave_prepare_kernel(const uint8_t *__restrict__ letters, const int64_t *__restrict__ offsets,
                                    int64_t pairs, uint32_t *__restrict__ keys, uint32_t *__restrict__ identity,
                                    int64_t *__restrict__ slot_bytes, int64_t *__restrict__ results,
                                    uint8_t *__restrict__ refused) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= pairs) return;
    const int64_t p0 = offsets[2 * warp], p2 = offsets[2 * warp + 2];
    bool bad = false;
    for (int64_t i = p0 + lane; i < p2; i += 32) bad = bad || letters[i] >= 0xFE;
    bad = __any_sync(kFull, bad);
    if (lane != 0) return;
    const int64_t letters_of_pair = p2 - p0;
    // Refused pairs sort last (key zero) and are left out of the launches; every other key is above zero.
    keys[warp] = bad ? 0u : uint32_t(letters_of_pair + 1 < 0xFFFFFFFFll ? letters_of_pair + 1 : 0xFFFFFFFFll);
    identity[warp] = uint32_t(warp);
    slot_bytes[warp] = 2 * letters_of_pair + 8;
    refused[warp] = bad ? 1 : 0;
    results[warp] = bad ? DINARA_UNSUPPORTED_SYMBOLS : kRetry;
}

// The CIGARs from their slots into one buffer, each turned round when it was written backwards.
__global__ void wave_gather_kernel(const char *__restrict__ slots, const int64_t *__restrict__ slot_offsets,
                                   const int64_t *__restrict__ lengths, const int64_t *__restrict__ offsets,
                                   char *__restrict__ out, int64_t count, bool backwards) {
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= count) return;
    const char *from = slots + slot_offsets[warp];
    const int64_t n = lengths[warp];
    char *to = out + offsets[warp];
    for (int64_t i = lane; i < n; i += 32) to[i] = backwards ? from[n - 1 - i] : from[i];
}

int64_t gcd(int64_t a, int64_t b) {
    while (b) {
        const int64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

CostPlan cost_plan(const dinara_costs *costs, const dinara_options *options) {
    CostPlan plan;
    int64_t x = 1, o = 0, e = 1, od = 0, ed = 1;
    if (costs) {
        if (costs->opening2 >= 0)
            throw Failure(DINARA_INVALID_MODE, "on the GPU, alignments under one gap piece");
        x = costs->mismatch;
        o = costs->opening;
        e = costs->extension;
        od = costs->deletion_extension > 0 ? costs->deletion_opening : o;
        ed = costs->deletion_extension > 0 ? costs->deletion_extension : e;
    }
    // Costs.affine's rules (modes.mojo:85-97): a mismatch and each gapped letter cost something, an
    // opening nothing below zero.
    if (x <= 0 || e <= 0 || ed <= 0 || o < 0 || od < 0)
        throw Failure(DINARA_INVALID_COSTS, "a mismatch or a gap's letter costing nothing, or an opening below zero");
    if (options) {
        if (options->band_low > INT64_MIN || options->band_high < INT64_MAX)
            throw Failure(DINARA_INVALID_MODE, "on the GPU, alignments with no band");
    }
    const int64_t scale = gcd(gcd(gcd(x, o), gcd(e, od)), ed);
    plan.x = x / scale;
    plan.oi = o / scale;
    plan.ei = e / scale;
    plan.od = od / scale;
    plan.ed = ed / scale;
    plan.scale = scale;
    // Unit costs (Costs.unit_scale, modes.mojo:158-163) take diagonal transition; the rest the wavefront.
    plan.edit = o == 0 && x == e && od == o && ed == e;
    const int64_t cap = options ? options->max_cost : -1;
    plan.ceiling = cap >= 0 ? cap / scale : INT32_MAX - 1;
    if (std::max({plan.x, plan.od + plan.ed, plan.oi + plan.ei}) > (1 << 20))
        throw Failure(DINARA_INVALID_COSTS, "costs whose steps pass 2^20 over their common factor");
    return plan;
}

int64_t cost_alignments(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                        const CostPlan &plan, bool right_ties, bool eqx, bool trace, int64_t *results) {
    cudaStream_t stream = gpu->stream;
    const int threads = 256;
    const unsigned warp_blocks = unsigned((pairs * 32 + threads - 1) / threads);
    uint32_t *keys = gpu->keys.ensure<uint32_t>(size_t(pairs));
    uint32_t *keys_sorted = gpu->keys_sorted.ensure<uint32_t>(size_t(pairs));
    uint32_t *identity = gpu->order.ensure<uint32_t>(size_t(pairs));
    uint32_t *order = gpu->order_sorted.ensure<uint32_t>(size_t(pairs));
    int64_t *slot_bytes = gpu->cigar_slots.ensure<int64_t>(2 * (size_t(pairs) + 1) + 2);
    int64_t *slot_offsets = slot_bytes + (pairs + 1);
    uint8_t *refused = gpu->flags.ensure<uint8_t>(size_t(pairs));
    wave_prepare_kernel<<<warp_blocks, threads, 0, stream>>>(letters, offsets, pairs, keys, identity, slot_bytes,
                                                             results, refused);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    DINARA_CUDA(cudaMemsetAsync(slot_bytes + pairs, 0, sizeof(int64_t), stream));
    size_t scan_bytes = 0, sort_bytes = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, slot_bytes, slot_offsets, int(pairs + 1), stream));
    DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, keys, keys_sorted, identity, order,
                                                          int(pairs), 0, 32, stream));
    void *space = gpu->sort_scratch.ensure<uint8_t>(std::max(scan_bytes, sort_bytes) + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, scan_bytes, slot_bytes, slot_offsets, int(pairs + 1), stream));
    DINARA_CUDA(cub::DeviceRadixSort::SortPairsDescending(space, sort_bytes, keys, keys_sorted, identity, order,
                                                          int(pairs), 0, 32, stream));
    int64_t slot_total = 0;
    read_back(gpu, &slot_total, slot_offsets + pairs, sizeof(int64_t));
    char *slots = trace ? gpu->walk_out.ensure<char>(size_t(slot_total) + 8) : nullptr;
    int64_t *lengths = gpu->cigar_lengths.ensure<int64_t>(size_t(pairs) + 1);
    DINARA_CUDA(cudaMemsetAsync(lengths, 0, (size_t(pairs) + 1) * sizeof(int64_t), stream));
    // Pairs with a refused letter sort last (key zero) and are left out of the launches.
    unsigned int *counters = gpu->counters.ensure<unsigned int>(64);
    uint32_t *retry = gpu->pending.ensure<uint32_t>(size_t(pairs));
    uint32_t *retry_next = gpu->pending_next.ensure<uint32_t>(size_t(pairs));
    // The refused pairs' count, to leave them out.
    DINARA_CUDA(cudaMemsetAsync(counters, 0, 64 * sizeof(unsigned int), stream));
    size_t count_bytes = 0;
    DINARA_CUDA(cub::DeviceReduce::Sum(nullptr, count_bytes, refused, counters + 8, int(pairs), stream));
    space = gpu->sort_scratch.ensure<uint8_t>(std::max({scan_bytes, sort_bytes, count_bytes}) + 256);
    DINARA_CUDA(cub::DeviceReduce::Sum(space, count_bytes, refused, counters + 8, int(pairs), stream));
    unsigned int refused_count = 0;
    read_back(gpu, &refused_count, counters + 8, sizeof(unsigned int));
    int64_t live = pairs - int64_t(refused_count);
    const uint32_t *launch_order = order;
    // Arenas: 256 KB a warp at first, for every resident warp; a pair that outgrows its arena runs again
    // with sixteen times the room on as many warps as the budget holds.
    int64_t arena_bytes = int64_t(256) << 10;
    const int64_t budget = int64_t(2) << 30;
    const int64_t resident_warps = int64_t(gpu->multiprocessors) * (2048 / 32);
    int rounds = 0;
    while (live > 0) {
        int64_t warps = std::min<int64_t>(resident_warps, budget / arena_bytes);
        warps = std::max<int64_t>(1, std::min<int64_t>(warps, live));
        const int64_t warps_per_block = kWaveBlock / 32;
        const int64_t blocks = (warps + warps_per_block - 1) / warps_per_block;
        uint8_t *arena = gpu->wavefront.ensure<uint8_t>(size_t(blocks * warps_per_block * arena_bytes));
        DINARA_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned int), stream));
        WaveArgs args;
        std::memset(&args, 0, sizeof args);
        args.letters = letters;
        args.offsets = offsets;
        args.order = launch_order;
        args.count = uint32_t(live);
        args.next = counters;
        args.x = int32_t(plan.x);
        args.od = int32_t(plan.od);
        args.ed = int32_t(plan.ed);
        args.oi = int32_t(plan.oi);
        args.ei = int32_t(plan.ei);
        args.scale = plan.scale;
        args.ceiling = plan.ceiling;
        args.reversed = !right_ties;
        args.eqx = eqx;
        args.trace = trace;
        args.arena = arena;
        args.arena_bytes = arena_bytes;
        args.table_entries = int32_t(std::min<int64_t>(arena_bytes / 16 / int64_t(sizeof(CostEntry)), INT32_MAX - 1));
        args.results = results;
        args.slot_offsets = slot_offsets;
        args.slots = slots;
        args.lengths = lengths;
        args.retry = retry;
        args.retry_count = counters + 1;
        ClockSpan clock(gpu, kClassTrace, stream);
        if (plan.edit)
            wavefront_kernel<true><<<unsigned(blocks), kWaveBlock, 0, stream>>>(args);
        else
            wavefront_kernel<false><<<unsigned(blocks), kWaveBlock, 0, stream>>>(args);
        DINARA_CUDA(cudaGetLastError());
        clock.stop();
        gpu->launches += 1;
        unsigned int again = 0;
        read_back(gpu, &again, counters + 1, sizeof(unsigned int));
        live = again;
        if (live == 0) break;
        arena_bytes *= 16;
        ++rounds;
        if (arena_bytes > budget || rounds > 3) {
            // Fronts past the whole budget: those pairs are refused for device memory.
            std::vector<uint32_t> left(static_cast<size_t>(live), 0u);
            DINARA_CUDA(cudaMemcpyAsync(left.data(), retry, size_t(live) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        stream));
            DINARA_CUDA(cudaStreamSynchronize(stream));
            const int64_t code = DINARA_OUT_OF_MEMORY;
            for (uint32_t p : left)
                DINARA_CUDA(cudaMemcpyAsync(results + p, &code, sizeof code, cudaMemcpyHostToDevice, stream));
            DINARA_CUDA(cudaStreamSynchronize(stream));
            break;
        }
        std::swap(retry, retry_next);
        launch_order = retry_next;
    }
    if (!trace) return 0;
    // The CIGARs' offsets, then each gathered into place.
    int64_t *cigar_offsets = gpu->cigar_offsets.ensure<int64_t>(size_t(pairs) + 2);
    DINARA_CUDA(cudaMemsetAsync(lengths + pairs, 0, sizeof(int64_t), stream));
    size_t offsets_bytes = 0;
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, offsets_bytes, lengths, cigar_offsets, int(pairs + 1), stream));
    space = gpu->sort_scratch.ensure<uint8_t>(offsets_bytes + 256);
    DINARA_CUDA(cub::DeviceScan::ExclusiveSum(space, offsets_bytes, lengths, cigar_offsets, int(pairs + 1), stream));
    int64_t total = 0;
    read_back(gpu, &total, cigar_offsets + pairs, sizeof(int64_t));
    char *out = gpu->cigar_bytes.ensure<char>(size_t(total) + 8);
    wave_gather_kernel<<<warp_blocks, threads, 0, stream>>>(slots, slot_offsets, lengths, cigar_offsets, out, pairs,
                                                            right_ties);
    DINARA_CUDA(cudaGetLastError());
    gpu->launches += 1;
    return total;
}

}  // namespace dinara
