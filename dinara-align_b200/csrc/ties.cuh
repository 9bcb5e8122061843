// Global alignments under Costs with the reference's Ties rule on the GPU (ties.cu).
#pragma once

#include "internal.cuh"

namespace dinara {

// Costs in the wavefront's terms: over their common factor (Penalties.scale), a deletion (a letter of
// the first sequence, the reference, alone) and an insertion each with an opening and an extension.
struct CostPlan {
    int64_t x = 1, od = 0, ed = 1, oi = 0, ei = 1;
    int64_t scale = 1;
    int64_t ceiling = 0;  // the largest cost over the common factor a pair may take
    bool edit = true;     // unit costs: diagonal transition and its trace
};

// Checks a dinara_costs (one gap piece; null for unit costs) and the options (no band; `max_cost`
// caps), throwing Failure for what the GPU does not take.
CostPlan cost_plan(const dinara_costs *costs, const dinara_options *options);

// Each pair's least cost into `results` (device, per pair; or its code: -1 a 0xFE/0xFF byte, -4 above
// the cap, -2 fronts past the device budget) and, with `trace`, its CIGAR by the Ties rule, Ties.RIGHT
// with `right_ties`; returns the CIGAR bytes' total and leaves their offsets (pairs + 1, device) in
// gpu->cigar_offsets and the bytes in gpu->cigar_bytes. Letters and offsets are on the device.
int64_t cost_alignments(dinara_gpu *gpu, int64_t pairs, const uint8_t *letters, const int64_t *offsets,
                        const CostPlan &plan, bool right_ties, bool eqx, bool trace, int64_t *results);

}  // namespace dinara
