"""Batches across the GPUs of one node, one process a GPU: every pair is independent, so a batch is split by
cost with no exchange while it runs, each rank aligns its share on its own GPU, and one gather brings the
results back in the batch's order.

The split is greedy, longest first: pairs in descending order of cells (rows x columns, or a predicted cost
when the caller has one), each to the rank with the least work so far, so the ranks finish together even
when a few long pairs carry most of the cells.
"""

from __future__ import annotations

import heapq
from typing import Callable, Optional, Sequence

import numpy as np

from . import Tape


def costs_of(tape: Tape) -> np.ndarray:
    """Each pair's cells (rows x columns), at least one."""
    rows = tape.offsets[1::2] - tape.offsets[0:-1:2]
    columns = tape.offsets[2::2] - tape.offsets[1::2]
    return np.maximum(rows * columns, 1).astype(np.float64)


def plan(costs: Sequence[float], world: int) -> list:
    """The pairs each of `world` ranks takes (index arrays, each ascending): longest first onto the least
    loaded rank."""
    if world < 1:
        raise ValueError("world: at least one rank")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, rank) for rank in range(world)]
    owned = [[] for _ in range(world)]
    for pair in order:
        load, rank = heapq.heappop(heap)
        owned[rank].append(int(pair))
        heapq.heappush(heap, (load + float(costs[pair]), rank))
    return [np.asarray(sorted(pairs), dtype=np.int64) for pairs in owned]


def subset(tape: Tape, pairs: np.ndarray) -> Tape:
    """The pairs `pairs` of a tape as a tape of their own, in that order."""
    pairs = np.asarray(pairs, dtype=np.int64)
    starts, middles, ends = tape.offsets[2 * pairs], tape.offsets[2 * pairs + 1], tape.offsets[2 * pairs + 2]
    lengths = ends - starts
    offsets = np.zeros(2 * len(pairs) + 1, dtype=np.int64)
    at = np.concatenate([[0], np.cumsum(lengths)])
    offsets[0:-1:2] = at[:-1]
    offsets[1::2] = at[:-1] + (middles - starts)
    offsets[-1] = at[-1]
    # One gather: letter j of the new tape comes from its pair's start plus its place within the pair.
    total = int(at[-1])
    source = np.arange(total, dtype=np.int64) + np.repeat(starts - at[:-1], lengths)
    letters = np.zeros(max(total, 1), dtype=np.uint8)
    letters[:total] = tape.letters[source]
    return Tape(letters, offsets)


def run(tape: Tape, align: Callable[[Tape], np.ndarray], group=None, costs: Optional[Sequence[float]] = None,
        root: int = 0) -> Optional[np.ndarray]:
    """Aligns a batch across the ranks of a torch.distributed process group: every rank passes the same
    batch and `align` (a function from a tape to one result a pair, e.g. `lambda t: dinara_align.scores_tape(t,
    scoring)`), runs it on its share, and the root gets every result in the batch's order (the others
    get None). The only collective is the gather at the end."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shares = plan(costs_of(tape) if costs is None else costs, world)
    mine = shares[rank]
    found = np.asarray(align(subset(tape, mine)) if len(mine) else np.zeros(0, dtype=np.int64))
    gathered = [None] * world if rank == root else None
    dist.gather_object((mine, found), gathered, dst=root, group=group)
    if rank != root:
        return None
    # One dtype for every rank's values: numbers promote to a common type, anything else (CIGAR strings,
    # alignments) is kept as objects, so no rank's values are cut to another's width.
    filled = [np.asarray(values) for _, values in gathered if len(values)]
    if filled and all(v.dtype.kind in "biuf" for v in filled):
        dtype = np.result_type(*filled)
    elif filled:
        dtype = object
    else:
        dtype = np.int64
    out = np.zeros(tape.pairs, dtype=dtype) if dtype is not object else np.empty(tape.pairs, dtype=object)
    for pairs, values in gathered:
        if len(pairs):
            out[pairs] = np.asarray(values, dtype=dtype) if dtype is not object else list(values)
    return out
