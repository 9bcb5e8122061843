"""Seeded synthetic batches shaped like the benchmark workloads, built with numpy.

Errors follow the reference's harness rule (benchmarks/harness.py:65-78): each letter independently
takes an edit with the pair's rate; a substitution always changes the letter, a deletion drops it, an
insertion keeps it and adds a random base after it. The split between the three is a parameter
(thirds, or 50/25/25). Sequences are uniform ACGT. The letters come back as one `Tape`, each pair's
reference (the seed sequence A) then its query (B, A with errors), as the reference's PairTape lays them.
"""

from __future__ import annotations

import numpy as np

from . import Tape

ASCII = np.frombuffer(b"ACGT", dtype=np.uint8)


def _segments(lengths: np.ndarray) -> tuple:
    """For a concatenation of segments of `lengths`: each element's segment and its place inside it."""
    starts = np.zeros(len(lengths) + 1, dtype=np.int64)
    np.cumsum(lengths, out=starts[1:])
    owner = np.repeat(np.arange(len(lengths), dtype=np.int64), lengths)
    within = np.arange(starts[-1], dtype=np.int64) - starts[:-1][owner]
    return owner, within, starts


def mutate(codes: np.ndarray, lengths: np.ndarray, rates: np.ndarray, split: tuple, rng: np.random.Generator) -> tuple:
    """Mutated copies of concatenated sequences (codes 0-3): (codes, lengths)."""
    owner, _, _ = _segments(lengths)
    rate = rates[owner]
    roll = rng.random(len(codes))
    s, d, _i = split
    substituted = roll < rate * s
    deleted = (roll >= rate * s) & (roll < rate * (s + d))
    inserted = (roll >= rate * (s + d)) & (roll < rate)
    letters = codes.copy()
    shift = rng.integers(1, 4, size=int(substituted.sum()), dtype=np.uint8)
    letters[substituted] = (letters[substituted] + shift) % 4
    emitted = 1 - deleted.astype(np.int64) + inserted.astype(np.int64)
    place = np.zeros(len(codes) + 1, dtype=np.int64)
    np.cumsum(emitted, out=place[1:])
    out = np.empty(place[-1], dtype=np.uint8)
    kept = ~deleted
    out[place[:-1][kept]] = letters[kept]
    out[place[:-1][inserted] + 1] = rng.integers(0, 4, size=int(inserted.sum()), dtype=np.uint8)
    new_lengths = np.bincount(owner, weights=emitted, minlength=len(lengths)).astype(np.int64)
    return out, new_lengths


def interleave(a: np.ndarray, a_lengths: np.ndarray, b: np.ndarray, b_lengths: np.ndarray) -> Tape:
    """Two concatenations as one tape of pairs (a_i, b_i), ASCII letters."""
    pairs = len(a_lengths)
    lengths = np.empty(2 * pairs, dtype=np.int64)
    lengths[0::2] = a_lengths
    lengths[1::2] = b_lengths
    offsets = np.zeros(2 * pairs + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    letters = np.empty(offsets[-1], dtype=np.uint8)
    owner, within, _ = _segments(a_lengths)
    letters[offsets[0:-1:2][owner] + within] = ASCII[a]
    owner, within, _ = _segments(b_lengths)
    letters[offsets[1::2][owner] + within] = ASCII[b]
    return Tape(letters, offsets)


def pairs_with_errors(rng: np.random.Generator, lengths: np.ndarray, rates, split: tuple) -> Tape:
    """Uniform ACGT references of `lengths`, each mutated at its rate."""
    lengths = np.asarray(lengths, dtype=np.int64)
    rates = np.broadcast_to(np.asarray(rates, dtype=np.float64), lengths.shape)
    a = rng.integers(0, 4, size=int(lengths.sum()), dtype=np.uint8)
    b, b_lengths = mutate(a, lengths, rates, split, rng)
    return interleave(a, lengths, b, b_lengths)


def log_uniform(rng: np.random.Generator, low: float, high: float, size: int) -> np.ndarray:
    return np.exp(rng.uniform(np.log(low), np.log(high), size=size))


THIRDS = (1 / 3, 1 / 3, 1 / 3)
HALF_QUARTERS = (0.5, 0.25, 0.25)


def unit_cost_uniform(pairs: int = 10_000, length: int = 250, rate: float = 0.02, seed: int = 1) -> Tape:
    """Global unit-cost batch: A uniform ACGT of one length, B = A at `rate` errors in thirds."""
    rng = np.random.default_rng(seed)
    return pairs_with_errors(rng, np.full(pairs, length), rate, THIRDS)


def affine_global(pairs: int = 1_000_000, low: int = 100, high: int = 300, rate: float = 0.05, seed: int = 2) -> Tape:
    """Gap-affine global batch: lengths uniform [low, high], 5% errors split 50/25/25."""
    rng = np.random.default_rng(seed)
    return pairs_with_errors(rng, rng.integers(low, high + 1, size=pairs), rate, HALF_QUARTERS)


def local_planted(pairs: int = 100_000, query_range=(150, 1000), target_range=(1000, 5000), rate: float = 0.08,
                  seed: int = 3) -> Tape:
    """Local batch: each query (150-1000 bp) mutated at `rate` (50/25/25) and planted at a uniform offset
    in a uniform ACGT target (1000-5000 bp); the target is the reference, the planted query the query."""
    rng = np.random.default_rng(seed)
    q_lengths = rng.integers(query_range[0], query_range[1] + 1, size=pairs).astype(np.int64)
    t_lengths = rng.integers(target_range[0], target_range[1] + 1, size=pairs).astype(np.int64)
    t_lengths = np.maximum(t_lengths, q_lengths)
    queries = rng.integers(0, 4, size=int(q_lengths.sum()), dtype=np.uint8)
    targets = rng.integers(0, 4, size=int(t_lengths.sum()), dtype=np.uint8)
    # Plant the unmutated query in the target; the query side carries the errors.
    _, _, t_starts = _segments(t_lengths)
    owner, within, q_starts = _segments(q_lengths)
    offset = (rng.random(pairs) * (t_lengths - q_lengths + 1)).astype(np.int64)
    targets[t_starts[:-1][owner] + offset[owner] + within] = queries
    mutated, m_lengths = mutate(queries, q_lengths, np.full(pairs, rate), HALF_QUARTERS, rng)
    return interleave(targets, t_lengths, mutated, m_lengths)


def uneven_unit_cost(pairs: int = 200_000, low: float = 100, high: float = 20_000, rate_range=(0.005, 0.15),
                     seed: int = 4) -> Tape:
    """Uneven unit-cost batch: lengths log-uniform [low, high], per-pair error uniform in `rate_range`
    (50/25/25)."""
    rng = np.random.default_rng(seed)
    lengths = np.round(log_uniform(rng, low, high, pairs)).astype(np.int64)
    rates = rng.uniform(rate_range[0], rate_range[1], size=pairs)
    return pairs_with_errors(rng, lengths, rates, HALF_QUARTERS)


def serving_request(rng: np.random.Generator, max_pairs: int = 4096, low: float = 100, high: float = 50_000,
                    rate_range=(0.01, 0.10)) -> Tape:
    """One serving request: 1-`max_pairs` pairs (log-uniform), lengths log-uniform, 1-10% errors."""
    count = max(1, int(round(log_uniform(rng, 1, max_pairs, 1)[0])))
    lengths = np.round(log_uniform(rng, low, high, count)).astype(np.int64)
    rates = rng.uniform(rate_range[0], rate_range[1], size=count)
    return pairs_with_errors(rng, lengths, rates, HALF_QUARTERS)
