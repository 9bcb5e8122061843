"""ctypes face of the CPU oracle (oracle/dinara_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by `__graft_entry__.smoke()` and by the CPU-baseline leg
of `bench.py`, always as the checker or the timed CPU restatement, never by the product package.

Letters are codes into a Scoring's alphabet; gaps are in the kernels' terms (`open` a gap's first
letter, `extend` each further one), as dinara_align/gotoh.mojo:40-60 keeps them.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "liboracle.so")

GLOBAL, LOCAL = 0, 1
GAP = 255

_lib = None


def build() -> str:
    """Compiles the oracle with its Makefile when the library is missing or older than its source."""
    source = os.path.join(HERE, "dinara_oracle.c")
    if not os.path.exists(LIBRARY) or os.path.getmtime(LIBRARY) < os.path.getmtime(source):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIBRARY


def lib() -> ctypes.CDLL:
    """The loaded oracle library, built first if needed."""
    global _lib
    if _lib is None:
        build()
        handle = ctypes.CDLL(LIBRARY)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        i8p = ctypes.POINTER(ctypes.c_int8)
        i64 = ctypes.c_int64
        i64p = ctypes.POINTER(ctypes.c_int64)
        i32 = ctypes.c_int32
        i32p = ctypes.POINTER(ctypes.c_int32)
        handle.oracle_gotoh_score.restype = i32
        handle.oracle_gotoh_score.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, i32, i64p, i64p]
        handle.oracle_gotoh_score_free.restype = i32
        handle.oracle_gotoh_score_free.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, i64, i64, i64, i64]
        handle.oracle_gotoh_extension_zdrop.restype = i32
        handle.oracle_gotoh_extension_zdrop.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, i64, i64,
                                                        ctypes.POINTER(i64), ctypes.POINTER(i64),
                                                        ctypes.POINTER(ctypes.c_int32)]
        handle.oracle_gotoh_extension.restype = i32
        handle.oracle_gotoh_extension.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, ctypes.POINTER(i64),
                                                  ctypes.POINTER(i64)]
        handle.oracle_gotoh_end_free.restype = i32
        handle.oracle_gotoh_end_free.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, i64, i64, i64, i64, i32,
                                                 ctypes.POINTER(i64), ctypes.POINTER(i64)]
        handle.oracle_gotoh_align.restype = i32
        handle.oracle_gotoh_align.argtypes = [u8p, i64, u8p, i64, i8p, i32, i32, i32, i32, u8p, u8p, i64p]
        handle.oracle_cigar.restype = i64
        handle.oracle_cigar.argtypes = [u8p, u8p, i64, i32, ctypes.c_char_p]
        for name in ("oracle_edit_distance_dp", "oracle_myers_distance"):
            getattr(handle, name).restype = i64
            getattr(handle, name).argtypes = [u8p, i64, u8p, i64]
        handle.oracle_band_doubling.restype = i64
        handle.oracle_band_doubling.argtypes = [u8p, i64, u8p, i64, i64, i64p, i64p]
        handle.oracle_banded_round.restype = i64
        handle.oracle_banded_round.argtypes = [u8p, i64, u8p, i64, i64, i64p]
        handle.oracle_score_reach_refuses.restype = i32
        handle.oracle_score_reach_refuses.argtypes = [i8p, i32, i32, i32, i64, i64, i32]
        handle.oracle_batch_scores.restype = None
        handle.oracle_batch_scores.argtypes = [i64, u8p, i64p, i8p, i32, i32, i32, i32, i32, i32p]
        handle.oracle_batch_alignments.restype = None
        handle.oracle_batch_alignments.argtypes = [i64, u8p, i64p, i8p, i32, i32, i32, i32, i32, i32, i32p,
                                                   ctypes.c_char_p, i64, i64p]
        handle.oracle_edit_cigar.restype = i64
        handle.oracle_edit_cigar.argtypes = [u8p, i64, u8p, i64, i32, i32, ctypes.c_char_p, i64]
        handle.oracle_affine_cigar.restype = i64
        handle.oracle_affine_cigar.argtypes = [u8p, i64, u8p, i64, i64, i64, i64, i64, i64, i64, i32, i32,
                                               ctypes.c_char_p, i64]
        handle.oracle_batch_wavefront.restype = None
        handle.oracle_batch_wavefront.argtypes = [i64, u8p, i64p, i64, i64, i64, i64, i64, i32, i32, i64p,
                                                  ctypes.c_char_p, i64, i64p]
        handle.oracle_batch_distances.restype = None
        handle.oracle_batch_distances.argtypes = [i64, u8p, i64p, i64, i32, i64p]
        _lib = handle
    return _lib


def _u8(array) -> tuple:
    if isinstance(array, (bytes, bytearray)):
        array = np.frombuffer(bytes(array), dtype=np.uint8)
    elif isinstance(array, str):
        array = np.frombuffer(array.encode("ascii"), dtype=np.uint8)
    data = np.ascontiguousarray(array, dtype=np.uint8)
    return data, data.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _i8(array) -> tuple:
    data = np.ascontiguousarray(array, dtype=np.int8)
    return data, data.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))


def codes(text, alphabet: str = "ACGT") -> np.ndarray:
    """`text` (str or bytes) as its letters' places in `alphabet` (common.mojo:277-286 translate)."""
    raw = text.encode("ascii") if isinstance(text, str) else bytes(text)
    table = np.full(256, 255, dtype=np.uint8)
    for place, letter in enumerate(alphabet.encode("ascii")):
        table[letter] = place
    out = table[np.frombuffer(raw, dtype=np.uint8)]
    if (out == 255).any():
        raise ValueError(f"a letter outside the alphabet {alphabet!r}")
    return out


def gotoh_score(first, second, table, size, open_, extend, mode=GLOBAL) -> tuple:
    """(score, end_row, end_column) of one pair in codes (the end is a local alignment's best cell)."""
    a, pa = _u8(first)
    b, pb = _u8(second)
    t, pt = _i8(table)
    row, column = ctypes.c_int64(), ctypes.c_int64()
    score = lib().oracle_gotoh_score(pa, len(a), pb, len(b), pt, size, open_, extend, mode, ctypes.byref(row),
                                     ctypes.byref(column))
    return score, row.value, column.value


def gotoh_score_free(a, b, table, size, open_, extend, reference_start=0, reference_end=0, query_start=0,
                     query_end=0) -> int:
    """The best score of a (codes, reference down the rows) against b with the given free letters at each
    end of each (scored.mojo:69-240)."""
    first, pa = _u8(a)
    second, pb = _u8(b)
    t, pt = _i8(table)
    big = (1 << 62)
    return int(lib().oracle_gotoh_score_free(pa, len(first), pb, len(second), pt, size, open_, extend,
                                             min(reference_start, big), min(reference_end, big),
                                             min(query_start, big), min(query_end, big)))


def gotoh_end_free(a, b, table, size, open_, extend, reference_start=0, reference_end=0, query_start=0,
                   query_end=0, highest=True) -> tuple:
    """(score, end_row, end_column) with free ends: the best end, of equal ones the furthest along the
    reference less the query (`highest`) or the least so (scored.mojo:69-100, 155-176)."""
    first, pa = _u8(a)
    second, pb = _u8(b)
    t, pt = _i8(table)
    big = (1 << 62)
    row, column = ctypes.c_int64(), ctypes.c_int64()
    score = lib().oracle_gotoh_end_free(pa, len(first), pb, len(second), pt, size, open_, extend,
                                        min(reference_start, big), min(reference_end, big), min(query_start, big),
                                        min(query_end, big), 1 if highest else 0, ctypes.byref(row),
                                        ctypes.byref(column))
    return int(score), row.value, column.value


def free_ends_alignment(a, b, table, size, open_, extend, reference_start=0, reference_end=0, query_start=0,
                        query_end=0, eqx=True) -> tuple:
    """(score, cigar, (reference start, reference end, query start, query end)) of a pair in codes with free
    ends under a Scoring, as the reference's host path places and aligns it (scoring.mojo:690-722 mode_span,
    scored.mojo:616-633 started_span, scoring.mojo:800-813): the best end, of equal ones the furthest along
    the reference less the query; the start by a sweep back over both prefixes to it, reversed, the letters
    free at the start free at its end, taking its end the least so; and the letters between them aligned
    globally by the full-matrix walk."""
    a = np.asarray(a, dtype=np.uint8)
    b = np.asarray(b, dtype=np.uint8)
    rs, re_ = min(reference_start, len(a)), min(reference_end, len(a))
    qs, qe = min(query_start, len(b)), min(query_end, len(b))
    score, end_row, end_column = gotoh_end_free(a, b, table, size, open_, extend, rs, re_, qs, qe, True)
    back, row, column = gotoh_end_free(a[:end_row][::-1].copy(), b[:end_column][::-1].copy(), table, size, open_,
                                       extend, 0, rs, 0, qs, False)
    start_row, start_column = end_row - row, end_column - column
    inner, cigar = gotoh_align(a[start_row:end_row], b[start_column:end_column], table, size, open_, extend,
                               GLOBAL, eqx)[:2]
    assert back == score == inner, (score, back, inner)
    return score, cigar, (start_row, end_row, start_column, end_column)


def gotoh_extension(a, b, table, size, open_, extend) -> tuple:
    """(score, stop_row, stop_column) of an extension from the origin (scored.mojo:69-100, 272-300)."""
    first, pa = _u8(a)
    second, pb = _u8(b)
    t, pt = _i8(table)
    row, column = ctypes.c_int64(), ctypes.c_int64()
    score = lib().oracle_gotoh_extension(pa, len(first), pb, len(second), pt, size, open_, extend, ctypes.byref(row),
                                         ctypes.byref(column))
    return int(score), row.value, column.value


def gotoh_extension_zdrop(a, b, table, size, open_, extend, zdrop) -> tuple:
    """(score, stop_row, stop_column, dropped) of an extension from the origin with a Z-drop (scored.mojo:272-300),
    its slack a diagonal the cheapest a gap grows a letter, -extend."""
    first, pa = _u8(a)
    second, pb = _u8(b)
    t, pt = _i8(table)
    row, column, dropped = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    score = lib().oracle_gotoh_extension_zdrop(pa, len(first), pb, len(second), pt, size, open_, extend, zdrop,
                                               -extend, ctypes.byref(row), ctypes.byref(column),
                                               ctypes.byref(dropped))
    return int(score), row.value, column.value, bool(dropped.value)


def extension_alignment(a, b, table, size, open_, extend, from_end=False, end_bonus=-1, eqx=True,
                        zdrop=-1) -> tuple:
    """(score, cigar, (reference start, reference end, query start, query end)) of an extension under a
    Scoring, as the reference's host path makes it (scoring.mojo:673-722 extension_span and mode_span,
    800-813): the best stop from the starts, or from the ends over both sequences reversed, with a Z-drop
    when `zdrop` is 0 or more; with an end bonus and no drop, the alignment reaching the query's far end
    (free ends: the reference's far end free) when its score plus the bonus passes the stop's; then the
    span's letters aligned globally."""
    a = np.asarray(a, dtype=np.uint8)
    b = np.asarray(b, dtype=np.uint8)
    n, m = len(a), len(b)
    x, y = (a[::-1].copy(), b[::-1].copy()) if from_end else (a, b)
    dropped = False
    if zdrop >= 0:
        score, row, column, dropped = gotoh_extension_zdrop(x, y, table, size, open_, extend, zdrop)
    else:
        score, row, column = gotoh_extension(x, y, table, size, open_, extend)
    span = (n - row, n, m - column, m) if from_end else (0, row, 0, column)
    if end_bonus > 0 and not dropped:
        big = 1 << 62
        counts = (big, 0, 0, 0) if from_end else (0, big, 0, 0)
        reach, _cigar, reach_span = free_ends_alignment(a, b, table, size, open_, extend, *counts, eqx=eqx)
        if reach + end_bonus > score:
            score, span = reach, reach_span
    inner, cigar = gotoh_align(a[span[0]:span[1]], b[span[2]:span[3]], table, size, open_, extend, GLOBAL, eqx)[:2]
    assert inner == score, (inner, score)
    return score, cigar, span


def gotoh_align(first, second, table, size, open_, extend, mode=GLOBAL, eqx=True) -> tuple:
    """(score, cigar, top, bottom): the full-matrix walk's alignment, rows as code arrays, 255 a gap."""
    a, pa = _u8(first)
    b, pb = _u8(second)
    t, pt = _i8(table)
    top = np.zeros(len(a) + len(b) + 1, dtype=np.uint8)
    bottom = np.zeros(len(a) + len(b) + 1, dtype=np.uint8)
    length = ctypes.c_int64()
    score = lib().oracle_gotoh_align(pa, len(a), pb, len(b), pt, size, open_, extend, mode,
                                     top.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                     bottom.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.byref(length))
    n = length.value
    out = ctypes.create_string_buffer(2 * n + 2)
    lib().oracle_cigar(top.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                       bottom.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, 1 if eqx else 0, out)
    return score, out.value.decode("ascii"), top[:n].copy(), bottom[:n].copy()


def edit_distance_dp(a, b) -> int:
    x, px = _u8(a)
    y, py = _u8(b)
    return lib().oracle_edit_distance_dp(px, len(x), py, len(y))


def myers_distance(a, b) -> int:
    x, px = _u8(a)
    y, py = _u8(b)
    return lib().oracle_myers_distance(px, len(x), py, len(y))


def band_doubling(a, b, start: int) -> tuple:
    """(distance, rounds, words swept) of plain band doubling from threshold `start`."""
    x, px = _u8(a)
    y, py = _u8(b)
    rounds, words = ctypes.c_int64(), ctypes.c_int64()
    distance = lib().oracle_band_doubling(px, len(x), py, len(y), start, ctypes.byref(rounds), ctypes.byref(words))
    return distance, rounds.value, words.value


def banded_round(a, b, threshold: int) -> int:
    x, px = _u8(a)
    y, py = _u8(b)
    return lib().oracle_banded_round(px, len(x), py, len(y), threshold, None)


def edit_cigar(first, second, right=False, eqx=True) -> tuple:
    """(distance, CIGAR) at unit costs by the Ties rule: Ties.RIGHT with `right`, else Ties.LEFT."""
    a, pa = _u8(first)
    b, pb = _u8(second)
    capacity = 2 * (len(a) + len(b)) + 8
    out = ctypes.create_string_buffer(capacity)
    distance = lib().oracle_edit_cigar(pa, len(a), pb, len(b), 1 if right else 0, 1 if eqx else 0, out, capacity)
    return distance, out.value.decode("ascii")


def affine_cigar(first, second, mismatch, opening, extension, deletion_opening=None, deletion_extension=None,
                 max_cost=-1, right=False, eqx=True) -> tuple:
    """(cost, CIGAR) under one-piece Costs by the wavefront and the Ties rule; cost -4 past `max_cost`.
    Deletions (letters of the first alone) cost as insertions unless their own costs are given."""
    a, pa = _u8(first)
    b, pb = _u8(second)
    capacity = 2 * (len(a) + len(b)) + 8
    out = ctypes.create_string_buffer(capacity)
    od = opening if deletion_opening is None else deletion_opening
    ed = extension if deletion_extension is None else deletion_extension
    cost = lib().oracle_affine_cigar(pa, len(a), pb, len(b), mismatch, od, ed, opening, extension, max_cost,
                                     1 if right else 0, 1 if eqx else 0, out, capacity)
    return cost, out.value.decode("ascii")


def score_reach_refuses(table, size, open_, extend, rows, columns, mode=GLOBAL) -> bool:
    t, pt = _i8(table)
    return bool(lib().oracle_score_reach_refuses(pt, size, open_, extend, rows, columns, mode))


def tape_of(firsts, seconds) -> tuple:
    """Pairs of code arrays as one tape and its offsets (scoring.mojo:267-340 PairTape)."""
    pieces, offsets, at = [], [0], 0
    for a, b in zip(firsts, seconds):
        pieces.append(np.asarray(a, dtype=np.uint8))
        at += len(a)
        offsets.append(at)
        pieces.append(np.asarray(b, dtype=np.uint8))
        at += len(b)
        offsets.append(at)
    tape = np.concatenate(pieces) if pieces else np.zeros(1, dtype=np.uint8)
    if len(tape) == 0:
        tape = np.zeros(1, dtype=np.uint8)
    return tape, np.asarray(offsets, dtype=np.int64)


def batch_scores(tape, offsets, table, size, open_, extend, mode=GLOBAL, threads=1) -> np.ndarray:
    pairs = (len(offsets) - 1) // 2
    t, pt = _u8(tape)
    o = np.ascontiguousarray(offsets, dtype=np.int64)
    s, ps = _i8(table)
    out = np.zeros(max(pairs, 1), dtype=np.int32)
    lib().oracle_batch_scores(pairs, pt, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ps, size, open_, extend,
                              mode, threads, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return out[:pairs]


def batch_alignments(tape, offsets, table, size, open_, extend, mode=GLOBAL, eqx=True, threads=1,
                     stride=None) -> tuple:
    """(scores, cigars as a list of str)."""
    pairs = (len(offsets) - 1) // 2
    t, pt = _u8(tape)
    o = np.ascontiguousarray(offsets, dtype=np.int64)
    s, ps = _i8(table)
    lengths = o[1::2][:pairs] - o[0::2][:pairs] + o[2::2][:pairs] - o[1::2][:pairs] if pairs else np.zeros(0)
    stride = stride or int(2 * (lengths.max() if pairs else 0) + 2)
    scores = np.zeros(max(pairs, 1), dtype=np.int32)
    cigars = ctypes.create_string_buffer(max(pairs, 1) * stride)
    cigar_lengths = np.zeros(max(pairs, 1), dtype=np.int64)
    lib().oracle_batch_alignments(pairs, pt, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ps, size, open_,
                                  extend, mode, 1 if eqx else 0, threads,
                                  scores.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), cigars, stride,
                                  cigar_lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    raw = cigars.raw
    out = [raw[p * stride: p * stride + int(cigar_lengths[p])].decode("ascii") for p in range(pairs)]
    return scores[:pairs], out


def batch_distances(tape, offsets, start=-1, threads=1) -> np.ndarray:
    """Unit-cost distances: plain band doubling from `start`, or the whole matrix for a negative start."""
    pairs = (len(offsets) - 1) // 2
    t, pt = _u8(tape)
    o = np.ascontiguousarray(offsets, dtype=np.int64)
    out = np.zeros(max(pairs, 1), dtype=np.int64)
    lib().oracle_batch_distances(pairs, pt, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), start, threads,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out[:pairs]


def dna_table(match: int, mismatch: int) -> np.ndarray:
    """Scoring.uniform's table over ACGT (common.mojo:255-266 uniform_matrix)."""
    return np.array([match if r == c else mismatch for r in range(4) for c in range(4)], dtype=np.int8)


def kernel_gaps(opening: int, extension: int) -> tuple:
    """A Scoring's (opening, extension) in the kernels' terms (scoring.mojo:202-215 gap_scores)."""
    return opening + extension, extension


def batch_wavefront(tape, offsets, mismatch, opening, extension, cigars=True, eqx=True, threads=1) -> tuple:
    """(costs, CIGARs or None) of every pair under Costs.affine(mismatch, opening, extension) by the
    wavefront, threaded: the reference's host path for a global alignment under a uniform Scoring."""
    pairs = (len(offsets) - 1) // 2
    t, pt = _u8(tape)
    o = np.ascontiguousarray(offsets, dtype=np.int64)
    costs = np.zeros(max(pairs, 1), dtype=np.int64)
    lengths = o[2::2][:pairs] - o[0::2][:pairs] if pairs else np.zeros(0, dtype=np.int64)
    stride = int(2 * (lengths.max() if pairs else 0) + 8)
    buffer = ctypes.create_string_buffer(max(pairs, 1) * stride) if cigars else None
    cigar_lengths = np.zeros(max(pairs, 1), dtype=np.int64)
    lib().oracle_batch_wavefront(pairs, pt, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), mismatch, opening,
                                 extension, opening, extension, 1 if eqx else 0, threads,
                                 costs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), buffer, stride,
                                 cigar_lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if not cigars:
        return costs[:pairs], None
    raw = buffer.raw
    return costs[:pairs], [raw[p * stride: p * stride + int(cigar_lengths[p])].decode("ascii") for p in range(pairs)]
