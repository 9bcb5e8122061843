"""dinara-align's batched alignment path on an NVIDIA B200.

The same Python surface as dinara-align's package (python/dinara_align/__init__.py in the reference) for
the batched GPU path: `Costs`, `Mode`, `Band`, `Scoring` and `Alignment` with the same fields and
factories, `distances` and `alignments` with the same signatures, the reference's batch `scores` under a
`Scoring` (api.mojo:843-892), and a `placement` keyword naming the GPU (api.mojo:1224, :849, :901).
Everything runs on the GPU through libdinara_gpu.so; a call the GPU path does not serve raises
ValueError, as the reference's GPU placement does (api.mojo:1240-1246, scoring.mojo:753-757).

>>> import dinara_align as da
>>> da.distances(["ACGTACGTTTGCA"], ["ACGTCGTTTTGCA"])
[2]
>>> da.scores(["ACGTTGCAGGGCATGACGT"], ["ACGTTGCACATGACGT"], da.Scoring.dna())
[22]
>>> da.alignments(["ACGTTGCAGGGCATGACGT"], ["ACGTTGCACATGACGT"], da.Scoring.dna())[0].cigar
'8=3D8='
"""

from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass, replace
from typing import Optional, Sequence, Union

import numpy as np

from . import _native as native

__all__ = [
    "Alignment",
    "Band",
    "Costs",
    "Mode",
    "Placement",
    "Scoring",
    "align",
    "alignments",
    "distance",
    "distances",
    "score",
    "scores",
    "Tape",
]

UNBOUNDED = 1 << 60
"""As many free letters as any sequence has, and a band edge past every diagonal (the reference's)."""

Text = Union[str, bytes]
_ENDS, _EXTENSION, _LOCAL = 0, 1, 2


def _text(sequence: Text) -> bytes:
    """A sequence as ASCII bytes: TypeError unless str or bytes, ValueError unless ASCII."""
    if isinstance(sequence, (bytes, bytearray)):
        return bytes(sequence)
    if not isinstance(sequence, str):
        raise TypeError(f"a sequence is a str or bytes, not {type(sequence).__name__}")
    if not sequence.isascii():
        raise ValueError("a sequence holds ASCII letters alone")
    return sequence.encode("ascii")


def _integers(*values) -> tuple:
    for value in values:
        if not isinstance(value, int):
            raise TypeError(f"an integer, not {type(value).__name__}")
    return values


@dataclass(frozen=True)
class Costs:
    """What each edit costs (the reference's `Costs`, fields in `dinara_costs` order). The GPU path
    measures unit costs, `Costs.edit()`."""

    mismatch: int = 1
    opening: int = 0
    extension: int = 1
    opening2: int = -1
    extension2: int = 0
    deletion_opening: int = 0
    deletion_extension: int = 0
    deletion_opening2: int = -1
    deletion_extension2: int = 0

    @staticmethod
    def edit() -> "Costs":
        return Costs()

    @staticmethod
    def linear(mismatch: int, gap: int) -> "Costs":
        return Costs(mismatch, 0, gap)

    @staticmethod
    def affine(mismatch: int, opening: int, extension: int) -> "Costs":
        return Costs(mismatch, opening, extension)

    @staticmethod
    def two_piece(mismatch: int, opening: int, extension: int, opening2: int, extension2: int) -> "Costs":
        if _integers(extension2)[0] <= 0 or _integers(opening2)[0] < 0:
            raise ValueError(f"second piece {opening2}, {extension2}: its extension must cost")
        return Costs(mismatch, opening, extension, opening2, extension2)

    def with_deletions(self, opening: int, extension: int, opening2: int = -1, extension2: int = 0) -> "Costs":
        """These costs with deletions (runs of reference letters alone) of their own, the others an
        insertion's, as bwa's `-O del,ins`."""
        if _integers(extension)[0] <= 0 or _integers(opening)[0] < 0 or (
                _integers(opening2)[0] >= 0 and _integers(extension2)[0] <= 0):
            raise ValueError(f"deletions {opening}, {extension}: an extension must cost")
        return replace(self, deletion_opening=opening, deletion_extension=extension, deletion_opening2=opening2,
                       deletion_extension2=extension2)

    def symmetric(self) -> bool:
        """Whether deletions cost what insertions do."""
        return self.deletion_extension == 0 or (
            self.deletion_opening, self.deletion_extension, self.deletion_opening2, self.deletion_extension2) == (
            self.opening, self.extension, self.opening2, self.extension2)

    def unit_scale(self) -> int:
        """The multiple of the edit distance these costs price every pair at, or 0 if they are not unit
        costs: a mismatch and a gap letter alike, no opening, one piece (modes.mojo:158-163)."""
        if self.opening2 >= 0 or self.opening != 0 or self.mismatch != self.extension or not self.symmetric():
            return 0
        return self.mismatch if self.mismatch > 0 else 0

    def _struct(self) -> native.CCosts:
        return native.CCosts(*_integers(self.mismatch, self.opening, self.extension, self.opening2, self.extension2,
                                        self.deletion_opening, self.deletion_extension, self.deletion_opening2,
                                        self.deletion_extension2))


class Anchor:
    """Which end of both sequences an extension is fixed at (the reference's)."""

    START = 0
    END = 1


@dataclass(frozen=True)
class Mode:
    """Which alignments count (the reference's `Mode`, fields in `dinara_mode` order). The GPU serves
    `Mode.GLOBAL` and, under a `Scoring`, `Mode.local()`, free ends (`INFIX`, `PREFIX`, `SUFFIX` and
    `ends_free(...)`) and `extension(0, ...)` (no match score of the mode's own), scores and alignments,
    the latter placed as the reference's host path places them."""

    kind: int = _ENDS
    reference_start: int = 0
    reference_end: int = 0
    query_start: int = 0
    query_end: int = 0
    match_score: int = 0
    anchor: int = Anchor.START
    zdrop: int = -1
    end_bonus: int = -1

    GLOBAL = None
    INFIX = None
    PREFIX = None
    SUFFIX = None

    @staticmethod
    def ends_free(reference_start=0, reference_end=0, query_start=0, query_end=0) -> "Mode":
        return Mode(_ENDS, reference_start, reference_end, query_start, query_end)

    def with_match_score(self, match_score: int) -> "Mode":
        return replace(self, match_score=match_score)

    @staticmethod
    def extension(match_score: int, anchor: int = Anchor.START, *, zdrop: int = -1, end_bonus: int = -1) -> "Mode":
        """A seed's extension from both starts (or `anchor` END, both ends), a match earning
        `match_score`. Under a `Scoring` (match score 0: the table's own) the GPU serves it, scores and
        alignments, with a Z-drop and an end bonus."""
        return Mode(_EXTENSION, match_score=match_score, anchor=anchor, zdrop=zdrop, end_bonus=end_bonus)

    @staticmethod
    def local(match_score: int = 0) -> "Mode":
        return Mode(_LOCAL, match_score=match_score)

    @staticmethod
    def overlap(match_score: int) -> "Mode":
        """Every end free and a match earning `match_score` (parasail's `sg`); the GPU path refuses it."""
        return Mode(_ENDS, UNBOUNDED, UNBOUNDED, UNBOUNDED, UNBOUNDED, match_score)

    def is_global(self) -> bool:
        return self.kind == _ENDS and not (self.reference_start or self.reference_end or self.query_start
                                           or self.query_end)

    def _struct(self) -> native.CMode:
        fields = _integers(self.kind, self.reference_start, self.reference_end, self.query_start, self.query_end,
                           self.match_score, self.anchor, self.zdrop, self.end_bonus)
        return native.CMode(*[min(value, UNBOUNDED) for value in fields])


Mode.GLOBAL = Mode()
Mode.INFIX = Mode(_ENDS, UNBOUNDED, UNBOUNDED, 0, 0)
Mode.PREFIX = Mode(_ENDS, 0, UNBOUNDED, 0, 0)
Mode.SUFFIX = Mode(_ENDS, UNBOUNDED, 0, 0, 0)


@dataclass(frozen=True)
class Band:
    low: int = -UNBOUNDED
    high: int = UNBOUNDED

    @staticmethod
    def around(width: int) -> "Band":
        return Band(-width, width)


@dataclass(frozen=True)
class Scoring:
    """A substitution table over an alphabet, row by row, and a gap of k letters scoring
    `opening + k * extension` (the reference's `Scoring`)."""

    alphabet: str
    table: tuple
    opening: int = -4
    extension: int = -2

    @staticmethod
    def dna() -> "Scoring":
        return Scoring.uniform(2, -4)

    @staticmethod
    def uniform(match: int, mismatch: int, opening: int = -4, extension: int = -2, alphabet: str = "ACGT") -> "Scoring":
        size = len(alphabet)
        table = tuple(match if row == column else mismatch for row in range(size) for column in range(size))
        return Scoring(alphabet, table, opening, extension)

    @staticmethod
    def tabulated(alphabet: str, table: Sequence[int], opening: int = -4, extension: int = -2) -> "Scoring":
        return Scoring(alphabet, tuple(table), opening, extension)

    def _struct(self) -> tuple:
        if not isinstance(self.alphabet, str) or not self.alphabet.isascii():
            raise ValueError("an alphabet is a str of ASCII letters")
        cells = list(_integers(*self.table))
        if any(cell < -128 or cell > 127 for cell in cells):
            raise ValueError("a table's cells lie within -128 and 127")
        size = len(self.alphabet)
        if len(cells) != size * size:
            raise ValueError(f"{len(cells)} scores for {size * size} pairs of letters")
        _integers(self.opening, self.extension)
        table = np.asarray(cells, dtype=np.int8)
        alphabet = self.alphabet.encode("ascii")
        struct = native.CScoring(alphabet, size, native.pointer(table, ctypes.c_int8), self.opening, self.extension)
        return struct, table, alphabet


@dataclass(frozen=True)
class Alignment:
    """An alignment of reference[reference_start:reference_end] against query[query_start:query_end] as a
    CIGAR over those letters ('=' 'X' or 'M', 'D' a reference letter alone, 'I' a query letter alone)."""

    cost: int
    score: int
    cigar: str
    reference_start: int
    reference_end: int
    query_start: int
    query_end: int

    def runs(self) -> list:
        out, length = [], 0
        for letter in self.cigar:
            if letter.isdigit():
                length = length * 10 + int(letter)
            else:
                out.append((length, letter))
                length = 0
        return out

    def gapped(self, reference: Text, query: Text) -> tuple:
        reference, query = _text(reference).decode(), _text(query).decode()
        top, bottom = [], []
        column, row = self.reference_start, self.query_start
        for length, operation in self.runs():
            if operation == "D":
                top.append(reference[column:column + length])
                bottom.append("-" * length)
                column += length
            elif operation == "I":
                top.append("-" * length)
                bottom.append(query[row:row + length])
                row += length
            else:
                top.append(reference[column:column + length])
                bottom.append(query[row:row + length])
                column += length
                row += length
        return "".join(top), "".join(bottom)

    def clipped_cigar(self, query_length: int, hard: bool = False) -> str:
        """The CIGAR as a SAM record carries it: the query's letters before and after the span clipped,
        soft ('S') or with `hard` hard ('H'); the record's POS is reference_start + 1."""
        clip = "H" if hard else "S"
        head = f"{self.query_start}{clip}" if self.query_start > 0 else ""
        tail = f"{query_length - self.query_end}{clip}" if query_length > self.query_end else ""
        return head + self.cigar + tail

    def edit_distance(self, reference: Text, query: Text) -> int:
        """SAM's NM: substitutions and gapped letters of the aligned span."""
        top, bottom = self.gapped(reference, query)
        return sum(a != b for a, b in zip(top, bottom))

    def identity(self, reference: Text, query: Text) -> float:
        """Matching columns over all columns of the alignment (BLAST's identity); 0 with no columns."""
        top, bottom = self.gapped(reference, query)
        return sum(a == b for a, b in zip(top, bottom)) / len(top) if top else 0.0

    def mismatch_string(self, reference: Text, query: Text) -> str:
        """SAM's MD tag: runs of matched reference letters, each mismatched reference letter, and '^'
        before each run of deleted ones; inserted query letters leave no mark."""
        top, bottom = self.gapped(reference, query)
        pieces, matched, in_deletion = [], 0, False
        for a, b in zip(top, bottom):
            if b == "-":
                if not in_deletion:
                    pieces.append(f"{matched}^")
                    matched, in_deletion = 0, True
                pieces.append(a)
                continue
            in_deletion = False
            if a == "-":
                continue
            if a == b:
                matched += 1
            else:
                pieces.append(f"{matched}{a}")
                matched = 0
        pieces.append(str(matched))
        return "".join(pieces)


@dataclass(frozen=True)
class Placement:
    """Where a batch runs: the GPU `gpu_id` (the reference's `Placement.on_gpu`, common.mojo:130-160)."""

    gpu_id: int = 0

    @staticmethod
    def on_gpu(gpu_id: int = 0) -> "Placement":
        return Placement(gpu_id)


class Tape:
    """Pairs laid end to end, the reference's PairTape (scoring.mojo:267-340): pair i's reference is
    `letters[offsets[2i]:offsets[2i+1]]` and its query `letters[offsets[2i+1]:offsets[2i+2]]`."""

    def __init__(self, letters: np.ndarray, offsets: np.ndarray):
        self.letters = np.ascontiguousarray(letters, dtype=np.uint8)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        if len(self.letters) == 0:
            self.letters = np.zeros(1, dtype=np.uint8)

    @property
    def pairs(self) -> int:
        return (len(self.offsets) - 1) // 2

    @staticmethod
    def of(references: Sequence[Text], queries: Sequence[Text]) -> "Tape":
        if len(references) != len(queries):
            raise ValueError(f"{len(references)} references against {len(queries)} queries")
        interleaved = [None] * (2 * len(references))
        interleaved[0::2] = [_text(item) for item in references]
        interleaved[1::2] = [_text(item) for item in queries]
        lengths = np.fromiter((len(item) for item in interleaved), dtype=np.int64, count=len(interleaved))
        offsets = np.zeros(len(interleaved) + 1, dtype=np.int64)
        np.cumsum(lengths, out=offsets[1:])
        letters = np.frombuffer(b"".join(interleaved), dtype=np.uint8)
        return Tape(letters, offsets)

    def reference(self, pair: int) -> bytes:
        return self.letters[self.offsets[2 * pair]:self.offsets[2 * pair + 1]].tobytes()

    def query(self, pair: int) -> bytes:
        return self.letters[self.offsets[2 * pair + 1]:self.offsets[2 * pair + 2]].tobytes()


def _placement(placement: Optional[Placement]) -> int:
    if placement is None:
        return 0
    if not isinstance(placement, Placement):
        raise TypeError("placement: a Placement")
    return placement.gpu_id


def _raise_first(statuses: np.ndarray, what: str) -> None:
    """Raises the first failing pair's refusal, as a serial loop of single calls would (api.mojo:826-840)."""
    failed = np.flatnonzero(statuses)
    if len(failed) == 0:
        return
    first = int(failed[0])
    code = int(statuses[first])
    if code == native.UNSUPPORTED_SYMBOLS:
        raise ValueError(f"pair {first}: a letter outside the {what}")
    if code == native.INVALID_COSTS:
        raise ValueError(f"pair {first}: scores past 32 bits")
    raise ValueError(f"pair {first}: code {code}")


def scores_tape(tape: Tape, scoring: Scoring, mode: Mode = Mode.GLOBAL, *, placement=None,
                statuses: bool = False):
    """Every pair's best score, global or local, on the GPU: an int32 array (and the per-pair statuses)."""
    handle = native.context(_placement(placement))
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    pairs = tape.pairs
    out = np.empty(max(pairs, 1), dtype=np.int32)
    codes = np.empty(max(pairs, 1), dtype=np.int64)
    code = native.lib().dinara_gpu_scores_tape(handle, pairs, tape.letters.ctypes.data,
                                                native.pointer(tape.offsets, ctypes.c_int64), ctypes.byref(struct),
                                                ctypes.byref(mode_struct), native.pointer(out, ctypes.c_int32),
                                                native.pointer(codes, ctypes.c_int64))
    native.check(code, handle)
    if statuses:
        return out[:pairs], codes[:pairs]
    _raise_first(codes[:pairs], "Scoring's alphabet")
    return out[:pairs]


def scores(references: Sequence[Text], queries: Sequence[Text], scoring: Scoring, mode: Mode = Mode.GLOBAL, *,
           placement: Optional[Placement] = None) -> list:
    """`score` for every pair under `scoring`, globally or locally (api.mojo:843-892)."""
    return [int(value) for value in scores_tape(Tape.of(references, queries), scoring, mode, placement=placement)]


def alignments_tape(tape: Tape, scoring: Scoring, mode: Mode = Mode.GLOBAL, *, eqx: bool = True, placement=None):
    """Every pair's alignment under `scoring` on the GPU, as arrays: (scores, spans[pairs, 4], cigar
    offsets, cigar bytes, statuses)."""
    handle = native.context(_placement(placement))
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    pairs = tape.pairs
    out = np.empty(max(pairs, 1), dtype=np.int32)
    spans = np.empty((max(pairs, 1), 4), dtype=np.int64)
    offsets = np.empty(pairs + 1, dtype=np.int64)
    codes = np.empty(max(pairs, 1), dtype=np.int64)
    buffer = ctypes.c_void_p()
    code = native.lib().dinara_gpu_alignments_tape(handle, pairs, tape.letters.ctypes.data,
                                                    native.pointer(tape.offsets, ctypes.c_int64),
                                                    ctypes.byref(struct), ctypes.byref(mode_struct), 1 if eqx else 0,
                                                    native.pointer(out, ctypes.c_int32),
                                                    native.pointer(spans, ctypes.c_int64),
                                                    native.pointer(offsets, ctypes.c_int64), ctypes.byref(buffer),
                                                    native.pointer(codes, ctypes.c_int64))
    native.check(code, handle)
    total = int(offsets[pairs]) if pairs else 0
    return out[:pairs], spans[:pairs], offsets, _owned_bytes(buffer.value, total), codes[:pairs]


def _owned_bytes(address: Optional[int], size: int) -> np.ndarray:
    """The library's CIGAR buffer as a uint8 array without a copy, freed (dinara_free) once the array and
    every view of it are gone."""
    if not address:
        return np.zeros(0, dtype=np.uint8)
    if size == 0:
        native.lib().dinara_free(address)
        return np.zeros(0, dtype=np.uint8)
    array = np.ctypeslib.as_array((ctypes.c_uint8 * size).from_address(address))
    weakref.finalize(array, native.lib().dinara_free, address)
    return array


def _cost_options(band: Optional[Band], max_cost: Optional[int], eqx: bool, ties: str,
                  max_memory: Optional[int]) -> native.COptions:
    """The options a Costs call takes on the GPU (the reference's `_options`, python/dinara_align/
    __init__.py:415-432): no band, a cap of zero or more, '='/'X' or 'M', ties left or right."""
    if ties not in ("left", "right"):
        raise ValueError("ties: 'left' or 'right'")
    if band is not None and (band.low > -UNBOUNDED or band.high < UNBOUNDED):
        raise ValueError("on the GPU, Costs take no band")
    cap = -1 if max_cost is None else _integers(max_cost)[0]
    if max_memory is not None:
        _integers(max_memory)
    return native.COptions(-(1 << 63), (1 << 63) - 1, cap, 1 if eqx else 0, 1 if ties == "right" else 0,
                           max_memory or 0)


def cost_alignments_tape(tape: Tape, costs: Costs = Costs(), *, max_cost: Optional[int] = None, ties: str = "left",
                         eqx: bool = True, trace: bool = True, placement=None):
    """Every pair's least cost under `costs`, globally, on the GPU, and with `trace` its CIGAR by the Ties
    rule: (costs int64 array, negative entries the pair's code; CIGAR offsets; CIGAR bytes)."""
    handle = native.context(_placement(placement))
    options = _cost_options(None, max_cost, eqx, ties, None)
    costs_struct = costs._struct()
    mode_struct = Mode.GLOBAL._struct()
    pairs = tape.pairs
    out = np.empty(max(pairs, 1), dtype=np.int64)
    offsets = np.zeros(pairs + 1, dtype=np.int64)
    buffer = ctypes.c_void_p()
    code = native.lib().dinara_gpu_cost_alignments_tape(
        handle, pairs, tape.letters.ctypes.data, native.pointer(tape.offsets, ctypes.c_int64),
        ctypes.byref(costs_struct), ctypes.byref(mode_struct), ctypes.byref(options), native.pointer(out, ctypes.c_int64),
        native.pointer(offsets, ctypes.c_int64) if trace else None, ctypes.byref(buffer) if trace else None)
    native.check(code, handle)
    total = int(offsets[pairs]) if (trace and pairs) else 0
    return out[:pairs], offsets, _owned_bytes(buffer.value, total) if trace else np.zeros(0, dtype=np.uint8)


def _check_cost_call(costs: Costs, mode: Mode) -> None:
    if not isinstance(costs, Costs):
        raise TypeError("costs: a Costs or a Scoring")
    if not mode.is_global() or mode.match_score > 0 or mode.kind != _ENDS:
        raise ValueError("on the GPU, Costs align globally")
    if costs.opening2 >= 0 or costs.deletion_opening2 >= 0:
        raise ValueError("on the GPU, Costs of one gap piece")
    if costs.mismatch <= 0:
        raise ValueError("a mismatch that costs nothing")


def _raise_code(pair: int, code: int) -> None:
    if code == native.UNSUPPORTED_SYMBOLS:
        raise ValueError(f"pair {pair}: a 0xFE or 0xFF byte")
    if code == native.OUT_OF_MEMORY:
        raise RuntimeError(f"dinara-align: pair {pair}: its fronts pass the device memory")
    raise ValueError(f"pair {pair}: code {code}")


def alignments(references: Sequence[Text], queries: Sequence[Text], costs: Union[Costs, Scoring] = Costs(),
               mode: Mode = Mode.GLOBAL, *, band: Optional[Band] = None, max_cost: Optional[int] = None,
               ties: str = "left", eqx: bool = True, max_memory: Optional[int] = None, threads: int = 0,
               placement: Optional[Placement] = None) -> list:
    """Every pair's alignment (the reference's `alignments` signature), None past `max_cost`. Under a
    `Costs` the CIGAR is the one `ties` names among equally good alignments (modes.mojo:402-426); under a
    `Scoring`, Gotoh's walk picks, as the reference's device path does (api.mojo:895-1006)."""
    if ties not in ("left", "right"):
        raise ValueError("ties: 'left' or 'right'")
    _integers(threads)
    tape = Tape.of(references, queries)
    if not isinstance(costs, Scoring):
        _check_cost_call(costs, mode)
        _cost_options(band, max_cost, eqx, ties, max_memory)
        if max_cost is not None and max_cost < 0:
            return [None] * tape.pairs
        found, offsets, data = cost_alignments_tape(tape, costs, max_cost=max_cost, ties=ties, eqx=eqx,
                                                    placement=placement)
        out = []
        for pair in range(tape.pairs):
            value = int(found[pair])
            if value == native.ABOVE_MAX:
                out.append(None)
                continue
            if value < 0:
                _raise_code(pair, value)
            cigar = data[offsets[pair]:offsets[pair + 1]].tobytes().decode("ascii")
            rows = int(tape.offsets[2 * pair + 1] - tape.offsets[2 * pair])
            columns = int(tape.offsets[2 * pair + 2] - tape.offsets[2 * pair + 1])
            out.append(Alignment(value, -value, cigar, 0, rows, 0, columns))
        return out
    if band is not None or max_cost is not None:
        raise ValueError("a Scoring takes no band or cap")
    found, spans, offsets, data, codes = alignments_tape(tape, costs, mode, eqx=eqx, placement=placement)
    _raise_first(codes, "Scoring's alphabet")
    out = []
    for pair in range(tape.pairs):
        cigar = data[offsets[pair]:offsets[pair + 1]].tobytes().decode("ascii")
        value = int(found[pair])
        span = spans[pair]
        out.append(Alignment(-value, value, cigar, int(span[0]), int(span[1]), int(span[2]), int(span[3])))
    return out


def distances_tape(tape: Tape, *, policy: int = native.BAND_PLAIN, start_thresholds=None, default_start: int = 0,
                   placement=None, report: bool = False):
    """Every pair's unit-cost global edit distance by band doubling on the GPU (int64 array; negative
    entries are the pair's own code), with the band report when asked."""
    handle = native.context(_placement(placement))
    pairs = tape.pairs
    out = np.empty(max(pairs, 1), dtype=np.int64)
    plan = native.CBandPlan(policy, None, default_start)
    starts = None
    if start_thresholds is not None:
        starts = np.ascontiguousarray(start_thresholds, dtype=np.int64)
        plan.start_thresholds = native.pointer(starts, ctypes.c_int64)
    summary = native.CBandReport()
    code = native.lib().dinara_gpu_distances_tape(handle, pairs, tape.letters.ctypes.data,
                                                   native.pointer(tape.offsets, ctypes.c_int64), ctypes.byref(plan),
                                                   native.pointer(out, ctypes.c_int64), ctypes.byref(summary))
    native.check(code, handle)
    if report:
        return out[:pairs], summary.as_dict()
    return out[:pairs]


def distances(references: Sequence[Text], queries: Sequence[Text], costs: Costs = Costs(), mode: Mode = Mode.GLOBAL,
              *, band: Optional[Band] = None, max_cost: Optional[int] = None, threads: int = 0,
              placement: Optional[Placement] = None) -> list:
    """Every pair's least cost (the reference's `distances` signature), None past `max_cost`, globally on
    the GPU: band doubling at unit costs with no cap (api.mojo:1237-1247), the gap-affine wavefront
    otherwise (api.mojo:622-716)."""
    if mode.match_score > 0:
        raise ValueError("a mode with a match score maximizes a score, which `align` finds")
    _check_cost_call(costs, mode)
    _cost_options(band, max_cost, True, "left", None)
    _integers(threads)
    tape = Tape.of(references, queries)
    scale = costs.unit_scale()
    if scale and max_cost is None:
        found = distances_tape(tape, placement=placement)
        if (found < 0).any():
            _raise_code(int(np.flatnonzero(found < 0)[0]), int(found[found < 0][0]))
        return [int(value) * scale for value in found]
    if max_cost is not None and max_cost < 0:
        return [None] * tape.pairs
    found, _offsets, _data = cost_alignments_tape(tape, costs, max_cost=max_cost, trace=False, placement=placement)
    out = []
    for pair, value in enumerate(found.tolist()):
        if value == native.ABOVE_MAX:
            out.append(None)
        elif value < 0:
            _raise_code(pair, value)
        else:
            out.append(value)
    return out


def distance(reference: Text, query: Text, costs: Costs = Costs(), mode: Mode = Mode.GLOBAL, *, band=None,
             max_cost=None, placement=None) -> Optional[int]:
    return distances([reference], [query], costs, mode, band=band, max_cost=max_cost, placement=placement)[0]


def score(reference: Text, query: Text, costs: Union[Costs, Scoring] = Costs(), mode: Mode = Mode.GLOBAL, *,
          band=None, placement=None) -> int:
    """The score `align` would give: under a `Scoring` its score, under `Costs` minus the least cost."""
    if isinstance(costs, Scoring):
        if band is not None:
            raise ValueError("a Scoring takes no band")
        return scores([reference], [query], costs, mode, placement=placement)[0]
    return -distance(reference, query, costs, mode, band=band, placement=placement)


def align(reference: Text, query: Text, costs: Union[Costs, Scoring] = Costs(), mode: Mode = Mode.GLOBAL, *,
          band=None, max_cost=None, ties: str = "left", eqx=True, max_memory=None,
          placement=None) -> Optional[Alignment]:
    return alignments([reference], [query], costs, mode, band=band, max_cost=max_cost, ties=ties, eqx=eqx,
                      max_memory=max_memory, placement=placement)[0]
