"""Gotoh scores and CIGARs on the GPU against the CPU oracle, bit for bit (the reference's
tests/test_alignment.mojo:3715-3990 device tests compare scores with the host; here the CIGAR is the
full-matrix walk's, as the reference's device walk gives it)."""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _scoring(da, entry):
    return da.Scoring(entry["alphabet"], tuple(entry["table"]), entry["opening"], entry["extension"])


def _oracle_batch(oracle, da, tape, scoring, local, aligned):
    size = len(scoring.alphabet)
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    codes = np.full(256, 255, dtype=np.uint8)
    for k, letter in enumerate(scoring.alphabet.encode()):
        codes[letter] = k
    coded = codes[tape.letters[: tape.offsets[-1]]] if tape.offsets[-1] else np.zeros(1, np.uint8)
    mode = oracle.LOCAL if local else oracle.GLOBAL
    if aligned:
        return oracle.batch_alignments(coded, tape.offsets, table, size, op, ex, mode, threads=8)
    return oracle.batch_scores(coded, tape.offsets, table, size, op, ex, mode, threads=8)


def test_known_answers(da):
    known = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    for entry in known:
        if entry["kind"] != "score":
            continue
        scoring = _scoring(da, entry["scoring"])
        mode = da.Mode.local() if entry["mode"] == "local" else da.Mode.GLOBAL
        assert da.scores([entry["reference"]], [entry["query"]], scoring, mode) == [entry["score"]], entry
        found = da.alignments([entry["reference"]], [entry["query"]], scoring, mode)[0]
        assert found.score == entry["score"], entry
        if "cigar" in entry:
            assert found.cigar == entry["cigar"], entry
        if "reference_start" in entry:
            assert found.reference_start == entry["reference_start"]
        if "query_end" in entry:
            assert found.query_end == entry["query_end"]
        if "cigar_m" in entry:
            assert da.alignments([entry["reference"]], [entry["query"]], scoring, mode, eqx=False)[0].cigar == entry[
                "cigar_m"]


def test_random_fixtures(da):
    data = json.load(open(os.path.join(GOLDEN, "random_pairs.json")))["pairs"]
    known = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    dna = _scoring(da, known[0]["scoring"])
    config2 = _scoring(da, known[8]["scoring"])
    refs = [entry["reference"] for entry in data]
    queries = [entry["query"] for entry in data]
    for name, scoring in (("dna", dna), ("config2", config2)):
        assert da.scores(refs, queries, scoring) == [entry[name]["global"] for entry in data]
        assert da.scores(refs, queries, scoring, da.Mode.local()) == [entry[name]["local"] for entry in data]
        found = da.alignments(refs, queries, scoring)
        assert [a.cigar for a in found] == [entry[name]["global_cigar"] for entry in data]
        local = da.alignments(refs, queries, scoring, da.Mode.local())
        assert [a.cigar for a in local] == [entry[name]["local_cigar"] for entry in data]
        assert [a.score for a in local] == [entry[name]["local"] for entry in data]


@pytest.mark.parametrize("local", [False, True])
def test_synthetic_scores_and_cigars(da, oracle, local):
    """Config-2-shaped pairs (100-300 bp, 5% errors), scores and CIGARs against the oracle."""
    from dinara_align import workloads

    tape = workloads.affine_global(3000, seed=21)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, scoring, local, True)
    got = da.scores_tape(tape, scoring, mode)
    np.testing.assert_array_equal(got, expected_scores)
    scores, spans, offsets, data, codes = da.alignments_tape(tape, scoring, mode)
    np.testing.assert_array_equal(scores, expected_scores)
    assert not codes.any()
    cigars = [data[offsets[p]:offsets[p + 1]].tobytes().decode() for p in range(tape.pairs)]
    assert cigars == expected_cigars


@pytest.mark.parametrize("local", [False, True])
def test_shapes_and_strips(da, oracle, local):
    """Every shape class and multi-strip pairs: widths 1..1500 columns, tall and flat pairs, empties."""
    rng = np.random.default_rng(8)
    widths = [0, 1, 2, 15, 16, 17, 63, 64, 65, 127, 128, 129, 255, 256, 257, 319, 320, 321, 511, 512, 513, 700, 1025,
              1500]
    refs, queries = [], []
    for w in widths:
        for h in (0, 1, 3, 40, 333, 1200):
            refs.append("".join(rng.choice(list("ACGT"), size=h)))
            queries.append("".join(rng.choice(list("ACGT"), size=w)))
    scoring = da.Scoring.dna()
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    tape = da.Tape.of(refs, queries)
    expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, scoring, local, True)
    assert da.scores(refs, queries, scoring, mode) == list(expected_scores)
    found = da.alignments(refs, queries, scoring, mode)
    assert [a.cigar for a in found] == expected_cigars
    assert [a.score for a in found] == list(expected_scores)


@pytest.mark.parametrize("local", [False, True])
def test_sixteen_bit_limits(da, oracle, local):
    """Whole-matrix scores where only some pairs fit the 16-bit pair sweep: large entries bring its limit
    down to a few hundred columns (locally) or rows and columns (globally), so pairs each side of it, and
    pairs of different shapes sharing a lane group, are scored in one batch."""
    rng = np.random.default_rng(77)
    scoring = da.Scoring.uniform(120, -120, -10, -5) if local else da.Scoring.uniform(60, -60, -20, -3)
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    refs, queries = [], []
    for _ in range(400):
        rows, columns = int(rng.integers(1, 700)), int(rng.integers(1, 700))
        a = rng.choice(list("ACGT"), size=max(rows, columns))
        b = a[:columns].copy()
        flips = rng.random(columns) < 0.05
        b[flips] = rng.choice(list("ACGT"), size=int(flips.sum()))
        refs.append("".join(a[:rows]))
        queries.append("".join(b))
    tape = da.Tape.of(refs, queries)
    expected = _oracle_batch(oracle, da, tape, scoring, local, False)
    np.testing.assert_array_equal(da.scores_tape(tape, scoring, mode), expected)


@pytest.mark.parametrize("local", [False, True])
def test_long_pairs_on_a_whole_block(da, oracle, local):
    """Pairs of at least 4,096 x 2,048 letters, scored on a whole block (strips of 4,096 columns): single
    and multiple strips, columns at and just past a strip's edge, next to shorter pairs."""
    rng = np.random.default_rng(91)
    scoring = da.Scoring.uniform(0, -4, -6, -2) if not local else da.Scoring.dna()
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    shapes = [(4096, 2048), (4095, 3000), (5000, 4096), (5000, 4097), (9000, 8500), (4100, 12000), (6000, 2047),
              (300, 250), (4500, 4480)]
    refs, queries = [], []
    for rows, columns in shapes:
        a = rng.choice(list("ACGT"), size=max(rows, columns))
        b = a[:columns].copy()
        flips = rng.random(columns) < 0.08
        b[flips] = rng.choice(list("ACGT"), size=int(flips.sum()))
        refs.append("".join(a[:rows]))
        queries.append("".join(b))
    tape = da.Tape.of(refs, queries)
    expected = _oracle_batch(oracle, da, tape, scoring, local, False)
    np.testing.assert_array_equal(da.scores_tape(tape, scoring, mode), expected)


def _cigar_score(reference, query, cigar, scoring):
    """The score of the alignment a CIGAR spells under a uniform Scoring (a gap of L letters scores
    opening + L x extension), with the letters it consumes on each side."""
    import re

    alphabet = scoring.alphabet
    table = np.asarray(scoring.table).reshape(len(alphabet), len(alphabet))
    score, r, q = 0, 0, 0
    for count, op in re.findall(r"(\d+)([=XMDI])", cigar):
        count = int(count)
        if op in "=XM":
            for k in range(count):
                score += int(table[alphabet.index(reference[r + k]), alphabet.index(query[q + k])])
            r += count
            q += count
        else:
            score += scoring.opening + count * scoring.extension
            if op == "D":
                r += count
            else:
                q += count
    return score, r, q


@pytest.mark.parametrize("scoring_name", ["config2", "dna", "steep", "wide"])
def test_long_cigars_over_a_proven_band(da, oracle, scoring_name):
    """Global CIGARs of long pairs (4,096 x 2,048 letters and more) recorded strip by strip over the band
    their widening band proved: few and many errors, a long deletion and a long insertion that take the
    path far off the main diagonal, a path that leaves the main diagonal and comes back, next to short
    pairs. Scores and CIGARs equal the whole-matrix oracle's; the recording sweeps well under the whole
    matrices' cells; and a 20 kbp pair's CIGAR spells the oracle's score."""
    import ctypes

    from dinara_align import _native as native, workloads

    rng = np.random.default_rng(83)
    scoring = da.Scoring.uniform(*SCORINGS[scoring_name])
    refs, queries = [], []
    tape = workloads.pairs_with_errors(rng, np.array([4300, 4600, 5000, 4800, 4400, 200, 180]),
                                       np.array([0.01, 0.05, 0.12, 0.3, 0.05, 0.05, 0.1]), workloads.HALF_QUARTERS)
    for p in range(tape.pairs):
        refs.append(tape.reference(p).decode())
        queries.append(tape.query(p).decode())
    a = "".join(rng.choice(list("ACGT"), size=4500))
    def letters(n):
        return "".join(rng.choice(list("ACGT"), size=n))

    refs += [a, a, a, a]
    queries += [a[:2000] + a[2600:],                 # 600 letters deleted
                a[:1500] + letters(700) + a[1500:],  # 700 inserted
                a[:1000] + a[1900:] + letters(900),  # off the main diagonal and back
                a[:2000] + letters(1800) + a[2000:]]  # the first band's ends 1,800 diagonals apart
    batch = da.Tape.of(refs, queries)
    expected_scores, expected_cigars = _oracle_batch(oracle, da, batch, scoring, False, True)
    found = da.alignments(refs, queries, scoring)
    assert [x.score for x in found] == list(expected_scores)
    assert [x.cigar for x in found] == expected_cigars

    # The recording swept the long pairs' bands, not their whole matrices.
    class Timing(ctypes.Structure):
        _fields_ = [("total_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("record_ms", ctypes.c_double),
                    ("launches", ctypes.c_int64), ("cells", ctypes.c_int64), ("class_ms", ctypes.c_double * 8),
                    ("class_launches", ctypes.c_int64 * 8), ("band_cells", ctypes.c_int64),
                    ("whole_cells", ctypes.c_int64)]

    lib = native.lib()
    handle = native.context(0)
    struct, _table, _alphabet = scoring._struct()
    mode = da.Mode.GLOBAL._struct()
    native.check(lib.dinara_gpu_resident_load(handle, batch.pairs, batch.letters.ctypes.data,
                                              native.pointer(batch.offsets, ctypes.c_int64), ctypes.byref(struct)),
                 handle)
    timing = Timing()
    native.check(lib.dinara_gpu_resident_align(handle, ctypes.byref(mode), 1, 1, ctypes.byref(timing)), handle)
    whole = sum(len(r) * len(q) for r, q in zip(refs, queries))
    assert 0 < timing.cells < 0.8 * whole

    # A 20 kbp pair: its CIGAR consumes both sequences and scores what the oracle's two-row sweep gives.
    b = "".join(rng.choice(list("ACGT"), size=20000))
    long_tape = workloads.pairs_with_errors(rng, np.array([20000]), 0.04, workloads.HALF_QUARTERS)
    long_refs = [b, long_tape.reference(0).decode()]
    long_queries = [b[:9000] + b[9400:], long_tape.query(0).decode()]
    got = da.alignments(long_refs, long_queries, scoring)
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    for reference, query, alignment in zip(long_refs, long_queries, got):
        want = oracle.gotoh_score(oracle.codes(reference), oracle.codes(query), table, 4, op, ex)[0]
        assert alignment.score == want
        assert _cigar_score(reference, query, alignment.cigar, scoring) == (want, len(reference), len(query))


def test_local_spans_placed_as_reference(da, oracle):
    """Local spans by as_alignment's rule (scoring.mojo:724-744): the aligned letters' last place."""
    refs = ["GGGGACGTACGTGGGG", "ACGTTTTTACGT" * 3, "TTTTACGTACGTTTTT"]
    queries = ["CCCCACGTTCGTCC", "ACGT", "ACGTACGT"]
    found = da.alignments(refs, queries, da.Scoring.dna(), da.Mode.local())
    for a, ref, query in zip(found, refs, queries):
        top, bottom = a.gapped(ref, query)
        letters_r = top.replace("-", "")
        letters_q = bottom.replace("-", "")
        assert a.reference_start == (ref.rfind(letters_r) if letters_r else 0)
        assert a.query_start == (query.rfind(letters_q) if letters_q else 0)
        assert ref[a.reference_start:a.reference_end] == letters_r
    assert (found[0].cigar, found[0].reference_start) == ("4=1X3=", 4)


def test_tables_beyond_four_letters(da, oracle):
    """A 20-letter table (the shared-memory path) and a table whose shifted entries pass 16 bits."""
    rng = np.random.default_rng(9)
    alphabet = "ACDEFGHIKLMNPQRSTVWY"
    table = tuple(int(v) for v in rng.integers(-6, 8, size=400))
    protein = da.Scoring.tabulated(alphabet, table, -10, -1)
    refs = ["".join(rng.choice(list(alphabet), size=rng.integers(0, 600))) for _ in range(80)]
    queries = ["".join(rng.choice(list(alphabet), size=rng.integers(0, 600))) for _ in range(80)]
    tape = da.Tape.of(refs, queries)
    for local in (False, True):
        mode = da.Mode.local() if local else da.Mode.GLOBAL
        expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, protein, local, True)
        assert da.scores(refs, queries, protein, mode) == list(expected_scores)
        assert [a.cigar for a in da.alignments(refs, queries, protein, mode)] == expected_cigars
    wide = da.Scoring.uniform(5, -3, -100, -20000)
    dna_refs = ["".join(rng.choice(list("ACGT"), size=rng.integers(1, 40))) for _ in range(30)]
    dna_queries = ["".join(rng.choice(list("ACGT"), size=rng.integers(1, 40))) for _ in range(30)]
    tape = da.Tape.of(dna_refs, dna_queries)
    expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, wide, False, True)
    assert da.scores(dna_refs, dna_queries, wide) == list(expected_scores)
    assert [a.cigar for a in da.alignments(dna_refs, dna_queries, wide)] == expected_cigars


def test_refusals(da):
    """What the reference refuses: letters outside the alphabet (per pair), scores past 2^28, bad
    Scorings and modes (the whole batch)."""
    scoring = da.Scoring.dna()
    scores, statuses = da.scores_tape(da.Tape.of(["ACGT", "ACNT", "A"], ["ACGT", "ACGT", "A"]), scoring,
                                      statuses=True)
    assert list(statuses) == [0, -1, 0]
    assert scores[0] == 8 and scores[2] == 2
    with pytest.raises(ValueError):
        da.scores(["ACNT"], ["ACGT"], scoring)
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACGT"], da.Scoring.uniform(2, -4, 3, -2))  # a gap that earns
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACGT"], da.Scoring("AC-T", tuple([1] * 16)))
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACGT"], scoring, da.Mode.extension(2))  # extensions stay on the host
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACGT"], scoring, da.Mode.INFIX.with_match_score(2))
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACGT"], scoring, da.Mode.local(2))
    huge = da.Scoring.uniform(2, -4, -4, -100000)
    _, statuses = da.scores_tape(da.Tape.of(["A" * 3000], ["A" * 3000]), huge, statuses=True)
    assert list(statuses) == [-3]


SCORINGS = {
    "config2": (0, -4, -6, -2),
    "dna": (2, -4, -4, -2),
    # A large step from cell to cell: only short pairs fit the 16-bit pair sweep, the rest take 32 bits.
    "steep": (10, -20, -30, -1),
    # Entries too large for the 16-bit pair sweep at any length: every band pair takes 32 bits.
    "wide": (100, -100, -4, -2),
}


@pytest.mark.parametrize("scoring_name", sorted(SCORINGS))
def test_band_proofs_and_leftovers(da, oracle, scoring_name):
    """Global pairs the proven band serves and pairs it leaves to the whole matrix: error rates from 0 to
    40%, length differences up to and past the band's 63 diagonals, long pairs, pairs each side of the
    16-bit pair sweep's length limit; scores and CIGARs must equal the whole-matrix oracle's either way."""
    from dinara_align import workloads

    rng = np.random.default_rng(41)
    scoring = da.Scoring.uniform(*SCORINGS[scoring_name])
    tapes = []
    for rate in (0.0, 0.02, 0.1, 0.25, 0.4):
        tapes.append(workloads.pairs_with_errors(rng, rng.integers(20, 700, size=120), rate,
                                                 workloads.HALF_QUARTERS))
    refs, queries = [], []
    for tape in tapes:
        for p in range(tape.pairs):
            refs.append(tape.reference(p).decode())
            queries.append(tape.query(p).decode())
    for extra in (30, 31, 32, 60, 62, 63, 64, 65, 90):
        a = "".join(rng.choice(list("ACGT"), size=300))
        refs.append(a)
        queries.append(a[: 300 - extra] if extra % 2 else a + "".join(rng.choice(list("ACGT"), size=extra)))
    a = "".join(rng.choice(list("ACGT"), size=4000))
    refs.append(a)
    queries.append(a[:1000] + a[1100:])
    tape = da.Tape.of(refs, queries)
    expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, scoring, False, True)
    assert da.scores(refs, queries, scoring) == list(expected_scores)
    found = da.alignments(refs, queries, scoring)
    assert [a.score for a in found] == list(expected_scores)
    assert [a.cigar for a in found] == expected_cigars


@pytest.mark.parametrize("local", [False, True])
def test_a_batch_in_units(da, oracle, local):
    """200,000 short pairs run as several units on two streams (letters sent a piece at a time, results
    moved out a unit at a time): scores, CIGARs, spans and statuses are the oracle's, from pageable
    letters, from page-locked letters, and from a tape whose offsets start past its first letter."""
    import torch

    from dinara_align import shards, workloads

    rng = np.random.default_rng(31)
    lengths = rng.integers(10, 90, size=200_000)
    tape = workloads.pairs_with_errors(rng, lengths, np.full(len(lengths), 0.05), workloads.HALF_QUARTERS)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    expected_scores, expected_cigars = _oracle_batch(oracle, da, tape, scoring, local, True)
    rows = tape.offsets[1::2] - tape.offsets[0:-1:2]
    columns = tape.offsets[2::2] - tape.offsets[1::2]
    # Spans of a few pairs from batches small enough to run as one unit.
    probes = np.r_[0:500, 99_800:100_300, 199_500:200_000]
    probe_spans = np.concatenate([da.alignments_tape(shards.subset(tape, part), scoring, mode)[1]
                                  for part in (probes[:500], probes[500:1000], probes[1000:])])

    def check(batch):
        np.testing.assert_array_equal(da.scores_tape(batch, scoring, mode), expected_scores)
        scores, spans, offsets, data, codes = da.alignments_tape(batch, scoring, mode)
        np.testing.assert_array_equal(scores, expected_scores)
        assert not codes.any()
        assert offsets[0] == 0 and offsets[-1] == len(data)
        cigars = data.tobytes().decode()
        assert [cigars[offsets[p]:offsets[p + 1]] for p in range(batch.pairs)] == expected_cigars
        if local:
            np.testing.assert_array_equal(spans[probes], probe_spans)
        else:
            np.testing.assert_array_equal(spans, np.stack([np.zeros_like(rows), rows, np.zeros_like(rows), columns], 1))

    check(tape)
    shift = 7
    pinned = torch.empty(len(tape.letters) + shift, dtype=torch.uint8, pin_memory=True).numpy()
    pinned[:shift] = ord("A")
    pinned[shift:] = tape.letters
    check(da.Tape(pinned, tape.offsets + shift))

    # A letter outside the alphabet in pairs of three different units flags those pairs alone.
    flagged = [5, 100_000, 199_999]
    letters = tape.letters.copy()
    for pair in flagged:
        letters[tape.offsets[2 * pair + 1]] = ord("N")
    marked = da.Tape(letters, tape.offsets)
    _, statuses = da.scores_tape(marked, scoring, mode, statuses=True)
    assert np.flatnonzero(statuses).tolist() == flagged
    codes = da.alignments_tape(marked, scoring, mode)[4]
    assert np.flatnonzero(codes).tolist() == flagged


def test_resident_batch_kept_across_other_calls(da):
    """A resident batch (letters packed once and kept on the device) keeps its letters and its results while
    the same context aligns other batches, large ones run in units included."""
    import ctypes

    from dinara_align import _native as native, workloads

    lib = native.lib()
    handle = native.context(0)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    struct, _table, _alphabet = scoring._struct()
    mode = da.Mode.GLOBAL._struct()
    kept = workloads.affine_global(3000, seed=61)
    expected = da.scores_tape(kept, scoring)
    other = workloads.affine_global(80_000, seed=62)

    native.check(lib.dinara_gpu_resident_load(handle, kept.pairs, kept.letters.ctypes.data,
                                              native.pointer(kept.offsets, ctypes.c_int64), ctypes.byref(struct)),
                 handle)
    got = np.zeros(kept.pairs, dtype=np.int32)
    for cigars in (1, 0):
        native.check(lib.dinara_gpu_resident_align(handle, ctypes.byref(mode), cigars, 1, None), handle)
        da.alignments_tape(other, scoring)  # between the run and its fetch
        got[:] = 0
        native.check(lib.dinara_gpu_resident_fetch(handle, native.pointer(got, ctypes.c_int32), None), handle)
        np.testing.assert_array_equal(got, expected)
        da.scores_tape(other, scoring)  # between two runs

    unit = workloads.unit_cost_uniform(2000, seed=63)
    expected_distances = da.distances_tape(unit)
    native.check(lib.dinara_gpu_resident_load(handle, unit.pairs, unit.letters.ctypes.data,
                                              native.pointer(unit.offsets, ctypes.c_int64), None), handle)
    plan = native.CBandPlan(native.BAND_PLAIN, None, 0)
    report = native.CBandReport()
    native.check(lib.dinara_gpu_resident_distances(handle, ctypes.byref(plan), ctypes.byref(report), None), handle)
    da.distances_tape(workloads.unit_cost_uniform(5000, seed=64))
    distances = np.zeros(unit.pairs, dtype=np.int64)
    native.check(lib.dinara_gpu_resident_fetch(handle, None, native.pointer(distances, ctypes.c_int64)), handle)
    np.testing.assert_array_equal(distances, expected_distances)
