"""Scores and alignments with free ends on the GPU against the oracle (the reference's host path for a
Scoring's free ends, scored.mojo:69-240 and scoring.mojo:690-813; its GPU refuses them): the reference's
literal, every preset its tests name (tests/test_alignment.mojo:2938-2943) on reads cut from and mutated
off their references, empty sides, pairs wider than one strip, and the refusals that stand."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BIG = 1 << 40


def _expected(oracle, scoring, refs, queries, mode):
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    size = len(scoring.alphabet)
    out = []
    for r, q in zip(refs, queries):
        out.append(oracle.gotoh_score_free(oracle.codes(r, scoring.alphabet), oracle.codes(q, scoring.alphabet), table,
                                           size, op, ex, min(mode.reference_start, BIG), min(mode.reference_end, BIG),
                                           min(mode.query_start, BIG), min(mode.query_end, BIG)))
    return out


def _reads(rng, count, longest):
    """References of 0-`longest` letters; queries cut from them and mutated, a sixth unrelated."""
    refs, queries = [], []
    for trial in range(count):
        n = int(rng.integers(0, longest + 1))
        ref = "".join(rng.choice(list("ACGT"), size=n))
        if trial % 6 == 0:
            query = "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, max(2, longest * 3 // 4)))))
        else:
            start = int(rng.integers(0, n // 4 + 1))
            stop = n - int(rng.integers(0, n // 4 + 1))
            piece = list(ref[start:max(start, stop)])
            rate = (0.0, 0.02, 0.1)[trial % 3]
            query = "".join(ch if rng.random() >= rate else rng.choice(list("ACGT")) for ch in piece
                            if rng.random() >= rate / 3)
        refs.append(ref)
        queries.append(query)
    return refs, queries


def test_reference_literal(da):
    """tests/test_python.py:103-104: the read placed inside its window by Mode.INFIX scores 16, at the
    reference's fifth letter, with the CIGAR 8=."""
    assert da.score("TTTTACGTACGTTTTT", "ACGTACGT", da.Scoring.dna(), da.Mode.INFIX) == 16
    placed = da.align("TTTTACGTACGTTTTT", "ACGTACGT", da.Scoring.dna(), da.Mode.INFIX)
    assert (placed.score, placed.reference_start, placed.cigar) == (16, 4, "8=")
    assert (placed.reference_end, placed.query_start, placed.query_end) == (12, 0, 8)
    assert da.scores(["TTTTACGTACGTTTTT"], ["ACGTACGT"], da.Scoring.dna(), da.Mode.PREFIX) == \
        [da.score("TTTTACGTACGTTTTT", "ACGTACGT", da.Scoring.dna(), da.Mode.PREFIX)]


@pytest.mark.parametrize("mode_name", ["INFIX", "PREFIX", "SUFFIX", "query_both", "few", "overlap"])
def test_presets_against_the_oracle(da, oracle, mode_name):
    modes = {"INFIX": da.Mode.INFIX, "PREFIX": da.Mode.PREFIX, "SUFFIX": da.Mode.SUFFIX,
             "query_both": da.Mode.ends_free(query_start=BIG, query_end=BIG),
             "few": da.Mode.ends_free(reference_start=8, reference_end=8, query_start=3, query_end=3),
             "overlap": da.Mode.ends_free(reference_end=40, query_start=40)}
    mode = modes[mode_name]
    rng = np.random.default_rng(sum(map(ord, mode_name)))
    refs, queries = _reads(rng, 240, 260)
    tabulated = da.Scoring.tabulated("ACGT", [5, -1, -2, -1, -1, 5, -3, -2, -2, -3, 5, -1, -1, -2, -1, 5], -6, -1)
    for scoring in (da.Scoring.dna(), tabulated):
        assert da.scores(refs, queries, scoring, mode) == _expected(oracle, scoring, refs, queries, mode)


def test_long_pairs_and_random_counts(da, oracle):
    """Pairs past one 512-column strip and tall ones, each batch with random free counts."""
    rng = np.random.default_rng(91)
    scoring = da.Scoring.dna()
    for batch in range(4):
        refs, queries = _reads(rng, 60, 2200)
        counts = [int(x) for x in rng.integers(0, 300, size=4)]
        mode = da.Mode.ends_free(*counts)
        assert da.scores(refs, queries, scoring, mode) == _expected(oracle, scoring, refs, queries, mode)


def _expected_alignments(oracle, scoring, refs, queries, mode):
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    size = len(scoring.alphabet)
    counts = [min(mode.reference_start, BIG), min(mode.reference_end, BIG), min(mode.query_start, BIG),
              min(mode.query_end, BIG)]
    return [oracle.free_ends_alignment(oracle.codes(r, scoring.alphabet), oracle.codes(q, scoring.alphabet), table,
                                       size, op, ex, *counts) for r, q in zip(refs, queries)]


@pytest.mark.parametrize("mode_name", ["INFIX", "PREFIX", "SUFFIX", "query_both", "few", "overlap"])
def test_alignments_against_the_oracle(da, oracle, mode_name):
    """Each preset's alignments: the score, the span as the reference places it (the best end furthest
    along the reference less the query, the start found back from it) and the span's global CIGAR, under
    two tables, on reads, unrelated pairs, repeats and empty sides, next to pairs past one strip."""
    modes = {"INFIX": da.Mode.INFIX, "PREFIX": da.Mode.PREFIX, "SUFFIX": da.Mode.SUFFIX,
             "query_both": da.Mode.ends_free(query_start=BIG, query_end=BIG),
             "few": da.Mode.ends_free(reference_start=8, reference_end=8, query_start=3, query_end=3),
             "overlap": da.Mode.ends_free(reference_end=40, query_start=40)}
    mode = modes[mode_name]
    rng = np.random.default_rng(sum(map(ord, mode_name)) + 1)
    refs, queries = _reads(rng, 160, 300)
    refs += ["ACACACACACACACAC", "", "ACGT", "", "AAAAAAAA"]
    queries += ["ACAC", "ACG", "", "", "AAAA"]
    long_refs, long_queries = _reads(rng, 6, 1400)
    refs += long_refs
    queries += long_queries
    tabulated = da.Scoring.tabulated("ACGT", [5, -1, -2, -1, -1, 5, -3, -2, -2, -3, 5, -1, -1, -2, -1, 5], -6, -1)
    for scoring in (da.Scoring.dna(), tabulated):
        found = da.alignments(refs, queries, scoring, mode)
        expected = _expected_alignments(oracle, scoring, refs, queries, mode)
        for k, (alignment, (score, cigar, span)) in enumerate(zip(found, expected)):
            got = (alignment.score, alignment.cigar, (alignment.reference_start, alignment.reference_end,
                                                      alignment.query_start, alignment.query_end))
            assert got == (score, cigar, span), (k, refs[k], queries[k])


def test_free_ends_refused_where_the_gpu_does_not_serve_them(da):
    """Negative counts stay refused, as does a match score of the mode's own beside the table's."""
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACG"], da.Scoring.dna(), da.Mode.ends_free(reference_start=-1))
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACG"], da.Scoring.dna(), da.Mode.ends_free(reference_start=-1))
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACG"], da.Scoring.dna(), da.Mode.INFIX.with_match_score(2))


def _expected_extensions(oracle, scoring, refs, queries, from_end, bonus):
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    size = len(scoring.alphabet)
    return [oracle.extension_alignment(oracle.codes(r, scoring.alphabet), oracle.codes(q, scoring.alphabet), table,
                                       size, op, ex, from_end, bonus) for r, q in zip(refs, queries)]


@pytest.mark.parametrize("anchor", ["start", "end"])
def test_extensions_against_the_oracle(da, oracle, anchor):
    """Extensions from both starts and from both ends (a seed's extension, scoring.mojo:673-722): with no end
    bonus, a small one and one near 2^62, and a Z-drop too large ever to stop the sweep (the reference's own
    check, tests/test_alignment.mojo:2576-2592), the scores, spans and CIGARs equal the oracle's under two
    tables, on reads sharing their anchor with the reference, unrelated pairs, empty sides and pairs past
    one strip; scores alone agree with the alignments'."""
    from_end = anchor == "end"
    rng = np.random.default_rng(97 + from_end)
    refs, queries = [], []
    for trial in range(150):
        n = int(rng.integers(0, 400 if trial % 25 else 1500))
        ref = "".join(rng.choice(list("ACGT"), size=n))
        shared = int(rng.integers(0, n + 1))
        piece = ref[n - shared:] if from_end else ref[:shared]
        rate = (0.0, 0.03, 0.1)[trial % 3]
        piece = "".join(ch if rng.random() >= rate else rng.choice(list("ACGT")) for ch in piece
                        if rng.random() >= rate / 3)
        tail = "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, 60))))
        query = "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, 200)))) if trial % 7 == 0 else (
            tail + piece if from_end else piece + tail)
        refs.append(ref)
        queries.append(query)
    refs += ["", "ACGT", ""]
    queries += ["ACG", "", ""]
    anchor_value = da.Anchor.END if from_end else da.Anchor.START
    tabulated = da.Scoring.tabulated("ACGT", [5, -1, -2, -1, -1, 5, -3, -2, -2, -3, 5, -1, -1, -2, -1, 5], -6, -1)
    for scoring in (da.Scoring.dna(), tabulated):
        for bonus in (-1, 12, 1 << 62):
            for zdrop in (-1, 1 << 62):
                mode = da.Mode.extension(0, anchor_value, zdrop=zdrop, end_bonus=bonus)
                found = da.alignments(refs, queries, scoring, mode)
                expected = _expected_extensions(oracle, scoring, refs, queries, from_end, bonus)
                for k, (alignment, (score, cigar, span)) in enumerate(zip(found, expected)):
                    got = (alignment.score, alignment.cigar, (alignment.reference_start, alignment.reference_end,
                                                              alignment.query_start, alignment.query_end))
                    assert got == (score, cigar, span), (k, refs[k], queries[k], bonus, zdrop)
                assert da.scores(refs, queries, scoring, mode) == [score for score, _c, _s in expected]


def test_extension_refusals(da):
    """An extension's match score beside the table's is the reference's own refusal."""
    with pytest.raises(ValueError):
        da.scores(["ACGT"], ["ACG"], da.Scoring.dna(), da.Mode.extension(1))
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACG"], da.Scoring.dna(), da.Mode.extension(2, zdrop=5))


def _expected_zdrop(oracle, scoring, refs, queries, from_end, bonus, zdrop):
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    size = len(scoring.alphabet)
    return [oracle.extension_alignment(oracle.codes(r, scoring.alphabet), oracle.codes(q, scoring.alphabet), table,
                                       size, op, ex, from_end, bonus, zdrop=zdrop) for r, q in zip(refs, queries)]


@pytest.mark.parametrize("anchor", ["start", "end"])
def test_extension_zdrops_against_the_oracle(da, oracle, anchor):
    """Extensions with Z-drops small enough to end the sweep (0, 5, 20, 60): each anti-diagonal's best kept on
    the device and read in order, the stop, the span and the CIGAR equal the oracle's, with and without an
    end bonus (a sweep ended early keeps its stop), on reads that share their anchor with the reference and
    then run into unrelated letters, under two tables; scores alone agree."""
    from_end = anchor == "end"
    rng = np.random.default_rng(131 + from_end)
    refs, queries = [], []
    for trial in range(120):
        n = int(rng.integers(0, 300 if trial % 30 else 1200))
        ref = "".join(rng.choice(list("ACGT"), size=n))
        shared = int(rng.integers(0, n + 1))
        piece = ref[n - shared:] if from_end else ref[:shared]
        piece = "".join(ch if rng.random() >= 0.04 else rng.choice(list("ACGT")) for ch in piece)
        tail = "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, 150))))
        refs.append(ref)
        queries.append(tail + piece if from_end else piece + tail)
    refs += ["", "ACGT"]
    queries += ["ACG", ""]
    anchor_value = da.Anchor.END if from_end else da.Anchor.START
    tabulated = da.Scoring.tabulated("ACGT", [5, -1, -2, -1, -1, 5, -3, -2, -2, -3, 5, -1, -1, -2, -1, 5], -6, -1)
    for scoring in (da.Scoring.dna(), tabulated):
        for zdrop in (0, 5, 20, 60):
            for bonus in (-1, 30):
                mode = da.Mode.extension(0, anchor_value, zdrop=zdrop, end_bonus=bonus)
                found = da.alignments(refs, queries, scoring, mode)
                expected = _expected_zdrop(oracle, scoring, refs, queries, from_end, bonus, zdrop)
                for k, (alignment, (score, cigar, span)) in enumerate(zip(found, expected)):
                    got = (alignment.score, alignment.cigar, (alignment.reference_start, alignment.reference_end,
                                                              alignment.query_start, alignment.query_end))
                    assert got == (score, cigar, span), (k, refs[k], queries[k], zdrop, bonus)
                assert da.scores(refs, queries, scoring, mode) == [score for score, _c, _s in expected]


def test_five_letter_alphabet(da, oracle):
    """A table of five letters puts pairs on the 8-bit tape and the shared-memory table: free-end scores and
    alignments (INFIX and a few letters each end) and extensions from both anchors against the oracle."""
    rng = np.random.default_rng(59)
    cells = [[6 if r == c else (-2 if 4 in (r, c) else -4) for c in range(5)] for r in range(5)]
    scoring = da.Scoring.tabulated("ACGTN", [v for row in cells for v in row], -5, -2)
    refs, queries = [], []
    for trial in range(120):
        n = int(rng.integers(0, 300 if trial % 20 else 900))
        ref = "".join(rng.choice(list("ACGTN"), size=n))
        start = int(rng.integers(0, n // 3 + 1))
        piece = ref[start:start + int(rng.integers(0, n - start + 1))]
        query = "".join(ch if rng.random() > 0.05 else rng.choice(list("ACGTN")) for ch in piece)
        if trial % 9 == 0:
            query = "".join(rng.choice(list("ACGTN"), size=int(rng.integers(0, 80))))
        refs.append(ref)
        queries.append(query)
    for mode in (da.Mode.INFIX, da.Mode.ends_free(reference_start=6, reference_end=9, query_start=2, query_end=4)):
        assert da.scores(refs, queries, scoring, mode) == _expected(oracle, scoring, refs, queries, mode)
        found = da.alignments(refs, queries, scoring, mode)
        expected = _expected_alignments(oracle, scoring, refs, queries, mode)
        assert [(a.score, a.cigar, (a.reference_start, a.reference_end, a.query_start, a.query_end))
                for a in found] == [tuple(e) for e in expected]
    for from_end in (False, True):
        mode = da.Mode.extension(0, da.Anchor.END if from_end else da.Anchor.START, end_bonus=9)
        found = da.alignments(refs, queries, scoring, mode)
        expected = _expected_extensions(oracle, scoring, refs, queries, from_end, 9)
        assert [(a.score, a.cigar, (a.reference_start, a.reference_end, a.query_start, a.query_end))
                for a in found] == [tuple(e) for e in expected]
