"""Parity at the shapes the workloads hold and at the reference-shaped C entry points, against the CPU oracle.

- Local planted queries (150-1,000 letters in 1,000-5,000-letter targets, 8% errors, Scoring.dna()),
  including the longest targets with the widest queries: the 16-bit pair local sweep near its limit.
- Serving-distribution pairs of 12-50 kbp, global gap-affine (4,6,2) scores: the long-pair sweeps.
- The reference's C batch shape (c/dinara.h:209-228): arrays of pointers and lengths, one result and
  one code a pair, CIGARs the caller frees with dinara_free.
(tests/test_alignment.mojo:3715-3990 are the reference's own device-against-host tests.)"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _coded(tape, alphabet="ACGT"):
    codes = np.full(256, 255, dtype=np.uint8)
    for k, letter in enumerate(alphabet.encode()):
        codes[letter] = k
    return codes[tape.letters[: tape.offsets[-1]]] if tape.offsets[-1] else np.zeros(1, np.uint8)


def _oracle(oracle, tape, scoring, local, aligned=False):
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    mode = oracle.LOCAL if local else oracle.GLOBAL
    if aligned:
        return oracle.batch_alignments(_coded(tape), tape.offsets, table, 4, op, ex, mode, threads=16)
    return oracle.batch_scores(_coded(tape), tape.offsets, table, 4, op, ex, mode, threads=16)


def test_local_planted_queries(da, oracle):
    """Config-3-shaped local scores, and the widest queries in the longest targets."""
    from dinara_align import workloads

    scoring = da.Scoring.dna()
    mode = da.Mode.local()
    tape = workloads.local_planted(300, seed=31)
    np.testing.assert_array_equal(da.scores_tape(tape, scoring, mode), _oracle(oracle, tape, scoring, True))
    widest = workloads.local_planted(24, query_range=(950, 1000), target_range=(4900, 5000), seed=32)
    np.testing.assert_array_equal(da.scores_tape(widest, scoring, mode), _oracle(oracle, widest, scoring, True))
    # Local CIGARs and spans on a share of them.
    few = workloads.local_planted(40, seed=33)
    expected_scores, expected_cigars = _oracle(oracle, few, scoring, True, aligned=True)
    scores, _spans, offsets, data, codes = da.alignments_tape(few, scoring, mode)
    np.testing.assert_array_equal(scores, expected_scores)
    assert not codes.any()
    assert [data[offsets[p]:offsets[p + 1]].tobytes().decode() for p in range(few.pairs)] == expected_cigars


@pytest.mark.parametrize("local", [False, True])
def test_serving_lengths(da, oracle, local):
    """Pairs of 12-50 kbp at 1-10% errors (the serving distribution's long end), scored against the oracle."""
    from dinara_align import workloads

    rng = np.random.default_rng(41)
    lengths = np.array([12_000, 20_000, 33_000, 50_000] if not local else [12_500, 30_000])
    tape = workloads.pairs_with_errors(rng, lengths, rng.uniform(0.01, 0.10, size=len(lengths)),
                                       workloads.HALF_QUARTERS)
    scoring = da.Scoring.uniform(0, -4, -6, -2) if not local else da.Scoring.dna()
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    np.testing.assert_array_equal(da.scores_tape(tape, scoring, mode), _oracle(oracle, tape, scoring, local))


class CAlignment(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in ("cost", "score", "reference_start", "reference_end",
                                                    "query_start", "query_end")] + [
        ("cigar", ctypes.c_void_p), ("cigar_length", ctypes.c_int64)]


def _pointer_arrays(texts):
    data = [t.encode() if isinstance(t, str) else t for t in texts]
    return (ctypes.c_char_p * len(data))(*data), (ctypes.c_int64 * len(data))(*[len(t) for t in data])


def _reference_batch(rng, count):
    refs, queries = [], []
    for _ in range(count):
        rows = int(rng.integers(0, 400))
        a = rng.choice(list("ACGT"), size=rows)
        b = a.copy()
        flips = rng.random(rows) < 0.06
        b[flips] = rng.choice(list("ACGT"), size=int(flips.sum()))
        cut = int(rng.integers(0, 5))
        refs.append("".join(a))
        queries.append("".join(b[cut:]) + "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, 6)))))
    refs += ["ACGTN", "", "ACGT"]  # a letter outside the alphabet, an empty side
    queries += ["ACGT", "GATTACA", ""]
    return refs, queries


@pytest.mark.parametrize("local", [False, True])
def test_reference_shaped_scores_and_alignments(da, oracle, local):
    lib = da._native.lib()
    vp, i64, i64p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)
    charpp = ctypes.POINTER(ctypes.c_char_p)
    lib.dinara_gpu_scores.restype = i64
    lib.dinara_gpu_scores.argtypes = [vp, i64, charpp, i64p, charpp, i64p, ctypes.POINTER(da._native.CScoring),
                                      ctypes.POINTER(da._native.CMode), ctypes.POINTER(ctypes.c_int32), i64p]
    lib.dinara_gpu_alignments.restype = i64
    lib.dinara_gpu_alignments.argtypes = [vp, i64, charpp, i64p, charpp, i64p, ctypes.POINTER(da._native.CScoring),
                                          ctypes.POINTER(da._native.CMode), i64, ctypes.POINTER(CAlignment), i64p]
    rng = np.random.default_rng(51 + local)
    refs, queries = _reference_batch(rng, 500)
    count = len(refs)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    mode = da.Mode.local() if local else da.Mode.GLOBAL
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    ref_ptrs, ref_lens = _pointer_arrays(refs)
    q_ptrs, q_lens = _pointer_arrays(queries)
    context = da._native.context(0)
    scores = (ctypes.c_int32 * count)()
    statuses = (ctypes.c_int64 * count)()
    code = lib.dinara_gpu_scores(context, count, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(struct),
                                 ctypes.byref(mode_struct), scores, statuses)
    assert code == 0
    good = list(range(count - 3)) + [count - 2, count - 1]
    assert list(statuses)[count - 3] == da._native.UNSUPPORTED_SYMBOLS
    assert all(statuses[k] == 0 for k in good)
    clean = da.Tape.of([refs[k] for k in good], [queries[k] for k in good])
    expected_scores, expected_cigars = _oracle(oracle, clean, scoring, local, aligned=True)
    assert [scores[k] for k in good] == list(expected_scores)

    alignments = (CAlignment * count)()
    code = lib.dinara_gpu_alignments(context, count, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(struct),
                                     ctypes.byref(mode_struct), 1, alignments, statuses)
    assert code == 0
    assert statuses[count - 3] == da._native.UNSUPPORTED_SYMBOLS and not alignments[count - 3].cigar
    expected_alignments = da.alignments([refs[k] for k in good], [queries[k] for k in good], scoring, mode)
    try:
        for place, k in enumerate(good):
            a = alignments[k]
            cigar = ctypes.string_at(a.cigar, a.cigar_length).decode()
            assert cigar == expected_cigars[place]
            assert a.score == expected_scores[place] and a.cost == -a.score
            e = expected_alignments[place]
            assert (a.reference_start, a.reference_end, a.query_start, a.query_end) == (
                e.reference_start, e.reference_end, e.query_start, e.query_end)
            if not local:
                assert (a.reference_start, a.reference_end, a.query_start, a.query_end) == (
                    0, len(refs[k]), 0, len(queries[k]))
    finally:
        for k in range(count):
            if alignments[k].cigar:
                lib.dinara_free(alignments[k].cigar)


def test_reference_shaped_distances(da, oracle):
    lib = da._native.lib()
    vp, i64, i64p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)
    charpp = ctypes.POINTER(ctypes.c_char_p)
    lib.dinara_gpu_distances.restype = i64
    lib.dinara_gpu_distances.argtypes = [vp, i64, charpp, i64p, charpp, i64p, ctypes.POINTER(da._native.CCosts),
                                         ctypes.POINTER(da._native.CMode), ctypes.POINTER(da._native.COptions), i64p]
    rng = np.random.default_rng(61)
    refs, queries = _reference_batch(rng, 400)
    refs.append(b"AC\xfeGT")  # a byte the unit-cost path refuses (c/dinara.h:15-17)
    queries.append(b"ACGT")
    count = len(refs)
    ref_ptrs, ref_lens = _pointer_arrays(refs)
    q_ptrs, q_lens = _pointer_arrays(queries)
    results = (ctypes.c_int64 * count)()
    context = da._native.context(0)
    code = lib.dinara_gpu_distances(context, count, ref_ptrs, ref_lens, q_ptrs, q_lens, None, None, None, results)
    assert code == 0
    expected = [oracle.edit_distance_dp(r if isinstance(r, bytes) else r.encode(),
                                        q if isinstance(q, bytes) else q.encode()) for r, q in zip(refs, queries)]
    assert list(results)[:-1] == expected[:-1]
    assert results[count - 1] == da._native.UNSUPPORTED_SYMBOLS
    # Unit costs scaled by two (Costs.affine(2, 0, 2)): every distance doubled.
    costs = da._native.CCosts(2, 0, 2, -1, 0, 0, 0, 0, 0)
    options = da._native.COptions(-(1 << 63), (1 << 63) - 1, -1, 1, 0, 0)
    code = lib.dinara_gpu_distances(context, count - 1, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(costs),
                                    ctypes.byref(da.Mode.GLOBAL._struct()), ctypes.byref(options), results)
    assert code == 0
    assert list(results)[: count - 1] == [2 * d for d in expected[:-1]]
    # A banded request is refused for the whole batch, as the reference's GPU placement refuses it.
    banded = da._native.COptions(-10, 10, -1, 1, 0, 0)
    assert lib.dinara_gpu_distances(context, count - 1, ref_ptrs, ref_lens, q_ptrs, q_lens, None, None,
                                    ctypes.byref(banded), results) == da._native.INVALID_MODE


@pytest.mark.parametrize("kind", ["infix", "extension"])
def test_reference_shaped_free_ends_and_extensions(da, oracle, kind):
    """The pointer-array entry point (the reference's batch shape) with free ends and with an extension (from
    the ends, a Z-drop and an end bonus): each alignment's score, span and CIGAR as the oracle places and
    aligns it, a pair with a letter outside the alphabet refused alone, the CIGARs freed by dinara_free."""
    lib = da._native.lib()
    vp, i64, i64p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)
    charpp = ctypes.POINTER(ctypes.c_char_p)
    lib.dinara_gpu_alignments.restype = i64
    lib.dinara_gpu_alignments.argtypes = [vp, i64, charpp, i64p, charpp, i64p, ctypes.POINTER(da._native.CScoring),
                                          ctypes.POINTER(da._native.CMode), i64, ctypes.POINTER(CAlignment), i64p]
    rng = np.random.default_rng(61 + (kind == "extension"))
    refs, queries = _reference_batch(rng, 300)
    count = len(refs)
    scoring = da.Scoring.dna()
    mode = da.Mode.INFIX if kind == "infix" else da.Mode.extension(0, da.Anchor.END, zdrop=10, end_bonus=5)
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    ref_ptrs, ref_lens = _pointer_arrays(refs)
    q_ptrs, q_lens = _pointer_arrays(queries)
    context = da._native.context(0)
    statuses = (ctypes.c_int64 * count)()
    alignments = (CAlignment * count)()
    code = lib.dinara_gpu_alignments(context, count, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(struct),
                                     ctypes.byref(mode_struct), 1, alignments, statuses)
    assert code == 0
    refused = count - 3
    assert statuses[refused] == da._native.UNSUPPORTED_SYMBOLS and not alignments[refused].cigar
    table = np.asarray(scoring.table, dtype=np.int8)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    big = 1 << 40
    try:
        for k in range(count):
            if k == refused:
                continue
            assert statuses[k] == 0
            a, b = oracle.codes(refs[k]), oracle.codes(queries[k])
            if kind == "infix":
                want = oracle.free_ends_alignment(a, b, table, 4, op, ex, big, big, 0, 0)
            else:
                want = oracle.extension_alignment(a, b, table, 4, op, ex, True, 5, zdrop=10)
            got = alignments[k]
            cigar = ctypes.string_at(got.cigar, got.cigar_length).decode() if got.cigar_length else ""
            assert (got.score, cigar, (got.reference_start, got.reference_end, got.query_start, got.query_end)) == (
                want[0], want[1], want[2]), k
            assert got.cost == -got.score
    finally:
        for k in range(count):
            if alignments[k].cigar:
                lib.dinara_free(alignments[k].cigar)
