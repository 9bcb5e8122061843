"""Alignments under Costs on the GPU, against the CPU oracle's restatement of the reference's Ties rule.

The reference's default `alignments(references, queries)` aligns at unit costs and writes, of equally
good alignments, the CIGAR its Ties rule names (modes.mojo:402-426; tests/test_alignment.mojo:2023-2222
pin the rule, tests/test_python.py:71-86 its known answers). Here every cost and CIGAR the GPU gives,
through the Python drop-in and through the reference's own C entry points, must equal the oracle's."""

import ctypes
import json
import os
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _costs(da, fields):
    return da.Costs(*fields)


def test_known_answers(da):
    known = [e for e in json.load(open(os.path.join(GOLDEN, "known_answers.json"))) if e["kind"] == "costs"]
    assert len(known) >= 10
    for entry in known:
        costs = _costs(da, entry["costs"])
        cap = entry.get("max_cost")
        found = da.align(entry["reference"], entry["query"], costs, ties=entry["ties"], eqx=entry["eqx"],
                         max_cost=cap)
        if entry["cost"] is None:
            assert found is None, entry
            assert da.distance(entry["reference"], entry["query"], costs, max_cost=cap) is None
            continue
        assert found.cost == entry["cost"] and found.score == -entry["cost"], entry
        if "cigar" in entry:
            assert found.cigar == entry["cigar"], entry
        assert da.distance(entry["reference"], entry["query"], costs, max_cost=cap) == entry["cost"]
        assert da.score(entry["reference"], entry["query"], costs) == -entry["cost"]


def _repeats(rng, longest=40):
    unit = "".join(rng.choice("ACGT") for _ in range(rng.randint(1, 4)))
    core = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, longest)))
    for _ in range(rng.randint(0, 6)):
        core += unit * rng.randint(1, 3) + "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 20)))
    rate = rng.choice([0.01, 0.03, 0.1, 0.25])
    out = []
    for letter in core:
        roll = rng.random()
        if roll < rate / 3:
            out.append(rng.choice("ACGT"))
        elif roll < 2 * rate / 3:
            continue
        elif roll < rate:
            out.append(letter + rng.choice("ACGT"))
        else:
            out.append(letter)
    return core, "".join(out)


def _expected(oracle, refs, queries, fields, right, eqx, cap=-1):
    x, o, e, _o2, _e2, do, de, _do2, _de2 = fields
    out = []
    for a, b in zip(refs, queries):
        if o == 0 and x == e and de == 0 and cap < 0:
            # Unit costs times x: the edit distance scaled (api.mojo:642-647), the same CIGAR.
            distance, cigar = oracle.edit_cigar(a, b, right=right, eqx=eqx)
            out.append((distance * x, cigar))
        else:
            out.append(oracle.affine_cigar(a, b, x, o, e, do if de else None, de if de else None, max_cost=cap,
                                           right=right, eqx=eqx))
    return out


COSTS = [[1, 0, 1, -1, 0, 0, 0, -1, 0], [4, 6, 2, -1, 0, 0, 0, -1, 0], [3, 1, 4, -1, 0, 0, 0, -1, 0],
         [4, 6, 2, -1, 0, 20, 5, -1, 0], [2, 0, 2, -1, 0, 0, 0, -1, 0], [5, 0, 3, -1, 0, 0, 0, -1, 0]]


@pytest.mark.parametrize("fields", COSTS)
def test_repeat_rich_pairs_follow_the_rule(da, oracle, fields):
    """Pairs built from repeats (ties everywhere) and empty sides, both tie rules, '='/'X' and 'M'."""
    rng = random.Random(101 + sum(fields))
    refs, queries = [], []
    for _ in range(400):
        a, b = _repeats(rng)
        refs.append(a)
        queries.append(b)
    refs += ["", "ACGT", "", "A" * 70]
    queries += ["", "", "GATTACA", "A" * 69 + "C"]
    costs = _costs(da, fields)
    for right in (False, True):
        for eqx in (True, False):
            found = da.alignments(refs, queries, costs, ties="right" if right else "left", eqx=eqx)
            expected = _expected(oracle, refs, queries, fields, right, eqx)
            assert [(a.cost, a.cigar) for a in found] == expected
            assert all((a.reference_end, a.query_end) == (len(r), len(q)) for a, r, q in zip(found, refs, queries))
    assert da.distances(refs, queries, costs) == [cost for cost, _ in _expected(oracle, refs, queries, fields,
                                                                                  False, True)]


@pytest.mark.parametrize("fields", [COSTS[0], COSTS[1]])
def test_read_batch_and_long_pairs(da, oracle, fields):
    """A batch shaped like short reads (100-300 bp, 5% errors), and pairs of 2-6 kbp at up to 12% whose
    fronts outgrow a warp's first arena and run again with larger ones."""
    from dinara_align import workloads

    tape = workloads.affine_global(3000, seed=71)
    refs = [tape.reference(p).decode() for p in range(tape.pairs)]
    queries = [tape.query(p).decode() for p in range(tape.pairs)]
    rng = np.random.default_rng(72)
    long_tape = workloads.pairs_with_errors(rng, rng.integers(2000, 6000, size=6), rng.uniform(0.04, 0.12, size=6),
                                            workloads.HALF_QUARTERS)
    refs += [long_tape.reference(p).decode() for p in range(long_tape.pairs)]
    queries += [long_tape.query(p).decode() for p in range(long_tape.pairs)]
    costs = _costs(da, fields)
    for right in (False, True):
        found = da.alignments(refs, queries, costs, ties="right" if right else "left")
        assert [(a.cost, a.cigar) for a in found] == _expected(oracle, refs, queries, fields, right, True)


def test_caps_and_refusals(da, oracle):
    """A cap leaves the pairs past it None, as the reference does; a 0xFE byte, a band, a second gap piece
    and a mode other than global are refused."""
    rng = random.Random(5)
    refs, queries = [], []
    for _ in range(200):
        a, b = _repeats(rng)
        refs.append(a)
        queries.append(b)
    fields = COSTS[1]
    costs = _costs(da, fields)
    expected = [cost for cost, _ in _expected(oracle, refs, queries, fields, False, True)]
    cap = int(np.median(expected))
    found = da.alignments(refs, queries, costs, max_cost=cap)
    capped = _expected(oracle, refs, queries, fields, False, True, cap=cap)
    for a, (cost, cigar), want in zip(found, capped, expected):
        if want > cap:
            assert a is None and cost == -4
        else:
            assert (a.cost, a.cigar) == (cost, cigar)
    assert da.distances(refs, queries, costs, max_cost=cap) == [c if c <= cap else None for c in expected]
    unit_cap = da.distances(refs, queries, da.Costs(), max_cost=3)
    unit = [oracle.edit_distance_dp(a, b) for a, b in zip(refs, queries)]
    assert unit_cap == [d if d <= 3 else None for d in unit]
    with pytest.raises(ValueError):
        da.alignments([b"AC\xfeT"], ["ACT"], costs)
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACT"], costs, band=da.Band.around(3))
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACT"], da.Costs.two_piece(4, 6, 2, 24, 1))
    with pytest.raises(ValueError):
        da.alignments(["ACGT"], ["ACT"], costs, da.Mode.INFIX)


class CAlignment(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in ("cost", "score", "reference_start", "reference_end",
                                                    "query_start", "query_end")] + [
        ("cigar", ctypes.c_void_p), ("cigar_length", ctypes.c_int64)]


def test_reference_named_c_entry_points(da, oracle):
    """The reference's own C functions (c/dinara.h:141-228) under their names: dinara_alignments,
    dinara_distances, dinara_align, dinara_distance and dinara_score, with its structs and codes."""
    lib = da._native.lib()
    i64, i64p, charpp = ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_char_p)
    costs_p, mode_p = ctypes.POINTER(da._native.CCosts), ctypes.POINTER(da._native.CMode)
    options_p = ctypes.POINTER(da._native.COptions)
    lib.dinara_alignments.restype = i64
    lib.dinara_alignments.argtypes = [i64, charpp, i64p, charpp, i64p, costs_p, mode_p, options_p, i64,
                                      ctypes.POINTER(CAlignment), i64p]
    lib.dinara_distances.restype = i64
    lib.dinara_distances.argtypes = [i64, charpp, i64p, charpp, i64p, costs_p, mode_p, options_p, i64, i64p]
    lib.dinara_distance.restype = i64
    lib.dinara_distance.argtypes = [ctypes.c_char_p, i64, ctypes.c_char_p, i64, costs_p, mode_p, options_p]
    lib.dinara_align.restype = i64
    lib.dinara_align.argtypes = [ctypes.c_char_p, i64, ctypes.c_char_p, i64, costs_p, mode_p, options_p,
                                 ctypes.POINTER(CAlignment)]
    lib.dinara_score.restype = i64
    lib.dinara_score.argtypes = [ctypes.c_char_p, i64, ctypes.c_char_p, i64, costs_p, mode_p, options_p, i64p]
    rng = random.Random(9)
    refs, queries = [], []
    for _ in range(300):
        a, b = _repeats(rng)
        refs.append(a.encode())
        queries.append(b.encode())
    refs.append(b"AC\xffGT")
    queries.append(b"ACGT")
    count = len(refs)
    ref_ptrs = (ctypes.c_char_p * count)(*refs)
    ref_lens = (ctypes.c_int64 * count)(*[len(r) for r in refs])
    q_ptrs = (ctypes.c_char_p * count)(*queries)
    q_lens = (ctypes.c_int64 * count)(*[len(q) for q in queries])
    for fields in (COSTS[0], COSTS[1]):
        costs = da._native.CCosts(*fields)
        for right in (0, 1):
            options = da._native.COptions(-(1 << 63), (1 << 63) - 1, -1, 1, right, 0)
            alignments = (CAlignment * count)()
            statuses = (ctypes.c_int64 * count)()
            assert lib.dinara_alignments(count, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(costs), None,
                                         ctypes.byref(options), 0, alignments, statuses) == 0
            expected = _expected(oracle, [r.decode() for r in refs[:-1]], [q.decode() for q in queries[:-1]], fields,
                                 bool(right), True)
            try:
                for k in range(count - 1):
                    a = alignments[k]
                    assert statuses[k] == 0
                    assert (a.cost, ctypes.string_at(a.cigar, a.cigar_length).decode()) == expected[k]
                    assert a.score == -a.cost and (a.reference_end, a.query_end) == (len(refs[k]), len(queries[k]))
                assert statuses[count - 1] == da._native.UNSUPPORTED_SYMBOLS and not alignments[count - 1].cigar
            finally:
                for k in range(count):
                    if alignments[k].cigar:
                        lib.dinara_free(alignments[k].cigar)
        results = (ctypes.c_int64 * count)()
        assert lib.dinara_distances(count, ref_ptrs, ref_lens, q_ptrs, q_lens, ctypes.byref(costs), None, None, 4,
                                    results) == 0
        assert list(results)[:-1] == [cost for cost, _ in expected]
        assert results[count - 1] == da._native.UNSUPPORTED_SYMBOLS
        a, b = refs[0], queries[0]
        assert lib.dinara_distance(a, len(a), b, len(b), ctypes.byref(costs), None, None) == expected[0][0]
        score = ctypes.c_int64()
        assert lib.dinara_score(a, len(a), b, len(b), ctypes.byref(costs), None, None, ctypes.byref(score)) == 0
        assert score.value == -expected[0][0]
        single = CAlignment()
        assert lib.dinara_align(a, len(a), b, len(b), ctypes.byref(costs), None, None, ctypes.byref(single)) == 0
        try:
            assert ctypes.string_at(single.cigar, single.cigar_length).decode() == \
                _expected(oracle, [a.decode()], [b.decode()], fields, False, True)[0][1]
        finally:
            lib.dinara_free(single.cigar)
    # A band, or a mode other than global, fails the whole batch (the GPU does not take them).
    banded = da._native.COptions(-3, 3, -1, 1, 0, 0)
    assert lib.dinara_distances(count, ref_ptrs, ref_lens, q_ptrs, q_lens, None, None, ctypes.byref(banded), 0,
                                results) == da._native.INVALID_MODE
    local = da.Mode.local(2)._struct()
    assert lib.dinara_distance(refs[0], len(refs[0]), queries[0], len(queries[0]), None, ctypes.byref(local),
                               None) == da._native.INVALID_MODE
