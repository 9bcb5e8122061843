"""The CPU oracle pinned against the reference's own known answers, and its formulations against each
other: the Gotoh walk by exhaustive enumeration on tiny pairs (the reference's
tests/test_alignment.mojo:93-243 strategy), the unit-cost distance by a plain dynamic program, Myers'
bit-vectors and band doubling."""

import itertools
import json
import os
import random

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _scoring(entry):
    table = np.asarray(entry["table"], dtype=np.int8)
    return table, len(entry["alphabet"]), entry["opening"] + entry["extension"], entry["extension"]


def costs_cigar(oracle, a, b, entry):
    """(cost, CIGAR) of a known answer under Costs: the unit-cost trace for unit costs with no cap (the
    reference's edit_cigar), else the wavefront's."""
    x, o, e, _o2, _e2, do, de, _do2, _de2 = entry["costs"]
    right = entry["ties"] == "right"
    cap = entry.get("max_cost", -1)
    if o == 0 and x == e and de == 0 and cap < 0:
        distance, cigar = oracle.edit_cigar(a, b, right=right, eqx=entry["eqx"])
        return distance * x, cigar
    return oracle.affine_cigar(a, b, x, o, e, do if de else None, de if de else None, max_cost=cap, right=right,
                               eqx=entry["eqx"])


def test_known_answers(oracle):
    """Every known answer the reference's tests give for this path (tests/golden/known_answers.json)."""
    known = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    assert len(known) >= 15
    for entry in known:
        a, b = entry["reference"], entry["query"]
        if entry["kind"] == "distance":
            assert oracle.edit_distance_dp(a, b) == entry["distance"], entry
            assert oracle.myers_distance(a, b) == entry["distance"], entry
            assert oracle.band_doubling(a, b, 0)[0] == entry["distance"], entry
            continue
        if entry["kind"] == "costs":
            cost, cigar = costs_cigar(oracle, a, b, entry)
            assert cost == (-4 if entry["cost"] is None else entry["cost"]), entry
            if "cigar" in entry:
                assert cigar == entry["cigar"], entry
            continue
        table, size, op, ex = _scoring(entry["scoring"])
        mode = oracle.LOCAL if entry["mode"] == "local" else oracle.GLOBAL
        ca, cb = oracle.codes(a, entry["scoring"]["alphabet"]), oracle.codes(b, entry["scoring"]["alphabet"])
        score, _, _ = oracle.gotoh_score(ca, cb, table, size, op, ex, mode)
        assert score == entry["score"], entry
        aligned, cigar, top, bottom = oracle.gotoh_align(ca, cb, table, size, op, ex, mode)
        assert aligned == entry["score"], entry
        if "cigar" in entry:
            assert cigar == entry["cigar"], entry
        if "cigar_m" in entry:
            assert oracle.gotoh_align(ca, cb, table, size, op, ex, mode, eqx=False)[1] == entry["cigar_m"]


def _enumerate_best(a, b, table, size, op, ex, local):
    """The best score of every alignment of two tiny sequences, by listing them all."""
    best = None

    def rescore(path):
        total, i, j, run, layer = 0, 0, 0, 0, None
        for move in path:
            if move == "M":
                total += int(table[a[i] * size + b[j]])
                i, j, layer = i + 1, j + 1, None
            else:
                total += ex if layer == move else op
                layer = move
                if move == "D":
                    i += 1
                else:
                    j += 1
        return total

    def walks(i, j):
        if i == len(a) and j == len(b):
            yield []
            return
        if i < len(a) and j < len(b):
            for rest in walks(i + 1, j + 1):
                yield ["M"] + rest
        if i < len(a):
            for rest in walks(i + 1, j):
                yield ["D"] + rest
        if j < len(b):
            for rest in walks(i, j + 1):
                yield ["I"] + rest

    if not local:
        return max(rescore(path) for path in walks(0, 0))
    best = 0
    for i0 in range(len(a) + 1):
        for i1 in range(i0, len(a) + 1):
            for j0 in range(len(b) + 1):
                for j1 in range(j0, len(b) + 1):
                    sub_a, sub_b = a[i0:i1], b[j0:j1]
                    value = _enumerate_best(sub_a, sub_b, table, size, op, ex, False) if (sub_a or sub_b) else 0
                    best = max(best, value)
    return best


def test_gotoh_against_enumeration(oracle):
    """Every pair over a two-letter alphabet with combined length at most five, global and local."""
    table = np.array([3, -2, -2, 3], dtype=np.int8)
    op, ex = oracle.kernel_gaps(-5, -1)
    words = [()]
    for n in range(1, 4):
        words += list(itertools.product((0, 1), repeat=n))
    for a in words:
        for b in words:
            if len(a) + len(b) > 5:
                continue
            for local in (False, True):
                expected = _enumerate_best(list(a), list(b), table, 2, op, ex, local)
                mode = oracle.LOCAL if local else oracle.GLOBAL
                got = oracle.gotoh_score(np.array(a, np.uint8), np.array(b, np.uint8), table, 2, op, ex, mode)[0]
                assert got == expected, (a, b, local)


def _rescore_cigar(cigar, a, b, table, size, op, ex, start_a=0, start_b=0):
    total, i, j = 0, start_a, start_b
    number = ""
    for ch in cigar:
        if ch.isdigit():
            number += ch
            continue
        k = int(number)
        number = ""
        if ch in "=XM":
            for _ in range(k):
                if ch == "=":
                    assert a[i] == b[j]
                if ch == "X":
                    assert a[i] != b[j]
                total += int(table[a[i] * size + b[j]])
                i, j = i + 1, j + 1
        elif ch == "D":
            total += op + (k - 1) * ex
            i += k
        else:
            total += op + (k - 1) * ex
            j += k
    return total, i, j


def test_random_fixtures(oracle):
    """The seeded fixtures: DP distances agree with Myers and band doubling; each fixture CIGAR rebuilds
    its pair and rescores to its score."""
    data = json.load(open(os.path.join(GOLDEN, "random_pairs.json")))["pairs"]
    dna = json.load(open(os.path.join(GOLDEN, "known_answers.json")))[0]["scoring"]
    table, size, op, ex = _scoring(dna)
    for entry in data:
        a, b = entry["reference"], entry["query"]
        assert oracle.myers_distance(a, b) == entry["distance"]
        assert oracle.band_doubling(a, b, 0)[0] == entry["distance"]
        ca, cb = oracle.codes(a), oracle.codes(b)
        score, cigar, _, _ = oracle.gotoh_align(ca, cb, table, size, op, ex)
        assert (score, cigar) == (entry["dna"]["global"], entry["dna"]["global_cigar"])
        total, i, j = _rescore_cigar(cigar, ca, cb, table, size, op, ex)
        assert (total, i, j) == (score, len(a), len(b))


def test_unit_cost_formulations_agree(oracle):
    """Plain DP, full-matrix Myers (device_edit.mojo's step) and band doubling from several starts, over
    lengths across word edges (the reference's 0..513 sweep, tests/test_alignment.mojo:560-586)."""
    rng = random.Random(11)
    lengths = [0, 1, 2, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513]
    for n in lengths:
        for rate in (0.0, 0.05, 0.3):
            a = "".join(rng.choice("ACGT") for _ in range(n))
            b = "".join(ch if rng.random() > rate else rng.choice(["", "A", ch + "C"]) for ch in a)
            if rng.random() < 0.3:
                b += "".join(rng.choice("ACGT") for _ in range(rng.randrange(0, 70)))
            d = oracle.edit_distance_dp(a, b)
            assert oracle.myers_distance(a, b) == d
            for start in (0, 1, 7, 64, 256):
                assert oracle.band_doubling(a, b, start)[0] == d
            for threshold in (0, 3, 40, 300):
                assert oracle.banded_round(a, b, threshold) >= d


def test_bytes_beyond_dna(oracle):
    """Unit costs take any byte as a letter matching only itself (c/dinara.h:15-17)."""
    a, b = b"kitten\x01\x7f", b"sitting\x7f"
    assert oracle.edit_distance_dp(a, b) == oracle.myers_distance(a, b) == oracle.band_doubling(a, b, 0)[0] == 3


def test_score_reach(oracle):
    """ScoreReach (scoring.mojo:218-249) refuses pairs whose scores could pass 2^28."""
    table = oracle.dna_table(2, -4)
    op, ex = oracle.kernel_gaps(-4, -2)
    assert not oracle.score_reach_refuses(table, 4, op, ex, 50_000, 50_000)
    assert oracle.score_reach_refuses(table, 4, op, ex, 20_000_000, 20_000_000)
    assert not oracle.score_reach_refuses(table, 4, op, ex, 40_000_000, 10, oracle.LOCAL)


def test_batches_match_singles(oracle):
    """The threaded batch entry points give each pair's single answer."""
    rng = np.random.default_rng(5)
    firsts = [rng.integers(0, 4, rng.integers(0, 90)).astype(np.uint8) for _ in range(60)]
    seconds = [rng.integers(0, 4, rng.integers(0, 90)).astype(np.uint8) for _ in range(60)]
    tape, offsets = oracle.tape_of(firsts, seconds)
    table = oracle.dna_table(2, -4)
    op, ex = oracle.kernel_gaps(-4, -2)
    for mode in (oracle.GLOBAL, oracle.LOCAL):
        scores = oracle.batch_scores(tape, offsets, table, 4, op, ex, mode, threads=4)
        aligned, cigars = oracle.batch_alignments(tape, offsets, table, 4, op, ex, mode, threads=3)
        for k, (a, b) in enumerate(zip(firsts, seconds)):
            single = oracle.gotoh_align(a, b, table, 4, op, ex, mode)
            assert scores[k] == single[0] == aligned[k]
            assert cigars[k] == single[1]
    distances = oracle.batch_distances(tape, offsets, start=0, threads=4)
    for k, (a, b) in enumerate(zip(firsts, seconds)):
        assert distances[k] == oracle.edit_distance_dp(a, b)


def test_mlp_oracle_gradients_by_finite_differences():
    """The predictor's CPU oracle: its analytic gradients against central differences."""
    import mlp_oracle

    rng = np.random.default_rng(2)
    flat = rng.normal(0, 0.2, size=mlp_oracle.PARAMETERS)
    x = rng.normal(0, 1, size=(7, 258))
    t = rng.uniform(0, 1, size=7)
    grads, _ = mlp_oracle.gradients(flat, x, t)
    for index in list(rng.integers(0, mlp_oracle.PARAMETERS, size=40)) + [mlp_oracle.PARAMETERS - 1]:
        step = 1e-6
        up, down = flat.copy(), flat.copy()
        up[index] += step
        down[index] -= step
        numeric = (mlp_oracle.gradients(up, x, t)[1] - mlp_oracle.gradients(down, x, t)[1]) / (2 * step)
        assert abs(numeric - grads[index]) <= 1e-5 + 1e-4 * abs(numeric)


def test_mlp_oracle_kmer_features():
    import mlp_oracle

    counts = mlp_oracle.kmer_counts(b"AAAACNAAAA")
    assert counts[0] == 2 and counts.sum() == 3  # AAAA twice, AAAC once; k-mers over N skipped
    f = mlp_oracle.features(b"AAAAA", b"AAAA")
    assert abs(f[0] - 32.0 * (2 - 1) ** 2 / 4.5) < 1e-12 and abs(f[256] - 0.8) < 1e-12
    # The squares of the differences lose their sign: the pair either way round reads the same.
    g = mlp_oracle.features(b"ACGTTGCAAC", b"ACGTAGCAAC")
    h = mlp_oracle.features(b"ACGTAGCAAC", b"ACGTTGCAAC")
    assert np.array_equal(g, h) and abs(g[:256].sum() - 32.0 * 8 / 10) < 1e-12


def _runs(cigar):
    out, length = [], 0
    for letter in cigar:
        if letter.isdigit():
            length = length * 10 + int(letter)
        else:
            out.append((length, letter))
            length = 0
    return out


def priced(cigar, reference, query, x, od, ed, oi, ei):
    """What a CIGAR costs over the pair it spells, checking that it spells it: substitutions x, a run of k
    reference letters alone od + k ed, of query letters oi + k ei (the reference's tests/test_python.py:
    26-46 `rows_cost`)."""
    total, i, j = 0, 0, 0
    for length, op in _runs(cigar):
        if op in "=XM":
            for _ in range(length):
                if op == "=":
                    assert reference[i] == query[j]
                if op == "X":
                    assert reference[i] != query[j]
                total += x if reference[i] != query[j] else 0
                i, j = i + 1, j + 1
        elif op == "D":
            total += od + length * ed
            i += length
        else:
            total += oi + length * ei
            j += length
    assert (i, j) == (len(reference), len(query))
    return total


def least_cost(a, b, x, od, ed, oi, ei):
    """The least gap-affine cost by the plain three-layer dynamic program."""
    big = 1 << 40
    n, m = len(a), len(b)
    H = [[big] * (m + 1) for _ in range(n + 1)]
    D = [[big] * (m + 1) for _ in range(n + 1)]
    I = [[big] * (m + 1) for _ in range(n + 1)]
    H[0][0] = 0
    for i in range(n + 1):
        for j in range(m + 1):
            if i > 0:
                D[i][j] = min(H[i - 1][j] + od + ed, D[i - 1][j] + ed)
            if j > 0:
                I[i][j] = min(H[i][j - 1] + oi + ei, I[i][j - 1] + ei)
            if i > 0 and j > 0:
                H[i][j] = H[i - 1][j - 1] + (0 if a[i - 1] == b[j - 1] else x)
            H[i][j] = min(H[i][j], D[i][j], I[i][j])
    return H[n][m]


def repeats(rng):
    """A pair rich in ties: runs of a short unit between random letters, and a mutated copy (the shape of
    the reference's tests/test_alignment.mojo:2023-2040 tie tests)."""
    unit = "".join(rng.choice("ACGT") for _ in range(rng.randint(1, 4)))
    core = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 30)))
    for _ in range(rng.randint(0, 5)):
        core += unit * rng.randint(1, 3) + "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 10)))
    rate = rng.choice([0.03, 0.1, 0.25])
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


@pytest.mark.parametrize("costs", [(1, 0, 1, 0, 1), (4, 6, 2, 6, 2), (3, 1, 4, 1, 4), (4, 6, 2, 20, 5), (2, 2, 3, 0, 1)])
def test_costs_cigars_are_optimal_and_follow_the_rule(oracle, costs):
    """Under Costs the CIGAR prices at the least cost (a plain DP's) and spells the pair; Ties.LEFT is
    Ties.RIGHT over both sequences reversed, read backwards (tests/test_alignment.mojo:2023-2200)."""
    x, od, ed, oi, ei = costs
    rng = random.Random(17 + sum(costs))
    unit = costs == (1, 0, 1, 0, 1)
    for _ in range(150):
        reference, query = repeats(rng)
        expected = least_cost(reference, query, x, od, ed, oi, ei)
        for right in (False, True):
            cost, cigar = oracle.affine_cigar(reference, query, x, oi, ei, od, ed, right=right)
            assert cost == expected
            assert priced(cigar, reference, query, x, od, ed, oi, ei) == expected
            mirrored = oracle.affine_cigar(reference[::-1], query[::-1], x, oi, ei, od, ed, right=not right)[1]
            assert "".join(f"{n}{op}" for n, op in reversed(_runs(mirrored))) == cigar
            if unit:
                # The unit-cost trace (edit_cigar) and the wavefront's agree, as the reference asserts for
                # a capped search against an uncapped one (tests/test_alignment.mojo:2212-2218).
                assert oracle.edit_cigar(reference, query, right=right) == (cost, cigar)


def test_batch_wavefront_matches_single_pairs(oracle):
    """The threaded wavefront batch (the reference's host path for a uniform Scoring, timed as a CPU
    baseline) gives every pair the single-pair search's cost and Ties.RIGHT CIGAR, and the plain DP's cost."""
    rng = random.Random(23)
    refs, queries = zip(*[repeats(rng) for _ in range(300)])
    tape, offsets = oracle.tape_of([np.frombuffer(r.encode(), np.uint8) for r in refs],
                                   [np.frombuffer(q.encode(), np.uint8) for q in queries])
    costs, cigars = oracle.batch_wavefront(tape, offsets, 4, 6, 2, threads=4)
    for k, (a, b) in enumerate(zip(refs, queries)):
        assert (costs[k], cigars[k]) == oracle.affine_cigar(a, b, 4, 6, 2, right=True)
        assert costs[k] == least_cost(a, b, 4, 6, 2, 6, 2)


def test_free_ends_known_answer(oracle):
    """The reference's literal (tests/test_python.py:103-104): the query placed inside the reference by
    Mode.INFIX under Scoring.dna() scores 16."""
    table = oracle.dna_table(2, -4)
    op, ex = oracle.kernel_gaps(-4, -2)
    unbounded = 1 << 40
    got = oracle.gotoh_score_free(oracle.codes("TTTTACGTACGTTTTT"), oracle.codes("ACGTACGT"), table, 4, op, ex,
                                  reference_start=unbounded, reference_end=unbounded)
    assert got == 16
    # No free letters is the global score.
    assert oracle.gotoh_score_free(oracle.codes("TTTTACGTACGTTTTT"), oracle.codes("ACGTACGT"), table, 4, op, ex) == \
        oracle.gotoh_score(oracle.codes("TTTTACGTACGTTTTT"), oracle.codes("ACGTACGT"), table, 4, op, ex)[0]


def _trimmed_best(oracle, a, b, table, op, ex, rs, re, qs, qe):
    """Free ends by brute force: the best global score over every trim the free letters allow, a start
    trimming one sequence's start (the alignment begins on the first row or the first column) and an end
    one sequence's end."""
    n, m = len(a), len(b)
    best = None
    starts = [(r0, 0) for r0 in range(min(rs, n) + 1)] + [(0, c0) for c0 in range(1, min(qs, m) + 1)]
    ends = [(r1, 0) for r1 in range(min(re, n) + 1)] + [(0, c1) for c1 in range(1, min(qe, m) + 1)]
    for r0, c0 in starts:
        for r1, c1 in ends:
            if r0 + r1 > n or c0 + c1 > m:
                continue
            score = oracle.gotoh_score(a[r0:n - r1], b[c0:m - c1], table, 4, op, ex)[0]
            best = score if best is None else max(best, score)
    return best


def test_free_ends_against_trimmed_global_alignments(oracle):
    """Every preset the reference names (INFIX, PREFIX, SUFFIX, the query's both ends, a few letters at
    each end, an overlap's; tests/test_alignment.mojo:2938-2943) and random counts, on short pairs and
    empty sides, under two tables: the oracle's free-end score is the best global score over the trims
    the free letters allow."""
    rng = np.random.default_rng(71)
    big = 1 << 40
    presets = [(big, big, 0, 0), (0, big, 0, 0), (big, 0, 0, 0), (0, 0, big, big), (8, 8, 3, 3), (0, 40, 40, 0)]
    for match, mismatch, opening, extension in ((2, -4, -4, -2), (1, -3, -5, -1)):
        table = oracle.dna_table(match, mismatch)
        op, ex = oracle.kernel_gaps(opening, extension)
        for trial in range(60):
            n, m = int(rng.integers(0, 14)), int(rng.integers(0, 12))
            a = rng.integers(0, 4, size=n).astype(np.uint8)
            b = a[: m].copy() if trial % 3 else rng.integers(0, 4, size=m).astype(np.uint8)
            b = b[rng.random(len(b)) > 0.1]
            counts = presets[trial % len(presets)] if trial < 36 else tuple(int(x) for x in rng.integers(0, 6, size=4))
            got = oracle.gotoh_score_free(a, b, table, 4, op, ex, *counts)
            assert got == _trimmed_best(oracle, a, b, table, op, ex, *counts), (a, b, counts)


def test_free_end_alignment_known_answer(oracle):
    """The reference's literal (tests/test_python.py:103-104): Mode.INFIX under Scoring.dna() places the
    query at the reference's fifth letter, scoring 16 with the CIGAR 8=."""
    table = oracle.dna_table(2, -4)
    op, ex = oracle.kernel_gaps(-4, -2)
    unbounded = 1 << 40
    score, cigar, span = oracle.free_ends_alignment(oracle.codes("TTTTACGTACGTTTTT"), oracle.codes("ACGTACGT"),
                                                    table, 4, op, ex, unbounded, unbounded, 0, 0)
    assert (score, span[0], cigar) == (16, 4, "8=")
    assert span == (4, 12, 0, 8)


def _placed_by_brute_force(oracle, a, b, table, op, ex, rs, re, qs, qe):
    """The score and span free ends give, by brute force: every allowed start (on the first column within
    `rs` reference letters, or on the first row within `qs` query letters) against every allowed end (on
    the last column within `re` letters of the last row, or on the last row within `qe` of the last
    column), each scored by the global alignment between them. The end is the best, of equal ones the
    furthest along the reference less the query; the start, of those reaching it at that score, the same."""
    n, m = len(a), len(b)
    rs, re, qs, qe = min(rs, n), min(re, n), min(qs, m), min(qe, m)
    starts = [(r, 0) for r in range(rs + 1)] + [(0, c) for c in range(1, qs + 1)]
    ends = [(n - r, m) for r in range(re + 1)] + [(n, m - c) for c in range(1, qe + 1)]

    def between(start, end):
        if start[0] > end[0] or start[1] > end[1]:
            return None
        return oracle.gotoh_score(a[start[0]:end[0]], b[start[1]:end[1]], table, 4, op, ex)[0]

    best, best_end = None, None
    for end in ends:
        values = [v for v in (between(start, end) for start in starts) if v is not None]
        if not values:
            continue
        value = max(values)
        if best is None or value > best or (value == best and end[0] - end[1] > best_end[0] - best_end[1]):
            best, best_end = value, end
    start = max((s for s in starts if between(s, best_end) == best), key=lambda s: s[0] - s[1])
    return best, (start[0], best_end[0], start[1], best_end[1])


def test_free_end_alignments_by_brute_force(oracle):
    """The oracle's free-end alignment against a brute force over every allowed start and end, for the
    presets and random counts of the score test, on short pairs, repeats and empty sides, under two tables:
    the same score and span, and the span's letters aligned globally scoring it."""
    rng = np.random.default_rng(73)
    big = 1 << 40
    presets = [(big, big, 0, 0), (0, big, 0, 0), (big, 0, 0, 0), (0, 0, big, big), (8, 8, 3, 3), (0, 40, 40, 0)]
    for match, mismatch, opening, extension in ((2, -4, -4, -2), (1, -3, -5, -1)):
        table = oracle.dna_table(match, mismatch)
        op, ex = oracle.kernel_gaps(opening, extension)
        for trial in range(60):
            n, m = int(rng.integers(0, 12)), int(rng.integers(0, 10))
            if trial % 4 == 3:
                a = np.tile(rng.integers(0, 4, size=2).astype(np.uint8), 6)[:n]  # repeats: many equal ends
            else:
                a = rng.integers(0, 4, size=n).astype(np.uint8)
            b = a[: m].copy() if trial % 3 else rng.integers(0, 4, size=m).astype(np.uint8)
            b = b[rng.random(len(b)) > 0.1]
            counts = presets[trial % len(presets)] if trial < 36 else tuple(int(x) for x in rng.integers(0, 6, size=4))
            score, cigar, span = oracle.free_ends_alignment(a, b, table, 4, op, ex, *counts)
            assert (score, span) == _placed_by_brute_force(oracle, a, b, table, op, ex, *counts), (a, b, counts)
            inner = oracle.gotoh_align(a[span[0]:span[1]], b[span[2]:span[3]], table, 4, op, ex)
            assert (inner[0], inner[1]) == (score, cigar)


def test_extensions_by_brute_force(oracle):
    """An extension's stop against a brute force over every prefix pair, each scored by its global alignment:
    the best above zero, of equal ones the furthest along both together, then along the reference, or the
    origin; from the ends, the same over both sequences reversed. With an end bonus the alignment reaching
    the query's far end wins when its score plus the bonus passes the stop's. The span's letters aligned
    globally score what the extension does."""
    rng = np.random.default_rng(79)
    big = 1 << 40
    for match, mismatch, opening, extension in ((2, -4, -4, -2), (1, -3, -5, -1)):
        table = oracle.dna_table(match, mismatch)
        op, ex = oracle.kernel_gaps(opening, extension)
        for trial in range(50):
            n, m = int(rng.integers(0, 12)), int(rng.integers(0, 12))
            a = rng.integers(0, 4, size=n).astype(np.uint8)
            if trial % 4 == 3:
                a = np.tile(rng.integers(0, 4, size=2).astype(np.uint8), 6)[:n]
            b = a[: m].copy() if trial % 3 else rng.integers(0, 4, size=m).astype(np.uint8)
            b = b[rng.random(len(b)) > 0.1]
            for from_end in (False, True):
                x, y = (a[::-1].copy(), b[::-1].copy()) if from_end else (a, b)
                best, stop = 0, (0, 0)
                for r in range(1, len(x) + 1):
                    for c in range(1, len(y) + 1):
                        value = oracle.gotoh_score(x[:r], y[:c], table, 4, op, ex)[0]
                        if value > 0 and (value > best or (value == best and (r + c > sum(stop) or (
                                r + c == sum(stop) and r > stop[0])))):
                            best, stop = value, (r, c)
                span = (len(x) - stop[0], len(x), len(y) - stop[1], len(y)) if from_end else (0, stop[0], 0, stop[1])
                score, cigar, got = oracle.extension_alignment(a, b, table, 4, op, ex, from_end)
                assert (score, got) == (best, span), (a, b, from_end)
                for bonus in (3, 50, 1 << 61):
                    counts = (big, 0, 0, 0) if from_end else (0, big, 0, 0)
                    reach, reach_cigar, reach_span = oracle.free_ends_alignment(a, b, table, 4, op, ex, *counts)
                    want = (reach, reach_cigar, reach_span) if reach + bonus > best else (best, cigar, span)
                    assert oracle.extension_alignment(a, b, table, 4, op, ex, from_end, bonus) == want


def test_extension_zdrop_by_brute_force(oracle):
    """An extension's Z-drop against a brute force: every prefix pair scored by its global alignment, each
    anti-diagonal's best (of equal ones the furthest along the reference), then the anti-diagonals in order
    as the reference reads them (scored.mojo:272-300): a best above zero at or above the best so far is
    the stop, one below it by more than the Z-drop plus the gap extension a diagonal apart ends the sweep.
    A Z-drop of 2^40 never ends it; with an end bonus a dropped sweep keeps its stop."""
    rng = np.random.default_rng(83)
    big = 1 << 40
    for match, mismatch, opening, extension in ((2, -4, -4, -2), (1, -3, -5, -1)):
        table = oracle.dna_table(match, mismatch)
        op, ex = oracle.kernel_gaps(opening, extension)
        for trial in range(40):
            n, m = int(rng.integers(0, 14)), int(rng.integers(0, 14))
            a = rng.integers(0, 4, size=n).astype(np.uint8)
            keep = int(rng.integers(0, n + 1))
            b = np.concatenate([a[:keep], rng.integers(0, 4, size=max(0, m - keep)).astype(np.uint8)])[:m]
            for zdrop in (0, 3, 7, big):
                most, furthest = {}, {}
                for r in range(1, n + 1):
                    for c in range(1, len(b) + 1):
                        value = oracle.gotoh_score(a[:r], b[:c], table, 4, op, ex)[0]
                        d = r + c
                        if d not in most or value > most[d] or (value == most[d] and r > furthest[d]):
                            most[d], furthest[d] = value, r
                best, best_row, best_d, dropped = 0, 0, 0, False
                for d in range(2, n + len(b) + 1) if n and len(b) else ():
                    if most[d] > 0 and most[d] >= best:
                        best, best_row, best_d = most[d], furthest[d], d
                    elif most[d] < best:
                        if best - most[d] > zdrop + (-ex) * abs((2 * furthest[d] - d) - (2 * best_row - best_d)):
                            dropped = True
                            break
                got = oracle.gotoh_extension_zdrop(a, b, table, 4, op, ex, zdrop)
                assert got == (best, best_row, best_d - best_row, dropped), (a, b, zdrop)
                if zdrop == big:
                    assert got[:3] == oracle.gotoh_extension(a, b, table, 4, op, ex)
                score, _cigar, span = oracle.extension_alignment(a, b, table, 4, op, ex, False, 1 << 61, zdrop=zdrop)
                if dropped:
                    assert (score, span) == (best, (0, best_row, 0, best_d - best_row))
