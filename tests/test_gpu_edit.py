"""Unit-cost distances on the GPU by band doubling against the oracle (the reference's
tests/test_alignment.mojo:3715-3760 test_device_edit_distances: 0-1500 bp pairs, other symbols, a long pair,
refusal of what the GPU placement does not serve)."""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _oracle_distances(oracle, tape):
    letters = tape.letters[: tape.offsets[-1]] if tape.offsets[-1] else np.zeros(1, np.uint8)
    return oracle.batch_distances(letters, tape.offsets, start=-1, threads=8)


def test_known_answers(da):
    known = [entry for entry in json.load(open(os.path.join(GOLDEN, "known_answers.json")))
             if entry["kind"] == "distance"]
    refs = [entry["reference"] for entry in known]
    queries = [entry["query"] for entry in known]
    assert da.distances(refs, queries) == [entry["distance"] for entry in known]


def test_random_fixtures(da):
    data = json.load(open(os.path.join(GOLDEN, "random_pairs.json")))["pairs"]
    refs = [entry["reference"] for entry in data]
    queries = [entry["query"] for entry in data]
    assert da.distances(refs, queries) == [entry["distance"] for entry in data]
    assert da.distances(refs, queries, da.Costs.linear(3, 3)) == [3 * entry["distance"] for entry in data]


@pytest.mark.parametrize("start", [0, 1, 16, 256])
def test_word_edges_and_starts(da, oracle, start):
    """Lengths across word edges (tests/test_alignment.mojo:560-586), every start threshold."""
    rng = np.random.default_rng(12)
    lengths = [1, 2, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 1000, 1500]
    refs, queries = [], []
    for n in lengths:
        for rate in (0.0, 0.02, 0.1, 0.4):
            a = rng.choice(list("ACGT"), size=n)
            b = [ch for ch in a if rng.random() > rate / 2]
            b = "".join(b) + "".join(rng.choice(list("ACGT"), size=int(rng.integers(0, 20))))
            refs.append("".join(a))
            queries.append(b)
            refs.append(b)
            queries.append("".join(a))
    tape = da.Tape.of(refs, queries)
    expected = _oracle_distances(oracle, tape)
    given = np.full(tape.pairs, start, dtype=np.int64)
    got = da.distances_tape(tape, policy=da._native.BAND_GIVEN, start_thresholds=given)
    np.testing.assert_array_equal(got, expected)


def test_uneven_batch(da, oracle):
    """A config-4-shaped batch (log-uniform 100 bp - 20 kbp, 0.5-15% errors), plain band doubling."""
    from dinara_align import workloads

    tape = workloads.uneven_unit_cost(600, seed=31)
    expected = _oracle_distances(oracle, tape)
    got, report = da.distances_tape(tape, report=True)
    np.testing.assert_array_equal(got, expected)
    assert report["words_swept"] > 0 and report["pair_rounds"] >= tape.pairs


def test_bytes_and_refusals(da, oracle):
    """Any byte is a letter matching only itself; 0xFE and 0xFF are refused per pair (c/dinara.h:15-17)."""
    refs = [b"kitten\x01\x7f", b"ACGTNNNNACGT", b"", b"AC\xfeGT", b"x" * 700]
    queries = [b"sitting\x7f", b"ACGTACGT", b"ACG", b"ACGT", b"y" + b"x" * 650]
    tape = da.Tape.of(refs, queries)
    got = da.distances_tape(tape)
    assert list(got[:3]) == [3, 4, 3]
    assert got[3] == -1
    assert got[4] == oracle.edit_distance_dp(refs[4], queries[4])
    # Gap-affine costs take the wavefront (tests/test_gpu_costs.py); two gap pieces are not served.
    assert da.distances(["ACGTAC"], ["ACGAC"], da.Costs.affine(4, 6, 2)) == [8]
    with pytest.raises(ValueError):
        da.distances(["ACGT"], ["ACGT"], da.Costs.two_piece(4, 6, 2, 24, 1))
    with pytest.raises(ValueError):
        da.distances(["ACGT"], ["ACGT"], mode=da.Mode.INFIX)
    with pytest.raises(ValueError):
        da.distances(["ACGT"], ["ACGT"], band=da.Band.around(3))


def test_a_large_batch(da, oracle):
    """100,000 pairs: distances are the oracle's from plain and from given first thresholds, from pageable
    and page-locked letters, and from a tape whose offsets start past its first letter; refused pairs far
    apart are refused alone, and the report's tallies cover every pair."""
    import torch

    from dinara_align import workloads

    rng = np.random.default_rng(41)
    lengths = rng.integers(20, 400, size=100_000)
    tape = workloads.pairs_with_errors(rng, lengths, rng.uniform(0.0, 0.15, size=len(lengths)),
                                       workloads.HALF_QUARTERS)
    expected = _oracle_distances(oracle, tape)
    got, report = da.distances_tape(tape, report=True)
    np.testing.assert_array_equal(got, expected)
    rows = tape.offsets[1::2] - tape.offsets[0:-1:2]
    columns = tape.offsets[2::2] - tape.offsets[1::2]
    assert report["full_cells"] == int((rows * columns).sum())
    assert report["pair_rounds"] >= tape.pairs and report["words_swept"] > 0
    given = np.full(tape.pairs, 1, dtype=np.int64)
    np.testing.assert_array_equal(
        da.distances_tape(tape, policy=da._native.BAND_GIVEN, start_thresholds=given), expected)

    shift = 5
    pinned = torch.empty(len(tape.letters) + shift, dtype=torch.uint8, pin_memory=True).numpy()
    pinned[:shift] = ord("C")
    pinned[shift:] = tape.letters
    np.testing.assert_array_equal(da.distances_tape(da.Tape(pinned, tape.offsets + shift)), expected)

    refused = [3, 50_000, 99_999]
    letters = tape.letters.copy()
    for pair in refused:
        letters[tape.offsets[2 * pair]] = 0xFE
    got = da.distances_tape(da.Tape(letters, tape.offsets))
    assert (got[refused] == -1).all()
    keep = np.setdiff1d(np.arange(tape.pairs), refused)
    np.testing.assert_array_equal(got[keep], expected[keep])


def test_autotuned_shapes_change_no_distance(da, oracle):
    """The band autotuner measures every window shape and a chain bound, installs them, and distances
    under the tuned shapes (and under a tuning that sends every band to its slowest shape) still equal
    the oracle's; a tuning read back installs again."""
    from dinara_align import tuning, workloads

    report = tuning.autotune(pairs=3000, length=(100, 6000), probe_length=2048)
    assert len(report["words_per_ms"]) == tuning.SHAPES
    assert all(rate > 0 for rate in report["words_per_ms"].values())
    assert f"{report['chain_words']}/{report['chain_share']:g}/{report['reach']}" in report["chain_ms"]
    tape = workloads.uneven_unit_cost(600, high=8000, seed=31)
    expected = _oracle_distances(oracle, tape)
    np.testing.assert_array_equal(da.distances_tape(tape), expected)
    kept = tuning.tuning()
    assert kept["chain_words"] == report["chain_words"]
    # Inverted costs: the chooser now prefers what the device measured slowest, and chains of one step.
    inverted = {"chain_words": 1, "chain_share": 0.0, "reach": 8, "full_grids": 1 - kept["full_grids"],
                "word_costs": [1.0 / cost for cost in kept["word_costs"]]}
    tuning.install(inverted)
    np.testing.assert_array_equal(da.distances_tape(tape), expected)
    tuning.install(kept)
    assert tuning.tuning() == kept
