"""The serving loop: requests submitted together run at once in their slots and each gets the scores it
gets alone; a request past the memory budget is refused, not run; waits are bounded."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_each_result_same_alone_and_in_the_mix(da):
    from dinara_align import serving, workloads

    rng = np.random.default_rng(23)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    requests = []
    for k in range(14):
        count = int(rng.integers(1, 300))
        lengths = np.round(workloads.log_uniform(rng, 50, 3000, count)).astype(np.int64)
        requests.append(workloads.pairs_with_errors(rng, lengths, rng.uniform(0.01, 0.1, size=count),
                                                    workloads.HALF_QUARTERS))
    alone = [da.scores_tape(tape, scoring, da.Mode.local() if k % 3 == 0 else da.Mode.GLOBAL)
             for k, tape in enumerate(requests)]
    with serving.Server(slots=4) as server:
        tickets = [server.submit(tape, scoring, da.Mode.local() if k % 3 == 0 else da.Mode.GLOBAL)
                   for k, tape in enumerate(requests)]
        for ticket, expected in zip(tickets, alone):
            code, scores, statuses, timing = server.wait(ticket)
            assert code == 0
            np.testing.assert_array_equal(scores, expected)
            assert timing["finished"] >= timing["admitted"] >= timing["submitted"]
        stats = server.stats()
        assert stats["completed"] == len(requests) and stats["queued"] == 0
        assert stats["resident_bytes"] <= stats["budget_bytes"]
        # Requests queued together behind busy slots shared device calls.
        assert 1 <= stats["calls"] < len(requests), stats


def test_budget_refusal_and_bounded_wait(da):
    from dinara_align import serving, workloads

    rng = np.random.default_rng(24)
    tape = workloads.pairs_with_errors(rng, np.full(20, 400), 0.05, workloads.HALF_QUARTERS)
    with serving.Server(slots=2, device_bytes=1 << 20) as server:
        code, _, _, _ = server.wait(server.submit(tape, da.Scoring.dna()))
        assert code == da._native.OUT_OF_MEMORY
    with serving.Server(slots=1) as server:
        ticket = server.submit(tape, da.Scoring.dna())
        code, scores, _, _ = server.wait(ticket, timeout=600)
        assert code == 0
        np.testing.assert_array_equal(scores, da.scores_tape(tape, da.Scoring.dna()))


def test_wait_runs_out_then_completes(da):
    """A wait shorter than the request's run gives DINARA_DEVICE_TIMEOUT and leaves the request queued or
    running; a later wait collects the same scores the request gets alone."""
    from dinara_align import serving, workloads

    rng = np.random.default_rng(25)
    tape = workloads.pairs_with_errors(rng, np.full(48, 10_000), 0.05, workloads.HALF_QUARTERS)
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    expected = da.scores_tape(tape, scoring)
    with serving.Server(slots=1) as server:
        ticket = server.submit(tape, scoring)
        code, _, _, _ = server.wait(ticket, timeout=0.001)
        assert code == da._native.DEVICE_TIMEOUT
        code, scores, statuses, _ = server.wait(ticket, timeout=600)
        assert code == 0
        np.testing.assert_array_equal(scores, expected)
        assert (statuses == 0).all()
