"""The multi-GPU path's host logic on CPU: the longest-first split and the gather back, run as two gloo
ranks (each rank's alignment stands in through the oracle, as the GPU path is not on this machine)."""

import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_plan_balances_and_covers():
    from dinara_align import shards

    costs = [100, 1, 1, 1, 50, 50, 3, 2]
    owned = shards.plan(costs, 2)
    assert sorted(np.concatenate(owned).tolist()) == list(range(len(costs)))
    loads = [sum(costs[p] for p in part) for part in owned]
    assert max(loads) - min(loads) <= 10  # 100 alone against 50 + 50 + the rest
    assert [len(part) for part in shards.plan([5, 4], 4)] == [1, 1, 0, 0]
    with pytest.raises(ValueError):
        shards.plan(costs, 0)


def test_subset_keeps_each_pair():
    import dinara_align as da
    from dinara_align import shards

    tape = da.Tape.of(["ACGT", "", "GGA"], ["AC", "TTT", ""])
    part = shards.subset(tape, np.array([2, 0]))
    assert [part.reference(0), part.query(0), part.reference(1), part.query(1)] == [b"GGA", b"", b"ACGT", b"AC"]


def _rank(rank, world, port, out_path, kind="distances"):
    sys.path.insert(0, os.path.join(HERE, "..", "dinara-align_b200"))
    sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
    import torch.distributed as dist

    import dinara_align as da
    import oracle
    from dinara_align import shards, workloads

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        if kind == "distances":
            tape = workloads.unit_cost_uniform(40, seed=5)

            def align(part):
                return oracle.batch_distances(part.letters[: part.offsets[-1]], part.offsets, start=256, threads=1)
        else:
            # Two pairs over three ranks: one rank owns nothing, and the others' strings differ in width.
            tape = da.Tape.of(["A" * 3, "C" * 30], ["G", "T" * 12])

            def align(part):
                return np.asarray([(part.reference(k) + part.query(k)).decode() for k in range(part.pairs)])

        found = shards.run(tape, align)
        if rank == 0:
            np.save(out_path, found, allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _spawn_ranks(world, out_path, kind):
    import multiprocessing as mp

    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        port = probe.getsockname()[1]
    context = mp.get_context("spawn")
    ranks = [context.Process(target=_rank, args=(r, world, port, out_path, kind)) for r in range(world)]
    for process in ranks:
        process.start()
    try:
        for process in ranks:
            process.join(timeout=120)
            assert process.exitcode == 0
    finally:
        for process in ranks:
            if process.is_alive():
                process.terminate()


def test_gather_keeps_strings_whole_with_an_empty_rank(tmp_path):
    import dinara_align as da  # noqa: F401  (the package path, set by conftest)

    out_path = str(tmp_path / "strings.npy")
    _spawn_ranks(3, out_path, "strings")
    assert np.load(out_path, allow_pickle=True).tolist() == ["AAAG", "C" * 30 + "T" * 12]


def test_two_gloo_ranks_gather_every_result(tmp_path):
    import multiprocessing as mp

    import dinara_align as da  # noqa: F401  (the package path, set by conftest)
    from dinara_align import workloads

    sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
    import oracle

    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        port = probe.getsockname()[1]
    out_path = str(tmp_path / "found.npy")
    context = mp.get_context("spawn")
    ranks = [context.Process(target=_rank, args=(r, 2, port, out_path)) for r in range(2)]
    for process in ranks:
        process.start()
    try:
        for process in ranks:
            process.join(timeout=120)
            assert process.exitcode == 0
    finally:
        for process in ranks:
            if process.is_alive():
                process.terminate()
    tape = workloads.unit_cost_uniform(40, seed=5)
    expected = oracle.batch_distances(tape.letters[: tape.offsets[-1]], tape.offsets, start=256, threads=1)
    np.testing.assert_array_equal(np.load(out_path), expected)
