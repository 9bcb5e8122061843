"""The allocation-free scores entry point (dinara_gpu_scores_static).

It serves callers that cannot allocate device memory (code inside another framework's memory pool, or
under a budget that forbids growth): they hand in their own device buffers and the call keeps its
working memory in a fixed device array. Here the test allocates the buffers itself (with torch), packs a
batch in the entry point's documented layout, and checks two calls in a row, global then local, against
the CPU oracle and against dinara_gpu_scores_tape on the same pairs. It also covers a batch past one
launch (more than 2^20 pairs), and the two refusals: a pair past the fixed array, and a pair whose
scores could pass 2^28. The file is named to run last."""

import ctypes
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


class PackedPair(ctypes.Structure):
    _fields_ = [("first_word", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("second_word", ctypes.c_uint32),
                ("columns", ctypes.c_uint32)]


def pack(sequences):
    """2-bit codes, 16 a word, each sequence from a 16-byte (4-word) boundary: (words, starts)."""
    starts, chunks, at = [], [], 0
    for codes in sequences:
        words = (len(codes) + 15) // 16
        padded = np.zeros(((words + 3) // 4) * 64, dtype=np.uint32)
        padded[: len(codes)] = codes
        packed = (padded.reshape(-1, 16) << (2 * np.arange(16, dtype=np.uint32))).sum(axis=1, dtype=np.uint64)
        starts.append(at)
        chunks.append(packed.astype(np.uint32))
        at += len(packed)
    return np.concatenate(chunks + [np.zeros(4, np.uint32)]), starts


def pack_short(codes, lengths):
    """Sequences of at most 16 letters (`codes` [count, 16], letters past each length ignored), each in
    its own four words, the first holding the letters: the same layout as `pack`, built at once."""
    count = len(lengths)
    masked = np.where(np.arange(16)[None, :] < lengths[:, None], codes, 0).astype(np.uint32)
    words = np.zeros((count + 1) * 4, dtype=np.uint32)
    words[0:4 * count:4] = (masked << (2 * np.arange(16, dtype=np.uint32))).sum(axis=1, dtype=np.uint64)
    return words, 4 * np.arange(count)


def bind(da):
    lib = da._native.lib()
    lib.dinara_gpu_scores_static.restype = ctypes.c_int64
    lib.dinara_gpu_scores_static.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.POINTER(da._native.CScoring), ctypes.POINTER(da._native.CMode),
                                             ctypes.c_void_p, ctypes.c_void_p]
    return lib


def shapes_on_device(starts, rows, columns):
    import torch

    shapes = np.zeros((len(rows), 4), dtype=np.uint32)
    shapes[:, 0] = starts[0::2]
    shapes[:, 1] = rows
    shapes[:, 2] = starts[1::2]
    shapes[:, 3] = columns
    return torch.from_numpy(shapes.view(np.int32).reshape(-1).copy()).cuda()


def oracle_scores(refs, queries, scoring, local, threads=8):
    import oracle

    tape, offsets = oracle.tape_of(refs, queries)
    op, ex = oracle.kernel_gaps(scoring.opening, scoring.extension)
    table = np.asarray(scoring.table, dtype=np.int8)
    return oracle.batch_scores(tape, offsets, table, 4, op, ex, oracle.LOCAL if local else oracle.GLOBAL,
                               threads=threads)


def test_static_scores_match_oracle_and_library(da):
    import torch

    lib = bind(da)
    rng = np.random.default_rng(77)
    refs, queries = [], []
    for rows, columns in [(0, 5), (7, 0), (1, 1), (150, 210), (300, 290), (40, 600), (2000, 1300), (900, 513),
                          (64, 64), (8191, 700)] + [(int(rng.integers(1, 400)), int(rng.integers(1, 700)))
                                                    for _ in range(300)]:
        a = rng.integers(0, 4, size=rows).astype(np.uint32)
        b = a[: min(rows, columns)].copy() if rows else np.zeros(0, np.uint32)
        b = np.concatenate([b, rng.integers(0, 4, size=max(0, columns - len(b))).astype(np.uint32)])[:columns]
        flip = rng.random(len(b)) < 0.05
        b[flip] = rng.integers(0, 4, size=int(flip.sum()))
        refs.append(a)
        queries.append(b)
    words, starts = pack([s for pair in zip(refs, queries) for s in pair])
    tape_device = torch.from_numpy(words.view(np.int32)).cuda()
    shapes_device = shapes_on_device(np.asarray(starts), [len(a) for a in refs], [len(b) for b in queries])
    scores_device = torch.zeros(len(refs), dtype=torch.int32, device="cuda")
    ascii_tape = da.Tape.of(["".join("ACGT"[c] for c in a) for a in refs],
                            ["".join("ACGT"[c] for c in b) for b in queries])
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    struct, _table, _alphabet = scoring._struct()
    stream = torch.cuda.current_stream().cuda_stream
    # Two calls in a row, global then local, each against the oracle and the library's own scores.
    for mode in (da.Mode.GLOBAL, da.Mode.local()):
        mode_struct = mode._struct()
        scores_device.fill_(12345)
        code = lib.dinara_gpu_scores_static(0, len(refs), tape_device.data_ptr(), shapes_device.data_ptr(),
                                            ctypes.byref(struct), ctypes.byref(mode_struct), scores_device.data_ptr(),
                                            stream)
        assert code == 0
        torch.cuda.synchronize()
        found = scores_device.cpu().numpy()
        local = mode is not da.Mode.GLOBAL
        np.testing.assert_array_equal(found, oracle_scores(refs, queries, scoring, local))
        np.testing.assert_array_equal(found, da.scores_tape(ascii_tape, scoring, mode))


def test_static_scores_past_one_launch(da):
    """More than 2^20 pairs go in two launches, each over its own slice of shapes and scores."""
    import torch

    lib = bind(da)
    rng = np.random.default_rng(78)
    count = (1 << 20) + 1500
    rows = rng.integers(0, 17, size=count)
    columns = rng.integers(0, 17, size=count)
    first = rng.integers(0, 4, size=(count, 16), dtype=np.uint8)
    second = first.copy()
    flip = rng.random((count, 16)) < 0.1
    second[flip] = rng.integers(0, 4, size=int(flip.sum()), dtype=np.uint8)
    codes = np.empty((2 * count, 16), dtype=np.uint8)
    codes[0::2], codes[1::2] = first, second
    lengths = np.empty(2 * count, dtype=np.int64)
    lengths[0::2], lengths[1::2] = rows, columns
    words, starts = pack_short(codes, lengths)
    tape_device = torch.from_numpy(words.view(np.int32)).cuda()
    shapes_device = shapes_on_device(starts, rows, columns)
    scores_device = torch.full((count,), 12345, dtype=torch.int32, device="cuda")
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    struct, _table, _alphabet = scoring._struct()
    code = lib.dinara_gpu_scores_static(0, count, tape_device.data_ptr(), shapes_device.data_ptr(),
                                        ctypes.byref(struct), ctypes.byref(da.Mode.GLOBAL._struct()),
                                        scores_device.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    refs = [first[k, : rows[k]] for k in range(count)]
    queries = [second[k, : columns[k]] for k in range(count)]
    np.testing.assert_array_equal(scores_device.cpu().numpy(), oracle_scores(refs, queries, scoring, False))


def test_static_scores_refusals(da):
    """A batch holding a pair past the fixed array (-2), or a pair whose scores could pass 2^28 (-3, as
    ScoreReach refuses it), runs nothing: the scores buffer keeps what it held."""
    import torch

    lib = bind(da)
    stream = torch.cuda.current_stream().cuda_stream
    tape_device = torch.zeros(4096, dtype=torch.int32, device="cuda")
    scores_device = torch.full((2,), 777, dtype=torch.int32, device="cuda")
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    struct, _table, _alphabet = scoring._struct()
    past_array = shapes_on_device(np.array([0, 0, 0, 0]), [10, 9000], [10, 600])
    code = lib.dinara_gpu_scores_static(0, 2, tape_device.data_ptr(), past_array.data_ptr(), ctypes.byref(struct),
                                        ctypes.byref(da.Mode.GLOBAL._struct()), scores_device.data_ptr(), stream)
    assert code == -2
    # Extension -16,000 keeps every shifted entry within 16 bits, but 8,150 + 400 letters reach past 2^28.
    heavy = da.Scoring.uniform(0, -4, -20000, -16000)
    heavy_struct, _table2, _alphabet2 = heavy._struct()
    past_reach = shapes_on_device(np.array([0, 0, 0, 0]), [10, 8150], [10, 400])
    code = lib.dinara_gpu_scores_static(0, 2, tape_device.data_ptr(), past_reach.data_ptr(), ctypes.byref(heavy_struct),
                                        ctypes.byref(da.Mode.GLOBAL._struct()), scores_device.data_ptr(), stream)
    assert code == -3
    torch.cuda.synchronize()
    assert scores_device.cpu().tolist() == [777, 777]
    # The same pair at the library's main entry point: refused by itself, with the same code.
    tape = da.Tape.of(["A" * 8150], ["A" * 400])
    _scores, statuses = da.scores_tape(tape, heavy, da.Mode.GLOBAL, statuses=True)
    assert statuses.tolist() == [-3]
