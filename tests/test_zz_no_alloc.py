"""The allocation-free scores entry point (dinara_gpu_scores_static) against the library's own scores.

It serves callers that cannot allocate device memory (code inside another framework's memory pool, or
under a budget that forbids growth): they hand in their own device buffers and the call keeps its
working memory in a fixed device array. Here the test allocates the buffers itself (with torch), packs a
batch in the entry point's documented layout, and checks two calls in a row, global then local, against
dinara_gpu_scores_tape on the same pairs. The file is named to run last."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def test_static_scores_match_library(da):
    import torch

    lib = da._native.lib()
    lib.dinara_gpu_scores_static.restype = ctypes.c_int64
    lib.dinara_gpu_scores_static.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.POINTER(da._native.CScoring), ctypes.POINTER(da._native.CMode),
                                             ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(77)
    refs, queries = [], []
    for rows, columns in [(0, 5), (7, 0), (1, 1), (150, 210), (300, 290), (40, 600), (2000, 1300), (900, 513),
                          (64, 64)] + [(int(rng.integers(1, 400)), int(rng.integers(1, 700))) for _ in range(300)]:
        a = rng.integers(0, 4, size=rows).astype(np.uint32)
        b = a[: min(rows, columns)].copy() if rows else np.zeros(0, np.uint32)
        b = np.concatenate([b, rng.integers(0, 4, size=max(0, columns - len(b))).astype(np.uint32)])[:columns]
        flip = rng.random(len(b)) < 0.05
        b[flip] = rng.integers(0, 4, size=int(flip.sum()))
        refs.append(a)
        queries.append(b)
    words, starts = pack([s for pair in zip(refs, queries) for s in pair])
    shapes = (PackedPair * len(refs))()
    for k in range(len(refs)):
        shapes[k] = PackedPair(starts[2 * k], len(refs[k]), starts[2 * k + 1], len(queries[k]))
    tape_device = torch.from_numpy(words.view(np.int32)).cuda()
    shapes_device = torch.frombuffer(bytearray(bytes(shapes)), dtype=torch.int32).cuda()
    scores_device = torch.zeros(len(refs), dtype=torch.int32, device="cuda")
    ascii_tape = da.Tape.of(["".join("ACGT"[c] for c in a) for a in refs],
                            ["".join("ACGT"[c] for c in b) for b in queries])
    scoring = da.Scoring.uniform(0, -4, -6, -2)
    struct, _table, _alphabet = scoring._struct()
    stream = torch.cuda.current_stream().cuda_stream
    for mode in (da.Mode.GLOBAL, da.Mode.local()):
        mode_struct = mode._struct()
        scores_device.fill_(12345)
        code = lib.dinara_gpu_scores_static(0, len(refs), tape_device.data_ptr(), shapes_device.data_ptr(),
                                            ctypes.byref(struct), ctypes.byref(mode_struct), scores_device.data_ptr(),
                                            stream)
        assert code == 0
        torch.cuda.synchronize()
        expected = da.scores_tape(ascii_tape, scoring, mode)
        np.testing.assert_array_equal(scores_device.cpu().numpy(), expected)
    # A pair past the fixed scratch (wider than 512 columns, more than 8,191 rows) is refused, nothing run.
    big = (PackedPair * 1)(PackedPair(0, 9000, 0, 600))
    big_device = torch.frombuffer(bytearray(bytes(big)), dtype=torch.int32).cuda()
    code = lib.dinara_gpu_scores_static(0, 1, tape_device.data_ptr(), big_device.data_ptr(), ctypes.byref(struct),
                                        ctypes.byref(da.Mode.GLOBAL._struct()), scores_device.data_ptr(), stream)
    assert code == -2
