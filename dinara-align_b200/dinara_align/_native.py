"""The B200 library (libdinara_gpu.so, built from dinara-align_b200/csrc) through ctypes.

Loading fails loudly: there is no CPU fallback for the GPU path, so a missing or unloadable library
raises `ImportError` at the first call that needs it.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libdinara_gpu.so")

# The C ABI's codes (include/dinara_gpu.h; the reference's c/dinara.h:35-49 for -1..-7).
UNSUPPORTED_SYMBOLS = -1
OUT_OF_MEMORY = -2
INVALID_COSTS = -3
ABOVE_MAX = -4
OUTSIDE_BAND = -5
INVALID_MODE = -6
INVALID_LENGTH = -7
DEVICE_FAILURE = -8
DEVICE_TIMEOUT = -9

ENDS_FREE, EXTENSION, LOCAL = 0, 1, 2
BAND_PLAIN, BAND_LEARNED, BAND_GIVEN = 0, 1, 2

i64 = ctypes.c_int64
i64p = ctypes.POINTER(ctypes.c_int64)
i32p = ctypes.POINTER(ctypes.c_int32)
f32p = ctypes.POINTER(ctypes.c_float)


class CScoring(ctypes.Structure):
    _fields_ = [("alphabet", ctypes.c_char_p), ("alphabet_size", i64), ("table", ctypes.POINTER(ctypes.c_int8)),
                ("opening", i64), ("extension", i64)]


class CMode(ctypes.Structure):
    _fields_ = [(name, i64) for name in ("kind", "reference_start", "reference_end", "query_start", "query_end",
                                         "match_score", "anchor", "zdrop", "end_bonus")]


class CCosts(ctypes.Structure):
    _fields_ = [(name, i64) for name in ("mismatch", "opening", "extension", "opening2", "extension2",
                                         "deletion_opening", "deletion_extension", "deletion_opening2",
                                         "deletion_extension2")]


class COptions(ctypes.Structure):
    _fields_ = [(name, i64) for name in ("band_low", "band_high", "max_cost", "eqx", "right_ties", "max_memory")]


class CBandPlan(ctypes.Structure):
    _fields_ = [("policy", i64), ("start_thresholds", i64p), ("default_start", i64)]


class CBandReport(ctypes.Structure):
    _fields_ = [("rounds", i64), ("pair_rounds", i64), ("words_swept", i64), ("full_cells", i64),
                ("first_round_hits", i64), ("overshoot", i64), ("undershoot", i64), ("kernel_ms", ctypes.c_double),
                ("predict_ms", ctypes.c_double), ("round_pairs", i64 * 16), ("round_launches", i64 * 16),
                ("round_ms", ctypes.c_double * 16)]

    def as_dict(self) -> dict:
        """The report as plain numbers, the per-round lists cut at the last round swept."""
        out = {}
        rounds = sum(1 for value in self.round_pairs if value > 0)
        for name, _ in self._fields_:
            value = getattr(self, name)
            out[name] = list(value)[:rounds] if name.startswith("round_") else value
        return out


_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """The loaded library, with every entry point's signature declared."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBRARY):
            raise ImportError(f"the B200 library is not built: {LIBRARY} is missing (run `make -C dinara-align_b200`)")
        handle = ctypes.CDLL(LIBRARY)
        vp = ctypes.c_void_p
        cp = ctypes.c_char_p
        handle.dinara_gpu_new.restype = vp
        handle.dinara_gpu_new.argtypes = [i64]
        handle.dinara_gpu_free.restype = None
        handle.dinara_gpu_free.argtypes = [vp]
        handle.dinara_gpu_last_error.restype = cp
        handle.dinara_gpu_last_error.argtypes = [vp]
        handle.dinara_gpu_device_info.restype = i64
        handle.dinara_gpu_device_info.argtypes = [vp, cp, i64, i64p]
        handle.dinara_free.restype = None
        handle.dinara_free.argtypes = [vp]
        handle.dinara_gpu_scores_tape.restype = i64
        handle.dinara_gpu_scores_tape.argtypes = [vp, i64, vp, i64p, ctypes.POINTER(CScoring), ctypes.POINTER(CMode),
                                                  i32p, i64p]
        handle.dinara_gpu_alignments_tape.restype = i64
        handle.dinara_gpu_alignments_tape.argtypes = [vp, i64, vp, i64p, ctypes.POINTER(CScoring),
                                                      ctypes.POINTER(CMode), i64, i32p, i64p, i64p,
                                                      ctypes.POINTER(ctypes.c_void_p), i64p]
        handle.dinara_gpu_cost_alignments_tape.restype = i64
        handle.dinara_gpu_cost_alignments_tape.argtypes = [vp, i64, vp, i64p, ctypes.POINTER(CCosts),
                                                           ctypes.POINTER(CMode), ctypes.POINTER(COptions), i64p, i64p,
                                                           ctypes.POINTER(ctypes.c_void_p)]
        handle.dinara_gpu_distances_tape.restype = i64
        handle.dinara_gpu_distances_tape.argtypes = [vp, i64, vp, i64p, ctypes.POINTER(CBandPlan), i64p,
                                                     ctypes.POINTER(CBandReport)]
        handle.dinara_gpu_resident_load.restype = i64
        handle.dinara_gpu_resident_load.argtypes = [vp, i64, vp, i64p, ctypes.POINTER(CScoring)]
        handle.dinara_gpu_resident_align.restype = i64
        handle.dinara_gpu_resident_align.argtypes = [vp, ctypes.POINTER(CMode), i64, i64, vp]
        handle.dinara_gpu_resident_distances.restype = i64
        handle.dinara_gpu_resident_distances.argtypes = [vp, ctypes.POINTER(CBandPlan), ctypes.POINTER(CBandReport),
                                                         vp]
        handle.dinara_gpu_resident_fetch.restype = i64
        handle.dinara_gpu_resident_fetch.argtypes = [vp, i32p, i64p]
        _lib = handle
        return _lib


_contexts: dict = {}


def context(device: int = 0) -> int:
    """The process's context on `device`, opened at first use and kept."""
    with _lock:
        found = _contexts.get(device)
    if found:
        return found
    handle = lib().dinara_gpu_new(device)
    if not handle:
        message = lib().dinara_gpu_last_error(None) or b"unknown failure"
        raise RuntimeError(f"dinara-align: cannot open GPU {device}: {message.decode(errors='replace')}")
    with _lock:
        _contexts[device] = handle
    return handle


def error_of(handle: int) -> str:
    message = lib().dinara_gpu_last_error(handle)
    return message.decode(errors="replace") if message else ""


def check(code: int, handle: int) -> None:
    """Raises the batch-wide failure `code` as ValueError (or RuntimeError for a device failure)."""
    if code == 0:
        return
    message = error_of(handle)
    if code in (DEVICE_FAILURE, DEVICE_TIMEOUT, OUT_OF_MEMORY):
        raise RuntimeError(f"dinara-align: {message} (code {code})")
    raise ValueError(message or f"code {code}")


def pointer(array: np.ndarray, ctype):
    return array.ctypes.data_as(ctypes.POINTER(ctype))
