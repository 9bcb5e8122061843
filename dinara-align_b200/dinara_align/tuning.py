"""The band autotuner from Python (no reference counterpart; see include/dinara_gpu.h): measure on a GPU
how fast each unit-cost window shape sweeps and which chain bound gives the fastest band doubling, keep
the result, and install it on a context later without measuring again."""

from __future__ import annotations

import ctypes
import json

import numpy as np

from . import Placement, _placement
from . import _native as native

SHAPES = 39


class TuneOptions(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("pairs", ctypes.c_int64), ("length_low", ctypes.c_double),
                ("length_high", ctypes.c_double), ("rate_low", ctypes.c_double), ("rate_high", ctypes.c_double),
                ("probe_length", ctypes.c_int64), ("measure_shapes", ctypes.c_int64)]


class TuneReport(ctypes.Structure):
    _fields_ = [("shapes", ctypes.c_int64), ("words_per_ms", ctypes.c_double * 40),
                ("chain_tried", ctypes.c_int64), ("chain_words_tried", ctypes.c_int64 * 8),
                ("chain_share_tried", ctypes.c_double * 8), ("reach_tried", ctypes.c_int64 * 8),
                ("chain_ms", ctypes.c_double * 8), ("chain_words", ctypes.c_int64), ("chain_share", ctypes.c_double),
                ("reach", ctypes.c_int64), ("full_grids", ctypes.c_int64), ("seconds", ctypes.c_double),
                ("chain_ms_near", ctypes.c_double * 8)]


class Tuning(ctypes.Structure):
    _fields_ = [("chain_words", ctypes.c_int64), ("chain_share", ctypes.c_double), ("reach", ctypes.c_int64),
                ("full_grids", ctypes.c_int64), ("word_costs", ctypes.c_float * 40)]


def _declare(lib):
    if getattr(lib, "_tuning_declared", False):
        return lib
    lib.dinara_gpu_band_autotune.restype = ctypes.c_int64
    lib.dinara_gpu_band_autotune.argtypes = [ctypes.c_void_p, ctypes.POINTER(TuneOptions), ctypes.POINTER(TuneReport)]
    lib.dinara_gpu_band_tuning.restype = ctypes.c_int64
    lib.dinara_gpu_band_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(Tuning)]
    lib._tuning_declared = True
    return lib


def shape_of(index: int) -> tuple:
    """(lanes, words a lane) of window shape `index`."""
    if index < 36:
        return 1 << (index // 6), index % 6 + 1
    return 32, (8, 12, 16)[index - 36]


def autotune(placement: Placement | None = None, *, pairs: int = 50_000, length=(100, 20_000), rate=(0.005, 0.15),
             probe_length: int = 4096, measure_shapes: bool = True, seed: int = 77) -> dict:
    """Measures and installs the band tuning on the placement's context; returns what it measured."""
    lib = _declare(native.lib())
    handle = native.context(_placement(placement))
    options = TuneOptions(seed, pairs, float(length[0]), float(length[1]), float(rate[0]), float(rate[1]),
                          probe_length, 1 if measure_shapes else 0)
    report = TuneReport()
    native.check(lib.dinara_gpu_band_autotune(handle, ctypes.byref(options), ctypes.byref(report)), handle)
    rates = {f"{g}x{k}": report.words_per_ms[s] for s in range(report.shapes) for g, k in [shape_of(s)]}
    # Keyed "floor/share/reach": the device time of plain doubling and of near starts together, and the near
    # starts' part alone (first thresholds near each distance, as a learned start gives them).
    keys = [f"{report.chain_words_tried[c]}/{report.chain_share_tried[c]:g}/{report.reach_tried[c]}"
            for c in range(report.chain_tried)]
    chains = {key: report.chain_ms[c] for c, key in enumerate(keys)}
    near = {key: report.chain_ms_near[c] for c, key in enumerate(keys)}
    return {"words_per_ms": rates, "chain_ms": chains, "chain_ms_near": near, "chain_words": int(report.chain_words),
            "chain_share": report.chain_share, "reach": int(report.reach), "full_grids": int(report.full_grids),
            "seconds": report.seconds}


def tuning_for_starts(report: dict, values: dict, near: bool) -> dict:
    """The tuning `values` (as `tuning()` returns it) with the chain bound an autotune `report` measured
    fastest for near starts (a learned start's rounds) or, without `near`, for plain doubling's."""
    times = {key: (report["chain_ms_near"][key] if near else report["chain_ms"][key] - report["chain_ms_near"][key])
             for key in report["chain_ms"]}
    floor, share, reach = min(times, key=times.get).split("/")
    return dict(values, chain_words=int(floor), chain_share=float(share), reach=int(reach))


def tuning(placement: Placement | None = None) -> dict:
    """The context's current tuning: its chain bound's floor and share, grid scheme and word costs."""
    lib = _declare(native.lib())
    handle = native.context(_placement(placement))
    values = Tuning()
    native.check(lib.dinara_gpu_band_tuning(handle, 0, ctypes.byref(values)), handle)
    return {"chain_words": int(values.chain_words), "chain_share": float(values.chain_share),
            "reach": int(values.reach), "full_grids": int(values.full_grids),
            "word_costs": [float(c) for c in values.word_costs[:SHAPES]]}


def install(values: dict, placement: Placement | None = None) -> None:
    """Installs a tuning that `tuning()` returned (on this or another run)."""
    lib = _declare(native.lib())
    handle = native.context(_placement(placement))
    costs = np.ascontiguousarray(values["word_costs"], dtype=np.float32)
    if costs.shape != (SHAPES,):
        raise ValueError(f"{costs.size} word costs for {SHAPES} shapes")
    given = Tuning()
    given.chain_words = int(values["chain_words"])
    given.chain_share = float(values.get("chain_share", 0.0))
    given.reach = int(values.get("reach", 5))
    given.full_grids = int(values.get("full_grids", 0))
    for s, cost in enumerate(costs):
        given.word_costs[s] = float(cost)
    native.check(lib.dinara_gpu_band_tuning(handle, 1, ctypes.byref(given)), handle)


def save(path: str, placement: Placement | None = None) -> None:
    with open(path, "w") as out:
        json.dump(tuning(placement), out)


def load(path: str, placement: Placement | None = None) -> None:
    with open(path) as source:
        install(json.load(source), placement)
