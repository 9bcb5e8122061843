"""The learned band predictor from Python: train it on the GPU, keep it as a versioned blob, and run band
doubling from its predictions (no reference counterpart; see include/dinara_gpu.h)."""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import Placement, Tape, _placement
from . import _native as native

PARAMETERS = 20801
INPUTS = 258
VERSION = 3


class TrainOptions(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("pairs", ctypes.c_int64), ("length_low", ctypes.c_double),
                ("length_high", ctypes.c_double), ("rate_low", ctypes.c_double), ("rate_high", ctypes.c_double),
                ("epochs", ctypes.c_int64), ("batch", ctypes.c_int64), ("learning_rate", ctypes.c_double),
                ("coverage", ctypes.c_double), ("slack", ctypes.c_double)]


class TrainReport(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("train_loss", ctypes.c_double), ("validation_loss", ctypes.c_double),
                ("margin", ctypes.c_double), ("slack", ctypes.c_double), ("held_out", ctypes.c_int64),
                ("seconds", ctypes.c_double)]


def _declare(lib):
    if getattr(lib, "_predictor_declared", False):
        return lib
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    f32p, i64p, f64p = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)
    lib.dinara_gpu_predictor_train.restype = i64
    lib.dinara_gpu_predictor_train.argtypes = [vp, ctypes.POINTER(TrainOptions), ctypes.POINTER(TrainReport)]
    lib.dinara_gpu_predictor_set.restype = i64
    lib.dinara_gpu_predictor_set.argtypes = [vp, f32p, ctypes.c_double, ctypes.c_double]
    lib.dinara_gpu_predictor_get.restype = i64
    lib.dinara_gpu_predictor_get.argtypes = [vp, f32p, f64p, f64p]
    lib.dinara_gpu_predictor_margins.restype = i64
    lib.dinara_gpu_predictor_margins.argtypes = [vp, i64, f64p]
    lib.dinara_gpu_predictor_features.restype = i64
    lib.dinara_gpu_predictor_features.argtypes = [vp, i64, vp, i64p, f32p]
    lib.dinara_gpu_predictor_gradients.restype = i64
    lib.dinara_gpu_predictor_gradients.argtypes = [vp, i64, f32p, f32p, f32p, f64p]
    lib.dinara_gpu_predictor_predict.restype = i64
    lib.dinara_gpu_predictor_predict.argtypes = [vp, i64, vp, i64p, f32p, i64p]
    lib._predictor_declared = True
    return lib


class Predictor:
    """The band predictor installed on one GPU's context."""

    def __init__(self, placement: Placement | None = None):
        self.handle = native.context(_placement(placement))
        self.lib = _declare(native.lib())
        self.seed = None

    def train(self, pairs: int = 1_000_000, *, seed: int = 2024, length=(100, 20_000), rate=(0.005, 0.15),
              epochs: int = 4, batch: int = 4096, learning_rate: float = 2e-3, coverage: float = 0.97,
              slack: float = 16.0) -> dict:
        """Trains on `pairs` pairs generated on the GPU from the uneven distribution (lengths log-uniform,
        error rate uniform, 50/25/25), their exact distances measured by plain band doubling."""
        options = TrainOptions(seed, pairs, float(length[0]), float(length[1]), float(rate[0]), float(rate[1]),
                               epochs, batch, learning_rate, coverage, slack)
        report = TrainReport()
        native.check(self.lib.dinara_gpu_predictor_train(self.handle, ctypes.byref(options), ctypes.byref(report)),
                     self.handle)
        self.seed = seed
        return {name: getattr(report, name) for name, _ in TrainReport._fields_}

    def parameters(self) -> tuple:
        """(flat parameters float32, margin, slack)."""
        out = np.zeros(PARAMETERS, dtype=np.float32)
        margin, slack = ctypes.c_double(), ctypes.c_double()
        native.check(self.lib.dinara_gpu_predictor_get(self.handle, native.pointer(out, ctypes.c_float),
                                                       ctypes.byref(margin), ctypes.byref(slack)), self.handle)
        return out, margin.value, slack.value

    def install(self, parameters, margin: float = 1.0, slack: float = 0.0) -> None:
        flat = np.ascontiguousarray(parameters, dtype=np.float32)
        if flat.shape != (PARAMETERS,):
            raise ValueError(f"{flat.size} parameters for {PARAMETERS}")
        native.check(self.lib.dinara_gpu_predictor_set(self.handle, native.pointer(flat, ctypes.c_float), margin,
                                                       slack), self.handle)

    def margins(self, values=None) -> list:
        """The margins by mean length (< 300, < 1,000, < 4,096, longer); installs `values` when given."""
        out = (ctypes.c_double * 4)(*(values if values is not None else (0.0,) * 4))
        native.check(self.lib.dinara_gpu_predictor_margins(self.handle, 0 if values is None else 1, out), self.handle)
        return list(out)

    def save(self, path: str) -> None:
        """A versioned blob: the parameters, the margins and slack, and the training seed."""
        flat, margin, slack = self.parameters()
        meta = json.dumps({"version": VERSION, "seed": self.seed, "margin": margin, "margins": self.margins(),
                           "slack": slack, "features": "squared 4-mer count differences x 32 / mean length, length ratio, summed squared 6-mer count differences / mean length"})
        np.savez(path, parameters=flat, meta=np.frombuffer(meta.encode(), dtype=np.uint8))

    def load(self, path: str) -> None:
        data = np.load(path)
        meta = json.loads(bytes(data["meta"]).decode())
        if meta.get("version") != VERSION:
            raise ValueError(f"predictor blob version {meta.get('version')}, expected {VERSION}")
        self.install(data["parameters"], meta["margin"], meta["slack"])
        self.margins(meta["margins"])
        self.seed = meta.get("seed")

    def features(self, tape: Tape) -> np.ndarray:
        out = np.zeros((max(tape.pairs, 1), INPUTS), dtype=np.float32)
        native.check(self.lib.dinara_gpu_predictor_features(self.handle, tape.pairs, tape.letters.ctypes.data,
                                                            native.pointer(tape.offsets, ctypes.c_int64),
                                                            native.pointer(out, ctypes.c_float)), self.handle)
        return out[:tape.pairs]

    def gradients(self, features: np.ndarray, targets: np.ndarray) -> tuple:
        x = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        out = np.zeros(PARAMETERS, dtype=np.float32)
        loss = ctypes.c_double()
        native.check(self.lib.dinara_gpu_predictor_gradients(self.handle, len(t), native.pointer(x, ctypes.c_float),
                                                             native.pointer(t, ctypes.c_float),
                                                             native.pointer(out, ctypes.c_float), ctypes.byref(loss)),
                     self.handle)
        return out, loss.value

    def predict(self, tape: Tape) -> tuple:
        """(predicted distances, first thresholds)."""
        predicted = np.zeros(max(tape.pairs, 1), dtype=np.float32)
        thresholds = np.zeros(max(tape.pairs, 1), dtype=np.int64)
        native.check(self.lib.dinara_gpu_predictor_predict(self.handle, tape.pairs, tape.letters.ctypes.data,
                                                           native.pointer(tape.offsets, ctypes.c_int64),
                                                           native.pointer(predicted, ctypes.c_float),
                                                           native.pointer(thresholds, ctypes.c_int64)), self.handle)
        return predicted[:tape.pairs], thresholds[:tape.pairs]


def default_blob() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "band_predictor.npz")
