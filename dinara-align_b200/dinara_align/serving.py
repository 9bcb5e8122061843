"""The serving loop from Python (include/dinara_gpu.h, dinara_server_*): submit batches of pairs at any time,
collect their scores, and drive an open-loop load of Poisson arrivals for latency and throughput."""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import Mode, Placement, Scoring, Tape, _placement
from . import _native as native


class ServerOptions(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int64), ("device_bytes", ctypes.c_int64)]


class RequestTiming(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_double), ("admitted", ctypes.c_double), ("finished", ctypes.c_double),
                ("pairs", ctypes.c_int64), ("device_bytes", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in ("queued", "running", "admitted", "completed", "refused",
                                                    "pairs_done", "resident_bytes", "budget_bytes")] + [
        ("clock", ctypes.c_double), ("calls", ctypes.c_int64)]


def _declare(lib):
    if getattr(lib, "_server_declared", False):
        return lib
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    lib.dinara_server_new.restype = vp
    lib.dinara_server_new.argtypes = [vp, ctypes.POINTER(ServerOptions)]
    lib.dinara_server_free.restype = None
    lib.dinara_server_free.argtypes = [vp]
    lib.dinara_server_submit.restype = i64
    lib.dinara_server_submit.argtypes = [vp, i64, vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(native.CScoring),
                                         ctypes.POINTER(native.CMode), ctypes.POINTER(ctypes.c_int64)]
    lib.dinara_server_wait.restype = i64
    lib.dinara_server_wait.argtypes = [vp, i64, i64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(RequestTiming)]
    lib.dinara_server_stats.restype = i64
    lib.dinara_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    lib._server_declared = True
    return lib


class Server:
    """A serving loop on one GPU: `slots` requests at once within a device-memory budget."""

    def __init__(self, slots: int = 4, device_bytes: int = 40 << 30, placement: Placement | None = None):
        self.lib = _declare(native.lib())
        self.context = native.context(_placement(placement))
        self.handle = self.lib.dinara_server_new(self.context, ctypes.byref(ServerOptions(slots, device_bytes)))
        if not self.handle:
            raise RuntimeError(f"dinara-align: no server: {native.error_of(self.context)}")
        self.pairs = {}

    def submit(self, tape: Tape, scoring: Scoring, mode: Mode = Mode.GLOBAL) -> int:
        struct, _table, _alphabet = scoring._struct()
        mode_struct = mode._struct()
        ticket = ctypes.c_int64()
        code = self.lib.dinara_server_submit(self.handle, tape.pairs, tape.letters.ctypes.data,
                                             native.pointer(tape.offsets, ctypes.c_int64), ctypes.byref(struct),
                                             ctypes.byref(mode_struct), ctypes.byref(ticket))
        if code != 0:
            raise ValueError(f"dinara-align: request refused (code {code})")
        self.pairs[ticket.value] = tape.pairs
        return ticket.value

    def wait(self, ticket: int, timeout: float = 600.0) -> tuple:
        """(code, scores, statuses, timing dict) of a request, waiting at most `timeout` seconds."""
        pairs = self.pairs.get(ticket, 0)
        scores = np.zeros(max(pairs, 1), dtype=np.int32)
        statuses = np.zeros(max(pairs, 1), dtype=np.int64)
        timing = RequestTiming()
        code = self.lib.dinara_server_wait(self.handle, ticket, int(timeout * 1000),
                                           native.pointer(scores, ctypes.c_int32),
                                           native.pointer(statuses, ctypes.c_int64), ctypes.byref(timing))
        if code != native.DEVICE_TIMEOUT:
            self.pairs.pop(ticket, None)
        return code, scores[:pairs], statuses[:pairs], {name: getattr(timing, name) for name, _ in RequestTiming._fields_}

    def stats(self) -> dict:
        out = ServerStats()
        self.lib.dinara_server_stats(self.handle, ctypes.byref(out))
        return {name: getattr(out, name) for name, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            self.lib.dinara_server_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def open_loop(server: Server, requests: list, rate: float, scoring: Scoring, mode: Mode = Mode.GLOBAL,
              seed: int = 5) -> dict:
    """Submits `requests` (Tapes) at Poisson arrivals of `rate` a second and waits for all: per-request
    latencies (submission to completion), achieved pairs/s, and the offered rate."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(requests))
    arrivals = np.cumsum(gaps)
    begin = time.perf_counter()
    tickets = []
    for tape, at in zip(requests, arrivals):
        delay = at - (time.perf_counter() - begin)
        if delay > 0:
            time.sleep(delay)
        tickets.append(server.submit(tape, scoring, mode))
    latencies, pairs, codes, first, last = [], 0, [], None, 0.0
    for ticket in tickets:
        code, scores, statuses, timing = server.wait(ticket)
        codes.append(code)
        latencies.append(timing["finished"] - timing["submitted"])
        pairs += timing["pairs"] if code == 0 else 0
        first = timing["submitted"] if first is None else min(first, timing["submitted"])
        last = max(last, timing["finished"])
    span = max(last - (first or 0.0), 1e-9)
    latencies = np.asarray(latencies)
    return {"requests": len(requests), "offered_requests_per_s": rate, "pairs": pairs, "pairs_per_s": pairs / span,
            "seconds": span, "p50_s": float(np.percentile(latencies, 50)), "p99_s": float(np.percentile(latencies, 99)),
            "refused": int(sum(1 for c in codes if c == native.OUT_OF_MEMORY)),
            "failed": int(sum(1 for c in codes if c not in (0, native.OUT_OF_MEMORY)))}
