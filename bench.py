"""Benchmark of the batched alignment path on B200s, one JSON line on rank 0.

Workload (default `affine`): 1,000,000 synthetic pairs, lengths uniform 100-300 bp, uniform ACGT, the query
the reference with 5% errors (substitutions/insertions/deletions 50/25/25), global gap-affine scores plus
CIGARs under mismatch 4, gap open 6, gap extend 2 (Scoring.uniform(0, -4, -6, -2)). A step is one pass of
the path over the batch: scheduling, the recording sweep, the walk back and the CIGARs, all on the device
with the packed letters resident in HBM (`value`); `e2e` times the same batch through the C ABI from host
buffers, copies included. Every rank takes its own batch (weak scaling; pairs are independent, so there is
no collective on the data path); `value` is all ranks' pairs over the slowest rank's device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload affine|...]
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dinara-align_b200"))

WORKLOADS = {
    "affine": "global gap-affine (4,6,2) scores + CIGAR, 1,000,000 pairs 100-300 bp, 5% errors 50/25/25",
    "local": "local scores under Scoring.dna(), 100,000 queries 150-1,000 bp planted in 1,000-5,000 bp targets, "
             "8% errors 50/25/25",
    "uneven": "global unit-cost distances by band doubling, 200,000 pairs log-uniform 100 bp-20 kbp, 0.5-15% "
              "errors 50/25/25",
    "unit250": "global unit-cost distances, 10,000 pairs of 250 bp, 2% errors in thirds",
}


def parse() -> argparse.Namespace:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=40)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--workload", choices=sorted(WORKLOADS), default="affine")
    parser.add_argument("--pairs", type=int, default=0, help="override the workload's pair count")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-cpu", action="store_true")
    parser.add_argument("--no-extras", action="store_true", help="skip the learned-band and serving sections")
    return parser.parse_args()


def make_workload(name: str, pairs: int, seed: int):
    from dinara_align import workloads

    if name == "affine":
        return workloads.affine_global(pairs or 1_000_000, seed=seed)
    if name == "local":
        return workloads.local_planted(pairs or 100_000, seed=seed)
    if name == "uneven":
        return workloads.uneven_unit_cost(pairs or 200_000, seed=seed)
    return workloads.unit_cost_uniform(pairs or 10_000, seed=seed)


class Clocks:
    """nvidia-smi samples of SM clock, max clock and throttle reasons, each with its time, from start() to
    stop(); summary() keeps those taken inside a window (the timed region). The sampler starts well before
    the timed region, since nvidia-smi takes a while to give its first sample."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.process = None
        self.file = None

    def start(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.process = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.process = None
        return self

    def stop(self):
        if self.process:
            self.process.terminate()
            self.process.wait(timeout=10)
            self.process = None

    def summary(self, begin: float, end: float) -> dict:
        """The samples taken between `begin` and `end` (time.time() seconds)."""
        if not self.file:
            return {}
        self.file.seek(0)
        sm, maxima, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                at = time.mktime(time.strptime(parts[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                at += float("0." + parts[0].split(".")[1]) if "." in parts[0] else 0.0
                clock, maximum = float(parts[1]), float(parts[2])
            except (ValueError, IndexError):
                continue
            if not begin <= at <= end:
                continue
            sm.append(clock)
            maxima.append(maximum)
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.file.name)
        self.file = None
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(maxima), "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_arm(args) -> None:
    """The reference's CPU path on this host: the oracle port (dinara-align's Mojo cannot be built here),
    on all host threads, over a bounded sample of the same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    threads = os.cpu_count() or 1
    line = cpu_measure(oracle, args.workload, threads, args.steps, args.warmup)
    line.update({"impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                 "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                            "timed_on": "the host's cores, a bounded sample of the workload (cpu_baseline.sample)"},
                 "data": "synthetic", "scaling": "weak", "vs_baseline": None})
    line["e2e"] = {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))


def cpu_measure(oracle, workload: str, threads: int, steps: int, warmup: int) -> dict:
    """The oracle timed on `threads` host threads over a bounded sample of the workload: pairs/s."""
    # Sized for roughly 10-30 s of CPU work on a 16-core host.
    sample_pairs = {"affine": 400_000, "local": 20_000, "uneven": 40_000, "unit250": 10_000}[workload]
    tape = make_workload(workload, sample_pairs, seed=1000)
    letters = tape.letters[: tape.offsets[-1]]
    if workload in ("affine", "local"):
        codes = np.full(256, 255, dtype=np.uint8)
        codes[np.frombuffer(b"ACGT", np.uint8)] = np.arange(4, dtype=np.uint8)
        coded = codes[letters]
        if workload == "affine":
            table = oracle.dna_table(0, -4)
            op, ex = oracle.kernel_gaps(-6, -2)

            def run():
                oracle.batch_alignments(coded, tape.offsets, table, 4, op, ex, oracle.GLOBAL, threads=threads)
        else:
            table = oracle.dna_table(2, -4)
            op, ex = oracle.kernel_gaps(-4, -2)

            def run():
                oracle.batch_scores(coded, tape.offsets, table, 4, op, ex, oracle.LOCAL, threads=threads)
    else:
        def run():
            oracle.batch_distances(letters, tape.offsets, start=256, threads=threads)
    run()
    times = []
    for _ in range(max(1, min(steps, 3))):
        begin = time.perf_counter()
        run()
        times.append(time.perf_counter() - begin)
    seconds = statistics.median(times)
    cells = int(((tape.offsets[1::2] - tape.offsets[0:-1:2]) * (tape.offsets[2::2] - tape.offsets[1::2])).sum())
    return {"metric": "pairs/s", "value": tape.pairs / seconds, "unit": "pairs/s", "higher_is_better": True,
            "gcups": cells / seconds / 1e9, "cpu_baseline": {
                "value": tape.pairs / seconds, "unit": "pairs/s", "cores": threads, "kind": "port",
                "sample": f"{tape.pairs} pairs of the {workload} workload (seed 1000), median of "
                          f"{len(times)} runs of {seconds:.2f} s"}}


def learned_band_section(da, native, lib, handle, steps: int) -> dict:
    """The uneven unit-cost batch (200,000 pairs, log-uniform 100 bp-20 kbp, 0.5-15% errors) swept by plain
    band doubling and by the learned band, each timed on the device with the letters resident; the
    predictor first trained on the GPU on 1,000,000 pairs of the same distribution."""
    from dinara_align import learned, workloads

    predictor = learned.Predictor()
    training = predictor.train(pairs=1_000_000, epochs=4, batch=4096, seed=2024)
    tape = workloads.uneven_unit_cost(200_000, seed=7)
    cells = int(((tape.offsets[1::2] - tape.offsets[0:-1:2]) * (tape.offsets[2::2] - tape.offsets[1::2])).sum())
    native.check(lib.dinara_gpu_resident_load(handle, tape.pairs, tape.letters.ctypes.data,
                                              tape.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), None),
                 handle)
    out = {"workload": WORKLOADS["uneven"], "pairs": tape.pairs, "full_matrix_cells": cells, "training": training}
    results = {}
    for name, policy in (("plain", native.BAND_PLAIN), ("learned", native.BAND_LEARNED)):
        times, report = [], native.CBandReport()
        for k in range(2 + steps):
            timing = Timing()
            plan = native.CBandPlan(policy, None, 0)
            report = native.CBandReport()
            native.check(lib.dinara_gpu_resident_distances(handle, ctypes.byref(plan), ctypes.byref(report),
                                                           ctypes.byref(timing)), handle)
            if k >= 2:
                times.append(timing.total_ms)
        found = np.zeros(tape.pairs, dtype=np.int64)
        lib.dinara_gpu_resident_fetch(handle, None, found.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        results[name] = found
        ms = statistics.median(times)
        out[name] = {"ms": ms, "pairs_per_s": tape.pairs / (ms / 1e3), "gcups": cells / (ms / 1e3) / 1e9,
                     "report": report.as_dict()}
    out["identical_distances"] = bool((results["plain"] == results["learned"]).all())
    out["speedup"] = out["learned"]["pairs_per_s"] / out["plain"]["pairs_per_s"]
    return out


def serving_section(da) -> dict:
    """Open-loop serving: Poisson arrivals at 2,000 requests/s, each 1-4,096 pairs (log-uniform), lengths
    log-uniform 100 bp-50 kbp, 1-10% errors, global gap-affine (4,6,2) scores, a 40 GB device budget; a bounded
    run of 100 requests, offered far past what the device sustains, so latency is mostly queueing and
    requests queued together share device calls."""
    from dinara_align import serving, workloads

    rng = np.random.default_rng(55)
    requests = [workloads.serving_request(rng) for _ in range(100)]
    scoring = da.Scoring.uniform(0, -4, -6, -2)

    def cells_of(batch):
        return int(sum(((t.offsets[1::2] - t.offsets[0:-1:2]) * (t.offsets[2::2] - t.offsets[1::2])).sum()
                       for t in batch))

    with serving.Server(slots=4, device_bytes=40 << 30) as server:
        out = serving.open_loop(server, requests, 2000.0, scoring)
        out["stats"] = server.stats()
    out["cells"] = cells_of(requests)
    out["gcups"] = out["cells"] / out["seconds"] / 1e9
    out["offered_pairs_per_s"] = 2000.0 * float(np.mean([t.pairs for t in requests]))
    # The same distribution offered at 5 requests/s, about a quarter of what the device sustains on these
    # requests: latency with little standing queue (40 requests, about 8 s).
    sustained = [workloads.serving_request(rng) for _ in range(40)]
    with serving.Server(slots=4, device_bytes=40 << 30) as server:
        steady = serving.open_loop(server, sustained, 5.0, scoring, seed=6)
        steady["stats"] = server.stats()
    steady["cells"] = cells_of(sustained)
    steady["gcups"] = steady["cells"] / steady["seconds"] / 1e9
    out["sustained_5_per_s"] = steady
    return out


def int32_peak(handle, lib) -> dict:
    lib.dinara_gpu_int32_peak.restype = ctypes.c_int64
    lib.dinara_gpu_int32_peak.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
    out = {}
    for kind, name in ((0, "viaddmax"), (1, "imnmx"), (2, "iadd3")):
        rate = ctypes.c_double()
        if lib.dinara_gpu_int32_peak(handle, kind, ctypes.byref(rate)) == 0:
            out[name] = rate.value
    return out


class Timing(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("record_ms", ctypes.c_double),
                ("launches", ctypes.c_int64), ("cells", ctypes.c_int64)]


def main() -> None:
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local_rank)
    # Clock samples from now on; the line keeps those inside the timed region.
    clocks = Clocks(local_rank).start()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import dinara_align as da
    from dinara_align import _native as native

    lib = native.lib()
    handle = native.context(local_rank)
    tape = make_workload(args.workload, args.pairs, seed=7 + rank)
    pairs = tape.pairs
    cells = int(((tape.offsets[1::2] - tape.offsets[0:-1:2]) * (tape.offsets[2::2] - tape.offsets[1::2])).sum())
    scoring = da.Scoring.uniform(0, -4, -6, -2) if args.workload == "affine" else da.Scoring.dna()
    mode = da.Mode.local() if args.workload == "local" else da.Mode.GLOBAL
    unit = args.workload in ("uneven", "unit250")

    lib.dinara_gpu_resident_load.restype = ctypes.c_int64
    lib.dinara_gpu_resident_load.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    lib.dinara_gpu_resident_align.restype = ctypes.c_int64
    lib.dinara_gpu_resident_align.argtypes = [ctypes.c_void_p, ctypes.POINTER(native.CMode), ctypes.c_int64,
                                              ctypes.c_int64, ctypes.POINTER(Timing)]
    lib.dinara_gpu_resident_distances.restype = ctypes.c_int64
    lib.dinara_gpu_resident_distances.argtypes = [ctypes.c_void_p, ctypes.POINTER(native.CBandPlan),
                                                  ctypes.POINTER(native.CBandReport), ctypes.POINTER(Timing)]
    lib.dinara_gpu_resident_fetch.restype = ctypes.c_int64
    lib.dinara_gpu_resident_fetch.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_int64)]
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    code = lib.dinara_gpu_resident_load(handle, pairs, tape.letters.ctypes.data,
                                        tape.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                        None if unit else ctypes.byref(struct))
    native.check(code, handle)

    band_report = {}

    def step() -> Timing:
        timing = Timing()
        if unit:
            plan = native.CBandPlan(native.BAND_PLAIN, None, 0)
            report = native.CBandReport()
            native.check(lib.dinara_gpu_resident_distances(handle, ctypes.byref(plan), ctypes.byref(report),
                                                           ctypes.byref(timing)), handle)
            band_report.update(report.as_dict())
        else:
            native.check(lib.dinara_gpu_resident_align(handle, ctypes.byref(mode_struct), 1 if args.workload ==
                                                       "affine" else 0, 1, ctypes.byref(timing)), handle)
        return timing

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    timings = []
    region_begin = time.time()
    for _ in range(args.steps):
        timings.append(step())
    torch.cuda.synchronize()
    region_end = time.time()
    clocks.stop()
    device_ms = sum(t.total_ms for t in timings)
    kernel_ms = sum(t.record_ms + t.kernel_ms for t in timings) / len(timings)
    launches = sum(t.launches for t in timings)
    slowest = device_ms
    if dist:
        value_t = torch.tensor([device_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(value_t, op=dist.ReduceOp.MAX)
        slowest = float(value_t.item())
    ms_per_step = slowest / args.steps
    value = world * pairs / (ms_per_step / 1e3)

    # The scorer alone (scores, no CIGAR) on the same resident batch: the int32 roofline's kernel.
    scorer = None
    if not unit:
        score_timings = []
        for k in range(args.warmup + args.steps):
            timing = Timing()
            native.check(lib.dinara_gpu_resident_align(handle, ctypes.byref(mode_struct), 0, 1, ctypes.byref(timing)),
                         handle)
            if k >= args.warmup:
                score_timings.append(timing)
        scorer = {"ms_per_step": sum(t.total_ms for t in score_timings) / len(score_timings),
                  "kernel_ms": sum(t.kernel_ms for t in score_timings) / len(score_timings),
                  "swept_cells": sum(t.cells for t in score_timings) / len(score_timings)}

    # End to end through the C ABI from host buffers (page-locked, as a serving caller keeps them),
    # copies inside the timed region.
    e2e = None
    if not args.no_e2e:
        letters_pinned = torch.empty(len(tape.letters), dtype=torch.uint8, pin_memory=True).numpy()
        letters_pinned[:] = tape.letters
        offsets_pinned = torch.empty(len(tape.offsets), dtype=torch.int64, pin_memory=True).numpy()
        offsets_pinned[:] = tape.offsets
        host_tape = da.Tape(letters_pinned, offsets_pinned)
        times = []
        h2d = int(tape.offsets[-1]) + tape.offsets.nbytes
        d2h = 0
        for k in range(2 + max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            begin = time.perf_counter()
            if unit:
                found = da.distances_tape(host_tape)
                d2h = found.nbytes
            elif args.workload == "affine":
                found, spans, offsets, data, codes = da.alignments_tape(host_tape, scoring, mode)
                d2h = found.nbytes + offsets.nbytes + len(data) + codes.nbytes + spans.nbytes
            else:
                found, codes = da.scores_tape(host_tape, scoring, mode, statuses=True)
                d2h = found.nbytes + codes.nbytes
            elapsed = time.perf_counter() - begin
            if k >= 2:
                times.append(elapsed)
        e2e_seconds = statistics.median(times)
        slow = e2e_seconds
        if dist:
            t = torch.tensor([e2e_seconds], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            slow = float(t.item())
        e2e = {"value": world * pairs / slow, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "seconds_per_step": slow, "host_buffers": "page-locked"}

    if rank == 0:
        peaks = int32_peak(handle, lib)
        ops_per_cell = 8 if args.workload == "local" else 7
        line = {
            "metric": "pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic",
            # Scores: 16-bit halves where a pair's values provably fit (exact), 32 bits otherwise.
            "dtype": "u64" if unit else "int16x2+int32",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "pairs_per_gpu": pairs,
                       "full_matrix_cells_per_gpu": cells, "l2": "inputs larger than L2 (packed tape and decisions)",
                       "parallelism": f"pairs sharded, {world} independent ranks"},
            "gcups": world * cells / (ms_per_step / 1e3) / 1e9,
            "gpu_launches": launches,
            "clocks": clocks.summary(region_begin, region_end),
            "e2e": e2e,
        }
        swept = sum(t.cells for t in timings) / len(timings)
        if not unit and "viaddmax" in peaks:
            peak = 2 * peaks["viaddmax"]
            achieved = swept * ops_per_cell / (kernel_ms / 1e3)
            line["roofline"] = {"bound": "int32", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gops/s",
                                "frac": achieved / peak, "ops_per_cell": ops_per_cell,
                                "swept_cells_per_step": swept, "kernel_ms_per_step": kernel_ms,
                                "kernel": "the recording sweep (band, then whole matrices for the rest) and the walk",
                                "peak_source": "measured in this run: DPX viaddmax chains on every SM, 2 ops each"}
        if unit and band_report and "viaddmax" in peaks and band_report.get("kernel_ms"):
            # A Myers/Hyyro word step is about 20 u64 operations (bit_parallel.mojo:10-11), 40 in int32 terms,
            # over the words the band kernels swept, against the same int32 peak as the scorers.
            peak = 2 * peaks["viaddmax"]
            achieved = band_report["words_swept"] * 40 / (band_report["kernel_ms"] / 1e3)
            line["roofline"] = {"bound": "int32", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gops/s",
                                "frac": achieved / peak, "traffic": None, "ops_per_word_step": 40,
                                "words_swept_per_step": band_report["words_swept"],
                                "kernel_ms_per_step": band_report["kernel_ms"],
                                "kernel": "the band kernels of every round (band_kernel, all window shapes)",
                                "peak_source": "measured in this run: DPX viaddmax chains on every SM, 2 ops each"}
        if "roofline" in line and args.workload == "affine":
            # DRAM bytes of the recording band sweep (dram__bytes_read.sum + dram__bytes_write.sum), from an
            # ncu capture of 200,000 pairs of this distribution (8,217 bytes a pair: the recorded decisions
            # and the sectors filled around their stores), scaled to this batch.
            line["roofline"]["traffic"] = 8217.0 * pairs
            line["roofline"]["traffic_unit"] = "bytes per launch of the recording band sweep"
        elif "roofline" in line:
            line["roofline"]["traffic"] = None
        if scorer and "viaddmax" in peaks:
            achieved = scorer["swept_cells"] * ops_per_cell / (scorer["kernel_ms"] / 1e3)
            scorer.update({"pairs_per_s": world * pairs / (scorer["ms_per_step"] / 1e3),
                           "gcups_full_matrix": cells / (scorer["kernel_ms"] / 1e3) / 1e9,
                           "roofline_frac": achieved / (2 * peaks["viaddmax"]),
                           "achieved_gops": achieved / 1e9})
            line["scorer"] = scorer
        if band_report:
            line["band_report"] = band_report
        if world == 1 and not args.no_extras and args.workload == "affine":
            line["learned_band"] = learned_band_section(da, native, lib, handle, max(1, min(args.steps, 3)))
            line["serving"] = serving_section(da)
        line["int32_peaks_instr_per_s"] = peaks
        if not args.no_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle

            line["cpu_baseline"] = cpu_measure(oracle, args.workload, os.cpu_count() or 1, 3, 1)["cpu_baseline"]
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
