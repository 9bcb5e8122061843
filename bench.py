"""Benchmark of the batched alignment path on B200s, one JSON line on rank 0.

Headline workload (default `uneven`, the metric's own comparison): 200,000 synthetic pairs, lengths
log-uniform 100 bp-20 kbp, per-pair error rate uniform 0.5-15% (substitutions/insertions/deletions
50/25/25), global unit-cost edit distances by band doubling. The learned band (a 258-64-64-1 network over
4-mer count differences and a 6-mer sketch, trained first on the GPU on 1,000,000 pairs of the same
distribution, whose exact distances plain band doubling measures) sets each pair's first threshold; plain
band doubling from the default band is run beside it as the check, and both must give the same distance on
every pair. Each arm sweeps with the band tuning's chain bound measured fastest for its own starts.

A step is one pass of the path over the batch with the letters resident in HBM (`value`, device time on
the context's stream); `e2e` times the same batch through the library's public call from page-locked host
buffers, copies included. Every rank takes its own batch (weak scaling; pairs are independent, so there is
no collective on the data path); `value` is all ranks' pairs over the slowest rank's device time.

Sections after the headline, each with its own device line, end-to-end figure, per-kernel rooflines, CPU
leg and a parity sample against the oracle: `affine` (1,000,000 pairs, 100-300 bp, 5% errors, global
(4,6,2) scores + CIGARs), `local` (100,000 planted queries, Scoring.dna()), `unit250` (10,000 pairs of
250 bp, 2% errors) and `serving` (open-loop Poisson arrivals).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload uneven|...]
"""

from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dinara-align_b200"))

WORKLOADS = {
    "uneven": "global unit-cost distances by band doubling, learned band against plain, 200,000 pairs log-uniform "
              "100 bp-20 kbp, 0.5-15% errors 50/25/25",
    "affine": "global gap-affine (4,6,2) scores + CIGAR, 1,000,000 pairs 100-300 bp, 5% errors 50/25/25",
    "local": "local scores under Scoring.dna(), 100,000 queries 150-1,000 bp planted in 1,000-5,000 bp targets, "
             "8% errors 50/25/25",
    "unit250": "global unit-cost distances, 10,000 pairs of 250 bp, 2% errors in thirds",
}

# The band tuning's chain bound, as the bench reports each arm's.
CHAIN_KEYS = ("chain_words", "chain_share", "reach")

# The host work the CPU legs sample, sized for roughly 10-30 s of CPU work on a 16-core host.
CPU_SAMPLE = {"uneven": 40_000, "affine": 400_000, "local": 20_000, "unit250": 10_000}


def parse() -> argparse.Namespace:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--workload", choices=list(WORKLOADS), default="uneven")
    parser.add_argument("--pairs", type=int, default=0, help="override the headline workload's pair count")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-cpu", action="store_true")
    parser.add_argument("--no-parity", action="store_true")
    parser.add_argument("--no-sections", action="store_true", help="only the headline workload")
    parser.add_argument("--arms", choices=["both", "learned", "plain"], default="both",
                        help="the uneven workload's arms to run (profiling one at a time)")
    parser.add_argument("--tuning", default="",
                        help="band tuning file: loaded when the file exists, else measured and saved there")
    parser.add_argument("--predictor", default="",
                        help="band predictor blob: loaded when the file exists, else trained and saved there")
    parser.add_argument("--selftest-ranks", action="store_true",
                        help="check the rank launch and the max-over-ranks timing on the CPU (gloo), no GPU work")
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


def cells_of(tape) -> int:
    return int(((tape.offsets[1::2] - tape.offsets[0:-1:2]) * (tape.offsets[2::2] - tape.offsets[1::2])).sum())


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


class Ranks:
    """This process's place among the ranks torchrun started (one a GPU), with the two collectives the
    bench takes: a barrier around the timed region and the max of the ranks' times after it."""

    def __init__(self, backend: str):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max(self, value: float) -> float:
        if not self.dist:
            return value
        import torch

        tensor = torch.tensor([value], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(tensor, op=self.dist.ReduceOp.MAX)
        return float(tensor.item())

    def close(self) -> None:
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def spawn_ranks(args) -> int:
    """`--gpus N` with N > 1 outside torchrun: starts N ranks on this node through torchrun, each running
    this script with the same arguments, and returns their exit status (rank 0 prints the line)."""
    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        port = probe.getsockname()[1]
    command = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(command)


def selftest_ranks(args) -> None:
    """The launch and timing protocol without a GPU: each rank times a host loop of its own length between
    barriers, and rank 0 prints the max over ranks, as the GPU arm does with device time."""
    ranks = Ranks("gloo")
    ranks.barrier()
    begin = time.perf_counter()
    total = 0
    for k in range(200_000 * (1 + ranks.rank)):
        total += k
    elapsed = time.perf_counter() - begin
    slowest = ranks.max(elapsed)
    if ranks.rank == 0:
        print(json.dumps({"metric": "selftest", "n_gpus": ranks.world, "slowest_s": slowest, "own_s": elapsed,
                          "steps": args.steps, "warmup": args.warmup}))
    ranks.close()


class Timing(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("record_ms", ctypes.c_double),
                ("launches", ctypes.c_int64), ("cells", ctypes.c_int64), ("class_ms", ctypes.c_double * 8),
                ("class_launches", ctypes.c_int64 * 8), ("band_cells", ctypes.c_int64),
                ("whole_cells", ctypes.c_int64)]


# dinara_timing.class_ms's kernel classes.
CLASS_BAND_RECORD, CLASS_BAND_SCORE, CLASS_WHOLE, CLASS_WALK, CLASS_UNIT_BAND, CLASS_PREDICT = 0, 1, 2, 3, 4, 5


def declare(lib, native):
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
    lib.dinara_gpu_int32_peak.restype = ctypes.c_int64
    lib.dinara_gpu_int32_peak.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]


def int32_peaks(handle, lib) -> dict:
    out = {}
    for kind, name in ((0, "viaddmax"), (1, "imnmx"), (2, "iadd3"), (3, "viaddmax_16x2")):
        rate = ctypes.c_double()
        if lib.dinara_gpu_int32_peak(handle, kind, ctypes.byref(rate)) == 0:
            out[name] = rate.value
    return out


def measured_hbm_gbs() -> tuple:
    """The pool's measured copy bandwidth (MEASURED_PEAKS.json) or the stated fallback, and which."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def timed_steps(step, steps: int, warmup: int, ranks) -> tuple:
    """W untimed steps, then K steps bracketed by a barrier and a device synchronize on both sides:
    (per-step results, wall-clock begin and end of the timed region)."""
    import torch

    for _ in range(warmup):
        step()
    ranks.barrier()
    torch.cuda.synchronize()
    begin = time.time()
    results = [step() for _ in range(steps)]
    torch.cuda.synchronize()
    ranks.barrier()
    return results, begin, time.time()


def pinned_tape(da, tape):
    """The tape in page-locked host memory, as a serving caller keeps its buffers."""
    import torch

    letters = torch.empty(len(tape.letters), dtype=torch.uint8, pin_memory=True).numpy()
    letters[:] = tape.letters
    offsets = torch.empty(len(tape.offsets), dtype=torch.int64, pin_memory=True).numpy()
    offsets[:] = tape.offsets
    return da.Tape(letters, offsets)


def sub_tape(tape, pairs):
    from dinara_align import shards

    return shards.subset(tape, np.sort(pairs))


def kernel_entry(name: str, ops: float, ms: float, peak_ops: float, launches: int, note: str, **extra) -> dict:
    """One kernel class's roofline entry: algorithmic int32 operations per step over its device time."""
    if ms <= 0:
        return {"kernel": name, "ms_per_step": ms, "note": "not launched"}
    achieved = ops / (ms / 1e3)
    out = {"kernel": name, "bound": "int32", "ms_per_step": ms, "launches_per_step": launches,
           "ops_per_step": ops, "achieved": achieved / 1e9, "peak": peak_ops / 1e9, "unit": "Gops/s",
           "frac": achieved / peak_ops, "work": note}
    out.update(extra)
    return out


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle


def coded(tape):
    codes = np.full(256, 255, dtype=np.uint8)
    codes[np.frombuffer(b"ACGT", np.uint8)] = np.arange(4, dtype=np.uint8)
    return codes[tape.letters[: tape.offsets[-1]]]


# ---------------------------------------------------------------------------------------------------------
# The CPU legs: the oracle (a C restatement of the reference's CPU algorithms) on the host's cores.


def cpu_measure(workload: str, threads: int, runs: int, gotoh: bool = False) -> dict:
    """The oracle timed on `threads` host threads over a bounded sample of the workload: pairs/s. For the
    global affine workload the reference's host path for a uniform Scoring is the gap-affine wavefront
    (scoring.mojo:414-440), restated in the oracle; `gotoh` times the full-matrix Gotoh walk instead."""
    oracle = oracle_module()
    tape = make_workload(workload, CPU_SAMPLE[workload], seed=1000)
    letters = tape.letters[: tape.offsets[-1]]
    if workload == "affine" and not gotoh:
        what = ("the gap-affine wavefront's costs and CIGARs under Costs.affine(4,6,2), one search from the start "
                "traced back (gap_affine.mojo:858-1010, 2028-2124), the reference's host path for a uniform Scoring")

        def run():
            oracle.batch_wavefront(letters, tape.offsets, 4, 6, 2, threads=threads)
    elif workload == "affine":
        table, (op, ex) = oracle.dna_table(0, -4), oracle.kernel_gaps(-6, -2)
        what = "full-matrix Gotoh scores and the walk's CIGARs (gotoh.mojo:285-510)"

        def run():
            oracle.batch_alignments(coded(tape), tape.offsets, table, 4, op, ex, oracle.GLOBAL, threads=threads)
    elif workload == "local":
        table, (op, ex) = oracle.dna_table(2, -4), oracle.kernel_gaps(-4, -2)
        what = "full-matrix local Gotoh scores (gotoh.mojo:285-362, beats :122-127)"

        def run():
            oracle.batch_scores(coded(tape), tape.offsets, table, 4, op, ex, oracle.LOCAL, threads=threads)
    else:
        what = "band doubling from the default band (band.mojo:526-657), Myers/Hyyro words"

        def run():
            oracle.batch_distances(letters, tape.offsets, start=256, threads=threads)
    run()
    times = []
    for _ in range(max(1, runs)):
        begin = time.perf_counter()
        run()
        times.append(time.perf_counter() - begin)
    seconds = statistics.median(times)
    return {"value": tape.pairs / seconds, "unit": "pairs/s", "cores": threads, "kind": "port",
            "gcups": cells_of(tape) / seconds / 1e9,
            "sample": f"{tape.pairs} pairs of the {workload} workload (seed 1000): {what}; median of {len(times)} "
                      f"runs of {seconds:.2f} s"}


def reference_arm(args) -> None:
    """The reference's CPU path on this host, timed on all host threads over a bounded sample of the same
    workload: the oracle port, since dinara-align's Mojo cannot be built here."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    threads = os.cpu_count() or 1
    base = cpu_measure(args.workload, threads, max(1, min(args.steps, 3)))
    line = {"metric": "pairs/s", "value": base["value"], "unit": "pairs/s", "higher_is_better": True,
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "timed_on": "the host's cores, a bounded sample of the workload (cpu_baseline.sample)"},
            "data": "synthetic", "scaling": "weak", "vs_baseline": None, "gcups": base["gcups"],
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}}
    line["e2e"] = {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------------------------
# The workloads on the GPU. Each returns the figures of its line: `value` and `ms_per_step` from the device
# time of `steps` timed steps (max over ranks), `e2e`, per-kernel rooflines and a parity sample.


def run_uneven(ctx, tape, steps, warmup) -> dict:
    """Config 4: the learned band against plain band doubling, letters resident; the predictor trained on
    the GPU first."""
    da, native, lib, handle, ranks, peaks = ctx["da"], ctx["native"], ctx["lib"], ctx["handle"], ctx["ranks"], \
        ctx["peaks"]
    from dinara_align import learned, tuning

    placement = da.Placement.on_gpu(ranks.local_rank)
    # The band autotuner first: both arms then sweep with the shapes it measured, each with the chain bound
    # it measured fastest for that arm's starts (plain doubling's, or near each distance as a learned start
    # is), and the predictor's margins are calibrated against the windows the learned arm's tuning gives.
    tuning_file = ctx.get("tuning", "")
    if tuning_file and os.path.exists(tuning_file):
        with open(tuning_file) as source:
            kept = json.load(source)
        arm_tunings = kept if "learned" in kept else {"learned": kept, "plain": kept}
        learned_tuning = arm_tunings["learned"]
        tuned = {"chain_words": learned_tuning["chain_words"], "chain_share": learned_tuning["chain_share"],
                 "chain_ms": {}, "seconds": 0.0, "words_per_ms": {}, "loaded": tuning_file}
    else:
        tuned = tuning.autotune(placement, pairs=tape.pairs)
        measured = tuning.tuning(placement)
        arm_tunings = {"learned": tuning.tuning_for_starts(tuned, measured, near=True),
                       "plain": tuning.tuning_for_starts(tuned, measured, near=False)}
        if tuning_file:
            with open(tuning_file, "w") as out_file:
                json.dump(arm_tunings, out_file)
    tuning.install(arm_tunings["learned"], placement)
    predictor = learned.Predictor(placement)
    blob = ctx.get("predictor", "")
    if blob and os.path.exists(blob):
        predictor.load(blob)
        training = {"loaded": blob}
    else:
        training = predictor.train(pairs=1_000_000, epochs=4, batch=1024, seed=2024)
        if blob:
            predictor.save(blob)
    native.check(lib.dinara_gpu_resident_load(handle, tape.pairs, tape.letters.ctypes.data,
                                              tape.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), None),
                 handle)
    reports = {}

    def stepper(policy, name):
        def step():
            timing, report = Timing(), native.CBandReport()
            plan = native.CBandPlan(policy, None, 0)
            native.check(lib.dinara_gpu_resident_distances(handle, ctypes.byref(plan), ctypes.byref(report),
                                                           ctypes.byref(timing)), handle)
            reports[name] = report.as_dict()
            return timing
        return step

    found = {}
    out = {}
    arms = [(name, policy) for name, policy in (("learned", native.BAND_LEARNED), ("plain", native.BAND_PLAIN))
            if ctx.get("arms", "both") in ("both", name)]
    for name, policy in arms:
        tuning.install(arm_tunings[name], placement)
        timings, begin, end = timed_steps(stepper(policy, name), steps, warmup, ranks)
        device_ms = ranks.max(sum(t.total_ms for t in timings))
        result = np.zeros(tape.pairs, dtype=np.int64)
        lib.dinara_gpu_resident_fetch(handle, None, result.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        found[name] = result
        per_step = device_ms / steps
        out[name] = {"ms_per_step": per_step, "pairs_per_s": ranks.world * tape.pairs / (per_step / 1e3),
                     "gcups_full_matrix": ranks.world * ctx["cells"] / (per_step / 1e3) / 1e9,
                     "launches_per_step": sum(t.launches for t in timings) / steps,
                     "band_ms_per_step": sum(t.class_ms[CLASS_UNIT_BAND] for t in timings) / steps,
                     "predict_ms_per_step": sum(t.class_ms[CLASS_PREDICT] for t in timings) / steps,
                     "report": reports[name], "timed_region": [begin, end]}
    tuning.install(arm_tunings["learned"], placement)  # the end-to-end calls run the learned band
    if len(out) == 1:
        # One arm alone (a profiling run): its own figures, no comparison.
        (name, only), = out.items()
        return {"value": only["pairs_per_s"], "ms_per_step": only["ms_per_step"],
                "gpu_launches": int(only["launches_per_step"] * steps), "timed_region": only["timed_region"],
                "arm": name, name: only, "training": training}
    line = {"value": out["learned"]["pairs_per_s"], "ms_per_step": out["learned"]["ms_per_step"],
            "gpu_launches": int(out["learned"]["launches_per_step"] * steps),
            "timed_region": out["learned"]["timed_region"],
            "plain_value": out["plain"]["pairs_per_s"], "plain_ms_per_step": out["plain"]["ms_per_step"],
            "speedup_learned_over_plain": out["learned"]["pairs_per_s"] / out["plain"]["pairs_per_s"],
            "identical_distances": bool((found["learned"] == found["plain"]).all()),
            "gcups": out["learned"]["gcups_full_matrix"], "plain_gcups": out["plain"]["gcups_full_matrix"],
            "learned": out["learned"], "plain": out["plain"], "training": training,
            "autotune": {"chain_words": tuned["chain_words"], "chain_share": tuned["chain_share"],
                         "chain_ms": tuned["chain_ms"], "chain_ms_near": tuned.get("chain_ms_near", {}),
                         "learned_chain": {k: arm_tunings["learned"][k] for k in CHAIN_KEYS},
                         "plain_chain": {k: arm_tunings["plain"][k] for k in CHAIN_KEYS},
                         "seconds": tuned["seconds"], "words_per_ms": tuned["words_per_ms"]}}
    # The dominant kernel: every round's band kernels. A Myers/Hyyro word step is about 20 u64 operations
    # (bit_parallel.mojo:10-11), 40 in int32 terms, over the words the rounds swept.
    kernels = []
    if "viaddmax" in peaks:
        peak = 2 * peaks["viaddmax"]
        for name in ("learned", "plain"):
            report = out[name]["report"]
            kernels.append(kernel_entry(f"band_kernel rounds ({name} band)", report["words_swept"] * 40,
                                        report["kernel_ms"], peak, sum(report["round_launches"]),
                                        "40 int32 ops a 64-cell word step, words the rounds swept",
                                        words_swept=report["words_swept"]))
        letters = int(tape.offsets[-1])
        predict_ms = out["learned"]["predict_ms_per_step"]
        if predict_ms > 0:
            hbm, hbm_source = measured_hbm_gbs()
            kernels.append({"kernel": "features_kernel + predict_kernel (learned band)", "bound": "hbm",
                            "ms_per_step": predict_ms, "bytes_per_step": letters,
                            "achieved": letters / (predict_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                            "frac": letters / (predict_ms / 1e3) / 1e9 / hbm, "peak_source": hbm_source,
                            "work": "each letter read once for the 4-mer sketch"})
        line["roofline"] = dict(kernels[0], traffic=None,
                                peak_source="measured in this run: DPX viaddmax chains on every SM, 2 ops each")
    line["kernels"] = kernels
    if ctx["e2e"]:
        host = pinned_tape(da, tape)
        times = []
        result = None
        for k in range(2 + 3):
            begin = time.perf_counter()
            result = da.distances_tape(host, policy=native.BAND_LEARNED, placement=placement)
            if k >= 2:
                times.append(time.perf_counter() - begin)
        slow = ranks.max(statistics.median(times))
        line["e2e"] = {"value": ranks.world * tape.pairs / slow, "unit": "pairs/s",
                       "h2d_bytes_per_step": int(tape.offsets[-1]) + tape.offsets.nbytes,
                       "d2h_bytes_per_step": result.nbytes, "seconds_per_step": slow,
                       "host_buffers": "page-locked", "call": "dinara_align.distances_tape(policy=BAND_LEARNED)"}
        line["e2e_identical"] = bool((result == found["learned"]).all())
    if ctx["parity"]:
        rng = np.random.default_rng(99)
        sample = rng.choice(tape.pairs, size=min(2000, tape.pairs), replace=False)
        part = sub_tape(tape, sample)
        oracle = oracle_module()
        expected = oracle.batch_distances(part.letters[: part.offsets[-1]], part.offsets, start=256, threads=16)
        got = found["learned"][np.sort(sample)]
        line["parity_sample"] = {"pairs": int(len(sample)), "mismatches": int((got != expected).sum()),
                                 "against": "the oracle's band doubling (band.mojo:526-657), seeded sample"}
    return line


def run_scoring(ctx, workload, tape, steps, warmup) -> dict:
    """Configs 2 (global scores + CIGARs) and 3 (local scores), letters resident and packed."""
    da, native, lib, handle, ranks, peaks = ctx["da"], ctx["native"], ctx["lib"], ctx["handle"], ctx["ranks"], \
        ctx["peaks"]
    affine = workload == "affine"
    scoring = da.Scoring.uniform(0, -4, -6, -2) if affine else da.Scoring.dna()
    mode = da.Mode.GLOBAL if affine else da.Mode.local()
    struct, _table, _alphabet = scoring._struct()
    mode_struct = mode._struct()
    native.check(lib.dinara_gpu_resident_load(handle, tape.pairs, tape.letters.ctypes.data,
                                              tape.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                              ctypes.byref(struct)), handle)

    def stepper(cigars):
        def step():
            timing = Timing()
            native.check(lib.dinara_gpu_resident_align(handle, ctypes.byref(mode_struct), cigars, 1,
                                                       ctypes.byref(timing)), handle)
            return timing
        return step

    timings, begin, end = timed_steps(stepper(1 if affine else 0), steps, warmup, ranks)
    device_ms = ranks.max(sum(t.total_ms for t in timings))
    per_step = device_ms / steps
    mean = lambda values: sum(values) / len(timings)  # noqa: E731
    line = {"value": ranks.world * tape.pairs / (per_step / 1e3), "ms_per_step": per_step,
            "gpu_launches": sum(t.launches for t in timings), "timed_region": [begin, end],
            "gcups": ranks.world * ctx["cells"] / (per_step / 1e3) / 1e9,
            "swept_cells_per_step": mean([t.cells for t in timings])}
    ops_per_cell = 7 if affine else 8
    kernels = []
    if "viaddmax" in peaks:
        peak = 2 * peaks["viaddmax"]
        hbm, hbm_source = measured_hbm_gbs()
        band_cells = mean([t.band_cells for t in timings])
        whole_cells = mean([t.whole_cells for t in timings])
        if affine:
            ms = mean([t.class_ms[CLASS_BAND_RECORD] for t in timings])
            # Recorded decisions: 4 bits a band cell, written once.
            kernels.append(kernel_entry("banded_pairs_kernel / banded_kernel, recording", band_cells * ops_per_cell,
                                        ms, peak, int(mean([t.class_launches[CLASS_BAND_RECORD] for t in timings])),
                                        "7 int32 ops a band cell (3 add + 4 max), DPX add-max as 2",
                                        band_cells=band_cells, decision_bytes=band_cells / 2,
                                        decision_gbs=(band_cells / 2) / (ms / 1e3) / 1e9 if ms else None,
                                        hbm_frac=(band_cells / 2) / (ms / 1e3) / 1e9 / hbm if ms else None,
                                        hbm_peak_source=hbm_source))
        ms = mean([t.class_ms[CLASS_WHOLE] for t in timings])
        kernels.append(kernel_entry("whole-matrix sweeps" + (" (the band's leftovers, recording)" if affine else ""),
                                    whole_cells * ops_per_cell, ms, peak,
                                    int(mean([t.class_launches[CLASS_WHOLE] for t in timings])),
                                    f"{ops_per_cell} int32 ops a cell", cells=whole_cells))
        if affine:
            ms = mean([t.class_ms[CLASS_WALK] for t in timings])
            kernels.append({"kernel": "walk_kernel", "bound": "latency", "ms_per_step": ms,
                            "pairs_per_s": tape.pairs / (ms / 1e3) if ms else None,
                            "work": "one dependent 4-bit decision read a CIGAR step, a thread a pair"})
        line["roofline"] = dict(kernels[0], traffic=6190.0 * tape.pairs if affine else None,
                                traffic_unit="bytes a step of the recording band sweep, its two launches (ncu "
                                             "capture of 200,000 pairs, 6,190 bytes a pair, scaled)"
                                if affine else None,
                                peak_source="measured in this run: DPX viaddmax chains on every SM, 2 ops each")
    line["kernels"] = kernels
    if affine:
        # The score-only sweep on the same resident batch.
        timings, _, _ = timed_steps(stepper(0), steps, warmup, ranks)
        ms = sum(t.total_ms for t in timings) / len(timings)
        kernel_ms = sum(t.class_ms[CLASS_BAND_SCORE] + t.class_ms[CLASS_WHOLE] for t in timings) / len(timings)
        cells = sum(t.cells for t in timings) / len(timings)
        scorer = {"ms_per_step": ms, "pairs_per_s": ranks.world * tape.pairs / (ms / 1e3),
                  "kernel_ms": kernel_ms, "swept_cells": cells}
        if "viaddmax" in peaks:
            achieved = cells * 7 / (kernel_ms / 1e3)
            scorer.update({"roofline_frac_int32_ops": achieved / (2 * peaks["viaddmax"]),
                           "achieved_gops": achieved / 1e9})
            if "viaddmax_16x2" in peaks:
                # A 16-bit pair instruction carries two cells: against the rate such instructions issue.
                scorer["roofline_frac_16x2_issue"] = achieved / (4 * peaks["viaddmax_16x2"])
        line["scorer"] = scorer
    found_scores = None
    if ctx["e2e"]:
        host = pinned_tape(da, tape)
        times = []
        result = None
        for k in range(2 + 3):
            begin_e = time.perf_counter()
            if affine:
                result = da.alignments_tape(host, scoring, mode, placement=da.Placement.on_gpu(ranks.local_rank))
                d2h = result[0].nbytes + result[2].nbytes + len(result[3]) + result[4].nbytes
            else:
                result = da.scores_tape(host, scoring, mode, statuses=True, placement=da.Placement.on_gpu(
                    ranks.local_rank))
                d2h = result[0].nbytes + result[1].nbytes
            if k >= 2:
                times.append(time.perf_counter() - begin_e)
        slow = ranks.max(statistics.median(times))
        line["e2e"] = {"value": ranks.world * tape.pairs / slow, "unit": "pairs/s",
                       "h2d_bytes_per_step": int(tape.offsets[-1]) + tape.offsets.nbytes, "d2h_bytes_per_step": d2h,
                       "seconds_per_step": slow, "host_buffers": "page-locked",
                       "call": "dinara_align.alignments_tape" if affine else "dinara_align.scores_tape"}
        found_scores = result
    if ctx["parity"] and found_scores is not None:
        oracle = oracle_module()
        rng = np.random.default_rng(98)
        sample = np.sort(rng.choice(tape.pairs, size=min(2000 if affine else 200, tape.pairs), replace=False))
        part = sub_tape(tape, sample)
        if affine:
            table, (op, ex) = oracle.dna_table(0, -4), oracle.kernel_gaps(-6, -2)
            scores, cigars = oracle.batch_alignments(coded(part), part.offsets, table, 4, op, ex, oracle.GLOBAL,
                                                     threads=16)
            got_scores, _spans, offsets, data, _codes = found_scores
            got_cigars = [data[offsets[p]:offsets[p + 1]].tobytes().decode() for p in sample]
            mismatches = int((got_scores[sample] != scores).sum()) + sum(
                1 for a, b in zip(got_cigars, cigars) if a != b)
            against = "the oracle's full-matrix Gotoh scores and walk CIGARs, seeded sample"
        else:
            table, (op, ex) = oracle.dna_table(2, -4), oracle.kernel_gaps(-4, -2)
            scores = oracle.batch_scores(coded(part), part.offsets, table, 4, op, ex, oracle.LOCAL, threads=16)
            mismatches = int((found_scores[0][sample] != scores).sum())
            against = "the oracle's full-matrix local Gotoh scores, seeded sample"
        line["parity_sample"] = {"pairs": int(len(sample)), "mismatches": mismatches, "against": against}
    return line


def run_unit250(ctx, tape, steps, warmup) -> dict:
    """Config 1: 10,000 pairs of 250 bp, plain band doubling, letters resident."""
    da, native, lib, handle, ranks = ctx["da"], ctx["native"], ctx["lib"], ctx["handle"], ctx["ranks"]
    native.check(lib.dinara_gpu_resident_load(handle, tape.pairs, tape.letters.ctypes.data,
                                              tape.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), None),
                 handle)

    def step():
        timing, report = Timing(), native.CBandReport()
        plan = native.CBandPlan(native.BAND_PLAIN, None, 0)
        native.check(lib.dinara_gpu_resident_distances(handle, ctypes.byref(plan), ctypes.byref(report),
                                                       ctypes.byref(timing)), handle)
        return timing

    timings, begin, end = timed_steps(step, steps, warmup, ranks)
    per_step = ranks.max(sum(t.total_ms for t in timings)) / steps
    line = {"value": ranks.world * tape.pairs / (per_step / 1e3), "ms_per_step": per_step,
            "gpu_launches": sum(t.launches for t in timings), "timed_region": [begin, end],
            "gcups": ranks.world * ctx["cells"] / (per_step / 1e3) / 1e9}
    found = np.zeros(tape.pairs, dtype=np.int64)
    lib.dinara_gpu_resident_fetch(handle, None, found.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if ctx["e2e"]:
        host = pinned_tape(da, tape)
        times = []
        for k in range(2 + 5):
            begin_e = time.perf_counter()
            result = da.distances_tape(host, placement=da.Placement.on_gpu(ranks.local_rank))
            if k >= 2:
                times.append(time.perf_counter() - begin_e)
        slow = ranks.max(statistics.median(times))
        line["e2e"] = {"value": ranks.world * tape.pairs / slow, "unit": "pairs/s",
                       "h2d_bytes_per_step": int(tape.offsets[-1]) + tape.offsets.nbytes,
                       "d2h_bytes_per_step": result.nbytes, "seconds_per_step": slow, "host_buffers": "page-locked",
                       "call": "dinara_align.distances_tape"}
    if ctx["parity"]:
        oracle = oracle_module()
        expected = oracle.batch_distances(tape.letters[: tape.offsets[-1]], tape.offsets, start=256, threads=16)
        line["parity_sample"] = {"pairs": tape.pairs, "mismatches": int((found != expected).sum()),
                                 "against": "the oracle's band doubling, every pair"}
    return line


def serving_section(da) -> dict:
    """Open-loop serving: Poisson arrivals at 2,000 requests/s, each 1-4,096 pairs (log-uniform), lengths
    log-uniform 100 bp-50 kbp, 1-10% errors, global gap-affine (4,6,2) scores, a 40 GB device budget; a bounded
    run of 100 requests, offered far past what the device sustains, so latency is mostly queueing and
    requests queued together share device calls."""
    from dinara_align import serving, workloads

    rng = np.random.default_rng(55)
    requests = [workloads.serving_request(rng) for _ in range(100)]
    scoring = da.Scoring.uniform(0, -4, -6, -2)

    def total_cells(batch):
        return int(sum(cells_of(t) for t in batch))

    with serving.Server(slots=4, device_bytes=40 << 30) as server:
        out = serving.open_loop(server, requests, 2000.0, scoring)
        out["stats"] = server.stats()
    out["cells"] = total_cells(requests)
    out["gcups"] = out["cells"] / out["seconds"] / 1e9
    out["offered_pairs_per_s"] = 2000.0 * float(np.mean([t.pairs for t in requests]))
    # The same distribution offered at 5 requests/s: latency with little standing queue (40 requests).
    sustained = [workloads.serving_request(rng) for _ in range(40)]
    with serving.Server(slots=4, device_bytes=40 << 30) as server:
        steady = serving.open_loop(server, sustained, 5.0, scoring, seed=6)
        steady["stats"] = server.stats()
    steady["cells"] = total_cells(sustained)
    steady["gcups"] = steady["cells"] / steady["seconds"] / 1e9
    out["sustained_5_per_s"] = steady
    return out


RUNNERS = {"uneven": run_uneven, "affine": lambda ctx, tape, s, w: run_scoring(ctx, "affine", tape, s, w),
           "local": lambda ctx, tape, s, w: run_scoring(ctx, "local", tape, s, w), "unit250": run_unit250}


def run_workload(ctx, workload: str, pairs: int, steps: int, warmup: int, cpu: bool) -> dict:
    tape = make_workload(workload, pairs, seed=7 + ctx["ranks"].rank)
    ctx["cells"] = cells_of(tape)
    line = RUNNERS[workload](ctx, tape, steps, warmup)
    line["config"] = {"workload": workload, "description": WORKLOADS[workload], "pairs_per_gpu": tape.pairs,
                      "full_matrix_cells_per_gpu": ctx["cells"],
                      "l2": "inputs larger than L2 (letters resident; packed tape and decisions)"
                            if workload != "unit250" else "letters 5 MB, within L2: the step is latency bound",
                      "parallelism": f"pairs sharded, {ctx['ranks'].world} independent ranks"}
    if cpu and ctx["ranks"].rank == 0:
        line["cpu_baseline"] = cpu_measure(workload, os.cpu_count() or 1, 1 if workload != "unit250" else 3)
        if workload == "affine":
            line["cpu_baseline_gotoh"] = cpu_measure(workload, os.cpu_count() or 1, 1, gotoh=True)
    return line


def main() -> None:
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    if args.selftest_ranks:
        selftest_ranks(args)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch

    ranks_env_local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(ranks_env_local)
    # Clock samples from now on; the line keeps those inside the headline's timed region.
    clocks = Clocks(ranks_env_local).start()
    ranks = Ranks("nccl")
    import dinara_align as da
    from dinara_align import _native as native

    lib = native.lib()
    declare(lib, native)
    handle = native.context(ranks.local_rank)
    peaks = int32_peaks(handle, lib)
    ctx = {"da": da, "native": native, "lib": lib, "handle": handle, "ranks": ranks, "peaks": peaks,
           "e2e": not args.no_e2e, "parity": not args.no_parity, "predictor": args.predictor,
           "tuning": args.tuning, "arms": args.arms}
    head = run_workload(ctx, args.workload, args.pairs, args.steps, args.warmup, not args.no_cpu)
    begin, end = head.pop("timed_region")
    sections = {}
    if ranks.world == 1 and not args.no_sections:
        for name in ("affine", "local", "unit250"):
            if name == args.workload:
                continue
            section = run_workload(ctx, name, 0, max(1, min(args.steps, 5)), 2, not args.no_cpu)
            section.pop("timed_region", None)
            sections[name] = section
        sections["serving"] = serving_section(da)
    clocks.stop()
    if ranks.rank == 0:
        line = {"metric": "pairs/s", "value": head.pop("value"), "unit": "pairs/s", "n_gpus": ranks.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": head.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
                # Unit cost: 64-bit Myers/Hyyro words. Scores: 16-bit halves where a pair's values provably
                # fit (exact), 32 bits otherwise.
                "dtype": "u64" if args.workload in ("uneven", "unit250") else "int16x2+int32",
                "config": head.pop("config"), "gpu_launches": head.pop("gpu_launches"),
                "clocks": clocks.summary(begin, end)}
        line.update(head)
        line["int32_peaks_instr_per_s"] = peaks
        line["sections"] = sections
        print(json.dumps(line))
    ranks.close()


if __name__ == "__main__":
    main()
