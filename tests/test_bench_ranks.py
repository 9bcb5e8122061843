"""bench.py's multi-GPU launch on the CPU: `--gpus 2` outside torchrun starts two ranks through torchrun
(127.0.0.1), each takes its place from the environment, and rank 0 alone prints the max over ranks of
their timed regions (the GPU arm's protocol, here over gloo with host loops standing in for device work)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_two_ranks_one_line():
    run = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--selftest-ranks",
                          "--steps", "1"], capture_output=True, text=True, timeout=300,
                         env={k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")})
    assert run.returncode == 0, run.stderr[-2000:]
    lines = [json.loads(line) for line in run.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2
    # Rank 1 loops twice as long as rank 0: the printed time is the slower rank's.
    assert lines[0]["slowest_s"] >= lines[0]["own_s"]
