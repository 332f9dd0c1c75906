"""bench.py's multi-GPU launcher, on CPU (no GPU needed).

``bench.py --gpus 2`` without a torchrun environment relaunches itself as
two ranks under torch.distributed.run; with ``--plan-only`` each rank joins
a gloo group, takes the timed region's collectives (barrier, maximum of the
elapsed times) and reports the frames it would process.  The ranks must
process distinct frames (seed 2 + rank), and the maximum must agree.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_two_ranks_process_distinct_frames():
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                          "--plan-only"], capture_output=True, text=True, timeout=300, env=env,
                         cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [line for line in res.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, res.stdout  # rank 0 alone prints
    report = json.loads(lines[0])
    assert report["world"] == 2
    assert [p["rank"] for p in report["plans"]] == [0, 1]
    assert [p["frame_seeds"] for p in report["plans"]] == [[2], [3]]
    assert report["max_over_ranks"] == 1.5


def test_launch_command_uses_one_process_per_gpu():
    sys.path.insert(0, ROOT)
    import bench

    cmd = bench.launch_command(8, ["--steps", "5"], 29500)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=8" in cmd and "--master-addr=127.0.0.1" in cmd
    assert cmd[-2:] == ["--steps", "5"]
