"""The multi-GPU replica logic on CPU: two gloo ranks (no GPU).

Frames shard round-robin with no data-path collective; the measurement's
collectives (barrier, maximum of elapsed times, sum of units) agree on every
rank; a rank's frames are disjoint from the other's and together cover the
workload.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from fauxice_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import json

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        frames = list(range(16))
        mine = replicas.shard(frames, rank, world)
        replicas.barrier()
        elapsed = 0.5 + rank  # rank 1 is the slowest
        slowest = replicas.max_over_ranks(elapsed)
        units = float(len(mine))
        total = replicas.sum_over_ranks(units)
        rate = replicas.throughput(units, elapsed)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as handle:
            json.dump({"mine": mine, "slowest": slowest, "total": total, "rate": rate}, handle)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import json

    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    results = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert results[0]["mine"] == list(range(0, 16, 2))
    assert results[1]["mine"] == list(range(1, 16, 2))
    assert sorted(results[0]["mine"] + results[1]["mine"]) == list(range(16))
    for r in results:
        assert r["slowest"] == 1.5
        assert r["total"] == 16.0
        assert r["rate"] == pytest.approx(16.0 / 1.5)


def test_single_process_needs_no_group():
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
    assert replicas.max_over_ranks(2.5) == 2.5
    assert replicas.throughput(10.0, 2.0) == 5.0
    with pytest.raises(ValueError):
        replicas.shard([1], 2, 2)
