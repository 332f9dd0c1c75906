"""Several GPUs: one process per GPU, each processing its own frames.

Frames are independent jobs (own prelude, own RNG chain), so the path shards
at frame granularity with no collective on the data path: rank r of N takes
frames r, r + N, r + 2N, ...  The only collectives are the measurement's:
barriers around the timed region and the maximum of the ranks' elapsed
times.  They take whatever backend the process group has (NCCL on GPUs,
gloo on CPU for tests).
"""

from __future__ import annotations

from typing import Sequence, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> list[T]:
    """The items rank ``rank`` of ``world`` processes (round-robin)."""

    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(items[rank::world])


def _device_for_backend():
    import torch
    import torch.distributed as dist

    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """The maximum of ``value`` over all ranks (the value itself alone)."""

    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    """The sum of ``value`` over all ranks (e.g. megapixels processed)."""

    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def throughput(units_per_rank: float, elapsed_per_rank_s: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""

    total = sum_over_ranks(units_per_rank)
    slowest = max_over_ranks(elapsed_per_rank_s)
    return total / slowest if slowest > 0 else float("inf")
