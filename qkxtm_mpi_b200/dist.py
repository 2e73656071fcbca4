"""Multi-GPU plumbing of the benchmark: one process per GPU, sources sharded by
rank (each rank solves its own point sources on its own replica of the gauge
field: independent work, no data-path collective), timings reduced with the
max over ranks.  torch.distributed is used only for the barrier and that one
scalar reduction (NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations

import datetime
import os


def env_rank() -> tuple[int, int, int]:
    """(RANK, WORLD_SIZE, LOCAL_RANK) from the launcher's environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def source_timeslice(rank: int, Lt: int) -> int:
    """Time slice of rank's point sources (distinct for up to Lt/2 ranks)."""
    return (2 * rank) % Lt


def init(backend: str, local_rank: int | None = None, timeout_s: int = 300) -> None:
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl" and local_rank is not None:
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float) -> float:
    """Max of x over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
