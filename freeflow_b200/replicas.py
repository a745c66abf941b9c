"""Multi-GPU runs of the fluid step: one independent replica per GPU.

One grid of the reference's configurations fits one GPU, and the step has no
exchange between grids, so N GPUs run N replicas. There is no collective on
the data path. A collective is used only for the timing:

- every rank times its own steps with CUDA events;
- the job's time is the maximum over ranks;
- the job's rate is the units all ranks processed divided by that time (weak scaling).

These helpers are the whole multi-rank protocol of ``bench.py``. They work
with any ``torch.distributed`` backend: NCCL on GPUs, gloo in the CPU tests.
"""
from __future__ import annotations

import os
from datetime import timedelta


def env_ranks() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment; 1 process by default."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 300.0, device=None) -> None:
    """Joins the process group when there is more than one rank; the short timeout makes ranks
    that wait for a failed peer end with an error instead of hanging."""
    import torch.distributed as dist

    _, world, _ = env_ranks()
    if world > 1 and not dist.is_initialized():
        kw = {"device_id": device} if device is not None else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of `value` over all ranks (the value itself for one process)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, seconds_max: float, world: int) -> float:
    """Units processed by all ranks per second of the slowest rank."""
    return world * units_per_rank / seconds_max


def shutdown() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
