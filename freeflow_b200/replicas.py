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
import socket
import subprocess
import sys
import time
from datetime import timedelta


def env_ranks() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment; 1 process by default."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def launch_local_ranks(argv: list[str], n: int, poll_s: float = 0.2) -> int:
    """Runs ``python argv...`` as `n` ranks on this node, as torchrun would: rank r gets
    RANK = LOCAL_RANK = r, WORLD_SIZE = n and a rendezvous on 127.0.0.1 at a free port.
    The ranks share this process's stdout and stderr.  If a rank fails, the others are
    terminated (by their own process handles).  Returns 0, or the first non-zero exit code."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, *argv], env=env))
    rc = 0
    while any(p.poll() is None for p in procs):
        failed = [p.returncode for p in procs if p.returncode not in (None, 0)]
        if failed:
            rc = failed[0]
            for p in procs:
                if p.poll() is None:
                    p.terminate()
            break
        time.sleep(poll_s)
    for p in procs:
        try:
            p.wait(timeout=60)
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
        if rc == 0 and p.returncode:
            rc = p.returncode
    return rc


def all_gather_objects(obj) -> list:
    """Every rank's `obj`, in rank order (just [obj] for one process)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


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
