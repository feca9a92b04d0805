"""Multi-GPU harness for independent replicas (one process per GPU).

The filter -> group_by -> aggregate path runs on one GPU per query; with N GPUs each rank runs
its own table (weak scaling) and the only cross-rank traffic is the timing reduction below, done
on the host-side process group (NCCL on GPUs, gloo on CPU tests). No data-path collective.
"""

from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment (1 process when absent)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def reduce_step_stats(ms: float, rows: int, device=None) -> tuple[float, int]:
    """Max step time and total rows over ranks; identity in a single process."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return ms, rows
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    r = torch.tensor([rows], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(r, op=dist.ReduceOp.SUM)
    return float(t.item()), int(r.item())


def barrier(device=None) -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if device is not None and str(device).startswith("cuda"):
            dist.barrier(device_ids=[int(str(device).split(":")[1]) if ":" in str(device) else 0])
        else:
            dist.barrier()
