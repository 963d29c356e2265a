"""Multi-process plumbing for the chemistry step (one process per GPU).

Cells are independent, so ranks never exchange field data: each rank steps
its own cells and the only collectives are the timing reduction (the job's
time is the slowest rank's) and the barriers around the timed region.
`bench.py` gives every rank a full field (weak scaling); `row_block` splits
one field's rows among ranks when a fixed field is shared (strong scaling).
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 600.0) -> None:
    """Process group from the launcher's environment (MASTER_ADDR/PORT)."""
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def row_block(n_rows: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous rows [start, stop) of `rank`; block sizes differ by at most
    one and the blocks cover 0..n_rows-1 exactly once in rank order."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank out of range")
    base, extra = divmod(n_rows, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
