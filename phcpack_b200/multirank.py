"""One process per GPU: the host-side pieces of running the path on N ranks.

The work units (systems, least-squares instances, paths) are independent, so
N ranks split them into contiguous ranges and exchange nothing on the data
path; the only collectives are the barrier around the timed region, the
maximum of the per-rank times and, where a caller wants every result on one
rank, a gather of the per-unit outputs at the end.  The functions take a
torch.distributed module (NCCL on GPUs, gloo on CPUs) or None for one rank.
"""
from __future__ import annotations

import numpy as np


def shard(n_units: int, rank: int, world: int) -> range:
    """The contiguous range of units of this rank: sizes differ by at most
    one, lower ranks take the larger shares."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _device(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value: float, dist=None) -> float:
    """The maximum of a per-rank value (a timed region) over all ranks."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(rows: np.ndarray, n_units: int, dist=None, dst: int = 0):
    """Gather per-unit result rows (shape (units of this rank, ...)) of every
    rank's shard into one array of n_units rows on rank dst, in unit order;
    other ranks get None."""
    if dist is None:
        return rows
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    width = int(np.prod(rows.shape[1:])) if rows.ndim > 1 else 1
    maxrows = max(len(shard(n_units, r, world)) for r in range(world))
    dev = _device(dist)
    buf = torch.zeros((maxrows, width), dtype=torch.float64, device=dev)
    mine = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.float64).reshape(len(rows), width))
    buf[:len(rows)] = mine.to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst)
    if rank != dst:
        return None
    out = np.concatenate([parts[r][:len(shard(n_units, r, world))].cpu().numpy() for r in range(world)])
    return out.reshape((n_units,) + rows.shape[1:]).astype(rows.dtype)
