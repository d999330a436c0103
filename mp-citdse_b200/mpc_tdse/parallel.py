"""Multi-GPU use of the propagation: pulses are independent, so a batch is
partitioned across ranks (one process per GPU) with no collective on the
data path; only the per-pulse results are gathered at the end, and timings
are reduced as the maximum over ranks.

The functions take an initialised torch.distributed process group (NCCL on
GPUs; gloo works the same way on CPU, which is how the tests run them).
"""
from __future__ import annotations

import numpy as np


def shard(n_items, rank, world):
    """Contiguous, balanced [start, stop) of n_items for this rank."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value, dist, device="cpu"):
    """Slowest rank's value (the time a multi-GPU step takes)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device="cpu"):
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_rows(local_rows, n_total, rank, world, dist, device="cpu"):
    """Reassembles a [n_total, ...] float64/complex128 array whose rows were
    computed shard by shard (`shard`): every rank gets the whole array."""
    import torch

    a = np.ascontiguousarray(local_rows)
    cplx = np.iscomplexobj(a)
    if cplx:
        a = a.view(np.float64)
    row_shape = a.shape[1:]
    width = int(np.prod(row_shape)) if row_shape else 1
    start, stop = shard(n_total, rank, world)
    if a.shape[0] != stop - start:
        raise ValueError("local rows do not match this rank's shard")
    full = torch.zeros((n_total, width), dtype=torch.float64, device=device)
    full[start:stop] = torch.from_numpy(a.reshape(stop - start, width)).to(device)
    dist.all_reduce(full, op=dist.ReduceOp.SUM)  # disjoint rows: a sum is a gather
    out = full.cpu().numpy().reshape((n_total,) + row_shape)
    return out.view(np.complex128) if cplx else out


def propagate_sharded(run_shard, items, rank, world, dist, device="cpu"):
    """Runs `run_shard(items[start:stop]) -> (rows, work_units, seconds)` on
    this rank's shard; returns (all rows, total units, slowest seconds)."""
    start, stop = shard(len(items), rank, world)
    rows, units, sec = run_shard(items[start:stop])
    allrows = gather_rows(rows, len(items), rank, world, dist, device)
    return allrows, sum_over_ranks(units, dist, device), max_over_ranks(sec, dist, device)
