"""Query sharding for one process per GPU.

Given the trained reference, every query cell is annotated independently (the score step, its
per-label quantiles and the fine-tune rounds only read that cell's row and the reference), so N
ranks each annotate one contiguous block of query rows and exchange nothing on the data path.
`gather_labels` collects the per-rank label arrays once at the end (all_gather over the process
group: NCCL between GPUs, gloo on CPU).  Each rank trains its own copy of the reference, as the
reference's single-process pipeline would (src/pipeline.cpp of STOmics/cusingler).
"""

from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

from .synth import CSR


def row_ranges(indptr: np.ndarray, world_size: int) -> list[tuple[int, int]]:
    """Contiguous row blocks [lo, hi) for `world_size` ranks, balanced by stored entries (the
    rank kernel's and the fine-tune's work grow with them).  Blocks may be empty when there are
    fewer rows than ranks; together they cover every row once, in order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    indptr = np.asarray(indptr)
    n_rows = len(indptr) - 1
    nnz = int(indptr[-1]) if n_rows > 0 else 0
    bounds = [0]
    for r in range(1, world_size):
        if nnz > 0:
            target = nnz * r / world_size
            lo = int(np.searchsorted(indptr, target, side="left"))
        else:
            lo = (n_rows * r) // world_size
        bounds.append(min(max(lo, bounds[-1]), n_rows))
    bounds.append(n_rows)
    return [(bounds[r], bounds[r + 1]) for r in range(world_size)]


def shard_of(csr: CSR, world_size: int, rank: int) -> tuple[int, int, CSR]:
    """(lo, hi, rows lo..hi-1 of `csr`) for `rank`; the slice shares the arrays of `csr`."""
    lo, hi = row_ranges(csr.indptr, world_size)[rank]
    return lo, hi, csr.rows(lo, hi)


def gather_labels(parts: Sequence[np.ndarray], group=None) -> list[np.ndarray]:
    """All-gather each of this rank's int32 label arrays (one entry per row of its shard, ranks in
    order) and return the concatenations, identical on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    n_local = torch.tensor([len(parts[0]) if parts else 0], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(max(sizes), 1)
    out = []
    for a in parts:
        buf = torch.zeros(cap, dtype=torch.int32, device=dev)
        buf[: len(a)] = torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev)
        got = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(got, buf, group=group)
        out.append(np.concatenate([g[: n].cpu().numpy() for g, n in zip(got, sizes)]).astype(np.int32))
    return out


def annotate_sharded(annotate: Callable[[CSR], Sequence[np.ndarray]], qry: CSR, group=None) -> list[np.ndarray]:
    """Annotate this rank's block of `qry` with `annotate` (e.g. ``Annotator.annotate``, which
    returns first and final labels) and gather the full label arrays on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    _, _, mine = shard_of(qry, world, rank)
    parts = annotate(mine) if mine.n_rows > 0 else None
    if parts is None:
        parts = [np.zeros(0, np.int32), np.zeros(0, np.int32)]
    return gather_labels([np.asarray(p, np.int32) for p in parts[:2]], group=group)
