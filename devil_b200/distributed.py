"""Gene sharding across ranks for devil's NB GLM path.

Genes are independent through the whole fit (IRLS, theta, bread, meat), so
each rank fits a contiguous range of genes with no exchange; the only
collective is the all-gather of the per-gene p-values, because the
Benjamini-Hochberg step (stats::p.adjust at R/test.R:127) ranks all genes
together.  With NCCL the gather runs over NVLink; the host logic is the same
for any torch.distributed backend (tests run it with gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_ranges(rowptr, world: int, n_cells: int):
    """Contiguous gene ranges balanced by per-gene cost (n dense cell terms
    plus the gene's nonzeros).  Returns a list of (begin, end)."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    G = len(rowptr) - 1
    cost = np.cumsum(np.diff(rowptr) + int(n_cells), dtype=np.float64)
    total = cost[-1] if G else 0.0
    bounds = [0]
    for r in range(1, world):
        bounds.append(int(np.searchsorted(cost, total * r / world, side="left")))
    bounds.append(G)
    bounds = np.maximum.accumulate(np.asarray(bounds))
    return [(int(bounds[r]), int(bounds[r + 1])) for r in range(world)]


def gather_vectors(local, group=None):
    """All-gather variable-length float64 vectors (rank order)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    t = torch.as_tensor(np.asarray(local, dtype=np.float64), device=dev)
    n = torch.tensor([t.numel()], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    mx = max(sizes) if sizes else 0
    pad = torch.full((mx,), float("nan"), dtype=torch.float64, device=dev)
    pad[: t.numel()] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return np.concatenate([p[:s].cpu().numpy() for p, s in zip(parts, sizes)])


def global_adjust(local_p, method="BH", group=None, adjust=None):
    """p.adjust over the p-values of every rank; returns this rank's slice.
    ``adjust`` defaults to the device implementation (devil_b200.p_adjust)."""
    import torch.distributed as dist

    if adjust is None:
        from .api import p_adjust as adjust
    full = gather_vectors(local_p, group)
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    sizes = gather_vectors(np.array([float(len(local_p))]), group).astype(np.int64)
    start = int(sizes[:rank].sum())
    adj = adjust(full, method)
    assert len(full) == int(sizes.sum()) and world == len(sizes)
    return adj[start:start + len(local_p)]


def global_adjust_tensor(local, method, adjust, group=None, sizes=None):
    """p.adjust over every rank's p-values, kept in torch tensors on the
    device of ``local`` (with NCCL: the GPU, so the gathered vector never
    crosses to the host).

    ``local`` is this rank's 1-D float64 tensor of p-values (ranks may hold
    different numbers of genes); ``adjust(full, method)`` returns the
    adjustment of the gathered vector in rank order (NaN = NA, not counted);
    ``sizes`` (the per-rank lengths, when already known) saves the exchange
    of the lengths.  Returns this rank's slice of the adjusted vector."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if sizes is None:
        n = torch.tensor([local.numel()], dtype=torch.int64, device=local.device)
        parts = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(parts, n, group=group)
        sizes = [int(s.item()) for s in parts]
    mx = max(sizes)
    pad = torch.full((mx,), float("nan"), dtype=torch.float64, device=local.device)
    pad[: local.numel()] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    full = torch.cat([parts[r][: sizes[r]] for r in range(world)])
    adj = adjust(full, method)
    start = int(sum(sizes[:rank]))
    return adj[start:start + local.numel()]
