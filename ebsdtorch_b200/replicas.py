"""Multi-GPU use of the single-GPU indexer: one process per GPU.

Dictionary indexing shards naturally by pattern: every pattern is matched
against the whole dictionary independently. With N ranks each rank indexes a
contiguous shard of the scan (or, in the benchmark, its own full map), so the
data path needs no collective. The only cross-rank steps are host-side
plumbing: timing as the maximum over ranks, and (optionally) gathering the
per-shard results to every rank once at the end.
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch


def shard_range(n_items: int, rank: int, world_size: int) -> Tuple[int, int]:
    """Contiguous [start, stop) of rank `rank`; shard sizes differ by at most one."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"invalid rank {rank} for world size {world_size}")
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. elapsed seconds) over all ranks."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_shards(local: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """All-gather per-rank row shards (as produced with shard_range) into the
    full (n_total, ...) tensor on every rank."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return local
    world = dist.get_world_size(group)
    sizes = [shard_range(n_total, r, world) for r in range(world)]
    longest = max(b - a for a, b in sizes)
    pad = torch.zeros((longest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[: b - a] for p, (a, b) in zip(parts, sizes)], dim=0)


def index_shard(index_fn, experiment_patterns, rank: Optional[int] = None, world_size: Optional[int] = None,
                gather: bool = True, **kwargs):
    """Run a drop-in indexing function (dictionary_index_orientations or
    pca_dictionary_index_orientations) on this rank's shard of the patterns.
    With gather=True the final orientations / metrics / phases of all shards
    are all-gathered into experiment_patterns on every rank; the per-shard
    raw top-k results stay local. Returns (start, stop) of the shard."""
    import torch.distributed as dist

    from .ebsd.experiment_pats import ExperimentPatterns

    if rank is None:
        rank = dist.get_rank() if dist.is_initialized() else 0
    if world_size is None:
        world_size = dist.get_world_size() if dist.is_initialized() else 1
    n = experiment_patterns.n_patterns
    a, b = shard_range(n, rank, world_size)
    part = ExperimentPatterns(experiment_patterns.patterns[a:b])
    index_fn(experiment_patterns=part, **kwargs)
    experiment_patterns.raw_indexing_results = part.raw_indexing_results
    experiment_patterns.shard = (a, b)
    if gather and world_size > 1:
        experiment_patterns.orientations = gather_shards(part.orientations.contiguous(), n)
        experiment_patterns.best_metrics = gather_shards(part.best_metrics.float().contiguous(), n)
        experiment_patterns.phases = gather_shards(part.phases.contiguous(), n)
    else:
        experiment_patterns.orientations = part.orientations
        experiment_patterns.best_metrics = part.best_metrics
        experiment_patterns.phases = part.phases
    return a, b
