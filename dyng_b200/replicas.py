"""Replicas and graph placement across GPUs (one process per GPU).

One sssp update does not shard across GPUs (every near-far step needs a global threshold and an
exchange of improved words; pointer jumping chases parents across any partition), so the unit
that spreads over GPUs is a whole graph: the benchmark runs one independent replica per GPU, and
a serving process places whole graphs (with their trees) on GPUs.  No data-path collective is
involved; torch.distributed carries only the barrier and the max-over-ranks time.
"""
from __future__ import annotations


def max_over_ranks(value: float) -> float:
    """The maximum of `value` over all ranks (the value itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    if device == "cuda":
        device = f"cuda:{torch.cuda.current_device()}"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, max_ms: float, world: int) -> float:
    """Units per second of the whole job: every rank processed `units_per_rank` units and the
    slowest took `max_ms` (weak scaling: per-rank work fixed as ranks are added)."""
    if max_ms <= 0:
        raise ValueError("whole_job_rate: the time must be positive")
    return world * units_per_rank / (max_ms / 1000.0)


def place_graphs(device_bytes, world: int, capacity_bytes: float | None = None):
    """Rank of each graph: largest first onto the least-loaded rank (ties to the lowest rank),
    so every rank computes the same placement from the same list.  With `capacity_bytes`, a
    graph that fits nowhere raises MemoryError."""
    if world < 1:
        raise ValueError("place_graphs: world must be >= 1")
    load = [0.0] * world
    rank = [0] * len(device_bytes)
    for i in sorted(range(len(device_bytes)), key=lambda j: (-device_bytes[j], j)):
        r = min(range(world), key=lambda k: (load[k], k))
        if capacity_bytes is not None and load[r] + device_bytes[i] > capacity_bytes:
            raise MemoryError(f"place_graphs: graph {i} ({device_bytes[i]} bytes) fits on no GPU")
        load[r] += device_bytes[i]
        rank[i] = r
    return rank
