"""Data-parallel replicas over several GPUs (one process per GPU).

Segments are independent (every sky depends on its own segment's spectra
only), so the multi-GPU form of the batched integrator is a set of replicas:
each rank integrates a contiguous shard of the segments with its own plan on
its own GPU, with no collective on the data path.  Two collectives remain,
both outside it: the maximum of the ranks' elapsed times (whole-job
throughput is timed by the slowest rank) and, optionally, gathering the
skies on one rank.  These helpers hold that host-side logic so that it runs
the same under NCCL on GPUs and under gloo on CPU tensors.
"""
from __future__ import annotations


def shard_range(n_seg: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous shard of n_seg segments: sizes
    differ by at most one, lower ranks take the extra segments."""
    if world <= 0 or not 0 <= rank < world or n_seg < 0:
        raise ValueError(f"bad shard request: {n_seg} segments, rank {rank} of {world}")
    q, r = divmod(n_seg, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank float over the default process group (the
    value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, elapsed_ms: float, device=None) -> tuple[float, float]:
    """(units/s of the whole job, the slowest rank's elapsed ms): every rank
    processed units_per_rank units per step."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    slowest = max_over_ranks(elapsed_ms, device)
    return world * units_per_rank * steps / (slowest / 1e3), slowest


def gather_skies(local, n_seg: int, dst: int = 0):
    """Gather every rank's shard of skies ([shard][nq] tensors, shards as
    shard_range cuts n_seg) into the full [n_seg][nq] tensor on rank dst
    (None elsewhere).  Shards are padded to a common length for the
    collective and trimmed afterwards."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    world, rank = dist.get_world_size(), dist.get_rank()
    start, stop = shard_range(n_seg, rank, world)
    if local.shape[0] != stop - start:
        raise ValueError(f"rank {rank} holds {local.shape[0]} skies, its shard has {stop - start}")
    longest = shard_range(n_seg, 0, world)[1]
    pad = torch.zeros((longest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    # complex skies travel as their real view; all_gather (gloo and NCCL)
    send = torch.view_as_real(pad) if pad.is_complex() else pad
    allp = [torch.empty_like(send) for _ in range(world)]
    dist.all_gather(allp, send)
    if rank != dst:
        return None
    out = []
    for r in range(world):
        a, b = shard_range(n_seg, r, world)
        part = torch.view_as_complex(allp[r]) if pad.is_complex() else allp[r]
        out.append(part[: b - a])
    return torch.cat(out, 0)
