"""Sequence sharding for one process per GPU.

The path shards by independent sequence: a depth map's SGM recurrences run across the whole
image, so one map stays on one GPU, and a batch of sequences is split into per-GPU groups.  No
collective touches the data path; ranks exchange only their timings and result statistics.
"""
from __future__ import annotations


def sequence_weight(cfg: dict, num_sources: int) -> int:
    """Work of one keyframe: voxels x sources (the cost volume dominates)."""
    return int(cfg["width"]) * int(cfg["height"]) * int(cfg["num_planes"]) * int(num_sources)


def shard_sequences(configs, world: int, num_sources: int):
    """Split sequence indices into `world` groups of balanced V*S (longest job first onto the
    least-loaded rank; deterministic, ties to the lower index and rank).  Returns a list of index
    lists, one per rank, each in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(configs)), key=lambda i: (-sequence_weight(configs[i], num_sources), i))
    load = [0] * world
    groups = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        groups[r].append(i)
        load[r] += sequence_weight(configs[i], num_sources)
    return [sorted(g) for g in groups]


def gather_stats(values, group=None):
    """All-gather of a small list of floats per rank (host tensors over gloo, device tensors over
    nccl); returns a list with one list per rank."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(list(values), dtype=torch.float64, device=dev)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [o.cpu().tolist() for o in out]
