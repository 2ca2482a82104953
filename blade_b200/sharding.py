"""Frequency sharding of one block across ranks (one process per GPU).

The beamform -> channelize -> detect path is independent per coarse channel:
every output channel f*R + k depends only on input channel f.  A block of F
channels is therefore split into contiguous channel ranges, one per rank, with
no exchange step on the data path; the only collectives are the optional gather
of the detector products to one rank and the max over ranks of a timing.  With
NCCL on GPUs (or gloo on CPUs) this is plain ``torch.distributed``.

Shapes follow the reference layouts: voltages [A, F, T, P] (frequency axis 1),
phasors [B, A, F, 1, P] (axis 2), detector products [B or A, F*R, T', O] (axis 1,
R output channels per input channel).
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch


def channel_range(F: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous [f0, f1) of rank `rank`: the first F % world ranks take one extra channel."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    base, extra = divmod(F, world)
    f0 = rank * base + min(rank, extra)
    return f0, f0 + base + (1 if rank < extra else 0)


def shard(t: torch.Tensor, axis: int, world: int, rank: int) -> torch.Tensor:
    """The rank's channel slice of `t` along its frequency axis (a view)."""
    f0, f1 = channel_range(t.shape[axis], world, rank)
    return t.narrow(axis, f0, f1 - f0)


def shard_block(voltages: torch.Tensor, phasors: torch.Tensor, world: int, rank: int):
    """(voltages [A, F, T, P], phasors [B, A, F, 1, P]) -> the rank's channel slices, contiguous."""
    return (shard(voltages, 1, world, rank).contiguous(), shard(phasors, 2, world, rank).contiguous())


def gather_channels(local: torch.Tensor, F: int, rate: int = 1, axis: int = 1, group=None,
                    dst: Optional[int] = 0) -> Optional[torch.Tensor]:
    """Concatenate every rank's products along `axis` in rank (channel) order.

    `local` holds the rank's channels (rate output channels per input channel).
    Shards of unequal size are padded to the largest for the collective and
    trimmed after.  dst = None gathers on every rank; otherwise only rank `dst`
    gets the result (the others get None)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = [(channel_range(F, world, r)[1] - channel_range(F, world, r)[0]) * rate for r in range(world)]
    if local.shape[axis] != sizes[rank]:
        raise ValueError(f"rank {rank} holds {local.shape[axis]} channels, expected {sizes[rank]}")
    width = max(sizes)
    pad = list(local.shape)
    pad[axis] = width
    buf = local.new_zeros(pad)
    buf.narrow(axis, 0, sizes[rank]).copy_(local)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    if dst is not None and rank != dst:
        return None
    return torch.cat([p.narrow(axis, 0, n) for p, n in zip(parts, sizes)], dim=axis)


def max_over_ranks(value: float, device: str = "cuda", group=None) -> float:
    """Largest `value` over the ranks (whole-job time is the slowest rank's)."""
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
