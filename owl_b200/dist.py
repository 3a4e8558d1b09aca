"""Multi-GPU plumbing: shots are independent, so each rank runs its own shots and
the stacked gradient is summed with one all-reduce (the reference's
allreduce_array of the gradient and misfit, src/inverse/2d/module_gradient.f90:398,411-413).
No collective runs inside the time loop."""
from __future__ import annotations

from typing import List, Sequence


def shard_shots(shots: Sequence, rank: int, world: int) -> List[int]:
    """Indices of the shots of `rank`: greedy balance of the trace counts
    (largest first, each to the least loaded rank), order kept within a rank."""
    if world <= 1:
        return list(range(len(shots)))
    load = [0] * world
    owner = [0] * len(shots)
    for i in sorted(range(len(shots)), key=lambda i: -max(1, len(shots[i].receivers))):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += max(1, len(shots[i].receivers))
    return [i for i in range(len(shots)) if owner[i] == rank]


def allreduce_sum(tensor, group=None):
    """In-place sum over ranks (NCCL for CUDA tensors, gloo for CPU tensors)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor
