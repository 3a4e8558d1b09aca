"""Multi-GPU plumbing: shots are independent, so each rank runs its own shots and
the stacked gradient and the per-shot misfits are summed with one all-reduce each
(the reference's allreduce_array of the gradient and the misfit,
src/inverse/2d/module_gradient.f90:398,411-413), in FP64. No collective runs
inside the time loop."""
from __future__ import annotations

from typing import List, Sequence, Tuple


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


class ShotSharding:
    """The shots of one rank out of a shot set, and the reductions that close one
    gradient evaluation over all ranks.

    Every rank must call `reduce` (and `any_rank`) the same number of times in
    the same order: they are collectives."""

    def __init__(self, shots: Sequence, rank: int, world: int, group=None):
        self.nshots = len(shots)
        self.rank, self.world, self.group = rank, world, group
        self.mine = shard_shots(shots, rank, world)

    def local(self, shots: Sequence) -> list:
        return [shots[i] for i in self.mine]

    def reduce(self, grad, misfit_local) -> Tuple["object", "object"]:
        """FP64 sums over ranks: the gradient (any float dtype; returned as a new
        float64 tensor) and the per-shot misfits of this rank's shots, placed at
        their index in the whole shot set (float64, length nshots)."""
        import torch
        g = grad.to(torch.float64)
        m = torch.zeros(self.nshots, dtype=torch.float64, device=grad.device)
        if len(self.mine):
            m[torch.as_tensor(self.mine, device=grad.device)] = misfit_local.to(torch.float64)
        allreduce_sum(g, self.group)
        allreduce_sum(m, self.group)
        return g, m

    def any_rank(self, flag: bool, device="cpu") -> bool:
        """True on every rank if `flag` is true on any rank (MAX all-reduce)."""
        import torch
        import torch.distributed as dist
        t = torch.tensor([1 if flag else 0], dtype=torch.int32, device=device)
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(self.group) > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return bool(t.item())
