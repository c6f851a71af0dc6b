"""Ray data parallelism over ranks (one process per GPU, torch.distributed).

Rays are independent, so a training step shards its rays over the ranks: each
rank projects and differentiates its own rays against replicated factors and
decoder, and the gradients are averaged across ranks once per step (the only
exchange; NCCL over NVLink on GPUs, gloo in the CPU tests). Node-error sums
(FP64) are summed across ranks the same way before the structure
optimisation.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_permutation(num_rays: int, batch: int, rank: int, world: int, epoch: int, seed: int = 1004):
    """This rank's ray indices for each step of an epoch: one global
    permutation (same seed on every rank) cut into steps of world * batch
    rays, of which this rank takes the rank-th slice. Ranks never share a
    ray within an epoch."""
    g = torch.Generator().manual_seed(seed + epoch)
    perm = torch.randperm(num_rays, generator=g)
    per_step = world * batch
    steps = num_rays // per_step
    return [perm[s * per_step + rank * batch: s * per_step + (rank + 1) * batch] for s in range(steps)]


def allreduce_gradients(params, world: int):
    """Average the .grad of every parameter over the ranks (in place)."""
    if world <= 1:
        return
    for p in params:
        if p.grad is not None:
            dist.all_reduce(p.grad, op=dist.ReduceOp.SUM)
            p.grad.div_(world)


def allreduce_node_error(loss_sum: torch.Tensor, weight_sum: torch.Tensor, world: int):
    """Sum the per-node FP64 loss and weight sums over the ranks (in place)."""
    if world <= 1:
        return
    dist.all_reduce(loss_sum, op=dist.ReduceOp.SUM)
    dist.all_reduce(weight_sum, op=dist.ReduceOp.SUM)
