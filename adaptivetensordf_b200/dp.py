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


def allreduce_gradients(params, world: int, bucket_bytes: int = 1 << 20):
    """Average the .grad of every parameter over the ranks (in place). Each
    gradient of at least bucket_bytes is reduced on its own; the smaller ones
    (decoder weights and biases, lines) travel together in one flat buffer per
    dtype, one collective instead of one each (their cost is latency, not
    bandwidth). Every rank issues the same collectives in the same order."""
    if world <= 1:
        return
    grads = [p.grad for p in params if p.grad is not None]
    small = {}
    for g in grads:
        if g.numel() * g.element_size() >= bucket_bytes:
            dist.all_reduce(g, op=dist.ReduceOp.SUM)
            g.div_(world)
        else:
            small.setdefault((g.dtype, g.device), []).append(g)
    for group in small.values():
        flat = torch.cat([g.reshape(-1) for g in group])
        dist.all_reduce(flat, op=dist.ReduceOp.SUM)
        flat.div_(world)
        off = 0
        for g in group:
            n = g.numel()
            g.copy_(flat[off:off + n].view(g.shape))
            off += n


def allreduce_node_error(loss_sum: torch.Tensor, weight_sum: torch.Tensor, world: int):
    """Sum the per-node FP64 loss and weight sums over the ranks (in place)."""
    if world <= 1:
        return
    dist.all_reduce(loss_sum, op=dist.ReduceOp.SUM)
    dist.all_reduce(weight_sum, op=dist.ReduceOp.SUM)
