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


# ----------------------------------------------------------------------------
# sharded optimizer step
# ----------------------------------------------------------------------------
def storage_flat(t: torch.Tensor) -> torch.Tensor:
    """A 1-D view of a dense tensor in its storage order (row-major, or
    NHWC for a channels-last 4-D tensor such as the factor planes)."""
    if t.is_contiguous():
        return t.view(-1)
    if t.dim() == 4 and t.is_contiguous(memory_format=torch.channels_last):
        return t.permute(0, 2, 3, 1).reshape(-1)
    raise ValueError("storage_flat: dense row-major or channels-last tensors only")


def adam_shard_torch(param, grad, exp_avg, exp_avg_sq, segments, step):
    """torch.optim.Adam's update (no amsgrad) on a flat shard, in place:
    segments are (start, end, lr, beta1, beta2, eps, weight_decay) ranges of
    the shard with their parameter's hyper-parameters. The plain torch form
    of the shard update (the CPU tests); on the GPU ShardedAdam runs
    atdf_adam_step_multi on the same ranges."""
    for a, b, lr, b1, b2, eps, wd in segments:
        p, g, m, v = param[a:b], grad[a:b], exp_avg[a:b], exp_avg_sq[a:b]
        if wd:
            g = g + wd * p
        m.mul_(b1).add_(g, alpha=1 - b1)
        v.mul_(b2).addcmul_(g, g, value=1 - b2)
        bc1 = 1 - b1 ** step
        bc2 = 1 - b2 ** step
        denom = (v.sqrt() / (bc2 ** 0.5)).add_(eps)
        p.addcdiv_(m, denom, value=-lr / bc1)


class _Domain:
    """Parameters sharded together: one flat storage-order layout padded to
    a multiple of the ranks, this rank's shard of FP32 masters and Adam
    moments, and the dtype the updated values are gathered in."""

    def __init__(self, idx, params, world, rank, gather_dtype, working):
        self.idx = idx
        self.working = working  # the parameters have working copies
        self.offsets = [0]
        for i in idx:
            self.offsets.append(self.offsets[-1] + params[i].numel())
        total = self.offsets[-1]
        self.shard = max(1, (total + world - 1) // world)
        self.padded = self.shard * world
        self.s0, self.s1 = rank * self.shard, min((rank + 1) * self.shard, total)
        dev = params[idx[0]].device
        self.master = torch.zeros(self.shard, device=dev, dtype=torch.float32)
        self.exp_avg = torch.zeros_like(self.master)
        self.exp_avg_sq = torch.zeros_like(self.master)
        self.gather_dtype = gather_dtype

    def ranges(self):
        """(slot in idx, start in the parameter, start in the shard, length)
        of every parameter's part inside this rank's shard."""
        out = []
        for k in range(len(self.idx)):
            a, b = max(self.offsets[k], self.s0), min(self.offsets[k + 1], self.s1)
            if a < b:
                out.append((k, a - self.offsets[k], a - self.s0, b - a))
        return out


def _grad_flat(p):
    g = p.grad
    if g.stride() != p.stride():  # one element order for parameter and gradient
        fmt = torch.channels_last if (p.dim() == 4 and p.is_contiguous(memory_format=torch.channels_last)) \
            else torch.contiguous_format
        g = g.contiguous(memory_format=fmt)
    return storage_flat(g)


class ShardedAdam:
    """The optimizer step of ray data parallelism, sharded over the ranks:

    1. the gradients, flattened in the parameters' storage order, are
       reduce-scattered: rank r receives the rank-summed gradient of its 1/N
       of the elements (all-reduced and sliced on backends without
       reduce-scatter, such as gloo);
    2. Adam updates only that shard (its FP32 master values and moments; a
       rank holds the moments of its shard only);
    3. the updated shard is all-gathered in the working precision: BF16 into
       the given working copies (the factor planes and lines of the BF16
       form) and FP32 into the other parameters (the decoder), so every rank
       projects from the same parameters.

    The parameters with working copies and the others are sharded as two
    separate flat domains, so only the small FP32 domain is gathered in
    FP32. Against an all-reduce of the gradients followed by a full Adam on
    every rank, each rank updates 1/N of the optimizer state per step and the
    factor gather carries BF16. The FP32 masters of the parameters with
    working copies are current only inside a rank's shard; gather_masters()
    completes them (before an evaluation or a checkpoint).

    ``update(master, grad, exp_avg, exp_avg_sq, segments, step)`` replaces
    the CUDA Adam kernel (atdf_adam_step_multi) on the shard, e.g.
    adam_shard_torch for CPU tensors."""

    def __init__(self, params, world: int, rank: int, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0,
                 working=None, param_lr=None, update=None):
        self.params = list(params)
        self.world, self.rank = world, rank
        self.hp = [(float((param_lr or {}).get(i, lr)), float(betas[0]), float(betas[1]), float(eps),
                    float(weight_decay)) for i in range(len(self.params))]
        self.working = working or {}  # parameter index -> working copy (same shape and layout)
        self.update = update
        self.step_count = 0
        low = [i for i in range(len(self.params)) if i in self.working]
        plain = [i for i in range(len(self.params)) if i not in self.working]
        self.domains = []
        if low:
            self.domains.append(_Domain(low, self.params, world, rank, self.working[low[0]].dtype, True))
        if plain:
            self.domains.append(_Domain(plain, self.params, world, rank, torch.float32, False))
        for d in self.domains:
            for k, pa, sa, n in d.ranges():
                d.master[sa:sa + n].copy_(storage_flat(self.params[d.idx[k]].detach())[pa:pa + n])

    def _reduce_scatter(self, d, flat):
        if self.world <= 1:
            return flat[:d.shard].clone()
        if dist.get_backend() == "nccl":
            out = torch.empty(d.shard, device=flat.device, dtype=flat.dtype)
            dist.reduce_scatter_tensor(out, flat, op=dist.ReduceOp.SUM)
            return out
        dist.all_reduce(flat, op=dist.ReduceOp.SUM)
        return flat[self.rank * d.shard:(self.rank + 1) * d.shard].clone()

    def _all_gather(self, d, shard):
        if self.world <= 1:
            return shard
        if dist.get_backend() == "nccl":
            out = torch.empty(d.padded, device=shard.device, dtype=shard.dtype)
            dist.all_gather_into_tensor(out, shard)
            return out
        parts = [torch.empty_like(shard) for _ in range(self.world)]
        dist.all_gather(parts, shard)
        return torch.cat(parts)

    @torch.no_grad()
    def step(self):
        """One update; every rank calls it at the same point (the same
        collectives in the same order)."""
        self.step_count += 1
        for d in self.domains:
            flat = torch.zeros(d.padded, device=d.master.device, dtype=torch.float32)
            for k, i in enumerate(d.idx):
                if self.params[i].grad is not None:
                    flat[d.offsets[k]:d.offsets[k + 1]].copy_(_grad_flat(self.params[i]))
            grad = self._reduce_scatter(d, flat).div_(self.world)
            segs = [(sa, sa + n) + self.hp[d.idx[k]] for k, pa, sa, n in d.ranges()]
            if self.update is not None:
                self.update(d.master, grad, d.exp_avg, d.exp_avg_sq, segs, self.step_count)
            else:
                self._adam_cuda(d, grad, segs)
            full = self._all_gather(d, d.master.to(d.gather_dtype))
            for k, i in enumerate(d.idx):
                a, b = d.offsets[k], d.offsets[k + 1]
                target = self.working[i] if d.working else self.params[i].detach()
                storage_flat(target).copy_(full[a:b])
            if d.working:  # the FP32 master is current in this rank's shard
                for k, pa, sa, n in d.ranges():
                    storage_flat(self.params[d.idx[k]].detach())[pa:pa + n].copy_(d.master[sa:sa + n])

    def _adam_cuda(self, d, grad, segs):
        import ctypes as ct

        from . import capi

        batch = []
        for (a, b, lr, b1, b2, eps, wd) in segs:
            t = capi.AdamTensor()
            t.n = b - a
            t.param = d.master.data_ptr() + 4 * a
            t.grad = grad.data_ptr() + 4 * a
            t.exp_avg = d.exp_avg.data_ptr() + 4 * a
            t.exp_avg_sq = d.exp_avg_sq.data_ptr() + 4 * a
            t.param_bf16 = None
            t.lr, t.beta1, t.beta2, t.eps, t.weight_decay, t.step = lr, b1, b2, eps, wd, self.step_count
            batch.append(t)
        if batch:
            arr = (capi.AdamTensor * len(batch))(*batch)
            st = capi.lib().atdf_adam_step_multi(len(batch), arr,
                                                 ct.c_void_p(torch.cuda.current_stream().cuda_stream))
            if st != 0:
                raise RuntimeError(f"atdf_adam_step_multi: {capi.lib().atdf_status_string(st).decode()}")

    @torch.no_grad()
    def gather_masters(self):
        """Complete the FP32 masters of the parameters with working copies on
        every rank (one FP32 all-gather of that domain)."""
        for d in self.domains:
            if not d.working:
                continue
            full = self._all_gather(d, d.master)
            for k, i in enumerate(d.idx):
                storage_flat(self.params[i].detach()).copy_(full[d.offsets[k]:d.offsets[k + 1]])
