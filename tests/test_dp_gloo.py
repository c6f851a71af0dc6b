"""Ray data parallelism on CPU with two gloo ranks: disjoint ray shards,
gradient averaging and node-error sums."""

import os
import socket

import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from adaptivetensordf_b200 import dp

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = dp.shard_permutation(1000, 64, rank, world, epoch=0)
        p = torch.nn.Parameter(torch.zeros(5))
        p.grad = torch.full((5,), float(rank + 1))
        q = torch.nn.Parameter(torch.zeros(2, 2))
        q.grad = torch.eye(2) * (rank + 1) * 10
        # a gradient above the bucket size (reduced alone, channels-last like
        # the planes) and two below it (reduced together in one flat buffer)
        big = torch.nn.Parameter(torch.zeros(2, 3, 4, 5).contiguous(memory_format=torch.channels_last))
        big.grad = (torch.arange(120.0).reshape(2, 3, 4, 5) * (rank + 1)).contiguous(
            memory_format=torch.channels_last)
        dp.allreduce_gradients([p, big, q], world, bucket_bytes=64)
        ls = torch.arange(4, dtype=torch.float64) * (rank + 1)
        ws = torch.ones(4, dtype=torch.float64)
        dp.allreduce_node_error(ls, ws, world)
        out[rank] = {"shards": [s.tolist() for s in shards], "p": p.grad.tolist(), "q": q.grad.tolist(),
                     "big": big.grad.tolist(), "ls": ls.tolist(), "ws": ws.tolist()}
    finally:
        dist.destroy_process_group()


def test_two_rank_data_parallel_step():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    a, b = res[0], res[1]
    assert len(a["shards"]) == len(b["shards"]) == 1000 // (2 * 64)
    for sa, sb in zip(a["shards"], b["shards"]):
        assert len(sa) == len(sb) == 64 and not set(sa) & set(sb)
    for r in (a, b):
        assert r["p"] == [1.5] * 5
        assert r["q"] == [[15.0, 0.0], [0.0, 15.0]]
        assert r["big"] == (torch.arange(120.0).reshape(2, 3, 4, 5) * 1.5).tolist()
        assert r["ls"] == [0.0, 3.0, 6.0, 9.0] and r["ws"] == [2.0] * 4


def _sharded_worker(rank, world, port, out):
    import torch.distributed as dist

    from adaptivetensordf_b200 import dp

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = _sharded_run(rank, world, dp)
    finally:
        dist.destroy_process_group()


def _model(seed=0):
    """Two factor planes (channels-last, with working copies) and a
    decoder-like weight and bias."""
    g = torch.Generator().manual_seed(seed)
    planes = [torch.rand((3, 4, 5, 5), generator=g).contiguous(memory_format=torch.channels_last)
              for _ in range(2)]
    dec = [torch.randn((7, 4), generator=g), torch.randn(7, generator=g)]
    return planes + dec


def _grads(step, rank):
    g = torch.Generator().manual_seed(100 * step + rank)
    return [torch.randn((3, 4, 5, 5), generator=g).contiguous(memory_format=torch.channels_last),
            torch.randn((3, 4, 5, 5), generator=g).contiguous(memory_format=torch.channels_last),
            torch.randn((7, 4), generator=g), torch.randn(7, generator=g)]


def _sharded_run(rank, world, dp):
    params = [p.clone() for p in _model()]
    working = {0: torch.zeros_like(params[0]), 1: torch.zeros_like(params[1])}
    opt = dp.ShardedAdam(params, world, rank, lr=1e-2, working=working, param_lr={2: 1e-3, 3: 1e-3},
                         update=dp.adam_shard_torch)
    for step in range(3):
        for p, g in zip(params, _grads(step, rank)):
            p.grad = g
        opt.step()
    out = {"working": [working[0].tolist(), working[1].tolist()], "dec": [params[2].tolist(), params[3].tolist()]}
    opt.gather_masters()
    out["masters"] = [params[0].tolist(), params[1].tolist()]
    return out


def test_two_rank_sharded_step_equals_one_rank_update():
    """ShardedAdam over two gloo ranks (reduce-scatter emulated by all-reduce
    and slicing, the shard's Adam in torch, all-gathers) gives the same
    parameters as torch.optim.Adam on one rank with the averaged gradients."""
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_sharded_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    ref = [torch.nn.Parameter(p.clone()) for p in _model()]
    opt = torch.optim.Adam([{"params": ref[:2], "lr": 1e-2}, {"params": ref[2:], "lr": 1e-3}])
    for step in range(3):
        g0, g1 = _grads(step, 0), _grads(step, 1)
        for p, a, b in zip(ref, g0, g1):
            p.grad = (a + b) / 2
        opt.step()
    for r in (0, 1):
        got = res[r]
        for k in range(2):
            assert torch.allclose(torch.tensor(got["working"][k]), ref[k].detach(), atol=1e-6)
            assert torch.allclose(torch.tensor(got["masters"][k]), ref[k].detach(), atol=1e-6)
        for k in range(2):
            assert torch.allclose(torch.tensor(got["dec"][k]), ref[2 + k].detach(), atol=1e-6)
