"""The fused Adam step (atdf_adam_step via adaptivetensordf_b200.optim.Adam)
against torch.optim.Adam: the same parameters and gradients for several
steps, with parameter groups, weight decay and a learning-rate change. The
two evaluate the update in a different operation order, so parameters agree
to ADAM_RTOL; the BF16 working copies written in the same pass must equal
the updated FP32 parameters rounded to BF16 exactly."""

import pytest
import torch

pytestmark = pytest.mark.gpu

ADAM_RTOL = 1e-5
ADAM_ATOL = 1e-7


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _pairs(seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    shapes = [(37, 16, 17, 17), (1, 16, 256, 1), (64, 16), (1,), (5, 3)]
    ours, ref = [], []
    for sh in shapes:
        x = torch.randn(sh, generator=g)
        if len(sh) == 4:
            x = x.contiguous(memory_format=torch.channels_last)
        a = x.cuda().requires_grad_(True)
        b = x.clone().cuda().requires_grad_(True)
        if len(sh) == 4:
            a = a.detach().contiguous(memory_format=torch.channels_last).requires_grad_(True)
            b = b.detach().contiguous(memory_format=torch.channels_last).requires_grad_(True)
        ours.append(a)
        ref.append(b)
    return ours, ref


def test_fused_adam_matches_torch_adam():
    from adaptivetensordf_b200 import optim

    ours, ref = _pairs(3)
    kw = dict(betas=(0.9, 0.99), eps=1e-8)
    oa = optim.Adam([{"params": ours[:2], "lr": 1e-2}, {"params": ours[2:], "lr": 5e-4, "weight_decay": 0.01}], **kw)
    ta = torch.optim.Adam([{"params": ref[:2], "lr": 1e-2}, {"params": ref[2:], "lr": 5e-4, "weight_decay": 0.01}],
                          **kw)
    g = torch.Generator(device="cpu").manual_seed(5)
    for step in range(6):
        for a, b in zip(ours, ref):
            gr = torch.randn(a.shape, generator=g).cuda()
            if a.dim() == 4:
                gr = gr.contiguous(memory_format=torch.channels_last)
            a.grad = gr.clone()
            b.grad = gr.clone()
        if step == 3:  # a schedule step: the new rate is read on the next update
            for grp_o, grp_t in zip(oa.param_groups, ta.param_groups):
                grp_o["lr"] *= 0.5
                grp_t["lr"] *= 0.5
        oa.step()
        ta.step()
    torch.cuda.synchronize()
    for a, b in zip(ours, ref):
        torch.testing.assert_close(a.detach(), b.detach(), rtol=ADAM_RTOL, atol=ADAM_ATOL)


def test_fused_adam_writes_the_bf16_copies():
    import adaptivetensordf_b200 as ab  # noqa: F401
    from adaptivetensordf_b200 import optim
    from adaptivetensordf_b200 import synthetic as syn

    tree = syn.make_tree(2, device="cuda")
    geo = syn.make_geometry(tree, 16, 17, (64, 17, 64), [64, 64], seed=9)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    params = syn.parameters(geo)
    ref = [p.detach().clone() for p in params]
    opt = optim.Adam(params, lr=1e-2, geometry=geo)
    tref = torch.optim.Adam([r.requires_grad_(True) for r in ref], lr=1e-2)
    g = torch.Generator(device="cpu").manual_seed(1)
    for _ in range(3):
        for p, r in zip(params, ref):
            gr = torch.randn(p.shape, generator=g).cuda().contiguous(memory_format=torch.preserve_format)
            gr = gr.as_strided(p.shape, p.stride()) if gr.stride() != p.stride() else gr
            p.grad = torch.empty_like(p).copy_(gr)
            r.grad = torch.empty_like(r).copy_(gr)
        opt.step()
        tref.step()
    torch.cuda.synchronize()
    for p, r in zip(params, ref):
        torch.testing.assert_close(p.detach(), r.detach(), rtol=ADAM_RTOL, atol=ADAM_ATOL)
    for m in range(3):
        assert torch.equal(geo.planes_bf16[m], geo.planes[m].detach().to(torch.bfloat16))
        assert torch.equal(geo.lines_bf16[m], geo.lines[m].detach().to(torch.bfloat16))


def test_single_tensor_entry_equals_the_batched_launch():
    """atdf_adam_step (one tensor per call) and atdf_adam_step_multi (every
    tensor in one launch, here 20 tensors: two launches of at most 16) apply
    the same arithmetic, so their results are identical."""
    import ctypes as ct

    from adaptivetensordf_b200 import capi

    L = capi.lib()
    g = torch.Generator(device="cpu").manual_seed(3)
    sizes = [1, 3, 5, 64, 1023, 4096, 70001] * 3
    sizes = sizes[:20]
    mk = lambda n: torch.randn(n, generator=g).cuda()  # noqa: E731
    a = [[mk(n) for _ in range(4)] for n in sizes]  # param, grad, m, v
    for t in a:
        t[3].abs_()
    b = [[x.clone() for x in t] for t in a]
    pb = [torch.empty(n, dtype=torch.bfloat16, device="cuda") for n in sizes]
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    for (p, gr, m, v), q in zip(a, pb):
        assert L.atdf_adam_step(p.numel(), capi.ptr(p), capi.ptr(gr), capi.ptr(m), capi.ptr(v), capi.ptr(q), 3e-3,
                                0.9, 0.999, 1e-8, 0.01, 7, stream) == 0
    arr = (capi.AdamTensor * len(sizes))()
    pb2 = [torch.empty_like(q) for q in pb]
    for i, ((p, gr, m, v), q) in enumerate(zip(b, pb2)):
        t = arr[i]
        t.n, t.param, t.grad, t.exp_avg, t.exp_avg_sq, t.param_bf16 = (p.numel(), p.data_ptr(), gr.data_ptr(),
                                                                         m.data_ptr(), v.data_ptr(), q.data_ptr())
        t.lr, t.beta1, t.beta2, t.eps, t.weight_decay, t.step = 3e-3, 0.9, 0.999, 1e-8, 0.01, 7
    assert L.atdf_adam_step_multi(len(sizes), arr, stream) == 0
    torch.cuda.synchronize()
    for ta, tb in zip(a, b):
        for x, y in zip(ta, tb):
            assert torch.equal(x, y)
    for q, q2 in zip(pb, pb2):
        assert torch.equal(q, q2)


def test_update_on_a_side_stream_matches_the_plain_step():
    """Adam(stream=side) with the geometry's params_ready event: the next
    projection runs its segment pass (atdf_project_segments), then waits for
    the update, then projects the segments (atdf_project_forward_segmented).
    Three training steps give the parameters of the same steps with the
    update on the current stream. The backward's line and decoder gradients
    are FP32 atomic sums, so two runs differ in the last bits, and Adam turns
    a last-bit change of a near-zero gradient into a step of up to 2 lr:
    two runs of the same path differ by about 1e-4 relative. A projection
    that read the parameters before their update would differ by about lr in
    every element (about 2e-2 relative here)."""
    import gc

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import optim
    from adaptivetensordf_b200 import synthetic as syn

    tree = syn.make_tree(3, device="cuda")
    rng = torch.Generator(device="cpu").manual_seed(5)
    R = 2048
    o = (torch.rand(R, 3, generator=rng) * 2 - 1) * 0.5
    d = torch.nn.functional.normalize(torch.randn(R, 3, generator=rng), dim=1)
    o = (o - 1.7 * d).cuda()
    d = d.cuda()
    y = torch.rand(1, R, generator=rng).cuda()
    runs = []
    for side in (None, torch.cuda.Stream()):
        geo = syn.make_geometry(tree, 16, 17, (128, 17, 128), [64, 64], seed=9)
        geo.precision = "bf16"
        geo.RefreshLowPrecision()
        params = syn.parameters(geo)
        opt = optim.Adam(params, lr=1e-2, geometry=geo, stream=side)
        for k in range(3):
            img = geo.ProjectRays(tree, ab.RayList(o, d), 16, 1 + k)
            loss, gimg = ab.MseLossAndGrad(img, y, 1.0)
            img.backward(gimg)
            opt.step()
            opt.zero_grad(set_to_none=True)
        if side is not None:
            assert geo.params_ready != 0
            opt.wait()
        torch.cuda.synchronize()
        runs.append(([p.detach().clone() for p in params], [b.clone() for b in geo.planes_bf16]))
        del opt
        gc.collect()
        assert geo.params_ready == 0  # the optimizer takes its event handle back
    for a, b in zip(runs[0][0] + runs[0][1], runs[1][0] + runs[1][1]):
        a, b = a.float(), b.float()
        assert float((a - b).norm() / a.norm().clamp_min(1e-30)) < 2e-3
