"""Parity of the CUDA path against the CPU oracle on seeded inputs.

Integer / index outputs (segment lists, sample counts, indices) must match
bit for bit; sample t / weight / position values too (both sides round once
per operation). Floating-point results of the field, decoder, projection and
gradients must agree with the FP64 oracle within the relative L2 tolerance
REL_TOL = 1e-5 stated by the target (FP32 arithmetic on the GPU)."""

import numpy as np
import pytest
import torch

from tests.scene import gpu_scene, oracle_views, rays_through_volume, rel_err

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _rays(o, d):
    import adaptivetensordf_b200 as ab

    return ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda())


@pytest.mark.parametrize("depth,quad,R,M", [(0, False, 64, 16), (2, False, 512, 32), (3, False, 777, 8),
                                            (4, False, 2048, 24), (3, True, 300, 16)])
def test_segments_and_samples_bit_exact(oracle, depth, quad, R, M):
    tree, geo, o, d = gpu_scene(depth, 8, 5, (9, 5, 9), [32], R, seed=depth, quad=quad)
    td = oracle_views(tree, geo)[0]
    segs_o, s_o = oracle.create_samples_for_rays(td, o, d, M)
    sg = tree.RaySegments(_rays(o, d), M)
    assert sg.num_segments == len(segs_o["n"])
    assert sg.num_samples == int(segs_o["n"].sum())
    for k_gpu, k_or in [("node", "node"), ("nsamp", "n"), ("ray", "ray"), ("first", "first"), ("tmin", "tmin"),
                        ("tmax", "tmax")]:
        assert np.array_equal(getattr(sg, k_gpu).cpu().numpy(), segs_o[k_or]), k_gpu
    s = tree.CreateSamplesForRays(_rays(o, d), M, False)
    for k in ["global_coordinate", "ray_t", "weight", "ray_index", "local_index_in_ray", "node_id"]:
        assert np.array_equal(getattr(s, k).cpu().numpy(), s_o[k]), k
    assert s.max_samples_per_ray == s_o["max_samples_per_ray"]


def test_samples_with_explicit_jitter_bit_exact(oracle):
    tree, geo, o, d = gpu_scene(3, 8, 5, (9, 5, 9), [32], 400, seed=5)
    td = oracle_views(tree, geo)[0]
    segs_o = oracle.ray_segments(td, o, d, 16)
    S = int(segs_o["n"].sum())
    rnd = np.random.default_rng(0).random(S).astype(np.float32)
    s_o = oracle.emit_samples(segs_o, o, d, rnd)
    s = tree.CreateSamplesForRaysWithRnd(_rays(o, d), 16, torch.from_numpy(rnd).cuda(), 0)
    for k in ["global_coordinate", "ray_t", "weight"]:
        assert np.array_equal(getattr(s, k).cpu().numpy(), s_o[k]), k
    # hashed jitter: the GPU draws exactly the oracle's values
    s2 = tree.CreateSamplesForRaysWithRnd(_rays(o, d), 16, None, 1234)
    rnd2 = oracle.jitter_for_segments(1234, segs_o)
    s2_o = oracle.emit_samples(segs_o, o, d, rnd2)
    assert np.array_equal(s2.ray_t.cpu().numpy(), s2_o["ray_t"])
    assert np.array_equal(s2.weight.cpu().numpy(), s2_o["weight"])


def test_edge_rays(oracle):
    """Empty batch, rays that miss, rays on split planes and grazing rays."""
    import adaptivetensordf_b200 as ab

    tree, geo, _, _ = gpu_scene(2, 8, 5, (9, 5, 9), [32], 1)
    td = oracle_views(tree, geo)[0]
    empty = ab.RayList(torch.zeros(0, 3, device="cuda"), torch.zeros(0, 3, device="cuda"))
    s = tree.CreateSamplesForRays(empty, 8, False)
    assert s.size() == 0
    o = np.array([[5, 5, -3], [-0.5, 0.0, -3], [0.0, 0.5, -3], [0.5, 0.5, -3], [0.0, 0.0, -3.0],
                  [-1.0, -1.0, -3.0], [1.0, 1.0, -3.0]], np.float32)
    d = np.array([[0, 0, 1]] * 5 + [[0, 0, 1], [0, 0, 1]], np.float32)
    d[4] = [1e-7, 0, 1]
    segs_o, s_o = oracle.create_samples_for_rays(td, o, d, 8)
    s = tree.CreateSamplesForRays(_rays(o, d), 8, False)
    assert np.array_equal(s.node_id.cpu().numpy(), s_o["node_id"])
    assert np.array_equal(s.weight.cpu().numpy(), s_o["weight"])
    assert np.array_equal(s.ray_index.cpu().numpy(), s_o["ray_index"])


def test_local_samples_and_node_id(oracle):
    tree, geo, o, d = gpu_scene(3, 8, 5, (9, 5, 9), [32], 200, seed=2)
    td = oracle_views(tree, geo)[0]
    s = tree.CreateSamplesForRays(_rays(o, d), 8, False)
    loc = tree.ComputeLocalSamples(s.global_coordinate, s.node_id)
    loc_o = oracle.local_samples(td, s.global_coordinate.cpu().numpy(), s.node_id.cpu().numpy())
    assert np.array_equal(loc.cpu().numpy(), loc_o)
    pts = np.random.default_rng(1).uniform(-1.1, 1.1, (5000, 3)).astype(np.float32)
    pts[:10] = 0.0
    ids, mask = tree.NodeIdForPositionGPU(torch.from_numpy(pts).cuda())
    ids_o, mask_o = oracle.node_id_for_position(td, pts)
    assert np.array_equal(ids.cpu().numpy(), ids_o)
    assert np.array_equal(mask.cpu().numpy(), mask_o)


def test_grid_sample_ops(oracle):
    import adaptivetensordf_b200 as ab

    rng = np.random.default_rng(0)
    for shape in [(5, 8, 17, 17), (3, 4, 6, 9)]:
        g = rng.normal(size=shape).astype(np.float32)
        S = 3000
        idx = rng.integers(0, shape[0], S)
        uv = rng.uniform(-1.2, 1.2, (S, 2)).astype(np.float32)
        gt = torch.from_numpy(g).cuda().requires_grad_(True)
        ut = torch.from_numpy(uv).cuda().requires_grad_(True)
        out = ab.IndirectGridSample2D(gt, torch.from_numpy(idx).cuda(), ut)
        out_o = oracle.grid_sample2d(g, idx, uv, np.float32)
        assert np.array_equal(out.detach().cpu().numpy(), out_o)
        go = rng.normal(size=out_o.shape).astype(np.float32)
        out.backward(torch.from_numpy(go).cuda())
        gg_o, gu_o = oracle.grid_sample2d_bwd(g, idx, uv, go, np.float64)
        assert rel_err(gt.grad.cpu().numpy(), gg_o) < REL_TOL
        assert np.array_equal(ut.grad.cpu().numpy(), oracle.grid_sample2d_bwd(g, idx, uv, go, np.float32)[1])
        # channels-last input gives the same result
        out_cl = ab.IndirectGridSample2D(gt.detach().contiguous(memory_format=torch.channels_last),
                                         torch.from_numpy(idx).cuda(), ut.detach())
        assert torch.equal(out_cl, out.detach())
    l = rng.normal(size=(2, 8, 33, 1)).astype(np.float32)
    idx = rng.integers(0, 2, 1000)
    u = rng.uniform(-1.1, 1.1, (1000, 1)).astype(np.float32)
    lt = torch.from_numpy(l).cuda().requires_grad_(True)
    ut = torch.from_numpy(u).cuda().requires_grad_(True)
    out = ab.IndirectGridSample1D(lt, torch.from_numpy(idx).cuda(), ut)
    assert np.array_equal(out.detach().cpu().numpy(), oracle.grid_sample1d(l, idx, u, np.float32))
    go = rng.normal(size=(1000, 8)).astype(np.float32)
    out.backward(torch.from_numpy(go).cuda())
    gl_o, gu_o = oracle.grid_sample1d_bwd(l, idx, u, go, np.float64)
    assert rel_err(lt.grad.cpu().numpy(), gl_o) < REL_TOL
    assert np.array_equal(ut.grad.cpu().numpy(), oracle.grid_sample1d_bwd(l, idx, u, go, np.float32)[1])


@pytest.mark.parametrize("tensor_op", ["add", "cat"])
def test_unfused_field_decoder_integral(oracle, tensor_op):
    """SampleVolumeIndirect + DecodeFeatures + IntegrateSamplesXRay (unfused
    composition of the drop-in ops) and its autograd backward."""
    import adaptivetensordf_b200 as ab

    R = 300
    tree, geo, o, d = gpu_scene(2, 8, 9, (33, 9, 33), [32, 32], R, seed=7, tensor_op=tensor_op)
    td, fd, md = oracle_views(tree, geo)
    s = tree.CreateSamplesForRays(_rays(o, d), 12, False)
    so = {k: getattr(s, k).cpu().numpy() for k in ["global_coordinate", "weight", "ray_index", "node_id"]}
    feat = geo.SampleVolumeIndirect_feature(tree, s.global_coordinate, s.node_id)
    feat_o = oracle.vm_features(fd, td, so["global_coordinate"], so["node_id"], np.float32)
    assert np.array_equal(feat.detach().cpu().numpy(), feat_o)
    img, ratio, ratio_inv = geo.ComputeImage(tree, s, 1, R)
    assert ratio is None and ratio_inv is None  # undefined, as in the reference's indirect path
    img_o = oracle.project_forward(fd, md, td, so, R, np.float64)
    assert rel_err(img.detach().cpu().numpy(), img_o) < REL_TOL
    gi = np.random.default_rng(3).normal(size=img_o.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd, md, td, so, R, gi, np.float64)
    for m in range(3):
        assert rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m]) < REL_TOL
        assert rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m]) < REL_TOL
    for li in range(len(md["layers"])):
        assert rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li]) < REL_TOL
        assert rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li]) < REL_TOL


@pytest.mark.parametrize("C,hidden,depth,G,lines,tensor_op,seed_j", [
    (8, [32], 2, 17, (64, 17, 64), "add", 0),
    (16, [64, 64], 3, 17, (128, 17, 128), "add", 99),
    (16, [64], 2, 9, (32, 9, 32), "add", 0),
    (8, [64, 64], 2, 17, (64, 17, 64), "cat", 5),
])
def test_fused_projection_forward_backward(oracle, C, hidden, depth, G, lines, tensor_op, seed_j):
    """Fused leaf-major forward and hand-written adjoint vs the FP64 oracle on
    the same samples."""
    import adaptivetensordf_b200 as ab

    R = 700
    M = 16
    tree, geo, o, d = gpu_scene(depth, C, G, lines, hidden, R, seed=C + depth, tensor_op=tensor_op)
    td, fd, md = oracle_views(tree, geo)
    img = geo.ProjectRays(tree, _rays(o, d), M, seed_j)
    segs_o = oracle.ray_segments(td, o, d, M)
    rnd = oracle.jitter_for_segments(seed_j, segs_o) if seed_j else None
    so = oracle.emit_samples(segs_o, o, d, rnd)
    img_o = oracle.project_forward(fd, md, td, so, R, np.float64)
    assert rel_err(img.detach().cpu().numpy(), img_o) < REL_TOL
    gi = np.random.default_rng(4).normal(size=img_o.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd, md, td, so, R, gi, np.float64)
    for m in range(3):
        assert rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m]) < REL_TOL, f"plane {m}"
        assert rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m]) < REL_TOL, f"line {m}"
    for li in range(len(md["layers"])):
        assert rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li]) < REL_TOL, f"W{li}"
        assert rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li]) < REL_TOL, f"b{li}"


def test_fused_out_of_roi_leaves(oracle):
    """Leaves outside the ROI (slot -1) decode zero features, as the reference
    does with a ground-truth volume."""
    R = 400
    tree, geo, o, d = gpu_scene(2, 8, 9, (32, 9, 32), [32], R, seed=3)
    slot = geo.leaf_slot.clone()
    ids = tree.active_node_ids
    slot[ids[::3]] = -1
    geo.leaf_slot = slot
    td, fd, md = oracle_views(tree, geo)
    img = geo.ProjectRays(tree, _rays(o, d), 8, 0)
    segs_o, so = oracle.create_samples_for_rays(td, o, d, 8)
    img_o = oracle.project_forward(fd, md, td, so, R, np.float64)
    assert rel_err(img.detach().cpu().numpy(), img_o) < REL_TOL
    gi = np.ones_like(img_o)
    img.backward(torch.ones_like(img))
    gr = oracle.project_backward(fd, md, td, so, R, gi, np.float64)
    for m in range(3):
        assert rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m]) < REL_TOL
    for li in range(len(md["layers"])):
        assert rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li]) < REL_TOL


def test_node_error_scoring(oracle):
    import adaptivetensordf_b200 as ab

    R = 500
    tree, geo, o, d = gpu_scene(2, 8, 9, (32, 9, 32), [32], R, seed=9)
    td, fd, md = oracle_views(tree, geo)
    y = np.random.default_rng(0).uniform(0, 2, (1, R)).astype(np.float32)
    img, ls, ws = geo.ProjectNodeError(tree, _rays(o, d), 8, 0, torch.from_numpy(y).cuda())
    segs_o, so = oracle.create_samples_for_rays(td, o, d, 8)
    prl = (img.cpu().numpy() - y) ** 2
    ls_o, ws_o = oracle.accumulate_loss_per_node(so, prl, len(td["node_depth"]))
    assert rel_err(ws.cpu().numpy(), ws_o) < 1e-12
    assert rel_err(ls.cpu().numpy(), ls_o) < 1e-9
    # unfused AccumulateSampleLossPerNode on the SampleList
    s = tree.CreateSamplesForRays(_rays(o, d), 8, False)
    ls2, ws2 = ab.AccumulateSampleLossPerNode(s, torch.from_numpy(prl).cuda(), tree.NumNodes())
    assert rel_err(ls2.cpu().numpy(), ls_o) < 1e-9


def test_mse_loss_and_grad():
    import adaptivetensordf_b200 as ab

    x = torch.randn(1, 1000, device="cuda")
    y = torch.randn(1, 1000, device="cuda")
    loss, g = ab.MseLossAndGrad(x, y, 1.0)
    assert abs(loss.item() - ((x - y) ** 2).mean().item()) < 1e-6
    assert torch.allclose(g, 2 * (x - y) / 1000, atol=1e-7)


def test_gradient_correction_bit_exact(oracle):
    """GradientCorrection (identity forward, g - (g.d) d backward) through the
    autograd op and through the C ABI, bit-exact against the oracle; an
    out-of-range ray index sets the index bit and leaves its row unwritten."""
    import ctypes as ct

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import capi

    rng = np.random.default_rng(5)
    R, S = 300, 20000
    d = rng.normal(size=(R, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ray = rng.integers(0, R, S)
    pos = rng.uniform(-1, 1, (S, 3)).astype(np.float32)
    g = rng.normal(size=(S, 3)).astype(np.float32)
    pt = torch.from_numpy(pos).cuda().requires_grad_(True)
    out = ab.GradientCorrection(pt, torch.from_numpy(d).cuda(), torch.from_numpy(ray).cuda())
    assert torch.equal(out.detach(), pt.detach())
    out.backward(torch.from_numpy(g).cuda())
    ref = oracle.gradient_correction_bwd(d, ray, g)
    assert np.array_equal(pt.grad.cpu().numpy(), ref)

    L = capi.lib()
    ray_bad = ray.copy()
    ray_bad[7] = R + 3
    dt, rt, gt = (torch.from_numpy(x).cuda() for x in (d, ray_bad, g))
    gout = torch.full((S, 3), 123.0, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.atdf_gradient_correction_backward(capi.ptr(dt), capi.ptr(rt), R, capi.ptr(gt), S, capi.ptr(gout),
                                               capi.ptr(err), stream) == 0
    torch.cuda.synchronize()
    assert err.item() == capi.DEVERR["index"]
    got = gout.cpu().numpy()
    assert np.all(got[7] == 123.0)
    keep = np.arange(S) != 7
    assert np.array_equal(got[keep], ref[keep])
