"""BF16 form of the fused projection (factor planes and lines in BF16, the
decoder on the tcgen05 tensor cores with FP32 accumulation) against the FP64
oracle.

The oracle runs on the same BF16-rounded factors and decoder weights, so the
remaining difference is the BF16 rounding of the decoder's activations and
gradients inside the tensor-core GEMMs. Tolerance: relative L2 error
BF16_TOL = 2e-2 for the image and for every gradient. The error against the
FP32 field (what the precision form costs) is printed per result."""

import numpy as np
import pytest
import torch

from tests.scene import gpu_scene, oracle_views, rel_err

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-2


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.bfloat16).to(torch.float64).numpy()


@pytest.mark.parametrize("depth,R,M,seed_j", [(2, 600, 16, 0), (3, 900, 12, 77), (4, 1500, 24, 5)])
def test_bf16_tensor_core_projection(oracle, depth, R, M, seed_j):
    import adaptivetensordf_b200 as ab

    L = (17 - 1) * (1 << depth)
    tree, geo, o, d = gpu_scene(depth, 16, 17, (L, 17, L), [64, 64], R, seed=depth + 30)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    td, fd, md = oracle_views(tree, geo)
    fd_b = {**fd, "planes": [_bf16(p) for p in fd["planes"]], "lines": [_bf16(l) for l in fd["lines"]]}
    md_b = {**md, "layers": [(_bf16(w), b.astype(np.float64)) for w, b in md["layers"]]}
    # the last layer (64 -> 1) runs on CUDA cores in FP32
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    rays = ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda())
    img = geo.ProjectRays(tree, rays, M, seed_j)
    segs = oracle.ray_segments(td, o, d, M)
    so = oracle.emit_samples(segs, o, d, oracle.jitter_for_segments(seed_j, segs) if seed_j else None)
    ref = oracle.project_forward(fd_b, md_b, td, so, R, np.float64)
    ref32 = oracle.project_forward(fd, md, td, so, R, np.float64)
    e = rel_err(img.detach().cpu().numpy(), ref)
    print(f"\nBF16 image: rel err {e:.2e} vs oracle on BF16 factors, "
          f"{rel_err(img.detach().cpu().numpy(), ref32):.2e} vs the FP32 field")
    assert e < BF16_TOL
    gi = np.random.default_rng(8).normal(size=ref.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd_b, md_b, td, so, R, gi, np.float64)
    errs = {}
    for m in range(3):
        errs[f"plane{m}"] = rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m])
        errs[f"line{m}"] = rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m])
    for li in range(3):
        errs[f"W{li}"] = rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li])
        errs[f"b{li}"] = rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li])
    print("BF16 gradients rel err: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v < BF16_TOL, k


@pytest.mark.parametrize("C", [16, 24])
def test_bf16_plane_gradient_dynamic_range(oracle, C):
    """The tensor-core backward sums each leaf's plane gradients as fixed-point
    integers with a per-leaf scale chosen from the first tiles, and sends a
    tile that would exceed the integer range to global memory in FP32 (the
    24-channel kernel zeroes a leaf's global gradient at its first such
    tile). Image gradients spread over twelve decades (random signs) make the
    tiles of a leaf differ by orders of magnitude, so both paths run; every
    leaf's plane gradient must still match the oracle to BF16_TOL of its own
    norm."""
    import adaptivetensordf_b200 as ab

    depth, R, M, seed_j = 3, 900, 12, 3
    L = (17 - 1) * (1 << depth)
    tree, geo, o, d = gpu_scene(depth, C, 17, (L, 17, L), [64, 64], R, seed=41)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    td, fd, md = oracle_views(tree, geo)
    fd_b = {**fd, "planes": [_bf16(p) for p in fd["planes"]], "lines": [_bf16(l) for l in fd["lines"]]}
    md_b = {**md, "layers": [(_bf16(w), b.astype(np.float64)) for w, b in md["layers"]]}
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    rays = ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda())
    img = geo.ProjectRays(tree, rays, M, seed_j)
    rng = np.random.default_rng(12)
    gi = (10.0 ** rng.uniform(-6, 6, size=(1, R))) * rng.choice([-1.0, 1.0], size=(1, R))
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    segs = oracle.ray_segments(td, o, d, M)
    so = oracle.emit_samples(segs, o, d, oracle.jitter_for_segments(seed_j, segs))
    gr = oracle.project_backward(fd_b, md_b, td, so, R, gi.astype(np.float32).astype(np.float64), np.float64)
    worst = 0.0
    for m in range(3):
        got, ref = geo.planes[m].grad.cpu().numpy(), gr["planes"][m]
        for s in range(ref.shape[0]):
            if np.abs(ref[s]).max() > 0:
                worst = max(worst, rel_err(got[s], ref[s]))
    print(f"\nworst per-leaf plane-gradient rel err over 12 decades of dI: {worst:.2e}")
    assert worst < BF16_TOL


def _bf16_views(tree, geo):
    td, fd, md = oracle_views(tree, geo)
    fd_b = {**fd, "planes": [_bf16(p) for p in fd["planes"]], "lines": [_bf16(l) for l in fd["lines"]]}
    md_b = {**md, "layers": [(_bf16(w), b.astype(np.float64)) for w, b in md["layers"]]}
    # the last layer (64 -> 1) runs on CUDA cores in FP32
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    return td, fd_b, md_b


def _mixed_depth_tree(max_depth, seed):
    """Active leaves at depths 2..max_depth: a seeded random refinement of the
    depth-2 octree (each leaf split with probability 0.4 while above
    max_depth), the kind of tree the structure refinement produces."""
    from adaptivetensordf_b200 import synthetic as syn

    rng = np.random.default_rng(seed)
    t = syn.make_tree(max_depth, 2, device="cpu")
    ch = t.node_children.numpy()
    depth = t.node_depth.numpy()
    leaves = list(np.nonzero(depth == 2)[0])
    active = []
    while leaves:
        n = leaves.pop()
        if depth[n] < max_depth and rng.random() < 0.4:
            leaves.extend(int(c) for c in ch[n] if c >= 0)
        else:
            active.append(n)
    return syn.tree_from_leaves(max_depth, np.array(active), device="cuda")


@pytest.mark.parametrize("depth,R,M,seed_j,mixed", [(2, 600, 16, 0, False), (4, 1500, 24, 5, False),
                                                      (5, 1200, 20, 9, True)])
def test_bf16_rank24_projection(oracle, depth, R, M, seed_j, mixed):
    """The 24-channel tensor-core kernels (K of the first layer padded to 32,
    one 128-row tile per backward CTA) against the FP64 oracle on the
    BF16-rounded parameters, on uniform and on mixed-depth trees."""
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn
    from tests.scene import rays_through_volume

    tree = _mixed_depth_tree(depth, 77) if mixed else syn.make_tree(depth, device="cuda")
    L = (17 - 1) * (1 << min(depth, 4))
    geo = syn.make_geometry(tree, 24, 17, (L, 17, L), [64, 64], seed=depth + 60)
    o, d = rays_through_volume(R, depth + 61)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    td, fd_b, md_b = _bf16_views(tree, geo)
    rays = ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda())
    img = geo.ProjectRays(tree, rays, M, seed_j)
    segs = oracle.ray_segments(td, o, d, M)
    so = oracle.emit_samples(segs, o, d, oracle.jitter_for_segments(seed_j, segs) if seed_j else None)
    ref = oracle.project_forward(fd_b, md_b, td, so, R, np.float64)
    errs = {"image": rel_err(img.detach().cpu().numpy(), ref)}
    gi = np.random.default_rng(18).normal(size=ref.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd_b, md_b, td, so, R, gi, np.float64)
    for m in range(3):
        errs[f"plane{m}"] = rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m])
        errs[f"line{m}"] = rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m])
    for li in range(3):
        errs[f"W{li}"] = rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li])
        errs[f"b{li}"] = rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li])
    print(f"\nrank-24 BF16 (depth {depth}{', mixed' if mixed else ''}, {tree.NumActiveNodes()} leaves): "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v < BF16_TOL, k
    geo.CheckErrors()
