"""Parity at the benchmark's scale: the depth-4 octree with all 4096 leaves,
rank-16 VM on 17^2 planes with lines (256, 17, 256), decoder 16 -> 64 -> 64
-> 1, 24 samples per leaf diagonal and interval jitter, on rays of the
61-tilt 256^2 parallel-beam series (the C2 training batch).

At this size the fused kernels run the paths small scenes never reach:
slots cut into several work items, the longest-first slot queue, the
per-item sample -> segment byte map and its binary-search fallback for items
of more than 4096 samples, and many CTAs contending for the slot queue.

* The segment and sample lists of a whole 16384-ray batch are compared bit
  for bit with the oracle.
* The fused FP32 projection and every gradient are compared with the FP64
  oracle (relative L2 <= 1e-5) on 2048 rays of that batch's tilts aimed at
  a 64 x 64-pixel window of the detector: the leaves they cross see about
  twice the batch's segments per leaf (multi-item slots).
* The BF16 tensor-core form is compared with the FP64 oracle run on the same
  BF16-rounded factors and weights, with per-quantity tolerances of about
  three times the measured error.
"""

import numpy as np
import pytest
import torch

from tests.scene import rel_err

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
# BF16 form against the FP64 oracle on the BF16-rounded parameters, about
# three times the measured errors (M = 24 / 96): the image carries the BF16
# rounding of the decoder's activations (1.4e-5 / 7e-6), the plane and line
# gradients also that of the backward's operands (1.9e-3 / 2.9e-3), the
# first-layer weights 2e-3, the other decoder parameters <= 1.4e-4
BF16_TOL = {"image": 5e-5, "plane": 6e-3, "line": 9e-3, "W": 6e-3, "b": 5e-4}


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _c2():
    from adaptivetensordf_b200.synthetic import CONFIGS

    return CONFIGS["C2"]


@pytest.fixture(scope="module")
def c2_model():
    from adaptivetensordf_b200 import synthetic as syn

    cfg = _c2()
    tree = syn.make_tree(cfg.tree_depth, device="cuda")
    return cfg, tree


def _window_rays(cfg, R, seed, x0=96, y0=96, w=64):
    """R rays of the C2 series (random tilts) through a w x w pixel window."""
    from adaptivetensordf_b200 import synthetic as syn

    rng = np.random.default_rng(seed)
    img = rng.integers(0, cfg.angles, R)
    px = x0 + rng.integers(0, w, R)
    py = y0 + rng.integers(0, w, R)
    return syn.parallel_beam_rays(syn.tilt_angles(cfg), cfg.detector, img, py * cfg.detector + px)


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.bfloat16).to(torch.float64).numpy()


def test_bench_batch_segments_and_samples_bit_exact(oracle, c2_model):
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    cfg, tree = c2_model
    o, d = syn.random_ray_batch(cfg, cfg.rays_per_batch, 1004)
    td = syn.tree_dict(tree)
    M, seed = cfg.max_samples_per_node, 101
    segs_o = oracle.ray_segments(td, o, d, M)
    rays = ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda())
    sg = tree.RaySegments(rays, M)
    assert sg.num_segments == len(segs_o["n"]) and sg.num_segments > 300000
    assert sg.num_samples == int(segs_o["n"].sum())
    for k_gpu, k_or in [("node", "node"), ("nsamp", "n"), ("ray", "ray"), ("first", "first"), ("tmin", "tmin"),
                        ("tmax", "tmax")]:
        assert np.array_equal(getattr(sg, k_gpu).cpu().numpy(), segs_o[k_or]), k_gpu
    s = tree.CreateSamplesForRaysWithRnd(rays, M, None, seed)
    s_o = oracle.emit_samples(segs_o, o, d, oracle.jitter_for_segments(seed, segs_o))
    for k in ["global_coordinate", "ray_t", "weight", "ray_index", "local_index_in_ray", "node_id"]:
        assert np.array_equal(getattr(s, k).cpu().numpy(), s_o[k]), k
    per_leaf = np.bincount(segs_o["node"], minlength=tree.NumNodes())[tree.active_node_ids.cpu().numpy()]
    print(f"\n{sg.num_segments} segments, {sg.num_samples} samples; segments per leaf: mean "
          f"{per_leaf.mean():.1f}, max {per_leaf.max()}, leaves with > 128: {(per_leaf > 128).sum()}")


def _scene(cfg, tree, R, seed, M):
    """M = 24: 2048 rays through a 64^2 window (about 190 segments in the
    busiest leaves); M = 96: 512 rays through a 16^2 window (items of up to
    about 4900 samples)."""
    from adaptivetensordf_b200 import synthetic as syn

    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    w = 64 if M == 24 else 16
    o, d = _window_rays(cfg, R, seed, 128 - w // 2, 128 - w // 2, w)
    return geo, o, d


def _oracle_samples(oracle, td, o, d, M, seed_j):
    segs = oracle.ray_segments(td, o, d, M)
    return segs, oracle.emit_samples(segs, o, d, oracle.jitter_for_segments(seed_j, segs))


@pytest.mark.parametrize("M", [24, 96])
def test_bench_shapes_fp32_dense_window(oracle, c2_model, M):
    """Fused FP32 forward and adjoint at the benchmark's model shapes; M = 96
    makes items of more than 4096 samples (the binary-search path)."""
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    cfg, tree = c2_model
    R, seed_j = (2048, 55) if M == 24 else (512, 56)
    geo, o, d = _scene(cfg, tree, R, 7 + M, M)
    td, fd, md = syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)
    segs, so = _oracle_samples(oracle, td, o, d, M, seed_j)
    per_leaf = np.bincount(segs["node"])
    samples = np.bincount(segs["node"], weights=segs["n"])
    touched = per_leaf > 0
    per_item = samples[touched] / np.ceil(per_leaf[touched] / 128)
    print(f"\nM={M}: {len(segs['n'])} segments, max per leaf {per_leaf.max()}, "
          f"leaves with > 128 segments {(per_leaf > 128).sum()}, items over 4096 samples {(per_item > 4096).sum()}")
    assert (per_leaf > 128).sum() > 5  # slots of several work items
    if M == 96:
        assert (per_item > 4096).sum() > 0  # items beyond the sample -> segment map
    img = geo.ProjectRays(tree, ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()), M, seed_j)
    ref = oracle.project_forward(fd, md, td, so, R, np.float64)
    assert rel_err(img.detach().cpu().numpy(), ref) < REL_TOL
    gi = np.random.default_rng(9).normal(size=ref.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd, md, td, so, R, gi, np.float64)
    for m in range(3):
        assert rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m]) < REL_TOL, f"plane {m}"
        assert rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m]) < REL_TOL, f"line {m}"
    for li in range(3):
        assert rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li]) < REL_TOL, f"W{li}"
        assert rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li]) < REL_TOL, f"b{li}"
    geo.CheckErrors()


@pytest.mark.parametrize("M", [24, 96])
def test_bench_shapes_bf16_dense_window(oracle, c2_model, M):
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    cfg, tree = c2_model
    R, seed_j = (2048, 57) if M == 24 else (512, 58)
    geo, o, d = _scene(cfg, tree, R, 17 + M, M)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    td, fd, md = syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)
    fd_b = {**fd, "planes": [_bf16(p) for p in fd["planes"]], "lines": [_bf16(x) for x in fd["lines"]]}
    md_b = {**md, "layers": [(_bf16(w), b.astype(np.float64)) for w, b in md["layers"]]}
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    segs, so = _oracle_samples(oracle, td, o, d, M, seed_j)
    img = geo.ProjectRays(tree, ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()), M, seed_j)
    ref = oracle.project_forward(fd_b, md_b, td, so, R, np.float64)
    errs = {"image": rel_err(img.detach().cpu().numpy(), ref)}
    gi = np.random.default_rng(10).normal(size=ref.shape)
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd_b, md_b, td, so, R, gi, np.float64)
    for m in range(3):
        errs[f"plane{m}"] = rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m])
        errs[f"line{m}"] = rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m])
    for li in range(3):
        errs[f"W{li}"] = rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li])
        errs[f"b{li}"] = rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li])
    print(f"\nBF16 at the benchmark's shapes (M={M}): " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v < BF16_TOL[k.rstrip("0123456789")], k
    geo.CheckErrors()


def test_c5_rank24_dense_window_bf16(oracle):
    """The rank-24 kernels at the C5 headline's shapes where they split work
    the most: 1536 rays of the C5 series through a 32 x 32-pixel window at the
    detector's centre cross the same central leaves, so a leaf's segments fill
    many work items (the forwards spread them over CTAs through the item
    queue; the backward walks them in one CTA), items exceed the forward's
    2048-sample map, and depth-3 leaves use the 40-row line windows. BF16
    projection and gradients against the FP64 oracle on the BF16-rounded
    parameters, with the tolerances above."""
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    cfg = syn.CONFIGS["C5"]
    tree = syn.adaptive_tree(cfg, syn.config_phantom(cfg, 1001), device="cuda")
    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    R, M, seed_j, w = 1536, cfg.max_samples_per_node, 61, 32
    rng = np.random.default_rng(77)
    img = rng.integers(0, cfg.angles, R)
    c0 = cfg.detector // 2 - w // 2
    px = c0 + rng.integers(0, w, R)
    py = c0 + rng.integers(0, w, R)
    o, d = syn.parallel_beam_rays(syn.tilt_angles(cfg), cfg.detector, img, py * cfg.detector + px, cfg.off_axis_deg)
    td, fd, md = syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)
    fd_b = {**fd, "planes": [_bf16(p) for p in fd["planes"]], "lines": [_bf16(x) for x in fd["lines"]]}
    md_b = {**md, "layers": [(_bf16(wt), b.astype(np.float64)) for wt, b in md["layers"]]}
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    segs, so = _oracle_samples(oracle, td, o, d, M, seed_j)
    per_leaf = np.bincount(segs["node"])
    samples = np.bincount(segs["node"], weights=segs["n"])
    depth = tree.node_depth.cpu().numpy()
    print(f"\n{len(segs['n'])} segments, {int(segs['n'].sum())} samples; max segments per leaf {per_leaf.max()}, "
          f"max samples per leaf {int(samples.max())}, depth-3 leaves hit {int((per_leaf[depth[:len(per_leaf)] == 3] > 0).sum())}")
    assert per_leaf.max() > 3 * 128  # a leaf of several work items
    assert samples.max() > 2 * 2048
    out = geo.ProjectRays(tree, ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()), M, seed_j)
    ref = oracle.project_forward(fd_b, md_b, td, so, R, np.float64)
    errs = {"image": rel_err(out.detach().cpu().numpy(), ref)}
    gi = np.random.default_rng(11).normal(size=ref.shape)
    out.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    gr = oracle.project_backward(fd_b, md_b, td, so, R, gi, np.float64)
    for m in range(3):
        errs[f"plane{m}"] = rel_err(geo.planes[m].grad.cpu().numpy(), gr["planes"][m])
        errs[f"line{m}"] = rel_err(geo.lines[m].grad.cpu().numpy(), gr["lines"][m])
    for li in range(3):
        errs[f"W{li}"] = rel_err(geo.decoder_weight[li].grad.cpu().numpy(), gr["W"][li])
        errs[f"b{li}"] = rel_err(geo.decoder_bias[li].grad.cpu().numpy(), gr["b"][li])
    print("rank-24 BF16 at C5's shapes: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v < BF16_TOL[k.rstrip("0123456789")], k
    geo.CheckErrors()
