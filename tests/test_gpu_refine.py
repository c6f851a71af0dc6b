"""Adaptive tree refinement on the GPU: moving the factor planes to the new
leaves preserves the field where the factorisation allows it, and a
refinement round inside training keeps the leaf budget."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _field(tree, geo, pts):
    nid, _ = tree.NodeIdForPositionGPU(pts)
    return geo.SampleVolumeIndirect(tree, pts, nid).view(-1)


def test_split_preserves_the_field():
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200 import synthetic as syn

    tree = syn.make_tree(3, active_depth=1)
    geo = syn.make_geometry(tree, 8, 9, (32, 9, 32), [32], seed=4)
    with torch.no_grad():
        geo.lines[1].fill_(1.0)  # the y line is leaf-local: keep it constant so splits are exact
    pts = torch.from_numpy(np.random.default_rng(0).uniform(-0.999, 0.999, (20000, 3)).astype(np.float32)).cuda()
    with torch.no_grad():
        before = _field(tree, geo, pts)
        ids = tree.active_node_ids.tolist()
        err = torch.zeros(tree.NumNodes())
        err[ids[2]] = 3.0
        err[ids[5]] = 1.0
        tree.SetErrorForActiveNodes(err, "override")
        tree.node_max_density = torch.ones(tree.NumNodes(), device="cuda")
        old_tree = recon._tree_like(tree, tree.node_active)
        old_planes = [p.detach().clone() for p in geo.planes]
        assert tree.OptimizeStructure(8 + 7 + 7, 1.1, 0.75)
        assert tree.NumActiveNodes() == 22
        geo.planes = [p.requires_grad_(True) for p in recon.transfer_planes(old_tree, tree, geo, old_planes)]
        geo.leaf_slot = tree.node_active_prefix_sum
        after = _field(tree, geo, pts)
    rel = float((after - before).norm() / before.norm())
    assert rel < 1e-5, rel


def test_merge_averages_children():
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200 import synthetic as syn

    tree = syn.make_tree(2, active_depth=2)
    geo = syn.make_geometry(tree, 8, 9, (32, 9, 32), [32], seed=5)
    with torch.no_grad():
        for p in geo.planes:
            p.fill_(0.25)  # identical children: the merged plane equals them
        tree.SetErrorForActiveNodes(torch.full((tree.NumNodes(),), 0.1), "override")
        tree.node_max_density = torch.ones(tree.NumNodes(), device="cuda")
        old_tree = recon._tree_like(tree, tree.node_active)
        old_planes = [p.detach().clone() for p in geo.planes]
        assert tree.OptimizeStructure(57, 1.1, 0.75)  # one merge of 8 leaves
        assert tree.NumActiveNodes() == 57
        new = recon.transfer_planes(old_tree, tree, geo, old_planes)
    for p in new:
        assert torch.allclose(p, torch.full_like(p, 0.25), atol=1e-6)


def test_refinement_inside_training_keeps_budget():
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200 import synthetic as syn

    cfg = syn.CONFIGS["C1"]
    data = recon.make_tilt_series(cfg)
    opt = recon.TrainOptions(epochs=4, batch=4096, max_samples_per_node=cfg.max_samples_per_node, init_scale=0.05,
                             start_depth=1, refine_every=2, max_active_nodes=36, stop_at_target=False)
    logs = []
    recs, _ = recon.train(cfg, "fp32", data, opt, log=logs.append)
    refined = [r for r in logs if "refined_epoch" in r]
    assert refined and refined[0]["leaves"] <= 36 and refined[0]["leaves"] > 8
    assert np.isfinite(recs[-1]["psnr"]) and recs[-1]["psnr"] > recs[0]["psnr"] - 1.0


def test_max_density_on_the_masked_corner_grid(oracle):
    """compute_max_density: the 20^3 corner-to-corner grid of every leaf
    (UniformGlobalSamples), each point masked by the tilt series' visibility
    (PointInAnyImage), the maximum of the decoded density; against the
    oracle's field and decoder at the same points and the numpy visibility
    mask."""
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200 import synthetic as syn
    from oracle import scene_oracle as so

    cfg = syn.Config("small", 32, 12, 7, 20.0, 24, 2, 8, 9, [32], 1024, 8)
    data = recon.make_tilt_series(cfg)
    tree, geo = recon.build_model(cfg, "fp32", init_scale=0.3)
    recon.compute_max_density(tree, geo, data)
    got = tree.node_max_density[tree.active_node_ids].cpu().numpy()
    ids = tree.active_node_ids
    pts = recon.uniform_global_samples(tree, ids, 20)
    P = pts.reshape(-1, 3).cpu().numpy()
    # the corner grid: first and last points are the leaf's corners
    assert torch.equal(pts[:, 0], tree.node_position_min[ids]) and torch.equal(pts[:, -1], tree.node_position_max[ids])
    node = ids[:, None].expand(-1, 8000).reshape(-1).cpu().numpy()
    td, fd, md = syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)
    dens = oracle.mlp_forward(md, oracle.vm_features(fd, td, P, node, np.float64), np.float64).reshape(-1)
    mask = so.point_in_any_image(P, data.cam_rotation, None, data.cam_intrinsics, data.width, data.height, 1,
                                 data.roi_min, data.roi_max)
    assert 0.0 < mask.mean() < 1.0  # the corners of the volume are outside the +-60 deg field of view
    ref = (dens * mask).reshape(len(ids), -1).max(1)
    assert np.abs(got - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
