"""CPU checks of the reconstruction driver's data generation."""

import numpy as np


def test_voxelize_boxes_matches_dense_voxelization():
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.recon import voxelize_boxes

    ph = syn.ellipsoid_phantom(20, 1001)
    a = syn.voxelize(ph, 40)
    b = voxelize_boxes(ph, 40)
    assert np.array_equal(a, b)
    assert 0 < a.mean() < 1


def _small_slab():
    import dataclasses

    from adaptivetensordf_b200 import synthetic as syn

    # the C5 refinement rule on a reduced phantom and leaf budget
    return dataclasses.replace(syn.CONFIGS["C5"], ellipsoids=300, target_leaves=700)


def test_adaptive_leaves_partition_the_specimen(oracle):
    """The adaptive tree's leaves are disjoint, lie in the slab, reach the
    maximum depth, and the tree built from them (the product's HyperTreeBase)
    has exactly those active leaves; the oracle's copy of the tree arrays
    gives the same leaves."""
    import torch

    from adaptivetensordf_b200 import synthetic as syn

    cfg = _small_slab()
    ph = syn.config_phantom(cfg)
    t = oracle.tree_build(cfg.tree_depth)
    leaves, culled = syn.adaptive_leaves(cfg, ph, t["node_position_min"], t["node_position_max"],
                                         t["node_children"], t["node_depth"])
    assert 0.95 * cfg.target_leaves <= len(leaves) <= 1.05 * cfg.target_leaves
    assert len(np.unique(leaves)) == len(leaves)
    depth = t["node_depth"][leaves]
    assert depth.min() >= cfg.start_depth and depth.max() == cfg.tree_depth
    lo, hi = t["node_position_min"][leaves], t["node_position_max"][leaves]
    assert np.all(hi[:, 2] > -cfg.slab) and np.all(lo[:, 2] < cfg.slab)
    # disjoint: no leaf is an ancestor of another (total volume = sum of parts)
    vol = np.prod(hi - lo, axis=1).sum()
    pts = np.random.default_rng(0).uniform(-1, 1, (20000, 3)) * np.array([1, 1, cfg.slab])
    inside = np.zeros(len(pts), int)
    for a, b in zip(lo, hi):
        inside += np.all((pts >= a) & (pts < b), axis=1)
    assert inside.max() == 1
    assert vol <= 8.0
    tree = syn.adaptive_tree(cfg, ph, device="cpu")
    assert np.array_equal(tree.active_node_ids.numpy(), leaves)
    assert int(tree.node_culled.sum()) == len(culled)
    assert not torch.any((tree.node_active == 1) & (tree.node_culled == 1))


def test_workload_generation_loads_nothing_native():
    """The reference arm of the benchmark generates the workload (phantom,
    rays, targets, adaptive leaves) without loading this package's native
    libraries."""
    import subprocess
    import sys

    code = (
        "import sys, dataclasses\n"
        "from adaptivetensordf_b200 import synthetic as syn\n"
        "from oracle import oracle as O\n"
        "cfg = dataclasses.replace(syn.CONFIGS['C5'], ellipsoids=100, target_leaves=200)\n"
        "ph = syn.config_phantom(cfg)\n"
        "o, d = syn.random_ray_batch(cfg, 64, 1)\n"
        "y = syn.analytic_projection(ph, o, d)\n"
        "t = O.tree_build(cfg.tree_depth)\n"
        "syn.adaptive_leaves(cfg, ph, t['node_position_min'], t['node_position_max'], t['node_children'],"
        " t['node_depth'])\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libatdf_b200' not in maps and '_atdf_host' not in maps, 'product library loaded'\n"
        "assert '_atdf_host' not in ''.join(sys.modules)\n"
        "print('ok')\n"
    )
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr[-2000:]


def test_analytic_projection_chunks_agree():
    """The ellipsoid chords summed in chunks equal one ellipsoid at a time."""
    from adaptivetensordf_b200 import synthetic as syn

    ph = syn.ellipsoid_phantom(37, 5)
    cfg = syn.CONFIGS["C2"]
    o, d = syn.random_ray_batch(cfg, 500, 3)
    a = syn.analytic_projection(ph, o, d, chunk=1)
    b = syn.analytic_projection(ph, o, d, chunk=16)
    assert np.allclose(a, b, rtol=1e-12, atol=1e-12) and a.max() > 0
