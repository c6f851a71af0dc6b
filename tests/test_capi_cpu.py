"""CPU checks of the boundary: the C-ABI library loads and exports every
symbol include/atdf.h declares; the host extension mirrors the reference's
tree construction; and the product path refuses CPU tensors (no fallback)."""

import ctypes as ct

import numpy as np
import pytest
import torch


def test_capi_exports_every_declared_symbol():
    from adaptivetensordf_b200 import capi

    names = capi.declared_symbols()
    assert len(names) >= 20
    lib = ct.CDLL(capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    L = capi.lib()
    assert L.atdf_version() == 100
    assert L.atdf_status_string(0) == b"ok"


def test_capi_argument_validation_without_gpu():
    """Invalid arguments are rejected on the host before any launch."""
    from adaptivetensordf_b200 import capi

    L = capi.lib()
    size = ct.c_size_t(0)
    assert L.atdf_project_workspace_size(1024, 4, 8, 4096, 1, ct.byref(size)) == 0
    assert size.value > 1024 * 24
    assert L.atdf_project_workspace_size(1024, 4, 5, 4096, 1, ct.byref(size)) == 1
    assert L.atdf_project_workspace_size(1024, 4, 8, 4096, 2, ct.byref(size)) == 1
    t = capi.Tree()
    assert L.atdf_ray_segments(ct.byref(t), None, None, 4, 8, None, None, None) == 1
    assert L.atdf_grid_sample2d_forward(None, 1, 1, 1, 1, None, None, None, 0, None, None, None) == 1


def test_host_tree_matches_oracle(oracle):
    import adaptivetensordf_b200 as ab

    for depth, quad in [(2, False), (3, True)]:
        t = ab.HyperTreeBase(3, depth)
        t.settree(quad, -0.5, 0.5)
        t.SetActive(depth)
        o = oracle.tree_build(depth, quad=quad, y_min=-0.5, y_max=0.5)
        assert np.array_equal(t.node_position_min.numpy(), o["node_position_min"])
        assert np.array_equal(t.node_position_max.numpy(), o["node_position_max"])
        assert np.array_equal(t.node_children.numpy(), o["node_children"])
        oracle.set_active_depth(o, depth)
        assert np.array_equal(t.active_node_ids.numpy(), o["active_node_ids"])
        assert np.array_equal(t.node_active_prefix_sum.numpy(), o["node_active_prefix_sum"])
        fl = t.node_flags.numpy()
        assert np.all(fl[o["active_node_ids"]] == 1) and fl[0] == 2


def test_host_set_error_for_active_nodes():
    import adaptivetensordf_b200 as ab

    t = ab.HyperTreeBase(3, 1)
    t.settree(False)
    t.SetActive(1)
    err = torch.arange(9, dtype=torch.float32)
    t.SetErrorForActiveNodes(err, "override")
    assert t.node_error[0].item() == -1 and t.node_error[1:].tolist() == list(range(1, 9))
    t.SetErrorForActiveNodes(torch.zeros(9), "min")
    assert t.node_error[1:].tolist() == [0.0] * 8


def test_product_path_refuses_cpu_tensors():
    import adaptivetensordf_b200 as ab

    g = torch.zeros(2, 3, 4, 4)
    with pytest.raises(RuntimeError, match="CUDA"):
        ab.IndirectGridSample2D(g, torch.zeros(3, dtype=torch.long), torch.zeros(3, 2))
    t = ab.HyperTreeBase(3, 1)
    t.settree(False)
    t.SetActive(1)
    rays = ab.RayList(torch.zeros(2, 3), torch.ones(2, 3))
    with pytest.raises(RuntimeError, match="CUDA"):
        t.CreateSamplesForRays(rays, 8, False)
