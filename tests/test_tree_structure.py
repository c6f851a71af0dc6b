"""CPU tests of the greedy tree-structure optimisation (the reference's
OR-Tools MIP, HyperTreeStructureOptimizer.cpp): splits go to the leaves with
the largest error x density, the active-leaf budget holds, and low-error
sibling groups merge to make room."""

import torch


def _tree(depth, active_depth):
    from adaptivetensordf_b200 import HyperTreeBase

    t = HyperTreeBase(3, depth)
    t.settree(False, -1.0, 1.0)
    t.SetActive(active_depth)
    return t


def test_split_highest_error_leaves_within_budget():
    t = _tree(3, 1)  # 8 active leaves at depth 1
    err = torch.zeros(t.NumNodes())
    ids = t.active_node_ids.tolist()
    err[ids[3]] = 5.0
    err[ids[6]] = 2.0
    err[ids[0]] = 0.1
    t.SetErrorForActiveNodes(err, "override")
    t.node_max_density = torch.ones(t.NumNodes())
    # budget for one split (8 - 1 + 8 = 15 leaves)
    assert t.OptimizeStructure(15, 1.1, 0.75)
    act = t.node_active
    assert int(act.sum()) == 15
    assert act[ids[3]] == 0 and all(act[c] == 1 for c in t.node_children[ids[3]].tolist())
    assert act[ids[6]] == 1
    assert list(t.active_node_ids.tolist()) == sorted(t.active_node_ids.tolist())
    assert int(t.node_active_prefix_sum[t.active_node_ids[-1]]) == 14


def test_merge_to_meet_budget_and_pay_for_splits():
    t = _tree(3, 2)  # 64 leaves at depth 2
    err = torch.full((t.NumNodes(),), 0.01)
    ids = t.active_node_ids.tolist()
    hot = ids[17]
    err[hot] = 10.0
    t.SetErrorForActiveNodes(err, "override")
    t.node_max_density = torch.ones(t.NumNodes())
    # budget 64: the split of the hot leaf (+7) must be paid by a merge (-7)
    assert t.OptimizeStructure(64, 1.1, 0.75)
    act = t.node_active
    assert int(act.sum()) <= 64
    assert act[hot] == 0
    parent_of_hot = int(t.node_parent[hot])
    assert act[parent_of_hot] == 0  # the hot leaf's own sibling group is not merged
    # budget smaller than the leaf count: merges only
    t2 = _tree(3, 2)
    t2.SetErrorForActiveNodes(torch.full((t2.NumNodes(),), 0.5), "override")
    t2.node_max_density = torch.ones(t2.NumNodes())
    assert t2.OptimizeStructure(40, 1.1, 0.75)
    assert int(t2.node_active.sum()) <= 40


def test_no_change_without_gain():
    t = _tree(2, 1)
    t.SetErrorForActiveNodes(torch.zeros(t.NumNodes()), "override")
    t.node_max_density = torch.ones(t.NumNodes())
    assert not t.OptimizeStructure(64, 1.1, 0.75)
    assert int(t.node_active.sum()) == 8
