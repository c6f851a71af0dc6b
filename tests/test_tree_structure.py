"""CPU tests of the tree-structure optimisation (the reference's OR-Tools MIP,
HyperTreeStructureOptimizer.cpp:5-392, solved exactly here by dynamic
programming): splits go to the leaves with the largest error x density, the
active-leaf budget holds, low-error sibling groups merge to make room, and
on small trees the solution's objective equals the brute-force optimum of
the same program."""

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


def _quad_tree(extra_split=None, culled=()):
    """Quad tree of depth 3 with its 16 depth-2 nodes active; optionally one
    of them split into its 4 children, and some depth-3 nodes culled."""
    from adaptivetensordf_b200 import HyperTreeBase

    t = HyperTreeBase(3, 3)
    t.settree(True, -1.0, 1.0)
    act = (t.node_depth == 2).to(torch.int32)
    if extra_split is not None:
        act[extra_split] = 0
        for c in t.node_children[extra_split].tolist():
            act[c] = 1
    cul = torch.zeros_like(act)
    for c in culled:
        cul[c] = 1
        act[c] = 0
    t.node_active = act
    t.node_culled = cul
    t.UpdateActive()
    return t


def _program(t, mf, sf):
    """The reference's program as items: (parent or -1, members) where a
    member is (node, none cost, split cost or None, live children)."""
    ns = t.NS()
    act = t.node_active.tolist()
    cul = t.node_culled.tolist()
    ch = t.node_children.tolist()
    err = [max(float(e), 0.0) for e in t.node_error.tolist()]
    den = [float(d) if d >= 0 else 1.0 for d in t.node_max_density.tolist()]

    def member(i):
        live = sum(1 for c in ch[i] if c >= 0 and not cul[c]) if ch[i][0] >= 0 else 0
        return (i, err[i] * den[i], sf * err[i] * den[i] if live else None, live)

    items, grouped = [], set()
    for p in range(len(act)):
        if ch[p][0] < 0 or act[p] == 1:
            continue
        kids = ch[p]
        na = sum(act[c] == 1 for c in kids)
        nc = sum(act[c] != 1 and cul[c] == 1 for c in kids)
        if na == 0 or na + nc != ns:
            continue
        mem = [member(c) for c in kids if act[c] == 1]
        merge = mf * sum(err[c] for c in kids if act[c] == 1) * max(den[c] for c in kids if act[c] == 1)
        items.append((p, mem, merge))
        grouped.update(c for c in kids if act[c] == 1)
    for i in range(len(act)):
        if act[i] == 1 and i not in grouped:
            items.append((-1, [member(i)], None))
    return items


def _brute_force(items, budget):
    import itertools

    per_item = []
    for parent, mem, merge in items:
        opts = []
        for combo in itertools.product(*[[0, 1] if m[2] is not None else [0] for m in mem]):
            opts.append((sum(m[3] if c else 1 for m, c in zip(mem, combo)),
                         sum(m[2] if c else m[1] for m, c in zip(mem, combo))))
        if parent >= 0:
            opts.append((1, merge))
        per_item.append(opts)
    best = {0: 0.0}  # count -> cheapest cost
    for opts in per_item:
        nxt = {}
        for b, c in best.items():
            for n, v in opts:
                if b + n <= budget and c + v < nxt.get(b + n, float("inf")):
                    nxt[b + n] = c + v
        best = nxt
    return min(best.values())


def _objective_of_result(items, act_after):
    total = 0.0
    for parent, mem, merge in items:
        if parent >= 0 and act_after[parent] == 1:
            total += merge
            continue
        for node, none, split, live in mem:
            total += none if act_after[node] == 1 else split
    return total


def test_exact_optimum_on_small_trees():
    import numpy as np

    rng = np.random.default_rng(7)
    for case in range(12):
        extra = [None, 9, 14][case % 3]
        t0 = _quad_tree(extra)
        depth3 = [n for n in range(t0.NumNodes()) if int(t0.node_depth[n]) == 3]
        culled = [int(c) for c in rng.choice(depth3, 6, replace=False)
                  if extra is None or int(t0.node_parent[int(c)]) != extra]
        t = _quad_tree(extra, culled)
        err = torch.from_numpy(rng.exponential(1.0, t.NumNodes()).astype(np.float32))
        err[torch.from_numpy(rng.random(t.NumNodes()) < 0.2)] = 0.0
        t.SetErrorForActiveNodes(err, "override")
        t.node_max_density = torch.from_numpy(rng.uniform(0.0, 1.0, t.NumNodes()).astype(np.float32))
        mf, sf = [(1.1, 0.75), (1.3, 0.5), (1.05, 0.9)][case % 3]
        items = _program(t, mf, sf)
        n_active = int(t.node_active.sum())
        for budget in (n_active - 6, n_active, n_active + 9, n_active + 30):
            opt = _brute_force(items, budget)
            tt = _quad_tree(extra, culled)
            tt.SetErrorForActiveNodes(err, "override")
            tt.node_max_density = t.node_max_density.clone()
            tt.OptimizeStructure(budget, mf, sf)
            after = tt.node_active.tolist()
            assert sum(after) <= budget
            got = _objective_of_result(items, after)
            assert abs(got - opt) <= 1e-9 * max(1.0, abs(opt)), (case, budget, got, opt)
