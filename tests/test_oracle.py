"""CPU checks of the oracle (test infrastructure) against closed-form known
answers and central finite differences. The reference ships no golden
vectors, so these are the oracle's pins (parity unpinned otherwise)."""

import math

import numpy as np
import pytest


def test_tree_build_octree(oracle):
    t = oracle.tree_build(2)
    assert len(t["node_depth"]) == 1 + 8 + 64
    # root and first child: child 0 is the lower octant, child 7 the upper one
    assert np.all(t["node_position_min"][0] == -1) and np.all(t["node_position_max"][0] == 1)
    assert np.all(t["node_position_min"][1] == -1) and np.all(t["node_position_max"][1] == 0)
    assert np.all(t["node_position_min"][8] == 0) and np.all(t["node_position_max"][8] == 1)
    # child 1 takes the upper half in x only (bit 0)
    assert list(t["node_position_min"][2]) == [0, -1, -1]
    assert list(t["node_children"][1]) == list(range(9, 17))
    oracle.set_active_depth(t, 2)
    assert len(t["active_node_ids"]) == 64 and t["active_node_ids"][0] == 9
    assert t["node_active_prefix_sum"][9] == 0 and t["node_active_prefix_sum"][0] == -1


def test_tree_build_quad(oracle):
    t = oracle.tree_build(2, quad=True, y_min=-0.5, y_max=0.5)
    assert len(t["node_depth"]) == 1 + 4 + 16
    assert np.all(t["node_position_min"][:, 1] == -0.5) and np.all(t["node_position_max"][:, 1] == 0.5)
    # child 1 splits x, child 2 splits z
    assert list(t["node_position_min"][2]) == [0, -0.5, -1]
    assert list(t["node_position_min"][3]) == [-1, -0.5, 0]


def test_intersect_box_cases(oracle):
    bmin, bmax = [0, 0, 0], [1, 1, 1]
    hit, t0, t1 = oracle.intersect_box(bmin, bmax, [0.5, 0.5, -2], [0, 0, 1])
    assert hit and t0 == 2.0 and t1 == 3.0
    # parallel ray on the min face is inside, on the max face outside ([min, max))
    assert oracle.intersect_box(bmin, bmax, [0.0, 0.5, -2], [0, 0, 1])[0]
    assert not oracle.intersect_box(bmin, bmax, [1.0, 0.5, -2], [0, 0, 1])[0]
    # miss and behind
    assert not oracle.intersect_box(bmin, bmax, [2, 2, -2], [0, 0, 1])[0]
    assert not oracle.intersect_box(bmin, bmax, [0.5, 0.5, 5], [0, 0, 1])[0]
    # origin inside: negative tmin
    hit, t0, t1 = oracle.intersect_box(bmin, bmax, [0.5, 0.5, 0.5], [0, 0, 1])
    assert hit and t0 == -0.5 and t1 == 0.5


def test_axis_aligned_samples_closed_form(oracle):
    """One leaf [-1,1]^3, ray along z: chord 2, diag 2*sqrt(3), n = ceil(M/sqrt(3))."""
    t = oracle.tree_build(0)
    oracle.set_active_depth(t, 0)
    o = np.array([[0.25, -0.5, -3.0]], np.float32)
    d = np.array([[0, 0, 1]], np.float32)
    M = 16
    segs, s = oracle.create_samples_for_rays(t, o, d, M)
    n = math.ceil(np.float32(np.float32(2.0) / np.float32(np.sqrt(np.float32(12.0)))) * M)
    assert segs["n"][0] == n
    assert segs["tmin"][0] == 2.0 and segs["tmax"][0] == 4.0
    step = 2.0 / n
    expect_t = 2.0 + (np.arange(n) + 0.5) * step
    assert np.allclose(s["ray_t"], expect_t, atol=1e-6)
    # midpoint samples: every Voronoi weight is one step (the end halves
    # reach to tmin / tmax)
    w = np.full(n, step)
    assert np.allclose(s["weight"], w, atol=1e-6)
    assert abs(s["weight"].sum() - 2.0) < 1e-5
    assert list(s["local_index_in_ray"]) == list(range(n))


def test_grazing_and_missing_rays(oracle):
    t = oracle.tree_build(1)
    oracle.set_active_depth(t, 1)
    # a ray along the y = 0 plane is parallel to the split plane: it lies in
    # the upper y cells ([0, 1) rule) only
    o = np.array([[-0.5, 0.0, -3.0], [5, 5, 5]], np.float32)
    d = np.array([[0, 0, 1], [0, 0, 1]], np.float32)
    segs = oracle.ray_segments(t, o, d, 8)
    nodes = segs["node"][segs["ray"] == 0]
    ymins = t["node_position_min"][nodes, 1]
    assert np.all(ymins == 0.0) and len(nodes) == 2
    assert segs["ray_seg_count"][1] == 0
    # a ray grazing an edge (hit length < 1e-5) is skipped
    o2 = np.array([[0.0, 0.0, -3.0]], np.float32)
    d2 = np.array([[1e-7, 0, 1]], np.float32)
    segs2 = oracle.ray_segments(t, o2, d2, 8)
    assert all(tmax - tmin >= 1e-5 for tmin, tmax in zip(segs2["tmin"], segs2["tmax"]))


def test_segments_sorted_and_contiguous(oracle):
    t = oracle.tree_build(3)
    oracle.set_active_depth(t, 3)
    rng = np.random.default_rng(3)
    R = 64
    th = rng.uniform(-1, 1, R)
    d = np.stack([np.sin(th), np.zeros(R), np.cos(th)], 1).astype(np.float32)
    o = (rng.uniform(-0.9, 0.9, (R, 3)) - np.sqrt(2) * d).astype(np.float32)
    segs = oracle.ray_segments(t, o, d, 8)
    for r in range(R):
        m = segs["ray"] == r
        tm = segs["tmin"][m]
        tx = segs["tmax"][m]
        assert np.all(np.diff(tm) >= 0)
        # consecutive leaves share their boundary along the ray
        assert np.allclose(tx[:-1], tm[1:], atol=1e-6)


def test_grid_sample_known_answers(oracle):
    rng = np.random.default_rng(0)
    g = rng.normal(size=(2, 3, 5, 7))
    # texel centres (align_corners = True) return texel values
    H, W = 5, 7
    ys, xs = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    uv = np.stack([xs.ravel() / (W - 1) * 2 - 1, ys.ravel() / (H - 1) * 2 - 1], 1)
    idx = np.ones(len(uv), np.int64)
    out = oracle.grid_sample2d(g, idx, uv, np.float64)
    assert np.allclose(out, g[1].reshape(3, -1).T, atol=1e-12)
    # outside the grid: border clamp
    out = oracle.grid_sample2d(g, np.array([0]), np.array([[3.0, -4.0]]), np.float64)
    assert np.allclose(out[0], g[0, :, 0, W - 1])
    # 1D: midpoint of two texels
    l = rng.normal(size=(1, 2, 4, 1))
    out = oracle.grid_sample1d(l, np.array([0]), np.array([[-1 + 1 / 3]]), np.float64)
    assert np.allclose(out[0], 0.5 * (l[0, :, 0, 0] + l[0, :, 1, 0]))


def _fd(fun, x, idx, h=1e-3):
    x[idx] += h
    fp = fun()
    x[idx] -= 2 * h
    fm = fun()
    x[idx] += h
    return (fp - fm) / (2 * h)


def test_grid_sample_adjoint_fd(oracle):
    rng = np.random.default_rng(1)
    g = rng.normal(size=(3, 4, 6, 5))
    S = 20
    idx = rng.integers(0, 3, S)
    uv = rng.uniform(-1.1, 1.1, (S, 2))
    go = rng.normal(size=(S, 4))
    gg, gu = oracle.grid_sample2d_bwd(g, idx, uv, go, np.float64)
    f = lambda: (oracle.grid_sample2d(g, idx, uv, np.float64) * go).sum()
    for i in [(0, 1, 2, 3), (2, 3, 5, 4), (1, 0, 0, 0)]:
        assert abs(_fd(f, g, i) - gg[i]) < 1e-7
    # uv derivative away from texel boundaries
    for s in range(3):
        for k in range(2):
            assert abs(_fd(f, uv, (s, k), 1e-6) - gu[s, k]) < 1e-4


def _random_scene(oracle, depth=2, C=4, G=5, L=9, cat=0, hidden=(8, 8), R=12, M=6, seed=0):
    rng = np.random.default_rng(seed)
    t = oracle.tree_build(depth)
    oracle.set_active_depth(t, depth)
    N = len(t["active_node_ids"])
    field = {
        "planes": [rng.uniform(-0.5, 0.5, (N, C, G, G)) for _ in range(3)],
        "lines": [rng.uniform(-0.5, 0.5, (1, C, L, 1)) for _ in range(3)],
        "leaf_slot": t["node_active_prefix_sum"],
        "cat": cat,
    }
    F = 3 * C if cat else C
    dims = [F, *hidden, 1]
    mlp = {"layers": [(rng.normal(0, 0.6, (dims[i + 1], dims[i])), rng.normal(0, 0.1, dims[i + 1]))
                      for i in range(len(dims) - 1)], "act": "silu", "last_act": "softplus", "beta": 2.0}
    th = rng.uniform(-1, 1, R)
    d = np.stack([np.sin(th), 0.1 * rng.normal(size=R), np.cos(th)], 1)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    o = (rng.uniform(-0.9, 0.9, (R, 3)) - np.sqrt(2) * d).astype(np.float32)
    segs, s = oracle.create_samples_for_rays(t, o, d, M)
    return t, field, mlp, o, d, segs, s


@pytest.mark.parametrize("cat", [0, 1])
def test_projection_adjoint_fd(oracle, cat):
    t, field, mlp, o, d, segs, s = _random_scene(oracle, cat=cat)
    R = o.shape[0]
    rng = np.random.default_rng(5)
    g = rng.normal(size=(1, R))
    grads = oracle.project_backward(field, mlp, t, s, R, g, np.float64)
    f = lambda: (oracle.project_forward(field, mlp, t, s, R, np.float64) * g).sum()
    for m in range(3):
        nz = np.argwhere(np.abs(grads["planes"][m]) > 1e-6)
        for i in nz[:: max(1, len(nz) // 3)][:3]:
            i = tuple(i)
            assert abs(_fd(f, field["planes"][m], i) - grads["planes"][m][i]) < 1e-7 * max(1, abs(grads["planes"][m][i])) + 1e-9
        nzl = np.argwhere(np.abs(grads["lines"][m]) > 1e-6)
        for i in nzl[:2]:
            i = tuple(i)
            assert abs(_fd(f, field["lines"][m], i) - grads["lines"][m][i]) < 1e-6
    for li, (W, b) in enumerate(mlp["layers"]):
        for i in [(0, 0), (W.shape[0] - 1, W.shape[1] - 1)]:
            assert abs(_fd(f, W, i) - grads["W"][li][i]) < 1e-5 * max(1, abs(grads["W"][li][i]))
        assert abs(_fd(f, b, (0,)) - grads["b"][li][0]) < 1e-5 * max(1, abs(grads["b"][li][0]))


def test_train_step_matches_composition(oracle):
    """The parallel CPU training step equals project fwd/bwd on the same samples."""
    t, field, mlp, o, d, segs, s = _random_scene(oracle, R=20, seed=3)
    R = o.shape[0]
    field32 = {**field, "planes": [p.astype(np.float32) for p in field["planes"]],
               "lines": [l.astype(np.float32) for l in field["lines"]]}
    mlp32 = {**mlp, "layers": [(w.astype(np.float32), b.astype(np.float32)) for w, b in mlp["layers"]]}
    y = np.random.default_rng(1).uniform(0, 1, R).astype(np.float32)
    loss, img, grads = oracle.train_step(t, field32, mlp32, o, d, y, 6, 0)
    img2 = oracle.project_forward(field32, mlp32, t, s, R, np.float64)
    assert np.allclose(img, img2, rtol=1e-5, atol=1e-6)
    gi = 2 * (img2 - y[None]) / R
    g2 = oracle.project_backward(field32, mlp32, t, s, R, gi, np.float64)
    for m in range(3):
        assert np.allclose(grads["planes"][m], g2["planes"][m], rtol=1e-4, atol=1e-7)
    for li in range(len(mlp["layers"])):
        assert np.allclose(grads["W"][li], g2["W"][li], rtol=1e-4, atol=1e-6)


def test_jitter_hash_and_node_error(oracle):
    a = [oracle.jitter(7, 3, 11, j) for j in range(100)]
    assert all(0.0 <= x < 1.0 for x in a)
    assert a == [oracle.jitter(7, 3, 11, j) for j in range(100)]
    assert abs(np.mean(a) - 0.5) < 0.1
    t, field, mlp, o, d, segs, s = _random_scene(oracle, R=10, seed=4)
    prl = np.random.default_rng(2).uniform(0, 1, (1, 10)).astype(np.float32)
    ls, ws = oracle.accumulate_loss_per_node(s, prl, len(t["node_depth"]))
    # the weights of one ray sum to its chord through the volume
    assert abs(ws.sum() - s["weight"].astype(np.float64).sum()) < 1e-9
    expect = np.zeros_like(ls)
    np.add.at(expect, s["node_id"], prl[0][s["ray_index"]].astype(np.float64) * s["weight"])
    assert np.allclose(ls, expect)


def test_gradient_correction_known_answers(oracle):
    """GradientCorrection's backward removes the gradient's component along
    the ray (GradientCorrection.cu:22-48): for a unit direction the result is
    orthogonal to it, a second application changes nothing, and a gradient
    along the ray vanishes. Axis-aligned cases are exact in FP32."""
    rng = np.random.default_rng(3)
    R, S = 50, 2000
    d = rng.normal(size=(R, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ray = rng.integers(0, R, S)
    g = rng.normal(size=(S, 3))
    out = oracle.gradient_correction_bwd(d, ray, g, np.float64)
    assert np.abs((out * d[ray]).sum(1)).max() < 1e-12
    again = oracle.gradient_correction_bwd(d, ray, out, np.float64)
    assert np.abs(again - out).max() < 1e-12
    along = oracle.gradient_correction_bwd(d, ray, 2.5 * d[ray], np.float64)
    assert np.abs(along).max() < 1e-12
    # FP32 restatement within rounding of the FP64 one
    out32 = oracle.gradient_correction_bwd(d.astype(np.float32), ray, g.astype(np.float32), np.float32)
    assert out32.dtype == np.float32 and np.abs(out32 - out).max() < 1e-5
    ax = np.array([[0.0, 0.0, 1.0]], np.float32)
    gg = np.array([[1.5, -2.0, 7.0]], np.float32)
    assert np.array_equal(oracle.gradient_correction_bwd(ax, [0], gg), np.array([[1.5, -2.0, 0.0]], np.float32))
