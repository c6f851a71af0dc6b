"""Device-side error words: every data-dependent problem a kernel meets sets a
bit in the caller's error word, skips the access and leaves the context
usable; the host layer turns a set bit into an exception (c10::Error, a
RuntimeError in Python). The reference only has a compiled-out assert
(hyperacorn/csrc/structure/HyperTree.cu:342) and a CHECK after the
out-of-bounds write has already happened (HyperTree.cu:554).

Each case is provoked with inputs whose every access was checked by reading
the kernels: capacities that are too small (the writes are guarded by the
capacity), a ray crossing more leaves than the hit list holds (the list
stops at 256), and ids beyond their arrays (rejected before the access).
Guard regions after each output must stay untouched."""

import ctypes as ct
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _stream():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def _segments(capi, R, cap, guard=64):
    """Segment arrays of `cap` entries plus a guard region filled with a
    sentinel; returns (struct, keep-alive dict)."""
    t = {
        "seg_off": torch.zeros(R + 1, dtype=torch.int64, device="cuda"),
        "smp_off": torch.zeros(R + 1, dtype=torch.int64, device="cuda"),
        "totals": torch.zeros(4, dtype=torch.int64, device="cuda"),
    }
    for k in ("node", "nsamp", "ray", "first"):
        t[k] = torch.full((cap + guard,), -7, dtype=torch.int32, device="cuda")
    for k in ("tmin", "tmax"):
        t[k] = torch.full((cap + guard,), -7.0, dtype=torch.float32, device="cuda")
    s = capi.Segments()
    s.ray_seg_offset = t["seg_off"].data_ptr()
    s.ray_sample_offset = t["smp_off"].data_ptr()
    s.node, s.tmin, s.tmax = t["node"].data_ptr(), t["tmin"].data_ptr(), t["tmax"].data_ptr()
    s.nsamp, s.ray, s.first = t["nsamp"].data_ptr(), t["ray"].data_ptr(), t["first"].data_ptr()
    s.capacity = cap
    s.totals = t["totals"].data_ptr()
    return s, t


def _rays(R, seed):
    from tests.scene import rays_through_volume

    o, d = rays_through_volume(R, seed)
    return torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()


def test_segment_capacity_bit_and_guard():
    from adaptivetensordf_b200 import capi
    from adaptivetensordf_b200 import synthetic as syn

    L = capi.lib()
    tree = syn.make_tree(3, device="cuda")
    t = capi.tree_struct(tree)
    R = 500
    o, d = _rays(R, 1)
    # enough room: no bit, and the count tells how much is needed
    full, keep_full = _segments(capi, R, R * 27)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.atdf_ray_segments(ct.byref(t), capi.ptr(o), capi.ptr(d), R, 16, ct.byref(full), capi.ptr(err),
                               _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() == 0
    need = int(keep_full["totals"][0].item())
    assert need > 100
    # a third of it: the bit is set, nothing is written past the capacity,
    # and the rays that fit are written as in the full run
    cap = need // 3
    small, keep = _segments(capi, R, cap)
    assert L.atdf_ray_segments(ct.byref(t), capi.ptr(o), capi.ptr(d), R, 16, ct.byref(small), capi.ptr(err),
                               _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() & capi.DEVERR["seg_capacity"]
    assert err.item() == capi.DEVERR["seg_capacity"]
    for k in ("node", "nsamp", "ray", "first", "tmin", "tmax"):
        assert torch.all(keep[k][cap:] == -7), k
    seg_off = keep["seg_off"].cpu().numpy()
    fits = np.nonzero(seg_off[1:] <= cap)[0]
    last = int(seg_off[fits[-1] + 1])
    for k in ("node", "nsamp", "ray", "first", "tmin", "tmax"):
        assert torch.equal(keep[k][:last], keep_full[k][:last]), k
    # the host layer raises instead of returning partial results
    import adaptivetensordf_b200 as ab

    sg = tree.RaySegments(ab.RayList(o, d), 16)
    assert sg.num_segments == need


def test_sample_capacity_bit_and_guard():
    from adaptivetensordf_b200 import capi
    from adaptivetensordf_b200 import synthetic as syn

    L = capi.lib()
    tree = syn.make_tree(2, device="cuda")
    t = capi.tree_struct(tree)
    R = 300
    o, d = _rays(R, 2)
    segs, keep = _segments(capi, R, R * 15)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.atdf_ray_segments(ct.byref(t), capi.ptr(o), capi.ptr(d), R, 8, ct.byref(segs), capi.ptr(err),
                               _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() == 0
    S = int(keep["totals"][1].item())
    cap, guard = S // 2, 128
    pos = torch.full((cap + guard, 3), -7.0, device="cuda")
    tt = torch.full((cap + guard,), -7.0, device="cuda")
    w = torch.full((cap + guard,), -7.0, device="cuda")
    ri = torch.full((cap + guard,), -7, dtype=torch.int64, device="cuda")
    li = torch.full((cap + guard,), -7, dtype=torch.int64, device="cuda")
    ni = torch.full((cap + guard,), -7, dtype=torch.int64, device="cuda")
    assert L.atdf_emit_samples(ct.byref(segs), R, capi.ptr(o), capi.ptr(d), None, 0, capi.ptr(pos), capi.ptr(tt),
                               capi.ptr(w), capi.ptr(ri), capi.ptr(li), capi.ptr(ni), cap, capi.ptr(err),
                               _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() == capi.DEVERR["sample_capacity"]
    assert torch.all(pos[cap:] == -7.0) and torch.all(tt[cap:] == -7.0) and torch.all(w[cap:] == -7.0)
    assert torch.all(ri[cap:] == -7) and torch.all(li[cap:] == -7) and torch.all(ni[cap:] == -7)
    assert torch.all(tt[:cap] != -7.0)  # everything below the capacity is written


def test_hit_overflow_bit():
    """A ray along the diagonal of a depth-8 quad tree (256 x 256 leaves in
    x and z) crosses about 511 leaves, more than the 256-entry hit list
    (the reference's max_intersections, HyperTree.cu:280)."""
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import capi
    from adaptivetensordf_b200 import synthetic as syn

    L = capi.lib()
    tree = syn.make_tree(8, device="cuda", quad=True)
    t = capi.tree_struct(tree)
    d = np.array([[1.0, 0.0, 1.0], [0.0, 0.0, 1.0]], np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.array([[-1.5 + 1e-3, 0.1, -1.5], [0.3, 0.1, -2.0]], np.float32)
    ot, dt = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    R = 2
    segs, keep = _segments(capi, R, R * 256)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.atdf_ray_segments(ct.byref(t), capi.ptr(ot), capi.ptr(dt), R, 4, ct.byref(segs), capi.ptr(err),
                               _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() == capi.DEVERR["hit_overflow"]
    off = keep["seg_off"].cpu().numpy()
    assert off[1] - off[0] == 256  # the list stops at its capacity
    assert off[2] - off[1] == 256  # the axis-aligned ray: 256 leaves in z, exactly full
    assert torch.all(keep["node"][2 * 256:] == -7)
    with pytest.raises(RuntimeError, match="more than 256 leaves"):
        tree.RaySegments(ab.RayList(ot[:1], dt[:1]), 4)
    # the context stays usable: the axis-aligned ray alone is fine
    sg = tree.RaySegments(ab.RayList(ot[1:], dt[1:]), 4)
    assert sg.num_segments == 256


def test_index_bits():
    """Node ids and plane slots beyond their arrays: the index bit is set, the
    access is skipped (zero features, untouched outputs), and the host layer
    raises."""
    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import capi
    from adaptivetensordf_b200 import synthetic as syn

    L = capi.lib()
    tree = syn.make_tree(2, device="cuda")
    geo = syn.make_geometry(tree, 8, 9, (32, 9, 32), [32], seed=4)
    nn = tree.NumNodes()
    # local samples with a node id past the tree
    P = 64
    pos = torch.rand(P, 3, device="cuda") * 2 - 1
    node = tree.active_node_ids[:P].clone()
    node[5] = nn + 10
    out = torch.full((P, 3), -7.0, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.atdf_local_samples(capi.ptr(pos), capi.ptr(node), P, 1, capi.ptr(tree.node_position_min),
                                capi.ptr(tree.node_position_max), nn, capi.ptr(out), capi.ptr(err),
                                _stream()) == 0
    torch.cuda.synchronize()
    assert err.item() == capi.DEVERR["index"]
    assert torch.all(out[5] == -7.0) and torch.all(out[6] != -7.0)
    # a plane slot past the planes (unfused feature op): zero features
    slot = geo.leaf_slot.clone()
    bad_leaf = int(tree.active_node_ids[3].item())
    slot[bad_leaf] = geo.planes[0].shape[0] + 4
    geo.leaf_slot = slot
    f, keep_f = capi.field_struct(geo)
    s = tree.CreateSamplesForRays(ab.RayList(*_rays(200, 3)), 8, False)
    S = s.size()
    feat = torch.full((S, 8), -7.0, device="cuda")
    err.zero_()
    assert L.atdf_vm_features_forward(ct.byref(f), capi.ptr(tree.node_position_min), capi.ptr(tree.node_position_max),
                                      nn, capi.ptr(s.global_coordinate), capi.ptr(s.node_id), S, capi.ptr(feat),
                                      capi.ptr(err), _stream()) == 0
    torch.cuda.synchronize()
    hit_bad = s.node_id == bad_leaf
    assert bool(hit_bad.any())
    assert err.item() == capi.DEVERR["index"]
    assert torch.all(feat[hit_bad] == 0.0) and torch.all(feat[~hit_bad] != -7.0)
    with pytest.raises(RuntimeError, match="index out of range"):
        geo.SampleVolumeIndirect_feature(tree, s.global_coordinate, s.node_id)
    # the fused projection: the segment joins the out-of-ROI bucket, the bit
    # accumulates in the geometry's error word (no read-back on the hot path)
    # and CheckErrors raises and clears it
    img = geo.ProjectRays(tree, ab.RayList(*_rays(200, 3)), 8, 0)
    img.sum().backward()
    with pytest.raises(RuntimeError, match="index out of range"):
        geo.CheckErrors()
    geo.CheckErrors()  # cleared
    # the context stays usable
    geo.leaf_slot = tree.node_active_prefix_sum.cuda()
    img = geo.ProjectRays(tree, ab.RayList(*_rays(200, 3)), 8, 0)
    assert bool(torch.isfinite(img).all())
    geo.CheckErrors()
