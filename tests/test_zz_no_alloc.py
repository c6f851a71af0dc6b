"""The forward projection entry point that allocates nothing.

Some callers cannot call cudaMalloc: a plugin whose host framework owns every
device allocation, or a loop where an allocation would synchronise the device.
atdf_project_forward_noalloc serves them by taking its workspace from a fixed
device array inside the library. This file is collected last so that a run
stopping at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

from tests.scene import rays_through_volume, rel_err

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def _call_both(L, capi, t, f, m, o, d, M, seed, stream):
    R = o.shape[0]
    o_t, d_t = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    size = ct.c_size_t(0)
    assert L.atdf_project_workspace_size(R, t.max_depth, t.ns, f.num_slots, 1, ct.byref(size)) == 0
    ws = torch.empty(size.value, dtype=torch.uint8, device="cuda")
    img_ref = torch.empty(1, R, device="cuda")
    img = torch.full((1, R), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.atdf_project_forward(ct.byref(t), ct.byref(f), ct.byref(m), capi.ptr(o_t), capi.ptr(d_t), R, M, seed,
                                  capi.ptr(img_ref), capi.ptr(ws), size.value, capi.ptr(err), stream) == 0
    assert L.atdf_project_forward_noalloc(ct.byref(t), ct.byref(f), ct.byref(m), capi.ptr(o_t), capi.ptr(d_t), R, M,
                                          seed, capi.ptr(img), capi.ptr(err), stream) == 0
    torch.cuda.synchronize()
    assert err.item() == 0
    return img.cpu().numpy(), img_ref.cpu().numpy()


def test_noalloc_forward_matches_allocating_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from adaptivetensordf_b200 import capi
    from adaptivetensordf_b200 import synthetic as syn

    L = capi.lib()
    tree = syn.make_tree(3, device="cuda")
    geo = syn.make_geometry(tree, 16, 17, (128, 17, 128), [64, 64], seed=5)
    t = capi.tree_struct(tree)
    f, keep_f = capi.field_struct(geo)
    m, keep_m = capi.mlp_struct(geo)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row: the second reuses the scratch the first one left
    for call, (R, seed) in enumerate([(3000, 11), (2200, 0)]):
        o, d = rays_through_volume(R, seed=100 + call)
        img, ref = _call_both(L, capi, t, f, m, o, d, 16, seed, stream)
        assert np.all(np.isfinite(img))
        assert rel_err(img, ref) < REL_TOL, call

    # a problem larger than the scratch array is refused before any launch
    big = 40000
    size = ct.c_size_t(0)
    assert L.atdf_project_workspace_size(big, t.max_depth, t.ns, f.num_slots, 1, ct.byref(size)) == 0
    assert size.value > (16 << 20)
    o, d = rays_through_volume(big, seed=7)
    o_t, d_t = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    img = torch.zeros(1, big, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = L.atdf_project_forward_noalloc(ct.byref(t), ct.byref(f), ct.byref(m), capi.ptr(o_t), capi.ptr(d_t), big, 16,
                                        0, capi.ptr(img), capi.ptr(err), stream)
    assert st == 3  # ATDF_ERR_WORKSPACE
    assert L.atdf_status_string(st) == b"workspace too small"
