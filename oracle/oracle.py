"""ctypes front end of the CPU oracle (oracle/atdf_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` leg of ``bench.py``, never by the product.
PARITY UNPINNED: the reference ships no golden vectors and cannot be built
here; the oracle is a restatement of its source, checked by known answers and
finite differences (see the header of atdf_oracle.cpp for the citations).

Arrays are numpy. Planes use the reference layout [N, C, H, W]; lines
[1, C, L, 1]; the decoder is a list of (W [out, in], b [out]) pairs.
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libatdf_oracle.so")

ACT = {"id": 0, "none": 0, "relu": 1, "silu": 2, "sigmoid": 3, "softplus": 4, "leakyrelu": 5, "abs": 6, "tanh": 7}

_lib = None


def build():
    """Compile the oracle library (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ct.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


P = ct.c_void_p
I64 = ct.c_int64
I32 = ct.c_int
F = ct.c_float


def _declare(L):
    L.orc_tree_build.restype = I64
    L.orc_tree_build.argtypes = [I32, I32, F, F, P, P, P, P, P]
    L.orc_intersect_box.restype = I32
    L.orc_intersect_box.argtypes = [P, P, P, P, P, P]
    L.orc_ray_segments.restype = I64
    L.orc_ray_segments.argtypes = [P, P, P, I64, P, P, I64, I32, P, P, I64, P, P, P, P, P, P]
    L.orc_emit_samples.restype = None
    L.orc_emit_samples.argtypes = [I64, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P]
    L.orc_jitter.restype = F
    L.orc_jitter.argtypes = [ct.c_uint64, ct.c_int32, ct.c_int32, ct.c_int32]
    L.orc_jitter_for_segments.restype = None
    L.orc_jitter_for_segments.argtypes = [ct.c_uint64, I64, P, P, P, P]
    L.orc_local_samples.restype = None
    L.orc_local_samples.argtypes = [I64, P, P, I64, P, P, P]
    L.orc_node_id_for_position.restype = None
    L.orc_node_id_for_position.argtypes = [I64, P, P, P, P, I32, P, I64, P, P]
    L.orc_accumulate_loss_per_node.restype = None
    L.orc_accumulate_loss_per_node.argtypes = [I64, P, P, P, P, I64, I64, I64, P, P]
    L.orc_num_threads.restype = I32
    L.orc_train_step_f32.restype = ct.c_double
    L.orc_train_step_f32.argtypes = (
        [P, P, P, I64, P, P, P, I64, I32, ct.c_uint64, I32, I32, P, P, P, P, P, P, P, P]
        + [I32, P, P, P, I32, I32, ct.c_double, P, P, P, P, P, P, P]
    )
    for suf in ("f32", "f64"):
        getattr(L, f"orc_grid_sample2d_fwd_{suf}").argtypes = [P, I64, I64, I32, I32, P, P, I64, P]
        getattr(L, f"orc_grid_sample2d_bwd_{suf}").argtypes = [P, I64, I64, I32, I32, P, P, I64, P, P, P]
        getattr(L, f"orc_grid_sample1d_fwd_{suf}").argtypes = [P, I64, I64, I32, P, P, I64, P]
        getattr(L, f"orc_grid_sample1d_bwd_{suf}").argtypes = [P, I64, I64, I32, P, P, I64, P, P, P]
        field = [I32, I32, P, P, P, P, P, P, P, P, P, P]
        mlp = [I32, P, P, P, I32, I32, ct.c_double]
        getattr(L, f"orc_vm_features_{suf}").argtypes = field + [I64, P, P, P]
        getattr(L, f"orc_vm_features_bwd_{suf}").argtypes = field + [I64, P, P, P, P, P]
        getattr(L, f"orc_mlp_fwd_{suf}").argtypes = mlp + [I64, P, P]
        getattr(L, f"orc_mlp_bwd_{suf}").argtypes = mlp + [I64, P, P, P, P, P]
        getattr(L, f"orc_project_fwd_{suf}").argtypes = field + mlp + [I64, P, P, P, P, I64, P]
        getattr(L, f"orc_project_bwd_{suf}").argtypes = field + mlp + [I64, P, P, P, P, I64, P, P, P, P, P]


def _p(a):
    return None if a is None else a.ctypes.data_as(P)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr_array(arrs):
    """Keeps the arrays alive with the pointer table."""
    t = (P * len(arrs))(*[a.ctypes.data for a in arrs])
    return t


def _suffix(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


# ----------------------------------------------------------------------------
# tree
# ----------------------------------------------------------------------------
def tree_build(max_depth, quad=False, y_min=-1.0, y_max=1.0):
    L = lib()
    n = L.orc_tree_build(max_depth, int(quad), y_min, y_max, None, None, None, None, None)
    ns = 4 if quad else 8
    t = {
        "node_position_min": np.zeros((n, 3), np.float32),
        "node_position_max": np.zeros((n, 3), np.float32),
        "node_children": np.zeros((n, ns), np.int32),
        "node_depth": np.zeros(n, np.int32),
        "node_parent": np.zeros(n, np.int32),
    }
    L.orc_tree_build(max_depth, int(quad), y_min, y_max, _p(t["node_position_min"]), _p(t["node_position_max"]),
                     _p(t["node_children"]), _p(t["node_depth"]), _p(t["node_parent"]))
    t["ns"] = ns
    t["max_depth"] = max_depth
    return t


def set_active(tree, node_active):
    """UpdateActive (HyperTree.cpp:550-588): active ids ascending and the
    active prefix sum (-1 for inactive nodes)."""
    node_active = np.asarray(node_active, np.int32)
    tree["node_active"] = node_active
    ids = np.nonzero(node_active == 1)[0].astype(np.int64)
    pref = -np.ones(len(node_active), np.int64)
    pref[ids] = np.arange(len(ids))
    tree["active_node_ids"] = ids
    tree["node_active_prefix_sum"] = pref
    return tree


def set_active_depth(tree, depth):
    """SetActive(depth) (HyperTree.cpp:544-548)."""
    return set_active(tree, (tree["node_depth"] == depth).astype(np.int32))


# ----------------------------------------------------------------------------
# sampling
# ----------------------------------------------------------------------------
def intersect_box(bmin, bmax, o, d):
    L = lib()
    a = [_c(x, np.float32) for x in (bmin, bmax, o, d)]
    tmin = np.zeros(1, np.float32)
    tmax = np.zeros(1, np.float32)
    hit = L.orc_intersect_box(*[_p(x) for x in a], _p(tmin), _p(tmax))
    return bool(hit), float(tmin[0]), float(tmax[0])


def ray_segments(tree, origin, direction, max_samples_per_node, active_ids=None):
    L = lib()
    if active_ids is None:
        active_ids = tree["active_node_ids"]
    act = _c(active_ids, np.int64)
    o = _c(origin, np.float32)
    d = _c(direction, np.float32)
    R = o.shape[0]
    pmin = _c(tree["node_position_min"], np.float32)
    pmax = _c(tree["node_position_max"], np.float32)
    sc = np.zeros(R, np.int64)
    nc = np.zeros(R, np.int64)
    total = L.orc_ray_segments(_p(pmin), _p(pmax), _p(act), len(act), _p(o), _p(d), R, int(max_samples_per_node),
                               _p(sc), _p(nc), 0, None, None, None, None, None, None)
    out = {
        "node": np.zeros(total, np.int32),
        "tmin": np.zeros(total, np.float32),
        "tmax": np.zeros(total, np.float32),
        "n": np.zeros(total, np.int32),
        "ray": np.zeros(total, np.int32),
        "first": np.zeros(total, np.int32),
    }
    L.orc_ray_segments(_p(pmin), _p(pmax), _p(act), len(act), _p(o), _p(d), R, int(max_samples_per_node),
                       _p(sc), _p(nc), total, _p(out["node"]), _p(out["tmin"]), _p(out["tmax"]), _p(out["n"]),
                       _p(out["ray"]), _p(out["first"]))
    out["ray_seg_count"] = sc
    out["ray_sample_count"] = nc
    return out


def jitter(seed, ray, node, j):
    return lib().orc_jitter(seed, ray, node, j)


def jitter_for_segments(seed, segs):
    S = int(segs["n"].sum())
    out = np.zeros(S, np.float32)
    lib().orc_jitter_for_segments(seed, len(segs["n"]), _p(segs["node"]), _p(segs["n"]), _p(segs["ray"]), _p(out))
    return out


def emit_samples(segs, origin, direction, rnd=None):
    """SampleList in canonical order: global_coordinate, ray_t, weight,
    ray_index, local_index_in_ray, node_id."""
    L = lib()
    S = int(segs["n"].astype(np.int64).sum())
    o = _c(origin, np.float32)
    d = _c(direction, np.float32)
    r = None if rnd is None else _c(rnd, np.float32)
    out = {
        "global_coordinate": np.zeros((S, 3), np.float32),
        "ray_t": np.zeros(S, np.float32),
        "weight": np.zeros(S, np.float32),
        "ray_index": np.zeros(S, np.int64),
        "local_index_in_ray": np.zeros(S, np.int64),
        "node_id": np.zeros(S, np.int64),
    }
    L.orc_emit_samples(len(segs["n"]), _p(segs["node"]), _p(segs["tmin"]), _p(segs["tmax"]), _p(segs["n"]),
                       _p(segs["ray"]), _p(segs["first"]), _p(o), _p(d), _p(r), _p(out["global_coordinate"]),
                       _p(out["ray_t"]), _p(out["weight"]), _p(out["ray_index"]), _p(out["local_index_in_ray"]),
                       _p(out["node_id"]))
    return out


def create_samples_for_rays(tree, origin, direction, max_samples_per_node, rnd=None):
    segs = ray_segments(tree, origin, direction, max_samples_per_node)
    s = emit_samples(segs, origin, direction, rnd)
    s["max_samples_per_ray"] = int(segs["ray_sample_count"].max()) if len(segs["ray_sample_count"]) else 0
    return segs, s


def local_samples(tree, pos, node, group=1):
    pos = _c(pos, np.float32)
    node = _c(node, np.int64)
    P_ = pos.reshape(-1, 3).shape[0]
    out = np.zeros((P_, 3), np.float32)
    lib().orc_local_samples(P_, _p(pos), _p(node), group, _p(_c(tree["node_position_min"], np.float32)),
                            _p(_c(tree["node_position_max"], np.float32)), _p(out))
    return out.reshape(pos.shape)


def node_id_for_position(tree, pos):
    pos = _c(pos, np.float32).reshape(-1, 3)
    n = pos.shape[0]
    oid = np.zeros(n, np.int64)
    mask = np.zeros(n, np.float32)
    lib().orc_node_id_for_position(n, _p(pos), _p(_c(tree["node_position_min"], np.float32)),
                                   _p(_c(tree["node_position_max"], np.float32)),
                                   _p(_c(tree["node_children"], np.int32)), tree["ns"],
                                   _p(_c(tree["node_active"], np.int32)), int(tree["active_node_ids"][0]), _p(oid),
                                   _p(mask))
    return oid, mask


# ----------------------------------------------------------------------------
# gathers
# ----------------------------------------------------------------------------
def grid_sample2d(grid, index, uv, dtype=np.float32):
    g = _c(grid, dtype)
    N, C, H, W = g.shape
    idx = _c(index, np.int64)
    u = _c(uv, dtype)
    S = idx.shape[0]
    out = np.zeros((S, C), dtype)
    getattr(lib(), f"orc_grid_sample2d_fwd_{_suffix(dtype)}")(_p(g), N, C, H, W, _p(idx), _p(u), S, _p(out))
    return out


def grid_sample2d_bwd(grid, index, uv, gout, dtype=np.float32):
    g = _c(grid, dtype)
    N, C, H, W = g.shape
    idx = _c(index, np.int64)
    u = _c(uv, dtype)
    go = _c(gout, dtype)
    S = idx.shape[0]
    gg = np.zeros_like(g)
    gu = np.zeros((S, 2), dtype)
    getattr(lib(), f"orc_grid_sample2d_bwd_{_suffix(dtype)}")(_p(g), N, C, H, W, _p(idx), _p(u), S, _p(go), _p(gg),
                                                              _p(gu))
    return gg, gu


def grid_sample1d(grid, index, uv, dtype=np.float32):
    g = _c(grid, dtype)
    N, C, W, _ = g.shape
    idx = _c(index, np.int64)
    u = _c(uv, dtype)
    S = idx.shape[0]
    out = np.zeros((S, C), dtype)
    getattr(lib(), f"orc_grid_sample1d_fwd_{_suffix(dtype)}")(_p(g), N, C, W, _p(idx), _p(u), S, _p(out))
    return out


def grid_sample1d_bwd(grid, index, uv, gout, dtype=np.float32):
    g = _c(grid, dtype)
    N, C, W, _ = g.shape
    idx = _c(index, np.int64)
    u = _c(uv, dtype)
    go = _c(gout, dtype)
    S = idx.shape[0]
    gg = np.zeros_like(g)
    gu = np.zeros((S, 1), dtype)
    getattr(lib(), f"orc_grid_sample1d_bwd_{_suffix(dtype)}")(_p(g), N, C, W, _p(idx), _p(u), S, _p(go), _p(gg),
                                                              _p(gu))
    return gg, gu


# ----------------------------------------------------------------------------
# field / decoder / projection
# ----------------------------------------------------------------------------
class _FieldArgs:
    def __init__(self, field, tree, dtype):
        self.planes = [_c(p, dtype) for p in field["planes"]]
        self.lines = [_c(l_, dtype) for l_ in field["lines"]]
        self.C = self.planes[0].shape[1]
        self.cat = int(field.get("cat", 0))
        self.ph = (ct.c_int * 3)(*[p.shape[2] for p in self.planes])
        self.pw = (ct.c_int * 3)(*[p.shape[3] for p in self.planes])
        self.ll = (ct.c_int * 3)(*[l_.shape[2] for l_ in self.lines])
        self.pt = _ptr_array(self.planes)
        self.lt = _ptr_array(self.lines)
        self.slot = _c(field["leaf_slot"], np.int64)
        self.pmin = _c(tree["node_position_min"], np.float32)
        self.pmax = _c(tree["node_position_max"], np.float32)
        self.rmin = _c(field.get("roi_min", (-1, -1, -1)), np.float32)
        self.rmax = _c(field.get("roi_max", (1, 1, 1)), np.float32)

    def args(self):
        return [self.C, self.cat, self.pt, self.ph, self.pw, self.lt, self.ll, _p(self.slot), _p(self.pmin),
                _p(self.pmax), _p(self.rmin), _p(self.rmax)]

    @property
    def F(self):
        return 3 * self.C if self.cat else self.C


class _MlpArgs:
    def __init__(self, mlp, dtype):
        self.W = [_c(w, dtype) for w, _ in mlp["layers"]]
        self.b = [_c(b, dtype) for _, b in mlp["layers"]]
        dims = [self.W[0].shape[1]] + [w.shape[0] for w in self.W]
        self.dims = (ct.c_int * len(dims))(*dims)
        self.n = len(self.W)
        self.Wt = _ptr_array(self.W)
        self.bt = _ptr_array(self.b)
        self.act = ACT[mlp.get("act", "silu")]
        self.last = ACT[mlp.get("last_act", "softplus")]
        self.beta = float(mlp.get("beta", 2.0))
        self.out = dims[-1]
        self.inp = dims[0]

    def args(self):
        return [self.n, self.dims, self.Wt, self.bt, self.act, self.last, self.beta]


def vm_features(field, tree, pos, node, dtype=np.float32):
    fa = _FieldArgs(field, tree, dtype)
    pos = _c(pos, np.float32)
    node = _c(node, np.int64)
    S = node.shape[0]
    out = np.zeros((S, fa.F), dtype)
    getattr(lib(), f"orc_vm_features_{_suffix(dtype)}")(*fa.args(), S, _p(pos), _p(node), _p(out))
    return out


def vm_features_bwd(field, tree, pos, node, gout, dtype=np.float32):
    fa = _FieldArgs(field, tree, dtype)
    pos = _c(pos, np.float32)
    node = _c(node, np.int64)
    go = _c(gout, dtype)
    S = node.shape[0]
    gp = [np.zeros_like(p) for p in fa.planes]
    gl = [np.zeros_like(l_) for l_ in fa.lines]
    getattr(lib(), f"orc_vm_features_bwd_{_suffix(dtype)}")(*fa.args(), S, _p(pos), _p(node), _p(go),
                                                            _ptr_array(gp), _ptr_array(gl))
    return gp, gl


def mlp_forward(mlp, x, dtype=np.float32):
    ma = _MlpArgs(mlp, dtype)
    x = _c(x, dtype)
    S = x.shape[0]
    out = np.zeros((S, ma.out), dtype)
    getattr(lib(), f"orc_mlp_fwd_{_suffix(dtype)}")(*ma.args(), S, _p(x), _p(out))
    return out


def mlp_backward(mlp, x, gout, dtype=np.float32):
    ma = _MlpArgs(mlp, dtype)
    x = _c(x, dtype)
    go = _c(gout, dtype)
    S = x.shape[0]
    dW = [np.zeros_like(w) for w in ma.W]
    db = [np.zeros_like(b) for b in ma.b]
    dx = np.zeros_like(x)
    getattr(lib(), f"orc_mlp_bwd_{_suffix(dtype)}")(*ma.args(), S, _p(x), _p(go), _ptr_array(dW), _ptr_array(db),
                                                    _p(dx))
    return dW, db, dx


def project_forward(field, mlp, tree, samples, num_rays, dtype=np.float32):
    """ComputeImage + IntegrateSamplesXRay: image [Cout, R]."""
    fa = _FieldArgs(field, tree, dtype)
    ma = _MlpArgs(mlp, dtype)
    pos = _c(samples["global_coordinate"], np.float32)
    w = _c(samples["weight"], np.float32)
    ray = _c(samples["ray_index"], np.int64)
    node = _c(samples["node_id"], np.int64)
    img = np.zeros((ma.out, num_rays), dtype)
    getattr(lib(), f"orc_project_fwd_{_suffix(dtype)}")(*fa.args(), *ma.args(), len(w), _p(pos), _p(w), _p(ray),
                                                        _p(node), num_rays, _p(img))
    return img


def project_backward(field, mlp, tree, samples, num_rays, gimage, dtype=np.float32):
    fa = _FieldArgs(field, tree, dtype)
    ma = _MlpArgs(mlp, dtype)
    pos = _c(samples["global_coordinate"], np.float32)
    w = _c(samples["weight"], np.float32)
    ray = _c(samples["ray_index"], np.int64)
    node = _c(samples["node_id"], np.int64)
    gi = _c(gimage, dtype)
    gp = [np.zeros_like(p) for p in fa.planes]
    gl = [np.zeros_like(l_) for l_ in fa.lines]
    dW = [np.zeros_like(x) for x in ma.W]
    db = [np.zeros_like(x) for x in ma.b]
    getattr(lib(), f"orc_project_bwd_{_suffix(dtype)}")(*fa.args(), *ma.args(), len(w), _p(pos), _p(w), _p(ray),
                                                        _p(node), num_rays, _p(gi), _ptr_array(gp), _ptr_array(gl),
                                                        _ptr_array(dW), _ptr_array(db))
    return {"planes": gp, "lines": gl, "W": dW, "b": db}


def accumulate_loss_per_node(samples, per_ray_loss, num_nodes):
    L = lib()
    prl = _c(per_ray_loss, np.float32)
    if prl.ndim == 1:
        prl = prl[None, :]
    C, R = prl.shape
    ray = _c(samples["ray_index"], np.int64)
    node = _c(samples["node_id"], np.int64)
    w = _c(samples["weight"], np.float32)
    ls = np.zeros(num_nodes, np.float64)
    ws = np.zeros(num_nodes, np.float64)
    L.orc_accumulate_loss_per_node(len(w), _p(ray), _p(node), _p(w), _p(prl), C, R, num_nodes, _p(ls), _p(ws))
    return ls, ws


def gradient_correction_bwd(direction, ray_index, grad, dtype=np.float32):
    """Backward of GradientCorrection
    (hyperacorn/csrc/modules/GradientCorrection.cu:22-48): per sample i with
    ray r = ray_index[i], g - (g . d) d with d = direction[r] as given (the
    reference does not normalise it). The dot product is summed left to
    right, every operation rounded to dtype on its own."""
    d = np.asarray(direction, dtype)[np.asarray(ray_index, np.int64)]
    g = np.asarray(grad, dtype)
    dot = (g[:, 0] * d[:, 0] + g[:, 1] * d[:, 1]) + g[:, 2] * d[:, 2]
    return g - dot[:, None] * d


def num_threads():
    return lib().orc_num_threads()


def train_step(tree, field, mlp, origin, direction, target, max_samples_per_node, seed):
    """One plain FP32 training step on the CPU (the timed CPU baseline).
    Returns (loss, image, grads)."""
    L = lib()
    fa = _FieldArgs(field, tree, np.float32)
    ma = _MlpArgs(mlp, np.float32)
    o = _c(origin, np.float32)
    d = _c(direction, np.float32)
    y = _c(target, np.float32).reshape(-1)
    R = o.shape[0]
    act = _c(tree["active_node_ids"], np.int64)
    img = np.zeros((ma.out, R), np.float32)
    gp = [np.zeros_like(p) for p in fa.planes]
    gl = [np.zeros_like(l_) for l_ in fa.lines]
    dW = [np.zeros_like(x) for x in ma.W]
    db = [np.zeros_like(x) for x in ma.b]
    pn = np.array([p.size for p in fa.planes], np.int64)
    ln = np.array([l_.size for l_ in fa.lines], np.int64)
    loss = L.orc_train_step_f32(_p(fa.pmin), _p(fa.pmax), _p(act), len(act), _p(o), _p(d), _p(y), R,
                                int(max_samples_per_node), seed, fa.C, fa.cat, fa.pt, fa.ph, fa.pw, fa.lt, fa.ll,
                                _p(fa.slot), _p(fa.rmin), _p(fa.rmax), *ma.args(), _p(pn), _p(ln), _p(img),
                                _ptr_array(gp), _ptr_array(gl), _ptr_array(dW), _ptr_array(db))
    return loss, img, {"planes": gp, "lines": gl, "W": dW, "b": db}
