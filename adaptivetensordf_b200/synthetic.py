"""Synthetic inputs of the benchmark configurations: ellipsoid phantoms,
parallel-beam tilt series, and random-initialised VM factors and decoders.

The reference trains on real cryo-ET tilt series that are not available
here; these seeded generators stand in for them with the shapes and value
distributions of the configurations:

* phantom: axis-aligned ellipsoids, centres U[-0.8, 0.8]^3, semi-axes
  U[0.05, 0.25]^3, densities U[0.1, 1.0], summed (clamped to 1 when
  voxelised) on a zero background in [-1, 1]^3;
* rays: parallel beam, tilt axis y, detector pixel centres on [-1, 1]^2,
  origin = R (u, v, 0) - sqrt(2) d with d = R (0, 0, 1), computed in float64
  and stored as float32 (hyperacorn/csrc/data/SceneBase.cpp:392-443);
* factors: uniform(-0.5, 0.5) planes / lines (vm_init_scale = 0.5, "uniform",
  hyperacorn/csrc/geometry/tensorfield.h:28-31);
* decoder: torch Linear layers with Kaiming-normal weights (fan_in, ReLU
  gain) and torch's default bias init (hyperacorn/csrc/geometry/Modules.h:30-36).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


# ----------------------------------------------------------------------------
# configurations
# ----------------------------------------------------------------------------
@dataclass
class Config:
    name: str
    volume: int
    ellipsoids: int
    angles: int
    angle_step: float
    detector: int
    tree_depth: int
    channels: int
    grid: int
    hidden: list = field(default_factory=lambda: [64, 64])
    rays_per_batch: int = 4096
    max_samples_per_node: int = 32
    noise: float = 0.0
    jitter: float = 0.0
    speckle: float = 0.0
    line_len: tuple | None = None
    # thin specimen: the phantom fills z in [-slab, slab] of the [-1, 1]^3
    # volume (its voxel grid is volume x volume x slab * volume)
    slab: float = 1.0
    # specimen tilt about x relative to the tilt axis (degrees)
    off_axis_deg: float = 0.0
    # adaptive tree: refined from start_depth toward target_leaves active
    # leaves (0: every node of depth tree_depth active)
    target_leaves: int = 0
    start_depth: int = 0
    # samples per ray of the learned proposal (0: none)
    proposal_budget: int = 0

    def lines(self):
        if self.line_len is not None:
            return tuple(self.line_len)
        n = (self.grid - 1) * (1 << self.tree_depth)
        return (n, self.grid, n)


CONFIGS = {
    # 64^3, 20 ellipsoids, 31 tilts at 4 deg, 64^2 detector, depth-2 octree
    # (64 leaves), rank-8 VM on 17^2 planes, decoder 8 -> 32 -> 1.
    "C1": Config("C1", 64, 20, 31, 4.0, 64, 2, 8, 17, [32], 4096, 32),
    # 256^3, 200 ellipsoids, 61 tilts at 2 deg, 256^2 detector, depth-4
    # octree, rank-16 VM, 17^2 planes; FCBlock default decoder 16->64->64->1.
    "C2": Config("C2", 256, 200, 61, 2.0, 256, 4, 16, 17, [64, 64], 16384, 24, noise=0.05, jitter=0.1),
    # 512^3, 1000 ellipsoids + 5% speckle, 512^2 detector, C=16, decoder
    # 16->64->64->1, 16384-ray batches, 256 samples per ray.
    # 29 samples per leaf diagonal: 260 uniform samples per ray on average
    # (28 gives 252), the configuration's 256.
    "C3": Config("C3", 512, 1000, 61, 2.0, 512, 4, 16, 17, [64, 64], 16384, 29, noise=0.05, jitter=0.1,
                 speckle=0.05),
    # the C2 volume and data, the uniform sampler at 256 samples per ray (29
    # per leaf diagonal) cut to 64 per ray by the learned proposal
    "C4": Config("C4", 256, 200, 61, 2.0, 256, 4, 16, 17, [64, 64], 16384, 29, noise=0.05, jitter=0.1,
                 proposal_budget=64),
    # thin slab 1024 x 1024 x 256 of 5000 ellipsoids, off-axis tilt drawn from
    # U[-5, 5] degrees (seed 1002), 81 tilts at 1.5 deg on a 1024^2 detector;
    # octree refined to depth 6 toward 4096 active leaves (empty leaves
    # culled), rank-24 VM on 17^2 planes with lines sized for depth 4,
    # decoder 24 -> 64 -> 64 -> 1, BF16; 119 samples per leaf diagonal give
    # 256 uniform samples per ray on average (about 4.9 leaves per ray)
    "C5": Config("C5", 1024, 5000, 81, 1.5, 1024, 6, 24, 17, [64, 64], 16384, 119, noise=0.05, jitter=0.1,
                 line_len=(256, 17, 256), slab=0.25,
                 off_axis_deg=float(np.random.default_rng(1002).uniform(-5.0, 5.0)), target_leaves=4096,
                 start_depth=3),
}


# ----------------------------------------------------------------------------
# phantom and rays
# ----------------------------------------------------------------------------
def ellipsoid_phantom(n: int, seed: int = 1001):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.8, 0.8, (n, 3))
    axes = rng.uniform(0.05, 0.25, (n, 3))
    dens = rng.uniform(0.1, 1.0, n)
    return {"centres": centres, "axes": axes, "density": dens}


def voxelize(ph, N: int, speckle: float = 0.0, seed: int = 1001, clamp: bool = True):
    """Phantom at the N^3 voxel centres of [-1, 1]^3 (z, y, x order)."""
    c = (np.arange(N) + 0.5) / N * 2 - 1
    vol = np.zeros((N, N, N), np.float64)
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    for cen, ax, d in zip(ph["centres"], ph["axes"], ph["density"]):
        q = ((xx - cen[0]) / ax[0]) ** 2 + ((yy - cen[1]) / ax[1]) ** 2 + ((zz - cen[2]) / ax[2]) ** 2
        vol += d * (q <= 1.0)
    if speckle > 0:
        rng = np.random.default_rng(seed + 7)
        m = rng.random(vol.shape) < speckle
        vol[m] += rng.uniform(0, 0.2, int(m.sum()))
    if clamp:
        vol = np.minimum(vol, 1.0)
    return vol


def slab_phantom(n: int, half_z: float, seed: int = 1001):
    """Ellipsoids of a thin specimen filling z in [-half_z, half_z]: the
    configurations' distributions (centres U[-0.8, 0.8]^3, semi-axes
    U[0.05, 0.25]^3, densities U[0.1, 1.0]) in the slab's own normalised frame,
    whose z is scaled by half_z into the volume."""
    ph = ellipsoid_phantom(n, seed)
    sc = np.array([1.0, 1.0, half_z])
    return {"centres": ph["centres"] * sc, "axes": ph["axes"] * sc, "density": ph["density"]}


def config_phantom(cfg: Config, seed: int = 1001):
    if cfg.slab < 1.0:
        return slab_phantom(cfg.ellipsoids, cfg.slab, seed)
    return ellipsoid_phantom(cfg.ellipsoids, seed)


def tilt_angles(cfg: Config):
    half = (cfg.angles - 1) / 2 * cfg.angle_step
    return np.array([-half + k * cfg.angle_step for k in range(cfg.angles)])


def parallel_beam_rays(angles_deg, detector: int, image_ids, pixel_ids, off_axis_deg: float = 0.0):
    """Rays of the given (tilt, pixel) pairs: float32 origin, direction [R, 3]."""
    th = np.deg2rad(np.asarray(angles_deg, np.float64)[image_ids])
    u = (pixel_ids % detector + 0.5) / detector * 2 - 1
    v = (pixel_ids // detector + 0.5) / detector * 2 - 1
    ct, st = np.cos(th), np.sin(th)
    d = np.stack([st, np.zeros_like(th), ct], 1)
    p = np.stack([u * ct, v, -u * st], 1)
    if off_axis_deg:
        a = math.radians(off_axis_deg)
        rx = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
        d = d @ rx.T
        p = p @ rx.T
    o = p - math.sqrt(2.0) * d
    return o.astype(np.float32), d.astype(np.float32)


def analytic_projection(ph, origin, direction, chunk: int = 256, device=None):
    """Line integrals of the (unclamped) ellipsoid sum along the rays, float64
    (ellipsoids in chunks of `chunk`); numpy, or torch on `device` when one
    is given (same arithmetic)."""
    xp = np
    if device is not None:
        xp = torch
        o = torch.as_tensor(np.asarray(origin, np.float64), device=device)
        d = torch.as_tensor(np.asarray(direction, np.float64), device=device)
        cen, ax, dens = (torch.as_tensor(ph[k], dtype=torch.float64, device=device)
                         for k in ("centres", "axes", "density"))
        out = torch.zeros(o.shape[0], dtype=torch.float64, device=device)
    else:
        o = np.asarray(origin, np.float64)
        d = np.asarray(direction, np.float64)
        cen, ax, dens = ph["centres"], ph["axes"], ph["density"]
        out = np.zeros(o.shape[0])
    for i in range(0, len(dens), chunk):
        c, a, dn = cen[i:i + chunk], ax[i:i + chunk], dens[i:i + chunk]
        oc = (o[:, None, :] - c[None]) / a[None]
        dc = d[:, None, :] / a[None]
        qa = (dc * dc).sum(2)
        qb = 2 * (oc * dc).sum(2)
        qc = (oc * oc).sum(2) - 1
        disc = qb * qb - 4 * qa * qc
        chord = xp.where(disc > 0, xp.sqrt(xp.clip(disc, 0.0, None)) / qa, xp.zeros_like(disc))
        out += (chord * dn[None]).sum(1)
    return out.cpu().numpy() if device is not None else out


def random_ray_batch(cfg: Config, R: int, seed: int):
    rng = np.random.default_rng(seed)
    img = rng.integers(0, cfg.angles, R)
    pix = rng.integers(0, cfg.detector * cfg.detector, R)
    return parallel_beam_rays(tilt_angles(cfg), cfg.detector, img, pix, cfg.off_axis_deg)


# ----------------------------------------------------------------------------
# model pieces
# ----------------------------------------------------------------------------
def make_tree(max_depth: int, active_depth: int | None = None, device: str = "cuda", quad: bool = False):
    from . import HyperTreeBase

    t = HyperTreeBase(3, max_depth)
    t.settree(quad, -1.0, 1.0)
    t.SetActive(max_depth if active_depth is None else active_depth)
    if device != "cpu":
        t.to(device)
    return t


def tree_from_leaves(max_depth: int, leaves, culled=None, device: str = "cuda"):
    """An octree of max_depth whose active leaves are the given node ids (a
    partition of the volume, possibly at mixed depths; culled node ids, whose
    region holds no leaf, are marked as such)."""
    from . import HyperTreeBase

    t = HyperTreeBase(3, max_depth)
    t.settree(False, -1.0, 1.0)
    act = torch.zeros(t.NumNodes(), dtype=torch.int32)
    act[torch.as_tensor(np.asarray(leaves, np.int64))] = 1
    t.node_active = act
    if culled is not None and len(culled):
        cul = torch.zeros(t.NumNodes(), dtype=torch.int32)
        cul[torch.as_tensor(np.asarray(culled, np.int64))] = 1
        t.node_culled = cul
    t.UpdateActive()
    if device != "cpu":
        t.to(device)
    return t


def _box_density_stats(ph, lo, hi, probe: int):
    """Variance and maximum of the phantom's density (ellipsoid sum, clamped
    to 1, float64) over the probe^3 cell-centre grid of each box [lo, hi],
    testing only the ellipsoids whose bounding box meets the box."""
    c, a, dn = ph["centres"], ph["axes"], ph["density"]
    emin, emax = c - a, c + a
    u = (np.arange(probe) + 0.5) / probe
    zz, yy, xx = np.meshgrid(u, u, u, indexing="ij")
    unit = np.stack([xx, yy, zz], -1).reshape(-1, 3)
    var = np.zeros(len(lo))
    mx = np.zeros(len(lo))
    for i in range(len(lo)):
        sel = np.nonzero(np.all((emax > lo[i]) & (emin < hi[i]), axis=1))[0]
        if len(sel) == 0:
            continue
        pts = lo[i] + unit * (hi[i] - lo[i])
        q = (((pts[:, None, :] - c[sel][None]) / a[sel][None]) ** 2).sum(-1)
        dens = np.minimum(((q <= 1.0) * dn[sel][None]).sum(1), 1.0)
        var[i] = dens.var()
        mx[i] = dens.max()
    return var, mx


def adaptive_leaves(cfg: Config, ph, node_min, node_max, node_children, node_depth, probe: int = 6,
                    split_share: float = 0.1):
    """Active leaves (and culled nodes) of the configuration's adaptive
    octree, refined from the phantom: start with the depth-start_depth cells
    that meet the specimen, then repeatedly split the leaves whose density
    varies most (variance of the phantom over a probe^3 grid of cell centres,
    rounded to 9 significant digits, ties by node id; the largest
    split_share of the candidates per round) until target_leaves active
    leaves or the maximum depth. Children outside the specimen or with no
    density on their probe grid are culled, as the structure refinement
    culls empty leaves. The phantom-derived error stands in for the trained
    field's error that the reference's refinement scores
    (hyper_train.cpp:1886-1912). Plain numpy in float64 on the tree's
    arrays, so any copy of the tree (this package's or another's) gives the
    same leaves."""
    mn = np.asarray(node_min, np.float64)
    mx = np.asarray(node_max, np.float64)
    ch = np.asarray(node_children)
    depth = np.asarray(node_depth)
    zlo, zhi = -cfg.slab, cfg.slab

    def keep(nodes):
        nodes = np.asarray(nodes, np.int64)
        nodes = nodes[(mx[nodes, 2] > zlo) & (mn[nodes, 2] < zhi)]
        var, dmax = _box_density_stats(ph, mn[nodes], mx[nodes], probe)
        full = dmax > 0
        score = np.array([float(f"{v:.9g}") for v in var[full]])
        return nodes[full], score

    leaves, score = keep(np.nonzero(depth == cfg.start_depth)[0])
    while len(leaves) < cfg.target_leaves:
        cand = np.nonzero((depth[leaves] < depth.max()) & (score > 0))[0]
        if len(cand) == 0:
            break
        room = (cfg.target_leaves - len(leaves)) // 7 + 1
        n = max(1, min(room, int(len(cand) * split_share) + 1))
        order = np.lexsort((leaves[cand], -score[cand]))
        pick = cand[order[:n]]
        kids = ch[leaves[pick]].reshape(-1)
        kn, ks = keep(kids[kids >= 0])
        rest = np.ones(len(leaves), bool)
        rest[pick] = False
        leaves = np.concatenate([leaves[rest], kn])
        score = np.concatenate([score[rest], ks])
    # culled: nodes with no active leaf in their subtree that lie in no leaf
    n = len(depth)
    act = np.zeros(n, bool)
    act[leaves] = True
    covered = act.copy()
    inside = np.zeros(n, bool)
    for nd in range(n - 1, -1, -1):  # children have larger ids than their parent
        c = ch[nd]
        c = c[c >= 0]
        if len(c) and covered[c].any():
            covered[nd] = True
    for nd in range(n):
        if act[nd] or inside[nd]:
            c = ch[nd]
            inside[c[c >= 0]] = True
    return np.sort(leaves), np.nonzero(~covered & ~inside)[0]


def adaptive_tree(cfg: Config, ph, device: str = "cuda"):
    """The configuration's adaptive octree (adaptive_leaves) as a
    HyperTreeBase on device."""
    from . import HyperTreeBase

    t = HyperTreeBase(3, cfg.tree_depth)
    t.settree(False, -1.0, 1.0)
    leaves, culled = adaptive_leaves(cfg, ph, t.node_position_min.numpy(), t.node_position_max.numpy(),
                                     t.node_children.numpy(), t.node_depth.numpy())
    return tree_from_leaves(cfg.tree_depth, leaves, culled, device)


def make_geometry(tree, channels: int, grid: int, lines, hidden, seed: int = 1003, device: str = "cuda",
                  init_scale: float = 0.5, tensor_op: str = "add", activation: str = "silu",
                  last_activation: str = "softplus", beta: float = 2.0):
    """GeometryTensorQO with one plane slot per active leaf (leaf_slot = the
    active prefix sum, i.e. the whole volume is the ROI)."""
    from . import GeometryTensorQO

    g = torch.Generator().manual_seed(seed)
    n_slots = int(tree.NumActiveNodes())
    planes = []
    for _ in range(3):
        p = (torch.rand((n_slots, channels, grid, grid), generator=g) * 2 - 1) * init_scale
        planes.append(p.to(device).contiguous(memory_format=torch.channels_last).requires_grad_(True))
    lns = []
    for L in lines:
        ln = (torch.rand((1, channels, L, 1), generator=g) * 2 - 1) * init_scale
        lns.append(ln.to(device).contiguous(memory_format=torch.channels_last).requires_grad_(True))
    geo = GeometryTensorQO()
    geo.planes = planes
    geo.lines = lns
    geo.leaf_slot = tree.node_active_prefix_sum.to(device)
    geo.tensor_op = tensor_op
    F = channels * (3 if tensor_op == "cat" else 1)
    dims = [F] + list(hidden) + [1]
    ws, bs = [], []
    for i in range(len(dims) - 1):
        fan_in = dims[i]
        w = torch.randn((dims[i + 1], fan_in), generator=g) * math.sqrt(2.0 / fan_in)
        bound = 1.0 / math.sqrt(fan_in)
        b = (torch.rand(dims[i + 1], generator=g) * 2 - 1) * bound
        ws.append(w.to(device).requires_grad_(True))
        bs.append(b.to(device).requires_grad_(True))
    geo.decoder_weight = ws
    geo.decoder_bias = bs
    geo.activation = activation
    geo.last_activation = last_activation
    geo.softplus_beta = beta
    return geo


def parameters(geo):
    return list(geo.planes) + list(geo.lines) + list(geo.decoder_weight) + list(geo.decoder_bias)


def field_dict(geo, tree):
    """Numpy copy of the field in the oracle's layout (reference [N, C, H, W])."""
    return {
        "planes": [p.detach().cpu().contiguous().numpy() for p in geo.planes],
        "lines": [ln.detach().cpu().contiguous().numpy() for ln in geo.lines],
        "leaf_slot": geo.leaf_slot.cpu().numpy(),
        "roi_min": np.array(geo.roi_min, np.float32),
        "roi_max": np.array(geo.roi_max, np.float32),
        "cat": 1 if geo.tensor_op == "cat" else 0,
    }


def mlp_dict(geo):
    return {
        "layers": [(w.detach().cpu().numpy(), b.detach().cpu().numpy())
                   for w, b in zip(geo.decoder_weight, geo.decoder_bias)],
        "act": geo.activation,
        "last_act": geo.last_activation,
        "beta": geo.softplus_beta,
    }


def tree_dict(tree):
    """Numpy copy of the tree buffers in the oracle's form."""
    return {
        "node_position_min": tree.node_position_min.cpu().numpy(),
        "node_position_max": tree.node_position_max.cpu().numpy(),
        "node_children": tree.node_children.cpu().numpy(),
        "node_depth": tree.node_depth.cpu().numpy(),
        "node_active": tree.node_active.cpu().numpy(),
        "active_node_ids": tree.active_node_ids.cpu().numpy(),
        "node_active_prefix_sum": tree.node_active_prefix_sum.cpu().numpy(),
        "ns": tree.NS(),
        "max_depth": tree.max_depth,
    }
