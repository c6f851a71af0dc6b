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
    "C3": Config("C3", 512, 1000, 61, 2.0, 512, 4, 16, 17, [64, 64], 16384, 24, noise=0.05, jitter=0.1,
                 speckle=0.05),
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


def analytic_projection(ph, origin, direction):
    """Line integrals of the (unclamped) ellipsoid sum along the rays, float64."""
    o = np.asarray(origin, np.float64)
    d = np.asarray(direction, np.float64)
    out = np.zeros(o.shape[0])
    for cen, ax, dens in zip(ph["centres"], ph["axes"], ph["density"]):
        oc = (o - cen) / ax
        dc = d / ax
        a = (dc * dc).sum(1)
        b = 2 * (oc * dc).sum(1)
        c = (oc * oc).sum(1) - 1
        disc = b * b - 4 * a * c
        m = disc > 0
        chord = np.zeros_like(out)
        chord[m] = np.sqrt(disc[m]) / a[m]
        out += dens * chord
    return out


def random_ray_batch(cfg: Config, R: int, seed: int):
    rng = np.random.default_rng(seed)
    img = rng.integers(0, cfg.angles, R)
    pix = rng.integers(0, cfg.detector * cfg.detector, R)
    return parallel_beam_rays(tilt_angles(cfg), cfg.detector, img, pix)


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
