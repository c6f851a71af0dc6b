"""Seeded scenes shared by the GPU parity tests: the same tree, rays, field and
decoder on the CUDA side (torch tensors through the product API) and on the
oracle side (numpy)."""

import math

import numpy as np
import torch


def rays_through_volume(R, seed, tilt=1.0, wobble=0.1):
    rng = np.random.default_rng(seed)
    th = rng.uniform(-tilt, tilt, R)
    d = np.stack([np.sin(th), wobble * rng.normal(size=R), np.cos(th)], 1)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    p = rng.uniform(-0.95, 0.95, (R, 3))
    o = p - math.sqrt(2.0) * d
    return o.astype(np.float32), d.astype(np.float32)


def gpu_scene(depth, C, G, lines, hidden, R, seed=0, tensor_op="add", activation="silu", quad=False,
              active_depth=None):
    from adaptivetensordf_b200 import synthetic as syn

    tree = syn.make_tree(depth, active_depth, device="cuda", quad=quad)
    geo = syn.make_geometry(tree, C, G, lines, hidden, seed=seed + 11, tensor_op=tensor_op, activation=activation)
    o, d = rays_through_volume(R, seed)
    return tree, geo, o, d


def oracle_views(tree, geo):
    from adaptivetensordf_b200 import synthetic as syn

    return syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / max(den, 1e-30)
