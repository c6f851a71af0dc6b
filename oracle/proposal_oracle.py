"""CPU restatement of the learned proposal sampler's kernels, in numpy.

TEST INFRASTRUCTURE ONLY: tests/ compare the CUDA kernels of
adaptivetensordf_b200/csrc/proposal.cu (atdf_proposal_features, _allocate,
_samples, _loss, _occupancy) with these functions; the proposal MLP itself
is checked against the C++ oracle's generic MLP (oracle.mlp_forward /
mlp_backward). Nothing in the product imports this module.

The proposal sampler has no counterpart in the reference (which places
max_samples_per_node uniform samples in every leaf a ray crosses,
hyperacorn/csrc/structure/HyperTree.cu:266-514), so these restate the
sampler's own definition: parity here is against this specification, not
against reference outputs.
"""

from __future__ import annotations

import numpy as np

BINS = 32
OUTPUTS = 33
INPUTS = 16
OCC = 9


def softplus1(x):
    x = np.asarray(x, np.float64)
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def octant(x, y, z):
    return (x > 0).astype(int) | ((y > 0).astype(int) << 1) | ((z > 0).astype(int) << 2)


def features(node_min, node_max, origin, direction, seg_node, seg_ray, tmin, tmax, occupancy):
    """[G, 16]: leaf-local entry point, leaf-local exit point, segment length
    / leaf diagonal, the leaf's mean occupancy, its 8 octant occupancies
    (occupancy [num_nodes, 9] or None)."""
    mn = node_min[seg_node].astype(np.float64)
    mx = node_max[seg_node].astype(np.float64)
    o = origin[seg_ray].astype(np.float64)
    d = direction[seg_ray].astype(np.float64)
    t0 = tmin.astype(np.float64)[:, None]
    t1 = tmax.astype(np.float64)[:, None]
    inv = 2.0 / (mx - mn)
    f = np.zeros((len(seg_node), INPUTS))
    f[:, 0:3] = (o + d * t0 - mn) * inv - 1
    f[:, 3:6] = (o + d * t1 - mn) * inv - 1
    f[:, 6] = (tmax - tmin) / np.sqrt(((mx - mn) ** 2).sum(1))
    if occupancy is not None:
        occ = occupancy.reshape(-1, OCC)[seg_node]
        f[:, 7] = occ[:, 8]
        f[:, 8:16] = occ[:, :8]
    return f


def allocate(ray_seg_offset, tmin, tmax, logits, budget, mass_mix, mass_power=1.0):
    """Per-segment sample counts and per-ray first indices, and the ray
    sample offsets [R + 1]: n = 1 + round(spare * share), share mixing the
    weight len * density^mass_power with the length."""
    R = len(ray_seg_offset) - 1
    G = int(ray_seg_offset[-1])
    n = np.zeros(G, np.int64)
    first = np.zeros(G, np.int64)
    off = np.zeros(R + 1, np.int64)
    length = (tmax - tmin).astype(np.float64)
    mass = length * np.power(np.maximum(softplus1(logits[:G, BINS]), 1e-20), mass_power)
    for r in range(R):
        b, e = int(ray_seg_offset[r]), int(ray_seg_offset[r + 1])
        nseg = e - b
        if nseg == 0:
            off[r + 1] = off[r]
            continue
        msum = mass[b:e].sum()
        lsum = length[b:e].sum()
        spare = max(budget - nseg, 0)
        run = 0
        for s in range(b, e):
            share = length[s] / lsum if lsum > 0 else 1.0 / nseg
            if msum > 0:
                share = (1 - mass_mix) * mass[s] / msum + mass_mix * share
            n[s] = 1 + int(np.floor(spare * share + 0.5))
            first[s] = run
            run += n[s]
        off[r + 1] = off[r] + run
    return n, first, off


def bin_probs(lg, bin_mix, power=1.0):
    lg = np.asarray(lg, np.float64)
    e = np.exp(power * (lg - lg.max(-1, keepdims=True)))
    p = e / e.sum(-1, keepdims=True)
    return p * (1 - bin_mix) + bin_mix / BINS


def samples(tmin, tmax, nsamp, logits, bin_mix, a=None, bin_power=1.0, importance=False):
    """t and weight of every segment's samples, concatenated in segment
    order: u_j = (j + a_j) / n, inverse CDF of the binned density (the
    predicted one raised to bin_power, mixed with uniform); weights are the
    Voronoi cells of the placed t within the segment, or with importance
    the importance weights 1 / (n q(t_j)) = bin width / (n p_bin). a:
    per-segment arrays of jitter (None: 0.5)."""
    ts, ws = [], []
    for s in range(len(nsamp)):
        n = int(nsamp[s])
        p = bin_probs(logits[s, :BINS], bin_mix, bin_power)
        cdf = np.concatenate([[0.0], np.cumsum(p)])
        t0, t1 = float(tmin[s]), float(tmax[s])
        binw = (t1 - t0) / BINS
        tt, tb = [], []
        for j in range(n):
            aj = 0.5 if a is None else float(a[s][j])
            u = (j + aj) / n
            b = int(np.searchsorted(cdf, u, side="right") - 1)
            b = min(max(b, 0), BINS - 1)
            frac = min(max((u - cdf[b]) / p[b], 0.0), 1.0)
            tt.append(min(max(t0 + (b + frac) * binw, t0), t1))
            tb.append(b)
        if importance:
            ts.extend(tt)
            ws.extend(binw / (n * p[b]) for b in tb)
            continue
        for j in range(n):
            lo = t0 if j == 0 else 0.5 * (tt[j - 1] + tt[j])
            hi = t1 if j == n - 1 else 0.5 * (tt[j + 1] + tt[j])
            ts.append(tt[j])
            ws.append(hi - lo)
    return np.array(ts), np.array(ws)


def loss(bins, logits, length, mass_weight, delta=1e-4):
    """Mean over segments of CE(normalised bins, softmax(bin logits)) +
    mass_weight * (log(softplus(z) len + delta) - log(m + delta))^2, its
    gradient with respect to the logits, and the target masses."""
    G = bins.shape[0]
    lg = logits[:G].astype(np.float64)
    h = np.maximum(bins.astype(np.float64), 0)
    m = h.sum(1)
    p = bin_probs(lg[:, :BINS], 0.0)
    hn = np.where(m[:, None] > 0, h / np.where(m > 0, m, 1)[:, None], 0.0)
    ce = -(hn * np.log(np.maximum(p, 1e-30))).sum(1)
    z = lg[:, BINS]
    mh = softplus1(z) * length
    e = np.log(mh + delta) - np.log(m + delta)
    total = (ce + mass_weight * e * e).sum() / G
    d = np.zeros_like(lg)
    d[:, :BINS] = np.where(m[:, None] > 0, p - hn, 0.0) / G
    sig = 1 / (1 + np.exp(-z))
    d[:, BINS] = mass_weight * 2 * e / (mh + delta) * length * sig / G
    return total, d, m


def node_occupancy_sums(bins, feats, length, seg_node, num_nodes):
    """Per leaf octant and leaf [num_nodes, 9]: target mass and crossed
    length, each bin placed at its centre between the entry and exit points."""
    nm = np.zeros((num_nodes, OCC))
    nl = np.zeros((num_nodes, OCC))
    h = np.maximum(bins.astype(np.float64), 0)
    c = (np.arange(BINS) + 0.5) / BINS
    for s in range(len(seg_node)):
        f = feats[s]
        pts = f[None, 0:3] + c[:, None] * (f[None, 3:6] - f[None, 0:3])
        q = octant(pts[:, 0], pts[:, 1], pts[:, 2])
        for b in range(BINS):
            nm[seg_node[s], q[b]] += h[s, b]
            nl[seg_node[s], q[b]] += length[s] / BINS
        nm[seg_node[s], 8] += h[s].sum()
        nl[seg_node[s], 8] += length[s]
    return nm, nl
