"""CPU checks of the proposal sampler's numpy restatement: the loss gradient
against central finite differences, the sampler's stratification and
weights, and the budget split."""

import numpy as np

from oracle import proposal_oracle as po


def test_proposal_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    G = 7
    lg = rng.normal(size=(G, po.OUTPUTS))
    bins = rng.gamma(0.5, 1.0, (G, po.BINS))
    bins[2] = 0.0
    length = rng.uniform(0.05, 0.3, G)
    L0, d, _ = po.loss(bins, lg, length, 0.3)
    h = 1e-6
    for s in range(G):
        for k in (0, 5, 31, 32):
            lp = lg.copy()
            lm = lg.copy()
            lp[s, k] += h
            lm[s, k] -= h
            fd = (po.loss(bins, lp, length, 0.3)[0] - po.loss(bins, lm, length, 0.3)[0]) / (2 * h)
            assert abs(fd - d[s, k]) < 1e-6 * max(1.0, abs(fd)), (s, k, fd, d[s, k])


def test_proposal_samples_are_stratified_and_weighted():
    """Uniform logits give the uniform stratified rule (t_j = tmin + (j + a)
    len / n, w = len / n); for any density the weights integrate a constant
    exactly in expectation over the jitter."""
    tmin = np.array([0.0, 1.0], np.float32)
    tmax = np.array([2.0, 1.5], np.float32)
    n = np.array([8, 5])
    lg = np.zeros((2, po.OUTPUTS))
    t, w = po.samples(tmin, tmax, n, lg, 0.2)
    assert np.allclose(t[:8], (np.arange(8) + 0.5) * 2 / 8)
    assert np.allclose(w[:8], 2 / 8) and np.allclose(w[8:], 0.5 / 5)
    rng = np.random.default_rng(1)
    lg = rng.normal(size=(2, po.OUTPUTS)) * 2
    K = 4000
    tot = np.zeros(2)
    for _ in range(K):
        a = [rng.random(8), rng.random(5)]
        _, w = po.samples(tmin, tmax, n, lg, 0.2, a)
        tot += [w[:8].sum(), w[8:].sum()]
    assert np.allclose(tot / K, tmax - tmin, rtol=2e-2)


def test_allocation_respects_budget():
    off = np.array([0, 3, 3, 10])
    G = 10
    rng = np.random.default_rng(2)
    tmin = rng.uniform(0, 1, G).astype(np.float32)
    tmax = (tmin + rng.uniform(0.01, 0.5, G)).astype(np.float32)
    lg = rng.normal(size=(G, po.OUTPUTS))
    n, first, ro = po.allocate(off, tmin, tmax, lg, 16, 0.25)
    assert np.all(n >= 1)
    assert ro[1] - ro[0] <= 16 and ro[2] == ro[1] and ro[3] - ro[2] <= 16
    assert list(first[:3]) == [0, n[0], n[0] + n[1]]


def test_octant_sums_split_each_segment():
    """Bins of a segment that crosses the leaf's x = 0 plane land in two
    octants; per-node sums add up to the segment totals."""
    feats = np.zeros((1, po.INPUTS))
    feats[0, 0:3] = [-0.9, -0.5, 0.5]
    feats[0, 3:6] = [0.9, -0.5, 0.5]
    bins = np.ones((1, po.BINS))
    nm, nl = po.node_occupancy_sums(bins, feats, np.array([2.0]), np.array([3]), 5)
    assert nm[3, 8] == 32 and abs(nl[3, 8] - 2.0) < 1e-12
    assert nm[3, 4] == 16 and nm[3, 5] == 16  # (x<=0, y<0, z>0) and (x>0, y<0, z>0)
    assert abs(nl[3, :8].sum() - 2.0) < 1e-12
