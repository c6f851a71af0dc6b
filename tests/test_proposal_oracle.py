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
    """Uniform logits give the uniform per-node rule (t_j = tmin + (j + a)
    len / n with Voronoi weights); for any density the weights of a segment
    tile it exactly, and denser placement integrates a bump more accurately."""
    tmin = np.array([0.0, 1.0], np.float32)
    tmax = np.array([2.0, 1.5], np.float32)
    n = np.array([8, 5])
    lg = np.zeros((2, po.OUTPUTS))
    t, w = po.samples(tmin, tmax, n, lg, 0.2)
    assert np.allclose(t[:8], (np.arange(8) + 0.5) * 2 / 8)
    assert np.allclose(w[:8], 2 / 8) and np.allclose(w[8:], 0.5 / 5)
    rng = np.random.default_rng(1)
    lg = rng.normal(size=(2, po.OUTPUTS)) * 2
    t, w = po.samples(tmin, tmax, n, lg, 0.2, [rng.random(8), rng.random(5)])
    assert np.allclose([w[:8].sum(), w[8:].sum()], tmax - tmin)
    # a narrow bump on a smooth background over a [0, 2] segment: placing
    # samples by the bump's density (square root) integrates it better than
    # uniform placement with the same count
    f = lambda x: np.exp(-((x - 0.6) / 0.05) ** 2) + 0.05 * np.sin(3 * x) + 0.06  # noqa: E731
    exact = 0.05 * np.sqrt(np.pi) + 0.05 * (1 - np.cos(6)) / 3 + 0.12
    c = (np.arange(po.BINS) + 0.5) / po.BINS * 2
    lg_bump = np.zeros((1, po.OUTPUTS))
    lg_bump[0, :po.BINS] = np.log(f(c))
    one = (np.array([0.0], np.float32), np.array([2.0], np.float32), np.array([12]))
    errs = {}
    for name, l in (("uniform", np.zeros((1, po.OUTPUTS))), ("bump", lg_bump)):
        e = []
        for _ in range(200):
            t, w = po.samples(*one, l, 0.2, [rng.random(12)], bin_power=0.5)
            e.append((f(t) * w).sum() - exact)
        errs[name] = np.sqrt(np.mean(np.square(e)))
    assert errs["bump"] < 0.75 * errs["uniform"], errs


def test_allocation_respects_budget():
    off = np.array([0, 3, 3, 10])
    G = 10
    rng = np.random.default_rng(2)
    tmin = rng.uniform(0, 1, G).astype(np.float32)
    tmax = (tmin + rng.uniform(0.01, 0.5, G)).astype(np.float32)
    lg = rng.normal(size=(G, po.OUTPUTS))
    n, first, ro = po.allocate(off, tmin, tmax, lg, 16, 0.25, 0.5)
    assert np.all(n >= 1)
    seg = np.diff(off)
    assert np.all(np.diff(ro) <= 16 + seg) and ro[2] == ro[1]
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


def test_importance_weights_are_unbiased():
    """With importance weights 1 / (n q(t)) and uniform jitter, the weighted
    sum of a density along a segment averages to its integral (for any
    proposal q with full support), while the Voronoi-cell weights of the
    same samples keep a bias when q is far from the density."""
    from oracle import proposal_oracle as po

    rng = np.random.default_rng(5)
    t0, t1, n = 0.3, 1.7, 6

    def rho(t):
        return np.where(t < 0.9, 0.05, 1.0 + 0.5 * np.sin(7 * t))

    grid = np.linspace(t0, t1, 200001)
    exact = np.trapezoid(rho(grid), grid)
    logits = rng.normal(0, 2.0, (1, po.BINS + 1))  # a poor proposal
    est_i, est_v = [], []
    for k in range(4000):
        a = [rng.random(n)]
        t, w = po.samples(np.array([t0]), np.array([t1]), np.array([n]), logits, 0.2, a, 1.0, importance=True)
        est_i.append((w * rho(t)).sum())
        t, w = po.samples(np.array([t0]), np.array([t1]), np.array([n]), logits, 0.2, a, 1.0, importance=False)
        est_v.append((w * rho(t)).sum())
    mi, se = np.mean(est_i), np.std(est_i) / np.sqrt(len(est_i))
    assert abs(mi - exact) < 4 * se + 1e-9, (mi, exact, se)
    # with a uniform proposal both rules place the same samples and weights
    flat = np.zeros((1, po.BINS + 1))
    t, wi = po.samples(np.array([t0]), np.array([t1]), np.array([n]), flat, 0.2, None, 1.0, importance=True)
    _, wv = po.samples(np.array([t0]), np.array([t1]), np.array([n]), flat, 0.2, None, 1.0, importance=False)
    assert np.allclose(wi, (t1 - t0) / n) and np.allclose(wv, (t1 - t0) / n)
    assert abs(np.mean(est_v) - exact) > 4 * np.std(est_v) / np.sqrt(len(est_v))  # the Voronoi rule is biased
