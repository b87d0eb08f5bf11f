"""The planner's CPU oracle checked against finite differences (CPU only)."""
import numpy as np

from oracle import planner_oracle as PO


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, PO.NPARAMS)
    x = rng.normal(0, 1, (12, 16))
    t = rng.normal(0, 1, (12, 3))
    mask = (rng.random((12, 3)) < 0.7).astype(float)
    g, _ = PO.grad(p, x, t, mask)
    h = 1e-6
    for i in rng.choice(np.arange(32, PO.NPARAMS), 60, replace=False):
        q = p.copy()
        q[i] += h
        lp = PO.grad(q, x, t, mask)[1]
        q[i] -= 2 * h
        lm = PO.grad(q, x, t, mask)[1]
        assert abs((lp - lm) / (2 * h) - g[i]) < 1e-5 * max(1.0, abs(g[i]))
    assert not g[:32].any()


def test_features_restatement_basic():
    lens = np.array([0, 10, 100, 1000], np.int64)
    dense = np.array([0, 0, 0, 1], bool)
    f = PO.features([np.array([1, 3, 9], np.uint32)], lens, dense, np.array([0, 32, 48, 256.0]),
                    (lens + 127) // 128, n_ads=4096, n_postings=1110, hybrid_min=50)
    assert f.shape == (1, 16)
    assert np.isclose(f[0, 0], np.log1p(2)) and np.isclose(f[0, 1], np.log1p(1010))
    assert np.isclose(f[0, 8], 1000 / 1010) and np.isclose(f[0, 11], np.log1p(1)) and f[0, 15] == 1.0
