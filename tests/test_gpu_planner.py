"""Learned planner kernels against the CPU oracle (oracle/planner_oracle.py).

Tolerances (FP32 device kernels against float64 numpy):
  features      rtol 1e-5, atol 1e-6
  MLP forward   rtol 1e-4, atol 1e-4
  gradients     |g_dev - g_ref| <= 1e-3 * max|g_ref| + 1e-4 * |g_ref|
  Adam step     rtol 1e-5, atol 1e-6
"""
import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, planner as P, workload as W
from adabool_b200 import _native as N
from oracle import oracle as O
from oracle import planner_oracle as PO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(dev):
    spec = W.ListsSpec(n_terms=3000, n_ads=65_537, nnz=300_000, zipf_s=1.1, max_len=25_000, seed=8)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off).astype(np.uint32)
    qoff, qt = W.gen_queries(W.QueriesSpec(40, "lognormal", 10.0, 1.5, 1, 400, seed=9), lens)
    qt = qt.copy()
    qt[3] = spec.n_terms + 7  # an out-of-range term
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, device=0)
    return dict(spec=spec, off=off, ads=ads, lens=lens, qoff=qoff, qt=qt, ix=ix)


def test_features_match_oracle(env):
    ix, qoff, qt = env["ix"], env["qoff"], env["qt"]
    got = P.features(ix, qoff, qt)
    lens = ix.list_lengths()
    exp = PO.features([qt[qoff[i]:qoff[i + 1]] for i in range(qoff.size - 1)], lens, (ix.list_flags() & 1) != 0,
                      ix.list_bytes().astype(np.float64), (lens.astype(np.int64) + 127) // 128, ix.n_ads,
                      ix.stats()["n_postings"], ix.tuning.heavy_min_len)
    assert np.allclose(got, exp, rtol=1e-5, atol=1e-6), np.abs(got - exp).max(0)


def _rand_problem(rng, n):
    x = rng.normal(0, 1, (n, 16)).astype(np.float32)
    t = rng.normal(3, 1, (n, 3)).astype(np.float32)
    mask = (rng.random((n, 3)) < 0.8).astype(np.float32)
    p = P.init_params(np.zeros(16), np.ones(16), seed=int(rng.integers(1000)))
    p[PO.OFF["b1"]:PO.OFF["W2"]] = rng.normal(0, 0.1, 64)
    return x, t, mask, p


def test_forward_and_gradient_match_oracle(dev):
    import torch
    rng = np.random.default_rng(5)
    for n in (1, 37, 5000):
        x, t, mask, p = _rand_problem(rng, n)
        y = P.mlp_predict(p, x)
        assert np.allclose(y, PO.forward(p, x.astype(np.float64))[2], rtol=1e-4, atol=1e-4)
        dp, dx, dt, dm = (torch.from_numpy(a).cuda() for a in (p, x, t, mask))
        g = torch.zeros(N.PLANNER_PARAMS, dtype=torch.float32, device="cuda")
        loss = torch.zeros(2, dtype=torch.float32, device="cuda")
        N.check(ab.lib().abf_mlp_grad(N.ptr(dp), N.ptr(dx), N.ptr(dt), N.ptr(dm), n, N.ptr(g), N.ptr(loss), None))
        torch.cuda.synchronize()
        g_ref, l_ref = PO.grad(p, x, t, mask)
        gd = g.cpu().numpy().astype(np.float64)
        tol = 1e-3 * np.abs(g_ref).max() + 1e-4 * np.abs(g_ref)
        assert np.all(np.abs(gd - g_ref) <= tol), np.abs(gd - g_ref).max()
        assert abs(loss[0].item() - l_ref) <= 1e-4 * max(l_ref, 1.0)
        assert loss[1].item() == float((mask != 0).sum())
        assert not gd[:32].any()  # standardisation entries get no gradient


def test_adam_step(dev):
    import torch
    rng = np.random.default_rng(1)
    p = rng.normal(0, 1, N.PLANNER_PARAMS).astype(np.float32)
    g = rng.normal(0, 1, N.PLANNER_PARAMS).astype(np.float32)
    m = rng.normal(0, 0.1, N.PLANNER_PARAMS).astype(np.float32)
    v = rng.random(N.PLANNER_PARAMS).astype(np.float32)
    dp, dg, dm, dv = (torch.from_numpy(a.copy()).cuda() for a in (p, g, m, v))
    step, lr, b1, b2, eps = 7, 1e-3, 0.9, 0.999, 1e-8
    N.check(ab.lib().abf_mlp_adam(N.ptr(dp), N.ptr(dg), N.ptr(dm), N.ptr(dv), step, lr, b1, b2, eps, None))
    torch.cuda.synchronize()
    m2 = b1 * m + (1 - b1) * g
    v2 = b2 * v + (1 - b2) * g * g
    p2 = p - lr * (m2 / (1 - b1 ** step)) / (np.sqrt(v2 / (1 - b2 ** step)) + eps)
    p2[:32] = p[:32]
    assert np.allclose(dp.cpu().numpy(), p2, rtol=1e-5, atol=1e-6)


def test_training_fits_a_smooth_target(dev):
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (20000, 16))
    T = np.stack([X[:, 0] * 0.5 + 1, np.abs(X[:, 1]), X[:, 2] ** 2 * 0.3], 1)
    r = P.train(X, T, epochs=60, batch=2048, lr=3e-3)
    base = ((T - T.mean(0)) ** 2).mean()
    assert r.val_loss < 0.1 * base, (r.val_loss, base)


def test_planner_choices_and_bit_exact_auto_batches(env):
    import torch
    ix, qoff, qt = env["ix"], env["qoff"], env["qt"]
    n = qoff.size - 1
    feats = P.features(ix, qoff, qt)
    rng = np.random.default_rng(3)
    p = P.init_params(feats.mean(0), feats.std(0), seed=4)
    P.install(ix, p)
    try:
        dt, do = P.device_batch(qoff, qt)
        pred = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        paths = torch.zeros(n, dtype=torch.uint8, device="cuda")
        N.check(ab.lib().abf_planner_predict(ix.handle, N.ptr(dt), N.ptr(do), n, N.ptr(pred), N.ptr(paths), None))
        torch.cuda.synchronize()
        y = P.mlp_predict(p, feats)
        assert np.allclose(pred.cpu().numpy(), y, rtol=1e-4, atol=1e-4)
        assert np.array_equal(paths.cpu().numpy(), np.array(N.PLANNER_PATHS)[y.argmin(1)])
        # random weights that favour every path somewhere: results stay exact
        p2 = p.copy()
        p2[PO.OFF["b3"]:] = [0.0, 0.0, 0.0]
        p2[PO.OFF["W3"]:PO.OFF["b3"]] = rng.normal(0, 1, 192)
        P.install(ix, p2)
        n_words = (env["spec"].n_ads + 31) // 32
        stride = (n_words + 3) // 4 * 4
        ws = ix.workspace(n, int(qoff[-1]))
        bms = torch.empty((n, stride), dtype=torch.int32, device="cuda")
        ix.set_tuning(probe_cap=64)  # every probe choice gets a probe slot (no fallback to UNION)
        ix.batch_run(ws, dt, do, n, bms, stride, path=ab.PATH_AUTO)
        ws.check()
        # the plan kernel's inline planner picks what the planner kernel picks
        N.check(ab.lib().abf_planner_predict(ix.handle, N.ptr(dt), N.ptr(do), n, None, N.ptr(paths), None))
        torch.cuda.synchronize()
        assert np.array_equal(ws.paths(n), paths.cpu().numpy())
        assert len(np.unique(ws.paths(n))) >= 2  # the random weights favour more than one path
        got = bms.cpu().numpy().view(np.uint32)
        for i in range(n):
            e = O.ids_to_bitmap(O.kway_union(env["off"], env["ads"], qt[qoff[i]:qoff[i + 1]]), n_words)
            assert np.array_equal(got[i, :n_words], e), i
    finally:
        P.uninstall(ix)
        ix.set_tuning(probe_cap=32)


def test_collect_labels_shapes(env):
    ix, qoff, qt = env["ix"], env["qoff"], env["qt"]
    t = P.collect_labels(ix, qoff[:11], qt[:qoff[10]])
    assert t.shape == (10, 3) and (t > 0).all()


def test_fixed_rule_paths_match_host_restatement(env):
    """Without a planner, ABF_PATH_AUTO takes the fixed rule in the plan
    kernel; the path of every query equals planner.fixed_rule_choice (the
    host restatement used to score the rule on labels)."""
    import torch
    ix, qoff, qt = env["ix"], env["qoff"], env["qt"]
    n = qoff.size - 1
    frac = P.touched_fraction(ix, qoff, qt)
    mx = P.max_list_len(ix, qoff, qt)
    fs = np.unique(frac)
    tau = float((fs[len(fs) // 2] + fs[len(fs) // 2 + 1]) / 2)  # between two queries' fractions
    hyb = int(np.median(mx[frac <= tau])) + 1
    old = ix.tuning
    ix.set_tuning(probe_min_fraction=tau, fixed_hybrid_min_len=hyb, probe_cap=64)
    try:
        n_words = (env["spec"].n_ads + 31) // 32
        stride = (n_words + 3) // 4 * 4
        ws = ix.workspace(n, int(qoff[-1]))
        bms = torch.empty((n, stride), dtype=torch.int32, device="cuda")
        dt, do = P.device_batch(qoff, qt)
        ix.batch_run(ws, dt, do, n, bms, stride, path=ab.PATH_AUTO)
        ws.check()
        want = np.array(N.PLANNER_PATHS)[P.fixed_rule_choice(ix, qoff, qt, tau, hyb)]
        got = ws.paths(n)
        assert len(np.unique(want)) == 3  # the thresholds split the queries over all three paths
        assert np.array_equal(got, want), (got, want)
    finally:
        ix.set_tuning(probe_min_fraction=old.probe_min_fraction, fixed_hybrid_min_len=old.fixed_hybrid_min_len,
                      probe_cap=32)
