"""CPU oracle for the learned planner (TEST INFRASTRUCTURE ONLY).

Float64 numpy restatements of the planner's 16 features
(adabool_b200/csrc/abf_planner.cu, query_features) and of the MLP's forward
pass and mean-squared-error gradient (mlp_grad_kernel), used by the tests to
check the device kernels. The planner has no counterpart in the reference,
so these restate this project's own definitions.
"""
from __future__ import annotations

import numpy as np

F, H, O = 16, 64, 3
OFF = {"mu": 0, "sd": 16, "W1": 32, "b1": 32 + H * F}
OFF["W2"] = OFF["b1"] + H
OFF["b2"] = OFF["W2"] + H * H
OFF["W3"] = OFF["b2"] + H
OFF["b3"] = OFF["W3"] + O * H
NPARAMS = OFF["b3"] + O


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF["W1"]:OFF["b1"]].reshape(H, F), p[OFF["b1"]:OFF["W2"]], p[OFF["W2"]:OFF["b2"]].reshape(H, H),
            p[OFF["b2"]:OFF["W3"]], p[OFF["W3"]:OFF["b3"]].reshape(O, H), p[OFF["b3"]:NPARAMS])


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    return h1, h2, h2 @ W3.T + b3


def grad(p, x, t, mask):
    """Gradient of sum(mask * (y - t)^2) / sum(mask) in the parameter layout."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    h1, h2, y = forward(p, x)
    m = (np.asarray(mask) != 0).astype(np.float64)
    ms = max(m.sum(), 1.0)
    r = m * (y - t)
    loss = (r * r).sum() / ms
    dy = 2 * r / ms
    g = np.zeros(NPARAMS)
    g[OFF["W3"]:OFF["b3"]] = (dy.T @ h2).ravel()
    g[OFF["b3"]:NPARAMS] = dy.sum(0)
    dh2 = (dy @ W3) * (h2 > 0)
    g[OFF["W2"]:OFF["b2"]] = (dh2.T @ h1).ravel()
    g[OFF["b2"]:OFF["W3"]] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g[OFF["W1"]:OFF["b1"]] = (dh1.T @ x).ravel()
    g[OFF["b1"]:OFF["W2"]] = dh1.sum(0)
    return g, loss


def features(q_terms_list, lens, dense, cbytes, nblocks, n_ads, n_postings, hybrid_min):
    """Features of every query of a batch (list of term arrays), float64."""
    n_q = len(q_terms_list)
    out = np.zeros((n_q, F))
    n_terms = len(lens)
    for q, terms in enumerate(q_terms_list):
        t = np.asarray([x for x in terms if x < n_terms], np.int64)
        ln = lens[t].astype(np.float64)
        d = dense[t].astype(bool)
        n = t.size
        S = ln.sum()
        mx = ln.max() if n else 0.0
        mean = S / max(n, 1)
        var = max((ln * ln).sum() / max(n, 1) - mean * mean, 0.0)
        Lg = np.log1p(-np.minimum(ln / n_ads, 0.999999)).sum()
        Sd = ln[d].sum()
        Bnd = nblocks[t][~d].sum()
        nl = int(((ln < hybrid_min) & ~d).sum())
        out[q] = [np.log1p(n), np.log1p(S), np.log1p(mx), np.log1p(mean), np.log1p(np.sqrt(var)),
                  np.log1p(cbytes[t].sum()), 1 - np.exp(Lg), np.log1p(d.sum()), Sd / max(S, 1.0), np.log1p(Bnd),
                  S / max(n_postings, 1), np.log1p(nl), q / max(n_q, 1), np.log1p(n_q), mx / n_ads, 1.0]
    return out
