"""Learned path planner: timing labels from the kernels, GPU training, evaluation.

The planner predicts, per query, log(microseconds) of each of the PROBE,
UNION and HYBRID paths from 16 device-computed features and takes the
cheapest (include/adabool.h, abf_planner_*). Here:

  collect_labels  answers each query alone through abf_batch_run once per
                  path and times it with CUDA events on the launching stream
  train           fits the MLP with the library's own forward/backward and
                  Adam kernels (abf_mlp_grad / abf_mlp_adam), MSE on log us
  fixed_rule      the fallback: probe when the query's lists cover more than
                  tau of all blocks, else HYBRID when one of its lists is as
                  dense as a bucket the reference stores as a bitset, else
                  list-union; tau from the crossover of the reference's own
                  kernels (measured on the oracle side) or from labels
  evaluate        regret against the per-query best path

Results are bit-exact whatever path is chosen; only time changes. The
reference has no planner: its drivers run both paths on every query
(test/adsfilter_q_all.cu:414-452).
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native as N
from ._native import check, lib, ptr, stream_ptr

F, HID, O = N.PLANNER_FEATURES, N.PLANNER_HIDDEN, N.PLANNER_OUTPUTS
PATHS = N.PLANNER_PATHS
OFF = {"mu": 0, "sd": 16, "W1": 32, "b1": 32 + HID * F}
OFF["W2"] = OFF["b1"] + HID
OFF["b2"] = OFF["W2"] + HID * HID
OFF["W3"] = OFF["b2"] + HID
OFF["b3"] = OFF["W3"] + O * HID
assert OFF["b3"] + O == N.PLANNER_PARAMS


def init_params(mu: np.ndarray, sd: np.ndarray, seed: int = 0) -> np.ndarray:
    """He-initialised parameters with the given feature standardisation."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N.PLANNER_PARAMS, np.float32)
    p[OFF["mu"]:OFF["mu"] + F] = mu
    p[OFF["sd"]:OFF["sd"] + F] = np.where(sd > 1e-6, sd, 1.0)
    p[OFF["W1"]:OFF["b1"]] = rng.normal(0, np.sqrt(2.0 / F), HID * F)
    p[OFF["W2"]:OFF["b2"]] = rng.normal(0, np.sqrt(2.0 / HID), HID * HID)
    p[OFF["W3"]:OFF["b3"]] = rng.normal(0, np.sqrt(1.0 / HID), O * HID)
    return p


def _torch():
    import torch
    return torch


def device_batch(q_off: np.ndarray, q_terms: np.ndarray, device: int = 0):
    torch = _torch()
    dt = torch.from_numpy(np.ascontiguousarray(q_terms, np.uint32).view(np.int32)).to(device) if q_terms.size else \
        torch.zeros(1, dtype=torch.int32, device=device)
    do = torch.from_numpy(np.ascontiguousarray(q_off, np.uint64).view(np.int64)).to(device)
    return dt, do


def features(index, q_off: np.ndarray, q_terms: np.ndarray, device: int = 0) -> np.ndarray:
    """Raw features (n x 16) computed by the library's device kernel."""
    torch = _torch()
    n = q_off.size - 1
    dt, do = device_batch(q_off, q_terms, device)
    out = torch.empty((max(n, 1), F), dtype=torch.float32, device=device)
    check(lib().abf_planner_features(index.handle, ptr(dt), ptr(do), n, ptr(out), None))
    torch.cuda.synchronize(device)
    return out[:n].cpu().numpy()


def collect_labels(index, q_off: np.ndarray, q_terms: np.ndarray, paths=PATHS, device: int = 0, chunk: int = 512,
                   verbose: bool = False) -> np.ndarray:
    """Device microseconds of each path for each query answered alone
    (bitmap only): n x len(paths)."""
    torch = _torch()
    n = q_off.size - 1
    dt, do = device_batch(q_off, q_terms, device)
    ws = index.workspace(1, max(int(q_off[-1]), 1))
    stride = (index.n_words + 3) // 4 * 4
    bm = torch.empty(stride, dtype=torch.int32, device=device)
    s = torch.cuda.Stream(device=device)
    out = np.zeros((n, len(paths)), np.float64)
    L = lib()

    def run(i, p):
        b = N.Batch(ptr(dt), C.c_void_p(do.data_ptr() + 8 * i), 1, None, p, ptr(bm), stride, None, 0, None)
        check(L.abf_batch_run(index.handle, ws.handle, C.byref(b), stream_ptr(s)))

    for i in range(min(n, 8)):  # warm-up
        for p in paths:
            run(i, p)
    s.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(chunk * len(paths))]
    t0 = time.time()
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        k = 0
        for i in range(c0, c1):
            for p in paths:
                ev[k][0].record(s)
                run(i, p)
                ev[k][1].record(s)
                k += 1
        s.synchronize()
        k = 0
        for i in range(c0, c1):
            for j in range(len(paths)):
                out[i, j] = ev[k][0].elapsed_time(ev[k][1]) * 1e3
                k += 1
        if verbose and (c0 // chunk) % 20 == 0:
            print(f"  labels {c1}/{n} ({time.time() - t0:.1f} s)", flush=True)
    ws.free()
    return out


def collect_labels_batched(index, q_off: np.ndarray, q_terms: np.ndarray, iso: np.ndarray, group: int = 512,
                           paths=PATHS, device: int = 0) -> np.ndarray:
    """Per-query labels in batch context: the queries are cut into groups of
    `group` (enough that the group's bitmaps do not fit in L2, as in a large
    batch), every group runs once per path as one batch with all its queries
    on that path, and each query's isolated time `iso` (n x paths) is scaled
    so the group's labels add up to the measured batch time of that path."""
    torch = _torch()
    n = q_off.size - 1
    dt, do = device_batch(q_off, q_terms, device)
    ws = index.workspace(group, max(int(q_off[-1]), 1))
    stride = (index.n_words + 3) // 4 * 4
    bms = torch.empty((group, stride), dtype=torch.int32, device=device)
    s = torch.cuda.Stream(device=device)
    L = lib()
    out = np.zeros_like(iso)

    def run(a, b, p):
        bt = N.Batch(ptr(dt), C.c_void_p(do.data_ptr() + 8 * a), b - a, None, p, ptr(bms), stride, None, 0, None)
        check(L.abf_batch_run(index.handle, ws.handle, C.byref(bt), stream_ptr(s)))

    run(0, min(n, group), PATHS[1])
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for a in range(0, n, group):
        b = min(n, a + group)
        for j, p in enumerate(paths):
            e0.record(s)
            run(a, b, p)
            e1.record(s)
            e1.synchronize()
            t_us = e0.elapsed_time(e1) * 1e3
            w = iso[a:b, j]
            out[a:b, j] = w * (t_us / max(w.sum(), 1e-9))
    ws.free()
    return out


@dataclass
class TrainResult:
    params: np.ndarray
    train_loss: float
    val_loss: float
    epochs: int
    seconds: float


def mlp_predict(params: np.ndarray, X: np.ndarray, device: int = 0) -> np.ndarray:
    """MLP outputs (n x 3) for raw features, through abf_mlp_forward."""
    torch = _torch()
    mu, sd = params[:F], params[F:2 * F]
    xs = ((X - mu) / sd).astype(np.float32)
    dp = torch.from_numpy(params.astype(np.float32)).to(device)
    dx = torch.from_numpy(np.ascontiguousarray(xs)).to(device)
    dy = torch.empty((max(len(X), 1), O), dtype=torch.float32, device=device)
    check(lib().abf_mlp_forward(ptr(dp), ptr(dx), len(X), ptr(dy), None))
    torch.cuda.synchronize(device)
    return dy[:len(X)].cpu().numpy()


def train(X: np.ndarray, T: np.ndarray, mask: np.ndarray | None = None, val_frac: float = 0.1, epochs: int = 200,
          batch: int = 8192, lr: float = 2e-3, seed: int = 0, device: int = 0, verbose: bool = False) -> TrainResult:
    """Adam on MSE of log-microsecond targets T (n x 3), GPU kernels only."""
    torch = _torch()
    L = lib()
    n = len(X)
    mask = np.ones_like(T, dtype=np.float32) if mask is None else mask.astype(np.float32)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    nv = max(1, int(n * val_frac))
    va, tr = perm[:nv], perm[nv:]
    mu = X[tr].mean(0)
    sd = X[tr].std(0)
    params = init_params(mu, sd, seed)
    sdd = np.where(sd > 1e-6, sd, 1.0)
    Xs = ((X - mu) / sdd).astype(np.float32)
    dev = torch.device("cuda", device)
    dx = torch.from_numpy(Xs).to(dev)
    dt = torch.from_numpy(T.astype(np.float32)).to(dev)
    dm = torch.from_numpy(mask).to(dev)
    dp = torch.from_numpy(params).to(dev)
    g = torch.zeros(N.PLANNER_PARAMS, dtype=torch.float32, device=dev)
    m1 = torch.zeros_like(g)
    m2 = torch.zeros_like(g)
    loss = torch.zeros(2, dtype=torch.float32, device=dev)
    tr_t = torch.from_numpy(tr).to(dev)
    va_t = torch.from_numpy(va).to(dev)
    xv, tv, mv = dx[va_t].contiguous(), dt[va_t].contiguous(), dm[va_t].contiguous()
    step = 0
    t0 = time.time()
    tl = vl = float("nan")
    for ep in range(epochs):
        order = tr_t[torch.randperm(tr_t.numel(), device=dev)]
        for b0 in range(0, order.numel(), batch):
            idx = order[b0:b0 + batch]
            xb, tb, mb = dx[idx].contiguous(), dt[idx].contiguous(), dm[idx].contiguous()
            check(L.abf_mlp_grad(ptr(dp), ptr(xb), ptr(tb), ptr(mb), idx.numel(), ptr(g), ptr(loss), None))
            step += 1
            check(L.abf_mlp_adam(ptr(dp), ptr(g), ptr(m1), ptr(m2), step, lr, 0.9, 0.999, 1e-8, None))
        if ep == epochs - 1 or (verbose and ep % 20 == 0):
            tl = float(loss[0].item())
            check(L.abf_mlp_grad(ptr(dp), ptr(xv), ptr(tv), ptr(mv), len(va), ptr(g), ptr(loss), None))
            vl = float(loss[0].item())
            if verbose:
                print(f"  epoch {ep}: train {tl:.4f} val {vl:.4f}", flush=True)
    return TrainResult(dp.cpu().numpy(), tl, vl, epochs, time.time() - t0)


def touched_fraction(index, q_off: np.ndarray, q_terms: np.ndarray) -> np.ndarray:
    """Fraction of all blocks the query's lists hold (the fixed rule's measure)."""
    lens = index.list_lengths().astype(np.int64)
    nblk = (lens + 127) // 128
    total = max(int(nblk.sum()), 1)
    valid = q_terms < index.n_terms
    b = np.where(valid, nblk[np.minimum(q_terms, index.n_terms - 1)], 0)
    s = np.add.reduceat(b, q_off[:-1].astype(np.int64)) if q_terms.size else np.zeros(q_off.size - 1)
    s = np.where(np.diff(q_off) == 0, 0, s)
    return s / total


def max_list_len(index, q_off: np.ndarray, q_terms: np.ndarray) -> np.ndarray:
    """Longest list of each query (0 for an empty one)."""
    lens = index.list_lengths().astype(np.int64)
    valid = q_terms < index.n_terms
    m = np.where(valid, lens[np.minimum(q_terms, index.n_terms - 1)], 0)
    out = np.maximum.reduceat(m, q_off[:-1].astype(np.int64)) if q_terms.size else np.zeros(q_off.size - 1)
    return np.where(np.diff(q_off) == 0, 0, out)


def fixed_rule_choice(index, q_off: np.ndarray, q_terms: np.ndarray, tau: float, hybrid_min: int) -> np.ndarray:
    """Output index (0 PROBE, 1 UNION, 2 HYBRID) the fixed rule of the plan
    kernel picks: PROBE when the query's lists hold more than tau of all
    blocks, else HYBRID when one of them has at least hybrid_min postings
    (0: never), else UNION."""
    frac = touched_fraction(index, q_off, q_terms)
    mx = max_list_len(index, q_off, q_terms)
    hyb = (mx >= hybrid_min) if hybrid_min else np.zeros(mx.shape, bool)
    return np.where(frac > tau, 0, np.where(hyb, 2, 1))


def calibrate_tau(frac: np.ndarray, times: np.ndarray) -> float:
    """tau minimising the total time of 'probe if frac > tau else union' on labelled queries."""
    cand = np.unique(np.concatenate([[0.0, 1.0], frac]))
    best, best_t = 1.0, np.inf
    for tau in cand:
        tot = np.where(frac > tau, times[:, 0], times[:, 1]).sum()
        if tot < best_t:
            best, best_t = float(tau), tot
    return best


def evaluate(times: np.ndarray, choice_idx: np.ndarray) -> dict:
    """Total time of a per-query choice against the per-query best (regret)."""
    best = times.min(1).sum()
    got = times[np.arange(len(times)), choice_idx].sum()
    return {"total_us": float(got), "best_us": float(best), "regret": float(got / best - 1.0),
            "agreement": float((choice_idx == times.argmin(1)).mean())}


def install(index, params: np.ndarray):
    check(lib().abf_planner_set(index.handle, ptr(np.ascontiguousarray(params, np.float32))))


def uninstall(index):
    check(lib().abf_planner_set(index.handle, None))


def save(params: np.ndarray, path, meta: dict | None = None):
    np.save(Path(path), params.astype(np.float32))
    if meta is not None:
        Path(str(path) + ".json").write_text(json.dumps(meta, indent=1))
