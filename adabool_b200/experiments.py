"""Measurements beyond the default bench step: the batched graph executor on
config c2 and the learned planner on it (config c3), against the plain
per-query fixed-threshold path. Run through ``bench.py --mode planner``.

c2: 16,384 queries (lognormal term counts, median 40, sigma 2, [1, 20000]) on
    c1's index, one CUDA-graph launch per batch, bitmaps packed per query.
c3: the planner trained on ~200k timing samples (each of 66,667 fresh seeded
    queries timed alone on PROBE, UNION and HYBRID), judged by regret against
    the per-query best path and by batch speed against the fixed rule.
"""
from __future__ import annotations

import time

import numpy as np

from . import _native as N
from . import planner as P
from . import workload as W
from .executor import GraphBatchExecutor
from .index import Index


def _autotune_union(ix, cfg, lens, sub_batch, device):
    """The kernels' tuning for this index from the autotuner on 1,024 seeded
    queries of the config's shape: the dense threshold and the dense group
    kernel timed on the list-union path, then the merge kernel's tile shape
    timed on the hybrid path with its merge threshold (n_ads / 1024) fixed,
    as the two paths use different kernels."""
    from . import autotune as AT
    q = W.QueriesSpec(1024, cfg.queries.kind, cfg.queries.median, cfg.queries.sigma, cfg.queries.lo,
                      cfg.queries.hi, seed=cfg.queries.seed + 104729)
    qoff, qt = W.gen_queries(q, lens)
    sb = min(sub_batch, 1024)
    tu = AT.autotune(ix, qoff, qt, path=N.PATH_UNION, sub_batch=sb, sample=1024, device=device)
    hm = max(128, cfg.lists.n_ads // 1024)
    ix.set_tuning(heavy_min_len=hm)
    knobs = {k: AT.KNOBS[k] for k in ("tile_words", "warps_per_tile", "ctas_per_sm")}
    knobs["heavy_min_len"] = [hm]
    th = AT.autotune(ix, qoff, qt, path=N.PATH_HYBRID, sub_batch=sb, sample=1024, knobs=knobs, grid=False,
                     device=device)
    return {"union": dict(tu.best), "hybrid_tile_shape": dict(th.best)}


def _chunked_features(ix, qoff, qt, chunk, device):
    """Features computed in batches of `chunk` queries (the inference batch
    size), so batch-position features mean the same at training time."""
    out = []
    for a in range(0, qoff.size - 1, chunk):
        b = min(qoff.size - 1, a + chunk)
        out.append(P.features(ix, (qoff[a:b + 1] - qoff[a]).astype(np.uint64), qt[qoff[a]:qoff[b]], device))
    return np.concatenate(out)


def _time_replays(ex, reps):
    torch = ex.torch
    ex.replay()
    ex.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ex.stream)
    for _ in range(reps):
        ex.replay()
    e1.record(ex.stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


# offsets (in log-microseconds) tried on the planner's HYBRID output when it
# is calibrated on whole-batch timings; 0 keeps the trained model
CALIBRATION_OFFSETS = (-0.2, -0.1, 0.0, 0.1, 0.2, 0.4, 0.8, 1.6)
HYBRID_OUT = list(N.PLANNER_PATHS).index(N.PATH_HYBRID)


def planner_experiment(n_train: int = 66_667, batch_config: str = "c2", reps: int = 3, device: int = 0,
                       per_query_sample: int = 2048, fixed_tau=None, verbose: bool = False) -> dict:
    """fixed_tau: the fixed rule's probe threshold (from the reference
    kernels' crossover, measured by the caller), or a callable
    (index, q_off, q_terms, frac) -> dict with "tau" run on the evaluation
    batch; None calibrates it on this library's own timing labels."""
    import torch
    t_start = time.time()
    cfg = W.CONFIGS[batch_config]
    L = cfg.lists
    off, ads = W.gen_lists(L)
    lens = np.diff(off).astype(np.uint32)
    ix = Index.from_csr(off, ads, L.n_terms, L.n_ads, device=device)
    del off, ads
    B = cfg.queries.n_queries
    tuned = _autotune_union(ix, cfg, lens, min(B, 2048), device)
    # HYBRID merges per tile every list of at least n_ads/1024 postings (UNION
    # merges only the dense-bitmap lists), so the three paths differ; probe
    # slots for a whole batch, so PROBE labels really run the probe
    ix.set_tuning(heavy_min_len=max(128, L.n_ads // 1024), probe_cap=B)
    # --- training labels on fresh queries ---
    tq = W.QueriesSpec(n_train, cfg.queries.kind, cfg.queries.median, cfg.queries.sigma, cfg.queries.lo,
                       cfg.queries.hi, seed=cfg.queries.seed + 7919)
    tqoff, tqt = W.gen_queries(tq, lens)
    t0 = time.time()
    t_iso = P.collect_labels(ix, tqoff, tqt, device=device, verbose=verbose)
    t_lab = P.collect_labels_batched(ix, tqoff, tqt, t_iso, group=B, device=device)
    torch.cuda.empty_cache()
    label_s = time.time() - t0
    Xtr = _chunked_features(ix, tqoff, tqt, B, device)
    t0 = time.time()
    tr = P.train(Xtr, np.log(t_lab), epochs=120, batch=8192, lr=2e-3, device=device, verbose=verbose)
    train_s = time.time() - t0
    frac_tr = P.touched_fraction(ix, tqoff, tqt)
    tau_labels = P.calibrate_tau(frac_tr, t_lab)
    # --- evaluation batch ---
    qoff, qt = W.gen_queries(cfg.queries, lens)
    n = qoff.size - 1
    tau_info = {"source": "this library's timing labels", "tau": tau_labels}
    if callable(fixed_tau):
        tau_info = dict(fixed_tau(ix, qoff, qt, P.touched_fraction(ix, qoff, qt)),
                        source="crossover of the reference's kernels")
    elif fixed_tau is not None:
        tau_info = {"source": "given", "tau": float(fixed_tau)}
    tau = float(tau_info.get("tau", tau_labels))
    hyb_min = int(ix.tuning.fixed_hybrid_min_len)
    e_iso = P.collect_labels(ix, qoff, qt, device=device)
    e_lab = P.collect_labels_batched(ix, qoff, qt, e_iso, group=B, device=device)
    torch.cuda.empty_cache()
    Xev = _chunked_features(ix, qoff, qt, B, device)
    choice_fx = P.fixed_rule_choice(ix, qoff, qt, tau, hyb_min)
    paths_of = np.array(N.PLANNER_PATHS, np.uint8)
    # --- batch throughput: one graph launch per batch of B queries ---
    ex = GraphBatchExecutor(ix, n, int(qoff[-1]), path=N.PATH_HYBRID, per_query_paths=True, device=device)
    ex.capture()
    batch = {}
    ref_bm = None
    mism = 0
    for name, ch in (("fixed_rule", choice_fx), ("oracle_best", e_lab.argmin(1)), ("always_union", np.ones(n, int)),
                     ("always_hybrid", np.full(n, 2))):
        ex.set_batch(qoff, qt, paths_of[ch])
        ms = _time_replays(ex, reps)
        batch[name] = {"ms": ms, "queries_per_s": n / (ms / 1e3)}
        if ref_bm is None:
            ref_bm = ex.bitmaps.clone()
        else:
            mism += int(not torch.equal(ref_bm, ex.bitmaps))
    del ex
    torch.cuda.empty_cache()
    # --- calibration: the labels are isolated times rescaled to batch totals,
    # which can misjudge a path's cost inside a large batch; one offset on the
    # HYBRID output, chosen by timing whole batches of fresh queries (not the
    # evaluation batch), corrects the planner for it ---
    cspec = W.QueriesSpec(n, cfg.queries.kind, cfg.queries.median, cfg.queries.sigma, cfg.queries.lo,
                          cfg.queries.hi, seed=cfg.queries.seed + 104729)
    cqoff, cqt = W.gen_queries(cspec, lens)
    exa = GraphBatchExecutor(ix, n, max(int(qoff[-1]), int(cqoff[-1])), path=N.PATH_AUTO, per_query_paths=False,
                             device=device)
    P.install(ix, tr.params)
    exa.capture()
    exa.set_batch(cqoff, cqt)
    calib, best_d, best_ms = {}, 0.0, float("inf")
    for d in CALIBRATION_OFFSETS:
        pc = tr.params.copy()
        pc[P.OFF["b3"] + HYBRID_OUT] += d
        P.install(ix, pc)
        ms = _time_replays(exa, reps)
        calib[f"{d:+.2f}"] = round(n / (ms / 1e3), 1)
        if ms < best_ms:
            best_d, best_ms = d, ms
    params = tr.params.copy()
    params[P.OFF["b3"] + HYBRID_OUT] += best_d
    P.install(ix, params)
    choice_pl = P.mlp_predict(params, Xev, device).argmin(1)
    choice_raw = P.mlp_predict(tr.params, Xev, device).argmin(1)
    regret = {"planner": P.evaluate(e_lab, choice_pl), "fixed_rule": P.evaluate(e_lab, choice_fx),
              "planner_uncalibrated": P.evaluate(e_lab, choice_raw),
              "always_probe": P.evaluate(e_lab, np.zeros(n, int)), "always_union": P.evaluate(e_lab, np.ones(n, int)),
              "always_hybrid": P.evaluate(e_lab, np.full(n, 2)),
              "planner_on_isolated_labels": P.evaluate(e_iso, choice_pl),
              "fixed_rule_on_isolated_labels": P.evaluate(e_iso, choice_fx)}
    exa.set_batch(qoff, qt)
    ms = _time_replays(exa, reps)
    batch["planner"] = {"ms": ms, "queries_per_s": n / (ms / 1e3), "note": "planner kernel inside the graph",
                        "hybrid_output_offset": best_d}
    P.install(ix, tr.params)
    ms_raw = _time_replays(exa, reps)
    batch["planner_uncalibrated"] = {"ms": ms_raw, "queries_per_s": n / (ms_raw / 1e3)}
    P.install(ix, params)
    mism += int(not torch.equal(ref_bm, exa.bitmaps))
    planner_bm = exa.bitmaps
    # --- plain per-query fixed-threshold path: each query alone, one call per query ---
    m = min(per_query_sample, n)
    ws = ix.workspace(1, int(qoff[-1]))
    stride = (ix.n_words + 3) // 4 * 4
    bm1 = torch.empty(stride, dtype=torch.int32, device=device)
    dt, do = P.device_batch(qoff, qt, device)
    s = torch.cuda.Stream(device=device)
    import ctypes as C
    Lb = N.lib()

    def one(i, choice):
        b = N.Batch(N.ptr(dt), C.c_void_p(do.data_ptr() + 8 * i), 1, None, int(paths_of[choice[i]]), N.ptr(bm1),
                    stride, None, 0, None)
        N.check(Lb.abf_batch_run(ix.handle, ws.handle, C.byref(b), N.stream_ptr(s)))

    def per_query_ms(choice):
        for i in range(min(m, 16)):
            one(i, choice)
        s.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for i in range(m):
            one(i, choice)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)

    pq_ms = per_query_ms(choice_fx)
    for i in range(0, m, max(1, m // 32)):  # per-query results equal the batch rows
        one(i, choice_fx)
        s.synchronize()
        mism += int(not torch.equal(bm1[:ix.n_words], planner_bm[i, :ix.n_words]))
    per_query = {"queries": m, "ms": pq_ms, "queries_per_s": m / (pq_ms / 1e3),
                 "note": "abf_batch_run with one query per call, fixed-rule path, back to back on one stream"}
    # the same per-query path with the threshold fitted to this library's own
    # labels instead of the reference's crossover (a stronger fixed rule)
    pq_lab_ms = per_query_ms(P.fixed_rule_choice(ix, qoff, qt, tau_labels, hyb_min))
    per_query_lab = {"queries": m, "ms": pq_lab_ms, "queries_per_s": m / (pq_lab_ms / 1e3), "tau": tau_labels}
    P.uninstall(ix)
    return {
        "batch_config": batch_config, "n_queries": n, "terms": int(qoff[-1]),
        "train": {"queries": n_train, "samples": int(t_lab.size), "label_seconds": round(label_s, 1),
                  "train_seconds": round(train_s, 1), "train_mse": tr.train_loss, "val_mse": tr.val_loss,
                  "epochs": tr.epochs},
        "fixed_rule": {"tau": tau, "hybrid_min_len": hyb_min, "tau_from": tau_info, "tau_from_labels": tau_labels},
        "regret": regret, "batch": batch, "per_query_fixed": per_query,
        "per_query_fixed_label_tau": per_query_lab,
        "speedup_planner_batch_over_per_query_fixed_label_tau":
            batch["planner"]["queries_per_s"] / per_query_lab["queries_per_s"],
        "speedup_planner_over_always_hybrid_batch":
            batch["planner"]["queries_per_s"] / batch["always_hybrid"]["queries_per_s"],
        "speedup_planner_over_best_constant_batch":
            batch["planner"]["queries_per_s"] / max(batch["always_hybrid"]["queries_per_s"],
                                                    batch["always_union"]["queries_per_s"]),
        "calibration": {"offsets_qps": calib, "chosen": best_d,
                        "batch": "a fresh batch of the same size and query distribution (seed + 104729)"},
        "speedup_planner_batch_over_per_query_fixed": batch["planner"]["queries_per_s"] / per_query["queries_per_s"],
        "speedup_planner_over_fixed_rule_batch": batch["planner"]["queries_per_s"] / batch["fixed_rule"]["queries_per_s"],
        "bitmap_mismatches_across_choices": mism,
        "path_share": {"planner": np.bincount(choice_pl, minlength=3).tolist(),
                       "planner_uncalibrated": np.bincount(choice_raw, minlength=3).tolist(),
                       "fixed_rule": np.bincount(choice_fx, minlength=3).tolist(),
                       "best": np.bincount(e_lab.argmin(1), minlength=3).tolist()},
        "tuning": dict(ix.tuning.as_dict(), dense_div=ix.dense_div), "autotuned_union": tuned,
        "seconds": round(time.time() - t_start, 1), "params": tr.params,
    }


def _train_for_groups(ix, qoff, qt, iso, groups, device, verbose=False):
    """Planner trained on labels measured in batches of several sizes, each
    with its features computed in batches of the same size."""
    X, Y = [], []
    for g in groups:
        Y.append(P.collect_labels_batched(ix, qoff, qt, iso, group=g, device=device))
        X.append(_chunked_features(ix, qoff, qt, g, device))
    X, Y = np.concatenate(X), np.concatenate(Y)
    tr = P.train(X, np.log(Y), epochs=120, batch=8192, lr=2e-3, device=device, verbose=verbose)
    return tr, X, Y


def serving_experiment(rates=(20_000, 50_000, 100_000, 200_000), offered_seconds: float = 0.5,
                       min_queries: int = 4000, n_train: int = 20_000, label_groups=(32, 256, 1024),
                       budget_bytes: int = 40 << 30, window_us: int = 100, max_batch_queries: int = 1024,
                       n_streams: int = 4, device: int = 0, planner_params=None, verbose: bool = False) -> dict:
    """Config c4: open-loop Poisson arrivals on c1's index, served by the
    batching server with the learned planner, by the same server with the
    fixed threshold rule, and by the plain per-query fixed-rule path (one
    query per abf_batch_run, one stream); throughput and latency
    percentiles per arrival rate."""
    import torch
    from .server import Server, latency_summary, poisson_arrivals
    t_start = time.time()
    cfg = W.CONFIGS["c4"]
    L = cfg.lists
    off, ads = W.gen_lists(L)
    lens = np.diff(off).astype(np.uint32)
    ix = Index.from_csr(off, ads, L.n_terms, L.n_ads, device=device)
    del off, ads
    tuned = _autotune_union(ix, cfg, lens, 256, device)
    ix.set_tuning(heavy_min_len=max(128, L.n_ads // 1024), probe_cap=max_batch_queries)
    # --- planner and fixed-rule threshold from batched timing labels ---
    tq = W.QueriesSpec(n_train, cfg.queries.kind, cfg.queries.median, cfg.queries.sigma, cfg.queries.lo,
                       cfg.queries.hi, seed=cfg.queries.seed + 7919)
    tqoff, tqt = W.gen_queries(tq, lens)
    t0 = time.time()
    iso = P.collect_labels(ix, tqoff, tqt, device=device, verbose=verbose)
    tr, _, Y = _train_for_groups(ix, tqoff, tqt, iso, label_groups, device, verbose)
    if planner_params is not None:
        tr.params = np.asarray(planner_params, np.float32)
    frac = np.tile(P.touched_fraction(ix, tqoff, tqt), len(label_groups))
    tau = P.calibrate_tau(frac, Y)
    ix.set_tuning(probe_min_fraction=tau)
    train_s = time.time() - t0
    torch.cuda.empty_cache()
    # --- arrivals ---
    n_max = max(int(max(rates) * offered_seconds), min_queries)
    qspec = W.QueriesSpec(n_max, cfg.queries.kind, cfg.queries.median, cfg.queries.sigma, cfg.queries.lo,
                          cfg.queries.hi, seed=cfg.queries.seed)
    qoff, qt = W.gen_queries(qspec, lens)
    servers = {
        "planner_batched": dict(path=N.PATH_AUTO, planner=True, max_batch_queries=max_batch_queries,
                                n_streams=n_streams, window_us=window_us),
        "fixed_rule_batched": dict(path=N.PATH_AUTO, planner=False, max_batch_queries=max_batch_queries,
                                   n_streams=n_streams, window_us=window_us),
        "per_query_fixed_rule": dict(path=N.PATH_AUTO, planner=False, max_batch_queries=1, n_streams=1,
                                     window_us=0),
    }
    runs = []
    for rate in rates:
        n = max(int(rate * offered_seconds), min_queries)
        arr = poisson_arrivals(rate, n, seed=int(rate))
        sub_off = qoff[:n + 1]
        sub_t = qt[:int(sub_off[-1])]
        ref_ids = None
        for name, sc in servers.items():
            if sc["planner"]:
                P.install(ix, tr.params)
            else:
                P.uninstall(ix)
            with Server(ix, budget_bytes=budget_bytes, window_us=sc["window_us"],
                        max_batch_queries=sc["max_batch_queries"], n_streams=sc["n_streams"],
                        path=sc["path"]) as srv:
                out = srv.run_trace(sub_off, sub_t, arr, timeout_s=600)
                st = srv.stats()
            mism = 0
            if ref_ids is None:
                ref_ids = out["n_ids"]
            else:
                mism = int((out["n_ids"] != ref_ids).sum())
            rec = {"rate_qps": rate, "server": name, "queries": n, "completed": out["completed"],
                   "rejected": out["rejected"], "failed": out["failed"], "seconds": out["seconds"],
                   "throughput_qps": out["completed"] / max(out["seconds"], 1e-9),
                   **latency_summary(out["latency_ns"]),
                   "queue_p50_us": float(np.percentile(out["queue_ns"][out["queue_ns"] != np.iinfo(np.uint64).max],
                                                       50)) / 1e3,
                   "batches": st["batches"], "mean_batch": st["completed"] / max(st["batches"], 1),
                   "max_batch": st["max_batch_queries_seen"], "admission_waits": st["admission_waits"],
                   "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9,
                   "paths": {N.PATH_NAMES[p]: int(c) for p, c in enumerate(st["path_queries"]) if c},
                   "id_count_mismatches_vs_first_server": mism}
            if verbose:
                print(rec, flush=True)
            runs.append(rec)
    P.uninstall(ix)
    return {"config": "c4", "index": {"n_terms": L.n_terms, "n_ads": L.n_ads, "nnz": L.nnz},
            "queries": {"median_terms": cfg.queries.median, "sigma": cfg.queries.sigma, "max_terms": cfg.queries.hi},
            "budget_bytes": budget_bytes, "window_us": window_us, "max_batch_queries": max_batch_queries,
            "n_streams": n_streams, "fixed_rule_tau": tau,
            "planner_train": {"queries": n_train, "groups": list(label_groups), "samples": int(Y.shape[0]),
                              "val_mse": tr.val_loss, "seconds": round(train_s, 1)},
            "runs": runs, "tuning": dict(ix.tuning.as_dict(), dense_div=ix.dense_div), "autotuned_union": tuned,
            "seconds": round(time.time() - t_start, 1), "params": tr.params}


def index_experiment(configs=("c0", "c1"), path_dir: str = "/tmp", device: int = 0, n_threads: int = 0) -> dict:
    """On-disk index and builder: per config, the parallel build from COO
    pairs and from CSR lists (host arrays -> device-resident index), the
    binary file's size, save time, and load time (one read + uploads)."""
    import os
    import torch
    from . import _native as NN
    out = {}
    for c in configs:
        cfg = W.CONFIGS[c] if isinstance(c, str) else c
        name = cfg.name
        L = cfg.lists
        off, ads = W.gen_lists(L)
        terms = np.repeat(np.arange(L.n_terms, dtype=np.uint32), np.diff(off).astype(np.int64))
        rec = {"n_terms": L.n_terms, "n_ads": L.n_ads, "nnz": int(ads.size)}
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ix = Index.from_coo(terms, ads, L.n_terms, L.n_ads, device=device, n_threads=n_threads)
        torch.cuda.synchronize()
        rec["build_coo_sorted_s"] = time.perf_counter() - t0
        del ix
        perm = np.random.default_rng(7).permutation(terms.size)  # COO pairs in no particular order
        t_coo, a_coo = terms[perm], ads[perm]
        del terms, perm
        t0 = time.perf_counter()
        ix = Index.from_coo(t_coo, a_coo, L.n_terms, L.n_ads, device=device, n_threads=n_threads)
        torch.cuda.synchronize()
        rec["build_coo_shuffled_s"] = time.perf_counter() - t0
        del ix, t_coo, a_coo
        t0 = time.perf_counter()
        ix = Index.from_csr(off, ads, L.n_terms, L.n_ads, device=device, n_threads=n_threads)
        torch.cuda.synchronize()
        rec["build_csr_s"] = time.perf_counter() - t0
        st = ix.stats()
        rec.update(payload_bytes=st["payload_bytes"], device_bytes=st["device_bytes"])
        f = os.path.join(path_dir, f"abf_index_{name}.bin")
        t0 = time.perf_counter()
        ix.save(f)
        rec["save_s"] = time.perf_counter() - t0
        rec["file_bytes"] = os.path.getsize(f)
        del ix
        t0 = time.perf_counter()
        ix2 = Index.load(f, device=device)
        torch.cuda.synchronize()
        rec["load_s"] = time.perf_counter() - t0
        rec["load_gbs"] = rec["file_bytes"] / rec["load_s"] / 1e9
        del ix2
        os.remove(f)
        rec["threads"] = n_threads or os.cpu_count()
        out[name] = rec
    return out
