#!/usr/bin/env python
"""Benchmark of the Boolean-filtering hot path on one or more B200s.

Workload (default, config c1): a synthetic filter matrix of 2^20 terms x 2^24
ads with ~500M postings (Zipf(1.05) list lengths clipped to [1, 5M], uniform
sorted unique ad ids per list) and 2,048 queries of distinct terms (lognormal
term counts, median 40, sigma 1.5, clipped to [1, 5000]; terms drawn with
probability proportional to list length). One step answers every query:
bitmap (2^24 bits) plus sorted uint32 id list per query, through the batched
API in sub-batches. Inputs are larger than L2 (the compressed index alone is
~0.8 GB), so no flush is needed between steps.

  value  queries/s with inputs already in HBM (device-timed, CUDA events);
         sub-batches alternate over --streams streams, each with its own
         workspace and output buffers
  e2e    the same through the public API from pinned host buffers: per
         sub-batch the query terms go host->device and every id list comes
         back device->host inside the timed region
  roofline / kernels
         per-kernel CUDA-event durations from the same steps run once more
         on a single stream (no overlap), against the bytes each kernel's
         design must move (dense bitmaps once per group-kernel launch, list
         blocks, bitmap writes and reads, 4 bytes per id)
  parity the untimed pass's ids of the first 256 queries against the CPU
         oracle run of the cpu_baseline leg (count + two checksums per query)
  reference_gpu
         the reference's own CUDA kernels on the same index and queries

Multi-GPU: replicas (each rank its own query set on its own copy of the
index, no collective on the data path), launched by torchrun; the time is
the max over ranks.

`--impl reference` times the reference's own CPU path (ComputeGroundTruth,
test/adsfilter_q_all.cu:196-208, built from the reference sources into
oracle/_ref) on the host cores, on a bounded sample of the same workload
(see run_reference).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "batched queries/s & postings GB/s vs HBM peak; learned vs fixed path planner"
# dram__bytes_read.sum + dram__bytes_write.sum of one launch divided by that
# launch's algorithmic bytes, from an ncu capture of the same kernel on the
# same workload at 1/4 scale (profiles/)
TRAFFIC_PER_ALGORITHMIC_BYTE: dict = {"compact": 1.000}
TRAFFIC_SOURCE: dict = {
    "compact": "ncu --set full of compact_kernel, config c1 at 1/4 scale, sub-batch 64: "
               "34.2 MB read + 752.3 MB written per launch = 1.000 x its algorithmic bytes "
               "(profiles/compact_kernel_c1x0.25.md)",
}
UNIT = "queries/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--config", default="c1")
    p.add_argument("--scale", type=float, default=1.0, help="shrink the workload (profiling / quick runs)")
    p.add_argument("--queries", type=int, default=0, help="override the query count")
    p.add_argument("--streams", type=int, default=2,
                   help="streams the sub-batches alternate over (each with its own workspace and buffers)")
    p.add_argument("--sub-batch", type=int, default=0,
                   help="queries per abf_batch_run call (0: tuned among 128/256/512, 256 without the tuner)")
    p.add_argument("--path", default="hybrid", choices=["auto", "probe", "union", "hybrid", "tile", "planner"])
    p.add_argument("--no-autotune", action="store_true", help="keep the library's default tuning")
    p.add_argument("--tuning", default="", help="apply a saved autotuner result (JSON) instead of tuning")
    p.add_argument("--tuning-set", default="",
                   help="explicit knobs instead of tuning, e.g. dense_div=256,tile_words=16384,group_min_queries=32")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (and with it the parity check)")
    p.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's CUDA kernels")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--out", default="", help="also append the JSON line to this file")
    p.add_argument("--mode", default="step", choices=["step", "planner", "serve", "index"],
                   help="step: the default benchmark; planner: configs c2/c3 (graph executor, learned planner); "
                        "serve: config c4 (Poisson arrivals through the serving loop); "
                        "index: parallel builder and binary index file vs the reference's BuildFrom")
    p.add_argument("--rates", default="20000,50000,100000,200000", help="serve mode: arrival rates (queries/s)")
    p.add_argument("--offered-seconds", type=float, default=0.5, help="serve mode: arrivals per rate, in seconds")
    p.add_argument("--planner-out", default="", help="planner mode: save the trained parameters (.npy)")
    p.add_argument("--train-queries", type=int, default=66_667)
    return p.parse_args()


# ---------------------------------------------------------------------------
def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def write_only_gbs(dev, gib: int = 4, reps: int = 5) -> float:
    """Write-only HBM rate of this GPU right now: best of `reps` fills of a
    `gib` GiB buffer, CUDA events. The compaction's traffic is almost all
    writes, so this is the ceiling it is also compared with."""
    import torch
    n = (gib << 30) // 4
    x = torch.empty(n, dtype=torch.int32, device=dev)
    x.fill_(1)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x.fill_(7)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del x
    torch.cuda.empty_cache()
    return 4.0 * n / (best / 1e3) / 1e9


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: the timed region begins once
            # it has produced its first sample, and only later ones count
            t_end = time.time() + 5.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.start = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        during = self.lines[getattr(self, "start", 0):] or self.lines[-1:]
        for ln in during:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def make_workload(cfg_name: str, scale: float, n_queries: int, rank: int):
    from adabool_b200 import workload as W
    cfg = W.CONFIGS[cfg_name]
    if scale != 1.0:
        cfg = W.scaled(cfg, scale)
    q = cfg.queries
    if n_queries:
        q.n_queries = n_queries
    q.seed = q.seed + 1000 * rank
    t0 = time.time()
    off, ads = W.gen_lists(cfg.lists)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(q, lens)
    return cfg, off, ads, lens, qoff, qterms, time.time() - t0


def split(qoff, qterms, sb):
    out = []
    nq = qoff.size - 1
    for a in range(0, nq, sb):
        b = min(nq, a + sb)
        o = (qoff[a:b + 1] - qoff[a]).astype(np.uint64)
        out.append((a, b, o, qterms[qoff[a]:qoff[b]].astype(np.uint32)))
    return out


def workload_config(cfg, n_postings: int, n_q: int) -> dict:
    """The `config` object of both arms' lines: the workload only (the
    execution settings of our arm go to its `execution` key)."""
    L, Q = cfg.lists, cfg.queries
    return {"workload": f"{cfg.name}: {L.n_terms} terms x {L.n_ads} ads, {n_postings} postings "
                        f"(Zipf {L.zipf_s:g} lengths clipped to [1, {L.max_len}], seed {L.seed}); {n_q} queries "
                        f"({Q.kind} term counts, median {Q.median:g}, sigma {Q.sigma:g}, [{Q.lo}, {Q.hi}], seed {Q.seed})",
            "output": "per query: bitmap over all ads + ascending uint32 ad ids",
            "l2": "inputs larger than L2 (no flush)"}


PARITY_QUERIES = 256  # queries whose ids get a checksum in the untimed pass


def id_checksums(ids, n: int, torch):
    """(sum of ids, sum of ids * position) mod 2^64 of an ascending id list on
    the device, the same checksums as the oracle's orc_cpu_batch_sums."""
    if n == 0:
        return 0, 0
    x = ids[:n].to(torch.int64) & 0xFFFFFFFF
    s1 = int(x.sum().item()) & 0xFFFFFFFFFFFFFFFF
    s2 = int((x * torch.arange(n, device=ids.device, dtype=torch.int64)).sum().item()) & 0xFFFFFFFFFFFFFFFF
    return s1, s2


def run_ours(args, rank, world, dev):
    import torch
    import adabool_b200 as ab
    from adabool_b200 import Index

    torch.cuda.set_device(dev)
    cfg, off, ads, lens, qoff, qterms, gen_s = make_workload(args.config, args.scale, args.queries, rank)
    L = cfg.lists
    t0 = time.time()
    ix = Index.from_csr(off, ads, L.n_terms, L.n_ads, device=dev)
    build_s = time.time() - t0
    n_q = qoff.size - 1
    n_words = (L.n_ads + 31) // 32
    stride = (n_words + 3) // 4 * 4
    path = {"auto": ab.PATH_AUTO, "probe": ab.PATH_PROBE, "union": ab.PATH_UNION, "hybrid": ab.PATH_HYBRID,
            "tile": ab.PATH_TILE, "planner": ab.PATH_AUTO}[args.path]
    tune_info = None
    if args.tuning_set:
        from adabool_b200 import autotune as AT
        kv = dict(x.split("=", 1) for x in args.tuning_set.split(",") if x)
        AT.apply(ix, {k: (float(v) if k == "probe_min_fraction" else int(v)) for k, v in kv.items()})
        tune_info = {"set": args.tuning_set}
    elif args.tuning:
        from adabool_b200 import autotune as AT
        AT.apply(ix, args.tuning)
        tune_info = {"from": args.tuning}
    elif not args.no_autotune:
        # untimed setup: the project's autotuner picks tile width, warps per
        # tile, the merge/scatter switch, dense-bitmap threshold, CTAs per SM
        from adabool_b200 import autotune as AT
        t0 = time.time()
        tr = AT.autotune(ix, qoff, qterms, path=path, sub_batch=args.sub_batch or 256, sample=1024, device=dev)
        tune_info = {"trials": len(tr.trials), "sample_ms": round(tr.best_ms, 3), "dense_div": tr.best.get("dense_div")}
        if not args.sub_batch:
            sbt = AT.tune_sub_batch(ix, qoff, qterms, path=path, candidates=(128, 256, 512), device=dev,
                                    n_streams=args.streams)
            args.sub_batch = sbt["best"]
            tune_info["sub_batch_ms"] = {str(k): round(v, 3) for k, v in sbt["ms"].items()}
        tune_info["seconds"] = round(time.time() - t0, 1)
    if not args.sub_batch:
        args.sub_batch = 256
    sbs = split(qoff, qterms, args.sub_batch)
    max_terms = max(int(s[3].size) for s in sbs) + 1
    # id capacity: the bound min(n_ads, sum of list lengths) per query
    qpost = np.add.reduceat(lens[qterms].astype(np.uint64), qoff[:-1].astype(np.int64)) if qterms.size else \
        np.zeros(n_q, np.uint64)
    qpost[np.diff(qoff) == 0] = 0
    bound = np.minimum(qpost, L.n_ads)
    cap = int(max(bound[a:b].sum() for a, b, _, _ in sbs)) + 1
    sbq = max(b - a for a, b, _, _ in sbs)

    # device-resident inputs per sub-batch
    d_in = [(torch.from_numpy(t.view(np.int32)).to(dev) if t.size else torch.zeros(1, dtype=torch.int32, device=dev),
             torch.from_numpy(o.view(np.int64)).to(dev), b - a) for a, b, o, t in sbs]
    n_streams = max(1, min(args.streams, len(sbs)))
    nbuf = max(n_streams, 1 if args.no_e2e else 2)
    ws = [ix.workspace(sbq, max_terms) for _ in range(nbuf)]
    bms = [torch.empty((sbq, stride), dtype=torch.int32, device=dev) for _ in range(nbuf)]
    ids = [torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(nbuf)]
    idoff = [torch.zeros(sbq + 1, dtype=torch.int64, device=dev) for _ in range(nbuf)]
    stream = torch.cuda.Stream(device=dev)
    streams = [stream] + [torch.cuda.Stream(device=dev) for _ in range(n_streams - 1)]
    fork = torch.cuda.Event()
    joins = [torch.cuda.Event() for _ in streams]

    def step():
        # sub-batch i runs on stream i % n with buffer set i % n, so one
        # sub-batch's compaction overlaps the next one's merge and scatter
        fork.record(stream)
        for s in streams[1:]:
            s.wait_event(fork)
        for i, (dt, do, nq) in enumerate(d_in):
            k = i % n_streams
            ix.batch_run(ws[k], dt, do, nq, bms[k], stride, path=path, d_ids=ids[k], d_id_offsets=idoff[k],
                         stream=streams[k])
        for s, e in zip(streams[1:], joins[1:]):
            e.record(s)
            stream.wait_event(e)

    # untimed pass: result sizes of every query and checksums of the first
    # PARITY_QUERIES queries' ids (compared with the oracle in cpu_baseline)
    n_par = min(PARITY_QUERIES, n_q)
    sums = np.zeros((n_par, 2), np.uint64)
    with torch.cuda.stream(stream):
        counts = np.zeros(n_q, np.uint64)
        for (a, b, _, _), (dt, do, nq) in zip(sbs, d_in):
            ix.batch_run(ws[0], dt, do, nq, bms[0], stride, path=path, d_ids=ids[0], d_id_offsets=idoff[0],
                         stream=stream)
            stream.synchronize()
            o = idoff[0][:nq + 1].cpu().numpy()
            counts[a:b] = np.diff(o)
            for i in range(a, min(b, n_par)):
                sums[i] = id_checksums(ids[0][int(o[i - a]):], int(o[i - a + 1] - o[i - a]), torch)
    ws[0].check(stream)

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    n_launch0 = ab.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    dist_barrier(world)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize(dev)
    launches = (ab.launch_count() - n_launch0) // max(args.steps, 1)
    ms_total = e0.elapsed_time(e1)
    ms_step = dist_max(ms_total / args.steps, world)
    dist_barrier(world)
    for w in ws:
        w.check(stream)

    # per-kernel CUDA-event times for the roofline: the same K steps once
    # more on one stream, so no kernel's duration includes another's
    # contention (in the timed region they overlap across streams)
    ix.profile(True)
    ix.profile_read()
    for _ in range(args.steps):
        for (dt, do, nq) in d_in:
            ix.batch_run(ws[0], dt, do, nq, bms[0], stride, path=path, d_ids=ids[0], d_id_offsets=idoff[0],
                         stream=stream)
    stream.synchronize()
    kern = ix.profile_read()
    ix.profile(False)

    # the same step without the id lists (bitmaps only, what the reference's
    # kernels produce), device-timed, for the reference-kernel comparison
    reps = max(1, args.steps // 2)
    with torch.cuda.stream(stream):
        def bm_step():
            for (dt, do, nq) in d_in:
                ix.batch_run(ws[0], dt, do, nq, bms[0], stride, path=path, stream=stream)
        bm_step()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(reps):
            bm_step()
        f1.record(stream)
        f1.synchronize()
    bitmaps_only_qps = n_q / (f0.elapsed_time(f1) / reps / 1e3)

    # ---- e2e through the public API from pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, ix, sbs, ws, bms, ids, idoff, stride, path, dev, world, n_q)

    # ---- physical bytes per kernel (roofline numerators) ----
    # every kernel is charged the bytes its design must move once: the dense
    # group kernel reads each dense bitmap once per launch and writes the
    # bitmaps of the queries it covers; the merge kernel reads the blocks of
    # the merged lists that have no dense bitmap (and, with the group kernel
    # on, reads back and rewrites the tiles of the queries that have such
    # lists); the scatter kernel reads the blocks of the scattered lists and
    # read-modify-writes one 4-byte word per posting; the compaction reads
    # each bitmap once and writes 4 bytes per id
    bm_bytes = L.n_ads / 8.0
    st = ix.stats()  # after tuning (the dense bitmaps follow dense_div)
    lbytes = ix.list_bytes().astype(np.float64)
    dense_t = (ix.list_flags() & 1) != 0
    hm = ix.tuning.heavy_min_len
    merged_t = {ab.PATH_HYBRID: dense_t | (lens >= hm), ab.PATH_TILE: np.ones_like(dense_t),
                ab.PATH_UNION: dense_t, ab.PATH_AUTO: dense_t,
                ab.PATH_PROBE: np.zeros_like(dense_t)}[path]
    seg = qoff[:-1].astype(np.int64)
    empty = np.diff(qoff) == 0

    def per_query(x):
        if not qterms.size:
            return np.zeros(n_q)
        return np.where(empty, 0.0, np.add.reduceat(x.astype(np.float64), seg))

    qt_m, qt_d = merged_t[qterms], dense_t[qterms]
    q_merge_nd = per_query(np.where(qt_m & ~qt_d, lbytes[qterms], 0.0))       # merged from blocks
    q_merge_nd_n = per_query((qt_m & ~qt_d).astype(np.float64))
    q_dense_n = per_query((qt_m & qt_d).astype(np.float64))                   # merged dense lists
    q_scat = per_query(np.where(~qt_m, lbytes[qterms], 0.0))
    q_scat_post = per_query(np.where(~qt_m, lens[qterms], 0).astype(np.float64))
    group_on = "dense_group" in kern
    alg = {"scatter_union": float(q_scat.sum() + 8.0 * q_scat_post.sum()),
           "compact": n_q * bm_bytes + 4.0 * float(counts.sum())}
    dense_only = (q_merge_nd_n == 0) & ~empty
    if group_on:
        g_launches = kern["dense_group"][0] / args.steps
        alg["dense_group"] = g_launches * float(st["dense_bytes"]) + float((~empty).sum()) * bm_bytes
        alg["tile_union"] = float(q_merge_nd[~dense_only & ~empty].sum()) + \
            2.0 * bm_bytes * float((~dense_only & ~empty).sum()) + bm_bytes * float(empty.sum())
    else:
        alg["tile_union"] = float(q_merge_nd.sum() + q_dense_n.sum() * bm_bytes) + n_q * bm_bytes
    hbm, peak_kind = peaks()
    cs = clk.summary()
    sm_mhz = (cs or {}).get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    smem_peak = n_sm * 128.0 * sm_mhz * 1e6 / 1e9  # GB/s: 128 bytes per clock per SM
    per_kernel = {}
    total_ms = sum(v[1] for v in kern.values())
    for name, (nl, tms) in kern.items():
        d = {"launches_per_step": nl / args.steps, "ms_per_step": tms / args.steps,
             "share": tms / max(total_ms, 1e-9)}
        if name in alg and tms > 0:
            d["bytes_per_step"] = alg[name]
            d["achieved_gbs"] = alg[name] * args.steps / (tms / 1e3) / 1e9
            d["frac_of_" + peak_kind] = d["achieved_gbs"] / hbm
        per_kernel[name] = d
    if group_on and kern["dense_group"][1] > 0:
        # its bound is the shared-memory pipe: one 256-byte row load per
        # (query, dense list, 64-word tile) named; a (query, tile) stops
        # reading rows once it is all ones, so the rows read are fewer
        pairs = float(q_dense_n.sum())
        g = per_kernel["dense_group"]
        g["bound"] = "shared memory"
        g["smem_gbs_rows_named"] = pairs * bm_bytes * args.steps / (kern["dense_group"][1] / 1e3) / 1e9
        g["smem_peak_gbs"] = round(smem_peak, 1)
        g["frac_of_smem_peak_rows_named"] = g["smem_gbs_rows_named"] / smem_peak
        g["smem_note"] = ("rows named by the queries' lists, an upper bound on the rows read: the merge of a "
                          "(query, tile) ends once it is all ones; ncu's shared-load wavefronts give the rows read")
        g["query_dense_pairs_per_step"] = pairs
    if "scatter_union" in per_kernel and kern["scatter_union"][1] > 0:
        sc = per_kernel["scatter_union"]
        sc["bound"] = "L2 atomics / issue"
        sc["postings_per_step"] = float(q_scat_post.sum())
        sc["postings_per_s"] = float(q_scat_post.sum()) * args.steps / (kern["scatter_union"][1] / 1e3)
        sc["bytes_note"] = ("blocks read plus a 4-byte read-modify-write per posting, an upper bound: ORs into "
                            "tiles the dense group kernel left all ones are skipped")
    dom = max(per_kernel, key=lambda k: per_kernel[k]["ms_per_step"]) if per_kernel else None
    roof = None
    if dom and "achieved_gbs" in per_kernel[dom]:
        a = per_kernel[dom]["achieved_gbs"]
        n_launch = max(kern[dom][0] / args.steps, 1.0)
        ratio = TRAFFIC_PER_ALGORITHMIC_BYTE.get(dom)
        # DRAM bytes per launch: measured ratio x this launch's algorithmic bytes
        traffic = round(ratio * alg[dom] / n_launch) if ratio is not None else None
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(a, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(a / hbm, 4), "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": round(alg[dom] / n_launch),
                "traffic_source": None if ratio is None else TRAFFIC_SOURCE.get(dom),
                "duration_source": "CUDA events around each launch in a single-stream pass of the same steps "
                                   "right after the timed region"}
        if dom == "compact":
            wgbs = write_only_gbs(dev)
            roof["write_only_gbs_live"] = round(wgbs, 1)
            roof["frac_of_write_only"] = round(a / wgbs, 4)
            roof["write_note"] = ("the compaction writes 4 bytes per id and reads 1 bit per ad (96 % writes on c1); "
                                  "write_only_gbs_live is a 4 GiB fill timed on this GPU after the profile pass")
    step_bytes = float(sum(alg.values()))
    postings = float(np.sum(qpost))
    value = n_q * world / (ms_step / 1e3)
    res = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Zipf lists, lognormal queries)",
        "config": workload_config(cfg, int(st["n_postings"]), n_q),
        "execution": {"path": args.path, "parallelism": f"replicas{world}",
                      "sub_batch": args.sub_batch, "streams": n_streams, "index_bytes": st["device_bytes"],
                      "tuning": dict(ix.tuning.as_dict(), dense_div=ix.dense_div), "autotune": tune_info},
        "postings_per_s": round(postings * world / (ms_step / 1e3), 1),
        "postings_raw_gbs": round(4 * postings * world / (ms_step / 1e3) / 1e9, 1),
        "algorithmic_gbs": round(step_bytes * world / (ms_step / 1e3) / 1e9, 1),
        "algorithmic_bytes_per_step": round(step_bytes),
        "bitmaps_only_qps": round(bitmaps_only_qps * world, 1),
        "roofline": roof, "kernels": per_kernel, "gpu_launches": int(launches),
        "result_ids_per_step": int(counts.sum()),
        "setup_s": {"generate": round(gen_s, 2), "build_upload": round(build_s, 2)},
    }
    if cs:
        res["clocks"] = cs
    if e2e:
        res["e2e"] = e2e
    return res, dict(off=off, ads=ads, qoff=qoff, qterms=qterms, counts=counts, sums=sums, ix=ix, cfg=cfg,
                     dev=dev)


def run_e2e(args, ix, sbs, ws, bms, ids, idoff, stride, path, dev, world, n_q):
    import torch
    streams = [torch.cuda.Stream(device=dev) for _ in range(2)]
    maxt = max(int(t.size) for _, _, _, t in sbs) + 1
    maxq = max(b - a for a, b, _, _ in sbs) + 1
    h_terms = [torch.from_numpy(t.view(np.int32) if t.size else np.zeros(1, np.int32)).pin_memory() for _, _, _, t in sbs]
    h_offs = [torch.from_numpy(o.view(np.int64)).pin_memory() for _, _, o, _ in sbs]
    d_terms = [torch.empty(maxt, dtype=torch.int32, device=dev) for _ in range(2)]
    d_offs = [torch.empty(maxq, dtype=torch.int64, device=dev) for _ in range(2)]
    h_idoff = [torch.empty(maxq, dtype=torch.int64).pin_memory() for _ in range(2)]
    h_ids = [torch.empty(ids[0].numel(), dtype=torch.int32).pin_memory() for _ in range(2)]
    ev_off = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    for e in done:
        e.record(streams[0])
    h2d = d2h = 0

    def one_step():
        nonlocal h2d, d2h
        h2d = d2h = 0
        for i, (a, b, o, t) in enumerate(sbs):
            k = i % 2
            s = streams[k]
            nq = b - a
            done[k].synchronize()  # pinned buffers of set k are free again
            with torch.cuda.stream(s):
                d_terms[k][:h_terms[i].numel()].copy_(h_terms[i], non_blocking=True)
                d_offs[k][:nq + 1].copy_(h_offs[i], non_blocking=True)
                ix.batch_run(ws[k], d_terms[k], d_offs[k], nq, bms[k], stride, path=path, d_ids=ids[k],
                             d_id_offsets=idoff[k], stream=s)
                h_idoff[k][:nq + 1].copy_(idoff[k][:nq + 1], non_blocking=True)
                ev_off[k].record(s)
            h2d += t.size * 4 + (nq + 1) * 8
            ev_off[k].synchronize()
            tot = int(h_idoff[k][nq])
            with torch.cuda.stream(s):
                if tot:
                    h_ids[k][:tot].copy_(ids[k][:tot], non_blocking=True)
                done[k].record(s)
            d2h += (nq + 1) * 8 + tot * 4
        for s in streams:
            s.synchronize()

    for _ in range(max(1, min(args.warmup, 2))):
        one_step()
    torch.cuda.synchronize(dev)
    dist_barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(streams[0])
    streams[1].wait_event(e0)
    for _ in range(args.steps):
        one_step()
    streams[0].wait_stream(streams[1])
    e1.record(streams[0])
    e1.synchronize()
    ms = dist_max(e0.elapsed_time(e1) / args.steps, world)
    return {"value": round(n_q * world / (ms / 1e3), 2), "unit": UNIT, "ms_per_step": round(ms, 3),
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "note": "query terms host->device and every sorted id list device->host, pinned buffers, 2 streams",
            "bound": f"PCIe: the device->host copy of the id lists, {d2h / (ms / 1e3) / 1e9:.1f} GB/s; kernel work "
                     "moves the device-timed value, not this one"}


def cpu_baseline(data: dict, seconds: float):
    """Oracle k-way merge (a port of the match-set semantics) on all host
    cores, on a bounded sample of the same queries. Its results are also the
    parity check of the untimed pass: per query the id count and two
    checksums of the ascending ids must equal ours."""
    from oracle import oracle as O
    off, ads, qoff, qterms = data["off"], data["ads"], data["qoff"], data["qterms"]
    n_threads = os.cpu_count() or 1
    lens = np.diff(off)
    # single-core rate on the first query with work
    i0 = int(np.argmax(np.diff(qoff) > 0))
    t0 = time.time()
    O.cpu_batch(off, ads, qoff[i0:i0 + 2] - qoff[i0], qterms[qoff[i0]:qoff[i0 + 1]], 1)
    one = max(time.time() - t0, 1e-6)
    post0 = float(lens[qterms[qoff[i0]:qoff[i0 + 1]]].sum())
    rate = post0 / one  # postings per second per core
    qpost = np.array([lens[qterms[qoff[i]:qoff[i + 1]]].sum() for i in range(qoff.size - 1)], np.float64)
    budget = rate * seconds * n_threads
    m = int(np.searchsorted(np.cumsum(qpost), budget)) + 1
    m = max(min(m, qoff.size - 1), min(n_threads, qoff.size - 1))
    t0 = time.time()
    counts, sums = O.cpu_batch(off, ads, qoff[:m + 1], qterms[:qoff[m]], n_threads, sums=True)
    dt = time.time() - t0
    # parity of our untimed pass against these oracle results
    k = min(m, data["sums"].shape[0])
    bad = [int(i) for i in range(k) if counts[i] != data["counts"][i] or
           not np.array_equal(sums[i], data["sums"][i])]
    parity = {"checked": k, "mismatches": len(bad), "first_mismatches": bad[:8],
              "against": "oracle heap k-way merge (orc_kway_union): per query the id count, the sum of the ids "
                         "and the sum of id x position (mod 2^64) of our ascending id list",
              "queries": f"the first {k} queries of the step"}
    return {"value": round(m / dt, 3), "unit": UNIT, "cores": n_threads, "kind": "port",
            "sample": f"first {m} queries of the same set ({qpost[:m].sum():.3g} postings), heap k-way merge "
                      f"to sorted ids, {n_threads} threads, {dt:.1f} s",
            "single_core_value": round(1.0 / one, 3), "single_core_sample": f"query {i0} ({post0:.3g} postings)"}, \
        parity


def reference_gpu(data: dict, sample: int = 32) -> dict:
    """The reference's own CUDA kernels (yxr620/AdaBool, compiled from its
    sources for sm_100a into oracle/_ref/libref_harness.so) on the same
    index and queries, beside ours. Its std::map builder cannot build 500M
    postings in reasonable time, so its arrays come from the oracle's
    restatement of that builder (pinned array for array against the real one
    by tests/test_oracle.py); the reference then derives its block metadata
    and runs its kernels unmodified. Per sampled query: Prepare(keys) +
    ListUnion_sparse (test/adsfilter_q_all.cu:427-438) and Prepare(len, bm) +
    ListUnion_dense (test/adsfilter_q_all.cu:414-425); one batch of 32
    through RunArraysImpl<32> (the path of BatchListUnion_dense) and the six
    RunSparseBatchListUnion launches of BatchListUnion_sparse
    (test/adsfilter_batch.cu:28-79). Kernels timed with CUDA events, the
    host Prepare with a host clock; every reference bitmap is compared with
    ours. Bitmaps only: the reference has no id-list kernel."""
    import ctypes as C
    import torch
    import adabool_b200 as ab
    from oracle import oracle as O
    H = O.ref_harness_lib()
    if H is None:
        return {"unavailable": "oracle/_ref/libref_harness.so was not built (needs the reference sources)"}
    off, ads, qoff, qterms, ix, cfg = (data[k] for k in ("off", "ads", "qoff", "qterms", "ix", "cfg"))
    L = cfg.lists
    t0 = time.time()
    mixed = O.Mixed.from_csr(off, ads)
    arrs = {f: [mixed.array(t, f) for t in range(O.NTYPES)] for f in ("key_seg", "headers", "keys", "arrays")}
    mixed.free()
    mixed_s = time.time() - t0

    def ptrs(lst, ct):
        return (ct * O.NTYPES)(*[x.ctypes.data_as(ct) if x.size else C.cast(None, ct) for x in lst])

    t0 = time.time()
    h = H.refq_gpu_load(ptrs(arrs["key_seg"], O.u32p), (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["key_seg"]]),
                        ptrs(arrs["headers"], O.u32p), (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["headers"]]),
                        ptrs(arrs["keys"], O.u32p), ptrs(arrs["arrays"], O.u8p),
                        (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["arrays"]]))
    load_s = time.time() - t0
    ref_bytes = int(sum(x.nbytes for v in arrs.values() for x in v))
    del arrs
    dev = data["dev"]
    n_words = (L.n_ads + 31) // 32
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    ours = torch.empty(n_words, dtype=torch.int32, device=dev)
    ref = torch.zeros(n_words + 64, dtype=torch.int32, device=dev)
    pm, km = C.c_float(), C.c_float()
    sparse, dense, ours_ms = [], [], []
    mismatches = 0
    n = min(sample, qoff.size - 1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch = {}
    try:
        for i in range(n):
            q = np.ascontiguousarray(qterms[qoff[i]:qoff[i + 1]], dtype=np.uint32)
            ix.query(q, ours, path=ab.PATH_HYBRID, stream=stream)  # warm
            e0.record(stream)
            ix.query(q, ours, path=ab.PATH_HYBRID, stream=stream)
            e1.record(stream)
            e1.synchronize()
            ours_ms.append(e0.elapsed_time(e1))
            want = ours.cpu().numpy()
            ref.zero_()
            rc = H.refq_gpu_sparse(h, q.ctypes.data_as(O.u32p), q.size, C.c_void_p(ref.data_ptr()), sp, C.byref(pm),
                                   C.byref(km))
            sparse.append((pm.value, km.value))
            mismatches += int(rc != 0 or not np.array_equal(ref[:n_words].cpu().numpy(), want))
            # padded so the reference's 16-byte bitmap reads stay inside the buffer
            qb = np.concatenate([O.term_bitmap_bytes(q, L.n_terms, pad_to=16), np.zeros(32, np.uint8)])
            ref.zero_()
            rc = H.refq_gpu_dense(h, qb.ctypes.data_as(O.u8p), qb.size, C.c_void_p(ref.data_ptr()), sp, C.byref(pm),
                                  C.byref(km))
            dense.append((pm.value, km.value))
            mismatches += int(rc != 0 or not np.array_equal(ref[:n_words].cpu().numpy(), want))
        B = min(32, qoff.size - 1)
        bqs = [np.ascontiguousarray(qterms[qoff[i]:qoff[i + 1]], dtype=np.uint32) for i in range(B)]
        qlen = ((L.n_terms + 7) // 8 + 15) // 16 * 16 + 32
        bm = np.zeros(B * qlen, np.uint8)
        for i, q in enumerate(bqs):
            b = O.term_bitmap_bytes(q, L.n_terms, pad_to=16)
            bm[i * qlen:i * qlen + b.size] = b
        res_len = (n_words + 3) // 4 * 4
        dres = torch.zeros(B * res_len, dtype=torch.int32, device=dev)
        got_d = None
        if B == 32:
            rc = H.refq_gpu_batch_dense32(h, bm.ctypes.data_as(O.u8p), qlen, C.c_void_p(dres.data_ptr()), res_len,
                                          sp, C.byref(pm), C.byref(km))
            batch["BatchListUnion_dense_b32"] = {"prep_ms": pm.value, "kernel_ms": km.value,
                                                 "kernel_qps": round(32e3 / km.value, 1), "rc": int(rc)}
            got_d = dres.cpu().numpy().reshape(B, res_len)
        keys = np.concatenate(bqs).astype(np.uint32)
        qidx = np.concatenate([np.full(q.size, i, np.uint32) for i, q in enumerate(bqs)])
        dres.zero_()
        rc = H.refq_gpu_batch_sparse(h, keys.ctypes.data_as(O.u32p), qidx.ctypes.data_as(O.u32p), keys.size,
                                     C.c_void_p(dres.data_ptr()), res_len * 4, sp, C.byref(pm), C.byref(km))
        batch[f"BatchListUnion_sparse_b{B}"] = {"prep_ms": pm.value, "kernel_ms": km.value,
                                                "kernel_qps": round(B * 1e3 / km.value, 1), "rc": int(rc)}
        got_s = dres.cpu().numpy().reshape(B, res_len)
        for i, q in enumerate(bqs):
            ix.query(q, ours, path=ab.PATH_HYBRID, stream=stream)
            want = ours.cpu().numpy()
            if got_d is not None:
                mismatches += int(not np.array_equal(got_d[i, :n_words], want))
            mismatches += int(not np.array_equal(got_s[i, :n_words], want))
    finally:
        H.refq_gpu_free(h)

    def stats(v):
        a = np.array(v)
        return {"prep_ms_mean": round(float(a[:, 0].mean()), 4), "kernel_ms_mean": round(float(a[:, 1].mean()), 4),
                "kernel_qps": round(float(1e3 / a[:, 1].mean()), 1),
                "with_prep_qps": round(float(1e3 / (a[:, 0] + a[:, 1]).mean()), 1)}

    return {"what": "reference CUDA kernels (built from its sources for sm_100a), bitmaps only, same index and "
                    "queries", "sample_queries": n,
            "ListUnion_sparse": stats(sparse), "ListUnion_dense": stats(dense), **batch,
            "ours_per_query_qps": round(float(1e3 / np.mean(ours_ms)), 1),
            "ours_per_query_note": "abf_query (HYBRID), one query per call, bitmap only, CUDA events",
            "bitmap_mismatches_vs_ours": mismatches, "reference_index_bytes": ref_bytes,
            "setup_s": {"mixed_build": round(mixed_s, 2), "reference_load": round(load_s, 2)}}


# ---------------------------------------------------------------------------
REF_COO_STRIDE = 16  # the reference arm scans every 16th COO pair and scales by 16


def run_reference(args):
    """The reference's CPU path on the host cores (bounded sample).

    The reference computes a query's match set on the CPU with
    ComputeGroundTruth (test/adsfilter_q_all.cu:196-208): one pass over every
    (term, ad) pair of the filter matrix with a std::set lookup of the term,
    inserting hits into a std::set of ads. It costs ~40 s per query at c1 on
    one core, so each step is a bounded sample: as many queries as host
    threads, one per thread, each scanning a 1/16 stride sample of the COO
    pairs (every 16th pair, so hits keep their proportion); the step time is
    scaled by 16 to a full scan. The workload comes from oracle/libwgen.so
    (the same generator source as the product library, built on its own), so
    this process loads no library of the product."""
    from oracle import oracle as O
    from adabool_b200 import workload as W
    W.use_generator_library(O.gen_lib(), "wgen_last_error_string")
    cfg, off, ads, lens, qoff, qterms, _ = make_workload(args.config, args.scale, args.queries, 0)
    n_q = qoff.size - 1
    n_threads = os.cpu_count() or 1
    H = O.ref_harness_lib()
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Zipf lists, lognormal queries)",
            "config": workload_config(cfg, int(off[-1]), n_q)}
    if H is not None:
        terms, ads_c = W.lists_to_coo(off, ads)
        ts = np.ascontiguousarray(terms[::REF_COO_STRIDE])
        as_ = np.ascontiguousarray(ads_c[::REF_COO_STRIDE])
        del terms, ads_c
        h = H.refq_cpu_load(O._p(ts, O.u32p), O._p(as_, O.u32p), ts.size)
        kind, scale = "reference", float(REF_COO_STRIDE)
        desc = (f"ComputeGroundTruth (the reference's CPU path: a std::set lookup per COO pair) over every "
                f"{REF_COO_STRIDE}th of the {int(off[-1])} COO pairs, time x{REF_COO_STRIDE}")

        def run(q0, m):
            counts = np.zeros(m, np.uint64)
            qo = np.ascontiguousarray(qoff[q0:q0 + m + 1] - qoff[q0])
            qt = np.ascontiguousarray(qterms[qoff[q0]:qoff[q0 + m]])
            H.refq_ground_truth_batch(h, O._p(qo, O.u64p), O._p(qt, O.u32p), m, n_threads, O._p(counts, O.u64p))
    else:
        kind, scale = "port", 1.0
        desc = "oracle heap k-way merge (the reference library was not built)"

        def run(q0, m):
            O.cpu_batch(off, ads, qoff[q0:q0 + m + 1] - qoff[q0], qterms[qoff[q0]:qoff[q0 + m]], n_threads)
    m = max(1, min(n_threads, n_q))
    nxt = 0
    times = []
    for k in range(args.warmup + args.steps):
        q0 = nxt if nxt + m <= n_q else 0
        nxt = q0 + m
        t0 = time.time()
        run(q0, m)
        if k >= args.warmup:
            times.append(time.time() - t0)
    sec = float(np.mean(times)) * scale  # per step of m queries over the full COO
    v = m / sec
    sample = (f"{desc}; each step {m} consecutive queries of the step's {n_q} (one per host thread), "
              f"{args.steps} steps")
    return dict(base, value=round(v, 4), ms_per_step=round(sec * 1e3, 1),
                cpu_baseline={"value": round(v, 4), "unit": UNIT, "cores": n_threads, "kind": kind, "sample": sample},
                e2e={"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


# ---------------------------------------------------------------------------
_PG = None


def dist_init(args):
    global _PG
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        _PG = dist
    return rank, world, local


def dist_barrier(world):
    if world > 1 and _PG is not None:
        _PG.barrier()


def dist_max(x: float, world: int) -> float:
    if world > 1 and _PG is not None:
        import torch
        dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        _PG.all_reduce(t, op=_PG.ReduceOp.MAX)
        return float(t.item())
    return x


def index_mode() -> dict:
    """Builder and binary file (ours, c0 / c1 at 1/16 / c1) beside the
    reference's own BuildFrom (src/AdaBool/inverted_list.h:348-374,
    compiled from its sources into oracle/_ref) on the same COO pairs, where
    its single-threaded std::map build finishes in seconds (c0, c1 at 1/16)."""
    from adabool_b200 import experiments as X
    from adabool_b200 import workload as W
    small = [W.CONFIGS["c0"], W.scaled(W.CONFIGS["c1"], 1 / 16)]
    r = {"metric": "index build / load seconds (host COO or CSR -> device-resident index)",
         "ours": X.index_experiment(configs=small + [W.CONFIGS["c1"]])}
    ref = {}
    try:
        from oracle import oracle as O
        if O.ref_build_lib() is None:
            raise RuntimeError("oracle/_ref/libref_build.so is not built")
        for cfg in small:
            name, L = cfg.name, cfg.lists
            off, ads = W.gen_lists(L)
            terms = np.repeat(np.arange(L.n_terms, dtype=np.uint32), np.diff(off).astype(np.int64))
            rec = {"nnz": int(ads.size), "threads": 1,
                   "note": "reference ivf_list::BuildFrom (host, std::map), no device upload"}
            t0 = time.perf_counter()
            m = O.Mixed.from_coo(terms, ads, source="reference")
            rec["build_from_sorted_s"] = time.perf_counter() - t0
            m.free()
            if ads.size <= 10_000_000:  # shuffled pairs: ~2.5 us per pair in its std::map
                perm = np.random.default_rng(7).permutation(terms.size)
                t0 = time.perf_counter()
                m = O.Mixed.from_coo(terms[perm], ads[perm], source="reference")
                rec["build_from_shuffled_s"] = time.perf_counter() - t0
                m.free()
            ref[name] = rec
    except Exception as e:  # the reference builder is an optional comparison
        ref["unavailable"] = str(e)
    r["reference_build_from"] = ref
    return r


def main():
    args = parse()
    if args.mode == "planner" and args.impl == "ours":
        from adabool_b200 import experiments as X
        from adabool_b200 import planner as P
        from adabool_b200 import workload as W

        def ref_tau(ix, qoff, qt, frac):
            # the fixed rule's threshold: crossover of the reference's own
            # kernels on the same index (oracle/ref_tau.py)
            from oracle import ref_tau as RT
            L = W.CONFIGS["c2"].lists
            off, ads = W.gen_lists(L)
            return RT.reference_tau(off, ads, L.n_terms, L.n_ads, qoff, qt, frac)

        r = X.planner_experiment(n_train=args.train_queries, fixed_tau=ref_tau, verbose=True)
        params = r.pop("params")
        if args.planner_out:
            P.save(params, args.planner_out, {k: r[k] for k in ("fixed_rule", "tuning", "train")})
        r["metric"] = METRIC
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")
        return 0
    if args.mode == "serve" and args.impl == "ours":
        from adabool_b200 import experiments as X
        rates = tuple(int(float(x)) for x in args.rates.split(","))
        r = X.serving_experiment(rates=rates, offered_seconds=args.offered_seconds,
                                 n_train=min(args.train_queries, 20_000), verbose=True)
        r.pop("params")
        r["metric"] = "serving throughput (queries/s) and p50/p99/p99.9 latency vs per-query fixed-rule path"
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")
        return 0
    if args.mode == "index" and args.impl == "ours":
        r = index_mode()
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")
        return 0
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        res = run_reference(args)
    else:
        rank, world, local = dist_init(args)
        res, data = run_ours(args, rank, world, local)
        if rank == 0 and not args.no_ref_gpu:
            res["reference_gpu"] = reference_gpu(data)
        if rank == 0 and not args.no_cpu:
            res["cpu_baseline"], res["parity"] = cpu_baseline(data, args.cpu_seconds)
        if _PG is not None:
            _PG.destroy_process_group()
        if rank != 0:
            return 0
    line = json.dumps(res)
    print(line, flush=True)
    if args.out:
        with open(args.out, "a") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
