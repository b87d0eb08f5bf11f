"""Autotuner for the batch kernels.

Times abf_batch_run (CUDA events on the launching stream) on a sample of
the caller's queries for candidate values of each knob -- merge tile width,
warps sharing a tile, the merge/scatter switch length (the dense/sparse
switch point of the hybrid path), CTAs per SM, blocks per scatter warp --
and keeps the fastest, one knob at a time (coordinate descent, a few
rounds). Results are bit-exact whatever the knobs; only time changes. The
outcome can be written to a JSON file and applied to a later index with
``apply``.

The reference fixes these at compile time (kKeyStep = 256, kThreadNum = 64,
test/adsfilter_q_all.cu:22-23) and has no tuner.
"""
from __future__ import annotations

import json
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _native as N

KNOBS = {
    "tile_words": [256, 512, 1024, 2048, 4096, 8192, 16384],
    "warps_per_tile": [1, 2, 4, 8],
    "ctas_per_sm": [2, 4, 6, 8],
    "scatter_blocks_per_warp": [1, 2, 4, 8],
    "dense_div": [16, 32, 64, 128, 256],  # lists with len * dense_div >= n_ads get dense bitmaps
    "group_min_queries": [0, 32],  # 0: no dense group kernel
}


def heavy_candidates(n_ads: int) -> list[int]:
    """Merge/scatter switch lengths: lists holding 1/4096 .. 1/16 of the ads."""
    return sorted({max(128, n_ads // d) for d in (4096, 1024, 512, 256, 128, 64, 32, 16)})


@dataclass
class TuneResult:
    best: dict
    best_ms: float
    trials: list = field(default_factory=list)

    def save(self, path):
        Path(path).write_text(json.dumps({"best": self.best, "best_ms": self.best_ms, "trials": self.trials},
                                         indent=1))


def apply(index, path_or_dict):
    d = path_or_dict if isinstance(path_or_dict, dict) else json.loads(Path(path_or_dict).read_text())["best"]
    if "dense_div" in d and d["dense_div"] != getattr(index, "dense_div", None):
        index.set_dense_div(d["dense_div"])
    index.set_tuning(**{k: v for k, v in d.items() if k in dict(N.Tuning._fields_)})


class _Runner:
    def __init__(self, index, q_off, q_terms, sub_batch, path, device, n_streams: int = 1):
        import torch
        self.torch = torch
        self.ix = index
        self.path = path
        n_q = q_off.size - 1
        self.stride = (index.n_words + 3) // 4 * 4
        self.sbs = []
        for a in range(0, n_q, sub_batch):
            b = min(n_q, a + sub_batch)
            o = (q_off[a:b + 1] - q_off[a]).astype(np.uint64)
            t = q_terms[q_off[a]:q_off[b]].astype(np.uint32)
            dt = torch.from_numpy(t.view(np.int32)).to(device) if t.size else torch.zeros(1, dtype=torch.int32,
                                                                                          device=device)
            self.sbs.append((dt, torch.from_numpy(o.view(np.int64)).to(device), b - a))
        mq = max(s[2] for s in self.sbs)
        mt = max(int(s[0].numel()) for s in self.sbs) + 1
        n = max(1, min(n_streams, len(self.sbs)))
        # sub-batch i runs on stream i % n with its own workspace and bitmaps
        self.wss = [index.workspace(mq, mt) for _ in range(n)]
        self.ws = self.wss[0]
        self.bms = [torch.empty((mq, self.stride), dtype=torch.int32, device=device) for _ in range(n)]
        self.streams = [torch.cuda.Stream(device=device) for _ in range(n)]
        self.stream = self.streams[0]

    def _pass(self):
        for i, (dt, do, nq) in enumerate(self.sbs):
            k = i % len(self.streams)
            self.ix.batch_run(self.wss[k], dt, do, nq, self.bms[k], self.stride, path=self.path,
                              stream=self.streams[k])

    def time_ms(self, reps: int) -> float:
        torch = self.torch
        self._pass()  # warm-up (tuning is read per launch: nothing to rebuild)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for s in self.streams[1:]:
            s.wait_event(e0)
        for _ in range(reps):
            self._pass()
        for s in self.streams[1:]:
            ev = torch.cuda.Event()
            ev.record(s)
            self.stream.wait_event(ev)
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def free(self):
        for w in self.wss:
            w.free()


# knobs that interact, searched jointly: which lists are dense decides which
# are merged, the tile width sets what a merge costs, and the group kernel
# changes what a dense list costs
GRID = ("dense_div", "heavy_min_len", "tile_words", "group_min_queries")


def autotune(index, q_off: np.ndarray, q_terms: np.ndarray, path: int = N.PATH_HYBRID, sub_batch: int = 256,
             sample: int = 1024, reps: int = 2, rounds: int = 2, knobs: dict | None = None, device: int = 0,
             grid: bool = True, verbose: bool = False) -> TuneResult:
    """Tuning on the first `sample` queries: a joint grid over the dense
    threshold, the merge/scatter switch and the tile width (which lists are
    dense decides which are merged, and the tile width sets what a merge
    costs), then coordinate descent over every knob from the grid's best.
    Leaves the best tuning set on the index and returns it with every trial."""
    n = min(sample, q_off.size - 1)
    run = _Runner(index, q_off[:n + 1], q_terms[:q_off[n]], sub_batch, path, device)
    space = dict(KNOBS if knobs is None else knobs)
    space.setdefault("heavy_min_len", heavy_candidates(index.n_ads))
    cur = index.tuning.as_dict()
    cur["dense_div"] = int(getattr(index, "dense_div", 32))
    tuning_knobs = [k for k in space if k != "dense_div"]

    def apply_cur():
        index.set_tuning(**{k: cur[k] for k in tuning_knobs})

    trials = []
    best_ms = run.time_ms(reps)
    trials.append({"tuning": dict(cur), "ms": best_ms})
    if grid and all(k in space for k in GRID):
        import itertools
        best_dd = cur["dense_div"]
        rest = GRID[1:]
        for dd in space["dense_div"]:
            index.set_dense_div(dd)
            for vals in itertools.product(*(space[k] for k in rest)):
                kv = dict(zip(rest, vals))
                cand = dict(cur, dense_div=dd, **kv)
                try:
                    index.set_tuning(**kv)
                except N.AbfError:
                    continue
                ms = run.time_ms(1)
                trials.append({"tuning": cand, "ms": ms})
                if ms < best_ms:
                    best_ms, cur, best_dd = ms, cand, dd
        if verbose:
            print(f"  grid best {best_ms:.3f} ms: {cur}", flush=True)
        index.set_dense_div(best_dd)
        apply_cur()
        best_ms = run.time_ms(reps)
    for _ in range(rounds):
        improved = False
        for knob, values in space.items():
            for v in values:
                if cur.get(knob) == v:
                    continue
                cand = dict(cur)
                cand[knob] = v
                try:
                    if knob == "dense_div":  # representation: rebuilds the dense bitmaps
                        index.set_dense_div(v)
                    else:
                        index.set_tuning(**{knob: v})
                except N.AbfError:
                    continue
                ms = run.time_ms(reps)
                trials.append({"tuning": cand, "ms": ms})
                if verbose:
                    print(f"  {knob}={v}: {ms:.3f} ms (best {best_ms:.3f})", flush=True)
                if ms < best_ms * 0.995:
                    best_ms, cur, improved = ms, cand, True
                if knob == "dense_div" and cur["dense_div"] != v:
                    index.set_dense_div(cur["dense_div"])
                apply_cur()
        if not improved:
            break
    apply_cur()
    if "dense_div" in space:
        index.dense_div = cur["dense_div"]
    run.free()
    return TuneResult(best=dict(cur), best_ms=best_ms, trials=trials)


def tune_sub_batch(index, q_off: np.ndarray, q_terms: np.ndarray, path: int = N.PATH_HYBRID,
                   candidates=(128, 256, 512, 1024), sample: int = 2048, reps: int = 2, device: int = 0,
                   n_streams: int = 1) -> dict:
    """Queries per abf_batch_run call: larger batches let co-resident merge
    tiles of different queries share L2, smaller ones keep the scatter's
    working set small and give the streams more calls to overlap. Times
    each candidate on the same sample, calls alternating over n_streams."""
    n = min(sample, q_off.size - 1)
    out = {}
    for sb in candidates:
        if sb > n:
            continue
        run = _Runner(index, q_off[:n + 1], q_terms[:q_off[n]], sb, path, device, n_streams)
        out[sb] = run.time_ms(reps)
        run.free()
        del run
    best = min(out, key=out.get)
    return {"best": best, "ms": out}
