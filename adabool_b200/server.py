"""Serving loop: Python face of ``abf_server_*`` (include/adabool.h).

The loop itself is native (csrc/abf_server.cpp): one server thread cuts
batches from a first-in first-out queue, admits them against a device pool
of ``budget_bytes`` (bitmap + worst-case id room per query), launches each
batch with ``abf_batch_run`` on one of ``n_streams`` streams, and hands back
device pointers to every query's bitmap and ascending ids, which stay in the
pool until released. ``run_trace`` replays an open-loop arrival schedule
from a native generator thread, so arrival rates of 10^5 queries/s are
reproduced without Python in the loop.

The reference has no serving layer (its drivers run one query or one batch
of at most 32 per host call: test/adsfilter_q_all.cu:412-440,
test/adsfilter_batch.cu:453-502).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class Result:
    ticket: int
    tag: int
    status: int
    path: int
    d_bitmap: int
    d_ids: int
    n_ids: int
    t_arrival_ns: int
    t_launch_ns: int
    t_done_ns: int
    batch_queries: int

    @property
    def latency_ns(self) -> int:
        return self.t_done_ns - self.t_arrival_ns


def clock_ns() -> int:
    return int(N.lib().abf_clock_ns())


def default_opts() -> N.ServerOpts:
    o = N.ServerOpts()
    N.check(N.lib().abf_server_default_opts(C.byref(o)))
    return o


class Server:
    def __init__(self, index, budget_bytes: int | None = None, window_us: int | None = None,
                 max_batch_queries: int | None = None, max_batch_terms: int | None = None,
                 n_streams: int | None = None, path: int | None = None, bitmaps: bool = True, ids: bool = True):
        o = default_opts()
        for name, v in (("budget_bytes", budget_bytes), ("window_us", window_us),
                        ("max_batch_queries", max_batch_queries), ("max_batch_terms", max_batch_terms),
                        ("n_streams", n_streams), ("path", path)):
            if v is not None:
                setattr(o, name, int(v))
        o.outputs = (N.SERVE_BITMAPS if bitmaps else 0) | (N.SERVE_IDS if ids else 0)
        self.opts = o
        self.index = index  # the index must outlive the server
        h = C.c_void_p()
        N.check(N.lib().abf_server_create(index.handle, C.byref(o), C.byref(h)))
        self.handle = h
        self._buf = (N.ServerResult * 256)()

    def submit(self, terms, tag: int = 0, arrival_ns: int = 0) -> int:
        t = np.ascontiguousarray(terms, dtype=np.uint32)
        ticket = C.c_uint64()
        N.check(N.lib().abf_server_submit(self.handle, N.ptr(t, N.u32p), t.size, int(tag), int(arrival_ns),
                                          C.byref(ticket)))
        return ticket.value

    def poll(self, max_results: int = 256, timeout_us: int = 0) -> list[Result]:
        if max_results > len(self._buf):
            self._buf = (N.ServerResult * max_results)()
        n = C.c_uint32()
        N.check(N.lib().abf_server_poll(self.handle, self._buf, max_results, int(timeout_us), C.byref(n)))
        out = []
        for i in range(n.value):
            r = self._buf[i]
            out.append(Result(r.ticket, r.tag, r.status, r.path, r.d_bitmap or 0, r.d_ids or 0, r.n_ids,
                              r.t_arrival_ns, r.t_launch_ns, r.t_done_ns, r.batch_queries))
        return out

    def release(self, ticket: int):
        N.check(N.lib().abf_server_release(self.handle, int(ticket)))

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(N.lib().abf_server_get_stats(self.handle, C.byref(s)))
        return s.as_dict()

    def run_trace(self, q_off: np.ndarray, q_terms: np.ndarray, arrival_ns: np.ndarray,
                  timeout_s: float = 120.0) -> dict:
        """Open-loop replay: query i arrives at start + arrival_ns[i]. Returns
        per-query latency and wait before launch (ns; UINT64_MAX for
        rejected or failed queries), id counts, paths and the run's totals."""
        n = q_off.size - 1
        off = np.ascontiguousarray(q_off, dtype=np.uint64)
        qt = np.ascontiguousarray(q_terms, dtype=np.uint32)
        arr = np.ascontiguousarray(arrival_ns, dtype=np.uint64)
        lat = np.zeros(n, np.uint64)
        qwait = np.zeros(n, np.uint64)
        nids = np.zeros(n, np.uint64)
        paths = np.zeros(n, np.uint8)
        ts = N.TraceStats()
        N.check(N.lib().abf_server_run_trace(self.handle, N.ptr(qt, N.u32p), N.ptr(off, N.u64p), n,
                                             N.ptr(arr, N.u64p), float(timeout_s), N.ptr(lat, N.u64p),
                                             N.ptr(qwait, N.u64p), N.ptr(nids, N.u64p), N.ptr(paths, N.u8p), C.byref(ts)))
        return {"latency_ns": lat, "queue_ns": qwait, "n_ids": nids, "paths": paths, "seconds": ts.seconds,
                "completed": ts.completed, "rejected": ts.rejected, "failed": ts.failed}

    def close(self):
        if getattr(self, "handle", None):
            N.check(N.lib().abf_server_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_view(addr: int, n: int, device: int = 0):
    """A torch int32 tensor over n words of device memory at addr (no copy);
    valid until the result that owns the memory is released."""
    import torch
    if n == 0:
        return torch.empty(0, dtype=torch.int32, device=torch.device("cuda", device))

    class _Arr:
        __cuda_array_interface__ = {"shape": (int(n),), "typestr": "<i4", "data": (int(addr), False),
                                    "version": 2, "strides": None}
    with torch.cuda.device(device):
        return torch.as_tensor(_Arr(), device=torch.device("cuda", device))


def poisson_arrivals(rate_qps: float, n: int, seed: int) -> np.ndarray:
    """Arrival times (ns from the start) of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e9 / rate_qps, size=n)
    return np.cumsum(gaps).astype(np.uint64)


def latency_summary(lat_ns: np.ndarray) -> dict:
    ok = lat_ns[lat_ns != np.iinfo(np.uint64).max].astype(np.float64) / 1e3
    if ok.size == 0:
        return {"p50_us": None, "p99_us": None, "p999_us": None, "mean_us": None, "max_us": None}
    return {"p50_us": float(np.percentile(ok, 50)), "p99_us": float(np.percentile(ok, 99)),
            "p999_us": float(np.percentile(ok, 99.9)), "mean_us": float(ok.mean()), "max_us": float(ok.max())}
