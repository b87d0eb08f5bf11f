"""Seeded synthetic workloads (include/abf_workload.h) and the benchmark shapes.

The reference measures on the AdsFilter dataset, which is not distributed
with it; these shapes stand in for it:

  c0  65,536 terms x 1,048,576 ads, ~8M postings, Zipf(1.1) lengths clipped to
      [1, 200k]; 256 queries of 4-64 distinct terms (uniform count).
  c1  2^20 terms x 2^24 ads, ~500M postings, Zipf(1.05) clipped to [1, 5M];
      2,048 queries, lognormal term counts (median 40, sigma 1.5, [1, 5000]).
  c2  c1's index; 16,384 queries, lognormal (median 40, sigma 2, [1, 20000]).
  c4  c1's index; serving arrivals, lognormal (median 40, sigma 2).

Query terms are distinct and drawn with probability proportional to list
length. Everything is a pure function of the seed.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import lib, ptr

_GEN_FUNCS = ("abf_gen_target_lengths", "abf_gen_lists_offsets", "abf_gen_lists_fill", "abf_gen_queries_offsets",
              "abf_gen_queries_fill")
_gen = None       # library the generators run from (None: libadabool.so)
_gen_err = None   # its last-error function


def use_generator_library(L, last_error: str = "abf_last_error_string"):
    """Runs the generators from the ctypes library L instead of libadabool.so
    (L exports the abf_gen_* functions of include/abf_workload.h, e.g. a
    standalone build of the same generator source); None restores the
    default. The data are the same: the generator is a pure function of its
    parameters."""
    global _gen, _gen_err
    if L is None:
        _gen = _gen_err = None
        return
    for name in _GEN_FUNCS:
        fn = getattr(L, name)
        fn.argtypes = N.PROTOTYPES[name]
        fn.restype = C.c_int
    err = getattr(L, last_error)
    err.argtypes = []
    err.restype = C.c_char_p
    _gen, _gen_err = L, err


def _g():
    return _gen if _gen is not None else lib()


def check(status: int):
    if status != N.ABF_OK:
        msg = (_gen_err() if _gen_err is not None else lib().abf_last_error_string()).decode(errors="replace")
        raise N.AbfError(status, msg)
    return status


@dataclass
class ListsSpec:
    n_terms: int
    n_ads: int
    nnz: int
    zipf_s: float
    max_len: int
    seed: int = 1


@dataclass
class QueriesSpec:
    n_queries: int
    kind: str = "lognormal"   # or "uniform"
    median: float = 40.0
    sigma: float = 1.5
    lo: int = 1
    hi: int = 5000
    seed: int = 2


@dataclass
class Config:
    name: str
    lists: ListsSpec
    queries: QueriesSpec
    note: str = ""
    extra: dict = field(default_factory=dict)


CONFIGS = {
    "c0": Config("c0", ListsSpec(65536, 1 << 20, 8_000_000, 1.1, 200_000, seed=11),
                 QueriesSpec(256, "uniform", lo=4, hi=64, seed=12)),
    "c1": Config("c1", ListsSpec(1 << 20, 1 << 24, 500_000_000, 1.05, 5_000_000, seed=21),
                 QueriesSpec(2048, "lognormal", 40.0, 1.5, 1, 5000, seed=22)),
    "c2": Config("c2", ListsSpec(1 << 20, 1 << 24, 500_000_000, 1.05, 5_000_000, seed=21),
                 QueriesSpec(16384, "lognormal", 40.0, 2.0, 1, 20000, seed=32)),
    "c4": Config("c4", ListsSpec(1 << 20, 1 << 24, 500_000_000, 1.05, 5_000_000, seed=21),
                 QueriesSpec(4096, "lognormal", 40.0, 2.0, 1, 20000, seed=42)),
}


def scaled(cfg: Config, factor: float, n_queries: int | None = None) -> Config:
    """Same shape, fewer terms/ads/postings (for tests and small profiles)."""
    L = cfg.lists
    nl = ListsSpec(max(16, int(L.n_terms * factor)), max(1024, int(L.n_ads * factor)), max(1000, int(L.nnz * factor)),
                   L.zipf_s, max(8, int(L.max_len * factor)), L.seed)
    Q = cfg.queries
    nq = QueriesSpec(n_queries or Q.n_queries, Q.kind, Q.median, Q.sigma, Q.lo, min(Q.hi, nl.n_terms), Q.seed)
    return Config(cfg.name + f"x{factor:g}", nl, nq)


def _lp(s: ListsSpec, n_threads: int) -> N.GenListsParams:
    return N.GenListsParams(s.n_terms, s.n_ads, s.nnz, s.zipf_s, s.max_len, s.seed, n_threads)


def gen_lists(s: ListsSpec, n_threads: int = 0):
    """CSR (offsets uint64[n_terms+1], ads uint32[nnz]) of the synthetic filter matrix."""
    p = _lp(s, n_threads)
    off = np.empty(s.n_terms + 1, dtype=np.uint64)
    check(_g().abf_gen_lists_offsets(C.byref(p), ptr(off, N.u64p)))
    ads = np.empty(int(off[-1]), dtype=np.uint32)
    check(_g().abf_gen_lists_fill(C.byref(p), ptr(off, N.u64p), ptr(ads, N.u32p)))
    return off, ads


def target_lengths(s: ListsSpec) -> np.ndarray:
    p = _lp(s, 0)
    out = np.empty(s.n_terms, dtype=np.uint32)
    check(_g().abf_gen_target_lengths(C.byref(p), ptr(out, N.u32p)))
    return out


def gen_queries(q: QueriesSpec, list_len: np.ndarray, n_threads: int = 0):
    """(offsets uint64[n_queries+1], terms uint32[...]) of the query set."""
    kind = N.QCOUNT_UNIFORM if q.kind == "uniform" else N.QCOUNT_LOGNORMAL
    p = N.GenQueriesParams(q.n_queries, kind, q.median, q.sigma, q.lo, q.hi, q.seed, n_threads)
    ll = np.ascontiguousarray(list_len, dtype=np.uint32)
    off = np.empty(q.n_queries + 1, dtype=np.uint64)
    check(_g().abf_gen_queries_offsets(C.byref(p), ptr(ll, N.u32p), ll.size, ptr(off, N.u64p)))
    terms = np.empty(int(off[-1]), dtype=np.uint32)
    check(_g().abf_gen_queries_fill(C.byref(p), ptr(ll, N.u32p), ll.size, ptr(off, N.u64p), ptr(terms, N.u32p)))
    return off, terms


def lists_to_coo(off: np.ndarray, ads: np.ndarray):
    terms = np.repeat(np.arange(off.size - 1, dtype=np.uint32), np.diff(off).astype(np.int64))
    return terms, ads
