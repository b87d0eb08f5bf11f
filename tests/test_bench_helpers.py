"""Host logic of bench.py on the CPU: the sub-batch split covers every query
once and rebases offsets, and the device-side id checksums that the bench
compares with the oracle are the same numbers the oracle computes (so the
bench line's parity check compares like with like)."""
import importlib.util
from pathlib import Path

import numpy as np
import torch

from adabool_b200 import workload as W
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_split_covers_every_query_once():
    b = _bench()
    rng = np.random.default_rng(1)
    for n, sb in ((1, 4), (7, 3), (2048, 512), (1000, 256)):
        counts = rng.integers(0, 9, n)
        qoff = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
        qt = rng.integers(0, 1 << 20, int(qoff[-1])).astype(np.uint32)
        parts = b.split(qoff, qt, sb)
        assert [p[0] for p in parts] == list(range(0, n, sb))
        assert parts[-1][1] == n
        for a, e, o, t in parts:
            assert o[0] == 0 and o.size == e - a + 1
            assert np.array_equal(t, qt[qoff[a]:qoff[e]])
            assert np.array_equal(np.diff(o), counts[a:e])


def test_id_checksums_match_the_oracle():
    b = _bench()
    spec = W.ListsSpec(n_terms=512, n_ads=1 << 24, nnz=400_000, zipf_s=1.05, max_len=200_000, seed=9)
    off, ads = W.gen_lists(spec)
    qoff, qt = W.gen_queries(W.QueriesSpec(12, "uniform", lo=1, hi=40, seed=4), np.diff(off).astype(np.uint32))
    counts, sums = O.cpu_batch(off, ads, qoff, qt, 2, sums=True)
    for i in range(qoff.size - 1):
        ids = O.kway_union(off, ads, qt[qoff[i]:qoff[i + 1]])
        assert ids.size == counts[i]
        t = torch.from_numpy(ids.view(np.int32).copy())
        s1, s2 = b.id_checksums(t, ids.size, torch)
        assert (s1, s2) == (int(sums[i, 0]), int(sums[i, 1]))


def test_id_checksums_wrap_like_uint64():
    """Sums past 2^63 (long dense id lists) wrap modulo 2^64 on both sides."""
    b = _bench()
    n = 6_000_000
    ids = (np.arange(n, dtype=np.uint64) * 2 + (1 << 23)).astype(np.uint32)  # ascending, up to ~2^24
    pos = np.arange(n, dtype=np.uint64)
    e1 = int(np.sum(ids.astype(np.uint64), dtype=np.uint64))
    e2 = int(np.sum(ids.astype(np.uint64) * pos, dtype=np.uint64))  # wraps modulo 2^64
    prod = ids.astype(np.uint64) * pos  # each term below 2^48: no wrap per term
    exact = sum(int(c) for c in prod.reshape(-1, 1000).sum(axis=1, dtype=np.uint64))  # chunk sums below 2^58
    assert exact >= 1 << 64 and e2 == exact % (1 << 64)  # the sum does wrap
    s1, s2 = b.id_checksums(torch.from_numpy(ids.view(np.int32).copy()), n, torch)
    assert (s1, s2) == (e1, e2)
