"""Bit-exact parity at the benchmark configurations, through the C ABI.

  c0  the whole configuration: 65,536 terms x 2^20 ads, 8M postings, all
      256 queries, every path, as one batch and query by query; bitmaps and
      ascending ids against the oracle's k-way merge (orc_kway_union, the
      reference's ComputeGroundTruth semantics, test/adsfilter_q_all.cu:196-208).
  c1  the full 2^20 x 2^24 index (500M postings) with the benchmark's dense
      representation; one launch of 512 of its queries writes more than 2^32
      ids, the regime where a 32-bit offset or count would wrap. Every query
      is checked through size-independent properties on the device (id count
      = bitmap popcount, ids strictly ascending, every id's bit set), a
      sample against the oracle (count + two checksums of the ids), three
      queries id for id.
  c2  16,384 queries on c1's index as one CUDA-graph launch through
      abf_batch_graph_*: every bitmap equals the same query run alone
      (abf_query, "bit-exact to config 1 run query by query"), a sample
      equals the oracle.
"""
import os

import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, workload as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PATHS = [ab.PATH_PROBE, ab.PATH_UNION, ab.PATH_HYBRID, ab.PATH_TILE, ab.PATH_AUTO]
THREADS = os.cpu_count() or 1


def _torch():
    import torch
    return torch


def _popcounts(rows, n_words):
    """Set bits per row of an int32 bitmap tensor (SWAR popcount on int64)."""
    torch = _torch()
    out = torch.zeros(rows.shape[0], dtype=torch.int64, device=rows.device)
    step = max(1, (1 << 27) // max(n_words, 1))
    for r0 in range(0, rows.shape[0], step):
        x = rows[r0:r0 + step, :n_words].to(torch.int64) & 0xFFFFFFFF
        x = x - ((x >> 1) & 0x55555555)
        x = (x & 0x33333333) + ((x >> 2) & 0x33333333)
        x = (x + (x >> 4)) & 0x0F0F0F0F
        x = ((x * 0x01010101) & 0xFFFFFFFF) >> 24
        out[r0:r0 + step] = x.sum(dim=1)
    return out


def _ids_match_bitmaps(bms, n_words, ids, idoff, n_ads):
    """Size-independent exactness of packed id lists against their bitmaps:
    count = popcount, strictly ascending, every id below n_ads with its bit
    set. Together these make the ids exactly the set bits."""
    torch = _torch()
    pc = _popcounts(bms, n_words)
    cnt = idoff[1:] - idoff[:-1]
    assert torch.equal(pc, cnt), "id counts differ from bitmap popcounts"
    o = idoff.cpu().numpy()
    for q in range(bms.shape[0]):
        a, b = int(o[q]), int(o[q + 1])
        if a == b:
            continue
        seg = ids[a:b].to(torch.int64) & 0xFFFFFFFF
        assert bool((seg[1:] > seg[:-1]).all()), f"query {q}: ids not strictly ascending"
        assert int(seg[-1]) < n_ads, f"query {q}: id past n_ads"
        words = bms[q, :n_words].to(torch.int64)[seg >> 5]
        assert bool(((words >> (seg & 31)) & 1).all()), f"query {q}: an id whose bit is clear"


def _checksums(ids, a, b):
    torch = _torch()
    n = b - a
    if n == 0:
        return 0, 0
    x = ids[a:b].to(torch.int64) & 0xFFFFFFFF
    s1 = int(x.sum().item()) & 0xFFFFFFFFFFFFFFFF
    s2 = int((x * torch.arange(n, device=ids.device, dtype=torch.int64)).sum().item()) & 0xFFFFFFFFFFFFFFFF
    return s1, s2


def _batch(ix, qoff, qterms, path, cap, torch):
    n_q = qoff.size - 1
    stride = (ix.n_words + 3) // 4 * 4
    ws = ix.workspace(n_q, int(qoff[-1]) + 1)
    bms = torch.full((n_q, stride), -1, dtype=torch.int32, device="cuda")  # garbage: must be overwritten
    ids = torch.empty(cap, dtype=torch.int32, device="cuda")
    idoff = torch.zeros(n_q + 1, dtype=torch.int64, device="cuda")
    d_terms = torch.from_numpy(np.ascontiguousarray(qterms, np.uint32).view(np.int32)).cuda()
    d_off = torch.from_numpy(np.ascontiguousarray(qoff, np.uint64).view(np.int64)).cuda()
    ix.batch_run(ws, d_terms, d_off, n_q, bms, stride, path=path, d_ids=ids, d_id_offsets=idoff)
    ws.check()
    return bms, ids, idoff


# ---------------------------------------------------------------------------
# c0: the whole configuration
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c0(dev):
    cfg = W.CONFIGS["c0"]
    off, ads = W.gen_lists(cfg.lists)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(cfg.queries, lens)
    assert qoff.size - 1 == 256 and ads.size > 7_000_000
    ix = Index.from_csr(off, ads, cfg.lists.n_terms, cfg.lists.n_ads, device=0)
    exp = [O.kway_union(off, ads, qterms[qoff[i]:qoff[i + 1]]) for i in range(qoff.size - 1)]
    return dict(cfg=cfg, off=off, ads=ads, qoff=qoff, qterms=qterms, ix=ix, exp=exp)


@pytest.mark.parametrize("path", PATHS)
def test_c0_every_query_as_one_batch(c0, path):
    torch = _torch()
    ix, qoff, qterms, exp = c0["ix"], c0["qoff"], c0["qterms"], c0["exp"]
    n_words = ix.n_words
    old = ix.tuning.probe_cap
    if path == ab.PATH_PROBE:
        ix.set_tuning(probe_cap=256)  # every query on the bitmap-probe (no list-union fallback)
    try:
        bms, ids, idoff = _batch(ix, qoff, qterms, path, sum(e.size for e in exp) + 1, torch)
    finally:
        ix.set_tuning(probe_cap=old)
    got_bm = bms.cpu().numpy().view(np.uint32)
    o = idoff.cpu().numpy()
    got = ids.cpu().numpy().view(np.uint32)
    for i, e in enumerate(exp):
        assert np.array_equal(got_bm[i, :n_words], O.ids_to_bitmap(e, n_words)), (path, i)
        assert np.array_equal(got[o[i]:o[i + 1]], e), (path, i)
    assert o[-1] == sum(e.size for e in exp)


@pytest.mark.parametrize("path", PATHS)
def test_c0_query_by_query(c0, path):
    torch = _torch()
    ix, qoff, qterms, exp = c0["ix"], c0["qoff"], c0["qterms"], c0["exp"]
    n_words = ix.n_words
    bm = torch.full((n_words,), -1, dtype=torch.int32, device="cuda")
    ids = torch.empty(max(e.size for e in exp) + 1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for i in range(0, qoff.size - 1, 3):
        ix.query(qterms[qoff[i]:qoff[i + 1]], bm, path=path, d_ids=ids, d_count=cnt)
        torch.cuda.synchronize()
        e = exp[i]
        assert np.array_equal(bm.cpu().numpy().view(np.uint32), O.ids_to_bitmap(e, n_words)), (path, i)
        n = int(cnt.item())
        assert n == e.size and np.array_equal(ids[:n].cpu().numpy().view(np.uint32), e), (path, i)


# ---------------------------------------------------------------------------
# c1 and c2: the full-scale index
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c1(dev):
    cfg = W.CONFIGS["c1"]
    off, ads = W.gen_lists(cfg.lists)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(cfg.queries, lens)
    ix = Index.from_csr(off, ads, cfg.lists.n_terms, cfg.lists.n_ads, device=0)
    ix.set_dense_div(256)  # the representation the benchmark's tuning settles on (638 dense bitmaps)
    yield dict(cfg=cfg, off=off, ads=ads, lens=lens, qoff=qoff, qterms=qterms, ix=ix)
    ix.free()
    _torch().cuda.empty_cache()


def test_c1_sub_batch_512_more_than_2_32_ids(c1):
    torch = _torch()
    ix, off, ads, lens = c1["ix"], c1["off"], c1["ads"], c1["lens"]
    n_ads = c1["cfg"].lists.n_ads
    nb = 512
    qoff = c1["qoff"][:nb + 1].copy()
    qterms = c1["qterms"][:qoff[-1]]
    qpost = np.array([int(lens[qterms[qoff[i]:qoff[i + 1]]].sum()) for i in range(nb)], np.int64)
    cap = int(np.minimum(qpost, n_ads).sum()) + 1
    bms, ids, idoff = _batch(ix, qoff, qterms, ab.PATH_HYBRID, cap, torch)
    o = idoff.cpu().numpy().astype(np.int64)
    assert o[-1] > (1 << 32), f"only {o[-1]} ids: the launch does not cross 2^32"
    _ids_match_bitmaps(bms, ix.n_words, ids, idoff, n_ads)
    # oracle sample: the longest queries, those packed past 2^32, a spread of others
    nt = np.diff(qoff)
    past = np.flatnonzero(o[:-1] >= (1 << 32))
    sample = sorted(set(np.argsort(-nt)[:12].tolist()) | set(past[:12].tolist()) |
                    set(range(0, nb, 43)) | {int(past[0]), nb - 1})
    sq = np.zeros(len(sample) + 1, np.uint64)
    sq[1:] = np.cumsum([nt[i] for i in sample])
    st = np.concatenate([qterms[qoff[i]:qoff[i + 1]] for i in sample]).astype(np.uint32)
    counts, sums = O.cpu_batch(off, ads, sq, st, THREADS, sums=True)
    for k, i in enumerate(sample):
        assert int(counts[k]) == o[i + 1] - o[i], f"query {i}: count"
        assert tuple(int(x) for x in sums[k]) == _checksums(ids, int(o[i]), int(o[i + 1])), f"query {i}: ids"
    # id for id: the longest query, the first one past 2^32, the last one
    for i in (int(np.argmax(nt)), int(past[0]), nb - 1):
        e = O.kway_union(off, ads, qterms[qoff[i]:qoff[i + 1]])
        assert np.array_equal(ids[int(o[i]):int(o[i + 1])].cpu().numpy().view(np.uint32), e), f"query {i}"
    del bms, ids
    torch.cuda.empty_cache()


def test_c2_graph_batch_equals_query_by_query(c1):
    torch = _torch()
    from adabool_b200.executor import GraphBatchExecutor
    ix, off, ads, lens = c1["ix"], c1["off"], c1["ads"], c1["lens"]
    cfg2 = W.CONFIGS["c2"]
    qoff, qterms = W.gen_queries(cfg2.queries, lens)
    n_q = qoff.size - 1
    assert n_q == 16384
    n_words = ix.n_words
    ex = GraphBatchExecutor(ix, n_q, int(qoff[-1]), path=ab.PATH_HYBRID).capture()
    assert ex.kernel_nodes >= 4
    ex.set_batch(qoff, qterms)
    ex.replay().synchronize()
    # every query alone through abf_query (its own plan, tile shape and
    # kernels), compared on the device
    one = torch.empty(n_words, dtype=torch.int32, device="cuda")
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    for i in range(n_q):
        ix.query(qterms[qoff[i]:qoff[i + 1]], one, path=ab.PATH_HYBRID, stream=stream)
        bad += (one != ex.bitmaps[i, :n_words]).any().to(torch.int64)
    assert int(bad.item()) == 0, f"{int(bad.item())} graph bitmaps differ from the same query run alone"
    # a sample against the oracle: the longest queries and a spread of others
    nt = np.diff(qoff)
    sample = sorted(set(np.argsort(-nt)[:4].tolist()) | set(range(0, n_q, 2047)))
    sq = np.zeros(len(sample) + 1, np.uint64)
    sq[1:] = np.cumsum([nt[i] for i in sample])
    st = np.concatenate([qterms[qoff[i]:qoff[i + 1]] for i in sample]).astype(np.uint32)
    counts, sums = O.cpu_batch(off, ads, sq, st, THREADS, sums=True)
    ids = torch.empty(ix.n_ads + 1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for k, i in enumerate(sample):
        ab.CollectIdsFromBitmap(ix, ex.bitmaps[i], ix.n_ads, ids, cnt)
        torch.cuda.synchronize()
        n = int(cnt.item())
        assert n == int(counts[k]), f"query {i}: count"
        assert _checksums(ids, 0, n) == tuple(int(x) for x in sums[k]), f"query {i}: ids"
    ex.free()
    del ex
    torch.cuda.empty_cache()
