"""Serving loop (abf_server_*): every query's bitmap and ids are the same
whether it runs alone (abf_query) or inside whatever batch the server cut,
admission never lets the pool's reservations exceed the budget, and an
open-loop Poisson trace completes with the same id counts.

The reference has no serving layer; the expected results are the single-
query path, which tests/test_gpu_parity.py pins against the oracle, plus an
oracle spot check here.
"""
import time

import numpy as np
import pytest

from adabool_b200 import Index, workload as W
from adabool_b200 import _native as N
from adabool_b200.server import Server, device_view, poisson_arrivals, latency_summary
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(dev):
    spec = W.ListsSpec(n_terms=8192, n_ads=200_003, nnz=1_500_000, zipf_s=1.05, max_len=60_000, seed=71)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off).astype(np.uint32)
    qoff, qt = W.gen_queries(W.QueriesSpec(300, "lognormal", 12.0, 2.0, 1, 2000, seed=72), lens)
    qs = [qt[qoff[i]:qoff[i + 1]] for i in range(qoff.size - 1)]
    heavy = int(np.argmax(lens))
    qs[5] = np.zeros(0, np.uint32)                                # empty query
    qs[9] = np.array([spec.n_terms + 1, heavy, heavy], np.uint32)  # out-of-range and repeated terms
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, device=0)
    return dict(spec=spec, off=off, ads=ads, lens=lens, qs=qs, ix=ix)


def _alone(ix, q, n_words, n_ads):
    import torch
    bm = torch.empty(n_words, dtype=torch.int32, device="cuda")
    ids = torch.empty(n_ads + 1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ix.query(q, bm, path=N.PATH_HYBRID, d_ids=ids, d_count=cnt)
    torch.cuda.synchronize()
    n = int(cnt.item())
    return bm.cpu().numpy().view(np.uint32), ids[:n].cpu().numpy().view(np.uint32)


def _drain(srv, n, timeout_s=60.0):
    out = []
    t_end = time.time() + timeout_s
    while len(out) < n:
        assert time.time() < t_end, "server did not finish in time"
        out += srv.poll(256, timeout_us=20_000)
    return out


@pytest.mark.parametrize("path", [N.PATH_AUTO, N.PATH_UNION, N.PATH_HYBRID, N.PATH_PROBE])
def test_same_result_alone_and_in_the_mix(setup, path):
    import torch
    ix, qs, spec = setup["ix"], setup["qs"], setup["spec"]
    n_words = (spec.n_ads + 31) // 32
    alone = [_alone(ix, q, n_words, spec.n_ads) for q in qs]
    with Server(ix, budget_bytes=256 << 20, window_us=200, max_batch_queries=64, n_streams=2, path=path) as srv:
        for i, q in enumerate(qs):
            srv.submit(q, tag=i)
        res = _drain(srv, len(qs))
        sizes = []
        for r in res:
            assert r.status == 0
            e_bm, e_ids = alone[r.tag]
            bm = device_view(r.d_bitmap, n_words).cpu().numpy().view(np.uint32)
            assert np.array_equal(bm, e_bm), f"bitmap of query {r.tag} differs in a batch of {r.batch_queries}"
            assert r.n_ids == e_ids.size
            ids = device_view(r.d_ids, r.n_ids).cpu().numpy().view(np.uint32)
            assert np.array_equal(ids, e_ids)
            sizes.append(r.batch_queries)
            srv.release(r.ticket)
        st = srv.stats()
        assert st["completed"] == len(qs) and st["released"] == len(qs)
        assert st["reserved_bytes"] == 0
        assert max(sizes) > 1, "every query ran alone: nothing was batched"
        torch.cuda.synchronize()
    # oracle spot check of the single-query results the mix was compared with
    for i in range(0, len(qs), 37):
        e = O.kway_union(setup["off"], setup["ads"], qs[i])
        assert np.array_equal(alone[i][1], e)


def test_admission_respects_budget(setup):
    ix, qs, spec = setup["ix"], setup["qs"], setup["spec"]
    lens = setup["lens"]
    stride_bytes = (spec.n_ads + 127) // 128 * 16
    # room of one query: its bitmap plus 4 bytes per possible id, 256-byte aligned
    rooms = [stride_bytes + (min(int(lens[q[q < spec.n_terms]].sum()), spec.n_ads) * 4 + 255) // 256 * 256
             for q in qs]
    budget = 6 * max(rooms)
    with Server(ix, budget_bytes=budget, window_us=50, max_batch_queries=8, n_streams=2,
                path=N.PATH_HYBRID) as srv:
        for i, q in enumerate(qs):
            srv.submit(q, tag=i)
        got = []
        held = []
        t_end = time.time() + 60
        while len(got) < len(qs):
            assert time.time() < t_end
            st = srv.stats()
            assert st["reserved_bytes"] <= budget
            res = srv.poll(256, timeout_us=20_000)
            got += res
            held += res
            if len(held) > 12 or not res:  # hold some results back, then release them
                for r in held:
                    srv.release(r.ticket)
                held = []
        for r in held:
            srv.release(r.ticket)
        st = srv.stats()
        assert st["peak_reserved_bytes"] <= budget
        assert st["admission_waits"] > 0, "the budget never held a query back"
        assert all(r.status == 0 for r in got)
        assert sorted(r.tag for r in got) == list(range(len(qs)))


def test_submit_errors(setup):
    ix, spec = setup["ix"], setup["spec"]
    stride_bytes = (spec.n_ads + 127) // 128 * 16
    heavy = int(np.argmax(setup["lens"]))
    with Server(ix, budget_bytes=stride_bytes + 4096, max_batch_terms=16, path=N.PATH_HYBRID) as srv:
        with pytest.raises(N.AbfError) as e:
            srv.submit(np.arange(17, dtype=np.uint32))
        assert e.value.status == 8
        with pytest.raises(N.AbfError) as e:
            srv.submit(np.array([heavy], np.uint32))  # id room alone exceeds the pool
        assert e.value.status == 8
        t = srv.submit(np.zeros(0, np.uint32), tag=3)  # an empty query fits
        r = _drain(srv, 1)[0]
        assert r.ticket == t and r.status == 0 and r.n_ids == 0
        with pytest.raises(N.AbfError):
            srv.release(t + 100)
        srv.release(t)
        assert srv.stats()["rejected"] == 2


def test_bitmaps_only_and_ids_only(setup):
    ix, qs, spec = setup["ix"], setup["qs"], setup["spec"]
    n_words = (spec.n_ads + 31) // 32
    sub = qs[:40]
    alone = [_alone(ix, q, n_words, spec.n_ads) for q in sub]
    for bitmaps, ids in ((True, False), (False, True)):
        with Server(ix, budget_bytes=128 << 20, bitmaps=bitmaps, ids=ids, path=N.PATH_HYBRID) as srv:
            for i, q in enumerate(sub):
                srv.submit(q, tag=i)
            for r in _drain(srv, len(sub)):
                assert r.status == 0
                if bitmaps:
                    assert r.d_ids == 0
                    bm = device_view(r.d_bitmap, n_words).cpu().numpy().view(np.uint32)
                    assert np.array_equal(bm, alone[r.tag][0])
                else:
                    assert r.d_bitmap == 0
                    got = device_view(r.d_ids, r.n_ids).cpu().numpy().view(np.uint32)
                    assert np.array_equal(got, alone[r.tag][1])
                srv.release(r.ticket)


def test_poisson_trace(setup):
    ix, qs, spec = setup["ix"], setup["qs"], setup["spec"]
    n_words = (spec.n_ads + 31) // 32
    reps = 7
    qlist = qs * reps
    q_off = np.zeros(len(qlist) + 1, np.uint64)
    q_off[1:] = np.cumsum([q.size for q in qlist])
    q_terms = np.concatenate(qlist).astype(np.uint32)
    arr = poisson_arrivals(20_000, len(qlist), seed=5)
    with Server(ix, budget_bytes=512 << 20, window_us=200, path=N.PATH_AUTO) as srv:
        out = srv.run_trace(q_off, q_terms, arr, timeout_s=60)
        st = srv.stats()
    assert out["completed"] == len(qlist) and out["rejected"] == 0 and out["failed"] == 0
    expect = np.array([_alone(ix, q, n_words, spec.n_ads)[1].size for q in qs] * reps, np.uint64)
    assert np.array_equal(out["n_ids"], expect)
    lat = latency_summary(out["latency_ns"])
    assert 0 < lat["p50_us"] <= lat["p99_us"] <= lat["p999_us"]
    assert st["batches"] < len(qlist)
    assert st["reserved_bytes"] == 0
