"""GPU parity: the CUDA paths against the CPU oracle (bit-exact), through the C ABI.

Expected values come from the oracle's k-way merge (pinned against the
reference's ComputeGroundTruth by tests/test_oracle.py) and from the
reference-derived golden vectors; the reference's own GPU kernels, built
from its sources, are run on the same inputs where their library exists.
"""
import ctypes as C

import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, workload as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PATHS = [ab.PATH_PROBE, ab.PATH_UNION, ab.PATH_HYBRID, ab.PATH_TILE, ab.PATH_AUTO]


def _torch():
    import torch
    return torch


def expected(off, ads, q, n_words):
    ids = O.kway_union(off, ads, q)
    return ids, O.ids_to_bitmap(ids, n_words)


@pytest.fixture(scope="module")
def small(dev):
    spec = W.ListsSpec(n_terms=4096, n_ads=70_001, nnz=400_000, zipf_s=1.1, max_len=30_000, seed=5)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(W.QueriesSpec(48, "lognormal", 12.0, 1.5, 1, 600, seed=6), lens)
    qs = [qterms[qoff[i]:qoff[i + 1]] for i in range(qoff.size - 1)]
    heavy = int(np.argmax(lens))
    qs += [np.zeros(0, np.uint32),                              # empty query
           np.array([spec.n_terms + 3, 1 << 30], np.uint32),     # only out-of-range terms
           np.array([heavy, heavy, 7, 7, heavy], np.uint32),     # repeated terms
           np.array([heavy], np.uint32),                         # one long list
           np.arange(0, spec.n_terms, 3, dtype=np.uint32)]       # a third of all terms
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, device=0, keep_host=True)
    # same lists without dense bitmaps: every long list merged from its blocks
    # through the directory
    ix_nodense = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, device=0, dense_div=None)
    assert ix.stats()["n_dense_lists"] > 0 and ix_nodense.stats()["n_directory_lists"] > 0
    return dict(spec=spec, off=off, ads=ads, qs=qs, ix=ix, ix_nodense=ix_nodense, n_words=(spec.n_ads + 31) // 32)


def test_decode_roundtrip_host(small):
    ix, off, ads = small["ix"], small["off"], small["ads"]
    for t in range(0, small["spec"].n_terms, 37):
        assert np.array_equal(ix.decode_list(t), ads[off[t]:off[t + 1]])


@pytest.mark.parametrize("variant", ["ix", "ix_nodense"])
@pytest.mark.parametrize("path", PATHS)
def test_query_every_path(small, path, variant):
    torch = _torch()
    ix, n_words = small[variant], small["n_words"]
    n_ads = small["spec"].n_ads
    bm = torch.full((n_words,), -1, dtype=torch.int32, device="cuda")  # garbage: must be overwritten
    ids = torch.empty(n_ads + 1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for q in small["qs"]:
        ix.query(q, bm, path=path, d_ids=ids, d_count=cnt)
        torch.cuda.synchronize()
        e_ids, e_bm = expected(small["off"], small["ads"], q, n_words)
        got_bm = bm.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_bm, e_bm), f"bitmap mismatch, path {path}, |q|={q.size}"
        n = int(cnt.item())
        assert n == e_ids.size
        assert np.array_equal(ids[:n].cpu().numpy().view(np.uint32), e_ids)


def test_batch_mixed_paths_and_probe_overflow(small):
    torch = _torch()
    ix, n_words = small["ix"], small["n_words"]
    qs = small["qs"]
    t = ix.tuning
    old = t.probe_cap
    ix.set_tuning(probe_cap=3)  # more probe queries than slots: the rest fall back to list-union
    try:
        ws = ix.workspace(len(qs), sum(q.size for q in qs) + 1)
        qoff = np.zeros(len(qs) + 1, np.uint64)
        qoff[1:] = np.cumsum([q.size for q in qs])
        flat = np.concatenate(qs).astype(np.uint32)
        rng = np.random.default_rng(3)
        paths = rng.choice([1, 2, 3, 4, 0, 1, 1], size=len(qs)).astype(np.uint8)
        stride = ((n_words + 3) // 4) * 4 + 4
        d_terms = torch.from_numpy(flat.view(np.int32)).cuda()
        d_off = torch.from_numpy(qoff.view(np.int64)).cuda()
        d_paths = torch.from_numpy(paths).cuda()
        bms = torch.full((len(qs), stride), 0x55, dtype=torch.int32, device="cuda")
        cap = sum(expected(small["off"], small["ads"], q, n_words)[0].size for q in qs)
        d_ids = torch.empty(cap + 5, dtype=torch.int32, device="cuda")
        d_idoff = torch.zeros(len(qs) + 1, dtype=torch.int64, device="cuda")
        ix.batch_run(ws, d_terms, d_off, len(qs), bms, stride, d_paths=d_paths, d_ids=d_ids, d_id_offsets=d_idoff)
        ws.check()
        got = bms.cpu().numpy().view(np.uint32)
        idoff = d_idoff.cpu().numpy().view(np.uint64)
        allids = d_ids.cpu().numpy().view(np.uint32)
        assert idoff[-1] == cap
        for i, q in enumerate(qs):
            e_ids, e_bm = expected(small["off"], small["ads"], q, n_words)
            assert np.array_equal(got[i, :n_words], e_bm), f"query {i} path {paths[i]}"
            assert np.array_equal(allids[idoff[i]:idoff[i + 1]], e_ids)
    finally:
        ix.set_tuning(probe_cap=old)


@pytest.mark.parametrize("dense_div", [16, 128, 512, 1024, 4096])
@pytest.mark.parametrize("path", [ab.PATH_UNION, ab.PATH_HYBRID, ab.PATH_AUTO, "mixed"])
def test_dense_group_kernel(small, dense_div, path):
    """The dense group kernel (one pass per tile over every dense-only query,
    dense slices staged by TMA) against the oracle, on and off, with 1, 2 or
    3 TMA boxes of dense bitmaps (12 / 83 / 295 / 553 of them: 64-word tiles
    double-buffered, then single-buffered) or too many for it (1,914)."""
    torch = _torch()
    ix, n_words, qs = small["ix"], small["n_words"], small["qs"]
    old_dd, old_gm = ix.dense_div, ix.tuning.group_min_queries
    qoff = np.zeros(len(qs) + 1, np.uint64)
    qoff[1:] = np.cumsum([q.size for q in qs])
    flat = np.concatenate(qs).astype(np.uint32)
    d_terms = torch.from_numpy(flat.view(np.int32)).cuda()
    d_off = torch.from_numpy(qoff.view(np.int64)).cuda()
    d_paths = None
    if path == "mixed":
        paths = np.random.default_rng(11).choice([1, 2, 3, 4, 0], size=len(qs)).astype(np.uint8)
        d_paths = torch.from_numpy(paths).cuda()
    stride = ((n_words + 3) // 4) * 4
    expect = [expected(small["off"], small["ads"], q, n_words)[1] for q in qs]
    try:
        ix.set_dense_div(dense_div)
        n_dense = ix.stats()["n_dense_lists"]
        ws = ix.workspace(len(qs), int(qoff[-1]) + 1)
        for gm in (0, 1):
            ix.set_tuning(group_min_queries=gm)
            bms = torch.full((len(qs), stride), -1, dtype=torch.int32, device="cuda")
            ix.batch_run(ws, d_terms, d_off, len(qs), bms, stride, path=0 if path == "mixed" else path,
                         d_paths=d_paths)
            ws.check()
            got = bms.cpu().numpy().view(np.uint32)
            for i in range(len(qs)):
                assert np.array_equal(got[i, :n_words], expect[i]), \
                    f"query {i}, dense_div {dense_div} ({n_dense} dense), group {gm}, path {path}"
        ws.free()
    finally:
        ix.set_dense_div(old_dd)
        ix.set_tuning(group_min_queries=old_gm)


def test_dense_group_windows(small):
    """Batches above 2,048 queries run the dense group kernel window by
    window; every bitmap equals the merge kernel's and, on a sample, the
    oracle's."""
    torch = _torch()
    ix, n_words, spec = small["ix"], small["n_words"], small["spec"]
    lens = np.diff(small["off"]).astype(np.uint32)
    qoff, qt = W.gen_queries(W.QueriesSpec(2300, "lognormal", 6.0, 1.5, 1, 200, seed=19), lens)
    n = qoff.size - 1
    stride = ((n_words + 3) // 4) * 4
    d_terms = torch.from_numpy(qt.astype(np.uint32).view(np.int32)).cuda()
    d_off = torch.from_numpy(qoff.astype(np.uint64).view(np.int64)).cuda()
    ws = ix.workspace(n, int(qoff[-1]) + 1)
    old_gm = ix.tuning.group_min_queries
    out = []
    try:
        for gm in (0, 1):
            ix.set_tuning(group_min_queries=gm)
            bms = torch.full((n, stride), -1, dtype=torch.int32, device="cuda")
            ix.batch_run(ws, d_terms, d_off, n, bms, stride, path=ab.PATH_UNION)
            ws.check()
            out.append(bms[:, :n_words].cpu().numpy().view(np.uint32))
    finally:
        ix.set_tuning(group_min_queries=old_gm)
        ws.free()
    assert np.array_equal(out[0], out[1])
    for i in list(range(0, n, 97)) + [2047, 2048, n - 1]:
        q = qt[qoff[i]:qoff[i + 1]]
        assert np.array_equal(out[1][i], expected(small["off"], small["ads"], q, n_words)[1]), f"query {i}"


@pytest.mark.parametrize("tile_words", [256, 512, 1024, 4096, 16384])
@pytest.mark.parametrize("warps", [1, 2, 4, 8])
def test_tuning_sweep_identical(small, tile_words, warps):
    torch = _torch()
    ix, n_words = small["ix"], small["n_words"]
    t0 = ix.tuning
    saved = {f: getattr(t0, f) for f, _ in t0._fields_}
    try:
        # fixed_tile_shape: single queries would otherwise run on adapted
        # (narrower, 8-warp) tiles, and this sweep is about every shape
        ix.set_tuning(tile_words=tile_words, warps_per_tile=warps, heavy_min_len=64, scatter_blocks_per_warp=3,
                      probe_chunk_blocks=128, fixed_tile_shape=1)
        bm = torch.empty(n_words, dtype=torch.int32, device="cuda")
        for q in small["qs"][::5]:
            for path in (ab.PATH_TILE, ab.PATH_HYBRID, ab.PATH_PROBE):
                ix.query(q, bm, path=path)
                torch.cuda.synchronize()
                assert np.array_equal(bm.cpu().numpy().view(np.uint32), expected(small["off"], small["ads"], q,
                                                                                 n_words)[1])
    finally:
        ix.set_tuning(**saved)


@pytest.mark.parametrize("variant", ["ix", "ix_nodense"])
def test_dense_div_rebuild(small, variant):
    """Changing the dense-bitmap threshold at run time (host copy kept, or
    fetched back from the device) keeps every result bit-exact."""
    torch = _torch()
    ix, n_words = small[variant], small["n_words"]
    bm = torch.empty(n_words, dtype=torch.int32, device="cuda")
    try:
        for dd in (8, 256, None, 32):
            ix.set_dense_div(dd)
            st = ix.stats()
            assert (st["n_dense_lists"] == 0) == (dd is None)
            for q in small["qs"][::4]:
                for path in (ab.PATH_HYBRID, ab.PATH_UNION):
                    ix.query(q, bm, path=path)
                    torch.cuda.synchronize()
                    assert np.array_equal(bm.cpu().numpy().view(np.uint32),
                                          expected(small["off"], small["ads"], q, n_words)[1])
    finally:
        ix.set_dense_div(128 if variant == "ix" else None)


def test_graph_executor_replays_bit_exact(small):
    """One graph launch per batch: two different batches replayed through the
    same captured graph (padded with empty queries) match the oracle."""
    torch = _torch()
    from adabool_b200.executor import GraphBatchExecutor
    ix, n_words = small["ix"], small["n_words"]
    qs = small["qs"]
    max_t = sum(q.size for q in qs) + 8
    cap = sum(expected(small["off"], small["ads"], q, n_words)[0].size for q in qs) + 8
    ex = GraphBatchExecutor(ix, len(qs) + 3, max_t, path=ab.PATH_HYBRID, with_ids=True, ids_capacity=cap,
                            per_query_paths=True).capture()
    rng = np.random.default_rng(11)
    for order in (np.arange(len(qs)), rng.permutation(len(qs))[:len(qs) - 5]):
        batch = [qs[i] for i in order]
        qoff = np.zeros(len(batch) + 1, np.uint64)
        qoff[1:] = np.cumsum([q.size for q in batch])
        flat = np.concatenate(batch).astype(np.uint32)
        paths = rng.choice([1, 2, 3, 4], size=len(batch)).astype(np.uint8)
        ex.set_batch(qoff, flat, paths)
        ex.replay().synchronize()
        got = ex.bitmaps.cpu().numpy().view(np.uint32)
        idoff = ex.d_id_off.cpu().numpy()
        ids = ex.d_ids.cpu().numpy().view(np.uint32)
        for i, q in enumerate(batch):
            e_ids, e_bm = expected(small["off"], small["ads"], q, n_words)
            assert np.array_equal(got[i, :n_words], e_bm), (i, paths[i])
            assert np.array_equal(ids[idoff[i]:idoff[i + 1]], e_ids)
        for i in range(len(batch), ex.max_q):  # padding queries are empty
            assert not got[i, :n_words].any()


def test_reference_api_or_semantics(small):
    """Prepare + ListUnion_* OR into the caller's buffer like the reference."""
    torch = _torch()
    ix, n_words, n_terms = small["ix"], small["n_words"], small["spec"].n_terms
    rng = np.random.default_rng(9)
    for q in small["qs"][::3]:
        e = expected(small["off"], small["ads"], q, n_words)[1]
        pre = rng.integers(0, 1 << 32, n_words, dtype=np.uint64).astype(np.uint32) & \
            rng.integers(0, 1 << 32, n_words, dtype=np.uint64).astype(np.uint32)
        # sparse
        d = torch.from_numpy(pre.view(np.int32).copy()).cuda()
        w = ix.Prepare(q)
        assert ab.ListUnion_sparse(w, d) == 0
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), pre | e)
        # dense: term bitmap bytes as the reference driver builds them
        qb = O.term_bitmap_bytes(q, n_terms, pad_to=1)
        d = torch.zeros(n_words, dtype=torch.int32, device="cuda")
        wd = ix.Prepare(qb.size, qb)
        assert ab.ListUnion_dense(wd, d) == 0
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), e)


@pytest.mark.parametrize("batch", [1, 5, 33, 70])
def test_batch_dense_any_size(small, batch):
    torch = _torch()
    ix, n_words, n_terms = small["ix"], small["n_words"], small["spec"].n_terms
    qs = [small["qs"][i % len(small["qs"])] for i in range(batch)]
    qlen = ((n_terms + 7) // 8 + 15) // 16 * 16
    host = np.concatenate([O.term_bitmap_bytes(q, n_terms, pad_to=16) for q in qs])
    assert host.size == batch * qlen
    res_len = ((n_words + 3) // 4) * 4
    for device_side in (False, True):
        d = torch.zeros(batch * res_len, dtype=torch.int32, device="cuda")
        if device_side:
            dq = torch.from_numpy(host.copy()).cuda()
            w = ix.PrepareBatchDevice(batch, qlen, dq)
        else:
            w = ix.PrepareBatch(batch, qlen, host)
        ab.BatchListUnion_dense(w, None, d, res_len)
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.uint32).reshape(batch, res_len)
        for i, q in enumerate(qs):
            assert np.array_equal(got[i, :n_words], expected(small["off"], small["ads"], q, n_words)[1])


def test_batch_dense_unaligned_device_bitmaps(small):
    """Caller bitmaps whose stride is not a multiple of 16 bytes: read without staging."""
    torch = _torch()
    ix, n_words, n_terms = small["ix"], small["n_words"], small["spec"].n_terms
    qs = small["qs"][:7]
    qlen = ((n_terms + 7) // 8 + 3) // 4 * 4 + 4  # multiple of 4, not of 16
    host = np.zeros(len(qs) * qlen, np.uint8)
    for i, q in enumerate(qs):
        b = O.term_bitmap_bytes(q, n_terms, pad_to=1)
        host[i * qlen:i * qlen + b.size] = b
    dq = torch.from_numpy(host).cuda()
    w = ix.PrepareBatchDevice(len(qs), qlen, dq)
    d = torch.zeros(len(qs) * n_words, dtype=torch.int32, device="cuda")
    ab.BatchListUnion_dense(w, None, d, n_words)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.uint32).reshape(len(qs), n_words)
    for i, q in enumerate(qs):
        assert np.array_equal(got[i], expected(small["off"], small["ads"], q, n_words)[1])


def test_batch_sparse_with_qidx(small):
    torch = _torch()
    ix, n_words = small["ix"], small["n_words"]
    qs = small["qs"][:9]
    keys = np.concatenate(qs).astype(np.uint32)
    qidx = np.concatenate([np.full(q.size, i, np.uint32) for i, q in enumerate(qs)])
    res_bytes = ((n_words * 4 + 15) // 16) * 16
    w = ix.Prepare(keys)
    d = torch.zeros(len(qs) * res_bytes // 4, dtype=torch.int32, device="cuda")
    dq = torch.from_numpy(qidx.view(np.int32)).cuda()
    ab.BatchListUnion_sparse(w, d, dq, res_bytes)
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.uint32).reshape(len(qs), res_bytes // 4)
    for i, q in enumerate(qs):
        assert np.array_equal(got[i, :n_words], expected(small["off"], small["ads"], q, n_words)[1])


@pytest.mark.parametrize("n_bits", [1, 31, 32, 33, 1000, 65536 + 7, 3 * 65536 * 32 + 5])
@pytest.mark.parametrize("density", [0.0, 0.01, 0.3, 0.5, 0.9, 1.0])
def test_collect_ids(small, n_bits, density):
    torch = _torch()
    rng = np.random.default_rng(n_bits)
    n_words = (n_bits + 31) // 32
    bits = rng.random(n_words * 32) < density
    words = np.packbits(bits, bitorder="little").view(np.uint32).copy()
    e = O.collect_ids(words, n_bits)
    d_bm = torch.from_numpy(words.view(np.int32).copy()).cuda()
    cap = max(e.size, 1)
    d_ids = torch.empty(cap, dtype=torch.int32, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ab.CollectIdsFromBitmap(small["ix"], d_bm, n_bits, d_ids, d_cnt)
    torch.cuda.synchronize()
    assert int(d_cnt.item()) == e.size
    assert np.array_equal(d_ids[:e.size].cpu().numpy().view(np.uint32), e)
    if e.size > 10:  # capacity below the count: count stays exact, prefix written
        small_cap = torch.empty(e.size // 2, dtype=torch.int32, device="cuda")
        ab.CollectIdsFromBitmap(small["ix"], d_bm, n_bits, small_cap, d_cnt)
        torch.cuda.synchronize()
        assert int(d_cnt.item()) == e.size
        assert np.array_equal(small_cap.cpu().numpy().view(np.uint32), e[:e.size // 2])
        # an id array that is not 16-byte aligned takes the plain-store path
        odd = torch.empty(cap + 1, dtype=torch.int32, device="cuda")[1:]
        ab.CollectIdsFromBitmap(small["ix"], d_bm, n_bits, odd, d_cnt)
        torch.cuda.synchronize()
        assert int(d_cnt.item()) == e.size
        assert np.array_equal(odd[:e.size].cpu().numpy().view(np.uint32), e)


def test_edge_lists(dev):
    """Runs of consecutive ids (0-bit gaps), 31-bit gaps, lengths at block
    boundaries, empty and single-id lists, ids at both ends of the range."""
    torch = _torch()
    n_ads = 1 << 31
    lists = [np.arange(0, 5000, dtype=np.uint32),                 # run: bits = 0
             np.array([0, n_ads - 1], np.uint32),                 # 31-bit gap
             np.arange(7, 7 + 3 * 128 * 5, 5, dtype=np.uint32),   # 3 full blocks
             np.zeros(0, np.uint32),                              # empty
             np.array([n_ads - 1], np.uint32),                    # single, last id
             np.arange(1000, 1000 + 129 * 1000, 1000, dtype=np.uint32)]  # 129 = block + 1
    off = np.zeros(len(lists) + 1, np.uint64)
    off[1:] = np.cumsum([l.size for l in lists])
    ads = np.concatenate(lists).astype(np.uint32)
    ix = Index.from_csr(off, ads, len(lists), n_ads, device=0, keep_host=True)
    for t, l in enumerate(lists):
        assert np.array_equal(ix.decode_list(t), l)
    n_words = n_ads // 32
    bm = torch.empty(n_words, dtype=torch.int32, device="cuda")
    ids = torch.empty(20000, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for q in ([0, 1, 2, 3, 4, 5], [1], [3], [2, 5], [0, 0, 4]):
        q = np.array(q, np.uint32)
        e = O.kway_union(off, ads, q)
        for path in (ab.PATH_UNION, ab.PATH_TILE, ab.PATH_PROBE, ab.PATH_HYBRID):
            ix.query(q, bm, path=path, d_ids=ids, d_count=cnt)
            torch.cuda.synchronize()
            n = int(cnt.item())
            assert n == e.size
            assert np.array_equal(ids[:n].cpu().numpy().view(np.uint32), e)
    del bm


def test_golden_vectors(dev, golden):
    """Match sets of the reference-derived fixtures through every path."""
    torch = _torch()
    for name in golden["case_names"]:
        t, a = golden[f"{name}/terms"], golden[f"{name}/ads"]
        n_terms, n_ads = int(t.max()) + 1, int(a.max()) + 1
        ix = Index.from_coo(t, a, n_terms, n_ads, device=0)
        n_words = (n_ads + 31) // 32
        qoff, qterms = golden[f"{name}/q_off"], golden[f"{name}/q_terms"]
        toff, tids = golden[f"{name}/truth_off"], golden[f"{name}/truth_ids"]
        bm = torch.empty(n_words, dtype=torch.int32, device="cuda")
        ids = torch.empty(n_ads + 1, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        for i in range(qoff.size - 1):
            q = qterms[qoff[i]:qoff[i + 1]]
            e = tids[toff[i]:toff[i + 1]]
            for path in PATHS:
                ix.query(q, bm, path=path, d_ids=ids, d_count=cnt)
                torch.cuda.synchronize()
                n = int(cnt.item())
                assert n == e.size, (name, i, path)
                assert np.array_equal(ids[:n].cpu().numpy().view(np.uint32), e), (name, i, path)
        ix.free()


# ---------------------------------------------------------------------------
# the reference's own kernels on the same inputs
# ---------------------------------------------------------------------------
def _ref_gpu_index(H, mixed):
    arrs = {f: [mixed.array(t, f) for t in range(O.NTYPES)] for f in ("key_seg", "headers", "keys", "arrays")}
    keep = []

    def ptrs(lst, ct):
        arr_t = ct * O.NTYPES
        keep.extend(lst)
        return arr_t(*[x.ctypes.data_as(ct) if x.size else C.cast(None, ct) for x in lst])

    ks = ptrs(arrs["key_seg"], O.u32p)
    hd = ptrs(arrs["headers"], O.u32p)
    ky = ptrs(arrs["keys"], O.u32p)
    ar = ptrs(arrs["arrays"], O.u8p)
    ksl = (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["key_seg"]])
    nr = (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["headers"]])
    al = (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["arrays"]])
    return H.refq_gpu_load(ks, ksl, hd, nr, ky, ar, al)


def test_reference_kernels_agree(small):
    H = O.ref_harness_lib()
    if H is None:
        pytest.skip("reference kernel library not built")
    torch = _torch()
    off, ads, spec = small["off"], small["ads"], small["spec"]
    n_words = small["n_words"]
    mixed = O.Mixed.from_csr(off, ads)
    h = _ref_gpu_index(H, mixed)
    try:
        pm, km = C.c_float(), C.c_float()
        stream = torch.cuda.current_stream()
        sp = C.c_void_p(stream.cuda_stream)
        for q in small["qs"]:
            e = expected(off, ads, q, n_words)[1]
            # oracle restatement of what the reference kernels compute
            assert np.array_equal(mixed.union(q, n_words), e)
            d = torch.zeros(n_words + 64, dtype=torch.int32, device="cuda")
            qq = np.ascontiguousarray(q, np.uint32)
            rc = H.refq_gpu_sparse(h, qq.ctypes.data_as(O.u32p), qq.size, C.c_void_p(d.data_ptr()), sp,
                                   C.byref(pm), C.byref(km))
            assert rc == 0
            assert np.array_equal(d[:n_words].cpu().numpy().view(np.uint32), e)
            qb = O.term_bitmap_bytes(q, spec.n_terms, pad_to=16)
            qb = np.concatenate([qb, np.zeros(32, np.uint8)])
            d.zero_()
            rc = H.refq_gpu_dense(h, qb.ctypes.data_as(O.u8p), qb.size, C.c_void_p(d.data_ptr()), sp,
                                  C.byref(pm), C.byref(km))
            assert rc == 0
            assert np.array_equal(d[:n_words].cpu().numpy().view(np.uint32), e)
            assert np.array_equal(mixed.probe(qb, n_words), e)
    finally:
        H.refq_gpu_free(h)
        mixed.free()


def test_batch_collect_ids(small):
    """abf_batch_collect_ids over a batch of bitmaps (empty, full, random
    densities, a stride wider than the bitmap), packed ids against the
    definition; with a short capacity the offsets stay exact and the ids
    that fit are written."""
    torch = _torch()
    ix, n_words = small["ix"], small["n_words"]
    n_ads = small["spec"].n_ads
    rng = np.random.default_rng(21)
    stride = ((n_words + 3) // 4) * 4 + 8
    dens = [0.0, 1.0, 0.5, 0.02, 0.9, 0.0001, 0.3]
    host = np.zeros((len(dens), stride), np.uint32)
    for i, d in enumerate(dens):
        bits = rng.random(stride * 32) < d
        host[i] = np.packbits(bits, bitorder="little").view(np.uint32)
    exp = [O.collect_ids(host[i, :n_words].copy(), n_ads) for i in range(len(dens))]
    total = sum(e.size for e in exp)
    d_bm = torch.from_numpy(host.view(np.int32)).cuda()
    ws = ix.workspace(len(dens), 1)
    for cap in (total + 5, total // 2):
        ids = torch.full((cap + 32,), -7, dtype=torch.int32, device="cuda")
        idoff = torch.zeros(len(dens) + 1, dtype=torch.int64, device="cuda")
        ab.BatchCollectIds(ix, ws, d_bm, stride, len(dens), ids[:cap], idoff)
        ws.check()
        o = idoff.cpu().numpy()
        got = ids.cpu().numpy().view(np.uint32)
        assert o[0] == 0 and o[-1] == total
        flat = np.concatenate(exp)
        for i, e in enumerate(exp):
            assert o[i + 1] - o[i] == e.size, i
        k = min(cap, total)
        assert np.array_equal(got[:k], flat[:k])
        assert (ids[cap:] == -7).all()
