"""The oracle against the reference-derived golden vectors (CPU only).

tests/golden/reference_vectors.npz holds outputs of the reference's own code
compiled from its sources (tests/golden/make_golden.py): BuildFrom's arrays,
ComputeGroundTruth's match sets and CollectIdsFromBitmap's id lists.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _csr(t, a):
    """Sorted unique per-term lists of COO pairs."""
    order = np.lexsort((a, t))
    t, a = t[order], a[order]
    keep = np.ones(t.size, bool)
    keep[1:] = (t[1:] != t[:-1]) | (a[1:] != a[:-1])
    t, a = t[keep], a[keep]
    n_terms = int(t.max()) + 1 if t.size else 1
    off = np.zeros(n_terms + 1, np.uint64)
    np.add.at(off, t.astype(np.int64) + 1, 1)
    return np.cumsum(off).astype(np.uint64), a.astype(np.uint32)


def test_kway_union_matches_reference_ground_truth(golden):
    for name in golden["case_names"]:
        t, a = golden[f"{name}/terms"], golden[f"{name}/ads"]
        off, ads = _csr(t, a)
        qoff, qterms = golden[f"{name}/q_off"], golden[f"{name}/q_terms"]
        toff, tids = golden[f"{name}/truth_off"], golden[f"{name}/truth_ids"]
        for i in range(qoff.size - 1):
            q = qterms[qoff[i]:qoff[i + 1]]
            e = tids[toff[i]:toff[i + 1]]
            assert np.array_equal(O.kway_union(off, ads, q), e), (name, i)
            assert np.array_equal(O.scan_union(t, a, q), e), (name, i)


def test_mixed_restatement_matches_reference_builder(golden):
    for name in golden["case_names"]:
        t, a = golden[f"{name}/terms"], golden[f"{name}/ads"]
        m = O.Mixed.from_coo(t, a, source="oracle")
        for ty in range(O.NTYPES):
            for f in O.FIELDS:
                assert np.array_equal(m.array(ty, f), golden[f"{name}/mixed/{ty}/{f}"]), (name, ty, f)
        m.free()


def test_mixed_decoders_match_ground_truth(golden):
    """Union and probe decoders of the mixed format give the match set
    (inputs without duplicate pairs)."""
    for name in golden["case_names"]:
        if name == "duplicates":
            continue
        t, a = golden[f"{name}/terms"], golden[f"{name}/ads"]
        n_words = (int(a.max()) + 32) // 32
        m = O.Mixed.from_coo(t, a)
        qoff, qterms = golden[f"{name}/q_off"], golden[f"{name}/q_terms"]
        toff, tids = golden[f"{name}/truth_off"], golden[f"{name}/truth_ids"]
        n_terms = int(t.max()) + 1
        for i in range(qoff.size - 1):
            q = qterms[qoff[i]:qoff[i + 1]]
            e = O.ids_to_bitmap(tids[toff[i]:toff[i + 1]], n_words)
            assert np.array_equal(m.union(q, n_words), e), (name, i)
            assert np.array_equal(m.probe(O.term_bitmap_bytes(q, n_terms), n_words), e), (name, i)
        m.free()


def test_duplicate_zero_byte_quirk():
    """The reference keeps duplicate pairs in its buckets and stops decoding an
    ARRAY record at the first zero byte past kMinNum
    (src/AdaBool/inverted_list.cu.h:84-93): bucket {0,0,0,3,5,7} of ARRAY8
    loses 3/5/7 only when the zero lands past kMinNum=5. Here low bytes
    {0 x 7, 9} (8 values, ARRAY8): payload = [0,0,0,0,0,0,9,0]; positions
    0..4 are unconditional, position 5 is 0 -> stop, so 9 is dropped."""
    t = np.full(8, 4, np.uint32)
    a = np.array([512] * 7 + [512 + 9], np.uint32)
    m = O.Mixed.from_coo(t, a)
    got = m.union(np.array([4], np.uint32), 32)
    assert O.collect_ids(got, 1024).tolist() == [512]
    ref = O.ref_build_lib()
    if ref is not None:
        r = O.Mixed.from_coo(t, a, source="reference")
        for f in O.FIELDS:
            assert np.array_equal(r.array(2, f), m.array(2, f))
    # the match-set oracle keeps 521: set semantics
    off = np.array([0, 0, 0, 0, 0, 2], np.uint64)
    assert O.kway_union(off, np.array([512, 521], np.uint32), [4]).tolist() == [512, 521]


@pytest.mark.parametrize("k", range(5))
def test_collect_ids_matches_reference(golden, k):
    bm = golden[f"collect/{k}/bitmap"]
    e = golden[f"collect/{k}/ids"]
    assert np.array_equal(O.collect_ids(bm, bm.size * 8), e)


def test_cpu_batch_counts():
    rng = np.random.default_rng(4)
    t = rng.integers(0, 200, 20000).astype(np.uint32)
    a = rng.integers(0, 50000, 20000).astype(np.uint32)
    off, ads = _csr(t, a)
    qs = [rng.choice(200, int(rng.integers(0, 30)), replace=False).astype(np.uint32) for _ in range(40)]
    qoff = np.zeros(len(qs) + 1, np.uint64)
    qoff[1:] = np.cumsum([q.size for q in qs])
    qt = np.concatenate(qs).astype(np.uint32)
    counts = O.cpu_batch(off, ads, qoff, qt, 3)
    for i, q in enumerate(qs):
        assert counts[i] == O.kway_union(off, ads, q).size


def test_reference_builder_if_present():
    """Where the reference sources exist, the restatement equals the real
    builder on a fresh random case too (beyond the committed fixtures)."""
    if O.ref_build_lib() is None:
        pytest.skip("reference builder not available here")
    rng = np.random.default_rng(77)
    t = rng.integers(0, 5000, 60000).astype(np.uint32)
    a = rng.integers(0, 1 << 22, 60000, dtype=np.uint32) & np.uint32(0xffffffcf)
    m1, m2 = O.Mixed.from_coo(t, a), O.Mixed.from_coo(t, a, source="reference")
    for ty in range(O.NTYPES):
        for f in O.FIELDS:
            assert np.array_equal(m1.array(ty, f), m2.array(ty, f)), (ty, f)


def test_standalone_generator_matches_library():
    """oracle/libwgen.so (the generator source built on its own, used by the
    reference's timing leg) yields the same workload as libadabool.so."""
    from adabool_b200 import workload as W
    spec = W.ListsSpec(n_terms=700, n_ads=90_001, nnz=60_000, zipf_s=1.1, max_len=9_000, seed=5)
    qs = W.QueriesSpec(50, "lognormal", 8.0, 1.5, 1, 100, seed=6)
    off_a, ads_a = W.gen_lists(spec)
    q_a = W.gen_queries(qs, np.diff(off_a).astype(np.uint32))
    W.use_generator_library(O.gen_lib(), "wgen_last_error_string")
    try:
        off_b, ads_b = W.gen_lists(spec)
        q_b = W.gen_queries(qs, np.diff(off_b).astype(np.uint32))
    finally:
        W.use_generator_library(None)
    assert np.array_equal(off_a, off_b) and np.array_equal(ads_a, ads_b)
    assert np.array_equal(q_a[0], q_b[0]) and np.array_equal(q_a[1], q_b[1])


def test_cpu_batch_checksums():
    from adabool_b200 import workload as W
    spec = W.ListsSpec(n_terms=300, n_ads=50_000, nnz=40_000, zipf_s=1.1, max_len=5_000, seed=9)
    off, ads = W.gen_lists(spec)
    qoff, qt = W.gen_queries(W.QueriesSpec(20, "lognormal", 6.0, 1.5, 1, 60, seed=3), np.diff(off).astype(np.uint32))
    counts, sums = O.cpu_batch(off, ads, qoff, qt, 3, sums=True)
    for i in range(qoff.size - 1):
        e = O.kway_union(off, ads, qt[qoff[i]:qoff[i + 1]]).astype(np.uint64)
        assert counts[i] == e.size
        assert sums[i, 0] == e.sum() and sums[i, 1] == (e * np.arange(e.size, dtype=np.uint64)).sum()
