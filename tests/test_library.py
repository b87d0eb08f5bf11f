"""libadabool on the host: exported symbols, the list format, the file format,
error behaviour and the workload generators (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, workload as W
from adabool_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s+(abf_[a-z_0-9]+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ab.lib()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert not (names - set(N.PROTOTYPES)), names - set(N.PROTOTYPES)
    assert lib.abf_abi_version() == 2


def rand_lists(rng, n_terms, n_ads, max_len):
    lists = []
    for t in range(n_terms):
        n = int(rng.integers(0, max_len))
        lists.append(np.unique(rng.integers(0, n_ads, n)).astype(np.uint32))
    off = np.zeros(n_terms + 1, np.uint64)
    off[1:] = np.cumsum([l.size for l in lists])
    return off, (np.concatenate(lists) if off[-1] else np.zeros(0, np.uint32)).astype(np.uint32)


@pytest.mark.parametrize("n_ads", [1, 33, 1000, 1 << 20, (1 << 31)])
def test_roundtrip_host_only(n_ads):
    rng = np.random.default_rng(n_ads % 1000)
    off, ads = rand_lists(rng, 300, n_ads, 600)
    ix = Index.from_csr(off, ads, 300, n_ads, host_only=True)
    st = ix.stats()
    assert st["n_postings"] == ads.size and st["on_device"] == 0
    for t in range(300):
        assert np.array_equal(ix.decode_list(t), ads[off[t]:off[t + 1]])
    assert np.array_equal(ix.list_lengths(), np.diff(off).astype(np.uint32))
    lb = ix.list_bytes()
    nblk = (np.diff(off) + 127) // 128
    assert np.all(lb >= 16 * nblk) and np.all(lb <= 16 * nblk + 16 * 32 * nblk)


def test_block_edge_lists():
    n_ads = 1 << 31
    lists = [np.arange(0, 1000, dtype=np.uint32),             # run of 1-gaps: 0-bit payload
             np.array([0, n_ads - 1], np.uint32),             # 31-bit gap
             np.arange(5, 5 + 128 * 3, dtype=np.uint32) * 7,  # exactly 3 blocks
             np.zeros(0, np.uint32),
             np.array([n_ads - 1], np.uint32),
             np.arange(0, 129 * 2, 2, dtype=np.uint32)]       # 129 ids: one full block + 1
    off = np.zeros(len(lists) + 1, np.uint64)
    off[1:] = np.cumsum([l.size for l in lists])
    ix = Index.from_csr(off, np.concatenate(lists).astype(np.uint32), len(lists), n_ads, host_only=True)
    for t, l in enumerate(lists):
        assert np.array_equal(ix.decode_list(t), l)
    st = ix.stats()
    assert st["n_blocks"] == 8 + 1 + 3 + 0 + 1 + 2


def test_dense_and_directory_tables():
    spec = W.ListsSpec(3000, 1 << 18, 600_000, 1.1, 60_000, seed=2)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off)
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, host_only=True)
    st = ix.stats()
    n_dense = int((lens * 128 >= spec.n_ads).sum())
    assert st["n_dense_lists"] == n_dense > 0
    assert st["dense_bytes"] == n_dense * ((spec.n_ads // 32 + 3) // 4 * 4) * 4
    assert st["n_directory_lists"] == int(((lens * 512 >= spec.n_ads) & (lens * 128 < spec.n_ads) & (lens > 128)).sum())
    none = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, host_only=True, dense_div=None)
    assert none.stats()["n_dense_lists"] == 0 and none.stats()["n_directory_lists"] > st["n_directory_lists"]


def test_coo_unsorted_duplicates_merged():
    rng = np.random.default_rng(5)
    t = rng.integers(0, 50, 5000).astype(np.uint32)
    a = rng.integers(0, 3000, 5000).astype(np.uint32)
    t = np.concatenate([t, t[:700]])
    a = np.concatenate([a, a[:700]])  # duplicate pairs
    ix = Index.from_coo(t, a, 50, 3000, host_only=True)
    for k in range(50):
        assert np.array_equal(ix.decode_list(k), np.unique(a[t == k]))
    # BuildFrom takes pairs and infers the domain like the reference drivers
    ix2 = Index.BuildFrom(np.stack([t, a], 1), host_only=True)
    assert ix2.n_terms == int(t.max()) + 1 and ix2.n_ads == int(a.max()) + 1


def test_range_errors():
    with pytest.raises(ab.AbfError) as e:
        Index.from_coo([0, 1], [5, 10], 2, 10, host_only=True)  # ad 10 >= n_ads
    assert e.value.status == 2
    with pytest.raises(ab.AbfError) as e:
        Index.from_coo([0, 2], [5, 6], 2, 10, host_only=True)  # term 2 >= n_terms
    assert e.value.status == 2
    with pytest.raises(ab.AbfError) as e:
        Index.from_csr([0, 1], [3], 1, (1 << 31) + 1, host_only=True)
    assert e.value.status == 2
    with pytest.raises(ab.AbfError) as e:
        Index.from_csr([0, 2, 1], [3, 4], 2, 10, host_only=True)  # offsets not monotone
    assert e.value.status == 1
    assert ab.lib().abf_last_error_string()


def test_device_calls_on_host_only_index_fail_cleanly():
    ix = Index.from_csr([0, 2], [1, 5], 1, 10, host_only=True)
    with pytest.raises(ab.AbfError) as e:
        ix.Prepare([0])
    assert e.value.status == 5
    with pytest.raises(ab.AbfError) as e:
        ix.workspace(4, 16)
    assert e.value.status == 5


def test_tuning_validation():
    ix = Index.from_csr([0, 2], [1, 5], 1, 10, host_only=True)
    t = ix.tuning
    assert t.tile_words in (256, 512, 1024, 2048, 4096, 8192, 16384) and t.heavy_min_len >= 128
    for bad in ({"tile_words": 300}, {"warps_per_tile": 3}, {"probe_chunk_blocks": 100}, {"ctas_per_sm": 0}):
        with pytest.raises(ab.AbfError):
            ix.set_tuning(**bad)
    ix.set_tuning(tile_words=512, warps_per_tile=2)
    assert ix.tuning.tile_words == 512 and ix.tuning.warps_per_tile == 2
    # the fields after probe_min_fraction survive a round trip through the C struct
    assert ix.tuning.group_min_queries == 32 and ix.tuning.fixed_tile_shape == 0
    ix.set_tuning(group_min_queries=0, fixed_tile_shape=1, probe_min_fraction=0.25)
    t = ix.tuning
    assert t.group_min_queries == 0 and t.fixed_tile_shape == 1 and abs(t.probe_min_fraction - 0.25) < 1e-7
    assert t.tile_words == 512 and t.warps_per_tile == 2


def test_save_load_roundtrip(tmp_path):
    rng = np.random.default_rng(8)
    off, ads = rand_lists(rng, 200, 100000, 900)
    ix = Index.from_csr(off, ads, 200, 100000, host_only=True)
    p = tmp_path / "idx.abf"
    ix.save(p)
    ix2 = Index.load(p, host_only=True)
    assert ix2.stats()["n_postings"] == ads.size
    for t in range(200):
        assert np.array_equal(ix2.decode_list(t), ads[off[t]:off[t + 1]])
    # truncated and corrupted files are refused
    raw = p.read_bytes()
    (tmp_path / "trunc.abf").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(ab.AbfError) as e:
        Index.load(tmp_path / "trunc.abf", host_only=True)
    assert e.value.status == 6
    bad = bytearray(raw)
    bad[0:8] = b"NOTANIDX"
    (tmp_path / "bad.abf").write_bytes(bytes(bad))
    with pytest.raises(ab.AbfError):
        Index.load(tmp_path / "bad.abf", host_only=True)


def test_generator_deterministic_across_threads():
    spec = W.ListsSpec(3000, 50000, 200000, 1.1, 20000, seed=9)
    p1 = N.GenListsParams(spec.n_terms, spec.n_ads, spec.nnz, spec.zipf_s, spec.max_len, spec.seed, 1)
    p4 = N.GenListsParams(spec.n_terms, spec.n_ads, spec.nnz, spec.zipf_s, spec.max_len, spec.seed, 4)
    o1 = np.empty(spec.n_terms + 1, np.uint64)
    o4 = np.empty(spec.n_terms + 1, np.uint64)
    N.check(ab.lib().abf_gen_lists_offsets(C.byref(p1), N.ptr(o1, N.u64p)))
    N.check(ab.lib().abf_gen_lists_offsets(C.byref(p4), N.ptr(o4, N.u64p)))
    assert np.array_equal(o1, o4)
    a1 = np.empty(int(o1[-1]), np.uint32)
    a4 = np.empty(int(o4[-1]), np.uint32)
    N.check(ab.lib().abf_gen_lists_fill(C.byref(p1), N.ptr(o1, N.u64p), N.ptr(a1, N.u32p)))
    N.check(ab.lib().abf_gen_lists_fill(C.byref(p4), N.ptr(o4, N.u64p), N.ptr(a4, N.u32p)))
    assert np.array_equal(a1, a4)
    lens = np.diff(o1)
    assert lens.min() >= 1 and abs(o1[-1] - spec.nnz) < 0.05 * spec.nnz
    for t in range(0, spec.n_terms, 50):  # sorted, unique, in range
        l = a1[o1[t]:o1[t + 1]]
        assert np.all(np.diff(l.astype(np.int64)) > 0) and (l.size == 0 or l[-1] < spec.n_ads)


def test_generated_lengths_follow_zipf():
    spec = W.ListsSpec(20000, 1 << 20, 2_000_000, 1.1, 100_000, seed=3)
    tl = W.target_lengths(spec)
    s = np.sort(tl)[::-1].astype(np.float64)
    assert s[0] <= spec.max_len and s[-1] >= 1
    # log-log slope of rank vs length over the unclipped middle ranks ~ -s
    r = np.arange(1, s.size + 1)
    sel = (s < spec.max_len * 0.9) & (s > 20)
    slope = np.polyfit(np.log(r[sel]), np.log(s[sel]), 1)[0]
    assert -1.25 < slope < -0.95
    assert abs(int(tl.sum()) - spec.nnz) < 0.01 * spec.nnz


@pytest.mark.parametrize("kind", ["uniform", "lognormal"])
def test_queries_distinct_and_bounded(kind):
    spec = W.ListsSpec(5000, 100000, 300000, 1.1, 20000, seed=4)
    lens = W.target_lengths(spec)
    q = W.QueriesSpec(300, kind, 40.0, 1.5, 4 if kind == "uniform" else 1, 64 if kind == "uniform" else 2000, seed=5)
    qoff, qt = W.gen_queries(q, lens)
    counts = np.diff(qoff)
    assert counts.min() >= q.lo and counts.max() <= q.hi
    for i in range(q.n_queries):
        t = qt[qoff[i]:qoff[i + 1]]
        assert np.unique(t).size == t.size and (t < spec.n_terms).all()
    # length-biased draws: hits per posting similar for long and short lists
    # (long lists are drawn less than proportionally: a term appears at most
    # once per query)
    hits = np.bincount(qt, minlength=spec.n_terms).astype(np.float64)
    order = np.argsort(lens)
    top, bottom = order[::-1][:50], order[:2500]
    if kind == "uniform":  # queries of <= 64 terms: far from saturating the long lists
        rate_top = hits[top].sum() / lens[top].sum()
        rate_bottom = hits[bottom].sum() / lens[bottom].sum()
        assert 0.2 < rate_top / rate_bottom < 1.5
    assert hits[top].mean() > 20 * max(hits[bottom].mean(), 1e-9)
    if kind == "lognormal":
        assert 25 <= np.median(counts) <= 60
