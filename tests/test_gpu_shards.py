"""Ad-range shards on one GPU: three shards of one index, each writing its
own word range of the full bitmaps, give the same bitmaps as the unsharded
index on every path (dense group kernel included), write nothing outside
their range, and their id lists, shifted and concatenated in shard order,
equal the unsharded ids."""
import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, planner as P, shards as S, workload as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPEC = W.ListsSpec(n_terms=16384, n_ads=300_000, nnz=3_000_000, zipf_s=1.1, max_len=120_000, seed=41)
SENTINEL = 0x5A5A5A5A


@pytest.fixture(scope="module")
def setup(dev):
    off, ads = W.gen_lists(SPEC)
    lens = np.diff(off).astype(np.uint32)
    qoff, qt = W.gen_queries(W.QueriesSpec(96, "lognormal", 30.0, 1.5, 1, 2000, seed=42), lens)
    full = Index.from_csr(off, ads, SPEC.n_terms, SPEC.n_ads, device=0)
    sh = S.AdRangeShards(off, ads, SPEC.n_terms, SPEC.n_ads, devices=[0, 0, 0])
    assert all(ix is not None for ix in sh.indexes)
    return dict(off=off, ads=ads, qoff=qoff, qt=qt, full=full, sh=sh)


def _bitmaps(n_q, stride, fill=0):
    import torch
    return torch.full((n_q, stride), fill, dtype=torch.int32, device="cuda")


@pytest.mark.parametrize("path", [ab.PATH_UNION, ab.PATH_HYBRID, ab.PATH_PROBE])
def test_shards_equal_unsharded_bitmaps(setup, path):
    import torch
    full, sh, qoff, qt = setup["full"], setup["sh"], setup["qoff"], setup["qt"]
    n_q, n_words = qoff.size - 1, (SPEC.n_ads + 31) // 32
    stride = (n_words + 3) // 4 * 4
    dt, do = P.device_batch(qoff, qt)
    ws = full.workspace(n_q, int(qoff[-1]))
    ref = _bitmaps(n_q, stride)
    full.batch_run(ws, dt, do, n_q, ref, stride, path=path)
    got = _bitmaps(n_q, stride, SENTINEL)
    sh.batch_run(sh.workspaces(n_q, int(qoff[-1])), dt, do, n_q, got, stride, path=path)
    torch.cuda.synchronize()
    assert torch.equal(got[:, :n_words], ref[:, :n_words])
    # oracle spot check on a few queries
    for i in range(0, n_q, 23):
        e = O.kway_union(setup["off"], setup["ads"], qt[qoff[i]:qoff[i + 1]])
        assert np.array_equal(got[i, :n_words].cpu().numpy().view(np.uint32), O.ids_to_bitmap(e, n_words))


def test_shard_writes_only_its_words(setup):
    import torch
    sh, qoff, qt = setup["sh"], setup["qoff"], setup["qt"]
    n_q, n_words = qoff.size - 1, (SPEC.n_ads + 31) // 32
    stride = (n_words + 3) // 4 * 4
    dt, do = P.device_batch(qoff, qt)
    lo, hi = sh.slices[1]
    ix = sh.indexes[1]
    got = _bitmaps(n_q, stride, SENTINEL)
    ix.batch_run(ix.workspace(n_q, int(qoff[-1])), dt, do, n_q, got[:, lo // 32:], stride, path=ab.PATH_UNION)
    torch.cuda.synchronize()
    g = got.cpu().numpy()
    w0, w1 = lo // 32, (hi + 31) // 32
    assert (g[:, :w0] == SENTINEL).all() and (g[:, w1:] == SENTINEL).all()


def test_shard_ids_concatenate(setup):
    import torch
    full, sh, qoff, qt = setup["full"], setup["sh"], setup["qoff"], setup["qt"]
    n_q = qoff.size - 1
    dt, do = P.device_batch(qoff, qt)

    def ids_of(ix, n_bits):
        w = (n_bits + 31) // 32
        stride = (w + 3) // 4 * 4
        bm = _bitmaps(n_q, stride)
        cap = n_q * n_bits
        d_ids = torch.empty(cap, dtype=torch.int32, device="cuda")
        d_off = torch.empty(n_q + 1, dtype=torch.int64, device="cuda")
        ix.batch_run(ix.workspace(n_q, int(qoff[-1])), dt, do, n_q, bm, stride, path=ab.PATH_UNION,
                     d_ids=d_ids, d_id_offsets=d_off)
        o = d_off.cpu().numpy()
        a = d_ids.cpu().numpy().view(np.uint32)
        return [a[o[i]:o[i + 1]] for i in range(n_q)]

    ref = ids_of(full, SPEC.n_ads)
    parts = [ids_of(ix, hi - lo) for ix, (lo, hi) in zip(sh.indexes, sh.slices)]
    for i in range(n_q):
        assert np.array_equal(S.merge_ids([p[i] for p in parts], sh.slices), ref[i])
