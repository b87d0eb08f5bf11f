"""Bounded device waits: a wait that runs out returns an error status.

Nothing here faults, traps or hangs the GPU. The self-test launches one CTA
that waits on an mbarrier armed for a copy that is never issued and one that
looks back at a compaction status word that nothing publishes (a flag that
nothing sets); both use the path kernels' own wait code with a short poll
limit, give up and set the workspace's error flag. The host then reads
ABF_ERR_TIMEOUT from abf_workspace_check, and the same workspace keeps
answering queries bit-exactly.
"""
import time

import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index, workload as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ABF_ERR_TIMEOUT = 7


@pytest.fixture(scope="module")
def tiny(dev):
    spec = W.ListsSpec(n_terms=512, n_ads=200_003, nnz=150_000, zipf_s=1.1, max_len=20_000, seed=41)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(W.QueriesSpec(40, "lognormal", 8.0, 1.5, 1, 100, seed=42), lens)
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, device=0)
    return dict(spec=spec, off=off, ads=ads, qoff=qoff, qterms=qterms, ix=ix)


def _run_batch(t, ws, path):
    import torch
    ix, qoff, qterms = t["ix"], t["qoff"], t["qterms"]
    n_q = qoff.size - 1
    n_words = (t["spec"].n_ads + 31) // 32
    stride = (n_words + 3) // 4 * 4
    exp = [O.kway_union(t["off"], t["ads"], qterms[qoff[i]:qoff[i + 1]]) for i in range(n_q)]
    bms = torch.empty((n_q, stride), dtype=torch.int32, device="cuda")
    ids = torch.empty(sum(e.size for e in exp) + 1, dtype=torch.int32, device="cuda")
    idoff = torch.zeros(n_q + 1, dtype=torch.int64, device="cuda")
    ix.batch_run(ws, torch.from_numpy(qterms.view(np.int32)).cuda(), torch.from_numpy(qoff.view(np.int64)).cuda(),
                 n_q, bms, stride, path=path, d_ids=ids, d_id_offsets=idoff)
    ws.check()
    got_bm = bms.cpu().numpy().view(np.uint32)
    o = idoff.cpu().numpy()
    got = ids.cpu().numpy().view(np.uint32)
    for i in range(n_q):
        assert np.array_equal(got_bm[i, :n_words], O.ids_to_bitmap(exp[i], n_words)), (path, i)
        assert np.array_equal(got[o[i]:o[i + 1]], exp[i]), (path, i)


def test_waits_run_out_and_report_timeout(tiny):
    ix, qoff, qterms = tiny["ix"], tiny["qoff"], tiny["qterms"]
    ws = ix.workspace(qoff.size - 1, qterms.size + 1)
    ws.check()  # starts clean
    t0 = time.time()
    ws.selftest_waits(1 << 12)
    with pytest.raises(ab.AbfError) as e:
        ws.check()
    assert e.value.status == ABF_ERR_TIMEOUT
    assert "code 3" in str(e.value)  # both the mbarrier wait (2) and the look-back wait (1) gave up
    assert time.time() - t0 < 30.0
    ws.check()  # the check cleared the flag
    # the context and the workspace still work: every path bit-exact
    for path in (ab.PATH_PROBE, ab.PATH_UNION, ab.PATH_HYBRID):
        _run_batch(tiny, ws, path)


def test_wait_limit_is_a_runtime_setting(tiny):
    """A workspace with a shorter (still ample) limit answers as before; a
    zero limit is refused."""
    ix, qoff, qterms = tiny["ix"], tiny["qoff"], tiny["qterms"]
    ws = ix.workspace(qoff.size - 1, qterms.size + 1)
    ws.set_wait_limit(1 << 20)
    for path in (ab.PATH_PROBE, ab.PATH_UNION, ab.PATH_AUTO):
        _run_batch(tiny, ws, path)
    with pytest.raises(ab.AbfError):
        ws.set_wait_limit(0)
