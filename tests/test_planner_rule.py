"""The fixed rule's host restatement (planner.fixed_rule_choice, used to
score the rule on measured labels) on a host-only index: the touched-block
fraction and the longest list of each query, with empty queries, repeated
terms and terms outside the index, against direct computations."""
import numpy as np

from adabool_b200 import Index, planner as P, workload as W


def test_fixed_rule_host_restatement():
    spec = W.ListsSpec(n_terms=3000, n_ads=200_000, nnz=600_000, zipf_s=1.1, max_len=60_000, seed=23)
    off, ads = W.gen_lists(spec)
    lens = np.diff(off).astype(np.int64)
    ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, host_only=True)
    assert np.array_equal(ix.list_lengths().astype(np.int64), lens)
    qs = [np.array([], np.uint32), np.array([5, 5, 5], np.uint32), np.array([spec.n_terms + 9], np.uint32),
          np.array([int(np.argmax(lens)), 1, 2], np.uint32), np.arange(0, spec.n_terms, 2, dtype=np.uint32)]
    q_off = np.concatenate([[0], np.cumsum([q.size for q in qs])]).astype(np.uint64)
    q_terms = np.concatenate(qs).astype(np.uint32)
    nblk = (lens + 127) // 128
    total = nblk.sum()
    frac = P.touched_fraction(ix, q_off, q_terms)
    mx = P.max_list_len(ix, q_off, q_terms)
    for i, q in enumerate(qs):
        v = q[q < spec.n_terms]
        assert np.isclose(frac[i], nblk[v].sum() / total)  # repeated terms count once per occurrence
        assert mx[i] == (lens[v].max() if v.size else 0)
    hyb = int(lens.max())  # only the query holding the longest list reaches it
    tau = float(frac[4]) - 1e-9  # only the query over half the terms passes tau
    choice = P.fixed_rule_choice(ix, q_off, q_terms, tau, hyb)
    assert choice.tolist() == [1, 1, 1, 2, 0]
    assert P.fixed_rule_choice(ix, q_off, q_terms, 1.0, 0).tolist() == [1] * 5  # no HYBRID switch, tau 1
