"""Ad-range shards on the host: the slices partition the ad space on aligned
boundaries, the per-shard CSR lists together equal the full lists, and two
gloo ranks, each answering every query from its own host shard index, gather
bitmaps and id lists equal to the single-process oracle."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from adabool_b200 import shards as S

SPEC = dict(n_terms=2000, n_ads=60000, nnz=150000, zipf_s=1.1, max_len=20000, seed=17)


def test_ad_slices_partition_aligned():
    for n_ads in (0, 1, 4096, 4097, 60000, 1 << 20):
        for world in (1, 2, 3, 8):
            sl = S.ad_slices(n_ads, world)
            assert len(sl) == world and sl[0][0] == 0 and sl[-1][1] == n_ads
            for (a, b), (c, d) in zip(sl, sl[1:]):
                assert b == c
            assert all(lo % S.SLICE_ALIGN == 0 or lo == n_ads for lo, _ in sl)


def test_shard_csr_reassembles_the_lists():
    from adabool_b200 import workload as W
    off, ads = W.gen_lists(W.ListsSpec(**SPEC))
    sl = S.ad_slices(SPEC["n_ads"], 3)
    parts = [S.shard_csr(off, ads, lo, hi) for lo, hi in sl]
    for t in range(0, SPEC["n_terms"], 97):
        got = S.merge_ids([a[o[t]:o[t + 1]] for o, a in parts], sl)
        assert np.array_equal(got, ads[off[t]:off[t + 1]])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        from pathlib import Path
        sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
        from adabool_b200 import Index, shards as S2, workload as W
        off, ads = W.gen_lists(W.ListsSpec(**SPEC))  # same seed on every rank
        sl = S2.ad_slices(SPEC["n_ads"], world)
        lo, hi = sl[rank]
        so, sa = S2.shard_csr(off, ads, lo, hi)
        ix = Index.from_csr(so, sa, SPEC["n_terms"], hi - lo, host_only=True)
        qoff, qt = W.gen_queries(W.QueriesSpec(23, "uniform", lo=1, hi=20, seed=3), np.diff(off).astype(np.uint32))
        w_local = (hi - lo + 31) // 32
        local = torch.zeros((qoff.size - 1, w_local), dtype=torch.int32)
        ids = []
        for i in range(qoff.size - 1):
            q = qt[qoff[i]:qoff[i + 1]]
            li = np.unique(np.concatenate([ix.decode_list(int(t)) for t in q])).astype(np.uint32) if q.size \
                else np.zeros(0, np.uint32)
            ids.append(li)
            words = np.zeros(w_local, np.uint32)
            np.bitwise_or.at(words, li >> 5, np.uint32(1) << (li & 31))
            local[i] = torch.from_numpy(words.view(np.int32))
        full = S2.gather_bitmap_slices(local, (SPEC["n_ads"] + 31) // 32, sl, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, ids)
        if rank == 0:
            merged = [S2.merge_ids([g[i] for g in gathered], sl) for i in range(qoff.size - 1)]
            np.save(os.path.join(out_dir, "bm.npy"), full.numpy().view(np.uint32))
            np.save(os.path.join(out_dir, "ids.npy"), np.concatenate(merged))
            np.save(os.path.join(out_dir, "cnt.npy"), np.array([m.size for m in merged]))
    finally:
        dist.destroy_process_group()


def test_two_rank_ad_shards_match_single_process(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    from adabool_b200 import workload as W
    from oracle import oracle as O
    off, ads = W.gen_lists(W.ListsSpec(**SPEC))
    qoff, qt = W.gen_queries(W.QueriesSpec(23, "uniform", lo=1, hi=20, seed=3), np.diff(off).astype(np.uint32))
    bm, ids, cnt = np.load(tmp_path / "bm.npy"), np.load(tmp_path / "ids.npy"), np.load(tmp_path / "cnt.npy")
    n_words = (SPEC["n_ads"] + 31) // 32
    pos = 0
    for i in range(qoff.size - 1):
        e = O.kway_union(off, ads, qt[qoff[i]:qoff[i + 1]])
        assert cnt[i] == e.size
        assert np.array_equal(ids[pos:pos + e.size], e)
        assert np.array_equal(bm[i], O.ids_to_bitmap(e, n_words))
        pos += e.size
