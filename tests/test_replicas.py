"""Replica sharding on two gloo ranks (CPU only): every rank answers its
share of the queries from its own host copy of the index; the gathered
answers equal the single-process oracle, and the timing reduction is the max
over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from adabool_b200 import replicas as R


def test_shard_range_partitions():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            parts = [R.shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            for (a, b), (c, d) in zip(parts, parts[1:]):
                assert b == c
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


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
        root = Path(__file__).resolve().parents[1]
        sys.path.insert(0, str(root))
        from adabool_b200 import Index, workload as W
        spec = W.ListsSpec(2000, 60000, 150000, 1.1, 20000, seed=17)
        off, ads = W.gen_lists(spec)  # same seed on every rank: identical replicas
        ix = Index.from_csr(off, ads, spec.n_terms, spec.n_ads, host_only=True)
        qoff, qt = W.gen_queries(W.QueriesSpec(37, "uniform", lo=1, hi=20, seed=3), np.diff(off).astype(np.uint32))
        loff, lt, first = R.shard_queries(qoff, qt, rank, world)
        counts = []
        for i in range(loff.size - 1):
            q = lt[loff[i]:loff[i + 1]]
            ids = np.unique(np.concatenate([ix.decode_list(int(t)) for t in q])) if q.size else np.zeros(0)
            counts.append(ids.size)
        gathered = [None] * world
        dist.all_gather_object(gathered, (first, counts))
        t_max = R.max_over_ranks(float(rank + 1), dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "res.npy"), np.array([t_max] + [c for f, cs in sorted(gathered) for c in cs]))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_match_single_process(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = np.load(tmp_path / "res.npy")
    assert res[0] == 2.0  # max over ranks
    from adabool_b200 import workload as W
    from oracle import oracle as O
    spec = W.ListsSpec(2000, 60000, 150000, 1.1, 20000, seed=17)
    off, ads = W.gen_lists(spec)
    qoff, qt = W.gen_queries(W.QueriesSpec(37, "uniform", lo=1, hi=20, seed=3), np.diff(off).astype(np.uint32))
    expect = [O.kway_union(off, ads, qt[qoff[i]:qoff[i + 1]]).size for i in range(qoff.size - 1)]
    assert res[1:].astype(int).tolist() == expect
