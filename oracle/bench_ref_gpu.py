"""Times the reference's own GPU path on the benchmark workload (measurement
infrastructure, not product).

The reference kernels are built from the reference sources into
oracle/_ref/libref_harness.so (oracle/build_oracle.py). Its index builder
(std::map, single-threaded) cannot build 500M postings in reasonable time, so
its arrays come from the oracle's restatement (orc_mixed_build_csr), which is
pinned array-for-array against the reference builder by tests/test_oracle.py;
the reference then computes its own block metadata and runs its kernels
unmodified. For each sampled query the script runs:

  * ListUnion_sparse after ivf_list::Prepare(keys)  (test/adsfilter_q_all.cu:427-438)
  * ListUnion_dense after ivf_list::Prepare(len, bm) (test/adsfilter_q_all.cu:414-425)
  * the batch paths for one batch of 32 queries: RunArraysImpl<32> and the
    six RunSparseBatchListUnion* launches (test/adsfilter_batch.cu:39-79)

timing the kernels with CUDA events and the host preparation with a host
clock, and checks every result bitmap against libadabool's on the same query.
Prints one JSON line.

    python oracle/bench_ref_gpu.py [--config c1] [--sample 32]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--config", default="c1")
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--sample", type=int, default=32)
    args = p.parse_args()
    import torch
    import adabool_b200 as ab
    from adabool_b200 import Index, workload as W
    from oracle import oracle as O

    H = O.ref_harness_lib()
    if H is None:
        print(json.dumps({"unavailable": "oracle/_ref/libref_harness.so not built"}))
        return 0
    cfg = W.CONFIGS[args.config]
    if args.scale != 1.0:
        cfg = W.scaled(cfg, args.scale)
    L = cfg.lists
    t0 = time.time()
    off, ads = W.gen_lists(L)
    lens = np.diff(off).astype(np.uint32)
    qoff, qterms = W.gen_queries(cfg.queries, lens)
    gen_s = time.time() - t0
    t0 = time.time()
    mixed = O.Mixed.from_csr(off, ads)
    mixed_s = time.time() - t0
    arrs = {f: [mixed.array(t, f) for t in range(O.NTYPES)] for f in ("key_seg", "headers", "keys", "arrays")}
    n_rec = [int(x.size) for x in arrs["headers"]]
    mixed.free()

    def ptrs(lst, ct):
        return (ct * O.NTYPES)(*[x.ctypes.data_as(ct) if x.size else C.cast(None, ct) for x in lst])

    t0 = time.time()
    h = H.refq_gpu_load(ptrs(arrs["key_seg"], O.u32p), (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["key_seg"]]),
                        ptrs(arrs["headers"], O.u32p), (C.c_uint64 * O.NTYPES)(*n_rec),
                        ptrs(arrs["keys"], O.u32p), ptrs(arrs["arrays"], O.u8p),
                        (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["arrays"]]))
    load_s = time.time() - t0
    del arrs

    ix = Index.from_csr(off, ads, L.n_terms, L.n_ads, device=0)
    n_words = (L.n_ads + 31) // 32
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    ours = torch.empty(n_words, dtype=torch.int32, device="cuda")
    ref = torch.zeros(n_words + 64, dtype=torch.int32, device="cuda")
    pm, km = C.c_float(), C.c_float()
    res = {"sparse": [], "dense": []}
    mismatches = 0
    n = min(args.sample, qoff.size - 1)
    for i in range(n):
        q = np.ascontiguousarray(qterms[qoff[i]:qoff[i + 1]], dtype=np.uint32)
        ix.query(q, ours, path=ab.PATH_HYBRID)
        torch.cuda.synchronize()
        want = ours.cpu().numpy()
        ref.zero_()
        rc = H.refq_gpu_sparse(h, q.ctypes.data_as(O.u32p), q.size, C.c_void_p(ref.data_ptr()), sp, C.byref(pm),
                               C.byref(km))
        res["sparse"].append((pm.value, km.value))
        mismatches += int(rc != 0 or not np.array_equal(ref[:n_words].cpu().numpy(), want))
        # padded so the reference's 16-byte bitmap reads stay inside the buffer
        qb = np.concatenate([O.term_bitmap_bytes(q, L.n_terms, pad_to=16), np.zeros(32, np.uint8)])
        ref.zero_()
        rc = H.refq_gpu_dense(h, qb.ctypes.data_as(O.u8p), qb.size, C.c_void_p(ref.data_ptr()), sp, C.byref(pm),
                              C.byref(km))
        res["dense"].append((pm.value, km.value))
        mismatches += int(rc != 0 or not np.array_equal(ref[:n_words].cpu().numpy(), want))
    # one batch of 32 queries through each batch path
    B = 32
    bqs = [np.ascontiguousarray(qterms[qoff[i]:qoff[i + 1]], dtype=np.uint32) for i in range(B)]
    qlen = ((L.n_terms + 7) // 8 + 15) // 16 * 16 + 32
    bm = np.zeros(B * qlen, np.uint8)
    for i, q in enumerate(bqs):
        b = O.term_bitmap_bytes(q, L.n_terms, pad_to=16)
        bm[i * qlen:i * qlen + b.size] = b
    res_len = (n_words + 3) // 4 * 4
    dres = torch.zeros(B * res_len, dtype=torch.int32, device="cuda")
    rc = H.refq_gpu_batch_dense32(h, bm.ctypes.data_as(O.u8p), qlen, C.c_void_p(dres.data_ptr()), res_len, sp,
                                  C.byref(pm), C.byref(km))
    bd = (pm.value, km.value, int(rc))
    got_d = dres.cpu().numpy().reshape(B, res_len)
    keys = np.concatenate(bqs).astype(np.uint32)
    qidx = np.concatenate([np.full(q.size, i, np.uint32) for i, q in enumerate(bqs)])
    dres.zero_()
    rc = H.refq_gpu_batch_sparse(h, keys.ctypes.data_as(O.u32p), qidx.ctypes.data_as(O.u32p), keys.size,
                                 C.c_void_p(dres.data_ptr()), res_len * 4, sp, C.byref(pm), C.byref(km))
    bs = (pm.value, km.value, int(rc))
    got_s = dres.cpu().numpy().reshape(B, res_len)
    for i, q in enumerate(bqs):
        ix.query(q, ours, path=ab.PATH_HYBRID)
        torch.cuda.synchronize()
        want = ours.cpu().numpy()
        mismatches += int(not np.array_equal(got_d[i, :n_words], want))
        mismatches += int(not np.array_equal(got_s[i, :n_words], want))
    H.refq_gpu_free(h)

    def stats(v):
        a = np.array(v)
        return {"prep_ms_mean": float(a[:, 0].mean()), "kernel_ms_mean": float(a[:, 1].mean()),
                "kernel_ms_median": float(np.median(a[:, 1])), "kernel_qps": float(1e3 / a[:, 1].mean()),
                "with_prep_qps": float(1e3 / (a[:, 0] + a[:, 1]).mean())}

    out = {"what": "reference GPU kernels (yxr620/AdaBool, built from its sources for sm_100a)",
           "config": cfg.name, "n_postings": int(off[-1]), "records_per_type": n_rec, "sample_queries": n,
           "sample_postings": float(lens[qterms[:qoff[n]]].sum()),
           "ListUnion_sparse": stats(res["sparse"]), "ListUnion_dense": stats(res["dense"]),
           "batch32_dense": {"prep_ms": bd[0], "kernel_ms": bd[1], "kernel_qps": 32e3 / bd[1], "rc": bd[2]},
           "batch32_sparse": {"prep_ms": bs[0], "kernel_ms": bs[1], "kernel_qps": 32e3 / bs[1], "rc": bs[2]},
           "mismatches_vs_libadabool": mismatches,
           "setup_s": {"generate": gen_s, "mixed_build": mixed_s, "reference_load": load_s}}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
