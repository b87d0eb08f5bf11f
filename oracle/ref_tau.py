"""The fixed rule's probe threshold from the reference's own CUDA kernels
(TEST AND BASELINE INFRASTRUCTURE ONLY; bench.py and tests/ call it).

The reference has no rule that picks a path: its drivers run both its dense
(bitmap-probe) and its sparse (list-union) path on every query
(test/adsfilter_q_all.cu:414-438). The fixed rule is therefore
build-defined -- probe when the query's lists hold more than tau of all
blocks -- and tau is the crossover of the reference's two paths on the same
index: ListUnion_dense scans the whole index, so its kernel time is about
constant per index; ListUnion_sparse's kernel time grows with the share of
the index the query touches. Both are timed with CUDA events around the
reference's kernel launches (its host-side Prepare is left out), a line
t_sparse = a + b * frac is fitted by least squares over a spread of query
sizes, and tau = (median t_dense - a) / b, clipped to [0, 1].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as O


def reference_tau(off, ads, n_terms: int, n_ads: int, q_off, q_terms, frac, sample: int = 48,
                  stream=None) -> dict:
    """tau from the reference kernels' crossover on this index; `frac` is
    each query's touched-block fraction in this library's format (the
    measure the plan kernel compares with tau). Needs the reference kernel
    library (oracle/_ref/libref_harness.so) and a CUDA device."""
    import torch
    H = O.ref_harness_lib()
    if H is None:
        return {"unavailable": "oracle/_ref/libref_harness.so was not built"}
    nonempty = np.flatnonzero(np.diff(q_off) > 0)
    order = nonempty[np.argsort(frac[nonempty], kind="stable")]
    pick = order[np.unique(np.linspace(0, order.size - 1, min(sample, order.size)).round().astype(np.int64))]
    mixed = O.Mixed.from_csr(off, ads)
    arrs = {f: [mixed.array(t, f) for t in range(O.NTYPES)] for f in ("key_seg", "headers", "keys", "arrays")}
    mixed.free()

    def ptrs(lst, ct):
        return (ct * O.NTYPES)(*[x.ctypes.data_as(ct) if x.size else C.cast(None, ct) for x in lst])

    h = H.refq_gpu_load(ptrs(arrs["key_seg"], O.u32p), (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["key_seg"]]),
                        ptrs(arrs["headers"], O.u32p), (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["headers"]]),
                        ptrs(arrs["keys"], O.u32p), ptrs(arrs["arrays"], O.u8p),
                        (C.c_uint64 * O.NTYPES)(*[x.size for x in arrs["arrays"]]))
    del arrs
    n_words = (n_ads + 31) // 32
    s = stream or torch.cuda.current_stream()
    sp = C.c_void_p(s.cuda_stream)
    d = torch.zeros(n_words + 64, dtype=torch.int32, device="cuda")
    pm, km = C.c_float(), C.c_float()
    ts, td, fs = [], [], []
    try:
        for _ in range(2):  # the first pass warms the kernels up
            ts, td, fs = [], [], []
            for i in pick:
                q = np.ascontiguousarray(q_terms[q_off[i]:q_off[i + 1]], dtype=np.uint32)
                d.zero_()
                rc = H.refq_gpu_sparse(h, q.ctypes.data_as(O.u32p), q.size, C.c_void_p(d.data_ptr()), sp,
                                       C.byref(pm), C.byref(km))
                if rc != 0:
                    raise RuntimeError(f"reference sparse path failed ({rc})")
                ts.append(km.value)
                qb = np.concatenate([O.term_bitmap_bytes(q, n_terms, pad_to=16), np.zeros(32, np.uint8)])
                d.zero_()
                rc = H.refq_gpu_dense(h, qb.ctypes.data_as(O.u8p), qb.size, C.c_void_p(d.data_ptr()), sp,
                                      C.byref(pm), C.byref(km))
                if rc != 0:
                    raise RuntimeError(f"reference dense path failed ({rc})")
                td.append(km.value)
                fs.append(float(frac[i]))
    finally:
        H.refq_gpu_free(h)
    fs, ts, td = np.array(fs), np.array(ts), np.array(td)
    A = np.stack([np.ones_like(fs), fs], 1)
    (a, b), *_ = np.linalg.lstsq(A, ts, rcond=None)
    dense = float(np.median(td))
    tau = float(np.clip((dense - a) / b, 0.0, 1.0)) if b > 0 else 1.0
    return {"tau": tau, "dense_kernel_ms": dense, "sparse_fit_ms": [float(a), float(b)],
            "queries": int(len(pick)), "frac_range": [float(fs.min()), float(fs.max())],
            "sparse_kernel_ms_range": [float(ts.min()), float(ts.max())]}
