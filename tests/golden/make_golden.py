"""Generates tests/golden/reference_vectors.npz from the reference itself.

Run where the reference source tree is present (it is read in place):

    python tests/golden/make_golden.py

Every expected value in the file comes from reference code compiled from
its own sources (oracle/build_oracle.py): the mixed-container arrays from
ivf_list::BuildFrom (src/AdaBool/inverted_list.h:348-478), the match sets
from ComputeGroundTruth (test/adsfilter_q_all.cu:196-208) and the id lists
from CollectIdsFromBitmap (test/adsfilter_q_all.cu:108-119). The inputs
are hand-written cases (every container type, a 40-value BITSET bucket,
1/2/4-byte key widths, duplicate pairs) and seeded random ones.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_vectors.npz"


def hand_cases(rng):
    cases = {}
    # 1. the reference's own doc example shape plus a BITSET bucket
    t, a = [], []
    # (term, high bucket, bucket size) -> ARRAY1, ARRAY4, ARRAY8, ARRAY16, ARRAY32, BITSET(40)
    for key, (hi, sz) in enumerate([(0, 1), (256, 3), (512, 7), (1024, 12), (2048, 25), (4096, 40)]):
        for v in rng.choice(256, sz, replace=False):
            t.append(key)
            a.append(hi + int(v))
    cases["containers"] = (np.array(t, np.uint32), np.array(a, np.uint32))
    # 2. key spans that force 1-, 2- and 4-byte key offsets in one type:
    #    600 single-id records (ARRAY1) spread over terms 0..599, 70000..,
    #    and 5,000,000 so blocks of 256 records see all three widths
    t = list(range(0, 300)) + list(range(70000, 70300)) + [5_000_000 + 3 * i for i in range(300)]
    a = [(i * 7919) % (1 << 20) for i in range(len(t))]
    cases["key_widths"] = (np.array(t, np.uint32), np.array(a, np.uint32))
    # 3. duplicate pairs, including a duplicated low byte 0 inside an ARRAY
    #    bucket (the reference keeps duplicates in its buckets)
    t = [5] * 8 + [6] * 3 + [7, 7]
    a = [1024, 1024, 1024, 1027, 1030, 1031, 1032, 1033, 7, 7, 9, 0, 0]
    cases["duplicates"] = (np.array(t, np.uint32), np.array(a, np.uint32))
    # 4. empty and single-term
    cases["single"] = (np.array([3], np.uint32), np.array([123456], np.uint32))
    return cases


def random_case(rng, n_terms, n_ads, nnz):
    # Zipf-ish term popularity so all container types appear
    w = 1.0 / np.arange(1, n_terms + 1) ** 1.1
    w /= w.sum()
    t = rng.choice(n_terms, size=nnz, p=w).astype(np.uint32)
    a = rng.integers(0, n_ads, nnz, dtype=np.uint32)
    return t, a


def main():
    rng = np.random.default_rng(20261203)
    hb = O.ref_build_lib()
    hh = O.ref_harness_lib()
    if hb is None or hh is None:
        raise SystemExit("reference libraries missing: run python oracle/build_oracle.py first")
    cases = hand_cases(rng)
    cases["random_small"] = random_case(rng, 400, 1 << 16, 20000)
    cases["random_medium"] = random_case(rng, 1500, 100_000, 30000)
    data = {}
    names = []
    for name, (t, a) in cases.items():
        names.append(name)
        data[f"{name}/terms"] = t
        data[f"{name}/ads"] = a
        ref = O.Mixed.from_coo(t, a, source="reference")
        for ty in range(O.NTYPES):
            for f in O.FIELDS:
                data[f"{name}/mixed/{ty}/{f}"] = ref.array(ty, f)
        ref.free()
        # queries: random term sets, some with out-of-range and repeated terms
        n_terms = int(t.max()) + 1
        qs = []
        for k in range(12):
            n = int(rng.integers(0, 24))
            q = rng.choice(t, size=n).astype(np.uint32) if n else np.zeros(0, np.uint32)
            if k % 3 == 0:
                q = np.concatenate([q, np.array([n_terms + 5, q[0] if q.size else 0], np.uint32)])
            qs.append(q)
        qoff = np.zeros(len(qs) + 1, np.uint64)
        qoff[1:] = np.cumsum([q.size for q in qs])
        qterms = np.concatenate(qs).astype(np.uint32) if qoff[-1] else np.zeros(0, np.uint32)
        data[f"{name}/q_off"] = qoff
        data[f"{name}/q_terms"] = qterms
        h = hh.refq_cpu_load(O._p(t, O.u32p), O._p(a, O.u32p), t.size)
        res, roff = [], [0]
        for q in qs:
            out = np.empty(max(a.size, 1), np.uint32)
            qq = np.ascontiguousarray(q, np.uint32)
            n = hh.refq_ground_truth(h, O._p(qq, O.u32p), qq.size, O._p(out, O.u32p), out.size)
            res.append(out[:n].copy())
            roff.append(roff[-1] + n)
        hh.refq_cpu_free(h)
        data[f"{name}/truth_off"] = np.array(roff, np.uint64)
        data[f"{name}/truth_ids"] = np.concatenate(res).astype(np.uint32) if roff[-1] else np.zeros(0, np.uint32)
    # CollectIdsFromBitmap on bitmaps with a ragged end
    for k, ncols in enumerate([1, 31, 33, 1000, 65536 + 7]):
        nb = (ncols + 7) // 8
        bm = (rng.random(nb) < 0.5).astype(np.uint8) * rng.integers(0, 256, nb, dtype=np.uint8)
        out = np.empty(nb * 8 + 1, np.uint32)
        n = hh.refq_collect_ids(O._p(bm, O.u8p), nb, O._p(out, O.u32p), out.size)
        data[f"collect/{k}/bitmap"] = bm
        data[f"collect/{k}/ids"] = out[:n].copy()
    data["case_names"] = np.array(names)
    np.savez_compressed(OUT, **data)
    print(OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
