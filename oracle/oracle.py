"""ctypes access to the oracle libraries (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs load this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build_oracle as B

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)

NTYPES = 6
FIELDS = ["key_seg", "headers", "keys", "arrays", "pos_seg", "blk_seg", "key_buf"]
BYTE_FIELDS = {"arrays", "key_buf"}

_orc = None
_refb = None
_refh = None


def _p(a, t):
    return a.ctypes.data_as(t)


def orc():
    global _orc
    if _orc is None:
        B.build_orc()
        L = C.CDLL(str(B.LIBORC))
        L.orc_kway_union.argtypes = [u64p, u32p, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint64]
        L.orc_kway_union.restype = C.c_uint64
        L.orc_scan_union.argtypes = [u32p, u32p, C.c_uint64, u32p, C.c_uint32, u32p, C.c_uint64]
        L.orc_scan_union.restype = C.c_uint64
        L.orc_ids_to_bitmap.argtypes = [u32p, C.c_uint64, u32p, C.c_uint64]
        L.orc_ids_to_bitmap.restype = None
        L.orc_collect_ids.argtypes = [u8p, C.c_uint64, C.c_uint64, u32p, C.c_uint64]
        L.orc_collect_ids.restype = C.c_uint64
        L.orc_cpu_batch.argtypes = [u64p, u32p, C.c_uint32, u64p, u32p, C.c_uint32, C.c_int, u64p]
        L.orc_cpu_batch.restype = C.c_uint64
        L.orc_cpu_batch_sums.argtypes = [u64p, u32p, C.c_uint32, u64p, u32p, C.c_uint32, C.c_int, u64p, u64p]
        L.orc_cpu_batch_sums.restype = C.c_uint64
        L.orc_mixed_build_coo.argtypes = [u32p, u32p, C.c_uint64, C.c_int]
        L.orc_mixed_build_coo.restype = C.c_void_p
        L.orc_mixed_build_csr.argtypes = [u64p, u32p, C.c_uint32, C.c_int]
        L.orc_mixed_build_csr.restype = C.c_void_p
        L.orc_mixed_free.argtypes = [C.c_void_p]
        L.orc_mixed_free.restype = None
        L.orc_mixed_array.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), u64p]
        L.orc_mixed_array.restype = C.c_int
        L.orc_mixed_union.argtypes = [C.c_void_p, u32p, C.c_uint64, u32p, C.c_uint64]
        L.orc_mixed_union.restype = None
        L.orc_mixed_probe.argtypes = [C.c_void_p, u8p, C.c_uint64, u32p, C.c_uint64]
        L.orc_mixed_probe.restype = None
        _orc = L
    return _orc


def ref_build_lib():
    """The reference's own BuildFrom (g++), or None where it was not built."""
    global _refb
    if _refb is None:
        if not B.REF_BUILD.exists():
            try:
                B.build_ref(with_gpu=False)
            except Exception:
                return None
        if not B.REF_BUILD.exists():
            return None
        L = C.CDLL(str(B.REF_BUILD))
        L.refb_build.argtypes = [u32p, u32p, C.c_uint64]
        L.refb_build.restype = C.c_void_p
        L.refb_array.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), u64p]
        L.refb_array.restype = C.c_int
        L.refb_free.argtypes = [C.c_void_p]
        L.refb_free.restype = None
        _refb = L
    return _refb


def ref_harness_lib():
    """The reference's driver (CPU ground truth + GPU kernels), or None."""
    global _refh
    if _refh is None:
        if not B.REF_HARNESS.exists():
            return None
        L = C.CDLL(str(B.REF_HARNESS))
        vp = C.c_void_p
        L.refq_cpu_load.argtypes = [u32p, u32p, C.c_uint64]
        L.refq_cpu_load.restype = vp
        L.refq_cpu_free.argtypes = [vp]
        L.refq_cpu_free.restype = None
        L.refq_ground_truth.argtypes = [vp, u32p, C.c_uint32, u32p, C.c_uint64]
        L.refq_ground_truth.restype = C.c_uint64
        L.refq_ground_truth_batch.argtypes = [vp, u64p, u32p, C.c_uint32, C.c_int, u64p]
        L.refq_ground_truth_batch.restype = C.c_uint64
        L.refq_collect_ids.argtypes = [u8p, C.c_uint64, u32p, C.c_uint64]
        L.refq_collect_ids.restype = C.c_uint64
        pp32 = C.POINTER(u32p)
        L.refq_gpu_load.argtypes = [pp32, u64p, pp32, u64p, pp32, C.POINTER(u8p), u64p]
        L.refq_gpu_load.restype = vp
        L.refq_gpu_free.argtypes = [vp]
        L.refq_gpu_free.restype = None
        fp = C.POINTER(C.c_float)
        L.refq_gpu_dense.argtypes = [vp, u8p, C.c_uint64, vp, vp, fp, fp]
        L.refq_gpu_dense.restype = C.c_int
        L.refq_gpu_sparse.argtypes = [vp, u32p, C.c_uint64, vp, vp, fp, fp]
        L.refq_gpu_sparse.restype = C.c_int
        L.refq_gpu_batch_dense32.argtypes = [vp, u8p, C.c_uint64, vp, C.c_uint32, vp, fp, fp]
        L.refq_gpu_batch_dense32.restype = C.c_int
        L.refq_gpu_batch_sparse.argtypes = [vp, u32p, u32p, C.c_uint64, vp, C.c_uint32, vp, fp, fp]
        L.refq_gpu_batch_sparse.restype = C.c_int
        _refh = L
    return _refh


# ---------------------------------------------------------------------------
def kway_union(off: np.ndarray, ads: np.ndarray, q) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.uint32)
    n_terms = off.size - 1
    cap = int(sum(int(off[t + 1] - off[t]) for t in q if t < n_terms))
    out = np.empty(max(cap, 1), dtype=np.uint32)
    n = orc().orc_kway_union(_p(off, u64p), _p(ads, u32p), n_terms, _p(q, u32p), q.size, _p(out, u32p), cap)
    return out[:n].copy()


def scan_union(terms: np.ndarray, ads: np.ndarray, q) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.uint32)
    out = np.empty(max(terms.size, 1), dtype=np.uint32)
    n = orc().orc_scan_union(_p(terms, u32p), _p(ads, u32p), terms.size, _p(q, u32p), q.size, _p(out, u32p),
                             out.size)
    return out[:n].copy()


def ids_to_bitmap(ids: np.ndarray, n_words: int) -> np.ndarray:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    w = np.zeros(n_words, dtype=np.uint32)
    orc().orc_ids_to_bitmap(_p(ids, u32p), ids.size, _p(w, u32p), n_words)
    return w


def collect_ids(words: np.ndarray, ncols: int) -> np.ndarray:
    b = np.ascontiguousarray(words).view(np.uint8)
    out = np.empty(max(ncols, 1), dtype=np.uint32)
    n = orc().orc_collect_ids(_p(b, u8p), b.size, ncols, _p(out, u32p), out.size)
    return out[:n].copy()


def cpu_batch(off, ads, q_off, q_terms, n_threads: int, sums: bool = False):
    """Heap k-way merge of every query on n_threads host threads: per-query
    id counts, and with sums=True also (sum of ids, sum of ids * position)
    mod 2^64 per query (an order-sensitive checksum of the sorted ids)."""
    counts = np.zeros(q_off.size - 1, dtype=np.uint64)
    q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
    q_terms = np.ascontiguousarray(q_terms, dtype=np.uint32)
    if not sums:
        orc().orc_cpu_batch(_p(off, u64p), _p(ads, u32p), off.size - 1, _p(q_off, u64p), _p(q_terms, u32p),
                            q_off.size - 1, n_threads, _p(counts, u64p))
        return counts
    s = np.zeros((q_off.size - 1, 2), dtype=np.uint64)
    orc().orc_cpu_batch_sums(_p(off, u64p), _p(ads, u32p), off.size - 1, _p(q_off, u64p), _p(q_terms, u32p),
                             q_off.size - 1, n_threads, _p(counts, u64p), _p(s, u64p))
    return counts, s


def gen_lib():
    """The standalone build of the workload generator (oracle/libwgen.so)."""
    B.build_wgen()
    return C.CDLL(str(B.LIBWGEN))


class Mixed:
    """The reference's mixed-container index, built by the oracle's restatement
    (source="oracle") or by the reference's own BuildFrom (source="reference")."""

    def __init__(self, handle, lib, getter, free):
        self._h, self._lib, self._get, self._free = handle, lib, getter, free

    @classmethod
    def from_coo(cls, terms, ads, source: str = "oracle", block_step: int = 256):
        t = np.ascontiguousarray(terms, dtype=np.uint32)
        a = np.ascontiguousarray(ads, dtype=np.uint32)
        if source == "oracle":
            L = orc()
            h = L.orc_mixed_build_coo(_p(t, u32p), _p(a, u32p), t.size, block_step)
            return cls(h, L, L.orc_mixed_array, L.orc_mixed_free)
        L = ref_build_lib()
        if L is None:
            raise RuntimeError("reference builder not available")
        h = L.refb_build(_p(t, u32p), _p(a, u32p), t.size)
        return cls(h, L, L.refb_array, L.refb_free)

    @classmethod
    def from_csr(cls, off, ads, block_step: int = 256):
        o = np.ascontiguousarray(off, dtype=np.uint64)
        a = np.ascontiguousarray(ads, dtype=np.uint32)
        L = orc()
        h = L.orc_mixed_build_csr(_p(o, u64p), _p(a, u32p), o.size - 1, block_step)
        return cls(h, L, L.orc_mixed_array, L.orc_mixed_free)

    def array(self, t: int, field: str) -> np.ndarray:
        p = C.c_void_p()
        n = C.c_uint64()
        rc = self._get(self._h, t, FIELDS.index(field), C.byref(p), C.byref(n))
        if rc != 0:
            raise ValueError("bad type/field")
        dt = np.uint8 if field in BYTE_FIELDS else np.uint32
        if n.value == 0 or not p.value:
            return np.zeros(0, dtype=dt)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8 if dt == np.uint8 else C.c_uint32)),
                                     shape=(n.value,)).copy()

    def union(self, keys, n_words: int) -> np.ndarray:
        k = np.ascontiguousarray(keys, dtype=np.uint32)
        res = np.zeros(n_words, dtype=np.uint32)
        orc().orc_mixed_union(self._h, _p(k, u32p), k.size, _p(res, u32p), n_words)
        return res

    def probe(self, qbm_bytes: np.ndarray, n_words: int) -> np.ndarray:
        b = np.ascontiguousarray(qbm_bytes, dtype=np.uint8)
        res = np.zeros(n_words, dtype=np.uint32)
        orc().orc_mixed_probe(self._h, _p(b, u8p), b.size, _p(res, u32p), n_words)
        return res

    def free(self):
        if self._h:
            self._free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def term_bitmap_bytes(q, n_terms: int, pad_to: int = 16) -> np.ndarray:
    """Byte bitmap of query terms (bit t of byte t/8), as the reference's
    drivers build it (test/adsfilter_q_all.cu:407-412), padded to pad_to."""
    nb = (n_terms + 7) // 8
    nb = (nb + pad_to - 1) // pad_to * pad_to
    b = np.zeros(nb, dtype=np.uint8)
    for t in np.asarray(q, dtype=np.uint64):
        if t < n_terms:
            b[t >> 3] |= np.uint8(1 << (t & 7))
    return b
