"""Index, workers and workspaces: Python mirror of the reference's operator API.

The names follow the reference so that code written against it reads the
same: ``Index.BuildFrom`` is ``ivf_list::BuildFrom``
(src/AdaBool/inverted_list.h:348), ``Index.Prepare`` is ``ivf_list::Prepare``
(src/AdaBool/inverted_list.h:481,530), the four ``*ListUnion_*`` functions are
the test drivers' operator entry points (test/adsfilter_q_all.cu:26-105,
test/adsfilter_batch.cu:27-79). The reference's entry points return
``cudaError_t`` and abort on allocation failure; these return 0 and raise
``AbfError`` on any failure.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional

import numpy as np

from . import _native as N
from ._native import check, lib, ptr, stream_ptr


def launch_count() -> int:
    """Kernel launches enqueued by libadabool since it was loaded."""
    return int(lib().abf_launch_count())


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


class Worker:
    """A prepared query (sparse: term ids; dense: term bitmaps)."""

    def __init__(self, handle: C.c_void_p, index: "Index", kind: str, keep=None):
        self._h = handle
        self.index = index
        self.kind = kind
        self._keep = keep  # caller device bitmaps of PrepareBatchDevice stay alive

    @property
    def handle(self):
        return self._h

    def free(self):
        if self._h:
            lib().abf_worker_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Workspace:
    """Scratch arrays for one in-flight batch (see abf_workspace_create)."""

    def __init__(self, index: "Index", max_queries: int, max_terms: int):
        h = C.c_void_p()
        check(lib().abf_workspace_create(index.handle, max_queries, max_terms, C.byref(h)))
        self._h = h
        self.index = index
        self.max_queries = max_queries
        self.max_terms = max_terms

    @property
    def handle(self):
        return self._h

    def check(self, stream=None):
        check(lib().abf_workspace_check(self._h, stream_ptr(stream)))

    def paths(self, n: int, stream=None) -> np.ndarray:
        """abf_path each of the last batch's first n queries ran on."""
        out = np.zeros(n, np.uint8)
        check(lib().abf_workspace_paths(self._h, ptr(out, N.u8p), n, stream_ptr(stream)))
        return out

    def set_wait_limit(self, polls: int):
        """Polls of every bounded device wait of this workspace's kernels."""
        check(lib().abf_workspace_set_wait_limit(self._h, int(polls)))

    def selftest_waits(self, polls: int, stream=None):
        """Makes one mbarrier wait and one look-back wait run out (see
        abf_workspace_selftest_waits); check() then raises ABF_ERR_TIMEOUT."""
        check(lib().abf_workspace_selftest_waits(self._h, int(polls), stream_ptr(stream)))

    def free(self):
        if self._h:
            lib().abf_workspace_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Index:
    """Compressed inverted lists of a terms x ads filter matrix."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        st = N.IndexStats()
        check(lib().abf_index_get_stats(self._h, C.byref(st)))
        self.n_terms = st.n_terms
        self.n_ads = st.n_ads
        self.n_words = (self.n_ads + 31) // 32
        self.dense_div = 128  # library default; set_dense_div / the builder's dense_div change it

    # ---- construction -------------------------------------------------
    @staticmethod
    def _opts(device, host_only, keep_host, n_threads, dense_div=0):
        """dense_div: 0 = library default, None = no dense bitmaps."""
        flags = (N.BUILD_HOST_ONLY if host_only else 0) | (N.BUILD_KEEP_HOST if keep_host else 0)
        return N.BuildOpts(device, flags, n_threads, N.DENSE_NONE if dense_div is None else int(dense_div))

    @classmethod
    def from_coo(cls, terms, ads, n_terms: int, n_ads: int, device: int = 0, host_only: bool = False,
                 keep_host: bool = False, n_threads: int = 0, dense_div=0) -> "Index":
        t, a = _u32(terms), _u32(ads)
        if t.shape != a.shape:
            raise ValueError("terms and ads differ in length")
        h = C.c_void_p()
        o = cls._opts(device, host_only, keep_host, n_threads, dense_div)
        check(lib().abf_index_build_coo(ptr(t, N.u32p), ptr(a, N.u32p), t.size, n_terms, n_ads, C.byref(o),
                                        C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, ads, n_terms: int, n_ads: int, device: int = 0, host_only: bool = False,
                 keep_host: bool = False, n_threads: int = 0, dense_div=0) -> "Index":
        off, a = _u64(offsets), _u32(ads)
        if off.size != n_terms + 1:
            raise ValueError("offsets must have n_terms + 1 entries")
        h = C.c_void_p()
        o = cls._opts(device, host_only, keep_host, n_threads, dense_div)
        check(lib().abf_index_build_csr(ptr(off, N.u64p), ptr(a, N.u32p), n_terms, n_ads, C.byref(o),
                                        C.byref(h)))
        return cls(h)

    @classmethod
    def BuildFrom(cls, pairs: Iterable, n_terms: Optional[int] = None, n_ads: Optional[int] = None,
                  **kw) -> "Index":
        """(term, ad) pairs -> index; domain defaults to max+1 like the reference's drivers
        (test/adsfilter_q_all.cu:359-360)."""
        arr = np.asarray(list(pairs) if not isinstance(pairs, np.ndarray) else pairs, dtype=np.uint32)
        arr = arr.reshape(-1, 2)
        n_terms = int(arr[:, 0].max()) + 1 if n_terms is None else n_terms
        n_ads = int(arr[:, 1].max()) + 1 if n_ads is None else n_ads
        return cls.from_coo(arr[:, 0], arr[:, 1], n_terms, n_ads, **kw)

    @classmethod
    def load(cls, path: str, device: int = 0, host_only: bool = False, keep_host: bool = False,
             dense_div=0) -> "Index":
        h = C.c_void_p()
        o = cls._opts(device, host_only, keep_host, 0, dense_div)
        check(lib().abf_index_load(str(path).encode(), C.byref(o), C.byref(h)))
        return cls(h)

    def save(self, path: str):
        check(lib().abf_index_save(self._h, str(path).encode()))

    def to_device(self, device: int = 0):
        check(lib().abf_index_to_device(self._h, device))

    @property
    def handle(self):
        return self._h

    def free(self):
        if self._h:
            lib().abf_index_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # ---- inspection ---------------------------------------------------
    def stats(self) -> dict:
        st = N.IndexStats()
        check(lib().abf_index_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def list_lengths(self) -> np.ndarray:
        out = np.empty(self.n_terms, dtype=np.uint32)
        check(lib().abf_index_list_lengths(self._h, ptr(out, N.u32p), self.n_terms))
        return out

    def decode_list(self, term: int) -> np.ndarray:
        n = C.c_uint64()
        check(lib().abf_index_decode_list(self._h, term, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.uint32)
        check(lib().abf_index_decode_list(self._h, term, ptr(out, N.u32p), out.size, C.byref(n)))
        return out

    def list_bytes(self) -> np.ndarray:
        """Compressed bytes of each term's list (payload + 16 B metadata per block)."""
        out = np.empty(self.n_terms, dtype=np.uint64)
        check(lib().abf_index_list_bytes(self._h, ptr(out, N.u64p), self.n_terms))
        return out

    def list_flags(self) -> np.ndarray:
        """Per-term flags: 1 = also a dense bitmap, 2 = per-tile block directory."""
        out = np.empty(self.n_terms, dtype=np.uint32)
        check(lib().abf_index_list_flags(self._h, ptr(out, N.u32p), self.n_terms))
        return out

    def profile(self, on: bool = True):
        check(lib().abf_profile_enable(self._h, 1 if on else 0))
        self._profiling = bool(on)

    def profile_read(self) -> dict:
        """{kernel: (launches, total_ms)} since the last read (synchronises)."""
        buf = (N.KernelTime * 16)()
        n = C.c_uint32()
        check(lib().abf_profile_read(self._h, C.cast(buf, C.c_void_p), 16, C.byref(n)))
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].total_ms)) for i in range(n.value)}

    @property
    def tuning(self) -> N.Tuning:
        t = N.Tuning()
        check(lib().abf_get_tuning(self._h, C.byref(t)))
        return t

    @tuning.setter
    def tuning(self, t: N.Tuning):
        check(lib().abf_set_tuning(self._h, C.byref(t)))

    def set_dense_div(self, dense_div):
        """Rebuild the dense bitmaps for lists with len * dense_div >= n_ads (None: no bitmaps)."""
        check(lib().abf_index_set_dense_div(self._h, N.DENSE_NONE if dense_div is None else int(dense_div)))
        self.dense_div = dense_div

    def set_tuning(self, **kw):
        t = self.tuning
        for k, v in kw.items():
            setattr(t, k, v)
        self.tuning = t

    # ---- reference-shaped workers -------------------------------------
    def Prepare(self, keys_or_len, query_bitmap=None) -> Worker:
        """Prepare(keys) -> sparse worker; Prepare(len, bitmap) -> dense worker."""
        h = C.c_void_p()
        if query_bitmap is None:
            k = _u32(keys_or_len)
            check(lib().abf_prepare_sparse(self._h, ptr(k, N.u32p), k.size, C.byref(h)))
            return Worker(h, self, "sparse")
        bm = np.ascontiguousarray(np.asarray(query_bitmap, dtype=np.uint8))
        check(lib().abf_prepare_dense(self._h, int(keys_or_len), ptr(bm, N.u8p), C.byref(h)))
        return Worker(h, self, "dense")

    def PrepareBatch(self, batch_size: int, length: int, query_bitmap) -> Worker:
        bm = np.ascontiguousarray(np.asarray(query_bitmap, dtype=np.uint8))
        h = C.c_void_p()
        check(lib().abf_prepare_batch(self._h, batch_size, length, ptr(bm, N.u8p), C.byref(h)))
        return Worker(h, self, "dense")

    def PrepareBatchDevice(self, batch_size: int, length: int, d_query_bitmap) -> Worker:
        h = C.c_void_p()
        check(lib().abf_prepare_batch_device(self._h, batch_size, length, ptr(d_query_bitmap), C.byref(h)))
        return Worker(h, self, "dense", keep=d_query_bitmap)

    # ---- native API ---------------------------------------------------
    def workspace(self, max_queries: int, max_terms: int) -> Workspace:
        return Workspace(self, max_queries, max_terms)

    def query(self, terms, d_bitmap, path: int = N.PATH_AUTO, d_ids=None, d_count=None, stream=None):
        t = _u32(terms)
        cap = 0 if d_ids is None else d_ids.numel()
        check(lib().abf_query(self._h, ptr(t, N.u32p), t.size, path, ptr(d_bitmap), ptr(d_ids), cap,
                              ptr(d_count), stream_ptr(stream)))

    def batch_run(self, ws: Workspace, d_terms, d_offsets, n_queries: int, d_bitmaps, stride_words: int,
                  path: int = N.PATH_AUTO, d_paths=None, d_ids=None, d_id_offsets=None, stream=None):
        b = N.Batch(ptr(d_terms), ptr(d_offsets), n_queries, ptr(d_paths), path, ptr(d_bitmaps), stride_words,
                    ptr(d_ids), 0 if d_ids is None else d_ids.numel(), ptr(d_id_offsets))
        check(lib().abf_batch_run(self._h, ws.handle, C.byref(b), stream_ptr(stream)))


# ---- reference operator entry points ----------------------------------
def ListUnion_dense(worker: Worker, d_res, stream=None) -> int:
    """Bitmap-probe of a dense worker ORed into d_res (test/adsfilter_q_all.cu:26-61)."""
    return check(lib().abf_list_union_dense(worker.handle, ptr(d_res), stream_ptr(stream)))


def ListUnion_sparse(worker: Worker, d_res, stream=None) -> int:
    """List-union of a sparse worker ORed into d_res (test/adsfilter_q_all.cu:64-105)."""
    return check(lib().abf_list_union_sparse(worker.handle, ptr(d_res), stream_ptr(stream)))


def BatchListUnion_dense(worker: Worker, stream, d_res, res_len_u32: int) -> int:
    """Batched probe, query b into d_res + b*res_len_u32 (test/adsfilter_batch.cu:28-36)."""
    return check(lib().abf_batch_list_union_dense(worker.handle, ptr(d_res), res_len_u32, stream_ptr(stream)))


def BatchListUnion_sparse(worker: Worker, d_res, d_qidx, res_len_per_batch_bytes: int, stream=None) -> int:
    """Batched union, key i into d_res + d_qidx[i]*res_len/4 (test/adsfilter_batch.cu:39-79)."""
    return check(lib().abf_batch_list_union_sparse(worker.handle, ptr(d_res), ptr(d_qidx),
                                                   res_len_per_batch_bytes, stream_ptr(stream)))


def BatchCollectIds(index: Index, ws: Workspace, d_bitmaps, stride_words: int, n_bitmaps: int, d_ids, d_id_offsets,
                    stream=None) -> int:
    """Packed ascending ids of a batch of device bitmaps (abf_batch_collect_ids)."""
    return check(lib().abf_batch_collect_ids(index.handle, ws.handle, ptr(d_bitmaps), stride_words, n_bitmaps,
                                             ptr(d_ids), 0 if d_ids is None else d_ids.numel(), ptr(d_id_offsets),
                                             stream_ptr(stream)))


def CollectIdsFromBitmap(index: Index, d_bitmap, n_bits: int, d_ids, d_count, stream=None) -> int:
    """Ascending ids of the set bits below n_bits, on the device (test/adsfilter_batch.cu:82-97)."""
    return check(lib().abf_collect_ids(index.handle, ptr(d_bitmap), n_bits, ptr(d_ids), d_ids.numel(),
                                       ptr(d_count), stream_ptr(stream)))
