"""Batch executor: one CUDA-graph launch per batch.

A batch of up to ``max_queries`` queries (``max_terms`` terms in total) is
answered by one replay of a CUDA graph that holds the whole of
``abf_batch_run``: planning, merge tiles, scatter, probe and (optionally)
compaction -- about ten kernel and memset nodes, launched by the host as a
single graph launch. The graph is captured by the C ABI
(``abf_batch_graph_create`` / ``abf_batch_graph_replay``), once for a fixed
batch size on fixed device buffers; each batch copies its terms/offsets (and
per-query paths) into those buffers on the executor's stream and replays.
Shorter batches are padded with empty queries, which cost one zeroed bitmap
each.

The reference launches six kernels per query (or per batch of at most 32)
from the host after a synchronous, allocating Prepare
(test/adsfilter_batch.cu:453-502); this has no counterpart there.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import check, lib, ptr, stream_ptr


class GraphBatchExecutor:
    def __init__(self, index, max_queries: int, max_terms: int, path: int = N.PATH_HYBRID,
                 with_ids: bool = False, ids_capacity: int = 0, per_query_paths: bool = False, device: int = 0):
        import torch
        self.torch = torch
        self.ix = index
        self.max_q = int(max_queries)
        self.max_t = int(max(max_terms, 1))
        self.path = path
        self.device = device
        self.stride = (index.n_words + 3) // 4 * 4
        dev = torch.device("cuda", device)
        self.d_terms = torch.zeros(self.max_t, dtype=torch.int32, device=dev)
        self.d_off = torch.zeros(self.max_q + 1, dtype=torch.int64, device=dev)
        self.d_paths = torch.full((self.max_q,), int(path), dtype=torch.uint8, device=dev) if per_query_paths \
            else None
        self.bitmaps = torch.empty((self.max_q, self.stride), dtype=torch.int32, device=dev)
        self.d_ids = torch.empty(max(int(ids_capacity), 1), dtype=torch.int32, device=dev) if with_ids else None
        self.d_id_off = torch.zeros(self.max_q + 1, dtype=torch.int64, device=dev) if with_ids else None
        self.ws = index.workspace(self.max_q, self.max_t)
        self.stream = torch.cuda.Stream(device=dev)
        self.graph = None
        self.kernel_nodes = 0
        self._n_set = 0
        # the batch the graph is captured from: the offsets start as all-empty
        # queries, a valid batch for the run that precedes the capture
        self._batch = N.Batch(ptr(self.d_terms), ptr(self.d_off), self.max_q, ptr(self.d_paths), int(path),
                              ptr(self.bitmaps), self.stride, ptr(self.d_ids),
                              0 if self.d_ids is None else self.d_ids.numel(), ptr(self.d_id_off))

    def capture(self):
        """Runs the batch once and captures it into a graph (abf_batch_graph_create)."""
        h = C.c_void_p()
        check(lib().abf_batch_graph_create(self.ix.handle, self.ws.handle, C.byref(self._batch),
                                           stream_ptr(self.stream), C.byref(h)))
        self.graph = h
        n = C.c_uint32()
        check(lib().abf_batch_graph_kernels(h, C.byref(n)))
        self.kernel_nodes = int(n.value)
        self.stream.synchronize()
        return self

    def set_batch(self, q_off: np.ndarray, q_terms: np.ndarray, paths: np.ndarray | None = None):
        """Copies a batch (host arrays) into the captured buffers, padding to max_queries."""
        torch = self.torch
        n = q_off.size - 1
        if n > self.max_q or q_off[-1] > self.max_t:
            raise ValueError("batch larger than the executor was built for")
        off = np.full(self.max_q + 1, q_off[-1], dtype=np.uint64)
        off[:n + 1] = q_off
        with torch.cuda.stream(self.stream):
            if q_terms.size:
                self.d_terms[:q_terms.size].copy_(torch.from_numpy(np.ascontiguousarray(q_terms, np.uint32)
                                                                   .view(np.int32)), non_blocking=False)
            self.d_off.copy_(torch.from_numpy(off.view(np.int64)))
            if paths is not None:
                if self.d_paths is None:
                    raise ValueError("executor built without per-query paths")
                p = np.full(self.max_q, int(self.path), np.uint8)
                p[:n] = paths
                self.d_paths.copy_(torch.from_numpy(p))
        self._n_set = n

    def set_batch_device(self, d_off, d_terms, n_queries: int):
        """Device-to-device form of set_batch (offsets already padded to max_queries + 1)."""
        with self.torch.cuda.stream(self.stream):
            self.d_terms[:d_terms.numel()].copy_(d_terms)
            self.d_off.copy_(d_off)
        self._n_set = n_queries

    def replay(self):
        """Launches the graph on the executor's stream (after set_batch's copies)."""
        if self.graph is None:
            self.capture()
        check(lib().abf_batch_graph_replay(self.graph, stream_ptr(self.stream)))
        return self

    def synchronize(self):
        self.stream.synchronize()

    def free(self):
        if self.graph is not None:
            lib().abf_batch_graph_destroy(self.graph)
            self.graph = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
