"""ctypes binding of libadabool.so (the C ABI in include/adabool.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any device entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libadabool.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
vp = C.c_void_p

ABF_OK = 0
STATUS_NAMES = {0: "ABF_OK", 1: "ABF_ERR_INVALID", 2: "ABF_ERR_RANGE", 3: "ABF_ERR_CUDA", 4: "ABF_ERR_OOM",
                5: "ABF_ERR_STATE", 6: "ABF_ERR_IO", 7: "ABF_ERR_TIMEOUT", 8: "ABF_ERR_CAPACITY",
                9: "ABF_ERR_INTERNAL"}

PATH_AUTO, PATH_PROBE, PATH_UNION, PATH_HYBRID, PATH_TILE = 0, 1, 2, 3, 4
PATH_NAMES = {PATH_AUTO: "auto", PATH_PROBE: "probe", PATH_UNION: "union", PATH_HYBRID: "hybrid",
              PATH_TILE: "tile"}

PLANNER_FEATURES = 16
PLANNER_HIDDEN = 64
PLANNER_OUTPUTS = 3
PLANNER_PARAMS = 2 * 16 + 64 * 16 + 64 + 64 * 64 + 64 + 3 * 64 + 3
PLANNER_PATHS = (1, 2, 3)  # outputs 0..2 predict PROBE, UNION, HYBRID

BUILD_HOST_ONLY = 1
BUILD_KEEP_HOST = 2
QCOUNT_UNIFORM = 0
QCOUNT_LOGNORMAL = 1


class BuildOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("flags", C.c_uint32), ("n_threads", C.c_int), ("dense_div", C.c_uint32)]


DENSE_NONE = 0xFFFFFFFF


class IndexStats(C.Structure):
    _fields_ = [("n_terms", C.c_uint32), ("n_ads", C.c_uint32), ("n_postings", C.c_uint64),
                ("n_blocks", C.c_uint64), ("payload_bytes", C.c_uint64), ("device_bytes", C.c_uint64),
                ("max_list_len", C.c_uint32), ("on_device", C.c_uint32), ("n_dense_lists", C.c_uint32),
                ("n_directory_lists", C.c_uint32), ("dense_bytes", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("tile_words", C.c_uint32), ("warps_per_tile", C.c_uint32), ("heavy_min_len", C.c_uint32),
                ("probe_chunk_blocks", C.c_uint32), ("scatter_blocks_per_warp", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("probe_cap", C.c_uint32), ("probe_min_fraction", C.c_float),
                ("group_min_queries", C.c_uint32), ("fixed_tile_shape", C.c_uint32),
                ("fixed_hybrid_min_len", C.c_uint32), ("compact_ctas_per_sm", C.c_uint32),
                ("group_tile_words", C.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Batch(C.Structure):
    _fields_ = [("d_terms", vp), ("d_offsets", vp), ("n_queries", C.c_uint32), ("d_paths", vp),
                ("path", C.c_int), ("d_bitmaps", vp), ("bitmap_stride_words", C.c_uint64), ("d_ids", vp),
                ("ids_capacity", C.c_uint64), ("d_id_offsets", vp)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_uint64), ("total_ms", C.c_double)]


class GenListsParams(C.Structure):
    _fields_ = [("n_terms", C.c_uint32), ("n_ads", C.c_uint32), ("nnz_target", C.c_uint64),
                ("zipf_s", C.c_double), ("max_len", C.c_uint32), ("seed", C.c_uint64), ("n_threads", C.c_int)]


class GenQueriesParams(C.Structure):
    _fields_ = [("n_queries", C.c_uint32), ("count_kind", C.c_int), ("median", C.c_double),
                ("sigma", C.c_double), ("lo", C.c_uint32), ("hi", C.c_uint32), ("seed", C.c_uint64),
                ("n_threads", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("window_us", C.c_uint32), ("max_batch_queries", C.c_uint32),
                ("max_batch_terms", C.c_uint64), ("n_streams", C.c_uint32), ("path", C.c_int),
                ("outputs", C.c_uint32)]


SERVE_BITMAPS = 1
SERVE_IDS = 2


class ServerResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int32), ("path", C.c_uint32),
                ("d_bitmap", vp), ("d_ids", vp), ("n_ids", C.c_uint64), ("t_arrival_ns", C.c_uint64),
                ("t_launch_ns", C.c_uint64), ("t_done_ns", C.c_uint64), ("batch_queries", C.c_uint32),
                ("pad_", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("submitted", "completed", "released", "rejected", "batches",
                                          "failed_batches", "waiting", "in_flight_batches", "pool_bytes",
                                          "reserved_bytes", "peak_reserved_bytes", "admission_waits")] + \
               [("path_queries", C.c_uint64 * 5), ("max_batch_queries_seen", C.c_uint64)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["path_queries"] = list(self.path_queries)
        return d


class TraceStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("failed", C.c_uint64)]


# (name, argtypes) of every exported entry point; restype is abf_status
# (c_int) unless listed in _RESTYPES.
PROTOTYPES = {
    "abf_index_build_coo": [u32p, u32p, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(BuildOpts), C.POINTER(vp)],
    "abf_index_build_csr": [u64p, u32p, C.c_uint32, C.c_uint32, C.POINTER(BuildOpts), C.POINTER(vp)],
    "abf_index_free": [vp],
    "abf_index_get_stats": [vp, C.POINTER(IndexStats)],
    "abf_index_list_lengths": [vp, u32p, C.c_uint32],
    "abf_index_decode_list": [vp, C.c_uint32, u32p, C.c_uint64, u64p],
    "abf_index_save": [vp, C.c_char_p],
    "abf_index_load": [C.c_char_p, C.POINTER(BuildOpts), C.POINTER(vp)],
    "abf_index_to_device": [vp, C.c_int],
    "abf_get_tuning": [vp, C.POINTER(Tuning)],
    "abf_set_tuning": [vp, C.POINTER(Tuning)],
    "abf_index_set_dense_div": [vp, C.c_uint32],
    "abf_prepare_sparse": [vp, u32p, C.c_uint64, C.POINTER(vp)],
    "abf_prepare_dense": [vp, C.c_uint64, u8p, C.POINTER(vp)],
    "abf_prepare_batch": [vp, C.c_uint64, C.c_uint64, u8p, C.POINTER(vp)],
    "abf_prepare_batch_device": [vp, C.c_uint64, C.c_uint64, vp, C.POINTER(vp)],
    "abf_worker_free": [vp],
    "abf_list_union_sparse": [vp, vp, vp],
    "abf_list_union_dense": [vp, vp, vp],
    "abf_batch_list_union_dense": [vp, vp, C.c_uint32, vp],
    "abf_batch_list_union_sparse": [vp, vp, vp, C.c_uint32, vp],
    "abf_collect_ids": [vp, vp, C.c_uint64, vp, C.c_uint64, vp, vp],
    "abf_batch_collect_ids": [vp, vp, vp, C.c_uint64, C.c_uint32, vp, C.c_uint64, vp, vp],
    "abf_collect_ids_noalloc": [vp, C.c_uint64, vp, C.c_uint64, vp, vp],
    "abf_collect_ids_noalloc_check": [vp],
    "abf_workspace_create": [vp, C.c_uint32, C.c_uint64, C.POINTER(vp)],
    "abf_workspace_free": [vp],
    "abf_workspace_check": [vp, vp],
    "abf_workspace_set_wait_limit": [vp, C.c_uint32],
    "abf_workspace_paths": [vp, u8p, C.c_uint32, vp],
    "abf_workspace_selftest_waits": [vp, C.c_uint32, vp],
    "abf_batch_run": [vp, vp, C.POINTER(Batch), vp],
    "abf_query": [vp, u32p, C.c_uint32, C.c_int, vp, vp, C.c_uint64, vp, vp],
    "abf_batch_graph_create": [vp, vp, C.POINTER(Batch), vp, C.POINTER(vp)],
    "abf_batch_graph_replay": [vp, vp],
    "abf_batch_graph_kernels": [vp, u32p],
    "abf_batch_graph_destroy": [vp],
    "abf_planner_features": [vp, vp, vp, C.c_uint32, vp, vp],
    "abf_planner_set": [vp, vp],
    "abf_planner_predict": [vp, vp, vp, C.c_uint32, vp, vp, vp],
    "abf_mlp_forward": [vp, vp, C.c_uint32, vp, vp],
    "abf_mlp_grad": [vp, vp, vp, vp, C.c_uint32, vp, vp, vp],
    "abf_mlp_adam": [vp, vp, vp, vp, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, vp],
    "abf_index_list_bytes": [vp, u64p, C.c_uint32],
    "abf_index_list_flags": [vp, u32p, C.c_uint32],
    "abf_profile_enable": [vp, C.c_int],
    "abf_profile_read": [vp, vp, C.c_uint32, u32p],
    "abf_clock_ns": [],
    "abf_server_default_opts": [C.POINTER(ServerOpts)],
    "abf_server_create": [vp, C.POINTER(ServerOpts), C.POINTER(vp)],
    "abf_server_submit": [vp, u32p, C.c_uint32, C.c_uint64, C.c_uint64, u64p],
    "abf_server_poll": [vp, C.POINTER(ServerResult), C.c_uint32, C.c_uint32, u32p],
    "abf_server_release": [vp, C.c_uint64],
    "abf_server_get_stats": [vp, C.POINTER(ServerStats)],
    "abf_server_destroy": [vp],
    "abf_server_run_trace": [vp, u32p, u64p, C.c_uint32, u64p, C.c_double, u64p, u64p, u64p, u8p,
                             C.POINTER(TraceStats)],
    "abf_last_error_string": [],
    "abf_status_string": [C.c_int],
    "abf_abi_version": [],
    "abf_launch_count": [],
    "abf_gen_target_lengths": [C.POINTER(GenListsParams), u32p],
    "abf_gen_lists_offsets": [C.POINTER(GenListsParams), u64p],
    "abf_gen_lists_fill": [C.POINTER(GenListsParams), u64p, u32p],
    "abf_gen_queries_offsets": [C.POINTER(GenQueriesParams), u32p, C.c_uint32, u64p],
    "abf_gen_queries_fill": [C.POINTER(GenQueriesParams), u32p, C.c_uint32, u64p, u32p],
}
_RESTYPES = {"abf_last_error_string": C.c_char_p, "abf_status_string": C.c_char_p,
             "abf_abi_version": C.c_uint32, "abf_launch_count": C.c_uint64, "abf_clock_ns": C.c_uint64}

_lib = None


class AbfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m adabool_b200.build` "
                               "(there is no fallback implementation)")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
        for name, args in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def check(status: int):
    if status != ABF_OK:
        raise AbfError(status, lib().abf_last_error_string().decode(errors="replace"))
    return status


def ptr(x, ctype=None):
    """Address of a numpy array or torch tensor as a ctypes pointer/void*."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        addr = x.data_ptr()
    elif hasattr(x, "ctypes"):
        addr = x.ctypes.data
    else:
        addr = int(x)
    return C.cast(addr, ctype) if ctype is not None else C.c_void_p(addr)


def stream_ptr(stream):
    """cudaStream_t of a torch stream (or an int handle); None = default stream."""
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))
