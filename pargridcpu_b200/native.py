"""ctypes binding of libfirmcore.so (the C ABI in include/firmcore.h).

The shared library is built in place (``pargridcpu_b200/libfirmcore.so``) by
``pargridcpu_b200/csrc/Makefile``.  Loading fails loudly when it is missing:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfirmcore.so")

FC_OK = 0
STATUS = {0: "FC_OK", 1: "FC_ERR_IO", 2: "FC_ERR_PARSE", 3: "FC_ERR_OOM", 4: "FC_ERR_BUDGET",
          5: "FC_ERR_DEVICE", 6: "FC_ERR_ITER_LIMIT", 7: "FC_ERR_INVALID", 8: "FC_ERR_TOO_LARGE",
          9: "FC_ERR_NO_DEVICE"}

# every function include/firmcore.h declares
EXPORTS = [
    "fc_status_string", "fc_abi_version", "fc_graph_load_dir", "fc_graph_from_pairs",
    "fc_graph_from_adjbuf", "fc_graph_free", "fc_graph_n", "fc_graph_layers", "fc_graph_layer_m",
    "fc_graph_id2vtx", "fc_graph_order", "fc_graph_csr", "fc_graph_upload",
    "fc_graph_release_device", "fc_graph_reset_results", "fc_graph_device_bytes", "fc_coreindex",
    "fc_densest", "fc_densest_members", "fc_cell_members", "fc_cells", "fc_coreindex_range",
    "fc_cells_range", "fc_batch_run", "fc_server_create",
    "fc_server_submit", "fc_server_wait", "fc_server_query", "fc_server_destroy", "fc_graph_stats",
    "fc_launch_count", "fc_coreindex_fixed_scratch", "fc_cell_index", "fc_cells_members",
    "fc_mlcd_query", "fc_probe_atomics", "fc_alloc_count", "fc_coreindex_densest",
]


class FcError(RuntimeError):
    def __init__(self, what, code):
        super().__init__(f"{what}: {STATUS.get(code, code)} ({lib().fc_status_string(code).decode()})")
        self.code = code


class DensestResult(C.Structure):
    _fields_ = [("beta", C.c_double), ("density", C.c_double), ("max_density_f", C.c_float),
                ("k", C.c_uint32), ("lmd", C.c_uint32), ("length", C.c_uint32),
                ("lstar", C.c_uint32), ("n_cells", C.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Cell(C.Structure):
    _fields_ = [("k", C.c_uint32), ("lmd", C.c_uint32), ("length", C.c_uint32),
                ("lstar", C.c_uint32), ("density", C.c_double)]


class BatchOptions(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("hub_threshold", C.c_uint32),
                ("use_cuda_graph", C.c_int), ("plain", C.c_int)]


class BatchReport(C.Structure):
    _fields_ = [("peel_ms", C.c_double), ("densest_ms", C.c_double),
                ("peel_launches", C.c_uint32), ("block_threads", C.c_uint32),
                ("hub_threshold", C.c_uint32), ("levels", C.c_uint32),
                ("used_cuda_graph", C.c_int), ("autotuned", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [("peel_ms", C.c_double), ("densest_ms", C.c_double),
                ("peel_launches", C.c_uint32), ("levels", C.c_uint32), ("subrounds", C.c_uint32),
                ("columns_per_launch", C.c_uint32), ("phase_ms", C.c_double * 3)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["phase_ms"] = list(self.phase_ms)
        return d


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_inflight", C.c_uint32),
                ("lanes", C.c_uint32), ("max_batch_graphs", C.c_uint32),
                ("block_threads", C.c_uint32), ("hub_threshold", C.c_uint32),
                ("plain", C.c_int), ("heavy_visits", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_uint64), ("batches", C.c_uint64),
                ("heavy_batches", C.c_uint64), ("graphs_peeled", C.c_uint64), ("uploads", C.c_uint64),
                ("evictions", C.c_uint64), ("resident_bytes", C.c_uint64),
                ("peak_bytes", C.c_uint64), ("busy_ms", C.c_double), ("overlap_ms", C.c_double),
                ("max_batch", C.c_uint32), ("lanes", C.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run pargridcpu_b200.build() "
                          "(make -C pargridcpu_b200/csrc)")
    L = C.CDLL(LIB_PATH)
    p, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    pp = C.POINTER(C.c_void_p)
    sig = {
        "fc_status_string": ([i32], C.c_char_p),
        "fc_abi_version": ([], i32),
        "fc_graph_load_dir": ([C.c_char_p, i32, i32, pp], i32),
        "fc_graph_from_pairs": ([u32, p, p, pp], i32),
        "fc_graph_from_adjbuf": ([u32, u32, p, p, pp], i32),
        "fc_graph_free": ([p], None),
        "fc_graph_n": ([p], u32),
        "fc_graph_layers": ([p], u32),
        "fc_graph_layer_m": ([p, u32], u64),
        "fc_graph_id2vtx": ([p, p], i32),
        "fc_graph_order": ([p, p], i32),
        "fc_graph_csr": ([p, p, p], i32),
        "fc_graph_upload": ([p, p], i32),
        "fc_graph_release_device": ([p], i32),
        "fc_graph_reset_results": ([p], i32),
        "fc_graph_device_bytes": ([p], u64),
        "fc_coreindex": ([p, p, i32, p], i32),
        "fc_densest": ([p, p, u32, p, p], i32),
        "fc_coreindex_densest": ([p, p, p, u32, p, p], i32),
        "fc_densest_members": ([p, p, p, p, p], i32),
        "fc_cell_members": ([p, u32, u32, p, u32, C.POINTER(u32), p], i32),
        "fc_cells": ([p, C.c_double, p, u32, C.POINTER(u32), p], i32),
        "fc_coreindex_range": ([p, u32, u32, p, i32, p], i32),
        "fc_cells_range": ([p, u32, u32, C.c_double, p, u32, C.POINTER(u32), p], i32),
        "fc_batch_run": ([p, u32, C.c_double, p, p, p, p, p], i32),
        "fc_server_create": ([p, pp], i32),
        "fc_server_submit": ([p, p, C.c_double, p, p, C.POINTER(u64)], i32),
        "fc_server_wait": ([p, u64, C.c_int64, C.POINTER(i32), C.POINTER(C.c_double)], i32),
        "fc_server_query": ([p, p], i32),
        "fc_server_destroy": ([p], i32),
        "fc_graph_stats": ([p, p], i32),
        "fc_launch_count": ([], u64),
        "fc_coreindex_fixed_scratch": ([u32, u32, u64, p, p, p, p, p], i32),
        "fc_cell_index": ([p, p, p, p, u64, C.POINTER(u64), p], i32),
        "fc_cells_members": ([p, p, p, u32, i32, p, p, u64, p], i32),
        "fc_mlcd_query": ([p, u32, u32, p, p, u32, p, p, u64, p], i32),
        "fc_probe_atomics": ([u64, u64, C.POINTER(C.c_double), p], i32),
        "fc_alloc_count": ([], u64),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(code, what):
    if code != FC_OK:
        raise FcError(what, code)


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def stream_handle(stream):
    """cudaStream_t as an int: None -> default stream; accepts torch.cuda.Stream."""
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))
