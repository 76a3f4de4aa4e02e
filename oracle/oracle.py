"""Test infrastructure, not product code: ctypes access to the CPU oracle.

Wraps ``liboracle.so`` (the plain-C restatement of the reference's hot path,
``firmcore_oracle.c``) and the reference checker ``_ref/ref_harness`` (the
reference's own sources compiled in place).  Only the tests, the smoke check
and the benchmark's CPU-baseline leg import this module, and only as the
checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
HARNESS = os.path.join(HERE, "_ref", "ref_harness")


class Cell(C.Structure):
    _fields_ = [("k", C.c_uint32), ("lmd", C.c_uint32), ("length", C.c_uint32),
                ("lstar", C.c_uint32), ("density", C.c_double)]


class DensestResult(C.Structure):
    _fields_ = [("max_density_f", C.c_float), ("density", C.c_double), ("k", C.c_uint32),
                ("lmd", C.c_uint32), ("length", C.c_uint32), ("lstar", C.c_uint32),
                ("n_cells", C.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB_PATH)
        p = C.c_void_p
        L.oracle_graph_from_pairs.argtypes = [C.c_uint32, p, p, C.POINTER(C.c_void_p)]
        L.oracle_graph_free.argtypes = [p]
        L.oracle_n.argtypes = [p]
        L.oracle_n.restype = C.c_uint32
        L.oracle_layers.argtypes = [p]
        L.oracle_layers.restype = C.c_uint32
        L.oracle_layer_m.argtypes = [p, C.c_uint32]
        L.oracle_layer_m.restype = C.c_uint64
        L.oracle_id2vtx.argtypes = [p, p]
        L.oracle_csr.argtypes = [p, p, p]
        L.oracle_coreindex.argtypes = [p, p]
        L.oracle_densest.argtypes = [p, p, C.c_double, C.POINTER(DensestResult), p, C.c_uint32,
                                     p, p]
        for name in ("oracle_cells_scan", "oracle_cells_sorted"):
            f = getattr(L, name)
            f.argtypes = [p, C.c_uint32, C.c_uint32, p, p, C.c_uint32, p, p]
            f.restype = C.c_uint64
        L.oracle_mlcd_query.argtypes = [p, C.c_uint32, C.c_uint32, p, p, C.c_uint32, p, p]
        L.oracle_mlcd_query.restype = C.c_uint64
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def flatten_pairs(layers):
    m = np.array([len(e) for e in layers], dtype=np.uint64)
    flat = (np.concatenate([np.ascontiguousarray(e, dtype=np.uint32).reshape(-1) for e in layers])
            if len(layers) else np.zeros(0, np.uint32))
    return m, np.ascontiguousarray(flat, dtype=np.uint32)


class OracleGraph:
    """A graph loaded with the reference loader's semantics, on the CPU."""

    def __init__(self, layers):
        self._keep = flatten_pairs(layers)
        m, flat = self._keep
        h = C.c_void_p()
        if lib().oracle_graph_from_pairs(len(layers), _ptr(m), _ptr(flat), C.byref(h)) != 0:
            raise MemoryError("oracle graph build failed")
        self.h = h
        self.n = lib().oracle_n(h)
        self.L = lib().oracle_layers(h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_graph_free(self.h)
            self.h = None

    def id2vtx(self):
        out = np.zeros(self.n, np.uint64)
        lib().oracle_id2vtx(self.h, _ptr(out))
        return out

    def layer_m(self):
        return np.array([lib().oracle_layer_m(self.h, l) for l in range(self.L)], np.uint64)

    def csr(self):
        off = np.zeros(self.L * (self.n + 1), np.uint64)
        adj = np.zeros(int(self.layer_m().sum()) + 1, np.uint32)
        lib().oracle_csr(self.h, _ptr(off), _ptr(adj))
        return off.reshape(self.L, self.n + 1), adj[:-1]

    def coreindex(self):
        t = np.zeros((self.L, self.n), np.uint32)
        if self.n and lib().oracle_coreindex(self.h, _ptr(t)) != 0:
            raise MemoryError("oracle coreindex failed")
        return t

    def densest(self, table, beta, with_cells=True):
        table = np.ascontiguousarray(table, dtype=np.uint32)
        res = DensestResult()
        cap = int(table.max(initial=0)) * self.L + 1 if with_cells else 0
        cells = (Cell * max(cap, 1))()
        nodes = np.zeros(max(self.n, 1), np.uint32)
        layers = np.zeros(max(self.L, 1), np.uint32)
        lib().oracle_densest(self.h, _ptr(table), float(beta), C.byref(res),
                             C.cast(cells, C.c_void_p) if with_cells else None, cap,
                             _ptr(nodes), _ptr(layers))
        out = dict(max_density_f=res.max_density_f, density=res.density, k=res.k, lmd=res.lmd,
                   length=res.length, lstar=res.lstar, n_cells=res.n_cells,
                   nodes=nodes[:res.length].copy() if res.k else np.zeros(0, np.uint32),
                   layers=layers[:res.lstar].copy() if res.k else np.zeros(0, np.uint32))
        if with_cells:
            nc = min(res.n_cells, cap)
            out["cells"] = np.array([(cells[i].k, cells[i].lmd, cells[i].length, cells[i].lstar)
                                     for i in range(nc)], dtype=np.uint32).reshape(-1, 4)
            out["cell_density"] = np.array([cells[i].density for i in range(nc)], np.float64)
        return out


def _split(offsets, nodes):
    return [nodes[offsets[i]:offsets[i + 1]].copy() for i in range(len(offsets) - 1)]


def _queries(ks, lmds):
    ks = np.ascontiguousarray(np.asarray(ks, dtype=np.uint32))
    lmds = np.ascontiguousarray(np.asarray(lmds, dtype=np.uint32))
    return ks, lmds, len(ks)


def cells_scan(table, ks, lmds):
    """getResCore's answers (Util/CoreIndexTime.h:8-40): per query (k, lmd)
    the nodes with core_lmd >= k, ascending ids."""
    table = np.ascontiguousarray(table, dtype=np.uint32)
    L, n = table.shape
    ks, lmds, nq = _queries(ks, lmds)
    off = np.zeros(nq + 1, np.uint64)
    lib().oracle_cells_scan(_ptr(table), n, L, _ptr(ks), _ptr(lmds), nq, _ptr(off), None)
    nodes = np.zeros(int(off[-1]) + 1, np.uint32)
    lib().oracle_cells_scan(_ptr(table), n, L, _ptr(ks), _ptr(lmds), nq, _ptr(off), _ptr(nodes))
    return _split(off, nodes)


def cells_sorted(table, ks, lmds):
    """getResCoreOffline's answers (Util/CoreIndexTime.h:43-59 after the sort
    of main.cpp:567-572): by ascending core, ids ascending within a core."""
    table = np.ascontiguousarray(table, dtype=np.uint32)
    L, n = table.shape
    ks, lmds, nq = _queries(ks, lmds)
    off = np.zeros(nq + 1, np.uint64)
    lib().oracle_cells_sorted(_ptr(table), n, L, _ptr(ks), _ptr(lmds), nq, _ptr(off), None)
    nodes = np.zeros(int(off[-1]) + 1, np.uint32)
    lib().oracle_cells_sorted(_ptr(table), n, L, _ptr(ks), _ptr(lmds), nq, _ptr(off),
                              _ptr(nodes))
    return _split(off, nodes)


def mlcd_query(cores, ks, lmds):
    """checktime's answers (Util/CheckMLCDTime.h:9-42) over the (n, P)
    coreness matrix, ascending ids."""
    cores = np.ascontiguousarray(cores, dtype=np.uint32)
    n, P = cores.shape
    ks, lmds, nq = _queries(ks, lmds)
    off = np.zeros(nq + 1, np.uint64)
    lib().oracle_mlcd_query(_ptr(cores), n, P, _ptr(ks), _ptr(lmds), nq, _ptr(off), None)
    nodes = np.zeros(int(off[-1]) + 1, np.uint32)
    lib().oracle_mlcd_query(_ptr(cores), n, P, _ptr(ks), _ptr(lmds), nq, _ptr(off), _ptr(nodes))
    return _split(off, nodes)


# ---- the reference itself ---------------------------------------------------

def harness_available():
    return os.path.exists(HARNESS)


def run_harness(src, mode, *args, timeout=3600):
    """Run the reference checker on a dataset directory (ending in '/') or an
    FCG1 file; returns its stdout."""
    cmd = [HARNESS, src, mode] + [str(a) for a in args]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)
    return r.stdout


def ref_table(src, L, n, mode="table", threads=1):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "t.bin")
        run_harness(src, mode, out, *([threads] if threads > 1 or mode == "pgtable" else []))
        return np.fromfile(out, dtype=np.uint32).reshape(L, n)


def ref_wds(src, beta, threads=1):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "w.txt")
        run_harness(src, "wds", out, repr(float(beta)), threads)
        res = dict(cells=[], nodes=np.zeros(0, np.uint32))
        for line in open(out):
            f = line.split()
            if f[0] == "result":
                res.update(max_density_f=float(f[1]), k=int(f[2]), lmd=int(f[3]),
                           length=int(f[4]))
            elif f[0] == "cell":
                res["cells"].append((int(f[1]), int(f[2]), int(f[3]), float(f[4]), int(f[5])))
            elif f[0] == "nodes":
                res["nodes"] = np.array([int(x) for x in f[1:]], np.uint32)
        return res


# ---- the loader's text parse ------------------------------------------------

_WS = b" \t\n\v\f\r"


def parse_layer_text(data: bytes):
    """Raw (u, v) pairs exactly as MultilayerGraph::LoadLayer collects them
    (Graph/MultilayerGraph.cpp:122-156): ``while (in.peek() != EOF) { in >> u
    >> v; if (u != v) keep(u, v); }`` with ``uint u, v`` and C++11 iostream
    rules -- a failed extraction at end of input leaves the variable unchanged
    and fails the stream; one that reads no digit stores 0; an out-of-range
    value stores UINT_MAX; a leading '-' negates modulo 2^32.  A pair whose
    variables were never assigned (undefined in the reference) is dropped."""
    pos, n = 0, len(data)
    state = {"fail": False, "eof": False}
    u = v = None
    out = []

    def extract(val):
        nonlocal pos
        if state["fail"] or state["eof"]:
            state["fail"] = True
            return val
        while pos < n and data[pos] in _WS:
            pos += 1
        if pos >= n:
            state["eof"] = state["fail"] = True
            return val
        neg = False
        if data[pos] in b"+-":
            neg = data[pos] == 45
            pos += 1
        start = pos
        while pos < n and 48 <= data[pos] <= 57:
            pos += 1
        if pos >= n:
            state["eof"] = True
        if pos == start:
            state["fail"] = True
            return 0
        mag = int(data[start:pos])
        if mag > 0xFFFFFFFF:
            state["fail"] = True
            return 0xFFFFFFFF
        return (-mag) & 0xFFFFFFFF if neg else mag

    while True:
        if state["fail"] or state["eof"] or pos >= n:
            break
        u = extract(u)
        v = extract(v)
        if u is not None and v is not None and u != v:
            out.append((u, v))
    return np.array(out, dtype=np.uint32).reshape(-1, 2)
