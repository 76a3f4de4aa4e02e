"""B200 FirmCore engine: the (k, lambda)-core index of every node over the whole
fcgrid and the per-cell densest-subgraph search, for multilayer graphs.

Python mirror of the reference's host interface (kouteisang/ParGridCPU):

* ``MultilayerGraph`` -- Graph/MultilayerGraph.h: ``LoadFromFile``,
  ``SetGraphOrder`` (via ``order=``), ``GetN``, ``getLayerNumber``,
  ``LoadId2VtxMap``, ``PrintStatistics``.
* ``CoreIndex.Execute / ExecuteParallel`` (CoreIndexParallel/CoreIndex.h:15-17)
  and ``FCSyncLeft.Execute / ExecuteMix`` (CoreParallel/FCSyncLeft.h:18,34):
  the full core table, ``table[lambda-1, v] = core_lambda(v)``.
* ``FCPathLevelLeft.Execute(mg, wds=True, beta)`` + ``WeightDenestSubgraph``
  (Core/FCPathLevelLeft.h:14, Core/FCTree.h:66): the densest subgraph.

Everything runs through the C ABI of ``libfirmcore.so`` on one CUDA device;
there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import native as _n

__all__ = ["MultilayerGraph", "CoreIndex", "FCSyncLeft", "FCPathLevelLeft", "batch_run",
           "Server", "build", "FcError", "launch_count", "mlcd_query"]

FcError = _n.FcError
HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8):
    """Compile libfirmcore.so and the CLI in place (sm_100a)."""
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"], check=True)


class MultilayerGraph:
    """A multilayer graph handle (host CSR; device CSR once uploaded)."""

    def __init__(self, handle):
        self._h = handle

    # -- construction (MultilayerGraph::LoadFromFile and friends) --
    @classmethod
    def LoadFromFile(cls, path, order=0, write_vtx_map=True):
        h = C.c_void_p()
        _n.check(_n.lib().fc_graph_load_dir(os.fsencode(path), int(order), int(write_vtx_map),
                                            C.byref(h)), f"load {path}")
        return cls(h)

    @classmethod
    def from_pairs(cls, layers):
        """``layers``: per-layer (m, 2) arrays of raw (u, v) ids in file order."""
        m = np.array([len(e) for e in layers], dtype=np.uint64)
        flat = (np.ascontiguousarray(np.concatenate(
            [np.ascontiguousarray(e, dtype=np.uint32).reshape(-1) for e in layers]))
            if len(layers) else np.zeros(0, np.uint32))
        h = C.c_void_p()
        _n.check(_n.lib().fc_graph_from_pairs(len(layers), _n.ptr(m), _n.ptr(flat), C.byref(h)),
                 "from_pairs")
        return cls(h)

    @classmethod
    def from_adjbuf(cls, n, bufs):
        """``bufs``: per-layer arrays in Graph::adj_lst_buf form ([deg, nbrs...] per node)."""
        keep = [np.ascontiguousarray(b, dtype=np.uint32) for b in bufs]
        arr = (C.c_void_p * max(len(keep), 1))(*[b.ctypes.data for b in keep])
        m = np.array([len(b) - n for b in keep], dtype=np.uint64)
        h = C.c_void_p()
        _n.check(_n.lib().fc_graph_from_adjbuf(n, len(keep), C.cast(arr, C.c_void_p), _n.ptr(m),
                                               C.byref(h)), "from_adjbuf")
        return cls(h)

    def free(self):
        if self._h:
            _n.lib().fc_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- accessors --
    @property
    def handle(self):
        return self._h

    @property
    def n(self):
        return _n.lib().fc_graph_n(self._h)

    @property
    def L(self):
        return _n.lib().fc_graph_layers(self._h)

    def GetN(self):
        return self.n

    def getLayerNumber(self):
        return self.L

    def layer_m(self):
        return np.array([_n.lib().fc_graph_layer_m(self._h, l) for l in range(self.L)], np.uint64)

    def id2vtx(self):
        out = np.zeros(self.n, np.uint64)
        _n.check(_n.lib().fc_graph_id2vtx(self._h, _n.ptr(out)), "id2vtx")
        return out

    LoadId2VtxMap = id2vtx

    def order(self):
        out = np.zeros(self.L, np.uint32)
        _n.check(_n.lib().fc_graph_order(self._h, _n.ptr(out)), "order")
        return out

    def csr(self):
        n, L = self.n, self.L
        m = self.layer_m()
        off = np.zeros(L * (n + 1), np.uint64)
        adj = np.zeros(int(m.sum()) + 1, np.uint32)
        _n.check(_n.lib().fc_graph_csr(self._h, _n.ptr(off), _n.ptr(adj)), "csr")
        return off.reshape(L, n + 1), adj[:-1]

    def PrintStatistics(self):
        m = (self.layer_m() >> 1).astype(np.uint64)
        s = f"|L| = {self.L}, |V| = {self.n}, |E| = {int(m.sum()) & 0xFFFFFFFF}, " \
            f"max_|E_i| = {int(m.max(initial=0))}"
        print(s)
        return s

    # -- device --
    def upload(self, stream=None):
        _n.check(_n.lib().fc_graph_upload(self._h, _n.stream_handle(stream)), "upload")

    def release_device(self):
        _n.check(_n.lib().fc_graph_release_device(self._h), "release_device")

    def reset_results(self):
        _n.check(_n.lib().fc_graph_reset_results(self._h), "reset_results")

    def stats(self):
        st = _n.Stats()
        _n.check(_n.lib().fc_graph_stats(self._h, C.byref(st)), "stats")
        return st.as_dict()

    def device_bytes(self):
        return _n.lib().fc_graph_device_bytes(self._h)

    # -- compute --
    def coreindex(self, out=None, stream=None, copy=True):
        """The L x n core table (uint32); ``out`` may be a host numpy array or
        a CUDA torch tensor (then the copy stays on the device, asynchronous).
        With copy=False the table is only computed (it stays resident)."""
        n, L = self.n, self.L
        if not copy:
            _n.check(_n.lib().fc_coreindex(self._h, None, 0, _n.stream_handle(stream)),
                     "coreindex")
            return None
        if out is None:
            out = np.zeros((L, n), np.uint32)
        if hasattr(out, "data_ptr"):  # torch tensor on the device
            _n.check(_n.lib().fc_coreindex(self._h, C.c_void_p(out.data_ptr()), 1,
                                           _n.stream_handle(stream)), "coreindex")
        else:
            _n.check(_n.lib().fc_coreindex(self._h, _n.ptr(out), 0, _n.stream_handle(stream)),
                     "coreindex")
        return out

    def densest(self, betas=(1.0,), stream=None):
        betas = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, np.float64)))
        res = (_n.DensestResult * len(betas))()
        _n.check(_n.lib().fc_densest(self._h, _n.ptr(betas), len(betas), C.cast(res, C.c_void_p),
                                     _n.stream_handle(stream)), "densest")
        return [r.as_dict() for r in res]

    def coreindex_densest(self, out=None, betas=(1.0,), stream=None):
        """The L x n core table into host memory (``out``, a new array when
        None) and the densest results for ``betas``, in one call: with a
        pinned ``out`` the table's copy overlaps the densest search.
        Returns (table, results)."""
        if out is None:
            out = np.zeros((self.L, self.n), np.uint32)
        betas = np.ascontiguousarray(np.atleast_1d(np.asarray(betas, np.float64)))
        res = (_n.DensestResult * len(betas))()
        _n.check(_n.lib().fc_coreindex_densest(self._h, _n.ptr(out), _n.ptr(betas), len(betas),
                                               C.cast(res, C.c_void_p),
                                               _n.stream_handle(stream)), "coreindex_densest")
        return out, [r.as_dict() for r in res]

    def densest_members(self, result):
        r = _n.DensestResult(**{k: result[k] for k, _ in _n.DensestResult._fields_})
        nodes = np.zeros(max(r.length, 1), np.uint32)
        layers = np.zeros(max(r.lstar, 1), np.uint32)
        _n.check(_n.lib().fc_densest_members(self._h, C.byref(r), _n.ptr(nodes), _n.ptr(layers),
                                             None), "densest_members")
        return nodes[:r.length], layers[:r.lstar]

    def cell_members(self, k, lmd, stream=None):
        """C_{k,lmd} = {v : core_lmd(v) >= k}, ascending internal ids (the
        `-m kpe -k -lmd` query, FCTree::saveCoreToLocal)."""
        nodes = np.zeros(max(self.n, 1), np.uint32)
        cnt = C.c_uint32()
        _n.check(_n.lib().fc_cell_members(self._h, int(k), int(lmd), _n.ptr(nodes), self.n,
                                          C.byref(cnt), _n.stream_handle(stream)), "cell_members")
        return nodes[:cnt.value].copy()

    def cell_index(self, stream=None):
        """Every cell as a prefix (the compact form of -m CoreMem / PathMem):
        (order, col_off, sizes) -- order[lambda-1] is column lambda's nodes by
        descending core, ids ascending within a core; C_{k,lambda} is
        order[lambda-1][:sizes[col_off[lambda-1] + k]]."""
        n, L = self.n, self.L
        off = np.zeros(L + 1, np.uint64)
        cnt = C.c_uint64()
        _n.check(_n.lib().fc_cell_index(self._h, None, _n.ptr(off), None, 0, C.byref(cnt),
                                        _n.stream_handle(stream)), "cell_index")
        order = np.zeros((L, n), np.uint32)
        sizes = np.zeros(max(cnt.value, 1), np.uint32)
        _n.check(_n.lib().fc_cell_index(self._h, _n.ptr(order), _n.ptr(off), _n.ptr(sizes),
                                        cnt.value, C.byref(cnt), _n.stream_handle(stream)),
                 "cell_index")
        return order, off, sizes[:cnt.value]

    def cells_members(self, ks, lmds, by_index=False, stream=None):
        """Many cells at once (-m CoreIndexTimeOnline / Offline): one array of
        node ids per query (k, lmd); ascending ids, or with by_index=True each
        cell's prefix of the cell index order."""
        ks = np.ascontiguousarray(np.asarray(ks, dtype=np.uint32))
        lmds = np.ascontiguousarray(np.asarray(lmds, dtype=np.uint32))
        nq = len(ks)
        off = np.zeros(nq + 1, np.uint64)
        h = _n.stream_handle(stream)
        _n.check(_n.lib().fc_cells_members(self._h, _n.ptr(ks), _n.ptr(lmds), nq, int(by_index),
                                           _n.ptr(off), None, 0, h), "cells_members")
        nodes = np.zeros(max(int(off[-1]), 1), np.uint32)
        _n.check(_n.lib().fc_cells_members(self._h, _n.ptr(ks), _n.ptr(lmds), nq, int(by_index),
                                           _n.ptr(off), _n.ptr(nodes), int(off[-1]), h),
                 "cells_members")
        return [nodes[off[i]:off[i + 1]].copy() for i in range(nq)]

    def coreindex_range(self, lmd_lo, lmd_hi, out=None, stream=None, copy=True):
        """Columns lmd_lo .. lmd_hi-1 of the core table, (lmd_hi - lmd_lo, n):
        one process's share when a graph is split by lambda range.  With
        copy=False the columns are only computed (they stay resident)."""
        h = _n.stream_handle(stream)
        if not copy:
            _n.check(_n.lib().fc_coreindex_range(self._h, int(lmd_lo), int(lmd_hi), None, 0, h),
                     "coreindex_range")
            return None
        if out is None:
            out = np.zeros((lmd_hi - lmd_lo, self.n), np.uint32)
        _n.check(_n.lib().fc_coreindex_range(self._h, int(lmd_lo), int(lmd_hi), _n.ptr(out), 0,
                                             h), "coreindex_range")
        return out

    def cells_range(self, lmd_lo, lmd_hi, beta=1.0, stream=None):
        """The cells of lambda lmd_lo .. lmd_hi-1 as (k, lmd, length, lstar,
        density) tuples, the form shard.merge_cells folds."""
        cnt = C.c_uint32()
        h = _n.stream_handle(stream)
        _n.check(_n.lib().fc_cells_range(self._h, int(lmd_lo), int(lmd_hi), float(beta), None, 0,
                                         C.byref(cnt), h), "cells_range")
        buf = (_n.Cell * max(cnt.value, 1))()
        _n.check(_n.lib().fc_cells_range(self._h, int(lmd_lo), int(lmd_hi), float(beta),
                                         C.cast(buf, C.c_void_p), cnt.value, C.byref(cnt), h),
                 "cells_range")
        return [(int(c.k), int(c.lmd), int(c.length), int(c.lstar), float(c.density))
                for c in buf[:cnt.value]]

    def cells(self, beta=1.0):
        cnt = C.c_uint32()
        _n.check(_n.lib().fc_cells(self._h, float(beta), None, 0, C.byref(cnt), None), "cells")
        buf = (_n.Cell * max(cnt.value, 1))()
        _n.check(_n.lib().fc_cells(self._h, float(beta), C.cast(buf, C.c_void_p), cnt.value,
                                   C.byref(cnt), None), "cells")
        rec = np.array([(c.k, c.lmd, c.length, c.lstar) for c in buf[:cnt.value]],
                       np.uint32).reshape(-1, 4)
        dens = np.array([c.density for c in buf[:cnt.value]], np.float64)
        return rec, dens


class CoreIndex:
    """CoreIndex::Execute / ExecuteParallel: the per-lambda core index table."""

    @staticmethod
    def Execute(mg: MultilayerGraph, id2vtx=None):
        return mg.coreindex()

    ExecuteParallel = Execute


class FCSyncLeft:
    """ParGrid / ParGridPlus: the same table."""

    @staticmethod
    def Execute(mg: MultilayerGraph, tree=None):
        return mg.coreindex()

    ExecuteMix = Execute


class FCPathLevelLeft:
    """WdsList: densest subgraph over the fcgrid cells."""

    @staticmethod
    def Execute(mg: MultilayerGraph, tree=None, wds=True, beta=1.0):
        return mg.densest([beta])[0] if wds else mg.coreindex()


def mlcd_query(cores, ks, lmds, stream=None):
    """The membership test of -m MLCDTime (checktime) on an (n, P) matrix of
    per-node coreness values: one ascending id array per query (k, lmd)."""
    cores = np.ascontiguousarray(cores, dtype=np.uint32)
    n, P = cores.shape
    ks = np.ascontiguousarray(np.asarray(ks, dtype=np.uint32))
    lmds = np.ascontiguousarray(np.asarray(lmds, dtype=np.uint32))
    nq = len(ks)
    off = np.zeros(nq + 1, np.uint64)
    h = _n.stream_handle(stream)
    _n.check(_n.lib().fc_mlcd_query(_n.ptr(cores), n, P, _n.ptr(ks), _n.ptr(lmds), nq,
                                    _n.ptr(off), None, 0, h), "mlcd_query")
    nodes = np.zeros(max(int(off[-1]), 1), np.uint32)
    _n.check(_n.lib().fc_mlcd_query(_n.ptr(cores), n, P, _n.ptr(ks), _n.ptr(lmds), nq,
                                    _n.ptr(off), _n.ptr(nodes), int(off[-1]), h), "mlcd_query")
    return [nodes[off[i]:off[i + 1]].copy() for i in range(nq)]


def probe_atomics(buffer_bytes, ops=1 << 28, stream=None):
    """Returned-value 4-byte atomic subtractions per second (1e9/s) at random
    addresses of a device buffer of ``buffer_bytes`` (fc_probe_atomics)."""
    r = C.c_double()
    _n.check(_n.lib().fc_probe_atomics(int(buffer_bytes), int(ops), C.byref(r),
                                       _n.stream_handle(stream)), "probe_atomics")
    return r.value


def launch_count():
    """Kernels libfirmcore has launched in this process."""
    return int(_n.lib().fc_launch_count())


def batch_run(graphs, beta=1.0, want_tables=True, block_threads=0, hub_threshold=0,
              use_cuda_graph=True, plain=False, stream=None):
    """Every (graph, lambda) column of many graphs in one batched launch plus
    the densest search (``plain=True``: the one-column-per-launch baseline);
    returns (tables, results, report)."""
    cnt = len(graphs)
    hs = (C.c_void_p * max(cnt, 1))(*[g.handle.value for g in graphs])
    tables = [np.zeros((g.L, g.n), np.uint32) for g in graphs] if want_tables else None
    tp = (C.c_void_p * max(cnt, 1))(*[t.ctypes.data for t in tables]) if want_tables else None
    res = (_n.DensestResult * max(cnt, 1))()
    opt = _n.BatchOptions(block_threads, hub_threshold, int(use_cuda_graph), int(plain))
    rep = _n.BatchReport()
    _n.check(_n.lib().fc_batch_run(C.cast(hs, C.c_void_p), cnt, float(beta),
                                   C.cast(tp, C.c_void_p) if tp is not None else None,
                                   C.cast(res, C.c_void_p), C.byref(opt), C.byref(rep),
                                   _n.stream_handle(stream)), "batch_run")
    return tables, [r.as_dict() for r in res[:cnt]], rep.as_dict()


class Server:
    """Continuous-batching request loop (fc_server_*): requests queue in
    arrival order, free lanes take every pending request that fits the
    device-memory budget as one batch; heavy requests run alone on three
    quarters of the SMs while light batches share the rest, so their work
    overlaps on the device.  ``plain=True`` is the one-at-a-time baseline."""

    def __init__(self, hbm_budget_bytes=0, max_inflight=0, lanes=0, max_batch_graphs=0,
                 block_threads=0, hub_threshold=0, plain=False, heavy_visits=0):
        opt = _n.ServerOptions(hbm_budget_bytes, max_inflight, lanes, max_batch_graphs,
                               block_threads, hub_threshold, int(plain), heavy_visits)
        h = C.c_void_p()
        _n.check(_n.lib().fc_server_create(C.byref(opt), C.byref(h)), "server_create")
        self._h = h
        self._keep = {}

    def submit(self, mg: MultilayerGraph, beta=1.0, want_table=True):
        """Queues a decomposition + densest request; returns its ticket."""
        table = np.zeros((mg.L, mg.n), np.uint32) if want_table else None
        res = _n.DensestResult()
        t = C.c_uint64()
        _n.check(_n.lib().fc_server_submit(self._h, mg.handle, float(beta), _n.ptr(table),
                                           C.byref(res), C.byref(t)), "server_submit")
        self._keep[t.value] = (mg, table, res)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """(table, densest result, latency ms) of a ticket; raises FcError with
        the request's own status when it failed."""
        st = C.c_int()
        lat = C.c_double()
        _n.check(_n.lib().fc_server_wait(self._h, ticket, timeout_ms, C.byref(st), C.byref(lat)),
                 "server_wait")
        mg, table, res = self._keep.pop(ticket)
        _n.check(st.value, "request")
        return table, res.as_dict(), lat.value

    def stats(self):
        out = _n.ServerStats()
        _n.check(_n.lib().fc_server_query(self._h, C.byref(out)), "server_query")
        return out.as_dict()

    def close(self):
        if self._h:
            _n.check(_n.lib().fc_server_destroy(self._h), "server_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
