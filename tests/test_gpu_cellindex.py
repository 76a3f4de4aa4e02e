"""Every cell at once on the GPU: the cell index (the compact form of every
cell, the counterpart of -m CoreMem / PathMem) and the batched cell queries
(-m CoreIndexTimeOnline / CoreIndexTimeOffline / MLCDTime), through the C
ABI, against the reference's own tables (golden fixtures) and the oracle's
restatements of getResCore, getResCoreOffline and checktime."""
import numpy as np
import pytest

import golden_cases as G
import oracle as O
from pargridcpu_b200 import FcError, MultilayerGraph, mlcd_query, synth

pytestmark = pytest.mark.gpu


def _check_index(g, table):
    order, off, sizes = g.cell_index()
    L, n = table.shape
    assert order.shape == (L, n) and len(off) == L + 1
    for l in range(L):
        col = table[l]
        kmax = int(col.max(initial=0))
        assert off[l + 1] - off[l] == kmax + 2
        # descending core, ascending ids within a core (a stable sort)
        want = np.argsort(-col.astype(np.int64), kind="stable")
        assert np.array_equal(order[l], want)
        s = sizes[off[l]:off[l + 1]]
        assert np.array_equal(s, [(col >= k).sum() for k in range(kmax + 2)])
    return order, off, sizes


def _queries(table, cells=None):
    L, n = table.shape
    ks, lmds = [], []
    if cells is not None:
        ks += [int(c[0]) for c in cells]
        lmds += [int(c[1]) for c in cells]
    for l in range(1, L + 1):
        km = int(table[l - 1].max(initial=0))
        ks += [0, 1, km, km + 1, km + 1000]
        lmds += [l] * 5
    return ks, lmds


@pytest.mark.parametrize("name", ["c1", "c2", "layers33", "mix0", "hubs", "tiny_dirty"])
def test_golden_cells_at_once(name):
    exp = G.expected(name)
    table = exp["table"]
    g = MultilayerGraph.from_pairs(G.inputs(name))
    order, off, sizes = _check_index(g, table)
    cells = exp["b1.0_cells"]
    for c in cells:  # every cell the reference reported, with its size
        assert sizes[off[c[1] - 1] + c[0]] == c[2]
    ks, lmds = _queries(table, cells)
    scan = g.cells_members(ks, lmds)
    want = O.cells_scan(table, ks, lmds)
    for a, b in zip(scan, want):
        assert np.array_equal(a, b)
    idx = g.cells_members(ks, lmds, by_index=True)
    srt = O.cells_sorted(table, ks, lmds)
    for a, b, k, lmd in zip(idx, want, ks, lmds):
        assert np.array_equal(a, order[lmd - 1][:len(b)])
        assert np.array_equal(np.sort(a), b)
    for a, b in zip(idx, srt):
        assert np.array_equal(np.sort(a), np.sort(b))


@pytest.mark.parametrize("make", [
    lambda: synth.chung_lu_graph(30000, 4, 240000, 2.1, 0.5, 9092),
    lambda: synth.erdos_renyi_graph(60, 600, 0.02, 0.1, 75),
    lambda: synth.chung_lu_graph(9000, 1, 30000, 2.2, 0.0, 71),
], ids=["cl_deep", "er_L600", "cl_L1"])
def test_random_cells_at_once(make):
    gen = make()
    table = O.OracleGraph(gen.layers).coreindex()
    g = MultilayerGraph.from_pairs(gen.layers)
    _check_index(g, table)
    rng = np.random.default_rng(3)
    L = table.shape[0]
    lmds = list(rng.integers(1, L + 1, size=200))
    ks = [int(rng.integers(0, table[l - 1].max() + 2)) for l in lmds]
    for by_index in (False, True):
        got = g.cells_members(ks, lmds, by_index=by_index)
        for a, b in zip(got, O.cells_scan(table, ks, lmds)):
            assert np.array_equal(np.sort(a) if by_index else a, b)


def test_index_follows_the_table():
    gen = synth.chung_lu_graph(6000, 5, 20000, 2.3, 0.4, 11)
    table = O.OracleGraph(gen.layers).coreindex()
    g = MultilayerGraph.from_pairs(gen.layers)
    g.coreindex_range(2, 4)            # a partial table first
    _check_index(g, table)             # the index peels the whole table
    g.reset_results()
    _check_index(g, table)             # and is rebuilt from the new one
    g.release_device()
    got = g.cells_members([3, 0], [1, 5], by_index=True)
    assert np.array_equal(np.sort(got[0]), np.nonzero(table[0] >= 3)[0])
    assert len(got[1]) == g.n


def test_invalid_lambda_is_refused():
    gen = synth.chung_lu_graph(500, 3, 1500, 2.3, 0.4, 12)
    g = MultilayerGraph.from_pairs(gen.layers)
    for lmd in (0, 4):
        with pytest.raises(FcError) as e:
            g.cells_members([1], [lmd])
        assert e.value.code == 7
    assert g.cells_members([], []) == []


def test_mlcd_query_matches_checktime():
    rng = np.random.default_rng(8)
    for n, P in ((5000, 7), (33, 1), (4097, 24)):
        cores = rng.integers(0, 40, size=(n, P)).astype(np.uint32)
        cores[::53, 0] = 0xFFFFFFFF
        nq = 60
        ks = list(rng.integers(0, 45, size=nq)) + [0, 0, 39]
        lmds = list(rng.integers(0, P + 2, size=nq)) + [0, P + 1, 1]
        got = mlcd_query(cores, ks, lmds)
        want = O.mlcd_query(cores, ks, lmds)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
