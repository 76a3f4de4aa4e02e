"""Parity of the CUDA path (through the C ABI) with the reference.

Golden fixtures were produced by the reference's own code; random cases are
checked against the oracle (pinned to the reference by test_oracle_golden).
Integer results (core tables, cells, node and layer sets) must be
bit-identical; so must the FP64 densities, since the device evaluates the
reference's expression in the same IEEE order (tolerance 0)."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

import golden_cases as G
import oracle as O
from pargridcpu_b200 import MultilayerGraph, native, synth

pytestmark = pytest.mark.gpu


def _check_all(g, exp, betas=G.BETAS, oracle_graph=None):
    table = g.coreindex()
    assert np.array_equal(table, exp["table"])
    res = g.densest(betas)
    for beta, r in zip(betas, res):
        tag = f"b{beta}"
        k, lmd, length = (int(x) for x in exp[f"{tag}_result"])
        assert (r["k"], r["lmd"], r["length"]) == (k, lmd, length), (beta, r)
        assert np.float32(r["max_density_f"]) == exp[f"{tag}_maxf"]
        rec, dens = g.cells(beta)
        assert np.array_equal(rec, exp[f"{tag}_cells"])
        assert np.array_equal(dens, exp[f"{tag}_cell_density"])
        if k:
            i = [j for j, c in enumerate(exp[f"{tag}_cells"]) if c[0] == k and c[1] == lmd][0]
            assert r["density"] == exp[f"{tag}_cell_density"][i]
            assert r["lstar"] == exp[f"{tag}_cells"][i][3]
            nodes, layers = g.densest_members(r)
            assert np.array_equal(nodes, exp[f"{tag}_nodes"])
            if oracle_graph is not None:
                o = oracle_graph.densest(table, beta, with_cells=False)
                assert np.array_equal(layers, o["layers"])
    return table


@pytest.mark.parametrize("name", G.SYNTH)
def test_golden_synth(name):
    layers = G.inputs(name)
    g = MultilayerGraph.from_pairs(layers)
    _check_all(g, G.expected(name), oracle_graph=O.OracleGraph(layers))


@pytest.mark.parametrize("name", G.TEXT)
def test_golden_text(name):
    exp = G.expected(name)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "mlg.conf"), "w") as f:
            f.write("".join(f"l{i}.txt\n" for i in range(len(G.texts(name)))))
        for i, t in enumerate(G.texts(name)):
            with open(os.path.join(d, f"l{i}.txt"), "w", newline="") as f:
                f.write(t)
        g = MultilayerGraph.LoadFromFile(d)
        if g.n:
            _check_all(g, exp)


RANDOM = [
    ("cl_L1", lambda: synth.chung_lu_graph(3000, 1, 9000, 2.2, 0.0, 71)),
    ("cl_L3_hubs", lambda: synth.chung_lu_graph(20000, 3, 80000, 2.02, 0.5, 72)),
    # cores up to 69, 392 rows over 512 entries: ordered rows, pruned and
    # strided chunk visits
    ("cl_deep", lambda: synth.chung_lu_graph(30000, 4, 240000, 2.1, 0.5, 9092)),
    ("cl_L12", lambda: synth.chung_lu_graph(5000, 12, 12000, 2.5, 0.4, 73)),
    ("er_L40", lambda: synth.erdos_renyi_graph(150, 40, 0.01, 0.08, 74)),
    ("er_L600", lambda: synth.erdos_renyi_graph(60, 600, 0.02, 0.1, 75)),
    ("dirty", lambda: synth.chung_lu_graph(2000, 5, 6000, 2.3, 0.3, 76, dirty=True)),
]


@pytest.mark.parametrize("name,make", RANDOM, ids=[r[0] for r in RANDOM])
def test_random_vs_oracle(name, make):
    gen = make()
    og = O.OracleGraph(gen.layers)
    ref = og.coreindex()
    g = MultilayerGraph.from_pairs(gen.layers)
    table = g.coreindex()
    assert np.array_equal(table, ref)
    for beta in (0.5, 1.0, 2.0):
        o = og.densest(ref, beta)
        r = g.densest([beta])[0]
        assert (r["k"], r["lmd"], r["length"], r["lstar"]) == (o["k"], o["lmd"], o["length"],
                                                                o["lstar"])
        assert r["density"] == o["density"]
        assert np.float32(r["max_density_f"]) == np.float32(o["max_density_f"])
        rec, dens = g.cells(beta)
        assert np.array_equal(rec, o["cells"]) and np.array_equal(dens, o["cell_density"])
        nodes, layers = g.densest_members(r)
        assert np.array_equal(nodes, o["nodes"]) and np.array_equal(layers, o["layers"])


@pytest.mark.parametrize("name", ["cl_L3_hubs", "cl_deep", "cl_L12"])
def test_endgame_on_and_off_agree(name, monkeypatch):
    """The three ways a single graph is peeled give the oracle's table: the
    default (the whole graph per column on a block or a cluster when it fits
    one), the grid-wide peel followed by the endgame on the survivors'
    subgraph, and the grid-wide peel alone."""
    gen = dict(RANDOM)[name]()
    ref = O.OracleGraph(gen.layers).coreindex()
    default = MultilayerGraph.from_pairs(gen.layers).coreindex()
    monkeypatch.setenv("FC_PEEL_WHOLE", "0")
    with_eg = MultilayerGraph.from_pairs(gen.layers).coreindex()
    monkeypatch.setenv("FC_PEEL_ENDGAME", "0")
    without = MultilayerGraph.from_pairs(gen.layers).coreindex()
    assert np.array_equal(default, ref)
    assert np.array_equal(with_eg, ref) and np.array_equal(without, ref)


def test_repeatable_and_reset():
    gen = synth.chung_lu_graph(30000, 4, 60000, 2.1, 0.5, 81)
    g = MultilayerGraph.from_pairs(gen.layers)
    a = g.coreindex()
    g.reset_results()
    b = g.coreindex()
    g.release_device()
    c = g.coreindex()
    assert np.array_equal(a, b) and np.array_equal(a, c)
    st = g.stats()
    assert st["peel_launches"] >= 1 and st["peel_ms"] > 0


def test_device_output():
    import torch
    gen = synth.chung_lu_graph(5000, 3, 12000, 2.3, 0.3, 82)
    g = MultilayerGraph.from_pairs(gen.layers)
    out = torch.zeros((g.L, g.n), dtype=torch.int32, device="cuda")
    g.coreindex(out=out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), g.coreindex())


def test_empty_and_edge_cases():
    # no edges at all (only self-loops): n = 0
    g = MultilayerGraph.from_pairs([np.array([[3, 3]], np.uint32)])
    assert g.n == 0
    assert g.coreindex().shape == (1, 0)
    assert g.densest([1.0])[0]["k"] == 0
    # one edge
    g = MultilayerGraph.from_pairs([np.array([[1, 2]], np.uint32), np.zeros((0, 2), np.uint32)])
    assert np.array_equal(g.coreindex(), np.array([[1, 1], [0, 0]], np.uint32))
    r = g.densest([1.0])[0]
    assert (r["k"], r["lmd"], r["length"]) == (1, 1, 2)


C3_FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "c3.npz")


@pytest.mark.skipif(not os.path.exists(C3_FIXTURE), reason="c3 fixture not generated")
@pytest.mark.parametrize("name", ["c1", "layers33", "hubs"])
def test_cell_members(name):
    """Any cell's node set from the device table equals {v : core >= k} of
    the reference's table, for k across the column's range and beyond."""
    exp = G.expected(name)["table"]
    g = MultilayerGraph.from_pairs(G.inputs(name))
    for lmd in sorted({1, 2, g.L // 2 + 1, g.L}):
        col = exp[lmd - 1]
        kmax = int(col.max())
        for k in sorted({0, 1, kmax // 2, kmax, kmax + 1}):
            want = np.nonzero(col >= k)[0].astype(np.uint32)
            assert np.array_equal(g.cell_members(k, lmd), want), (lmd, k)
    with pytest.raises(native.FcError):
        g.cell_members(1, g.L + 1)


def test_deadline_ends_the_run_with_an_error_and_the_device_stays_usable(monkeypatch):
    """Every wait and loop of the grid-wide peel kernel is bounded by the
    run's deadline: a run past it ends with an error status (no fault, no
    trap), and the next call on the same context gets the reference's table.
    (c1 would otherwise be peeled on thread-block clusters, whole graph per
    column, without the grid-wide kernel.)"""
    g = MultilayerGraph.from_pairs(G.inputs("c1"))
    monkeypatch.setenv("FC_PEEL_WHOLE", "0")
    monkeypatch.setenv("FC_PEEL_DEADLINE_MS", "0")
    with pytest.raises(native.FcError) as e:
        g.coreindex()
    assert e.value.code == 6  # FC_ERR_ITER_LIMIT
    monkeypatch.delenv("FC_PEEL_DEADLINE_MS")
    assert np.array_equal(g.coreindex(), G.expected("c1")["table"])
    monkeypatch.delenv("FC_PEEL_WHOLE")
    g.reset_results()
    assert np.array_equal(g.coreindex(), G.expected("c1")["table"])


def test_c3_full_size():
    """The 2.5M-node, 34M-edge, 4-layer configuration at full size: table hash
    and densest results against the reference's own output."""
    exp = dict(np.load(C3_FIXTURE))
    man = G.MANIFEST["c3"]
    gen = synth.config_graph("c3")
    assert G.pairs_sha(gen.layers) == man["pairs_sha256"]
    g = MultilayerGraph.from_pairs(gen.layers)
    table = g.coreindex()
    assert hashlib.sha256(np.ascontiguousarray(table).tobytes()).hexdigest() == man["table_sha256"]
    # size-independent properties too
    assert np.all(table[1:] <= table[:-1])
    for beta in G.BETAS:
        tag = f"b{beta}"
        r = g.densest([beta])[0]
        k, lmd, length = (int(x) for x in exp[f"{tag}_result"])
        assert (r["k"], r["lmd"], r["length"]) == (k, lmd, length)
        assert np.float32(r["max_density_f"]) == exp[f"{tag}_maxf"]
        rec, dens = g.cells(beta)
        assert np.array_equal(rec, exp[f"{tag}_cells"])
        assert np.array_equal(dens, exp[f"{tag}_cell_density"])
        nodes, _ = g.densest_members(r)
        assert np.array_equal(nodes, exp[f"{tag}_nodes"])


def test_c5_large_graph():
    """The serving configuration's large graph (2.6M nodes, 24 layers, 48M
    edges, the first seed the serving benchmark draws): table hash, per-lambda
    maxima and densest result against the reference's own output
    (tests/golden/c5_large.json); containment across lambda holds."""
    import json
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c5_large.json")))
    f = fx["graph"]
    gen = synth._make(fx["params"])
    assert G.pairs_sha(gen.layers) == f["pairs_sha256"]
    g = MultilayerGraph.from_pairs(gen.layers)
    assert (g.n, g.L) == (f["n"], f["L"])
    table = g.coreindex()
    assert [int(x) for x in table.max(axis=1)] == f["kmax"]
    assert hashlib.sha256(np.ascontiguousarray(table).tobytes()).hexdigest() == f["table_sha256"]
    assert np.all(table[1:] <= table[:-1])
    r = g.densest([fx["beta"]])[0]
    assert (r["k"], r["lmd"], r["length"], r["lstar"]) == (f["k"], f["lmd"], f["length"], f["lstar"])
    assert r["density"] == f["density"]
    assert np.float32(r["max_density_f"]) == np.float32(f["max_density_f"])
    nodes, _ = g.densest_members(r)
    assert hashlib.sha256(np.ascontiguousarray(nodes, dtype="<u4").tobytes()).hexdigest() == \
        f["nodes_sha256"]


@pytest.mark.parametrize("name", ["c1", "layers33", "mix0", "hubs"])
@pytest.mark.parametrize("pinned", [True, False])
def test_coreindex_densest_in_one_call(name, pinned):
    """fc_coreindex_densest: the table and every beta's result equal the
    separate calls' (and the reference's), whether the table's copy overlaps
    the densest search (pinned buffer) or precedes it (pageable buffer)."""
    import torch

    exp = G.expected(name)
    g = MultilayerGraph.from_pairs(G.inputs(name))
    if pinned:
        out = torch.zeros((g.L, g.n), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    else:
        out = np.zeros((g.L, g.n), np.uint32)
    table, res = g.coreindex_densest(out, G.BETAS)
    assert table is out
    assert np.array_equal(table, exp["table"])
    g2 = MultilayerGraph.from_pairs(G.inputs(name))
    sep = g2.densest(G.BETAS)
    assert np.array_equal(g2.coreindex(), exp["table"])
    for beta, r, s in zip(G.BETAS, res, sep):
        assert r == s, beta
        k, lmd, length = (int(x) for x in exp[f"b{beta}_result"])
        assert (r["k"], r["lmd"], r["length"]) == (k, lmd, length), (beta, r)
    # a second call on the resident table peels nothing and gives the same
    out2 = np.zeros_like(out)
    table2, res2 = g.coreindex_densest(out2, G.BETAS)
    assert np.array_equal(table2, table) and res2 == res
