"""Batched decomposition (fc_batch_run): one persistent launch over many
graphs must give every graph exactly the table and densest result it gets
alone -- checked against the reference's golden outputs and the oracle, in
the batched form (with and without CUDA-graph capture, autotuned and with
fixed configurations) and in the plain one-column-per-launch form."""
import numpy as np
import pytest

import golden_cases as G
import oracle as O
from pargridcpu_b200 import MultilayerGraph, batch_run, synth

pytestmark = pytest.mark.gpu


def _batch_inputs():
    gens = [G.inputs(name) for name in ("mix0", "mix1", "mix2", "mix3", "tiny_dirty", "layers33")]
    gens += [synth.chung_lu_graph(800, 1, 2400, 2.2, 0.0, 301).layers,
             synth.chung_lu_graph(3000, 2, 6000, 2.4, 0.5, 302).layers,
             synth.erdos_renyi_graph(50, 40, 0.02, 0.1, 303).layers,
             synth.chung_lu_graph(12000, 7, 30000, 2.05, 0.3, 304).layers,
             [np.array([[1, 2]], np.uint32)]]
    gens += [g.layers for g in synth.batch_mix(count=10, seed=305, n_lo=500, n_hi=8000)]
    return gens


@pytest.fixture(scope="module")
def batch():
    layers = _batch_inputs()
    expected = []
    for ls in layers:
        og = O.OracleGraph(ls)
        t = og.coreindex()
        expected.append((t, og.densest(t, 1.0, with_cells=False)))
    return layers, expected


def _check(tables, results, expected):
    for i, ((t, o), got_t, r) in enumerate(zip(expected, tables, results)):
        assert np.array_equal(got_t, t), f"graph {i}: table"
        assert (r["k"], r["lmd"], r["length"], r["lstar"]) == (o["k"], o["lmd"], o["length"],
                                                                o["lstar"]), f"graph {i}"
        assert r["density"] == o["density"], f"graph {i}: density"
        assert np.float32(r["max_density_f"]) == np.float32(o["max_density_f"])


@pytest.mark.parametrize("mode", [
    dict(),                                                  # autotuned, CUDA graph
    dict(use_cuda_graph=False),
    dict(block_threads=1024, hub_threshold=16),
    dict(block_threads=512, hub_threshold=64, use_cuda_graph=False),
    dict(plain=True),
], ids=["auto", "no-graph", "t1024-h16", "t512-h64", "plain"])
def test_batch_matches_oracle(batch, mode):
    layers, expected = batch
    graphs = [MultilayerGraph.from_pairs(ls) for ls in layers]
    tables, results, report = batch_run(graphs, beta=1.0, **mode)
    _check(tables, results, expected)
    if not mode.get("plain"):
        assert report["peel_launches"] >= 1
        assert report["block_threads"] in (512, 1024)
    print(mode, report)


def test_batch_golden_fixtures():
    names = ["mix0", "mix1", "mix2", "mix3", "c1", "c2"]
    graphs = [MultilayerGraph.from_pairs(G.inputs(n)) for n in names]
    tables, results, _ = batch_run(graphs, beta=2.0)
    for name, t, r in zip(names, tables, results):
        exp = G.expected(name)
        assert np.array_equal(t, exp["table"]), name
        k, lmd, length = (int(x) for x in exp["b2.0_result"])
        assert (r["k"], r["lmd"], r["length"]) == (k, lmd, length), name
        assert np.float32(r["max_density_f"]) == exp["b2.0_maxf"]


def test_batch_same_as_alone():
    gens = synth.batch_mix(count=6, seed=306, n_lo=2000, n_hi=30000)
    graphs = [MultilayerGraph.from_pairs(g.layers) for g in gens]
    tables, results, _ = batch_run(graphs, beta=1.0)
    for g, t, r in zip(gens, tables, results):
        alone = MultilayerGraph.from_pairs(g.layers)
        assert np.array_equal(alone.coreindex(), t)
        a = alone.densest([1.0])[0]
        assert (a["k"], a["lmd"], a["length"], a["density"]) == (r["k"], r["lmd"], r["length"],
                                                                 r["density"])


def test_batch_with_empty_graph_and_empty_layer():
    """A graph without edges and a graph with an empty layer, between ordinary
    ones: every result equals the oracle's, the empty graph's is all zero."""
    ordinary = synth.chung_lu_graph(2000, 3, 5000, 2.3, 0.3, 350).layers
    empty = [np.zeros((0, 2), np.uint32), np.zeros((0, 2), np.uint32)]
    gap = [ordinary[0], np.zeros((0, 2), np.uint32), ordinary[1]]
    layers = [ordinary, empty, gap]
    graphs = [MultilayerGraph.from_pairs(ls) for ls in layers]
    tables, results, _ = batch_run(graphs, beta=1.0)
    assert graphs[1].n == 0 and tables[1].size == 0
    assert (results[1]["k"], results[1]["lmd"], results[1]["length"]) == (0, 0, 0)
    for i in (0, 2):
        og = O.OracleGraph(layers[i])
        t = og.coreindex()
        o = og.densest(t, 1.0, with_cells=False)
        assert np.array_equal(tables[i], t)
        assert (results[i]["k"], results[i]["lmd"], results[i]["length"], results[i]["density"]) == \
            (o["k"], o["lmd"], o["length"], o["density"])


def _c4_graphs():
    """The full 256-graph mix (seed 404), regenerated from its seeds on the
    host's cores, and its pinned reference results."""
    import hashlib
    import json
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    fx = json.load(open(os.path.join(G.GOLDEN, "c4_mix.json")))
    params = synth.batch_params(**{k: fx["generator"][k] for k in ("count", "seed")})
    with ProcessPoolExecutor(os.cpu_count() or 1, mp_context=mp.get_context("spawn")) as ex:
        gens = list(ex.map(synth._make, params, chunksize=1))
    for gen, f in zip(gens, fx["graphs"]):
        assert G.pairs_sha(gen.layers) == f["pairs_sha256"], f["name"]
    return gens, fx["graphs"], hashlib


def test_c4_mix_batched_equals_the_reference():
    """All 256 graphs of the mix in one batched run: every table (SHA-256)
    and every densest result equal the reference's own (tests/golden/
    c4_mix.json, made by the reference's get_index2 and WdsList)."""
    gens, fx, hashlib = _c4_graphs()
    graphs = [MultilayerGraph.from_pairs(g.layers) for g in gens]
    tables, results, rep = batch_run(graphs, beta=1.0)
    for i, (g, t, r, f) in enumerate(zip(graphs, tables, results, fx)):
        assert (g.n, g.L) == (f["n"], f["L"]), i
        assert hashlib.sha256(np.ascontiguousarray(t).tobytes()).hexdigest() == \
            f["table_sha256"], f"graph {i}: table"
        assert (r["k"], r["lmd"], r["length"]) == (f["k"], f["lmd"], f["length"]), i
        assert np.float32(r["max_density_f"]) == np.float32(f["max_density_f"]), i
        if r["k"]:
            assert r["density"] == f["density"] and r["lstar"] == f["lstar"], i
            nodes, _ = g.densest_members(r)
            assert hashlib.sha256(np.ascontiguousarray(nodes, dtype="<u4").tobytes()) \
                .hexdigest() == f["nodes_sha256"], i
