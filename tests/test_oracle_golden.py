"""The oracle pinned against the reference: every golden fixture was produced
by the reference's own code (tests/golden/make_golden.py), and the oracle must
reproduce it exactly."""
import os
import tempfile

import numpy as np
import pytest

import golden_cases as G
import oracle as O


def _check_densest(og, table, exp, beta):
    tag = f"b{beta}"
    got = og.densest(table, beta)
    k, lmd, length = (int(x) for x in exp[f"{tag}_result"])
    assert (got["k"], got["lmd"], got["length"]) == (k, lmd, length)
    assert np.float32(got["max_density_f"]) == exp[f"{tag}_maxf"]
    assert np.array_equal(got["cells"], exp[f"{tag}_cells"])
    # per-cell FP64 densities are bit-identical, not merely close
    assert np.array_equal(got["cell_density"], exp[f"{tag}_cell_density"])
    assert np.array_equal(got["nodes"], exp[f"{tag}_nodes"])


@pytest.mark.parametrize("name", G.SYNTH)
def test_oracle_matches_reference(name):
    exp = G.expected(name)
    og = O.OracleGraph(G.inputs(name))
    assert og.n == G.MANIFEST[name]["n"] and og.L == G.MANIFEST[name]["L"]
    assert np.array_equal(og.id2vtx(), exp["id2vtx"])
    assert np.array_equal(og.layer_m(), exp["layer_m"])
    table = og.coreindex()
    assert np.array_equal(table, exp["table"])
    # the reference's two routes agree with each other as well
    assert np.array_equal(exp["pgtable"], exp["table"])
    for beta in G.BETAS:
        _check_densest(og, table, exp, beta)


@pytest.mark.parametrize("name", G.TEXT)
def test_oracle_text_parse(name):
    exp = G.expected(name)
    layers = [O.parse_layer_text(t.encode()) for t in G.texts(name)]
    og = O.OracleGraph(layers)
    assert og.n == G.MANIFEST[name]["n"]
    assert np.array_equal(og.id2vtx(), exp["id2vtx"])
    if og.n:
        table = og.coreindex()
        assert np.array_equal(table, exp["table"])
        for beta in G.BETAS:
            _check_densest(og, table, exp, beta)


def test_parse_quirks():
    p = O.parse_layer_text
    # trailing newline: the last pair is read twice (a duplicate, later dropped)
    assert p(b"1 2\n").tolist() == [[1, 2], [1, 2]]
    assert p(b"1 2").tolist() == [[1, 2]]
    # a lone number pairs with the previous v
    assert p(b"1 2\n4\n").tolist() == [[1, 2], [4, 2]]
    # self-loops dropped, negative wraps, text stops the parse with u = 0
    assert p(b"3 3\n-1 2\n").tolist() == [[4294967295, 2], [4294967295, 2]]
    assert p(b"1 2\nx 5\n").tolist() == [[1, 2], [0, 2]]
    assert p(b"").shape == (0, 2)


def test_oracle_invariants_random():
    """Metamorphic properties on random small graphs: layer permutation
    invariance and containment core_{l+1} <= core_l."""
    from pargridcpu_b200 import synth
    for seed in range(6):
        g = synth.chung_lu_graph(150, 6, 400, 2.3, 0.4, 1000 + seed)
        t = O.OracleGraph(g.layers).coreindex()
        assert np.all(t[1:] <= t[:-1])
        perm = np.random.default_rng(seed).permutation(6)
        # permuting layers keeps every node's id (first-seen order may change)
        og2 = O.OracleGraph([g.layers[i] for i in perm])
        t2 = og2.coreindex()
        og1 = O.OracleGraph(g.layers)
        pos1 = {int(x): i for i, x in enumerate(og1.id2vtx())}
        idx = np.array([pos1[int(x)] for x in og2.id2vtx()])
        assert np.array_equal(t2, t[:, idx])


@pytest.mark.skipif(not O.harness_available(), reason="reference checker not built")
def test_harness_on_random_text_dataset():
    """A fresh seeded dataset through the reference's own text loader, beyond
    the stored fixtures."""
    from pargridcpu_b200 import synth
    g = synth.chung_lu_graph(400, 4, 900, 2.2, 0.3, 4242, dirty=True)
    with tempfile.TemporaryDirectory() as d:
        synth.write_dataset(g, d)
        og = O.OracleGraph(g.layers)
        ref = O.ref_table(d + "/", og.L, og.n)
        assert np.array_equal(og.coreindex(), ref)
        w = O.ref_wds(d + "/", 1.0)
        got = og.densest(ref, 1.0)
        assert (got["k"], got["lmd"], got["length"]) == (w["k"], w["lmd"], w["length"])
        assert os.path.exists(os.path.join(d, "__vtx_map.txt"))
