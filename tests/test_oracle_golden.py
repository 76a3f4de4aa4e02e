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


# ---- the query-time restatements (Util/CoreIndexTime.h, Util/CheckMLCDTime.h)

@pytest.mark.parametrize("name", ["c1_small", "tiny_dirty", "layers33", "mix0"])
def test_query_restatements_answer_the_reference_cells(name):
    """Every cell the reference's own run reported, asked back through the
    getResCore / getResCoreOffline restatements, has the reference's size."""
    exp = G.expected(name)
    table = exp["table"]
    cells = exp["b1.0_cells"]
    ks = [int(c[0]) for c in cells] + [0, int(table.max()) + 1]
    lmds = [int(c[1]) for c in cells] + [1, table.shape[0]]
    scan = O.cells_scan(table, ks, lmds)
    srt = O.cells_sorted(table, ks, lmds)
    for i, c in enumerate(cells):
        assert len(scan[i]) == c[2]
    assert len(scan[-2]) == table.shape[1] and len(scan[-1]) == 0
    for a, b, k, lmd in zip(scan, srt, ks, lmds):
        assert np.array_equal(a, np.nonzero(table[lmd - 1] >= k)[0])
        assert np.array_equal(np.sort(b), a)
        assert np.all(np.diff(table[lmd - 1][b].astype(np.int64)) >= 0)


def test_mlcd_restatement():
    rng = np.random.default_rng(5)
    cores = rng.integers(0, 9, size=(700, 6)).astype(np.uint32)
    cores[::37, 2] = 0xFFFFFFFF  # a negative int read as unsigned, as the reference compares
    ks = [0, 1, 3, 5, 8, 9, 4, 2]
    lmds = [0, 1, 2, 6, 1, 1, 7, 3]
    got = O.mlcd_query(cores, ks, lmds)
    for k, lmd, g in zip(ks, lmds, got):
        want = np.nonzero((cores >= k).sum(axis=1) >= max(lmd, 1))[0]
        assert np.array_equal(g, want)


def test_oracle_matches_reference_on_the_c4_mix_sample():
    """The smallest graphs of the 256-graph mix against the reference's own
    results for them (tests/golden/c4_mix.json)."""
    import hashlib
    import json
    from pargridcpu_b200 import synth
    fx = json.load(open(os.path.join(G.GOLDEN, "c4_mix.json")))
    params = synth.batch_params(**{k: fx["generator"][k] for k in ("count", "seed")})
    small = sorted(range(len(params)), key=lambda i: fx["graphs"][i]["entries"])[:6]
    for i in small:
        f = fx["graphs"][i]
        gen = synth._make(params[i])
        assert G.pairs_sha(gen.layers) == f["pairs_sha256"]
        og = O.OracleGraph(gen.layers)
        t = og.coreindex()
        assert hashlib.sha256(np.ascontiguousarray(t).tobytes()).hexdigest() == f["table_sha256"]
        d = og.densest(t, 1.0, with_cells=False)
        assert (d["k"], d["lmd"], d["length"]) == (f["k"], f["lmd"], f["length"])
        assert np.float32(d["max_density_f"]) == np.float32(f["max_density_f"])
        if d["k"]:
            assert d["density"] == f["density"]


def brute_force_table(layers, ids):
    """The (k, lambda)-core index straight from its definition, for tiny
    graphs: core_lambda(v) is the largest k such that v belongs to a node set
    in which every node has at least k neighbours inside the set in at least
    lambda layers.  For each lambda and k = 1, 2, ... nodes are removed from
    the previous k's set until every one left qualifies (the largest such set
    is unique: the union of qualifying sets qualifies).  Self-loops and
    repeated pairs count once, as undirected edges without loops."""
    L, n = len(layers), len(ids)
    pos = {int(v): i for i, v in enumerate(ids)}
    nb = [[set() for _ in range(n)] for _ in range(L)]
    for l, e in enumerate(layers):
        for u, v in np.asarray(e, np.int64).reshape(-1, 2):
            if u != v:
                nb[l][pos[int(u)]].add(pos[int(v)])
                nb[l][pos[int(v)]].add(pos[int(u)])
    t = np.zeros((L, n), np.uint32)
    for lam in range(1, L + 1):
        alive = set(range(n))
        k = 1
        while alive:
            changed = True
            while changed:
                changed = False
                for v in list(alive):
                    if sum(len(nb[l][v] & alive) >= k for l in range(L)) < lam:
                        alive.discard(v)
                        changed = True
            for v in alive:
                t[lam - 1, v] = k
            k += 1
    return t


def _tiny_cases():
    from pargridcpu_b200 import synth
    rng = np.random.default_rng(77)
    cases = []
    for seed in range(4):  # random multilayer graphs
        g = synth.chung_lu_graph(48, 5, 120, 2.2, 0.5, 500 + seed)
        cases.append((f"chung_lu_{seed}", g.layers))
    cases.append(("one_layer", synth.chung_lu_graph(60, 1, 200, 2.2, 0.0, 42).layers))
    # more than 32 layers: Top-lambda over a block of layers
    cases.append(("33_layers", synth.erdos_renyi_graph(24, 33, 0.1, 0.3, 43).layers))
    # an empty layer, nodes isolated in some layers, repeated pairs, self-loops
    a = rng.integers(0, 30, (150, 2))
    b = rng.integers(10, 40, (90, 2))
    dup = np.concatenate([a[:40], a[:40], [[5, 5], [7, 7], [5, 9]]])
    cases.append(("empty_dup_loops", [a, np.zeros((0, 2), np.int64), b, dup]))
    return cases


@pytest.mark.parametrize("name,layers", _tiny_cases(), ids=[c[0] for c in _tiny_cases()])
def test_oracle_matches_the_definition_on_tiny_graphs(name, layers):
    og = O.OracleGraph(layers)
    assert np.array_equal(og.coreindex(), brute_force_table(layers, og.id2vtx()))


def test_node_relabelling_permutes_the_table():
    """Renaming the vertex ids (a bijection) leaves the first-seen numbering's
    positions, hence the table, unchanged, and id2vtx renamed alike."""
    from pargridcpu_b200 import synth
    g = synth.chung_lu_graph(200, 4, 700, 2.3, 0.4, 909)
    og = O.OracleGraph(g.layers)
    top = int(max(int(np.asarray(e).max(initial=0)) for e in g.layers)) + 1
    ren = np.random.default_rng(5).permutation(top).astype(np.int64) * 3 + 11
    og2 = O.OracleGraph([ren[np.asarray(e, np.int64)] for e in g.layers])
    assert np.array_equal(og2.coreindex(), og.coreindex())
    assert np.array_equal(og2.id2vtx(), ren[og.id2vtx().astype(np.int64)].astype(np.uint64))
