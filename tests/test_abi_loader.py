"""The C-ABI library without a GPU: every declared symbol is exported, the
loader reproduces the reference loader's results (golden fixtures made by the
reference itself), and compute calls fail loudly instead of falling back to
the CPU."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import golden_cases as G
import oracle as O
from pargridcpu_b200 import MultilayerGraph, native, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "firmcore.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fc_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_exports():
    decl = declared_functions()
    assert decl == sorted(native.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (fc_\w+)", out))
    missing = [f for f in decl if f not in exported]
    assert not missing, missing
    lib = native.lib()
    for f in decl:
        assert getattr(lib, f) is not None
    assert lib.fc_abi_version() == 1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("name", G.SYNTH)
def test_loader_from_pairs_matches_reference(name):
    exp = G.expected(name)
    layers = G.inputs(name)
    g = MultilayerGraph.from_pairs(layers)
    assert g.n == G.MANIFEST[name]["n"] and g.L == G.MANIFEST[name]["L"]
    assert np.array_equal(g.id2vtx(), exp["id2vtx"])
    assert np.array_equal(g.layer_m(), exp["layer_m"])
    off, adj = g.csr()
    o_off, o_adj = O.OracleGraph(layers).csr()
    assert np.array_equal(off, o_off) and np.array_equal(adj, o_adj)


def test_csr_build_split_over_threads_matches_oracle():
    """Few layers and many nodes: each layer's rows are sorted and deduplicated
    on several host threads (node ranges of equal entry counts); the CSR must
    still equal the oracle's, duplicates and self loops included."""
    gen = synth.chung_lu_graph(30000, 2, 120000, 2.1, 0.4, 97, dirty=True)
    g = MultilayerGraph.from_pairs(gen.layers)
    off, adj = g.csr()
    o_off, o_adj = O.OracleGraph(gen.layers).csr()
    assert np.array_equal(off, o_off) and np.array_equal(adj, o_adj)


def _write_texts(d, texts):
    with open(os.path.join(d, "mlg.conf"), "w") as f:
        f.write("".join(f"l{i}.txt\n" for i in range(len(texts))))
    for i, t in enumerate(texts):
        with open(os.path.join(d, f"l{i}.txt"), "w", newline="") as f:
            f.write(t)


@pytest.mark.parametrize("name", G.TEXT)
def test_loader_text_matches_reference(name):
    exp = G.expected(name)
    with tempfile.TemporaryDirectory() as d:
        _write_texts(d, G.texts(name))
        g = MultilayerGraph.LoadFromFile(d, write_vtx_map=True)
        assert g.n == G.MANIFEST[name]["n"]
        assert np.array_equal(g.id2vtx(), exp["id2vtx"])
        vm = open(os.path.join(d, "__vtx_map.txt")).read().split()
        ids = np.array(vm, dtype=np.uint64).reshape(-1, 2)
        assert np.array_equal(ids[:, 0], exp["id2vtx"]) and np.array_equal(
            ids[:, 1], np.arange(g.n))


def test_loader_text_same_as_pairs():
    g0 = synth.chung_lu_graph(800, 3, 3000, 2.3, 0.3, 99, dirty=True)
    with tempfile.TemporaryDirectory() as d:
        synth.write_dataset(g0, d)
        a = MultilayerGraph.LoadFromFile(d, write_vtx_map=False)
        assert not os.path.exists(os.path.join(d, "__vtx_map.txt"))
    b = MultilayerGraph.from_pairs(g0.layers)
    assert np.array_equal(a.id2vtx(), b.id2vtx())
    for x, y in zip(a.csr(), b.csr()):
        assert np.array_equal(x, y)


def _ref_order(o, m, n):
    """SetGraphOrder's permutation (Graph/MultilayerGraph.cpp:9-45), for inputs
    without ties."""
    if o in (1, 2):
        key = [np.float32(np.float32(x >> 1) / np.float32(n)) for x in m]
    else:
        key = list(m)
    idx = sorted(range(len(m)), key=lambda i: key[i], reverse=(o in (2, 4)))
    return idx


@pytest.mark.parametrize("o", [1, 2, 3, 4])
def test_layer_order(o):
    rng = np.random.default_rng(o)
    layers = []
    for l, m in enumerate([30, 80, 10, 55]):
        e = rng.integers(0, 40, size=(m, 2)).astype(np.uint32)
        layers.append(e)
    with tempfile.TemporaryDirectory() as d:
        synth.write_dataset(synth.Graph(layers), d)
        g0 = MultilayerGraph.LoadFromFile(d, order=0, write_vtx_map=False)
        g = MultilayerGraph.LoadFromFile(d, order=o, write_vtx_map=False)
    m0 = [int(x) for x in g0.layer_m()]
    assert len(set(m0)) == len(m0)
    want = _ref_order(o, m0, g0.n)
    assert list(g.order()) == want
    assert [int(x) for x in g.layer_m()] == [m0[i] for i in want]


def test_adjbuf_roundtrip():
    layers = synth.chung_lu_graph(300, 3, 900, 2.4, 0.2, 5).layers
    a = MultilayerGraph.from_pairs(layers)
    off, adj = a.csr()
    n = a.n
    bufs = []
    for l in range(a.L):
        rows = []
        for v in range(n):
            r = adj[off[l, v]:off[l, v + 1]]
            rows.append(np.concatenate([[len(r)], r]))
        bufs.append(np.concatenate(rows).astype(np.uint32))
    b = MultilayerGraph.from_adjbuf(n, bufs)
    for x, y in zip(a.csr(), b.csr()):
        assert np.array_equal(x, y)
    bad = [x.copy() for x in bufs]
    bad[0][0] = 10 ** 6  # a row longer than the buffer
    with pytest.raises(native.FcError):
        MultilayerGraph.from_adjbuf(n, bad)


def test_load_errors():
    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(native.FcError) as e:
            MultilayerGraph.LoadFromFile(d)
        assert e.value.code == 1
        with open(os.path.join(d, "mlg.conf"), "w") as f:
            f.write("missing.txt\n")
        with pytest.raises(native.FcError) as e:
            MultilayerGraph.LoadFromFile(d)
        assert e.value.code == 1


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    g = MultilayerGraph.from_pairs(G.inputs("tiny_dirty"))
    with pytest.raises(native.FcError) as e:
        g.coreindex()
    assert e.value.code == 9
    with pytest.raises(native.FcError) as e:
        g.densest([1.0])
    assert e.value.code == 9


def test_lambda_range_bounds_checked_on_host():
    """fc_coreindex_range / fc_cells_range reject a range outside
    1 <= lo < hi <= L+1 before touching a device."""
    g = MultilayerGraph.from_pairs(G.inputs("tiny_dirty"))
    for lo, hi in [(0, 1), (2, 2), (3, 2), (1, g.L + 2)]:
        rc = native.lib().fc_coreindex_range(g._h, lo, hi, None, 0, None)
        assert rc == 7
        with pytest.raises(native.FcError) as e:
            g.cells_range(lo, hi)
        assert e.value.code == 7


def test_cli_help_runs_without_gpu():
    """The drop-in CLI loads a dataset and prints the reference's header lines
    before any device work."""
    exe = os.path.join(ROOT, "pargridcpu_b200", "firmcore_baseline")
    with tempfile.TemporaryDirectory() as d:
        ds = os.path.join(d, "dataset", "tiny")
        synth.write_dataset(synth.chung_lu_graph(50, 2, 80, 2.5, 0.0, 1), ds)
        wd = os.path.join(d, "bin")
        os.makedirs(wd)
        r = subprocess.run([exe, "-d", "tiny", "-m", "fcgrid"], cwd=wd, capture_output=True,
                           text=True)
        assert r.returncode == 0, r.stderr
        assert "method = fcgrid dataset = tiny" in r.stdout
        assert "|L| = 2, |V| = " in r.stdout
        assert "kupper = " in r.stdout and "lmdupper = 2" in r.stdout
