"""The drop-in CLI on a GPU: `firmcore_baseline` run the way the reference's
binary is run (dataset under ../dataset/<name>/, outputs under ../output/)
prints the reference's lines and writes the reference's files, with the
values of the reference's algorithm (the oracle on the same input)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from pargridcpu_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "pargridcpu_b200", "firmcore_baseline")


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    base = tmp_path_factory.mktemp("cli")
    g = synth.chung_lu_graph(3000, 5, 9000, 2.3, 0.3, 77)
    synth.write_dataset(g, str(base / "dataset" / "tiny"))
    os.makedirs(base / "bin")
    os.makedirs(base / "output")
    og = O.OracleGraph(g.layers)
    return base, og, og.coreindex()


def _run(base, *args):
    r = subprocess.run([EXE, "-d", "tiny", *args], cwd=base / "bin", capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _field(out, name):
    for line in out.splitlines():
        if line.startswith(name + " = "):
            return line.split(" = ", 1)[1].strip()
    raise AssertionError(f"{name} not printed:\n{out}")


def test_pargrid_table(setup):
    base, og, table = setup
    out = _run(base, "-m", "ParGrid", "-num_thread", "8", "-table", str(base / "t.bin"))
    assert "Path left Core Parallel Sync Elapsed time:" in out
    got = np.fromfile(base / "t.bin", dtype=np.uint32).reshape(og.L, og.n)
    assert np.array_equal(got, table)


def test_wdslist_lines(setup):
    base, og, table = setup
    out = _run(base, "-m", "WdsList", "-beta", "1")
    d = og.densest(table, 1.0, with_cells=False)
    assert int(_field(out, "res_k")) == d["k"]
    assert int(_field(out, "res_lmd")) == d["lmd"]
    assert int(_field(out, "res_len")) == d["length"]
    # printed as the reference prints its float maximum (6 significant digits)
    assert float(_field(out, "maximum_density")) == pytest.approx(d["max_density_f"], rel=1e-5)


def test_kpe_cell_file(setup):
    base, og, table = setup
    lmd = 2
    k = max(1, int(table[lmd - 1].max()) // 2)
    out = _run(base, "-m", "kpe", "-k", str(k), "-lmd", str(lmd))
    path = base / "output" / f"tiny_k_{k}_lmd_{lmd}_serial.txt"
    assert _field(out, "res_file") == f"../output/tiny_k_{k}_lmd_{lmd}_serial.txt"
    lines = path.read_text().splitlines()
    want = np.nonzero(table[lmd - 1] >= k)[0]
    assert lines[0] == f"########## k_{k}_lmd_{lmd}_length_{len(want)}"
    vtx = (base / "dataset" / "tiny" / "__vtx_map.txt").read_text().split()
    id2vtx = {int(vtx[i + 1]): vtx[i] for i in range(0, len(vtx), 2)}
    assert lines[1:] == [id2vtx[int(v)] for v in want]


@pytest.mark.parametrize("method,line", [
    ("ParGridPlus", "Mix Core/Path Parallel Sync Elapsed time:"),
    ("CoreIndex", "CoreIndex Serial Elapsed time:"),
    ("ParCoreIndex", "CoreIndex Parallel Elapsed time:"),
])
def test_table_methods(setup, method, line):
    """-m ParGridPlus / CoreIndex / ParCoreIndex (main.cpp:277-400): the
    reference's lines, and the same table."""
    base, og, table = setup
    out = _run(base, "-m", method, "-num_thread", "4", "-table", str(base / f"{method}.bin"))
    assert line in out and "mem = " in out
    if method != "ParGridPlus":
        assert _field(out, "n_layer") == str(og.L)
        assert _field(out, "n_vertex") == str(og.n)
    got = np.fromfile(base / f"{method}.bin", dtype=np.uint32).reshape(og.L, og.n)
    assert np.array_equal(got, table)


def test_wdscoreindex_lines(setup):
    """-m WdsCoreIndex (main.cpp:444-451) prints the densest cell's density
    and label; the label is the fold's winner (WdsList's answer)."""
    base, og, table = setup
    out = _run(base, "-m", "WdsCoreIndex", "-beta", "1")
    assert "I am the WDS CoreIndex" in out and "Wds CoreIndex Time = " in out
    d = og.densest(table, 1.0, with_cells=False)
    assert float(_field(out, "maximum_density")) == pytest.approx(d["max_density_f"], rel=1e-5)
    assert (int(_field(out, "res_k")), int(_field(out, "res_lmd"))) == (d["k"], d["lmd"])


@pytest.mark.parametrize("method,line", [
    ("CoreMem", "CoreParallel Sync with Memory reduction Elapsed time:"),
    ("PathMem", "PathParallel with Memory reduction Elapsed time:"),
])
def test_mem_methods_write_every_cell(setup, method, line):
    """-m CoreMem / PathMem (main.cpp:331-362): every cell in compact form."""
    base, og, table = setup
    path = base / f"{method}.cells"
    out = _run(base, "-m", method, "-cells", str(path))
    assert line in out and "Memory reduction mem = " in out
    raw = path.read_bytes()
    L, n = np.frombuffer(raw[:8], np.uint32)
    assert (L, n) == (og.L, og.n)
    off = np.frombuffer(raw[8:8 + 8 * (L + 1)], np.uint64)
    at = 8 + 8 * (L + 1)
    sizes = np.frombuffer(raw[at:at + 4 * int(off[-1])], np.uint32)
    order = np.frombuffer(raw[at + 4 * int(off[-1]):], np.uint32).reshape(L, n)
    for l in range(L):
        for k in range(int(table[l].max()) + 2):
            cell = order[l][:sizes[off[l] + k]]
            assert np.array_equal(np.sort(cell), np.nonzero(table[l] >= k)[0])


def _qblocks(path):
    out, cur = [], None
    for ln in path.read_text().splitlines():
        if ln.startswith("##########"):
            cur = (ln, [])
            out.append(cur)
        else:
            cur[1].append(int(ln))
    return out


@pytest.mark.parametrize("method", ["CoreIndexTimeOnline", "CoreIndexTimeOffline"])
def test_query_methods(setup, method):
    """-m CoreIndexTimeOnline / Offline (main.cpp:493-582): a klmd list of
    cells answered from the table; every answer is {v : core_lmd(v) >= k}."""
    base, og, table = setup
    pairs = [(1, 1), (3, 2), (int(table[0].max()), 1), (2, og.L), (10 ** 6, 3), (0, 4), (2, 99)]
    (base / "q.klmd").write_text("".join(f"{k} {l}\n" for k, l in pairs))
    qout = base / f"{method}.q"
    out = _run(base, "-m", method, "-klmd", str(base / "q.klmd"), "-qout", str(qout))
    assert "Elapsed time: " in out
    vtx = (base / "dataset" / "tiny" / "__vtx_map.txt").read_text().split()
    raw2id = {int(vtx[i]): int(vtx[i + 1]) for i in range(0, len(vtx), 2)}
    blocks = _qblocks(qout)
    kept = [(k, l) for k, l in pairs if 1 <= l <= og.L]  # lambda 99 is not a column
    assert len(blocks) == len(kept)
    for (k, l), (head, ids) in zip(kept, blocks):
        want = np.nonzero(table[l - 1] >= k)[0]
        assert head == f"########## k_{k}_lmd_{l}_length_{len(want)}"
        got = np.array([raw2id[i] for i in ids], dtype=np.int64)
        if method == "CoreIndexTimeOnline":
            assert np.array_equal(got, want)
        else:
            assert np.array_equal(np.sort(got), want)


def test_mlcd_method(setup):
    """-m MLCDTime (main.cpp:453-491): checktime's membership test on a
    coreness file."""
    base, og, table = setup
    rng = np.random.default_rng(1)
    cores = rng.integers(0, 12, size=(500, 5))
    (base / "c.cores").write_text("".join(" ".join(map(str, r)) + "\n" for r in cores))
    pairs = [(0, 0), (3, 2), (11, 1), (5, 5), (7, 3)]
    (base / "m.klmd").write_text("".join(f"{k} {l}\n" for k, l in pairs))
    qout = base / "mlcd.q"
    out = _run(base, "-m", "MLCDTime", "-klmd", str(base / "m.klmd"), "-cores",
               str(base / "c.cores"), "-qout", str(qout))
    assert "Elapsed time: " in out
    want = O.mlcd_query(cores.astype(np.uint32), [p[0] for p in pairs], [p[1] for p in pairs])
    for (head, ids), w in zip(_qblocks(qout), want):
        assert ids == [int(x) for x in w]
