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
