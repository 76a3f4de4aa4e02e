"""Generate the golden fixtures in this directory from the reference itself.

Every expected output here comes from the reference's own code: its sources
compiled in place by ``oracle/Makefile`` into ``oracle/_ref/ref_harness``,
which loads each input through the reference loader
(``MultilayerGraph::LoadFromFile`` on a text dataset; the c3 case, 34M edges,
goes through the harness's binary path instead) and runs

* ``get_index2`` per lambda (CoreIndex) for the core table,
* ParGrid's ``PeelSync`` on ParGrid's schedule for a second copy of the table,
* ``FCPathLevelLeft::Execute(wds=true)`` + ``FCTree::WeightDenestSubgraph``
  (WdsList) for beta in {0.5, 1.0, 2.0}.

Inputs are not stored: they are regenerated from the seeds in
``manifest.json`` by ``pargridcpu_b200.synth`` and checked against the stored
SHA-256 of their raw pairs.  Loader edge cases are stored as raw file text.

The batched mix (256 graphs, seed 404) and one large serving graph (n=2.6M,
L=24) are pinned the same way as c3, by hashes: ``--with-c4`` writes
``c4_mix.json`` (per graph: input and table SHA-256, per-lambda maxima, the
WdsList result for beta = 1 and its node set's SHA-256), ``--with-c5``
``c5_large.json`` (the same for the large graph).

Usage: python tests/golden/make_golden.py [--with-c3] [--with-c4] [--with-c5]
Needs the reference checkout (oracle/Makefile's REF) to build the checker.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from pargridcpu_b200 import synth  # noqa: E402
import oracle as O  # noqa: E402

BETAS = (0.5, 1.0, 2.0)
SCRATCH = os.path.join(HERE, "_scratch")

# name -> generator call (kind, kwargs); regenerated by tests via synth_case()
CASES = {
    "tiny_dirty": ("chung_lu", dict(n=300, n_layers=5, m_per_layer=1200, gamma=2.3, copy=0.3,
                                    seed=7, dirty=True)),
    "c1": ("config", dict(name="c1")),
    "c2": ("config", dict(name="c2")),
    "c1_small": ("config", dict(name="c1", scale=0.2)),
    "single_layer": ("chung_lu", dict(n=500, n_layers=1, m_per_layer=2000, gamma=2.2, copy=0.0,
                                      seed=11)),
    "layers33": ("chung_lu", dict(n=400, n_layers=33, m_per_layer=600, gamma=2.4, copy=0.5,
                                  seed=12)),
    "layers70": ("erdos_renyi", dict(n=90, n_layers=70, p_lo=0.02, p_hi=0.12, seed=13)),
    "er_small": ("erdos_renyi", dict(n=60, n_layers=40, p_lo=0.02, p_hi=0.1, seed=5)),
    "hubs": ("chung_lu", dict(n=20_000, n_layers=4, m_per_layer=60_000, gamma=2.05, copy=0.5,
                              seed=14)),
}
for i in range(4):
    CASES[f"mix{i}"] = ("mix", dict(index=i))

# raw layer-file texts that pin the loader's parse (MultilayerGraph.cpp:104-166)
TEXT_CASES = {
    "text_no_trailing_newline": ["1 2\n2 3\n3 1", "3 4\n4 1"],
    "text_trailing_blank": ["10 20\n20 30\n30 10\n\n\n", "30 40 \n  40 10\n"],
    "text_selfloops_dups": ["5 5\n5 6\n6 5\n5 6\n7 7\n6 7\n", "7 5\n5 7\n9 9\n"],
    "text_incomplete_pair": ["1 2\n2 3\n4\n", "2 1\n"],
    "text_empty_layer": ["1 2\n2 3\n3 1\n1 4\n", "", "4 2\n2 1\n"],
    "text_tabs_crlf": ["1\t2\r\n2\t3\r\n3\t1\r\n", "1 3\r\n"],
}

MIX_PARAMS = dict(count=4, seed=404, n_lo=1_000, n_hi=6_000)


def synth_case(name):
    """Regenerate a case's raw per-layer pairs."""
    kind, kw = CASES[name]
    if kind == "config":
        return synth.config_graph(**kw).layers
    if kind == "chung_lu":
        return synth.chung_lu_graph(**kw).layers
    if kind == "erdos_renyi":
        return synth.erdos_renyi_graph(**kw).layers
    if kind == "mix":
        return synth.batch_mix(**MIX_PARAMS)[kw["index"]].layers
    raise KeyError(kind)


def pairs_sha(layers):
    h = hashlib.sha256()
    for e in layers:
        a = np.ascontiguousarray(e, dtype="<u4")
        h.update(np.uint64(len(a)).tobytes())
        h.update(a.tobytes())
    return h.hexdigest()


def _ref_outputs(src, L, n, with_pg=True):
    out = {}
    out["table"] = O.ref_table(src, L, n, "table")
    if with_pg:
        out["pgtable"] = O.ref_table(src, L, n, "pgtable", threads=4)
    for beta in BETAS:
        w = O.ref_wds(src, beta, threads=4)
        tag = f"b{beta}"
        out[f"{tag}_result"] = np.array([w.get("k", 0), w.get("lmd", 0), w.get("length", 0)],
                                        np.uint32)
        out[f"{tag}_maxf"] = np.float32(w.get("max_density_f", 0.0))
        cells = w["cells"]
        out[f"{tag}_cells"] = np.array([(c[0], c[1], c[2], c[4]) for c in cells],
                                       np.uint32).reshape(-1, 4)
        out[f"{tag}_cell_density"] = np.array([c[3] for c in cells], np.float64)
        out[f"{tag}_nodes"] = w["nodes"].astype(np.uint32)
    return out


def _read_vtx_map(d, n):
    vm = np.loadtxt(os.path.join(d, "__vtx_map.txt"), dtype=np.uint64, ndmin=2).reshape(-1, 2)
    id2vtx = np.zeros(n, np.uint64)
    id2vtx[vm[:, 1].astype(np.int64)] = vm[:, 0]
    return id2vtx


def make_case(name, manifest):
    layers = synth_case(name)
    d = os.path.join(SCRATCH, name) + "/"
    shutil.rmtree(d, ignore_errors=True)
    synth.write_dataset(synth.Graph(layers), d)
    og = O.OracleGraph(layers)
    n, L = og.n, og.L
    out = _ref_outputs(d, L, n)
    out["id2vtx"] = _read_vtx_map(d, n)
    out["layer_m"] = og.layer_m()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    manifest[name] = dict(kind="synth", n=int(n), L=int(L), pairs_sha256=pairs_sha(layers),
                          pairs=int(sum(len(e) for e in layers)))
    print(name, n, L, flush=True)


def make_text_case(name, texts, manifest):
    d = os.path.join(SCRATCH, name) + "/"
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    with open(os.path.join(d, "mlg.conf"), "w") as f:
        f.write("".join(f"l{i}.txt\n" for i in range(len(texts))))
    for i, t in enumerate(texts):
        with open(os.path.join(d, f"l{i}.txt"), "w", newline="") as f:
            f.write(t)
    # n and L as the reference loader sees them: read from the harness log
    r = subprocess.run([O.HARNESS, d, "table", os.path.join(d, "t.bin")], capture_output=True,
                       text=True, check=True)
    head = r.stderr.split()
    n = int([x for x in head if x.startswith("n=")][0][2:])
    L = int([x for x in head if x.startswith("L=")][0][2:])
    out = _ref_outputs(d, L, n) if n else {"table": np.zeros((L, 0), np.uint32)}
    out["id2vtx"] = _read_vtx_map(d, n) if n else np.zeros(0, np.uint64)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    manifest[name] = dict(kind="text", n=n, L=L, texts=texts)
    print(name, n, L, flush=True)


def make_c3(manifest):
    """Full-size c3: too large to store, so its table is kept as a SHA-256,
    with per-lambda maxima and the densest results."""
    g = synth.config_graph("c3")
    os.makedirs(SCRATCH, exist_ok=True)
    fcg = os.path.join(SCRATCH, "c3.fcg")
    synth.write_fcg(g, fcg)
    og = O.OracleGraph(g.layers)
    n, L = og.n, og.L
    table = O.ref_table(fcg, L, n, "table")
    out = {"table_kmax": table.max(axis=1).astype(np.uint32),
           "table_hist": np.stack([np.bincount(t, minlength=int(table.max()) + 1)
                                   for t in table]).astype(np.uint64)}
    for beta in BETAS:
        w = O.ref_wds(fcg, beta, threads=8)
        tag = f"b{beta}"
        out[f"{tag}_result"] = np.array([w["k"], w["lmd"], w["length"]], np.uint32)
        out[f"{tag}_maxf"] = np.float32(w["max_density_f"])
        out[f"{tag}_cells"] = np.array([(c[0], c[1], c[2], c[4]) for c in w["cells"]],
                                       np.uint32).reshape(-1, 4)
        out[f"{tag}_cell_density"] = np.array([c[3] for c in w["cells"]], np.float64)
        out[f"{tag}_nodes"] = w["nodes"].astype(np.uint32)
    np.savez_compressed(os.path.join(HERE, "c3.npz"), **out)
    manifest["c3"] = dict(kind="synth_large", n=int(n), L=int(L), pairs_sha256=pairs_sha(g.layers),
                          pairs=g.n_pairs,
                          table_sha256=hashlib.sha256(np.ascontiguousarray(table).tobytes())
                          .hexdigest())
    print("c3", n, L, flush=True)


def _pin_graph(args):
    """One graph's reference outputs as hashes (a worker of make_c4/make_c5)."""
    params, tag, threads = args
    g = synth._make(params)
    os.makedirs(SCRATCH, exist_ok=True)
    fcg = os.path.join(SCRATCH, f"{tag}.fcg")
    synth.write_fcg(g, fcg)
    og = O.OracleGraph(g.layers)
    n, L = og.n, og.L
    table = O.ref_table(fcg, L, n, "table", threads=threads)
    w = O.ref_wds(fcg, 1.0, threads=threads)
    os.remove(fcg)
    win = [c for c in w["cells"] if (c[0], c[1]) == (w.get("k", 0), w.get("lmd", 0))]
    return dict(name=params["name"], n=int(n), L=int(L), pairs_sha256=pairs_sha(g.layers),
                entries=int(og.layer_m().sum()),
                table_sha256=hashlib.sha256(np.ascontiguousarray(table).tobytes()).hexdigest(),
                kmax=[int(x) for x in table.max(axis=1)] if n else [0] * L,
                k=int(w.get("k", 0)), lmd=int(w.get("lmd", 0)), length=int(w.get("length", 0)),
                max_density_f=float(np.float32(w.get("max_density_f", 0.0))),
                density=float(win[0][3]) if win else 0.0,
                lstar=int(win[0][4]) if win else 0,
                n_cells=len(w["cells"]),
                nodes_sha256=hashlib.sha256(np.ascontiguousarray(w["nodes"], dtype="<u4")
                                            .tobytes()).hexdigest())


C4_MIX = dict(count=256, seed=404)


def make_c4(workers):
    """The full 256-graph mix (batch_params(256, seed=404)): every graph's
    table and densest result from the reference, as hashes."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    params = synth.batch_params(**C4_MIX)
    jobs = [(p, f"c4_{i}", 1) for i, p in enumerate(params)]
    # the largest graphs first, so the pool ends together
    order = sorted(range(len(jobs)), key=lambda i: -params[i]["n"] * params[i]["n_layers"]
                   * params[i]["m_per_layer"] / max(1, params[i]["n"]))
    out = [None] * len(jobs)
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        futs = {i: ex.submit(_pin_graph, jobs[i]) for i in order}
        for i in order:
            out[i] = futs[i].result()
            print("c4", i, out[i]["n"], out[i]["L"], flush=True)
    with open(os.path.join(HERE, "c4_mix.json"), "w") as f:
        json.dump(dict(generator=dict(C4_MIX, fn="synth.batch_params"), beta=1.0, graphs=out),
                  f, indent=0)


def make_c5(workers):
    """The serving configuration's large graph (CONFIGS['c5_large'], the
    first of the seeds the benchmark draws: seed + 0)."""
    c = synth.CONFIGS["c5_large"]
    p = dict(n=c["n"], n_layers=c["L"], m_per_layer=c["m"], gamma=c["gamma"], copy=c["copy"],
             seed=c["seed"], name="large0")
    r = _pin_graph((p, "c5", workers))
    with open(os.path.join(HERE, "c5_large.json"), "w") as f:
        json.dump(dict(params=p, beta=1.0, graph=r), f, indent=1)
    print("c5", r["n"], r["L"], flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--with-c3", action="store_true")
    ap.add_argument("--with-c4", action="store_true")
    ap.add_argument("--with-c5", action="store_true")
    ap.add_argument("--only", default=None)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "liboracle.so"],
                   check=True, stdout=subprocess.DEVNULL)
    mpath = os.path.join(HERE, "manifest.json")
    manifest = json.load(open(mpath)) if os.path.exists(mpath) else {}
    manifest["_generator"] = dict(mix=MIX_PARAMS, betas=list(BETAS))
    if a.with_c4 or a.with_c5:
        if a.with_c4:
            make_c4(a.workers)
        if a.with_c5:
            make_c5(a.workers)
        return
    for name in CASES:
        if a.only and name != a.only:
            continue
        make_case(name, manifest)
    for name, texts in TEXT_CASES.items():
        if a.only and name != a.only:
            continue
        make_text_case(name, texts, manifest)
    if a.with_c3:
        make_c3(manifest)
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    shutil.rmtree(SCRATCH, ignore_errors=True)


if __name__ == "__main__":
    main()
