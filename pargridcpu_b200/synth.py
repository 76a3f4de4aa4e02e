"""Seeded synthetic multilayer graphs in the reference loader's input form.

The reference is benchmarked on twelve public datasets that are not available
here, so every workload is a seeded synthetic graph with the shapes the
benchmark configurations name:

* ``c1``: n=20,000, L=7, ~20,000 edges per layer, Chung-Lu gamma=2.5, 30% of
  each layer copied from layer 0.
* ``c2``: n=220, L=360, each layer Erdos-Renyi with p ~ U[0.01, 0.06].
* ``c3``: n=2.5M, L=4, 34M edges (8.5M per layer), Chung-Lu gamma=2.1, 50%
  copied from layer 0.
* ``c4``: a batch of 256 graphs, n log-uniform in [1k, 200k], L uniform in
  [2, 24], mean per-layer degree log-uniform in [2, 32], gamma ~ U[2, 3], copy
  fraction ~ U[0, 0.6].
* ``c5``: the c4 distribution plus 2% large graphs (n=2.6M, L=24, ~48M edges,
  gamma=2.2, 40% copy), for the serving loop.

A graph is a list of per-layer ``(m_l, 2)`` uint32 arrays of raw (u, v) ids in
file order -- exactly what ``MultilayerGraph::LoadLayer`` reads from a layer
file (Graph/MultilayerGraph.cpp:104-166).  Node labels are a random
permutation, so the loader's first-seen remap is exercised.  Self-loops and
duplicate edges are not generated unless asked for (``dirty=True``).

Chung-Lu layer: weights w_i = (i+1)^(-1/(gamma-1)); both endpoints drawn with
probability proportional to w (inverse-CDF sampling); self-loops and repeats
dropped; redrawn until the layer has its target edge count.  Layer copy: a
``copy`` fraction of layer 0's edges, sampled without replacement, then filled
with fresh draws.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Graph", "chung_lu_graph", "erdos_renyi_graph", "config_graph", "batch_mix",
    "write_fcg", "read_fcg", "write_dataset", "CONFIGS",
]


@dataclass
class Graph:
    """Raw per-layer edge lists (file order) plus the parameters that made them."""
    layers: list
    name: str = ""
    params: dict = field(default_factory=dict)

    @property
    def n_layers(self) -> int:
        return len(self.layers)

    @property
    def n_pairs(self) -> int:
        return int(sum(len(x) for x in self.layers))


def _cl_sampler(rng, n, gamma):
    w = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (gamma - 1.0))
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    perm = rng.permutation(n).astype(np.int64)

    def draw(k):
        a = perm[np.minimum(np.searchsorted(cdf, rng.random(k), side="right"), n - 1)]
        b = perm[np.minimum(np.searchsorted(cdf, rng.random(k), side="right"), n - 1)]
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        keep = lo != hi
        return lo[keep] * n + hi[keep]
    return draw


def _unique(x):
    """Sorted distinct values (same output as np.unique, sort-based)."""
    x = np.sort(x)
    if len(x) < 2:
        return x
    keep = np.empty(len(x), bool)
    keep[0] = True
    np.not_equal(x[1:], x[:-1], out=keep[1:])
    return x[keep]


def _fill(draw, base, target):
    ub = _unique(base)
    s = ub
    while len(s) < target:
        need = target - len(s)
        s = _unique(np.concatenate([s, draw(int(need * 1.3) + 64)]))
    if len(s) > target:
        # keep all of base, trim the fresh draws at random
        extra = s[~np.isin(s, ub, assume_unique=True)]
        keep = np.random.default_rng(len(s)).choice(len(extra), target - len(ub), replace=False)
        s = np.sort(np.concatenate([ub, extra[keep]]))
    return s


def _pairs(keys, n, rng):
    keys = keys.copy()
    rng.shuffle(keys)
    u = (keys // n).astype(np.uint32)
    v = (keys % n).astype(np.uint32)
    swap = rng.random(len(keys)) < 0.5
    uu = np.where(swap, v, u)
    vv = np.where(swap, u, v)
    return np.stack([uu, vv], 1)


def chung_lu_graph(n, n_layers, m_per_layer, gamma, copy, seed, name="", dirty=False):
    """Chung-Lu multilayer graph; ``m_per_layer`` undirected edges per layer."""
    rng = np.random.default_rng(seed)
    draw = _cl_sampler(rng, n, gamma)
    m = int(min(m_per_layer, n * (n - 1) // 2))
    l0 = _fill(draw, np.empty(0, np.int64), m)
    layers = []
    for l in range(n_layers):
        if l == 0:
            keys = l0
        else:
            base = rng.choice(l0, int(copy * m), replace=False) if copy > 0 else np.empty(0, np.int64)
            keys = _fill(draw, base, m)
        layers.append(_pairs(keys, n, rng))
    g = Graph(layers, name, dict(kind="chung_lu", n=n, L=n_layers, m=m, gamma=gamma, copy=copy,
                                 seed=seed))
    if dirty:
        _dirty(g, rng)
    return g


def erdos_renyi_graph(n, n_layers, p_lo, p_hi, seed, name=""):
    """Independent Erdos-Renyi layers with p ~ U[p_lo, p_hi] per layer."""
    rng = np.random.default_rng(seed)
    iu, ju = np.triu_indices(n, 1)
    keys_all = iu.astype(np.int64) * n + ju
    layers = []
    ps = []
    for _ in range(n_layers):
        p = rng.uniform(p_lo, p_hi)
        ps.append(p)
        keys = keys_all[rng.random(len(keys_all)) < p]
        layers.append(_pairs(keys, n, rng))
    return Graph(layers, name, dict(kind="erdos_renyi", n=n, L=n_layers, p_lo=p_lo, p_hi=p_hi,
                                    seed=seed))


def _dirty(g, rng):
    """Add self-loops and repeated / reversed edges (the loader drops them)."""
    for l, e in enumerate(g.layers):
        if len(e) == 0:
            continue
        k = max(1, len(e) // 20)
        dup = e[rng.integers(0, len(e), k)]
        rev = dup[:, ::-1]
        loops = np.repeat(e[rng.integers(0, len(e), k), :1], 2, axis=1)
        allp = np.concatenate([e, dup, rev, loops])
        g.layers[l] = allp[rng.permutation(len(allp))].astype(np.uint32)


CONFIGS = {
    "c1": dict(kind="chung_lu", n=20_000, L=7, m=20_000, gamma=2.5, copy=0.3, seed=101),
    "c2": dict(kind="erdos_renyi", n=220, L=360, p_lo=0.01, p_hi=0.06, seed=202),
    "c3": dict(kind="chung_lu", n=2_500_000, L=4, m=8_500_000, gamma=2.1, copy=0.5, seed=303),
    "c5_large": dict(kind="chung_lu", n=2_600_000, L=24, m=2_000_000, gamma=2.2, copy=0.4,
                     seed=505),
}


def config_graph(name, scale=1.0, seed=None):
    """One of the named configurations; ``scale`` shrinks n and m for tests."""
    c = dict(CONFIGS[name])
    if seed is not None:
        c["seed"] = seed
    if c["kind"] == "chung_lu":
        n = max(16, int(c["n"] * scale))
        m = max(8, int(c["m"] * scale))
        return chung_lu_graph(n, c["L"], m, c["gamma"], c["copy"], c["seed"], name=name)
    return erdos_renyi_graph(c["n"], c["L"], c["p_lo"], c["p_hi"], c["seed"], name=name)


def batch_params(count=256, seed=404, n_lo=1_000, n_hi=200_000, large_frac=0.0, large=None):
    """The per-graph parameters of batch_mix (cheap; no graph is built)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if large_frac > 0 and rng.random() < large_frac:
            c = large or CONFIGS["c5_large"]
            out.append(dict(n=c["n"], n_layers=c["L"], m_per_layer=c["m"], gamma=c["gamma"],
                            copy=c["copy"], seed=int(rng.integers(1 << 30)), name=f"large{i}"))
            continue
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        L = int(rng.integers(2, 25))
        deg = float(np.exp(rng.uniform(np.log(2), np.log(32))))
        gamma = float(rng.uniform(2.0, 3.0))
        copy = float(rng.uniform(0.0, 0.6))
        m = max(1, int(n * deg / 2))
        out.append(dict(n=n, n_layers=L, m_per_layer=m, gamma=gamma, copy=copy,
                        seed=int(rng.integers(1 << 30)), name=f"g{i}"))
    return out


def _make(p):
    return chung_lu_graph(**p)


def batch_mix(count=256, seed=404, n_lo=1_000, n_hi=200_000, large_frac=0.0, large=None,
              workers=0):
    """The uneven batch: per graph n log-uniform in [n_lo, n_hi], L uniform in
    [2, 24], mean per-layer degree log-uniform in [2, 32], gamma ~ U[2, 3], copy
    ~ U[0, 0.6].  With ``large_frac`` > 0 that share of graphs is drawn from
    ``large`` (a CONFIGS-style dict) instead.  Each graph has its own seed, so
    ``workers`` > 1 (a spawned process pool) builds the same graphs."""
    params = batch_params(count, seed, n_lo, n_hi, large_frac, large)
    if workers and workers > 1 and count > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_make, params, chunksize=1))
    return [_make(p) for p in params]


# ---- files -----------------------------------------------------------------

def write_fcg(g: Graph, path: str) -> None:
    """FCG1 binary: b"FCG1", uint32 L, then per layer uint64 m and m (u,v)
    uint32 pairs in file order (little endian)."""
    with open(path, "wb") as f:
        f.write(b"FCG1")
        f.write(struct.pack("<I", g.n_layers))
        for e in g.layers:
            e = np.ascontiguousarray(e, dtype="<u4")
            f.write(struct.pack("<Q", len(e)))
            f.write(e.tobytes())


def read_fcg(path: str) -> Graph:
    with open(path, "rb") as f:
        if f.read(4) != b"FCG1":
            raise ValueError("not an FCG1 file")
        (L,) = struct.unpack("<I", f.read(4))
        layers = []
        for _ in range(L):
            (m,) = struct.unpack("<Q", f.read(8))
            layers.append(np.frombuffer(f.read(8 * m), dtype="<u4").reshape(m, 2).copy())
    return Graph(layers, os.path.basename(path))


def write_dataset(g: Graph, directory: str, trailing_newline=True) -> None:
    """The reference's dataset layout: ``mlg.conf`` naming one layer file per
    line, and one ``u v`` line per edge in each layer file."""
    os.makedirs(directory, exist_ok=True)
    names = [f"l{i}.txt" for i in range(g.n_layers)]
    with open(os.path.join(directory, "mlg.conf"), "w") as f:
        f.write("\n".join(names) + "\n")
    for name, e in zip(names, g.layers):
        with open(os.path.join(directory, name), "w") as f:
            if len(e):
                body = "\n".join(f"{int(a)} {int(b)}" for a, b in e) if len(e) < 200_000 else \
                    _fast_lines(e)
                f.write(body + ("\n" if trailing_newline else ""))


def _fast_lines(e):
    return "\n".join(map(" ".join, np.asarray(e).astype(str).tolist()))
