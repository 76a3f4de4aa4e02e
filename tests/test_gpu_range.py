"""One graph split by lambda range (fc_coreindex_range / fc_cells_range): each
range's table is the matching slice of the whole table, each range's cells
are the whole graph's cells of those lambdas, and the fold of all ranges'
cells (the reference's order and float running maximum) is the whole graph's
densest result.  A handle that computed a range still gives the whole table
and densest result afterwards."""
import numpy as np
import pytest

import golden_cases as G
from pargridcpu_b200 import MultilayerGraph, shard, synth

pytestmark = pytest.mark.gpu

FIELDS = ("k", "lmd", "length", "lstar", "density", "max_density_f")


def _cases():
    yield "c1", G.inputs("c1")
    yield "layers33", G.inputs("layers33")
    yield "mix0", G.inputs("mix0")
    yield "chung_lu", synth.chung_lu_graph(40000, 9, 150000, 2.2, 0.4, 410).layers


@pytest.mark.parametrize("name,layers", list(_cases()), ids=lambda x: x if isinstance(x, str) else "")
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("beta", [1.0, 2.0])
def test_ranges_give_the_whole_graph(name, layers, world, beta):
    whole = MultilayerGraph.from_pairs(layers)
    table = whole.coreindex()
    res = whole.densest([beta])[0]
    rec, dens = whole.cells(beta)
    L = whole.L
    per_rank = []
    for lo, hi in shard.column_ranges(L, world):
        if lo >= hi:
            continue
        g = MultilayerGraph.from_pairs(layers)      # one process's own handle
        part = g.coreindex_range(lo, hi)
        assert np.array_equal(part, table[lo - 1:hi - 1])
        cells = g.cells_range(lo, hi, beta)
        want = [(int(r[0]), int(r[1]), int(r[2]), int(r[3]), float(d))
                for r, d in zip(rec, dens) if lo <= r[1] < hi]
        assert cells == want
        per_rank.append(cells)
        # the same handle then answers for the whole graph
        assert np.array_equal(g.coreindex(), table)
        got = g.densest([beta])[0]
        for f in FIELDS:
            assert got[f] == res[f], f
    merged = shard.merge_cells(per_rank[::-1])
    for f in FIELDS:
        assert merged[f] == res[f], f


def test_range_inside_resident_table_and_nested_ranges():
    """A range inside an already computed table or range is copied, not
    recomputed; a range outside the computed one is computed."""
    layers = G.inputs("layers33")
    whole = MultilayerGraph.from_pairs(layers)
    table = whole.coreindex()
    L = whole.L
    g = MultilayerGraph.from_pairs(layers)
    assert np.array_equal(g.coreindex_range(2, L + 1), table[1:])
    assert np.array_equal(g.coreindex_range(3, L), table[2:L - 1])   # inside
    assert np.array_equal(g.coreindex_range(1, 2), table[:1])        # outside
    assert np.array_equal(whole.coreindex_range(1, L + 1), table)    # whole table resident
    assert np.array_equal(whole.coreindex_range(L, L + 1), table[L - 1:])
