"""The serving loop (fc_server_*): requests that run batched with others,
while other batches run beside them on the device, get exactly the results
they get alone; requests that arrive while a large one runs do not queue
behind it; admission respects the device-memory budget (rejecting what can
never fit, releasing resident graphs to make room) without changing any
result; the plain one-at-a-time form agrees."""
import time

import numpy as np
import pytest

import golden_cases as G
from pargridcpu_b200 import MultilayerGraph, Server, native, synth

pytestmark = pytest.mark.gpu

FIELDS = ("k", "lmd", "length", "lstar", "density", "max_density_f")


def _alone(layers, beta):
    g = MultilayerGraph.from_pairs(layers)
    return g.coreindex(), g.densest([beta])[0]


def _same(table, res, exp):
    t, d = exp
    assert np.array_equal(table, t)
    for f in FIELDS:
        assert res[f] == d[f], f


@pytest.fixture(scope="module")
def mix():
    """(layers, beta) requests: golden mixes, assorted small graphs, one graph
    asked twice with different betas, a single-edge graph."""
    reqs = [(G.inputs(f"mix{i}"), 1.0) for i in range(4)]
    reqs += [(g.layers, 0.5 + 0.25 * (i % 3))
             for i, g in enumerate(synth.batch_mix(count=8, seed=310, n_lo=500, n_hi=20000))]
    twice = synth.chung_lu_graph(5000, 6, 12000, 2.3, 0.4, 311).layers
    reqs += [(twice, 1.0), (twice, 2.0)]
    reqs += [(G.inputs("layers33"), 1.0), ([np.array([[1, 2]], np.uint32)], 1.0)]
    return reqs


def test_server_results_same_alone_and_in_mix(mix):
    expected = [_alone(ls, b) for ls, b in mix]
    graphs = {}
    for ls, _ in mix:  # one handle per distinct input, as a caller would hold them
        graphs.setdefault(id(ls), MultilayerGraph.from_pairs(ls))
    srv = Server(lanes=2)
    try:
        order = np.random.default_rng(5).permutation(len(mix))
        tickets = {}
        for i in order:
            ls, beta = mix[i]
            tickets[i] = srv.submit(graphs[id(ls)], beta)
        for i, t in tickets.items():
            table, res, lat = srv.wait(t, timeout_ms=120000)
            _same(table, res, expected[i])
            assert lat > 0
        st = srv.stats()
    finally:
        srv.close()
    print(st)
    assert st["requests_done"] == len(mix)
    assert st["batches"] < len(mix)          # requests were batched together
    assert st["max_batch"] > 1
    assert st["graphs_peeled"] <= len(graphs) + st["batches"]


def test_server_small_requests_pass_a_large_one():
    """A large request is on one lane; requests submitted after it start on
    the other lane and complete first, with the same results as alone."""
    big = synth.chung_lu_graph(1_000_000, 12, 2_000_000, 2.2, 0.4, 320).layers
    small = [g.layers for g in synth.batch_mix(count=6, seed=321, n_lo=500, n_hi=3000)]
    exp_small = [_alone(ls, 1.0) for ls in small]
    gbig = MultilayerGraph.from_pairs(big)
    gsmall = [MultilayerGraph.from_pairs(ls) for ls in small]
    srv = Server(lanes=2, heavy_visits=100_000_000)  # the large graph is heavy
    try:
        t0 = time.perf_counter()
        tb = srv.submit(gbig, 1.0, want_table=False)
        deadline = time.perf_counter() + 30
        while srv.stats()["batches"] < 1 and time.perf_counter() < deadline:
            time.sleep(0.0005)
        ts = [(time.perf_counter(), srv.submit(g, 1.0)) for g in gsmall]
        done_small = []
        for (ts_sub, t), e in zip(ts, exp_small):
            table, res, lat = srv.wait(t, timeout_ms=120000)
            _same(table, res, e)
            done_small.append(ts_sub - t0 + lat / 1e3)
        _, _, lat_big = srv.wait(tb, timeout_ms=120000)
        st = srv.stats()
    finally:
        srv.close()
    print(st, "big ms", lat_big, "small done s", done_small)
    assert max(done_small) < lat_big / 1e3
    assert st["overlap_ms"] > 0 and st["heavy_batches"] == 1


def test_server_plain_same():
    reqs = [(G.inputs(f"mix{i}"), 1.0) for i in range(4)]
    expected = [_alone(ls, b) for ls, b in reqs]
    srv = Server(plain=True)
    try:
        ts = [srv.submit(MultilayerGraph.from_pairs(ls), b) for ls, b in reqs]
        for t, e in zip(ts, expected):
            table, res, _ = srv.wait(t, timeout_ms=120000)
            _same(table, res, e)
        st = srv.stats()
    finally:
        srv.close()
    assert st["batches"] == len(reqs) and st["lanes"] == 1


def test_server_budget_rejects_what_cannot_fit():
    g = MultilayerGraph.from_pairs(G.inputs("c1"))
    srv = Server(hbm_budget_bytes=1 << 20)
    try:
        t = srv.submit(g, 1.0)
        with pytest.raises(native.FcError) as e:
            srv.wait(t, timeout_ms=60000)
        assert e.value.code == 4  # FC_ERR_BUDGET
    finally:
        srv.close()


def test_server_evicts_resident_graphs_for_room():
    """A budget that holds two resident graphs and one running batch: each
    later request releases the least recently used copy, and every result
    stays exact.  The graphs have one shape; a first server's counters after
    one request give the resident and scratch bytes of one graph."""
    gens = [synth.chung_lu_graph(20000, 8, 60000, 2.3, 0.3, 340 + i).layers for i in range(5)]
    expected = [_alone(ls, 1.0) for ls in gens]
    graphs = [MultilayerGraph.from_pairs(ls) for ls in gens]
    probe = Server(lanes=1)
    try:
        table, res, _ = probe.wait(probe.submit(graphs[0], 1.0), timeout_ms=120000)
        _same(table, res, expected[0])
        st0 = probe.stats()
    finally:
        probe.close()
    gb = st0["resident_bytes"]                # one resident copy
    wb = st0["peak_bytes"] - gb               # one batch's scratch
    assert gb > 0 and wb > 0
    srv = Server(hbm_budget_bytes=2 * gb + wb + gb // 2, lanes=1)
    try:
        for _ in range(2):
            for g, e in zip(graphs, expected):
                table, res, _ = srv.wait(srv.submit(g, 1.0), timeout_ms=120000)
                _same(table, res, e)
        st = srv.stats()
    finally:
        srv.close()
    print(st)
    assert st["evictions"] > 0 and st["uploads"] > len(graphs)


def test_server_empty_graph():
    g = MultilayerGraph.from_pairs([np.zeros((0, 2), np.uint32)])
    srv = Server()
    try:
        table, res, _ = srv.wait(srv.submit(g, 1.0), timeout_ms=60000)
    finally:
        srv.close()
    assert table.size == 0 and (res["k"], res["lmd"], res["length"]) == (0, 0, 0)
