"""Sharding the path over ranks, on the CPU: the work-balanced graph
assignment and the lambda ranges are deterministic and cover everything
once; the merged fold of per-rank cells reproduces the reference's densest
result; and two gloo ranks (world_size 2, one process each) that split a
batch by graph and one graph by lambda range gather exactly the
single-process results.  The oracle computes each rank's share."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import golden_cases as G
import oracle as O
from pargridcpu_b200 import shard, synth


def _oracle_cells(layers, beta):
    og = O.OracleGraph(layers)
    t = og.coreindex()
    d = og.densest(t, beta, with_cells=True)
    cells = [(int(k), int(l), int(n), int(s), float(dd))
             for (k, l, n, s), dd in zip(d["cells"], d["cell_density"])]
    return og, t, d, cells


def _same_result(merged, d):
    assert (merged["k"], merged["lmd"], merged["length"], merged["lstar"]) == \
        (d["k"], d["lmd"], d["length"], d["lstar"])
    assert merged["density"] == d["density"]
    assert np.float32(merged["max_density_f"]) == np.float32(d["max_density_f"])


def test_assign_graphs_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    works = [int(x) for x in rng.lognormal(18, 2, size=200)]
    for world in (1, 2, 3, 8):
        a = shard.assign_graphs(works, world)
        assert a == shard.assign_graphs(works, world)
        assert sorted(set(a)) == list(range(min(world, len(works))))
        loads = [sum(w for w, r in zip(works, a) if r == k) for k in range(world)]
        # LPT bound: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(works) / world + max(works)


def test_column_ranges_cover_once():
    for L in (1, 2, 7, 24, 360):
        for world in (1, 2, 3, 8):
            rs = shard.column_ranges(L, world)
            cols = [c for lo, hi in rs for c in range(lo, hi)]
            assert cols == list(range(1, L + 1))
            assert max(hi - lo for lo, hi in rs) - min(hi - lo for lo, hi in rs) <= 1


@pytest.mark.parametrize("name", ["mix0", "layers33", "c1", "er_small"])
@pytest.mark.parametrize("beta", [0.5, 1.0, 2.0])
def test_fold_of_split_cells_is_the_reference_fold(name, beta):
    _, _, d, cells = _oracle_cells(G.inputs(name), beta)
    _same_result(shard.fold_cells(cells), d)
    L = max(c[1] for c in cells)
    for world in (2, 3):
        parts = [[c for c in cells if lo <= c[1] < hi] for lo, hi in shard.column_ranges(L, world)]
        _same_result(shard.merge_cells(parts[::-1]), d)  # any gather order


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        # (1) a batch split by graph
        gens = [g.layers for g in synth.batch_mix(count=6, seed=340, n_lo=300, n_hi=3000)]
        ogs = [O.OracleGraph(ls) for ls in gens]
        works = [shard.graph_work(o.n, o.L, int(o.layer_m().sum()) * 2) for o in ogs]
        owner = shard.assign_graphs(works, world)
        mine = []
        for i, o in enumerate(ogs):
            if owner[i] != rank:
                continue
            t = o.coreindex()
            d = o.densest(t, 1.0, with_cells=False)
            mine.append((i, t.tobytes(), (d["k"], d["lmd"], d["length"], d["density"])))
        got = [None] * world
        dist.all_gather_object(got, mine)
        # (2) one graph split by lambda range
        og, t, d, cells = _oracle_cells(G.inputs("c1"), 1.0)
        lo, hi = shard.column_ranges(og.L, world)[rank]
        merged = shard.gather_cells([c for c in cells if lo <= c[1] < hi])
        if rank == 0:
            flat = sorted(x for part in got for x in part)
            assert [x[0] for x in flat] == list(range(len(gens)))  # every graph once
            for i, tb, res in flat:
                o = ogs[i]
                t0 = o.coreindex()
                d0 = o.densest(t0, 1.0, with_cells=False)
                assert tb == t0.tobytes()
                assert res == (d0["k"], d0["lmd"], d0["length"], d0["density"])
            _same_result(merged, d)
            open(os.path.join(out_dir, "ok"), "w").write("ok")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_batch_and_columns(tmp_path):
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert (tmp_path / "ok").exists()
