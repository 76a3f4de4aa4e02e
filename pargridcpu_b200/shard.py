"""Sharding the hot path over ranks (one process per GPU).

The path needs no exchange inside its loop, so ranks share work two ways:

* whole graphs of a batch, assigned by estimated work (``assign_graphs``):
  each rank runs the batched decomposition of its own graphs, and nothing
  crosses ranks but the results;
* the lambda columns of one graph (``column_ranges``): the columns are
  independent given the graph, so each rank peels a contiguous lambda range,
  and the densest search merges the ranks' per-cell results with the
  reference's own fold (``merge_cells``).

The fold (Core/FCTree.cpp:69-82 with main.cpp:403-424) walks the cells in
preorder -- lambda-major, k ascending -- keeping a float running maximum and
replacing the best cell when ``density >= maximum`` (the later cell wins ties
and float near-ties).  Because the maximum is rounded to float after each
update, the fold is not associative: the merge gathers every rank's cells
(at most sum over lambda of kmax of them) and folds them again in order,
rather than comparing the ranks' own winners.
"""
from __future__ import annotations

import heapq

import numpy as np

__all__ = ["graph_work", "assign_graphs", "column_ranges", "fold_cells", "merge_cells",
           "gather_cells"]


def graph_work(n, L, entries):
    """Edge visits of a full fcgrid (every lambda column visits every
    directed entry once) plus the degree-table writes, as the cost model."""
    return int(entries) * int(L) + int(n) * int(L) * int(L)


def assign_graphs(works, world):
    """Rank of each graph: longest-processing-time-first onto the least
    loaded rank (ties to the lower rank).  Deterministic, so every rank
    computes the same assignment without communicating."""
    order = sorted(range(len(works)), key=lambda i: (-int(works[i]), i))
    heap = [(0, r) for r in range(world)]
    out = [0] * len(works)
    for i in order:
        load, r = heapq.heappop(heap)
        out[i] = r
        heapq.heappush(heap, (load + int(works[i]), r))
    return out


def column_ranges(L, world):
    """Contiguous lambda ranges [lo, hi) (1-based lambda, hi exclusive), one
    per rank, sizes differing by at most one; ranks beyond L get empty
    ranges."""
    out = []
    base, extra = divmod(L, world)
    lo = 1
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def fold_cells(cells):
    """The reference's fold over cells (k, lmd, length, lstar, density), in
    preorder.  Returns the winning cell's fields and the float maximum."""
    best = dict(k=0, lmd=0, length=0, lstar=0, density=0.0)
    maxf = np.float32(0.0)
    for c in sorted(cells, key=lambda c: (c[1], c[0])):
        d = float(c[4])
        if d >= float(maxf):
            maxf = np.float32(d)
            best = dict(k=int(c[0]), lmd=int(c[1]), length=int(c[2]), lstar=int(c[3]), density=d)
    best["max_density_f"] = float(maxf)
    return best


def merge_cells(per_rank):
    """Fold of the cells of all ranks (each rank's list for its own lambda
    range, in any order)."""
    return fold_cells([c for cells in per_rank for c in cells])


def gather_cells(cells, group=None):
    """All ranks' cells on every rank (torch.distributed all_gather_object),
    then the merged fold."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    out = [None] * world
    dist.all_gather_object(out, list(cells), group=group)
    return merge_cells(out)
