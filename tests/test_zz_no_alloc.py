"""fc_coreindex_fixed_scratch through the C ABI.

This entry point serves callers that cannot allocate device memory -- an
application whose memory manager already holds the whole device, or a
latency-bound loop that cannot take the stall of a device allocation.  They
pass a graph and an output table in device memory they own; the library's
scratch comes from one fixed 64 MiB device array.  Its table must equal the
one fc_coreindex (the allocating path) returns, call after call, since every
call reuses the same scratch.

The caller's device buffers here are made by torch: the test plays the part
of such a caller, which owns its memory."""
import ctypes as C

import numpy as np
import pytest

from pargridcpu_b200 import MultilayerGraph, native, synth

pytestmark = pytest.mark.gpu

FC_OK, FC_ERR_INVALID, FC_ERR_TOO_LARGE = 0, 7, 8


def node_major(g):
    """The kernels' input layout from the host CSR: node_ptr[n+1], slots
    u*L + l (node-major rows, layers in order) and deg0[n*L]."""
    off, adj = g.csr()
    n, L = g.n, g.L
    deg = (off[:, 1:] - off[:, :-1]).astype(np.int64)          # (L, n)
    deg0 = np.ascontiguousarray(deg.T)                          # (n, L)
    node_ptr = np.zeros(n + 1, np.int64)
    node_ptr[1:] = np.cumsum(deg0.sum(axis=1))
    within = np.cumsum(deg0, axis=1) - deg0                     # offset of layer l in row v
    slots = np.empty(int(node_ptr[-1]), np.uint32)
    for l in range(L):
        lo, hi = int(off[l, 0]), int(off[l, n])
        owner = np.repeat(np.arange(n), deg[l])
        j = np.arange(hi - lo) - (off[l, owner].astype(np.int64) - lo)
        slots[node_ptr[owner] + within[owner, l] + j] = adj[lo:hi].astype(np.uint32) * L + l
    return node_ptr.astype(np.uint32), slots, deg0.reshape(-1).astype(np.uint32)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _call(n, L, entries, d_ptr, d_adj, d_deg0, d_out):
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    return native.lib().fc_coreindex_fixed_scratch(n, L, entries, vp(d_ptr), vp(d_adj),
                                                   vp(d_deg0), vp(d_out), None)


def test_fixed_scratch_matches_allocating_path():
    import torch
    # two column groups: the six columns do not all fit the 64 MiB at once
    gen = synth.chung_lu_graph(200_000, 6, 200_000, 2.2, 0.4, 9090)
    g = MultilayerGraph.from_pairs(gen.layers)
    ref = g.coreindex()
    node_ptr, slots, deg0 = node_major(g)
    d_ptr, d_adj, d_deg0 = _dev(node_ptr), _dev(slots), _dev(deg0)
    out = torch.empty((g.L, g.n), dtype=torch.int32, device="cuda")
    for call in range(2):
        out.fill_(-1 - call)  # stale contents must not leak into the result
        rc = _call(g.n, g.L, len(slots), d_ptr, d_adj, d_deg0, out)
        torch.cuda.synchronize()
        assert rc == FC_OK, native.STATUS.get(rc, rc)
        got = out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, ref), f"call {call}"


def test_fixed_scratch_deep_graph_with_long_rows():
    """Cores up to 69 and rows of up to 42,012 entries in the caller's own
    (unordered) layout: past level 16 long rows are visited strided, which
    must not depend on the rows being ordered."""
    import torch
    gen = synth.chung_lu_graph(30_000, 4, 240_000, 2.1, 0.5, 9092)
    g = MultilayerGraph.from_pairs(gen.layers)
    ref = g.coreindex()
    assert ref.max() > 16
    node_ptr, slots, deg0 = node_major(g)
    assert np.diff(node_ptr.astype(np.int64)).max() > 512
    d_ptr, d_adj, d_deg0 = _dev(node_ptr), _dev(slots), _dev(deg0)
    out = torch.empty((g.L, g.n), dtype=torch.int32, device="cuda")
    rc = _call(g.n, g.L, len(slots), d_ptr, d_adj, d_deg0, out)
    torch.cuda.synchronize()
    assert rc == FC_OK, native.STATUS.get(rc, rc)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_fixed_scratch_small_graph_twice():
    import torch
    gen = synth.erdos_renyi_graph(120, 40, 0.02, 0.1, 9091)
    g = MultilayerGraph.from_pairs(gen.layers)
    ref = g.coreindex()
    node_ptr, slots, deg0 = node_major(g)
    d_ptr, d_adj, d_deg0 = _dev(node_ptr), _dev(slots), _dev(deg0)
    out = torch.empty((g.L, g.n), dtype=torch.int32, device="cuda")
    for call in range(2):
        out.fill_(12345)
        assert _call(g.n, g.L, len(slots), d_ptr, d_adj, d_deg0, out) == FC_OK
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_fixed_scratch_rejects_oversize():
    import torch
    tiny = torch.zeros(16, dtype=torch.int32, device="cuda")
    # one column of 50M nodes x 8 layers needs far more than 64 MiB: rejected
    # on the host, before anything reads these (too small) buffers
    assert _call(50_000_000, 8, 1000, tiny, tiny, tiny, tiny) == FC_ERR_TOO_LARGE


def test_fixed_scratch_allocates_nothing():
    """The property the entry point exists for: once a device is set up (its
    first call), calls create no device or pinned allocation, stream or
    event (the library's own count) and take no device memory."""
    import torch
    gen = synth.chung_lu_graph(20_000, 5, 60_000, 2.3, 0.4, 9093)
    g = MultilayerGraph.from_pairs(gen.layers)
    ref = g.coreindex()
    node_ptr, slots, deg0 = node_major(g)
    d_ptr, d_adj, d_deg0 = _dev(node_ptr), _dev(slots), _dev(deg0)
    out = torch.empty((g.L, g.n), dtype=torch.int32, device="cuda")
    assert _call(g.n, g.L, len(slots), d_ptr, d_adj, d_deg0, out) == FC_OK  # set-up call
    torch.cuda.synchronize()
    allocs = native.lib().fc_alloc_count()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        out.fill_(7)
        assert _call(g.n, g.L, len(slots), d_ptr, d_adj, d_deg0, out) == FC_OK
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
    assert native.lib().fc_alloc_count() == allocs
    assert torch.cuda.mem_get_info()[0] == free0


def test_fixed_scratch_rejects_a_malformed_csr():
    """A CSR the peel could not index safely is refused on the device before
    the peel runs, and the next well-formed call is unaffected."""
    import torch
    gen = synth.erdos_renyi_graph(150, 12, 0.02, 0.1, 9094)
    g = MultilayerGraph.from_pairs(gen.layers)
    ref = g.coreindex()
    node_ptr, slots, deg0 = node_major(g)
    n, L, e = g.n, g.L, len(slots)
    out = torch.empty((L, n), dtype=torch.int32, device="cuda")
    bad_slot = slots.copy()
    bad_slot[e // 2] = n * L            # names no degree counter
    bad_ptr = node_ptr.copy()
    bad_ptr[n // 2] = bad_ptr[n // 2 + 1] + 1  # a row of negative length
    short_ptr = node_ptr.copy()
    short_ptr[n] = e - 1                # ends before the entries do
    for p, s_ in ((node_ptr, bad_slot), (bad_ptr, slots), (short_ptr, slots)):
        rc = _call(n, L, e, _dev(p), _dev(s_), _dev(deg0), out)
        torch.cuda.synchronize()
        assert rc == FC_ERR_INVALID
    assert _call(n, L, e, _dev(node_ptr), _dev(slots), _dev(deg0), out) == FC_OK
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
