"""cuts_count_noalloc: counting for callers that cannot allocate GPU memory.

Such a caller (code inside a framework that owns every device allocation)
holds the graph and an output buffer in its own device memory -- here torch
tensors stand in for it -- and the engine adds no allocation of its own: its
scratch is a fixed device array.  Each case calls the entry point twice in a
row through the C ABI (the second call must not see the first call's state)
and checks every count against the existing batched entry point, which
allocates its scratch normally.  Counts are exact integers: equality.
"""
import ctypes as C

import numpy as np
import pytest

import cuts_b200 as cb
from tests.helpers import csr_from_arcs, directed_er

pytestmark = pytest.mark.gpu


def _device_layout(oo, oa, io=None, ia=None):
    """info (u32 pairs: offset, length) and adjacency as device tensors."""
    import torch

    def info(off):
        off = off.astype(np.int64)
        return torch.from_numpy(np.stack([off[:-1], np.diff(off)], 1).astype(np.int32).copy()).cuda()

    adj_all = oa.astype(np.uint32)
    io_t = None
    if io is not None:
        shift = np.int64(len(oa))
        adj_all = np.concatenate([oa, ia]).astype(np.uint32)
        io_t = info(io.astype(np.int64) + shift)
    adj = torch.from_numpy(adj_all.view(np.int32).copy()).cuda()
    return info(oo), io_t, adj


def _queries(seed0, n):
    qs = []
    for s in range(n):
        k = 2 + s % 5
        qs.append(cb.Query.from_arcs(k, cb.random_query_arcs(k, 0.45, seed0 + s)))
    for name in ["triangle", "4-cycle", "house", "4-clique+pendant"]:
        qs.append(cb.Query.from_arcs(*cb.named_query_arcs(name)))
    return qs


def _run_twice(n, info_out, info_in, adj, qs, want):
    import torch
    counts = torch.full((len(qs),), -1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        cb.count_noalloc(info_out.data_ptr(), info_in.data_ptr() if info_in is not None else None,
                         adj.data_ptr(), n, qs, counts.data_ptr())
        torch.cuda.synchronize()
        assert [int(x) for x in counts.cpu()] == want


def test_noalloc_matches_batched_entry_point_power_law():
    h = cb.HostGraph.chung_lu(3000, 12000, 2.2, 2.0, 60.0, seed=8)
    g = h.upload(0)
    qs = _queries(4000, 40)
    want, status, _ = g.count_batch(qs)
    assert status == [0] * len(qs)
    oo, oa, _, _ = h.csr()
    info_out, _, adj = _device_layout(oo, oa)
    _run_twice(h.n, info_out, None, adj, qs, want)


def test_noalloc_matches_batched_entry_point_directed():
    n, src, dst = directed_er(1500, 12.0, seed=21)
    oo, oa, io, ia, _, _ = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    rng = np.random.default_rng(3)
    qs = []
    for t in range(24):
        k = 3 + t % 4
        und = cb.random_query_arcs(k, 0.5, 600 + t)
        qs.append(cb.Query.from_arcs(k, [a for a in und if a[0] < a[1] or rng.random() < 0.6]))
    want, status, _ = g.count_batch(qs)
    info_out, info_in, adj = _device_layout(oo, oa, io, ia)
    _run_twice(n, info_out, info_in, adj, qs, want)


def test_noalloc_rejects_beyond_limits():
    import torch
    h = cb.HostGraph.erdos_renyi(200, 0.05, seed=1)
    oo, oa, _, _ = h.csr()
    info_out, _, adj = _device_layout(oo, oa)
    counts = torch.zeros(70, dtype=torch.int64, device="cuda")
    tri = cb.Query.from_arcs(*cb.named_query_arcs("triangle"))
    with pytest.raises(cb.CutsError) as e:
        cb.count_noalloc(info_out.data_ptr(), None, adj.data_ptr(), h.n, [tri] * 65, counts.data_ptr())
    assert e.value.code == cb.ERR_LIMIT
    big = cb.Query.from_arcs(11, [(a, b) for a in range(11) for b in range(11) if a != b])
    with pytest.raises(cb.CutsError) as e:
        cb.count_noalloc(info_out.data_ptr(), None, adj.data_ptr(), h.n, [big], counts.data_ptr())
    assert e.value.code == cb.ERR_LIMIT
    with pytest.raises(cb.CutsError) as e:
        cb.count_noalloc(info_out.data_ptr(), None, adj.data_ptr(), h.n, [tri], counts.data_ptr(),
                         flags=cb.FLAG_SYMMETRY_BREAK)
    assert e.value.code == cb.ERR_ARG
