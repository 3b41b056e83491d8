"""cuts_count_noalloc: counting for callers that cannot allocate GPU memory.

Such a caller (code inside a framework that owns every device allocation)
holds the graph and an output buffer in its own device memory -- here torch
tensors stand in for it -- and the engine adds no allocation of its own: its
scratch is a fixed device array.  Each case calls the entry point twice in a
row through the C ABI (the second call must not see the first call's state)
and checks every count against the existing batched entry point, which
allocates its scratch normally, and against the CPU oracle.  Counts are
exact integers: equality.
"""
import ctypes as C

import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import csr_from_arcs, directed_er, oracle_graph_from_host

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


def _query(k, arcs):
    q = cb.Query.from_arcs(k, arcs)
    q.test_arcs = list(arcs)  # kept for the oracle
    return q


def _queries(seed0, n):
    qs = []
    for s in range(n):
        k = 2 + s % 5
        qs.append(_query(k, cb.random_query_arcs(k, 0.45, seed0 + s)))
    for name in ["triangle", "4-cycle", "house", "4-clique+pendant"]:
        qs.append(_query(*cb.named_query_arcs(name)))
    return qs


def _run_twice(n, info_out, info_in, adj, qs, want, stream=None):
    """Two calls in a row, on the default stream or on a caller's stream."""
    import torch
    counts = torch.full((len(qs),), -1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        if stream is None:
            cb.count_noalloc(info_out.data_ptr(), info_in.data_ptr() if info_in is not None else None,
                             adj.data_ptr(), n, qs, counts.data_ptr())
            torch.cuda.synchronize()
        else:
            with torch.cuda.stream(stream):
                cb.count_noalloc(info_out.data_ptr(), info_in.data_ptr() if info_in is not None else None,
                                 adj.data_ptr(), n, qs, counts.data_ptr(), stream=stream.cuda_stream)
            stream.synchronize()
        assert [int(x) for x in counts.cpu()] == want


def _oracle_counts(od, qs):
    out = []
    for q in qs:
        k = q.k
        out.append(O.count(od, O.Graph.from_arcs(k, q.test_arcs), q.order)[0])
    return out


def test_noalloc_matches_batched_entry_point_power_law():
    h = cb.HostGraph.chung_lu(3000, 12000, 2.2, 2.0, 60.0, seed=8)
    g = h.upload(0)
    qs = _queries(4000, 40)
    want, status, _ = g.count_batch(qs)
    assert status == [0] * len(qs)
    assert want == _oracle_counts(oracle_graph_from_host(h), qs)
    oo, oa, _, _ = h.csr()
    info_out, _, adj = _device_layout(oo, oa)
    _run_twice(h.n, info_out, None, adj, qs, want)


def test_noalloc_on_a_caller_stream_matches_oracle():
    import torch
    h = cb.HostGraph.erdos_renyi(2500, 9.0 / 2499, seed=17)
    qs = _queries(4200, 20)
    want = _oracle_counts(oracle_graph_from_host(h), qs)
    oo, oa, _, _ = h.csr()
    info_out, _, adj = _device_layout(oo, oa)
    _run_twice(h.n, info_out, None, adj, qs, want, stream=torch.cuda.Stream())


def test_noalloc_empty_inputs():
    import torch
    h = cb.HostGraph.erdos_renyi(200, 0.05, seed=1)
    oo, oa, _, _ = h.csr()
    info_out, _, adj = _device_layout(oo, oa)
    tri = cb.Query.from_arcs(*cb.named_query_arcs("triangle"))
    # nq == 0: returns OK and leaves the counts buffer as it was
    guard = torch.full((2,), 7, dtype=torch.int64, device="cuda")
    cb.count_noalloc(info_out.data_ptr(), None, adj.data_ptr(), h.n, [], guard.data_ptr())
    torch.cuda.synchronize()
    assert [int(x) for x in guard.cpu()] == [7, 7]
    # n == 0: every query counts zero
    counts = torch.full((3,), 7, dtype=torch.int64, device="cuda")
    cb.count_noalloc(info_out.data_ptr(), None, adj.data_ptr(), 0, [tri] * 3, counts.data_ptr())
    torch.cuda.synchronize()
    assert [int(x) for x in counts.cpu()] == [0, 0, 0]


def test_noalloc_matches_batched_entry_point_directed():
    n, src, dst = directed_er(1500, 12.0, seed=21)
    oo, oa, io, ia, _, _ = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    rng = np.random.default_rng(3)
    qs = []
    for t in range(24):
        k = 3 + t % 4
        und = cb.random_query_arcs(k, 0.5, 600 + t)
        qs.append(_query(k, [a for a in und if a[0] < a[1] or rng.random() < 0.6]))
    want, status, _ = g.count_batch(qs)
    od = O.Graph.from_arrays(n, src, dst)
    assert want == _oracle_counts(od, qs)
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
