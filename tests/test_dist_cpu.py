"""The multi-rank path: world_size-2 gloo ranks each count their root stripe
(u % 2 == rank) and reduce with cuts_b200.dist.reduce_counts, as bench.py
does over NCCL.  On CPU the stripes are counted by the oracle (this checks
the striping and the reduction); the gpu-marked test runs the engine's own
sharded count in two processes."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import cuts_b200 as cb


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as O
    from cuts_b200.dist import reduce_counts
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    h = cb.HostGraph.erdos_renyi(3000, 10.0 / 2999, seed=6)
    oo, oa, _, _ = h.csr()
    od = O.Graph.from_csr(h.n, oo, oa)
    counts = []
    for name in ["triangle", "4-cycle", "house"]:
        k, arcs = cb.named_query_arcs(name)
        counts.append(O.count_striped(od, O.Graph.from_arcs(k, arcs), rank, world, nthreads=2)[0])
    tot, ms = reduce_counts(counts, 10.0 * (rank + 1))
    if rank == 0:
        full = [O.count(od, O.Graph.from_arcs(*cb.named_query_arcs(nm)))[0]
                for nm in ["triangle", "4-cycle", "house"]]
        out.put((tot, ms, full))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_stripes_reduce_to_full_count():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tot, ms, full = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tot == full
    assert ms == 20.0


def test_stripes_partition_levels():
    from oracle import oracle as O
    h = cb.HostGraph.chung_lu(3000, 12000, 2.2, 2.0, 60.0, seed=3)
    oo, oa, _, _ = h.csr()
    od = O.Graph.from_csr(h.n, oo, oa)
    k, arcs = cb.named_query_arcs("house")
    q = O.Graph.from_arcs(k, arcs)
    full = O.count(od, q)
    parts = [O.count_striped(od, q, r, 3) for r in range(3)]
    assert sum(p[0] for p in parts) == full[0]
    assert [sum(p[1][i] for p in parts) for i in range(k)] == full[1]


def _engine_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from cuts_b200.dist import reduce_counts
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    g = h.upload(0)
    counts, ms = [], 0.0
    for name in ["triangle", "4-cycle", "house", "4-clique+pendant"]:
        q = cb.Query.from_arcs(*cb.named_query_arcs(name))
        for flags in (0, cb.FLAG_SYMMETRY_BREAK):
            r = g.count_sharded(q, rank, world, chunks=2, flags=flags)
            counts.append(r.count)
            ms += r.ms
    tot, mx = reduce_counts(counts, ms)
    if rank == 0:
        out.put(tot)
    g.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_engine_processes_reduce_to_oracle_count():
    """Two processes, one per rank (both on GPU 0: their kernels never wait
    on each other), each count their root stripe with the engine and reduce
    over gloo; the sums equal the oracle's full counts."""
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_engine_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tot = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    oo, oa, _, _ = h.csr()
    od = O.Graph.from_csr(h.n, oo, oa)
    want = []
    for name in ["triangle", "4-cycle", "house", "4-clique+pendant"]:
        k, arcs = cb.named_query_arcs(name)
        c = O.count(od, O.Graph.from_arcs(k, arcs))[0]
        want += [c, c]
    assert tot == want
