"""The multi-GPU host path on CPU: world_size-2 gloo ranks each count their
root stripe (u % 2 == rank, computed here by the oracle in place of a GPU)
and reduce with cuts_b200.dist.reduce_counts, as bench.py does over NCCL."""
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
