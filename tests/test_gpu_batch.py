"""Batched engine on a GPU: per-query counts of one persistent launch (replayed
from its CUDA graph) against the CPU oracle, plus the time-budget status."""
import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import csr_from_arcs, directed_er, oracle_graph_from_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pl():
    h = cb.HostGraph.chung_lu(3000, 12000, 2.2, 2.0, 60.0, seed=8)
    return h, h.upload(0), oracle_graph_from_host(h)


def _queries(n, seed0):
    out = []
    for s in range(n):
        k = 3 + (s * 7 + seed0) % 3
        p = [0.3, 0.45, 0.6][s % 3]
        out.append((k, cb.random_query_arcs(k, p, seed0 + s)))
    return out


_WANT = {}


@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK])
def test_batch_counts_match_oracle(pl, flags):
    h, g, od = pl
    qdefs = _queries(48, 500)
    qs = [cb.Query.from_arcs(k, a) for k, a in qdefs]
    if "pl48" not in _WANT:
        _WANT["pl48"] = [O.count(od, O.Graph.from_arcs(k, a))[0] for k, a in qdefs]
    want = _WANT["pl48"]
    b = g.batch(qs, flags=flags)
    for rep in range(2):  # second run replays the captured graph
        counts, status, ms = b.run()
        assert status == [0] * len(qs)
        assert counts == want


@pytest.mark.parametrize("grain,grab,bps", [(1, 1, 0), (7, 3, 1), (256, 8, 2)])
def test_batch_tuning_does_not_change_counts(pl, grain, grab, bps):
    h, g, od = pl
    qdefs = _queries(16, 900)
    qs = [cb.Query.from_arcs(k, a) for k, a in qdefs]
    want = [g.count(q).count for q in qs]
    counts, status, _ = g.batch(qs, grain=grain, tasks_per_grab=grab, blocks_per_sm=bps).run()
    assert counts == want and status == [0] * len(qs)


def test_batch_named_and_edge_cases(pl):
    h, g, od = pl
    names = ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant", "3-prism", "6-cycle"]
    qs = [cb.Query.from_arcs(*cb.named_query_arcs(nm)) for nm in names]
    # an edge (k = 2), a 6-clique (no match at all), and an 11-clique (beyond
    # the batched kernel's 10 vertices: counted by the level engine; its
    # levels die out after a few steps in a sparse graph)
    qs.append(cb.Query.from_arcs(2, [(0, 1), (1, 0)]))
    clique = [(a, b) for a in range(6) for b in range(6) if a != b]
    qs.append(cb.Query.from_arcs(6, clique))
    clique11 = [(a, b) for a in range(11) for b in range(11) if a != b]
    qs.append(cb.Query.from_arcs(11, clique11))
    want = [g.count(q).count for q in qs]
    counts, status, _ = g.count_batch(qs)
    assert counts == want and status == [0] * len(qs)
    assert counts[-3] == h.info()[1]  # the edge query: every arc


def test_batch_directed():
    n, src, dst = directed_er(1200, 12.0, seed=13)
    oo, oa, io, ia, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    od = O.Graph.from_arrays(n, s, d)
    rng = np.random.default_rng(1)
    qdefs = []
    for t in range(20):
        k = 3 + t % 4
        und = cb.random_query_arcs(k, 0.5, 300 + t)
        qdefs.append((k, [a for a in und if a[0] < a[1] or rng.random() < 0.6]))
    qs = [cb.Query.from_arcs(k, a) for k, a in qdefs]
    want = [O.count(od, O.Graph.from_arcs(k, a))[0] for k, a in qdefs]
    counts, status, _ = g.count_batch(qs)
    assert counts == want


def test_batch_budget_marks_unfinished():
    """A tiny device-time budget ends the launch; unfinished queries say so,
    finished ones keep exact counts, and the graph stays usable."""
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    g = h.upload(0)
    qs = [cb.Query.from_arcs(*cb.named_query_arcs("5-cycle")) for _ in range(8)]
    b = g.batch(qs)
    counts, status, ms = b.run(budget_ms=0.05)
    assert any(s == cb.ERR_BUDGET for s in status)
    full, st2, _ = b.run()
    assert st2 == [0] * len(qs) and len(set(full)) == 1
    for c, s in zip(counts, status):
        if s == 0:
            assert c == full[0]
    assert g.count(qs[0]).count == full[0]


def test_level_engine_budget():
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    g = h.upload(0)
    g.set_level_cap(4096)  # many chunks, so the budget is checked often
    q = cb.Query.from_arcs(*cb.named_query_arcs("house"))
    r, done = g.count_budget(q, 0.001)
    assert not done
    g.set_level_cap(0)
    r, done = g.count_budget(q, 0.0)
    assert done and r.count == g.count(q).count


def test_level_engine_device_budget():
    """One large chunk: the kernels' own deadline stops the run well before
    the work would end (the host check between chunks never runs)."""
    import time
    h = cb.HostGraph.chung_lu(20000, 80000, 2.1, 2.0, 2000.0, seed=9)
    g = h.upload(0)
    q = cb.Query.from_arcs(*cb.named_query_arcs("6-cycle"))
    sample, sdone = g.count_sample(q, 0, 64, budget_ms=5000.0)
    full_est_ms = sample.ms * 64 if sdone else 5000.0 * 64
    assert full_est_ms > 200  # the whole count takes far longer than the budget
    t = time.perf_counter()
    r, done = g.count_budget(q, 20.0, chunks=1)
    wall = time.perf_counter() - t
    assert not done
    assert wall < 0.5 * full_est_ms / 1e3 + 0.1
    # a budget the run fits in: exact (a root stripe, to stay short)
    if sdone:
        r2, done2 = g.count_sample(q, 0, 64, budget_ms=1e7)
        assert done2 and r2.count == sample.count


def test_batch_query_budget_drops_only_the_heavy_query():
    """A per-query limit: the heavy query placed first is dropped once it has
    used its share, the cheap ones behind it finish with exact counts."""
    h = cb.HostGraph.chung_lu(20000, 80000, 2.1, 2.0, 2000.0, seed=9)
    g = h.upload(0)
    # a 7-vertex path: ~1e15 embeddings around the degree-2,000 hubs
    path7 = [(a, b) for i in range(6) for a, b in ((i, i + 1), (i + 1, i))]
    heavy = cb.Query.from_arcs(7, path7)
    cheap = [cb.Query.from_arcs(*cb.named_query_arcs(n)) for n in ("triangle", "4-clique+pendant", "triangle")]
    b = g.batch([heavy] + cheap)
    b.set_query_budget(200.0)
    counts, status, ms = b.run()
    assert status[0] == cb.ERR_BUDGET
    assert status[1:] == [0, 0, 0]
    for c, q in zip(counts[1:], cheap):
        assert c == g.count(q).count
    b.set_query_budget(0.0)
    b2 = g.batch(cheap)
    c2, s2, _ = b2.run()
    assert s2 == [0, 0, 0] and c2 == counts[1:]


def test_batch_shards_partition_every_query():
    """One launch per shard (as one per GPU): the per-query counts of the
    shards add up to the unsharded counts, for every shard count."""
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    g = h.upload(0)
    qs = [cb.Query.from_arcs(*cb.named_query_arcs(n)) for n in ("triangle", "4-cycle", "house", "4-clique+pendant")]
    qs += [cb.Query.from_arcs(k, cb.random_query_arcs(k, 0.4, 70 + k)) for k in (3, 4, 5)]
    full, st, _ = g.batch(qs).run()
    assert st == [0] * len(qs)
    for nshards in (2, 3, 7):
        tot = [0] * len(qs)
        for r in range(nshards):
            b = g.batch(qs)
            b.set_shard(r, nshards)
            c, s, _ = b.run()
            assert s == [0] * len(qs)
            tot = [a + x for a, x in zip(tot, c)]
        assert tot == full
    with pytest.raises(cb.CutsError):
        g.batch(qs).set_shard(3, 3)


@pytest.mark.parametrize("name,flags", [("triangle", 0), ("4-clique+pendant", cb.FLAG_SYMMETRY_BREAK),
                                        ("house", 0)])
def test_count_autotuner(name, flags):
    """The level engine's chunk / tile tuner: every configuration gives the
    oracle's count, the best one is kept on the graph and reproduces it."""
    from cuts_b200 import autotune
    from oracle import oracle as O
    from tests.helpers import oracle_graph_from_host
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    g = h.upload(0)
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    best, times = autotune.tune_count(g, q, flags=flags, chunks=(1, 3), splits=(8, 64, 256),
                                      level_caps=(0, 4096), reps=2)
    assert len(times) == 2 * 3 * 2 and best in times and times[best] == min(times.values())
    want = O.count(oracle_graph_from_host(h), O.Graph.from_arcs(k, arcs), q.order)[0]
    assert g.count(q, chunks=best[0], flags=flags).count == want


@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK])
def test_batch_routes_fused_queries_to_the_level_engine(pl, flags, monkeypatch):
    """Queries of 4+ vertices whose count the level engine fuses (or
    orbit-folds) leave the persistent launch; the counts are the same either
    way and equal the oracle's."""
    h, g, od = pl
    names = ["4-clique+pendant", "house", "4-cycle", "triangle"]
    qdefs = [cb.named_query_arcs(nm) for nm in names] + _queries(12, 4400)
    qs = [cb.Query.from_arcs(k, a) for k, a in qdefs]
    want = [O.count(od, O.Graph.from_arcs(k, a))[0] for k, a in qdefs]
    routed = g.batch(qs, flags=flags)
    monkeypatch.setenv("CUTS_BATCH_ROUTE", "0")
    kept = g.batch(qs, flags=flags)
    c1, s1, _ = routed.run()
    c2, s2, _ = kept.run()
    assert s1 == s2 == [0] * len(qs)
    assert c1 == c2 == want
    assert routed.info()[0] < kept.info()[0]  # fewer tasks in the launch
