"""Engine counts vs the CPU oracle on the same seeded inputs (bit-exact).

Every case compares the total count and, where the order is the same, every
per-level table size |L_i| (which pins the per-level semantics, not only the
final number).
"""
import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import csr_from_arcs, directed_er, oracle_graph_from_host

pytestmark = pytest.mark.gpu

NAMED = ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant", "3-prism", "6-cycle"]


@pytest.fixture(scope="module")
def er2k():
    h = cb.HostGraph.erdos_renyi(2000, 10.0 / 1999, seed=3)
    return h, h.upload(0), oracle_graph_from_host(h)


@pytest.fixture(scope="module")
def cl5k():
    # power law, exponent 2.1, degree cap 100: 5-cycles ~3.5e7, 6-cycles ~1.1e9
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    return h, h.upload(0), oracle_graph_from_host(h)


_ORACLE = {}


def oracle_count(od, k, arcs, order):
    # the entry keeps its graph alive, so an id is never reused for another graph
    key = (id(od), k, tuple(arcs), tuple(order))
    if key not in _ORACLE or _ORACLE[key][0] is not od:
        _ORACLE[key] = (od, O.count(od, O.Graph.from_arcs(k, arcs), order))
    return _ORACLE[key][1]


def _check(g, od, k, arcs, flags=0, chunks=1, levels=True):
    q = cb.Query.from_arcs(k, arcs)
    cnt, lv, _ = oracle_count(od, k, arcs, q.order)
    r = g.count(q, chunks=chunks, flags=flags, stats=True)
    assert r.count == cnt
    if levels:
        assert r.level_sizes == lv
    return cnt


@pytest.mark.parametrize("name", NAMED)
def test_named_er(er2k, name):
    h, g, od = er2k
    k, arcs = cb.named_query_arcs(name)
    _check(g, od, k, arcs)


PL_NAMED = ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant", "3-prism"]


@pytest.mark.parametrize("name", PL_NAMED)
def test_named_power_law(cl5k, name):
    h, g, od = cl5k
    k, arcs = cb.named_query_arcs(name)
    _check(g, od, k, arcs)


@pytest.mark.parametrize("seed", range(12))
def test_random_queries(er2k, seed):
    h, g, od = er2k
    k = 4 + seed % 4
    arcs = cb.random_query_arcs(k, 0.3, seed)
    _check(g, od, k, arcs)


@pytest.mark.parametrize("name", ["4-cycle", "house", "5-cycle"])
def test_forced_chunking(er2k, name):
    """A tiny level capacity forces the planner to cut every level."""
    h, g, od = er2k
    k, arcs = cb.named_query_arcs(name)
    g.set_level_cap(1024)
    try:
        q = cb.Query.from_arcs(k, arcs)
        r = g.count(q, stats=True)
        cnt, lv, _ = O.count(od, O.Graph.from_arcs(k, arcs), q.order)
        assert r.count == cnt and r.level_sizes == lv
        assert r.chunks > k  # really chunked
    finally:
        g.set_level_cap(0)


@pytest.mark.parametrize("trunks", [1, 2, 4, 7])
def test_trunks(er2k, trunks):
    h, g, od = er2k
    k, arcs = cb.named_query_arcs("house")
    _check(g, od, k, arcs, chunks=trunks)


@pytest.mark.parametrize("name", PL_NAMED)
def test_symmetry_breaking(cl5k, name):
    h, g, od = cl5k
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    cnt, _, _ = oracle_count(od, k, arcs, q.order)
    assert g.count(q, flags=cb.FLAG_SYMMETRY_BREAK).count == cnt


def test_heavy_count_engines_agree(cl5k):
    """6-cycles (~1e9 embeddings, beyond the oracle's seconds): the level
    engine, the level engine with symmetry breaking, chunked, and the
    depth-first batched engine are independent paths and must agree."""
    h, g, od = cl5k
    q = cb.Query.from_arcs(*cb.named_query_arcs("6-cycle"))
    a = g.count(q).count
    assert a > 10**8
    assert g.count(q, flags=cb.FLAG_SYMMETRY_BREAK).count == a
    assert g.count(q, chunks=5).count == a
    counts, status, _ = g.count_batch([q, q])
    assert counts == [a, a] and status == [0, 0]


@pytest.mark.parametrize("name", ["triangle", "4-clique+pendant", "5-cycle"])
def test_no_closed_form(er2k, name):
    h, g, od = er2k
    k, arcs = cb.named_query_arcs(name)
    _check(g, od, k, arcs, flags=cb.FLAG_NO_CLOSED_FORM)


def test_directed_graph_and_queries():
    n, src, dst = directed_er(1500, 14.0, seed=11)
    oo, oa, io, ia, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    assert not g.info()[2]
    od = O.Graph.from_arrays(n, s, d)
    rng = np.random.default_rng(0)
    for t in range(10):
        k = 3 + t % 4
        und = cb.random_query_arcs(k, 0.5, 100 + t)
        # orient: keep each arc with prob 0.7 but keep the query connected
        arcs = [a for a in und if rng.random() < 0.7 or a[0] < a[1]]
        _check(g, od, k, arcs)


def test_self_loops():
    """Self-loops in the data graph count in degrees; a query self-loop is
    only a signature constraint, as in the reference."""
    n = 300
    h = cb.HostGraph.erdos_renyi(n, 0.05, seed=2)
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(oo.astype(np.int64)))
    loops = np.arange(0, n, 3, dtype=np.uint32)
    src = np.concatenate([src, loops])
    dst = np.concatenate([oa, loops])
    oo2, oa2, io2, ia2, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo2, oa2, io2, ia2)
    od = O.Graph.from_arrays(n, s, d)
    k, arcs = cb.named_query_arcs("triangle")
    _check(g, od, k, arcs)
    _check(g, od, 3, arcs + [(2, 2)])
    _check(g, od, 3, arcs + [(0, 0)])


def test_small_queries_and_empty():
    h = cb.HostGraph.erdos_renyi(500, 0.02, seed=9)
    g = h.upload(0)
    od = oracle_graph_from_host(h)
    # one vertex: the reference reports 0 (count only added at iter == k-1 >= 1)
    q1 = cb.Query.from_arcs(1, [])
    assert g.count(q1).count == 0
    # one edge: every arc
    cnt = _check(g, od, 2, [(0, 1), (1, 0)])
    assert cnt == h.info()[1]
    # no match: 6-clique in a sparse graph
    edges = [(a, b) for a in range(6) for b in range(6) if a != b]
    assert g.count(cb.Query.from_arcs(6, edges)).count == 0
    # empty data graph
    e = cb.HostGraph.erdos_renyi(50, 0.0, seed=0).upload(0)
    assert e.count(cb.Query.from_arcs(3, cb.named_query_arcs("triangle")[1])).count == 0


def test_known_answers():
    """Closed forms: K_n holds n!/(n-k)! embeddings of any k-vertex
    connected symmetric query; a star K_{1,s} (s >= 2) in K_{1,d} has
    d!/(d-s)! (the centre must map to the centre)."""
    import math
    n = 9
    edges = [(a, b) for a in range(n) for b in range(n) if a != b]
    src = np.array([a for a, _ in edges], np.uint32)
    dst = np.array([b for _, b in edges], np.uint32)
    oo, oa, io, ia, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa)
    for name in NAMED:
        k, arcs = cb.named_query_arcs(name)
        want = math.factorial(n) // math.factorial(n - k)
        assert g.count(cb.Query.from_arcs(k, arcs)).count == want
        assert g.count(cb.Query.from_arcs(k, arcs), flags=cb.FLAG_SYMMETRY_BREAK).count == want
    dstar = 12
    sedges = [(0, i) for i in range(1, dstar + 1)]
    sarcs = sedges + [(b, a) for a, b in sedges]
    s2 = np.array([a for a, _ in sarcs], np.uint32)
    d2 = np.array([b for _, b in sarcs], np.uint32)
    oo, oa, _, _, _, _ = csr_from_arcs(dstar + 1, s2, d2)
    g = cb.Graph.from_csr(dstar + 1, oo, oa)
    for s_ in (2, 3, 4):
        qarcs = [(0, i) for i in range(1, s_ + 1)] + [(i, 0) for i in range(1, s_ + 1)]
        want = math.factorial(dstar) // math.factorial(dstar - s_)
        assert g.count(cb.Query.from_arcs(s_ + 1, qarcs)).count == want


@pytest.mark.parametrize("name", ["triangle", "house", "4-clique+pendant"])
def test_sharded_counts_sum(cl5k, name):
    """Root stripes u % N == r partition the count and every level."""
    h, g, od = cl5k
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    full = g.count(q, stats=True)
    parts = [g.count_sharded(q, r, 3) for r in range(3)]
    assert sum(p.count for p in parts) == full.count
    assert [sum(p.level_sizes[i] for p in parts) for i in range(k)] == full.level_sizes


# queries whose last vertex hangs off an earlier one: the last level is a
# closed form and folds into level k-2 (unless a symmetry condition ties it
# to the penultimate vertex)
FOLD_QUERIES = {
    "star3": (4, [(0, 1), (1, 0), (0, 2), (2, 0), (0, 3), (3, 0)]),
    "tailed-triangle": (4, [(0, 1), (1, 0), (1, 2), (2, 1), (2, 0), (0, 2), (0, 3), (3, 0)]),
    "4-clique+pendant": cb.named_query_arcs("4-clique+pendant"),
    "path4": (4, [(0, 1), (1, 0), (1, 2), (2, 1), (2, 3), (3, 2)]),
    "directed-fan": (4, [(0, 1), (1, 2), (2, 0), (0, 3)]),
}


@pytest.mark.parametrize("name", sorted(FOLD_QUERIES))
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK, cb.FLAG_NO_CLOSED_FORM])
def test_fold_and_guaranteed_members(er2k, cl5k, name, flags):
    k, arcs = FOLD_QUERIES[name]
    for h, g, od in (er2k, cl5k):
        q = cb.Query.from_arcs(k, arcs)
        cnt, lv, _ = oracle_count(od, k, arcs, q.order)
        r = g.count(q, flags=flags, stats=True)
        assert r.count == cnt
        if flags != cb.FLAG_SYMMETRY_BREAK:
            assert r.level_sizes == lv
        r4 = g.count(q, flags=flags, chunks=3)
        assert r4.count == cnt


FUSE_QUERIES = {
    "triangle": cb.named_query_arcs("triangle"),
    "4-clique": (4, [(a, b) for a in range(4) for b in range(4) if a != b]),
    "5-clique": (5, [(a, b) for a in range(5) for b in range(5) if a != b]),
    "4-clique+pendant": cb.named_query_arcs("4-clique+pendant"),
    "diamond": (4, [(0, 1), (1, 0), (0, 2), (2, 0), (1, 2), (2, 1), (1, 3), (3, 1), (2, 3), (3, 2)]),
    "house": cb.named_query_arcs("house"),
    "directed-triangle-mixed": (3, [(0, 1), (1, 2), (0, 2), (2, 0)]),
    "directed-4-clique": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (3, 1)]),
}


@pytest.mark.parametrize("name", sorted(FUSE_QUERIES))
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK])
def test_fused_levels(er2k, cl5k, name, flags):
    """The counted level fused with the one before (per-parent candidate sets
    in scratch) against the oracle, levels included, and against the unfused
    plan; directed queries on a directed graph too."""
    k, arcs = FUSE_QUERIES[name]
    graphs = [er2k, cl5k]
    if name.startswith("directed"):
        n, src, dst = directed_er(1500, 14.0, seed=11)
        oo, oa, io, ia, s_, d_ = csr_from_arcs(n, src, dst)
        graphs = [(None, cb.Graph.from_csr(n, oo, oa, io, ia), O.Graph.from_arrays(n, s_, d_))]
    for h, g, od in graphs:
        q = cb.Query.from_arcs(k, arcs)
        cnt, lv, _ = oracle_count(od, k, arcs, q.order)
        r = g.count(q, flags=flags, stats=True)
        assert r.count == cnt
        if flags == 0:
            assert r.level_sizes == lv
        assert g.count(q, flags=flags | cb.FLAG_NO_FUSE).count == cnt
        assert g.count(q, flags=flags, chunks=5).count == cnt


def test_fused_with_forced_chunking(cl5k):
    h, g, od = cl5k
    k, arcs = cb.named_query_arcs("4-clique+pendant")
    q = cb.Query.from_arcs(k, arcs)
    cnt, lv, _ = oracle_count(od, k, arcs, q.order)
    g.set_level_cap(2048)
    try:
        r = g.count(q, stats=True)
        assert r.count == cnt and r.level_sizes == lv
    finally:
        g.set_level_cap(0)


@pytest.mark.parametrize("split", ["0", "1", "7", "40"])
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK])
def test_fused_split_parents(er2k, cl5k, monkeypatch, split, flags):
    """Parents whose candidate set exceeds the split threshold are deferred to
    the second phase (groups of 32 vertices spread over all warps); with small
    thresholds nearly every parent goes there, and with threshold 0 on the
    power-law graph the saved-set pool runs out, so the in-place fallback is
    taken too.  Counts and level sizes against the oracle."""
    monkeypatch.setenv("CUTS_FUSE_SPLIT", split)
    for name in ("triangle", "4-clique", "4-clique+pendant", "diamond", "house"):
        k, arcs = FUSE_QUERIES[name]
        for h, g, od in (er2k, cl5k):
            q = cb.Query.from_arcs(k, arcs)
            cnt, lv, _ = oracle_count(od, k, arcs, q.order)
            r = g.count(q, flags=flags, stats=True)
            assert r.count == cnt, (name, split)
            if flags == 0:
                assert r.level_sizes == lv, (name, split)


def test_fused_split_directed(monkeypatch):
    monkeypatch.setenv("CUTS_FUSE_SPLIT", "3")
    n, src, dst = directed_er(1500, 14.0, seed=11)
    oo, oa, io, ia, s_, d_ = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    od = O.Graph.from_arrays(n, s_, d_)
    for name in ("directed-triangle-mixed", "directed-4-clique"):
        k, arcs = FUSE_QUERIES[name]
        q = cb.Query.from_arcs(k, arcs)
        cnt, lv, _ = oracle_count(od, k, arcs, q.order)
        r = g.count(q, stats=True)
        assert r.count == cnt and r.level_sizes == lv


def test_fused_hub_graph_matches_unfused():
    """A graph with hubs of degree > 256 (the default split threshold): the
    fused plan, with its deferred hub parents, against the unfused plan."""
    h = cb.HostGraph.chung_lu(20000, 80000, 2.1, 2.0, 2000.0, seed=9)
    g = h.upload(0)
    assert h.info()[3] > 256
    for name in ("triangle", "4-clique", "4-clique+pendant", "diamond"):
        k, arcs = FUSE_QUERIES[name]
        q = cb.Query.from_arcs(k, arcs)
        for flags in (0, cb.FLAG_SYMMETRY_BREAK):
            a = g.count(q, flags=flags, stats=True)
            b = g.count(q, flags=flags | cb.FLAG_NO_FUSE, stats=True)
            assert a.count == b.count, (name, flags)
            assert a.level_sizes == b.level_sizes, (name, flags)


ORBIT_QUERIES = {
    "4-clique+pendant": cb.named_query_arcs("4-clique+pendant"),
    "5-clique+pendant": (6, [(a, b) for a in range(6) for b in range(6)
                             if a != b and (a < 5 and b < 5 or {a, b} == {0, 5})]),
    "paw": (4, [(0, 1), (1, 0), (1, 2), (2, 1), (0, 2), (2, 0), (0, 3), (3, 0)]),
    "diamond+pendant": (5, [(a, b) for u, v in [(0, 1), (0, 2), (1, 2), (1, 3), (2, 3), (1, 4)]
                            for a, b in ((u, v), (v, u))]),
    "dir3cycle+pendant": (4, [(0, 1), (1, 2), (2, 0), (0, 3)]),
}


@pytest.fixture(scope="module")
def loops_graph():
    """Symmetric ER graph with a self-loop on every third vertex."""
    n = 200
    h = cb.HostGraph.erdos_renyi(n, 0.15, seed=4)
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(oo.astype(np.int64)))
    loops = np.arange(0, n, 3, dtype=np.uint32)
    src = np.concatenate([src, loops])
    dst = np.concatenate([oa, loops])
    oo2, oa2, io2, ia2, s, d = csr_from_arcs(n, src, dst)
    return None, cb.Graph.from_csr(n, oo2, oa2, io2, ia2), O.Graph.from_arrays(n, s, d)


@pytest.mark.parametrize("name", sorted(ORBIT_QUERIES))
def test_orbit_fold(er2k, cl5k, loops_graph, monkeypatch, name):
    """Symmetry breaking on the core of a query whose last vertex is a
    pendant, weighted by the pendant's attachment orbit: counts against the
    oracle through the fused kernel, the flattened kernel (no fusion), with
    chunking, with every parent split into the fused kernel's second phase,
    and against the plan that breaks the whole query's symmetry."""
    k, arcs = ORBIT_QUERIES[name]
    q = cb.Query.from_arcs(k, arcs)
    lv, _ = q.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)
    assert lv[k - 1]["ofold"], name
    S = cb.FLAG_SYMMETRY_BREAK
    # a graph whose lowest clique vertices have no other edges: a class
    # representative puts a vertex without a pendant neighbour first
    und = ([(a, b) for a in range(5) for b in range(a + 1, 5)] + [(4, 5), (4, 6), (1, 5), (2, 5)] +
           [(9, 10), (9, 11), (10, 11), (10, 12), (10, 13)] +
           [(a, b) for a in range(14, 18) for b in range(a + 1, 18)] + [(17, 18), (17, 19)] +
           [(a, b) for a in range(20, 26) for b in range(a + 1, 26)] + [(25, 26)])
    src = np.array([a for a, b in und] + [b for a, b in und], np.uint32)
    dst = np.array([b for a, b in und] + [a for a, b in und], np.uint32)
    oo, oa, io, ia, s_, d_ = csr_from_arcs(27, src, dst)
    edge = (None, cb.Graph.from_csr(27, oo, oa, io, ia), O.Graph.from_arrays(27, s_, d_))
    for h, g, od in (er2k, cl5k, loops_graph, edge):
        cnt, _, _ = oracle_count(od, k, arcs, q.order)
        assert g.count(q, flags=S).count == cnt
        assert g.count(q, flags=S | cb.FLAG_NO_FUSE).count == cnt
        assert g.count(q, flags=S | cb.FLAG_NO_ORBIT_FOLD).count == cnt
        assert g.count(q, flags=S, chunks=3).count == cnt
        monkeypatch.setenv("CUTS_FUSE_SPLIT", "0")
        assert g.count(q, flags=S).count == cnt
        monkeypatch.delenv("CUTS_FUSE_SPLIT")


@pytest.fixture(scope="module")
def sparse5k():
    # mean degree 1.6 (arcs < 2n): the regime where the reference switches to
    # its 8-lane kernel (AVG_DEGREE = arcs / n + 2 <= 3, host_funcs.cu:33,145)
    h = cb.HostGraph.erdos_renyi(5000, 1.6 / 4999, seed=31)
    n, arcs, sym, maxd = h.info()
    assert arcs < 2 * n
    return h, h.upload(0), oracle_graph_from_host(h)


@pytest.mark.parametrize("name", ["3-path", "4-path", "5-path", "3-star", "triangle", "4-cycle"])
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK, cb.FLAG_NO_CLOSED_FORM])
def test_sparse_graph(sparse5k, name, flags):
    h, g, od = sparse5k
    k, arcs = cb.named_query_arcs(name)
    cnt = _check(g, od, k, arcs, flags=flags, chunks=3, levels=not (flags & cb.FLAG_SYMMETRY_BREAK))
    if name.endswith("path") or name.endswith("star"):
        assert cnt > 0


def _pendant_queries():
    """Queries whose last two vertices are pendants on earlier ones: stars,
    paths, a triangle with two tails on one / two vertices, random trees."""
    qs = [cb.named_query_arcs(n) for n in ("3-star", "4-path", "5-path")]
    sym = lambda es: [a for e in es for a in (e, e[::-1])]
    qs.append((5, sym([(0, 1), (1, 2), (2, 0), (0, 3), (0, 4)])))          # two tails on one vertex
    qs.append((5, sym([(0, 1), (1, 2), (2, 0), (0, 3), (1, 4)])))          # tails on two vertices
    qs.append((6, sym([(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (2, 5)])))  # square with two tails
    qs.append((5, sym([(0, 1), (0, 2), (0, 3), (0, 4)])))                  # 4-star
    for s in range(6):
        k = 5 + s % 3
        qs.append((k, cb.random_query_arcs(k, 0.0, 9100 + s)))            # random trees
    return qs


@pytest.fixture(scope="module")
def cl1k():
    # power law with degree cap 20: the 7-vertex trees below have ~1e9 matches,
    # which the oracle enumerates in a few seconds (on cl5k they take hours)
    h = cb.HostGraph.chung_lu(1000, 2500, 2.1, 2.0, 20.0, seed=5)
    return h, h.upload(0), oracle_graph_from_host(h)


@pytest.mark.parametrize("i", range(13))
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK, cb.FLAG_NO_PAIR_FOLD])
def test_pendant_pair_fold(cl1k, i, flags):
    h, g, od = cl1k
    k, arcs = _pendant_queries()[i]
    q = cb.Query.from_arcs(k, arcs)
    plan, _ = q.plan_levels(True, flags)
    cnt = _check(g, od, k, arcs, flags=flags, chunks=2, levels=not (flags & cb.FLAG_SYMMETRY_BREAK))
    assert cnt > 0
    # stars and tails of two leaves on one vertex are folded; the others
    # (pendants on two different vertices) check the unfolded plan
    folded = i in (0, 3, 6, 9, 11) and not (flags & cb.FLAG_NO_PAIR_FOLD)
    assert plan[k - 3]["fold2"] in ((1, 2) if folded else (0,))


def test_pendant_pair_fold_directed():
    n, src, dst = directed_er(1500, 14.0, seed=33)
    oo, oa, io, ia, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    od = O.Graph.from_arrays(n, s, d)
    for arcs in ([(0, 1), (1, 2), (2, 0), (0, 3), (4, 0)], [(0, 1), (1, 2), (1, 3), (3, 4), (3, 5)],
                 [(0, 1), (2, 1), (0, 3), (0, 4)]):
        k = 1 + max(max(a) for a in arcs)
        _check(g, od, k, arcs, chunks=1)
