"""The oracle's own generator, degree relabelling, ordering conditions and
count-only last level (CPU): each checked against an independent route to the
same number."""
import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import oracle_graph_from_host


@pytest.mark.parametrize("n,m,gamma,cap,seed", [(3000, 12000, 2.2, 60.0, 8), (20000, 150000, 2.1, 2000.0, 0)])
def test_oracle_generator_equals_engine_generator(n, m, gamma, cap, seed):
    h = cb.HostGraph.chung_lu(n, m, gamma, 2.0, cap, seed)
    og = O.Graph.chung_lu(n, m, gamma, 2.0, cap, seed)
    oo, oa, _, _ = h.csr()
    a, b, c, d = og.csr()
    assert np.array_equal(oo.astype(np.uint64), a) and np.array_equal(oa.astype(np.uint32), b)
    assert og.arcs == 2 * m


def test_relabel_by_degree():
    og = O.Graph.chung_lu(4000, 20000, 2.1, 2.0, 200.0, 4)
    rg, orig = og.relabel_by_degree()
    oo = og.csr()[0].astype(np.int64)
    deg = np.diff(oo)
    assert sorted(orig.tolist()) == list(range(4000))
    # ranks ascend by (degree, old id)
    keys = [(int(deg[v]), int(v)) for v in orig]
    assert keys == sorted(keys)
    ro = rg.csr()[0].astype(np.int64)
    assert np.array_equal(np.diff(ro), deg[orig])
    k, arcs = cb.named_query_arcs("house")
    assert O.count(rg, O.Graph.from_arcs(k, arcs))[:2] == O.count(og, O.Graph.from_arcs(k, arcs))[:2]


def _conditions(plan):
    out = []
    for i, lv in enumerate(plan):
        for j in range(i):
            if (lv["gt"] >> j) & 1:
                out.append((j, i))
            if (lv["lt"] >> j) & 1:
                out.append((i, j))
    return out


@pytest.mark.parametrize("name", ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant", "3-prism",
                                  "4-path", "3-star"])
def test_conditions_times_automorphisms_is_the_plain_count(name):
    h = cb.HostGraph.chung_lu(1500, 7000, 2.2, 2.0, 60.0, 2)
    od, _ = oracle_graph_from_host(h).relabel_by_degree()
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    oq = O.Graph.from_arcs(k, arcs)
    plain = O.count(od, oq, q.order)[0]
    plan, aut = q.plan_levels(True, cb.FLAG_SYMMETRY_BREAK | cb.FLAG_NO_ORBIT_FOLD)
    cnt, _ = O.count_ex(od, oq, q.order, _conditions(plan))
    assert cnt * aut == plain
    # stripes of the conditioned count partition it
    assert sum(O.count_ex(od, oq, q.order, _conditions(plan), r, 3)[0] for r in range(3)) == cnt


def test_orbit_decomposition_is_the_plain_count():
    h = cb.HostGraph.chung_lu(1500, 7000, 2.2, 2.0, 60.0, 2)
    od, _ = oracle_graph_from_host(h).relabel_by_degree()
    k, arcs = cb.named_query_arcs("4-clique+pendant")
    q = cb.Query.from_arcs(k, arcs)
    order = q.order
    plan, mult = q.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)
    orbit = plan[k - 1]["ofold"]
    e = order[k - 1]
    core = [(a, b) for a, b in arcs if e not in (a, b)]
    raw = sum(O.count_ex(od, O.Graph.from_arcs(k, core + [(order[x], e), (e, order[x])]), order,
                         _conditions(plan))[0] for x in range(k - 1) if (orbit >> x) & 1)
    assert raw * mult == O.count(od, O.Graph.from_arcs(k, arcs), order)[0]


@pytest.mark.parametrize("name", ["4-clique+pendant", "4-path", "3-star", "triangle", "house"])
def test_closed_last_level_is_the_same_count(name):
    h = cb.HostGraph.chung_lu(2000, 9000, 2.2, 2.0, 80.0, 6)
    od, _ = oracle_graph_from_host(h).relabel_by_degree()
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    oq = O.Graph.from_arcs(k, arcs)
    plan, _ = q.plan_levels(True, cb.FLAG_SYMMETRY_BREAK | cb.FLAG_NO_ORBIT_FOLD)
    for conds in ([], _conditions(plan)):
        assert O.count_ex(od, oq, q.order, conds, 0, 2, opts=O.OPT_CLOSED_LAST) == \
            O.count_ex(od, oq, q.order, conds, 0, 2)


def test_closed_last_level_directed_graph():
    from tests.helpers import directed_er
    n, src, dst = directed_er(800, 10.0, seed=9)
    od = O.Graph.from_arrays(n, src, dst)
    for arcs in ([(0, 1), (1, 2), (2, 0), (2, 3)], [(0, 1), (1, 2), (2, 3), (3, 2)], [(0, 1), (2, 1)]):
        k = 1 + max(max(a) for a in arcs)
        oq = O.Graph.from_arcs(k, arcs)
        assert O.count_ex(od, oq, None, [], opts=O.OPT_CLOSED_LAST) == O.count_ex(od, oq)
