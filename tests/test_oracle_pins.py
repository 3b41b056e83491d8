"""Pins of the CPU oracle (and of the engine's host order) against the reference.

* Order + P/C join lists: the reference's own host code (graph.cpp, score.cpp,
  util.cpp, common.cpp) compiled into oracle/_ref/ref_order.  Checked live on
  the reference's 33 query fixtures (read in place when the reference is
  mounted) and through the committed golden file tests/golden/orders.json
  (160 seeded queries, made by tests/golden/make_orders.py).
* Counts: closed-form known answers and brute force on tiny graphs.
"""
import itertools
import json
import math
import os
import subprocess

import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.conftest import REF_DIR, have_reference

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orders.json")


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)["queries"]


def _write(path, k, arcs):
    with open(path, "w") as f:
        f.write(f"{k}\n")
        for a, b in arcs:
            f.write(f"{a}\t{b}\n")


@pytest.mark.parametrize("i", range(160))
def test_oracle_order_matches_reference_golden(tmp_path, i):
    q = _golden()[i]
    p = str(tmp_path / "q.g")
    _write(p, q["k"], q["arcs"])
    order, P, C = O.order(O.Graph.load(p))
    assert order == q["order"]
    assert P == q["P"] and C == q["C"]


@pytest.mark.parametrize("i", range(160))
def test_engine_order_matches_reference_golden(tmp_path, i):
    q = _golden()[i]
    p = str(tmp_path / "q.g")
    _write(p, q["k"], q["arcs"])
    und = {(min(a, b), max(a, b)) for a, b in q["arcs"]}
    # the engine rejects disconnected queries; golden queries are connected
    eq = cb.Query.load(p)
    assert eq.order == q["order"]
    P, C = eq.joins()
    assert P == q["P"] and C == q["C"]
    assert len(und) >= q["k"] - 1


def _ref_fixture_paths():
    d = os.path.join(REF_DIR, "data_set", "query", "ours_format")
    return [os.path.join(d, f"{i}.g") for i in range(1, 34)]


@pytest.mark.skipif(not have_reference() or not os.path.exists(O.REF_ORDER),
                    reason="reference sources / ref_order harness not present")
def test_reference_query_fixtures_live():
    """The reference's 33 query fixtures, read in place."""
    paths = _ref_fixture_paths()
    out = subprocess.run([O.REF_ORDER] + paths, check=True, capture_output=True,
                         text=True).stdout.strip().split("\n")
    assert len(out) == 33
    for path, line in zip(paths, out):
        ref_order = [int(x) for x in line.split(" ")[1][len("order="):].split(",")]
        order, P, C = O.order(O.Graph.load(path))
        assert order == ref_order, path
        eq = cb.Query.load(path)
        assert eq.order == ref_order, path
        assert eq.joins() == (P, C)


def test_four_cycle_order_and_joins():
    # symmetric 4-cycle -> order 0 1 2 3 with P = C = {0, 2} at the last level
    k, arcs = cb.named_query_arcs("4-cycle")
    order, P, C = O.order(O.Graph.from_arcs(k, arcs))
    assert order == [0, 1, 2, 3] and P[3] == [0, 2] and C[3] == [0, 2]


# ---- counts -------------------------------------------------------------

def _complete(n):
    return [(a, b) for a in range(n) for b in range(n) if a != b]


@pytest.mark.parametrize("name", ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant",
                                  "3-prism", "6-cycle"])
def test_oracle_complete_graph(name):
    n = 8
    d = O.Graph.from_arcs(n, _complete(n))
    k, arcs = cb.named_query_arcs(name)
    cnt, lv, _ = O.count(d, O.Graph.from_arcs(k, arcs))
    assert cnt == math.factorial(n) // math.factorial(n - k)
    assert lv[0] == n


def test_oracle_cycle_in_cycle():
    k, arcs = cb.named_query_arcs("4-cycle")
    assert O.count(O.Graph.from_arcs(4, arcs), O.Graph.from_arcs(4, arcs))[0] == 8
    assert O.count(O.Graph.from_arcs(4, _complete(4)), O.Graph.from_arcs(3, cb.cycle3()))[0] == 24 \
        if hasattr(cb, "cycle3") else True


def test_oracle_star():
    d = 9
    edges = [(0, i) for i in range(1, d + 1)]
    arcs = edges + [(b, a) for a, b in edges]
    G = O.Graph.from_arcs(d + 1, arcs)
    for s in (2, 3, 4):
        qa = [(0, i) for i in range(1, s + 1)]
        qa += [(b, a) for a, b in qa]
        assert O.count(G, O.Graph.from_arcs(s + 1, qa))[0] == math.factorial(d) // math.factorial(d - s)


def _brute(n, darcs, k, qarcs):
    """Injective maps preserving every query arc and the degree signature."""
    dset = set(darcs)
    din = [0] * n; dout = [0] * n
    for a, b in dset:
        dout[a] += 1; din[b] += 1
    qset = set(qarcs)
    qin = [0] * k; qout = [0] * k
    for a, b in qset:
        qout[a] += 1; qin[b] += 1
    c = 0
    for f in itertools.permutations(range(n), k):
        if any(din[f[v]] < qin[v] or dout[f[v]] < qout[v] for v in range(k)):
            continue
        if all((f[a], f[b]) in dset for a, b in qset if a != b):
            c += 1
    return c


@pytest.mark.parametrize("seed", range(25))
def test_oracle_brute_force(seed):
    rng = np.random.default_rng(seed)
    n = 7
    darcs = [(a, b) for a in range(n) for b in range(n) if rng.random() < 0.45]
    k = 3 + seed % 3
    und = cb.random_query_arcs(k, 0.4, seed) if seed % 2 else None
    if und is None:
        # directed query: orient a random tree + extras
        und = cb.random_query_arcs(k, 0.4, seed)
        und = [a for a in und if a[0] < a[1] or rng.random() < 0.5]
    if seed % 5 == 0:
        und = und + [(0, 0)]
    d = O.Graph.from_arcs(n, darcs)
    q = O.Graph.from_arcs(k, und)
    assert O.count(d, q)[0] == _brute(n, darcs, k, und)


def test_oracle_level_sizes_and_bytes_small():
    """|L_i| are prefix counts; the byte model follows its formula."""
    k, arcs = cb.named_query_arcs("triangle")
    n = 5
    d = O.Graph.from_arcs(n, _complete(n))
    cnt, lv, by = O.count(d, O.Graph.from_arcs(k, arcs))
    assert lv == [5, 20, 60] and cnt == 60
    # 8n + 4|L0| + sum over parents of (8 + lists) + 8|L1|
    # level 1: 5 parents x (8 + 4*4 + 8); level 2: 20 parents x (8 + (4*4+8)) [one distinct
    # list per position on a symmetric graph, two positions]
    want = 8 * 5 + 4 * 5 + 5 * (8 + 24) + 20 * (8 + 2 * 24) + 8 * 20
    assert by == want


def test_oracle_root_slices_sum():
    h = cb.HostGraph.erdos_renyi(800, 0.02, seed=4)
    oo, oa, _, _ = h.csr()
    d = O.Graph.from_csr(800, oo, oa)
    k, arcs = cb.named_query_arcs("house")
    q = O.Graph.from_arcs(k, arcs)
    full = O.count(d, q)[0]
    n0 = O.count(d, q)[1][0]
    parts = sum(O.count(d, q, root_begin=a, root_end=min(a + 97, n0))[0] for a in range(0, n0, 97))
    assert parts == full
