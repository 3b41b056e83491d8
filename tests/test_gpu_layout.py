"""The data graph's device layout: built on the device from CSR arrays
(validation, symmetry check, degree-ranked ids, padded sorted lists).
Counts never depend on the labelling; invalid CSR input is rejected with the
loader's messages; the id map takes the dump back to the caller's ids."""
import os
import subprocess
import sys

import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import csr_from_arcs, directed_er, oracle_graph_from_host

pytestmark = pytest.mark.gpu


def _sym_csr(n, edges):
    src = np.array([a for a, b in edges] + [b for a, b in edges], np.uint32)
    dst = np.array([b for a, b in edges] + [a for a, b in edges], np.uint32)
    oo, oa, io, ia, _, _ = csr_from_arcs(n, src, dst)
    return oo, oa, io, ia


def test_from_csr_rejects_invalid_input():
    oo, oa, io, ia = _sym_csr(5, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0)])
    g = cb.Graph.from_csr(5, oo, oa)  # symmetric, in-lists omitted
    assert g.info()[2] is True
    bad = oa.copy()
    bad[0], bad[1] = bad[1], bad[0]  # vertex 0's list out of order
    with pytest.raises(cb.CutsError, match="strictly sorted"):
        cb.Graph.from_csr(5, oo, bad)
    big = oa.copy()
    big[-1] = 9  # id out of range
    with pytest.raises(cb.CutsError, match="out of range"):
        cb.Graph.from_csr(5, oo, big)
    off = oo.copy()
    off[2] = off[3] + 1  # offsets not monotone
    with pytest.raises(cb.CutsError, match="monotone"):
        cb.Graph.from_csr(5, off, oa)
    # a directed cycle without in-lists
    src = np.arange(5, dtype=np.uint32)
    dst = (src + 1) % 5
    doo, doa, dio, dia, _, _ = csr_from_arcs(5, src, dst)
    with pytest.raises(cb.CutsError, match="not symmetric"):
        cb.Graph.from_csr(5, doo, doa)
    d = cb.Graph.from_csr(5, doo, doa, dio, dia)
    assert d.info()[2] is False
    # in-lists equal to the out-lists: symmetric
    s = cb.Graph.from_csr(5, oo, oa, oo, oa)
    assert s.info()[2] is True
    # the first graph still counts after the rejected builds
    assert g.count(cb.Query.from_arcs(*cb.named_query_arcs("5-cycle"))).count == 10


def _drop_arc(oo, oa, u, v):
    """The CSR without the arc u -> v."""
    x = int(oo[u]) + int(np.searchsorted(oa[oo[u]:oo[u + 1]], v))
    assert oa[x] == v
    oo2 = oo.copy()
    oo2[u + 1:] -= 1
    return oo2, np.delete(oa, x)


def test_symmetry_check_finds_every_missing_reverse():
    """The symmetry check searches only the arcs that go down in (degree,
    id) order and compares the numbers of arcs going up and down: a missing
    reverse is found on either side, from a hub or from a leaf."""
    # star 0-1, 0-2 plus the arc 3 -> 0 alone (an up arc: leaf to hub), and
    # 0 -> 3 alone (a down arc: hub to leaf)
    for extra in ([(3, 0)], [(0, 3)]):
        src = np.array([0, 1, 0, 2] + [a for a, b in extra], np.uint32)
        dst = np.array([1, 0, 2, 0] + [b for a, b in extra], np.uint32)
        oo, oa, _, _, _, _ = csr_from_arcs(4, src, dst)
        with pytest.raises(cb.CutsError, match="not symmetric"):
            cb.Graph.from_csr(4, oo, oa)
    # a power-law graph, self-loops added: symmetric; without one arc (hub
    # to leaf, leaf to hub, equal degrees): not
    h = cb.HostGraph.chung_lu(3000, 9000, 2.1, 2.0, 200.0, seed=12)
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(h.n, dtype=np.uint32), np.diff(oo).astype(np.int64))
    loops = np.arange(0, h.n, 7, dtype=np.uint32)
    lo, la, _, _, _, _ = csr_from_arcs(h.n, np.concatenate([src, loops]), np.concatenate([oa, loops]))
    assert cb.Graph.from_csr(h.n, lo, la).info()[2] is True
    deg = np.diff(oo)
    hub = int(np.argmax(deg))
    leaf = int(oa[oo[hub]:oo[hub + 1]][np.argmin(deg[oa[oo[hub]:oo[hub + 1]]])])
    pairs = [(hub, leaf), (leaf, hub)]
    for u in range(h.n):  # an arc between two vertices of equal degree
        vs = oa[oo[u]:oo[u + 1]]
        same = vs[deg[vs] == deg[u]]
        if len(same):
            pairs += [(u, int(same[0])), (int(same[0]), u)]
            break
    assert len(pairs) == 4
    for u, v in pairs:
        oo2, oa2 = _drop_arc(oo, oa, u, v)
        with pytest.raises(cb.CutsError, match="not symmetric"):
            cb.Graph.from_csr(h.n, oo2, oa2)


def test_host_and_csr_paths_agree():
    h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
    oo, oa, _, _ = h.csr()
    g1 = h.upload(0)
    g2 = cb.Graph.from_csr(h.n, oo, oa)
    assert g1.info() == g2.info()
    for name in ("triangle", "4-cycle", "house", "4-clique+pendant"):
        q = cb.Query.from_arcs(*cb.named_query_arcs(name))
        for fl in (0, cb.FLAG_SYMMETRY_BREAK):
            a = g1.count(q, flags=fl, stats=True)
            b = g2.count(q, flags=fl, stats=True)
            assert a.count == b.count and a.level_sizes == b.level_sizes


_RELABEL_OFF = """
import sys, os, json
sys.path.insert(0, os.getcwd())
import numpy as np
import cuts_b200 as cb
from tests.helpers import csr_from_arcs, directed_er
h = cb.HostGraph.chung_lu(5000, 20000, 2.1, 2.0, 100.0, seed=5)
g = h.upload(0)
out = []
for name in ("triangle", "house", "4-clique+pendant"):
    q = cb.Query.from_arcs(*cb.named_query_arcs(name))
    out.append([g.count(q, flags=f, stats=True).count for f in (0, 1)])
n, s, d = directed_er(1500, 14.0, seed=11)
oo, oa, io, ia, _, _ = csr_from_arcs(n, s, d)
dg = cb.Graph.from_csr(n, oo, oa, io, ia)
q = cb.Query.from_arcs(3, [(0, 1), (1, 2), (0, 2), (2, 0)])
out.append([dg.count(q, flags=0).count])
print(json.dumps(out))
"""


def test_counts_do_not_depend_on_the_labelling():
    """The same counts with degree-ranked ids and with the caller's ids
    (CUTS_NO_RELABEL=1, read when a graph is built), in separate processes."""
    res = []
    for env in ({}, {"CUTS_NO_RELABEL": "1"}):
        e = dict(os.environ, **env)
        r = subprocess.run([sys.executable, "-c", _RELABEL_OFF], capture_output=True, text=True, env=e,
                           cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))), timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res.append(r.stdout.strip().splitlines()[-1])
    assert res[0] == res[1]


def test_self_loops_detected_after_relabelling():
    """A graph whose only self-loop sits on a hub: the loop flag must follow
    the vertex to its degree rank (the fold's membership tests depend on it)."""
    edges = [(0, i) for i in range(1, 40)] + [(1, 2), (2, 3), (1, 3)]
    n = 40
    src = np.array([a for a, b in edges] + [b for a, b in edges] + [0], np.uint32)
    dst = np.array([b for a, b in edges] + [a for a, b in edges] + [0], np.uint32)
    oo, oa, io, ia, s_, d_ = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    od = O.Graph.from_arrays(n, s_, d_)
    for name in ("4-clique+pendant", "triangle"):
        k, arcs = cb.named_query_arcs(name)
        q = cb.Query.from_arcs(k, arcs)
        want = O.count(od, O.Graph.from_arcs(k, arcs), q.order)[0]
        for fl in (0, cb.FLAG_SYMMETRY_BREAK):
            assert g.count(q, flags=fl).count == want
    paw = (4, [(0, 1), (1, 0), (1, 2), (2, 1), (0, 2), (2, 0), (0, 3), (3, 0)])
    q = cb.Query.from_arcs(*paw)
    want = O.count(od, O.Graph.from_arcs(*paw), q.order)[0]
    assert g.count(q, flags=cb.FLAG_SYMMETRY_BREAK).count == want
