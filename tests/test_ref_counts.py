"""Counts pinned by the reference binary itself (tests/golden/ref_counts.json,
recorded on a B200 by tests/golden/make_ref_counts.py from the unmodified
reference built for sm_100a): the oracle on CPU and the engine on a GPU must
reproduce every recorded count."""
import json
import os

import pytest

import cuts_b200 as cb
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_counts.json")
pytestmark = pytest.mark.skipif(not os.path.exists(GOLDEN), reason="reference counts not recorded")


def _cases():
    if not os.path.exists(GOLDEN):
        return []
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


_GRAPHS = {}


def _graph(case):
    key = case["graph"]
    if key not in _GRAPHS:
        p = case["graph_params"]
        if case["graph_kind"] == "er":
            h = cb.HostGraph.erdos_renyi(p["n"], p["p"], p["seed"])
        else:
            h = cb.HostGraph.chung_lu(p["n"], p["m"], p["gamma"], p["wmin"], p["cap"], p["seed"])
        oo, oa, _, _ = h.csr()
        _GRAPHS[key] = (h, O.Graph.from_csr(h.n, oo, oa), None)
    return _GRAPHS[key]


def test_reference_is_self_consistent():
    for c in _cases():
        assert c["ref_count"] == c["ref_count_trunks4"], c["graph"] + "/" + c["query"]


@pytest.mark.parametrize("i", range(len(_cases())))
def test_oracle_reproduces_reference(i):
    c = _cases()[i]
    h, od, _ = _graph(c)
    k, arcs = c["k"], [tuple(a) for a in c["arcs"]]
    assert O.count(od, O.Graph.from_arcs(k, arcs))[0] == c["ref_count"]


@pytest.mark.gpu
def test_engine_reproduces_reference():
    dev = {}
    for c in _cases():
        h, od, _ = _graph(c)
        if c["graph"] not in dev:
            dev[c["graph"]] = h.upload(0)
        g = dev[c["graph"]]
        q = cb.Query.from_arcs(c["k"], [tuple(a) for a in c["arcs"]])
        assert g.count(q).count == c["ref_count"], c["graph"] + "/" + c["query"]
        assert g.count(q, chunks=4, flags=cb.FLAG_SYMMETRY_BREAK).count == c["ref_count"]
