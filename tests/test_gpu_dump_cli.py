"""The reference-facing surface on a GPU: the `cuts` command and its result
line, the Python mirror of search()/search_dfs_bfs_strategy(), and the
ans.txt match dump (compared as a set with the oracle's enumeration)."""
import os
import re
import subprocess

import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O
from tests.helpers import csr_from_arcs, directed_er, oracle_graph_from_host

pytestmark = pytest.mark.gpu

LINE = re.compile(r"^(\((\d+),(\d+)\))+$")


def _parse_dump(path, order):
    rows = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            assert LINE.match(line), line
            pairs = [(int(a), int(b)) for a, b in re.findall(r"\((\d+),(\d+)\)", line)]
            assert [a for a, _ in pairs] == order  # pairs in matching order
            by_q = dict(pairs)
            rows.append(tuple(by_q[v] for v in range(len(order))))
    return rows


@pytest.mark.parametrize("name", ["triangle", "4-cycle", "house", "4-clique+pendant"])
def test_dump_matches_oracle_set(tmp_path, name):
    h = cb.HostGraph.erdos_renyi(400, 0.04, seed=21)
    g = h.upload(0)
    k, arcs = cb.named_query_arcs(name)
    q = cb.Query.from_arcs(k, arcs)
    path = str(tmp_path / "ans.txt")
    n = g.dump(q, path)
    rows = _parse_dump(path, q.order)
    assert n == len(rows) == g.count(q).count
    want = O.enumerate_matches(oracle_graph_from_host(h), O.Graph.from_arcs(k, arcs), q.order)
    assert sorted(rows) == sorted(want)


def test_dump_directed_and_chunked(tmp_path):
    n, src, dst = directed_er(600, 12.0, seed=5)
    oo, oa, io, ia, s, d = csr_from_arcs(n, src, dst)
    g = cb.Graph.from_csr(n, oo, oa, io, ia)
    g.set_level_cap(256)  # force chunked levels, the final one included
    arcs = [(0, 1), (1, 2), (2, 0), (2, 3)]
    q = cb.Query.from_arcs(4, arcs)
    path = str(tmp_path / "ans.txt")
    g.dump(q, path)
    rows = _parse_dump(path, q.order)
    want = O.enumerate_matches(O.Graph.from_arrays(n, s, d), O.Graph.from_arcs(4, arcs), q.order)
    assert sorted(rows) == sorted(want)


def _files(tmp_path):
    h = cb.HostGraph.erdos_renyi(3000, 8.0 / 2999, seed=0)
    dpath = str(tmp_path / "er.g")
    h.write(dpath)
    k, arcs = cb.named_query_arcs("4-cycle")
    qpath = str(tmp_path / "c4.g")
    cb.write_query(qpath, k, arcs)
    cnt = O.count(oracle_graph_from_host(h), O.Graph.from_arcs(k, arcs))[0]
    return dpath, qpath, cnt


def test_cli_result_line(tmp_path):
    dpath, qpath, cnt = _files(tmp_path)
    r = subprocess.run([cb.CLI_PATH, dpath, qpath], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().split("\n")
    assert lines[:4] == ["start loading graph file from disk to memory...", "graph loading complete...",
                         "start copying graph to gpu...", "end copying graph to gpu..."]
    m = re.match(r"^er\.g,c4\.g,([0-9.e+-]+)ms,(\d+)$", lines[4])
    assert m and int(m.group(2)) == cnt
    r = subprocess.run([cb.CLI_PATH, dpath, qpath, "4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    lines = r.stdout.strip().split("\n")
    assert lines[3] == "finish copying graph to gpu..."
    assert lines[4].endswith(f"ms,{cnt}")


def test_cli_dump_and_base_name(tmp_path):
    dpath, qpath, cnt = _files(tmp_path)
    env = dict(os.environ, CUTS_WRITE_TO_DISK="1")
    # relative paths without '/': base_name() gives "" (common.cpp:19-26)
    r = subprocess.run([cb.CLI_PATH, "er.g", "c4.g"], capture_output=True, text=True,
                       cwd=str(tmp_path), env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().split("\n")
    assert re.match(r"^,,[0-9.e+-]+ms,%d$" % cnt, lines[4])
    assert lines[5:] == ["start writting matching results to disk,ans.txt",
                         "finish writting matching results to disk,ans.txt"]
    with open(tmp_path / "ans.txt") as f:
        assert sum(1 for _ in f) == cnt


def test_python_mirror(tmp_path, capfd):
    dpath, qpath, cnt = _files(tmp_path)
    assert cb.search(qpath, dpath) == cnt
    assert cb.search_dfs_bfs_strategy(qpath, dpath, False, 3) == cnt
    out = capfd.readouterr().out
    assert out.count(f"er.g,c4.g,") == 2
    with pytest.raises(cb.CutsError):
        cb.search_dfs_bfs_strategy(qpath, dpath, False, 0)


_DUMPS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_dumps.json")


def _dump_cases():
    if not os.path.exists(_DUMPS):
        return []
    import json
    with open(_DUMPS) as f:
        return json.load(f)["cases"]


@pytest.mark.skipif(not _dump_cases(), reason="reference dumps not recorded")
def test_dump_sets_equal_reference_binary(tmp_path):
    """Match sets identical to the ans.txt the reference binary wrote
    (tests/golden/ref_dumps.json): same canonical digest, same line count."""
    import hashlib
    graphs = {}
    for c in _dump_cases():
        key = c["graph"]
        if key not in graphs:
            p = c["graph_params"]
            h = (cb.HostGraph.erdos_renyi(p["n"], p["p"], p["seed"]) if c["graph_kind"] == "er" else
                 cb.HostGraph.chung_lu(p["n"], p["m"], p["gamma"], p["wmin"], p["cap"], p["seed"]))
            graphs[key] = h.upload(0)
        g = graphs[key]
        k, arcs = cb.named_query_arcs(c["query"])
        q = cb.Query.from_arcs(k, arcs)
        path = str(tmp_path / f"{key}_{c['query']}.txt")
        n = g.dump(q, path)
        rows = _parse_dump(path, q.order)
        hsh = hashlib.sha256()
        for r in sorted(rows):
            hsh.update((" ".join(str(x) for x in r) + "\n").encode())
        assert n == len(rows) == c["lines"], (key, c["query"])
        assert hsh.hexdigest() == c["sha256"] == c["oracle_sha256"], (key, c["query"])


def test_sharded_dump_partitions_the_full_dump(tmp_path):
    h = cb.HostGraph.chung_lu(3000, 12000, 2.2, 2.0, 60.0, seed=8)
    g = h.upload(0)
    for name in ["triangle", "house"]:
        k, arcs = cb.named_query_arcs(name)
        q = cb.Query.from_arcs(k, arcs)
        full = str(tmp_path / f"{name}_full.txt")
        n = g.dump(q, full)
        rows = sorted(_parse_dump(full, q.order))
        parts = []
        for r in range(3):
            path = str(tmp_path / f"{name}_{r}.txt")
            nr = g.dump(q, path, r, 3)
            pr = _parse_dump(path, q.order)
            assert nr == len(pr) == g.count_sharded(q, r, 3).count
            parts += pr
        assert n == len(rows) and sorted(parts) == rows
