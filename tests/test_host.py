"""Host-side logic on CPU: the C-ABI library, loader semantics, generators,
query plans, CLI argument handling.  No GPU compute is called."""
import os
import re
import subprocess

import numpy as np
import pytest

import cuts_b200 as cb
from oracle import oracle as O


def test_library_exports_every_header_symbol():
    with open(cb.HEADER_PATH) as f:
        src = f.read()
    declared = set(re.findall(r"\b(cuts_[a-z0-9_]+)\s*\(", src))
    assert len(declared) >= 25
    lib = cb.lib()
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    # and nothing exported beyond the header (plus C++ internals, hidden by the namespace)
    out = subprocess.run(["nm", "-D", "--defined-only", cb.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (cuts_[a-z0-9_]+)$", out, re.M))
    assert exported == declared


def test_version():
    assert cb.lib().cuts_version().decode().startswith("cuts_b200")


CASES = {
    "plain": "4\n0\t1\n1\t2\n2\t3\n3\t0\n",
    "crlf": "4\r\n0\t1\r\n1\t2\r\n2\t3\r\n",
    "no_tab_lines_skipped": "5\n# comment\n0\t1\n\n1 2\n3\t4\n",
    "duplicates": "3\n0\t1\n0\t1\n1\t2\n0\t1\n",
    "self_loops": "3\n0\t0\n0\t1\n2\t2\n",
    "stoi_prefix": "6\t junk\n 1\t2xyz\n+3\t 4\n5\t0\t9\n",
    "no_trailing_newline": "3\n0\t1\n1\t2",
    "isolated": "10\n0\t9\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_loader_matches_oracle(tmp_path, name):
    p = str(tmp_path / "g.txt")
    with open(p, "w", newline="") as f:
        f.write(CASES[name])
    og = O.Graph.load(p)
    h = cb.HostGraph.load(p)
    n, arcs, sym, _ = h.info()
    assert n == og.n
    oo, oa, io, ia = og.csr()
    po, pa, pi, pia = h.csr()
    assert np.array_equal(oo, po) and np.array_equal(oa, pa)
    assert sym == og.symmetric()
    if not sym:
        assert np.array_equal(io, pi) and np.array_equal(ia, pia)


REF_LOADER_JSON = os.path.join(os.path.dirname(__file__), "golden", "ref_loader.json")
REF_LOAD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "ref_load")


@pytest.mark.parametrize("name", sorted(CASES))
def test_loader_matches_reference_loader(tmp_path, name):
    """This loader builds the CSR that the reference's own loader builds
    (file_reader, util.cpp:19-52; Graph(1, path), graph.cpp:18-61) on every
    edge case: vertex and arc counts, out-lists and in-lists.  Fixtures from
    the reference loader compiled from its sources
    (tests/golden/make_ref_loader.py); the binary is run live as well where
    it has been built."""
    import json
    with open(REF_LOADER_JSON) as f:
        want = json.load(f)[name]
    p = str(tmp_path / "g.txt")
    with open(p, "w", newline="") as f:
        f.write(CASES[name])
    if os.path.exists(REF_LOAD):
        from tests.golden.make_ref_loader import run_ref_load
        assert run_ref_load(p) == want
    h = cb.HostGraph.load(p)
    n, arcs, sym, _ = h.info()
    assert (n, arcs) == (want["V"], want["E"])
    oo, oa, io, ia = h.csr()
    assert oo.tolist() == want["out_off"] and oa.tolist() == want["out_adj"]
    if sym:  # one CSR kept: the reference's in-lists are the same lists
        assert want["in_off"] == want["out_off"] and want["in_adj"] == want["out_adj"]
    else:
        assert io.tolist() == want["in_off"] and ia.tolist() == want["in_adj"]


@pytest.mark.skipif(not os.path.exists(REF_LOAD), reason="reference loader not built here")
def test_loader_matches_reference_loader_on_random_files(tmp_path):
    """Seeded random files -- directed arcs with repeats and self-loops in
    random line order, CRLF line ends on some lines -- loaded by the
    reference's loader and by this one: the same CSR."""
    from tests.golden.make_ref_loader import run_ref_load
    rng = np.random.default_rng(5)
    for n, m in ((50, 400), (3000, 40000)):
        src = rng.integers(0, n, m)
        dst = rng.integers(0, n, m)
        src = np.concatenate([src, src[: m // 10]])  # repeated arcs
        dst = np.concatenate([dst, dst[: m // 10]])
        perm = rng.permutation(len(src))
        ends = rng.choice(["\n", "\r\n"], len(src))
        p = str(tmp_path / f"r{n}.txt")
        with open(p, "w", newline="") as f:
            f.write(f"{n}\n" + "".join(f"{src[i]}\t{dst[i]}{ends[i]}" for i in perm))
        want = run_ref_load(p)
        h = cb.HostGraph.load(p)
        n2, arcs, sym, _ = h.info()
        assert (n2, arcs) == (want["V"], want["E"])
        oo, oa, io, ia = h.csr()
        assert oo.tolist() == want["out_off"] and oa.tolist() == want["out_adj"]
        assert not sym and io.tolist() == want["in_off"] and ia.tolist() == want["in_adj"]


def test_loader_symmetry_finds_every_missing_reverse(tmp_path):
    """The loader's symmetry check searches only the arcs going down in
    (degree, id) order and compares the numbers going up and down: a graph
    with self-loops is symmetric, the same graph without one arc (leaf to
    hub, hub to leaf, between equal degrees) is not."""
    h = cb.HostGraph.chung_lu(2000, 6000, 2.1, 2.0, 150.0, seed=21)
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(h.n), np.diff(oo).astype(np.int64))
    deg = np.diff(oo)
    hub = int(np.argmax(deg))
    nb = oa[oo[hub]:oo[hub + 1]]
    leaf = int(nb[np.argmin(deg[nb])])
    same = next((u, int(v)) for u in range(h.n) for v in oa[oo[u]:oo[u + 1]] if deg[v] == deg[u] and v != u)
    loops = np.arange(0, h.n, 5)

    def load(drop):
        keep = ~((src == drop[0]) & (oa == drop[1])) if drop else np.ones(len(oa), bool)
        s = np.concatenate([src[keep], loops])
        d = np.concatenate([oa[keep], loops])
        p = str(tmp_path / "g.txt")
        with open(p, "w") as f:
            f.write(f"{h.n}\n" + "".join(f"{a}\t{b}\n" for a, b in zip(s, d)))
        return cb.HostGraph.load(p).info()[2]

    assert load(None) is True
    for drop in [(hub, leaf), (leaf, hub), same, same[::-1]]:
        assert load(drop) is False, drop


@pytest.mark.parametrize("text,code", [
    ("", cb.ERR_PARSE),
    ("x\n0\t1\n", cb.ERR_PARSE),
    ("3\n0\t5\n", cb.ERR_PARSE),
    ("3\n-1\t2\n", cb.ERR_PARSE),
    ("3\n0\tx\n", cb.ERR_PARSE),
    ("3\n99999999999\t1\n", cb.ERR_PARSE),
])
def test_loader_errors(tmp_path, text, code):
    p = str(tmp_path / "bad.txt")
    with open(p, "w") as f:
        f.write(text)
    with pytest.raises(cb.CutsError) as e:
        cb.HostGraph.load(p)
    assert e.value.code == code


def test_missing_file():
    with pytest.raises(cb.CutsError) as e:
        cb.HostGraph.load("/nonexistent/graph.txt")
    assert e.value.code == cb.ERR_IO


def test_write_roundtrip(tmp_path):
    h = cb.HostGraph.erdos_renyi(3000, 0.003, seed=7)
    p = str(tmp_path / "er.txt")
    h.write(p)
    h2 = cb.HostGraph.load(p)
    a, b = h.csr(), h2.csr()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_er_generator():
    h = cb.HostGraph.erdos_renyi(10000, 8.0 / 9999, seed=0)
    n, arcs, sym, _ = h.info()
    assert n == 10000 and sym
    assert abs(arcs / n - 8.0) < 0.3
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(n), np.diff(oo.astype(np.int64)))
    assert not np.any(src == oa)  # no loops
    h2 = cb.HostGraph.erdos_renyi(10000, 8.0 / 9999, seed=0)
    assert np.array_equal(h2.csr()[1], oa)
    h3 = cb.HostGraph.erdos_renyi(10000, 8.0 / 9999, seed=1)
    assert not np.array_equal(h3.csr()[1][:1000], oa[:1000])


def test_chung_lu_generator():
    n, m = 20000, 100000
    h = cb.HostGraph.chung_lu(n, m, 2.1, 2.0, 500.0, seed=0)
    nn, arcs, sym, maxd = h.info()
    assert nn == n and sym and arcs == 2 * m
    oo, oa, _, _ = h.csr()
    src = np.repeat(np.arange(n), np.diff(oo.astype(np.int64)))
    assert not np.any(src == oa)
    deg = np.diff(oo.astype(np.int64))
    assert maxd == deg.max() and maxd > 20 * deg.mean()  # heavy tail
    h2 = cb.HostGraph.chung_lu(n, m, 2.1, 2.0, 500.0, seed=0)
    assert np.array_equal(h2.csr()[1], oa)


def test_random_query_connected():
    for seed in range(50):
        k = 3 + seed % 6
        arcs = cb.random_query_arcs(k, 0.3, seed)
        q = cb.Query.from_arcs(k, arcs)  # raises when disconnected
        assert sorted(q.order) == list(range(k))
        assert all((b, a) in arcs for a, b in arcs)


def test_query_errors():
    with pytest.raises(cb.CutsError) as e:
        cb.Query.from_arcs(4, [(0, 1), (1, 0), (2, 3), (3, 2)])
    assert e.value.code == cb.ERR_QUERY
    with pytest.raises(cb.CutsError) as e:
        cb.Query.from_edges(17, [(i, i + 1) for i in range(16)])
    assert e.value.code == cb.ERR_QUERY
    q = cb.Query.from_edges(4, [(0, 1), (1, 2), (2, 3)])
    with pytest.raises(cb.CutsError):
        q.set_order([0, 2, 1, 3])  # position 1 has no arc to position 0
    q.set_order([1, 2, 0, 3])
    assert q.order == [1, 2, 0, 3]


@pytest.mark.parametrize("name,aut", [("triangle", 6), ("4-cycle", 8), ("5-cycle", 10),
                                      ("6-cycle", 12), ("house", 2), ("4-clique+pendant", 6),
                                      ("3-prism", 12)])
def test_automorphism_counts(name, aut):
    k, arcs = cb.named_query_arcs(name)
    assert cb.Query.from_arcs(k, arcs).automorphisms() == aut


def test_automorphisms_directed():
    # directed 3-cycle: rotations only
    assert cb.Query.from_arcs(3, [(0, 1), (1, 2), (2, 0)]).automorphisms() == 3
    # directed path: identity only
    assert cb.Query.from_arcs(3, [(0, 1), (1, 2)]).automorphisms() == 1


def test_cli_usage_and_bad_trunks(tmp_path):
    r = subprocess.run([cb.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 255
    assert "args data_graph path,query_graph_path" in r.stdout
    r = subprocess.run([cb.CLI_PATH, "a", "b", "0"], capture_output=True, text=True)
    assert r.returncode == 255 and "invalid trunks" in r.stdout
    r = subprocess.run([cb.CLI_PATH, "/nonexistent/d.txt", "/nonexistent/q.g"],
                       capture_output=True, text=True)
    assert r.returncode == 255 and "failed" in r.stdout


def test_plan_fold_and_guarantees():
    # 4-clique 0..3 + pendant 4 on 0: the pendant is last, joined to position of 0
    q = cb.Query.from_arcs(*cb.named_query_arcs("4-clique+pendant"))
    lv, aut = q.plan_levels(True, 0)
    k = q.k
    assert q.order[-1] == 4 and aut == 1
    last, pen = lv[k - 1], lv[k - 2]
    assert last["closed"] == 1 and last["sig"] == 0 and pen["fold"] == 1
    pos0 = q.order.index(0)
    # every other clique vertex is a query neighbour of 0: guaranteed in N(m0)
    want = sum(1 << j for j in range(k - 1) if j != pos0)
    assert last["guar"] == want
    # intermediate levels keep the signature test; level 0 too
    assert all(l["sig"] == 1 for l in lv[:-1])
    # no closed form, no fold
    lv2, _ = q.plan_levels(True, cb.FLAG_NO_CLOSED_FORM)
    assert lv2[k - 1]["closed"] == 0 and lv2[k - 2]["fold"] == 0
    # symmetry breaking on a triangle: constraints, |Aut| = 6, no fold (closed form
    # needs a single joined list)
    t = cb.Query.from_arcs(*cb.named_query_arcs("triangle"))
    lv3, aut3 = t.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)
    assert aut3 == 6 and lv3[2]["closed"] == 0 and lv3[1]["fold"] == 0
    assert lv3[1]["gt"] | lv3[1]["lt"] and lv3[2]["gt"] | lv3[2]["lt"]


def test_plan_directed_guarantees():
    # directed: 0->1, 1->2, 0->3 ; last vertex 3 joined by out-list of m0; 1 is in
    # out(m0) (arc 0->1) but 2 is not guaranteed
    q = cb.Query.from_arcs(4, [(0, 1), (1, 2), (0, 3)])
    q.set_order([0, 1, 2, 3])
    lv, _ = q.plan_levels(False, 0)
    assert lv[3]["closed"] == 1
    assert lv[3]["guar"] == 0b010
    lv_sym, _ = q.plan_levels(True, 0)
    assert lv_sym[3]["guar"] == 0b010  # 2 is not adjacent to 0 at all


def test_plan_fuse_conditions():
    tri = cb.Query.from_arcs(*cb.named_query_arcs("triangle"))
    lv, _ = tri.plan_levels(True, 0)
    assert lv[2]["fuse"] == 1
    assert tri.plan_levels(True, cb.FLAG_NO_FUSE)[0][2]["fuse"] == 0
    # 4-clique+pendant: the folded level k-2 (the 4-clique vertex) is fused
    cp = cb.Query.from_arcs(*cb.named_query_arcs("4-clique+pendant"))
    lv, _ = cp.plan_levels(True, 0)
    assert lv[3]["fold"] == 1 and lv[3]["fuse"] == 1
    # 4-cycle: the last vertex does not join the previous one's lists -> no fuse
    c4 = cb.Query.from_arcs(*cb.named_query_arcs("4-cycle"))
    assert all(l["fuse"] == 0 for l in c4.plan_levels(True, 0)[0])


def test_binary_csr_cache(tmp_path):
    for h in (cb.HostGraph.erdos_renyi(5000, 0.002, seed=3),):
        p = str(tmp_path / "g.csr")
        h.save_binary(p)
        h2 = cb.HostGraph.load_binary(p)
        assert h2.info() == h.info()
        for a, b in zip(h.csr(), h2.csr()):
            assert (a is None and b is None) or np.array_equal(a, b)
    # directed graph round trip through text then binary
    p_txt = str(tmp_path / "d.txt")
    with open(p_txt, "w") as f:
        f.write("5\n0\t1\n1\t2\n2\t0\n3\t4\n")
    d = cb.HostGraph.load(p_txt)
    d.save_binary(str(tmp_path / "d.csr"))
    d2 = cb.HostGraph.load_binary(str(tmp_path / "d.csr"))
    assert d2.info() == d.info() and not d2.info()[2]
    for a, b in zip(d.csr(), d2.csr()):
        assert np.array_equal(a, b)
    with open(tmp_path / "bad.csr", "wb") as f:
        f.write(b"NOTACSR!")
    with pytest.raises(cb.CutsError) as e:
        cb.HostGraph.load_binary(str(tmp_path / "bad.csr"))
    assert e.value.code == cb.ERR_PARSE


def test_converters(tmp_path):
    from cuts_b200 import convert
    snap = tmp_path / "s.txt"
    snap.write_text("# comment line\n# another\n0\t5\n5\t0\n2\t3\n")
    n = convert.snap_to_cuts(str(snap), str(tmp_path / "s.g"))
    assert n == 6
    h = cb.HostGraph.load(str(tmp_path / "s.g"))
    assert h.info()[:2] == (6, 3)
    q = tmp_path / "q.g"
    q.write_text("3\n0\t1\n1\t2\n2\t0\n")
    convert.cuts_to_gsi(str(q), str(tmp_path / "q.gsi"))
    lines = (tmp_path / "q.gsi").read_text().splitlines()
    assert lines[0] == "t # 0" and lines[1] == "3 3 1 1" and lines[-1] == "t # -1"
    assert lines[2:5] == ["v 0 1", "v 1 1", "v 2 1"] and lines[5] == "e 0 1 1"


def _und(edges):
    return [(a, b) for u, v in edges for a, b in ((u, v), (v, u))]


ORBIT_QUERIES = {
    # name: (k, arcs, expected orbit size or 0 for "no orbit fold")
    "4-clique+pendant": cb.named_query_arcs("4-clique+pendant") + (4,),
    "paw": (4, _und([(0, 1), (1, 2), (0, 2), (0, 3)]), 3),
    "5-clique+pendant": (6, _und([(a, b) for a in range(5) for b in range(a + 1, 5)] + [(0, 5)]), 5),
    "4-cycle+pendant": (5, _und([(0, 1), (1, 2), (2, 3), (3, 0), (0, 4)]), 0),
    "diamond+pendant-deg3": (5, _und([(0, 1), (0, 2), (1, 2), (1, 3), (2, 3), (1, 4)]), 0),
    "diamond+pendant-deg2": (5, _und([(0, 1), (0, 2), (1, 2), (1, 3), (2, 3), (0, 4)]), 0),
    "path4": (4, _und([(0, 1), (1, 2), (2, 3)]), 0),
    "star4": (5, _und([(0, 1), (0, 2), (0, 3), (0, 4)]), 0),
    # a directed 3-cycle with an out-pendant: the rotations move the attachment
    "dir3cycle+pendant": (4, [(0, 1), (1, 2), (2, 0), (0, 3)], 3),
}


def _brute_orbit_total(q, qarcs, lv, aut, n, out_adj, in_adj):
    """aut x sum over core embeddings that satisfy the plan's masks and
    signatures of the orbit weight -- the orbit fold's formula evaluated by
    a plain depth-first search."""
    k = q.k
    order = q.order
    e = order[k - 1]
    arcs = set(qarcs)
    core = order[:k - 1]
    a = [v for v in core if (v, e) in arcs or (e, v) in arcs][0]
    L = out_adj if (a, e) in arcs else in_adj
    omask = lv[k - 1]["ofold"]
    total = 0
    m = []

    def fits(i, v):
        if v in m:
            return False
        if lv[i]["sig"] and (len(in_adj[v]) < lv[i]["qin"] or len(out_adj[v]) < lv[i]["qout"]):
            return False
        for j in range(i):
            if (core[i], core[j]) in arcs and m[j] not in out_adj[v]:
                return False
            if (core[j], core[i]) in arcs and v not in out_adj[m[j]]:
                return False
            if ((lv[i]["gt"] >> j) & 1) and not v > m[j]:
                return False
            if ((lv[i]["lt"] >> j) & 1) and not v < m[j]:
                return False
        return True

    def dfs(i):
        nonlocal total
        if i == k - 1:
            mset = set(m)
            for x in range(k - 1):
                if (omask >> x) & 1:
                    total += len(L[m[x]] - mset)
            return
        for v in range(n):
            if fits(i, v):
                m.append(v)
                dfs(i + 1)
                m.pop()

    dfs(0)
    return total * aut


def _orbit_graphs(directed, k):
    """Small data graphs: random ones, dense and sparse, and one whose
    lowest-id clique vertices have no edges outside their clique (so a class
    representative puts a vertex without a pendant neighbour at the
    attachment's position)."""
    out = []
    for dens in (0.55, 0.3):
        rng = np.random.default_rng(7 + k)
        n = 9
        src, dst = [], []
        for u in range(n):
            for v in range(n):
                if u != v and rng.random() < dens:
                    src.append(u); dst.append(v)
                    if not directed:
                        src.append(v); dst.append(u)
        out.append((n, src, dst))
    # K5 on 0..4 with pendants on 4; a triangle 9-10-11 whose lowest vertex
    # has no other edge; a K4 14..17 whose lowest three have no other edge;
    # a K6 20..25 with one extra edge on 25
    und = ([(a, b) for a in range(5) for b in range(a + 1, 5)] + [(4, 5), (4, 6), (4, 7), (4, 8),
                                                                   (1, 5), (2, 5), (2, 6)] +
           [(9, 10), (9, 11), (10, 11), (10, 12), (10, 13)] +
           [(a, b) for a in range(14, 18) for b in range(a + 1, 18)] + [(17, 18), (17, 19)] +
           [(a, b) for a in range(20, 26) for b in range(a + 1, 26)] + [(25, 26)])
    src = [a for a, b in und] + ([] if directed else [b for a, b in und])
    dst = [b for a, b in und] + ([] if directed else [a for a, b in und])
    out.append((27, src, dst))
    return out


@pytest.mark.parametrize("name", sorted(ORBIT_QUERIES))
@pytest.mark.parametrize("directed", [False, True])
def test_orbit_fold_plan_is_exact(name, directed):
    """The orbit fold's plan (core symmetry conditions, signatures,
    multiplier, orbit positions) evaluated by brute force equals the
    oracle's count."""
    k, arcs, _ = ORBIT_QUERIES[name]
    for n, src, dst in _orbit_graphs(directed, k):
        _orbit_case(name, directed, k, arcs, n, src, dst)


def _orbit_case(name, directed, k, arcs, n, src, dst):
    if directed:
        arcs = [(a, b) for a, b in arcs if a < b] + [(b, a) for a, b in arcs if a > b and (a + b) % 3 == 0]
    out_adj = [set() for _ in range(n)]
    in_adj = [set() for _ in range(n)]
    for u, v in zip(src, dst):
        out_adj[u].add(v)
        in_adj[v].add(u)
    sym = all(u in out_adj[v] for u in range(n) for v in out_adj[u])
    q = cb.Query.from_arcs(k, arcs)
    lv, aut = q.plan_levels(sym, cb.FLAG_SYMMETRY_BREAK)
    og = O.Graph.from_arrays(n, np.array(src, np.uint32), np.array(dst, np.uint32))
    want = O.count(og, O.Graph.from_arcs(k, arcs), q.order)[0]
    if lv[k - 1]["ofold"]:
        assert lv[k - 2]["fold"] == 1
        got = _brute_orbit_total(q, arcs, lv, aut, n, out_adj, in_adj)
        assert got == want, (name, directed, lv[k - 1]["ofold"], aut)
    lvn, autn = q.plan_levels(sym, cb.FLAG_SYMMETRY_BREAK | cb.FLAG_NO_ORBIT_FOLD)
    assert all(l["ofold"] == 0 for l in lvn)


def _pair_queries():
    """Queries whose last two vertices may be pendants on one vertex: stars,
    tails on one or two vertices, a path, random trees."""
    sym = lambda es: [a for e in es for a in (e, e[::-1])]
    qs = [cb.named_query_arcs(x) for x in ("3-star", "4-path")]
    qs.append((5, sym([(0, 1), (1, 2), (2, 0), (0, 3), (0, 4)])))  # two tails on one vertex
    qs.append((5, sym([(0, 1), (1, 2), (2, 0), (0, 3), (1, 4)])))  # tails on two vertices
    qs.append((5, sym([(0, 1), (0, 2), (0, 3), (0, 4)])))          # 4-star
    qs += [(5 + s % 2, cb.random_query_arcs(5 + s % 2, 0.0, 9100 + s)) for s in range(4)]
    return qs


def _brute_pair_total(q, qarcs, lv, aut, n, out_adj, in_adj):
    """aut x the pendant-pair closed form as the counting kernel evaluates
    it: every embedding of the first k - 2 positions that satisfies the
    plan's masks and signatures, times |A'| |B'| - |A' n B'| (kind 1) or
    C(|A'|, 2) (kind 2), A' and B' the two pendants' windows of their list
    minus the matched vertices (no signature test for the pendants: the
    plan holds that the joins imply it)."""
    k = q.k
    order = q.order
    arcs = set(qarcs)
    kind = lv[k - 3]["fold2"]
    m = []
    total = 0

    def fits(i, v):
        if v in m:
            return False
        if lv[i]["sig"] and (len(in_adj[v]) < lv[i]["qin"] or len(out_adj[v]) < lv[i]["qout"]):
            return False
        for j in range(i):
            if (order[i], order[j]) in arcs and m[j] not in out_adj[v]:
                return False
            if (order[j], order[i]) in arcs and v not in out_adj[m[j]]:
                return False
            if ((lv[i]["gt"] >> j) & 1) and not v > m[j]:
                return False
            if ((lv[i]["lt"] >> j) & 1) and not v < m[j]:
                return False
        return True

    def window(pos):
        x = order[pos]
        a = [j for j in range(k - 2) if (order[j], x) in arcs or (x, order[j]) in arcs]
        assert len(a) == 1
        j = a[0]
        lst = out_adj[m[j]] if (order[j], x) in arcs else in_adj[m[j]]
        lo, hi = 0, 1 << 40
        for jj in range(k - 2):  # conditions on earlier positions (the pen bit excluded)
            if (lv[pos]["gt"] >> jj) & 1:
                lo = max(lo, m[jj] + 1)
            if (lv[pos]["lt"] >> jj) & 1:
                hi = min(hi, m[jj])
        return {t for t in lst if lo <= t < hi} - set(m)

    def dfs(i):
        nonlocal total
        if i == k - 2:
            A, B = window(k - 2), window(k - 1)
            total += len(A) * (len(A) - 1) // 2 if kind == 2 else len(A) * len(B) - len(A & B)
            return
        for v in range(n):
            if fits(i, v):
                m.append(v)
                dfs(i + 1)
                m.pop()

    dfs(0)
    return total * aut


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("flags", [0, cb.FLAG_SYMMETRY_BREAK])
def test_pendant_pair_plan_is_exact(directed, flags):
    """Where the plan folds a pendant pair, its closed form over the plan's
    own masks equals the oracle's count; every fold is on one list."""
    folded = 0
    for qi, (k, arcs) in enumerate(_pair_queries()):
        if directed:
            arcs = [(a, b) for a, b in arcs if a < b]
        for n, src, dst in _orbit_graphs(directed, k):
            out_adj = [set() for _ in range(n)]
            in_adj = [set() for _ in range(n)]
            for u, v in zip(src, dst):
                out_adj[u].add(v)
                in_adj[v].add(u)
            sym = all(u in out_adj[v] for u in range(n) for v in out_adj[u])
            q = cb.Query.from_arcs(k, arcs)
            lv, aut = q.plan_levels(sym, flags)
            if not lv[k - 3]["fold2"]:
                continue
            folded += 1
            og = O.Graph.from_arrays(n, np.array(src, np.uint32), np.array(dst, np.uint32))
            want = O.count(og, O.Graph.from_arcs(k, arcs), q.order)[0]
            assert _brute_pair_total(q, arcs, lv, aut, n, out_adj, in_adj) == want, (qi, directed, flags)
    assert folded >= 6


def test_orbit_fold_plan_shape():
    q = cb.Query.from_arcs(*cb.named_query_arcs("4-clique+pendant"))
    lv, aut = q.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)
    k = q.k
    # core K4 (|Aut| 24), the pendant's clique vertex has an orbit of 4
    assert bin(lv[k - 1]["ofold"]).count("1") == 4 and aut == 6
    assert lv[k - 2]["fold"] == 1 and lv[k - 2]["fuse"] == 1
    # the core's chain orders all four clique positions
    assert lv[1]["gt"] and lv[2]["gt"] and lv[3]["gt"]
    # without symmetry breaking: the plain fold, no orbit
    lv0, aut0 = q.plan_levels(True, 0)
    assert lv0[k - 1]["ofold"] == 0 and aut0 == 1


def test_query_prefix_keeps_the_first_levels_plan():
    """A prefix query's plan is the full plan's first j levels: same joins and
    signatures, the signature tested at every level, no closed form."""
    for k, arcs in [cb.named_query_arcs("house"), cb.named_query_arcs("4-clique+pendant"),
                    (6, cb.random_query_arcs(6, 0.3, 3)), (5, [(0, 1), (1, 2), (2, 0), (0, 3), (3, 4)])]:
        q = cb.Query.from_arcs(k, arcs)
        full, _ = q.plan_levels(True, 0)
        for j in range(1, k + 1):
            p = q.prefix(j)
            assert p.k == j and p.order == list(range(j))
            lv, aut = p.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)  # prefixes count plainly
            assert aut == 1
            for i in range(j):
                for key in ("joins", "qin", "qout", "gt", "lt"):
                    assert lv[i][key] == (full[i][key] if key not in ("gt", "lt") else 0), (k, j, i, key)
                assert lv[i]["sig"] == 1 and lv[i]["closed"] == 0 and lv[i]["ofold"] == 0
    with pytest.raises(cb.CutsError):
        q.prefix(0)


def test_pendant_pair_plan():
    """The pendant-pair closed form is planned where the last two vertices
    are pendants on the same earlier position: independent pendants (kind
    1), or interchangeable ones ordered by symmetry breaking (kind 2); never
    with CUTS_FLAG_NO_PAIR_FOLD, not when the two are adjacent, and not for
    pendants on two different positions (a path's ends)."""
    star = cb.Query.from_arcs(*cb.named_query_arcs("3-star"))
    lv, aut = star.plan_levels(True, 0)
    assert lv[1]["fold2"] == 1 and lv[2]["fold"] == 0 and aut == 1
    lv, aut = star.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)
    assert lv[1]["fold2"] == 2 and aut == 6
    lv, _ = star.plan_levels(True, cb.FLAG_NO_PAIR_FOLD)
    assert all(x["fold2"] == 0 for x in lv)
    path = cb.Query.from_arcs(*cb.named_query_arcs("4-path"))
    assert all(x["fold2"] == 0 for x in path.plan_levels(True, 0)[0])
    sym = lambda es: [a for e in es for a in (e, e[::-1])]
    tails = cb.Query.from_arcs(5, sym([(0, 1), (1, 2), (2, 0), (0, 3), (0, 4)]))  # two tails on one vertex
    assert tails.plan_levels(True, 0)[0][2]["fold2"] == 1
    assert tails.plan_levels(True, cb.FLAG_SYMMETRY_BREAK)[0][2]["fold2"] == 2
    # a triangle's last two vertices are adjacent: no pendant pair
    tri = cb.Query.from_arcs(*cb.named_query_arcs("4-clique+pendant"))
    assert all(x["fold2"] == 0 for x in tri.plan_levels(True, 0)[0])
