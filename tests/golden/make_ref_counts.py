"""Generate tests/golden/ref_counts.json: counts of the reference binary built
for sm_100a by `make -C oracle ref` (oracle/_ref/cuts_ref_b148: the reference
with its grid set to 148 SMs and its fixed buffers resized so it can start and
stay in bounds on a B200 host -- the stock build's 280 GB managed reservation
fails there -- the algorithm untouched) on this project's seeded inputs.
Runs on a GPU machine:

    python tests/golden/make_ref_counts.py

Every input is checked safe for the reference before it runs (the
reference's unchecked buffers): maximum degree below its per-warp candidate
helper (15,112 entries in the stock build, 32,880 in this resized one), level
sizes (from this project's oracle) far below its u32 tables and its
(resized) 4e9-word final table, and a mean degree above 2 (arcs >= 2n): on
sparser graphs the reference switches to its 8-lane kernel, whose last level
reads shared memory at warp * 112 + i for up to 128 warps per block
(device_funcs.cu:708-716) -- far past its 5,120-entry array, an out-of-range
shared-memory access -- so it is not run there.  Each case runs
`cuts <data> <query>` and `cuts <data> <query> 4`; the fixture records the
graph and query recipes (not their text) with the counts the reference
printed.  `large_cases` adds the benchmark's 1M-vertex graph (triangle,
maximum degree 21,618 < 32,880; ~2e7 level-1 entries).
"""
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import cuts_b200 as cb  # noqa: E402
from oracle import oracle as O  # noqa: E402

HELPER_SAFE_DEGREE = 32768
GRAPHS = {
    "er2k": ("er", dict(n=2000, p=10.0 / 1999, seed=3)),
    "er10k": ("er", dict(n=10000, p=8.0 / 9999, seed=0)),
    "cl3k": ("cl", dict(n=3000, m=12000, gamma=2.2, wmin=2.0, cap=60.0, seed=8)),
    "cl5k": ("cl", dict(n=5000, m=20000, gamma=2.1, wmin=2.0, cap=100.0, seed=5)),
}


def make_graph(kind, p):
    if kind == "er":
        return cb.HostGraph.erdos_renyi(p["n"], p["p"], p["seed"])
    return cb.HostGraph.chung_lu(p["n"], p["m"], p["gamma"], p["wmin"], p["cap"], p["seed"])


def queries():
    qs = {name: cb.named_query_arcs(name) for name in
          ["triangle", "4-cycle", "5-cycle", "house", "4-clique+pendant", "3-prism",
           "3-path", "4-path", "3-star"]}
    for s in range(8):
        k = 4 + s % 3
        qs[f"rand{k}_{s}"] = (k, cb.random_query_arcs(k, 0.35, 700 + s))
    # directed queries (orientation of random undirected ones)
    for s in range(4):
        k = 3 + s % 3
        und = cb.random_query_arcs(k, 0.6, 800 + s)
        qs[f"dir{k}_{s}"] = (k, [a for a in und if (a[0] + a[1] + s) % 3 != 0 or a[0] < a[1]])
    return qs


LINE = re.compile(r"^(.*),(.*),([0-9.e+-]+)ms,(\d+)$")


def run_ref(binary, dpath, qpath, trunks=None, timeout=600):
    cmd = [binary, dpath, qpath] + ([str(trunks)] if trunks else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    for line in r.stdout.splitlines()[::-1]:
        m = LINE.match(line.strip())
        if m:
            return int(m.group(4)), float(m.group(3))
    raise RuntimeError(f"no result line from {cmd}: rc={r.returncode} {r.stdout[-500:]} {r.stderr[-500:]}")


LARGE = {"c2": dict(n=1_000_000, m=10_000_000, gamma=2.1, wmin=2.0, cap=20000.0, seed=0)}


def large_cases(binary):
    cases = []
    with tempfile.TemporaryDirectory() as d:
        p = LARGE["c2"]
        h = cb.HostGraph.chung_lu(p["n"], p["m"], p["gamma"], p["wmin"], p["cap"], p["seed"])
        n, arcs, sym, maxd = h.info()
        assert maxd < HELPER_SAFE_DEGREE and arcs >= 2 * n, (maxd, arcs)
        dpath = os.path.join(d, "c2.g")
        h.write(dpath)
        k, qarcs = cb.named_query_arcs("triangle")
        qpath = os.path.join(d, "triangle.g")
        cb.write_query(qpath, k, qarcs)
        c1, ms1 = run_ref(binary, dpath, qpath, timeout=1800)
        c4, ms4 = run_ref(binary, dpath, qpath, 4, timeout=1800)
        cases.append({"graph": "c2", "graph_kind": "cl", "graph_params": p, "query": "triangle", "k": k,
                      "arcs": qarcs, "ref_count": c1, "ref_count_trunks4": c4, "ref_ms": ms1,
                      "ref_ms_trunks4": ms4})
        print("c2 triangle", c1, c4, f"{ms1:.1f}ms", f"{ms4:.1f}ms", flush=True)
    return cases


def main():
    binary = O.REF_CUTS.replace("cuts_ref", "cuts_ref_b148")
    assert os.path.exists(binary), "build it: make -C oracle ref"
    out = {"generator": "tests/golden/make_ref_counts.py", "binary": "oracle/_ref/cuts_ref_b148",
           "cases": []}
    with tempfile.TemporaryDirectory() as d:
        for gname, (kind, params) in GRAPHS.items():
            h = make_graph(kind, params)
            n, arcs, sym, maxd = h.info()
            assert maxd < HELPER_SAFE_DEGREE and arcs >= 2 * n, (gname, maxd, arcs)
            dpath = os.path.join(d, gname + ".g")
            h.write(dpath)
            oo, oa, _, _ = h.csr()
            od = O.Graph.from_csr(n, oo, oa)
            for qname, (k, qarcs) in queries().items():
                q = cb.Query.from_arcs(k, qarcs)
                cnt, lv, _ = O.count(od, O.Graph.from_arcs(k, qarcs), q.order)
                # the reference stores every level of a trunk in one u32 table of
                # ~3.6e9 words and writes each match into its final table
                if sum(lv[:-1]) > 5e8 or cnt > 2e9:
                    continue
                qpath = os.path.join(d, qname + ".g")
                cb.write_query(qpath, k, qarcs)
                c1, ms1 = run_ref(binary, dpath, qpath)
                c4, ms4 = run_ref(binary, dpath, qpath, 4)
                out["cases"].append({"graph": gname, "graph_kind": kind, "graph_params": params,
                                     "query": qname, "k": k, "arcs": qarcs, "ref_count": c1,
                                     "ref_count_trunks4": c4, "ref_ms": ms1, "ref_ms_trunks4": ms4,
                                     "oracle_count": cnt})
                print(gname, qname, c1, c4, cnt, f"{ms1:.2f}ms", flush=True)
    out["large_cases"] = large_cases(binary)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_counts.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {len(out['cases'])} cases to {dst}")


if __name__ == "__main__":
    main()
