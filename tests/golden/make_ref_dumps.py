"""Generate tests/golden/ref_dumps.json: the match sets the reference binary
itself writes to ans.txt, recorded as canonical digests.

The binary is oracle/_ref/cuts_ref_b148_dump (`make -C oracle ref`): the
reference built for sm_100a with its grid set to 148 SMs, its fixed buffers
resized for a B200 host, and its hard-coded `write_to_disk = false`
(main.cu:31) switched on; its dump is write_match_to_disk (util.cpp:53-74)
over the final table the last level fills (device_funcs.cu:363-391).  Runs on
a GPU machine:

    python tests/golden/make_ref_dumps.py

Each case runs `cuts_ref_b148_dump <data> <query>` in a scratch directory
and reads the ans.txt it leaves.  A line "(q,d)(q,d)..." is canonicalised to
the tuple of data vertices indexed by query vertex; the set of tuples, sorted,
is written one per line ("d0 d1 ...\\n") and hashed with SHA-256.  The fixture
keeps the digest and the number of lines, and the digest of the oracle's own
enumeration of the same case (it must agree).  Inputs are the small seeded
graphs of make_ref_counts.py, checked safe for the reference the same way
(maximum degree below its helper, mean degree above 2, at most 2e6 matches).
"""
import hashlib
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

GRAPHS = {
    "er2k": ("er", dict(n=2000, p=10.0 / 1999, seed=3)),
    "cl3k": ("cl", dict(n=3000, m=12000, gamma=2.2, wmin=2.0, cap=60.0, seed=8)),
}
QUERIES = ["triangle", "4-cycle", "house", "4-clique+pendant", "3-path", "3-star"]
PAIR = re.compile(r"\((\d+),(\d+)\)")


def make_graph(kind, p):
    if kind == "er":
        return cb.HostGraph.erdos_renyi(p["n"], p["p"], p["seed"])
    return cb.HostGraph.chung_lu(p["n"], p["m"], p["gamma"], p["wmin"], p["cap"], p["seed"])


def canonical_rows_from_lines(lines, k):
    rows = []
    for line in lines:
        line = line.strip()
        if not line:
            continue
        by_q = dict((int(a), int(b)) for a, b in PAIR.findall(line))
        rows.append(tuple(by_q[v] for v in range(k)))
    return rows


def digest(rows):
    h = hashlib.sha256()
    for r in sorted(rows):
        h.update((" ".join(str(x) for x in r) + "\n").encode())
    return h.hexdigest()


def main():
    binary = os.path.join(ROOT, "oracle", "_ref", "cuts_ref_b148_dump")
    assert os.path.exists(binary), "build it: make -C oracle ref"
    out = {"generator": "tests/golden/make_ref_dumps.py", "binary": "oracle/_ref/cuts_ref_b148_dump",
           "canonical": "sorted tuples of data vertices by query vertex, one per line, space separated",
           "cases": []}
    with tempfile.TemporaryDirectory() as d:
        for gname, (kind, params) in GRAPHS.items():
            h = make_graph(kind, params)
            n, arcs, sym, maxd = h.info()
            assert maxd < 32768 and arcs >= 2 * n, (gname, maxd, arcs)
            dpath = os.path.join(d, gname + ".g")
            h.write(dpath)
            oo, oa, _, _ = h.csr()
            od = O.Graph.from_csr(n, oo, oa)
            for qname in QUERIES:
                k, qarcs = cb.named_query_arcs(qname)
                q = cb.Query.from_arcs(k, qarcs)
                cnt, lv, _ = O.count(od, O.Graph.from_arcs(k, qarcs), q.order)
                if cnt > 2_000_000 or sum(lv[:-1]) > 5e8:
                    continue
                qpath = os.path.join(d, qname + ".g")
                cb.write_query(qpath, k, qarcs)
                work = os.path.join(d, f"run_{gname}_{qname}")
                os.makedirs(work)
                r = subprocess.run([binary, dpath, qpath], capture_output=True, text=True, timeout=600,
                                   cwd=work)
                assert r.returncode == 0, (gname, qname, r.stdout[-500:], r.stderr[-500:])
                with open(os.path.join(work, "ans.txt")) as f:
                    rows = canonical_rows_from_lines(f, k)
                want = O.enumerate_matches(od, O.Graph.from_arcs(k, qarcs), q.order)
                case = {"graph": gname, "graph_kind": kind, "graph_params": params, "query": qname,
                        "k": k, "lines": len(rows), "sha256": digest(rows), "oracle_count": cnt,
                        "oracle_sha256": digest(want)}
                out["cases"].append(case)
                print(gname, qname, len(rows), cnt, case["sha256"] == case["oracle_sha256"], flush=True)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_dumps.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['cases'])} cases to {dst}")


if __name__ == "__main__":
    main()
