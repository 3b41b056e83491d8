"""Generate tests/golden/orders.json: the reference's own matching order and
P/C join lists for a fixed set of seeded queries.

Runs oracle/_ref/ref_order, the harness linked against the reference's
unmodified graph.cpp/score.cpp/util.cpp/common.cpp (built by
`make -C oracle ref`).  The queries are this project's own seeded random
queries (undirected and directed), written to a temporary directory; the
fixture stores each query's arcs together with the reference's output, so
the pin can be checked without the reference present.

    python tests/golden/make_orders.py
"""
import json
import os
import random
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_ORDER  # noqa: E402


def seeded_queries():
    rng = random.Random(20240601)
    out = []
    for i in range(160):
        k = rng.randint(2, 12)
        p = rng.choice([0.0, 0.1, 0.2, 0.3, 0.5, 0.8])
        edges = set()
        for v in range(1, k):  # random attachment spanning tree
            edges.add((rng.randrange(v), v))
        for a in range(k):
            for b in range(a + 1, k):
                if rng.random() < p:
                    edges.add((a, b))
        directed = i % 3 == 2
        arcs = []
        for a, b in sorted(edges):
            if directed:
                r = rng.random()
                if r < 0.4:
                    arcs.append((a, b))
                elif r < 0.8:
                    arcs.append((b, a))
                else:
                    arcs += [(a, b), (b, a)]
            else:
                arcs += [(a, b), (b, a)]
        if i % 11 == 5:  # occasional self-loop
            v = rng.randrange(k)
            arcs.append((v, v))
        rng.shuffle(arcs)
        out.append({"k": k, "arcs": arcs})
    return out


def parse_line(line):
    _, order, P, Cs = line.split(" ")
    order = [int(x) for x in order[len("order="):].split(",")]

    def lists(s):
        res = []
        for part in s.split(";"):
            _, vals = part.split(":")
            res.append([int(x) for x in vals.split(",")] if vals else [])
        return res

    return order, lists(P[2:]), lists(Cs[2:])


def main():
    qs = seeded_queries()
    with tempfile.TemporaryDirectory() as d:
        paths = []
        for i, q in enumerate(qs):
            p = os.path.join(d, f"q{i}.g")
            with open(p, "w") as f:
                f.write(f"{q['k']}\n")
                for a, b in q["arcs"]:
                    f.write(f"{a}\t{b}\n")
            paths.append(p)
        out = subprocess.run([REF_ORDER] + paths, check=True, capture_output=True, text=True).stdout
    lines = out.strip().split("\n")
    assert len(lines) == len(qs)
    for q, line in zip(qs, lines):
        q["order"], q["P"], q["C"] = parse_line(line)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "orders.json")
    with open(dst, "w") as f:
        json.dump({"generator": "tests/golden/make_orders.py", "source": "oracle/_ref/ref_order",
                   "queries": qs}, f, separators=(",", ":"))
    print(f"wrote {len(qs)} reference orders to {dst}")


if __name__ == "__main__":
    main()
