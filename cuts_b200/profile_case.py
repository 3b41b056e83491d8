"""One small, self-contained counting run, sized for an ncu capture.

    python -m cuts_b200.profile_case [--query triangle] [--graph c2]
                                     [--arena-mb 1024] [--repeat 2] [--batch N]

Builds the seeded workload graph, keeps the trie arena small (so a profiler
that saves and restores device memory between passes has little to move),
warms up once and counts the query `--repeat` times (or runs a batch of N
seeded random queries through the batched engine with --batch).
"""
import argparse
import sys
import time

import cuts_b200 as cb

GRAPHS = {
    # mid-size plain-method workload: 1M vertices, 10M edges, exponent 2.1, cap 20,000
    "c2": lambda: cb.HostGraph.chung_lu(1_000_000, 10_000_000, 2.1, 2.0, 20000.0, 0),
    # small plain-method workload: ER, 10,000 vertices, mean degree 8
    "c1": lambda: cb.HostGraph.erdos_renyi(10_000, 8.0 / 9_999, 0),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--graph", default="c2", choices=sorted(GRAPHS))
    ap.add_argument("--query", default="triangle")
    ap.add_argument("--arena-mb", type=int, default=1024)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--chunks", type=int, default=4)
    ap.add_argument("--flags", type=int, default=0)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--stripe", type=int, default=1,
                    help="count only the roots u with u %% stripe == 0 (a smaller case)")
    a = ap.parse_args(argv)
    h = GRAPHS[a.graph]()
    g = h.upload(0)
    g.set_arena_bytes(a.arena_mb << 20)
    if a.batch:
        qs = []
        for s in range(a.batch):
            k = 3 + s % 5
            qs.append(cb.Query.from_arcs(k, cb.random_query_arcs(k, [0.2, 0.4, 0.6][s % 3], s)))
        b = g.batch(qs, flags=a.flags)
        b.run()
        for _ in range(a.repeat):
            counts, status, ms = b.run()
            print(f"batch {a.batch}: {ms:.3f} ms, {sum(counts)} matches, "
                  f"{sum(1 for s in status if s)} unfinished", flush=True)
        return 0
    q = cb.Query.from_arcs(*cb.named_query_arcs(a.query))

    def run():
        if a.stripe > 1:
            return g.count_sharded(q, 0, a.stripe, chunks=a.chunks, flags=a.flags)
        return g.count(q, chunks=a.chunks, flags=a.flags, stats=True)

    run()
    for _ in range(a.repeat):
        t = time.perf_counter()
        r = run()
        print(f"{a.query}: count {r.count} in {r.ms:.3f} ms (wall {1e3 * (time.perf_counter() - t):.1f}), "
              f"levels {r.level_sizes}, launches {r.launches}, chunks {r.chunks}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
