#!/usr/bin/env python
"""Benchmark: exact subgraph-isomorphism counting on one B200.

Workload (the mid-size plain-method configuration): an undirected Chung-Lu
graph with n = 1,000,000 vertices and exactly 10,000,000 distinct edges
(expected degrees from a power law with exponent 2.1, minimum 2, capped at
20,000; seed 0), int32 CSR resident in HBM; queries triangle and 4-clique +
pendant, each counted exactly along the score.cpp order with the root level
cut into 4 chunks, as the reference's `cuts <data> <query> 4`.  The input is
synthetic (this project's seeded generator): the reference's SNAP graphs are
not used.  The configuration's other two queries, house and 5-cycle, are not
in the timed step: root-sampled level sizes put ~2.5e12 and ~4.5e13 partial
matches at their third level (~1.4e13 and ~2.7e14 embeddings), beyond an
exact enumeration in a benchmark run by this or any vertex-at-a-time engine.

One step = the two counts.  value = matches per second of device time
(sum of counts / sum of device times; each count timed by CUDA events on the
engine's stream from its first kernel to its last, as the reference times
its search).  L2 is flushed (a 512 MB write) before every count, outside the
timed intervals.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuts|reference]

With N > 1 (torchrun, one rank per GPU) the roots are striped over ranks
(u % N == rank, as the reference's multi-node level 0) and the four counts are
summed over ranks; the total work is fixed, so scaling is "strong".

--impl reference times the CPU oracle (a C/OpenMP restatement of the
reference's algorithm, the same join order) on this host's cores over a
bounded root sample of the same workload; the reference itself has no CPU
implementation of the search.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "chung-lu n=1e6 m=1e7 gamma=2.1 cap=2e4 seed=0; triangle, 4-clique+pendant; chunks=4",
    "n": 1_000_000, "m": 10_000_000, "gamma": 2.1, "wmin": 2.0, "cap": 20000.0, "seed": 0,
    "queries": ["triangle", "4-clique+pendant"],
    "chunks": 4,
}
METRIC = "matches/s (exact counts, 1M-vertex power-law graph)"
UNIT = "matches/s"


def _env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Clocks:
    """nvidia-smi samples of one GPU during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def make_graph():
    import cuts_b200 as cb
    w = WORKLOAD
    return cb.HostGraph.chung_lu(w["n"], w["m"], w["gamma"], w["wmin"], w["cap"], w["seed"])


def make_queries():
    import cuts_b200 as cb
    return [(name,) + cb.named_query_arcs(name) for name in WORKLOAD["queries"]]


# ---------------------------------------------------------------------------
# CPU oracle (cpu_baseline and --impl reference)
# ---------------------------------------------------------------------------

def cpu_sample(h, queries, budget_s=20.0):
    """Time the oracle on a root sample of each query, sized so the whole sample
    takes about budget_s seconds; returns (matches/s, cores, description)."""
    from oracle import oracle as O
    import numpy as np
    oo, oa, _, _ = h.csr()
    od = O.Graph.from_csr(h.n, oo, oa)
    cores = os.cpu_count() or 1
    total_cnt, total_t, parts = 0, 0.0, []
    per_q = budget_s / len(queries)
    import cuts_b200 as cb
    for name, k, arcs in queries:
        order = cb.Query.from_arcs(k, arcs).order
        oq = O.Graph.from_arcs(k, arcs)
        n0 = h.n
        # grow a contiguous root slice (vertex-id order; weights are i.i.d. per
        # vertex, so a slice is an unbiased sample) until it takes per_q / 4
        span = 8
        while True:
            t0 = time.perf_counter()
            cnt, lv, _ = O.count(od, oq, order, 0, span, cores)
            dt = time.perf_counter() - t0
            if dt >= per_q / 4 or span >= n0:
                break
            span = min(n0, span * 4 if dt < per_q / 64 else span * 2)
        total_cnt += cnt
        total_t += dt
        parts.append(f"{name}: first {span} roots ({100.0 * span / n0:.3f}% of L_0) {dt:.2f}s")
    return total_cnt / max(total_t, 1e-9), cores, "; ".join(parts)


REF_SAFE_DEGREE = 32768 + 112   # cuts_ref_b148: per-warp helper of 32,768 words past 112 in smem
REF_TABLE_WORDS = 3.5e9          # its trie table (u32 words, every level of a trunk)
REF_FINAL_WORDS = 4.5e10         # its managed final table


def reference_gpu(h, queries, level_sizes, counts, chunks):
    """Time the reference binary (built for sm_100a, 148-SM grid, enlarged
    candidate helper) on the workload's queries that it can run without
    overflowing its fixed tables; the others are reported as unsafe and not
    launched.  Returns {query: {...}}."""
    import re
    import tempfile
    from oracle import oracle as O
    binary = O.REF_CUTS.replace("cuts_ref", "cuts_ref_b148")
    out = {}
    if not os.path.exists(binary):
        return {"unavailable": "oracle/_ref/cuts_ref_b148 not built"}
    n, arcs, sym, maxd = h.info()
    with tempfile.TemporaryDirectory() as d:
        dpath = os.path.join(d, "data.g")
        h.write(dpath)
        import cuts_b200 as cb
        for (name, k, qarcs), lv, cnt in zip(queries, level_sizes, counts):
            stored = sum(lv[:-1])
            final_words = cnt + (k - 1) * (lv[-2] if k >= 2 else 0)
            if maxd >= REF_SAFE_DEGREE or stored > REF_TABLE_WORDS or final_words > REF_FINAL_WORDS:
                out[name] = {"run": False, "reason": f"would overflow the reference's fixed tables "
                                                     f"(levels {stored:.3g} words, final {final_words:.3g})"}
                continue
            qpath = os.path.join(d, name + ".g")
            cb.write_query(qpath, k, qarcs)
            t0 = time.perf_counter()
            r = subprocess.run([binary, dpath, qpath, str(chunks)], capture_output=True, text=True,
                               timeout=1800)
            wall = time.perf_counter() - t0
            m = None
            for line in r.stdout.splitlines()[::-1]:
                m = re.match(r"^(.*),(.*),([0-9.e+-]+)ms,(\d+)$", line.strip())
                if m:
                    break
            if not m:
                out[name] = {"run": True, "failed": (r.stdout + r.stderr)[-300:]}
                continue
            out[name] = {"run": True, "ms": float(m.group(3)), "count": int(m.group(4)),
                         "count_matches": int(m.group(4)) == cnt, "wall_s_with_load": wall}
    return out


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    h = make_graph()
    queries = make_queries()
    for _ in range(args.warmup):
        cpu_sample(h, queries, budget_s=args.cpu_budget / 2)
    vals, desc, cores = [], "", 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, cores, desc = cpu_sample(h, queries, budget_s=args.cpu_budget / 2)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded Chung-Lu generator)",
        "config": {"workload": WORKLOAD["workload"], "sample": "root slices per query"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# other configurations (reports, not the headline line)
# ---------------------------------------------------------------------------

def run_other_workload(args):
    import torch
    import cuts_b200 as cb
    from cuts_b200 import workloads as W
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    name = {"learned": "mid", "batched": "batched", "large": "large"}[args.workload]
    h = W.graph(name)
    g = h.upload(0)
    n, arcs, sym, maxd = h.info()
    gen_s = time.perf_counter() - t0
    rep = {"workload": args.workload, "graph": {"n": n, "arcs": arcs, "max_degree": maxd,
                                                "gen_upload_s": gen_s}}
    if args.workload == "learned":
        rep.update(W.run_learned(g, budget_ms=args.budget_ms, flags=args.flags))
    elif args.workload == "batched":
        rep.update(W.run_batched(g, flags=args.flags, query_budget_ms=args.batch_query_ms,
                                 budget_ms=args.batch_launch_ms))
    else:
        g.set_arena_bytes(48 << 30)
        res = {}
        qdefs = [("6-cycle",) + cb.named_query_arcs("6-cycle"), ("3-prism",) + cb.named_query_arcs("3-prism")]
        rq = None
        for s in range(1000):  # first seeded connected 6-vertex query with exactly 8 edges
            a = cb.random_query_arcs(6, 0.3, 5000 + s)
            if len(a) == 16:
                rq = ("random6e8", 6, a)
                break
        qdefs.append(rq)
        for qname, k, qarcs in qdefs:
            q = cb.Query.from_arcs(k, qarcs)
            fl = args.flags | cb.FLAG_SYMMETRY_BREAK
            est = None
            for stride in (1 << 20, 1 << 16, 1 << 12):  # root-stripe estimates, growing
                rs, ok = g.count_sample(q, 0, stride, budget_ms=10000.0, flags=fl)
                if not ok:
                    break
                est = {"stride": stride, "ms": rs.ms, "est_count": rs.count * stride,
                       "est_levels": [x * stride for x in rs.level_sizes],
                       "est_full_s": rs.ms * stride / 1e3}
            r, done = g.count_budget(q, args.budget_ms, chunks=8, flags=fl)
            res[qname] = {"finished": done, "count": r.count if done else None, "ms": r.ms,
                          "levels": r.level_sizes if done else None, "estimate": est}
        rep["queries"] = res
    print(json.dumps(rep), flush=True)
    return 0


# ---------------------------------------------------------------------------
# engine
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuts", choices=["cuts", "reference"])
    ap.add_argument("--flags", type=int, default=1,
                    help="CUTS_FLAG_* bits; default 1 = symmetry breaking (exact: one embedding "
                         "per automorphism orbit, scaled by |Aut(Q)|)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="also time the reference binary where it is safe to run")
    ap.add_argument("--workload", default="mid", choices=["mid", "learned", "batched", "large"],
                    help="mid = the headline line; the others print their own report line")
    ap.add_argument("--budget-ms", type=float, default=5000.0,
                    help="per-query time budget of the learned / large workloads")
    ap.add_argument("--batch-query-ms", type=float, default=50.0,
                    help="batched workload: each query's share of GPU time")
    ap.add_argument("--batch-launch-ms", type=float, default=60000.0,
                    help="batched workload: the launch's device-time budget")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "mid":
        return run_other_workload(args)

    import numpy as np
    import torch
    import cuts_b200 as cb

    rank, world, local = _env_rank()
    dev = local
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    h = make_graph()
    n, arcs, sym, maxd = h.info()
    g = h.upload(dev)
    queries = [(name, cb.Query.from_arcs(k, a)) for name, k, a in make_queries()]
    chunks = WORKLOAD["chunks"]
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.int32, device=f"cuda:{dev}")

    def count(q):
        if world > 1:
            return g.count_sharded(q, rank, world, chunks=chunks, flags=args.flags)
        return g.count(q, chunks=chunks, flags=args.flags, stats=True)

    def step(record):
        ms, cnts, launches = 0.0, [], 0
        for name, q in queries:
            flush.fill_(len(cnts))
            torch.cuda.synchronize(dev)
            r = count(q)
            ms += r.ms
            cnts.append(r.count)
            launches += r.launches
            if record is not None:
                record.append((name, r.count, r.ms))
        return ms, cnts, launches

    for _ in range(args.warmup):
        step(None)

    clocks = Clocks(dev)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    t0 = time.perf_counter()
    total_ms, launches, per_query = 0.0, 0, []
    counts = None
    for _ in range(args.steps):
        ms, cnts, la = step(per_query)
        total_ms += ms
        launches += la
        counts = cnts
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    if pg:
        pg.barrier()
    clk = clocks.stop()

    max_ms = total_ms
    if pg:
        from cuts_b200.dist import reduce_counts
        counts, max_ms = reduce_counts(counts, total_ms, device=f"cuda:{dev}")
    step_matches = sum(counts)
    value = step_matches * args.steps / (max_ms / 1e3)

    # end to end through the C ABI, on every rank (each its root stripe):
    # host CSR (pinned) -> device layout, counts, D2H of the counts; the
    # step's time is the slowest rank's wall clock
    oo, oa, _, _ = h.csr()
    oo_p = torch.from_numpy(oo.view(np.int64)).pin_memory().numpy().view(np.uint64)
    oa_p = torch.from_numpy(oa.view(np.int32)).pin_memory().numpy().view(np.uint32)
    h2d = oo_p.nbytes + oa_p.nbytes
    e2e_t = []
    for it in range(max(1, min(args.steps, 3)) + 1):
        if pg:
            pg.barrier()
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        g2 = cb.Graph.from_csr(n, oo_p, oa_p, device=dev)
        cnt_e = []
        for name, q in queries:
            if world > 1:
                cnt_e.append(g2.count_sharded(q, rank, world, chunks=chunks, flags=args.flags).count)
            else:
                cnt_e.append(g2.count(q, chunks=chunks, flags=args.flags).count)
        g2.close()
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t1
        if pg:
            from cuts_b200.dist import reduce_counts
            cnt_e, dt_ms = reduce_counts(cnt_e, dt * 1e3, device=f"cuda:{dev}")
            dt = dt_ms / 1e3
        if it > 0:  # first pass warms the allocator
            e2e_t.append(dt)
        assert sum(cnt_e) == step_matches
    e2e_val = step_matches / statistics.median(e2e_t)

    result = None
    if rank == 0:
        # live per-kernel timing for the roofline: one profiled pass (event
        # pairs around every level launch) plus the traffic model
        kern = {"last_level": [0.0, 0, 0], "expand": [0.0, 0, 0]}
        if world == 1:
            for name, q in queries:
                flush.fill_(7)
                torch.cuda.synchronize(dev)
                r = g.count(q, chunks=chunks, flags=args.flags, stats=True, profile=True,
                            alg_bytes=True)
                kern["last_level"][0] += r.last_level_ms
                kern["last_level"][1] += r.last_level_launches
                kern["last_level"][2] += r.last_level_bytes
                kern["expand"][0] += r.expand_ms
                kern["expand"][1] += r.expand_launches
        peak, peak_kind = measured_peaks()
        ll_ms, ll_n, ll_bytes = kern["last_level"]
        achieved = (ll_bytes / max(ll_n, 1)) / ((ll_ms / max(ll_n, 1)) / 1e3) / 1e9 if ll_ms else None
        traffic = ncu_traffic().get("last_level_bytes_per_launch")
        # the counting kernel of each query: fused with the level before, or flat
        sym = h.info()[2]
        kinds = []
        for name, q in queries:
            lv, _ = q.plan_levels(sym, args.flags)
            fused = any(x["fuse"] for x in lv) and os.environ.get("CUTS_NO_FUSE") != "1"
            kinds.append(f"{'k_fused' if fused else 'k_level_flat'}<count> ({name})")
        roofline = {
            "kernel": "last counted level: " + ", ".join(kinds),
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "peak_source": peak_kind,
            "alg_bytes_per_launch": ll_bytes / max(ll_n, 1) if ll_n else None,
            "avg_launch_ms": ll_ms / max(ll_n, 1) if ll_n else None,
            "share_of_kernel_time": ll_ms / max(ll_ms + kern["expand"][0], 1e-12) if ll_ms else None,
        }


        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, cores, desc = cpu_sample(h, [(nm,) + cb.named_query_arcs(nm) for nm, _ in queries],
                                        budget_s=args.cpu_budget)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}

        ref_gpu = None
        if args.ref_gpu and world == 1:
            lvls = []
            for name, q in queries:
                lvls.append(g.count(q, chunks=chunks, stats=True).level_sizes)
            ref_gpu = reference_gpu(h, make_queries(), lvls, counts, chunks)

        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu generator; SNAP graphs not used)",
            "config": {"workload": WORKLOAD["workload"], "n": n, "arcs": arcs, "max_degree": maxd,
                       "flags": args.flags, "l2": "flushed (512 MB write) before every count",
                       "parallelism": f"root stripes x{world}" if world > 1 else "1 GPU"},
            "counts": dict(zip([nm for nm, _ in queries], counts)),
            "ms_per_query": {nm: statistics.mean([t for a, c, t in per_query if a == nm])
                             for nm, _ in queries} if world == 1 else None,
            "wall_s_timed": wall,
            "clocks": clk,
            "gpu_launches": launches,
            "roofline": roofline,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d) * world,
                    "d2h_bytes_per_step": 8 * len(queries) * world,
                    "note": "wall clock, slowest rank: CSR copy to each GPU + on-device layout + "
                            "the counts (each rank its root stripe) + count reads"},
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
        }
        print(json.dumps(result), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
