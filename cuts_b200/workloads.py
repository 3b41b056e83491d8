"""Seeded workloads beyond the headline benchmark.

* learned: the 1M-vertex power-law graph (exponent 2.1, cap 20,000, 10M
  edges); 200 random connected queries (5-8 vertices, spanning tree plus
  extra edges at density 0.3, seeds 0..199); the cost model trained on
  per-level sizes of 2,000 other queries (seeds 10,000..11,999); plain
  (score order, one query at a time) against learned order + one batched
  launch.
* batched: a 4M-vertex power-law graph (exponent 2.2, 40M edges, cap
  20,000); 4,096 random connected queries of 3-7 vertices, density
  0.2-0.6, in one persistent CUDA-graph launch, launch shape autotuned.
* large: a 16M-vertex power-law graph (exponent 2.1, cap 100,000, 256M
  edges, ~2 GB int32 CSR); 6-cycle, 3-prism and a seeded random 6-vertex /
  8-edge query in 8 chunks.

Queries whose exact count does not finish within the stated time budget are
reported as unfinished, never as a count.
"""
from __future__ import annotations

import math
import time
from typing import Dict, List, Tuple

import numpy as np

import cuts_b200 as cb
from cuts_b200 import learned as L


def eval_queries(n: int = 200, seed0: int = 0, kmin: int = 5, kmax: int = 8, p: float = 0.3):
    rng = np.random.default_rng(12345 + seed0)
    out = []
    for s in range(n):
        k = int(rng.integers(kmin, kmax + 1))
        out.append((k, cb.random_query_arcs(k, p, seed0 + s)))
    return out


def batched_queries(n: int = 4096, seed0: int = 0):
    rng = np.random.default_rng(777 + seed0)
    out = []
    for s in range(n):
        k = int(rng.integers(3, 8))
        p = float(rng.uniform(0.2, 0.6))
        out.append((k, cb.random_query_arcs(k, p, seed0 + s)))
    return out


def graph(name: str) -> "cb.HostGraph":
    if name == "mid":
        return cb.HostGraph.chung_lu(1_000_000, 10_000_000, 2.1, 2.0, 20000.0, 0)
    if name == "batched":
        return cb.HostGraph.chung_lu(4_000_000, 40_000_000, 2.2, 2.0, 20000.0, 0)
    if name == "large":
        return cb.HostGraph.chung_lu(16_000_000, 256_000_000, 2.1, 2.0, 100000.0, 0)
    raise ValueError(name)


def _log(*a):
    import sys
    print(*a, file=sys.stderr, flush=True)


def plain_pass(g: "cb.Graph", queries, budget_ms: float, flags: int = 0, orders=None, tag="plain"):
    """One query at a time through the level engine, each under budget_ms
    (host check between chunks, device deadline inside the kernels); the
    score order unless `orders` gives one per query."""
    res = []
    t0 = time.perf_counter()
    for i, (k, arcs) in enumerate(queries):
        q = cb.Query.from_arcs(k, arcs)
        if orders is not None:
            q.set_order(orders[i])
        r, done = g.count_budget(q, budget_ms, flags=flags)
        res.append((done, r.count if done else None, r.ms))
        if (i + 1) % 50 == 0:
            _log(f"{tag}: {i + 1}/{len(queries)} queries, {sum(d for d, _, _ in res)} finished, "
                 f"{time.perf_counter() - t0:.1f} s")
    return res, time.perf_counter() - t0


def train_model(g: "cb.Graph", n_train: int = 2000, orders_per_query: int = 4, stride: int = 1 << 16,
                epochs: int = 400, seed: int = 10000, time_budget_s: float = 120.0,
                run_budget_ms: float = 100.0):
    train_q = eval_queries(n_train, seed0=seed)
    t0 = time.perf_counter()
    samples = L.collect(g, train_q, orders_per_query=orders_per_query, stride=stride, seed=1,
                        time_budget_s=time_budget_s, run_budget_ms=run_budget_ms, prefixes=True)
    t_collect = time.perf_counter() - t0
    _log(f"training data: {len(samples)} runs in {t_collect:.1f} s")
    X, y, _ = L.features(g, train_q, samples)
    t1 = time.perf_counter()
    model = L.train(X, y, epochs=epochs, batch=4096, lr=2e-3)
    t_train = time.perf_counter() - t1
    info = {"samples": len(samples), "queries_logged": len({s.query for s in samples}),
            "complete_runs": sum(1 for s in samples if len(s.levels) == train_q[s.query][0]),
            "rows": int(len(y)), "collect_s": t_collect, "train_s": t_train,
            "fit_mae_nats": L.prediction_error(model, X, y)}
    _log(f"model: {info}")
    return model, info


def estimate_orders(g: "cb.Graph", qdefs, orders_a, orders_b, stride: int, budget_ms: float,
                    flags: int = 0, shard: int = 1):
    """Estimated device time of a full exact count of each query under two
    orders, from the same root stripe (u % stride == shard; the stripe's time
    x stride); None where the stripe itself exceeds budget_ms."""
    out = []
    t0 = time.perf_counter()
    for i, (k, arcs) in enumerate(qdefs):
        row = []
        for orders in (orders_a, orders_b):
            q = cb.Query.from_arcs(k, arcs)
            q.set_order(orders[i])
            r, done = g.count_sample(q, shard, stride, budget_ms, flags)
            row.append(r.ms * stride if done else None)
        out.append(row)
        if (i + 1) % 50 == 0:
            _log(f"estimates: {i + 1}/{len(qdefs)} queries, {time.perf_counter() - t0:.1f} s")
    return out


def run_learned(g: "cb.Graph", n_eval: int = 200, n_train: int = 2000, budget_ms: float = 100.0,
                model=None, train_budget_s: float = 120.0, flags: int = 0,
                est_stride: int = 1 << 12, est_budget_ms: float = 300.0,
                choose_stride: int = 1 << 14, choose_budget_ms: float = 100.0):
    """The 200 evaluation queries three ways, each query under the same
    budget of budget_ms of the whole GPU:
      plain    -- score order, level engine, one query at a time;
      learned  -- the learned order (the model's three best proposals and the
                  score order timed on a root stripe of 1/choose_stride of
                  the roots, the fastest kept), level engine, one query at a
                  time;
      learned_batched -- the learned order, all queries in one persistent
                  launch (cheapest measured first), each limited to
                  budget_ms of GPU time by the batched kernel's per-query limit.
    queries/s = finished queries / seconds (planning included).  Alongside:
    the estimated device time of each query's full exact count under the
    score and the learned order, from another root stripe (shard 1), so the
    choice and its evaluation use different roots."""
    info = {}
    if model is None:
        model, info = train_model(g, n_train=n_train, time_budget_s=train_budget_s)
    qdefs = eval_queries(n_eval)
    plain, plain_s = plain_pass(g, qdefs, budget_ms, flags)
    t0 = time.perf_counter()
    qs, works, orders = [], [], []
    switched = model_switched = 0
    for k, arcs in qdefs:
        q = cb.Query.from_arcs(k, arcs)
        score = list(q.order)
        _, pw, sw = q.plan(g, cb.ORDER_LEARNED, model, beam=256, margin=2.0)
        model_switched += pw < sw
        q.set_order(score)
        # the model's proposals, measured on a small root stripe (shard 0)
        order, times = L.choose_order(g, q, model, proposals=3, stride=choose_stride,
                                      budget_ms=choose_budget_ms, flags=flags)
        switched += order != score
        qs.append(q)
        t = times.get(tuple(order))
        works.append(t if t is not None else math.inf)
        orders.append(order)
    plan_s = time.perf_counter() - t0
    _log(f"planned {n_eval} queries in {plan_s:.1f} s: {switched} orders changed by measured "
         f"proposals, {model_switched} by the model alone")
    score_orders = [cb.Query.from_arcs(k, arcs).order for k, arcs in qdefs]
    est = estimate_orders(g, qdefs, score_orders, orders, est_stride, est_budget_ms, flags)
    both = [(a, b) for a, b in est if a is not None and b is not None]
    est_rep = {
        "stride": est_stride, "stripe_budget_ms": est_budget_ms,
        "queries_estimated_both": len(both),
        "score_only": sum(1 for a, b in est if a is not None and b is None),
        "learned_only": sum(1 for a, b in est if a is None and b is not None),
        "sum_est_s_score": sum(a for a, _ in both) / 1e3,
        "sum_est_s_learned": sum(b for _, b in both) / 1e3,
        "geomean_speedup": (math.exp(sum(math.log(max(a, 1e-3) / max(b, 1e-3)) for a, b in both) / len(both))
                            if both else None),
        "learned_faster": sum(1 for a, b in both if b < a * 0.9),
        "learned_slower": sum(1 for a, b in both if b > a * 1.1),
        "est_full_s_quantiles_score": ([float(x) for x in np.quantile([a / 1e3 for a, _ in both],
                                                                       [0.1, 0.5, 0.9])] if both else None),
    }
    _log(f"estimates: {est_rep}")
    learned, learned_s = plain_pass(g, qdefs, budget_ms, flags, orders=orders, tag="learned")
    # cheapest measured stripe first
    rank = sorted(range(n_eval), key=lambda i: works[i])
    b = g.batch([qs[i] for i in rank], flags=flags)
    b.set_query_budget(budget_ms)
    t1 = time.perf_counter()
    counts_r, status_r, ms = b.run(budget_ms * n_eval)
    batch_wall = time.perf_counter() - t1
    counts = [0] * n_eval
    status = [0] * n_eval
    for j, i in enumerate(rank):
        counts[i], status[i] = counts_r[j], status_r[j]
    lb_s = plan_s + batch_wall
    done_p = [d for d, _, _ in plain]
    done_l = [d for d, _, _ in learned]
    done_b = [s == 0 for s in status]
    agree = all(c == pc for (d, pc, _), c, s in zip(plain, counts, status) if d and s == 0)
    agree = agree and all(lc == pc for (d, pc, _), (dl, lc, _) in zip(plain, learned) if d and dl)
    fin_k = lambda done: {k: sum(1 for (kk, _), d in zip(qdefs, done) if d and kk == k) for k in range(5, 9)}
    return {
        "queries": n_eval, "budget_ms_per_query": budget_ms,
        "plain": {"finished": sum(done_p), "seconds": plain_s,
                  "queries_per_s": sum(done_p) / plain_s, "finished_by_k": fin_k(done_p)},
        "learned": {"finished": sum(done_l), "seconds": plan_s + learned_s, "plan_s": plan_s,
                    "queries_per_s": sum(done_l) / (plan_s + learned_s), "orders_changed": switched,
                    "orders_changed_by_model_alone": model_switched,
                    "finished_by_k": fin_k(done_l)},
        "learned_batched": {"finished": sum(done_b), "seconds": lb_s, "plan_s": plan_s,
                            "launch_ms": ms, "launch_wall_s": batch_wall,
                            "queries_per_s": sum(done_b) / lb_s, "finished_by_k": fin_k(done_b)},
        "counts_agree_where_both_finished": agree,
        "estimated_full_counts": est_rep,
        "training": info,
    }


def stripe_estimates(g: "cb.Graph", qs, stride: int = 1 << 16, budget_ms: float = 20.0,
                     flags: int = 0):
    """Estimated work (sum of level sizes) of each query from one root stripe;
    inf when the stripe itself exceeds budget_ms."""
    est = []
    for q in qs:
        r, done = g.count_sample(q, 0, stride, budget_ms, flags)
        est.append(float(sum(r.level_sizes)) * stride if done else math.inf)
    return est


def run_batched(g: "cb.Graph", n: int = 4096, budget_ms: float = 60000.0, tune_sample: int = 256,
                flags: int = 0, query_budget_ms: float = 50.0):
    """4,096 queries in one persistent launch, cheapest estimated first, each
    limited to query_budget_ms of the whole GPU and the launch to budget_ms;
    shape autotuned on a sample."""
    from cuts_b200 import autotune
    qdefs = batched_queries(n)
    qs0 = [cb.Query.from_arcs(k, a) for k, a in qdefs]
    t_est = time.perf_counter()
    est = stripe_estimates(g, qs0, flags=flags)
    rank = sorted(range(n), key=lambda i: est[i])
    qs = [qs0[i] for i in rank]
    est_s = time.perf_counter() - t_est
    t0 = time.perf_counter()
    best, times = autotune.tune_batch(g, qs[:tune_sample], flags=flags, budget_ms=2000.0,
                                      query_budget_ms=query_budget_ms)
    tune_s = time.perf_counter() - t0
    b = g.batch(qs, flags=flags, grain=best[0], tasks_per_grab=best[1], blocks_per_sm=best[2])
    b.set_query_budget(query_budget_ms)
    _log(f"batched: estimates {est_s:.1f} s, tuned {best} in {tune_s:.1f} s")
    counts, status, ms = b.run(budget_ms)
    fin = sum(1 for s in status if s == 0)
    # the finished queries again, as a batch of their own (no unfinished
    # query holding the launch), and one at a time through the level engine
    # (count_budget, 10x the per-query share as a safety bound)
    fin_qs = [q for q, st in zip(qs, status) if st == 0]
    rerun = None
    if fin_qs:
        b2 = g.batch(fin_qs, flags=flags, grain=best[0], tasks_per_grab=best[1], blocks_per_sm=best[2])
        b2.run()  # capture
        c2, s2, ms2 = b2.run()
        assert c2 == [c for c, st in zip(counts, status) if st == 0]
        rerun = {"finished": sum(1 for x in s2 if x == 0), "ms": ms2,
                 "queries_per_s": len(fin_qs) / max(ms2 / 1e3, 1e-9)}
        b2.close()
    plain_ms, plain_done = 0.0, 0
    for q, c, st in zip(qs, counts, status):
        if st != 0:
            continue
        r, done = g.count_budget(q, 10 * query_budget_ms if query_budget_ms > 0 else 0.0, flags=flags)
        if done:
            assert r.count == c
            plain_ms += r.ms
            plain_done += 1
    return {"queries": n, "finished": fin, "launch_ms": ms, "queries_per_s": fin / (ms / 1e3),
            "finished_set_as_batch": rerun,
            "one_at_a_time": {"finished": plain_done, "ms": plain_ms,
                              "queries_per_s": plain_done / max(plain_ms / 1e3, 1e-9)},
            "query_budget_ms": query_budget_ms, "launch_budget_ms": budget_ms,
            "tuned": list(best), "tune_s": tune_s, "estimate_s": est_s, "tasks": b.info()[0],
            "matches_finished": int(sum(c for c, s in zip(counts, status) if s == 0)),
            "finished_by_k": {k: sum(1 for i, s in zip(rank, status) if s == 0 and qdefs[i][0] == k)
                              for k in range(3, 8)}}
