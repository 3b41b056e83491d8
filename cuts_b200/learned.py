"""Learned matching order: training data, training and evaluation.

The cost model predicts log(1 + |L_i|), the size of trie level i, from the
per-step features of an order (query-vertex degree, back-edge count to the
matched set, data-graph degree tails, the signature survival rate and the
parent level's size).  Training data are the per-level table sizes the
plain engine reports for the score order and for random connected orders of
seeded training queries; on large graphs each run covers a root stripe
(u % stride == 0) and its level sizes are scaled by the stride, which is
an unbiased estimate because the stripes partition every level.

The model is trained by the engine's own FP32 kernels (cuts_mlp_train) and
used by cuts_plan(..., CUTS_ORDER_LEARNED, ...), which keeps the score order
whenever the model does not promise enough saving.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

import cuts_b200 as cb


def random_order(k: int, arcs: Sequence[Tuple[int, int]], rng: np.random.Generator) -> List[int]:
    """A uniformly drawn connected-prefix order."""
    nb = [set() for _ in range(k)]
    for a, b in arcs:
        if a != b:
            nb[a].add(b)
            nb[b].add(a)
    order = [int(rng.integers(k))]
    used = {order[0]}
    while len(order) < k:
        front = sorted({w for u in order for w in nb[u]} - used)
        v = int(rng.choice(front))
        order.append(v)
        used.add(v)
    return order


@dataclass
class Sample:
    query: int
    order: List[int]
    levels: List[int]      # estimated |L_i|
    ms: float
    score: bool


def level_sizes(g: "cb.Graph", q: "cb.Query", stride: int, budget_ms: float = 0.0):
    """Per-level sizes of q's current order, from the root stripe 0 of `stride`
    (scaled by the stride); None when the run exceeds budget_ms."""
    if stride <= 1 and budget_ms <= 0:
        r = g.count(q, stats=True)
        return r.level_sizes, r.ms
    r, done = g.count_sample(q, 0, max(stride, 1), budget_ms)
    if not done:
        return None, budget_ms
    return [x * max(stride, 1) for x in r.level_sizes], r.ms


def prefix_level_sizes(g: "cb.Graph", q: "cb.Query", stride: int, budget_ms: float):
    """The sizes of q's first levels under its current order: the prefix
    queries of 2, 3, ... positions (q's signatures kept) are counted on the
    root stripe until one exceeds budget_ms; returns the longest complete
    list (at least |L_0|) and the time spent."""
    best, spent = None, 0.0
    for j in range(2, q.k + 1):
        lv, ms = level_sizes(g, q.prefix(j), stride, budget_ms)
        spent += ms
        if lv is None:
            break
        best = lv
    return best, spent


def collect(g: "cb.Graph", queries: Sequence[Tuple[int, list]], orders_per_query: int = 4,
            stride: int = 1, seed: int = 0, time_budget_s: float = 1e9,
            run_budget_ms: float = 0.0, prefixes: bool = False) -> List[Sample]:
    """Per-level sizes of the score order and random orders of each query.
    With `prefixes`, a run that does not fit run_budget_ms still yields the
    sizes of the levels its prefixes reach (Sample.levels is then shorter
    than k)."""
    rng = np.random.default_rng(seed)
    out: List[Sample] = []
    t0 = time.time()
    for qi, (k, arcs) in enumerate(queries):
        if time.time() - t0 > time_budget_s:
            break
        q = cb.Query.from_arcs(k, arcs)
        score = q.order
        orders = [score] + [random_order(k, arcs, rng) for _ in range(orders_per_query - 1)]
        for j, o in enumerate(orders):
            q.set_order(o)
            if prefixes:
                lv, ms = prefix_level_sizes(g, q, stride, run_budget_ms)
            else:
                lv, ms = level_sizes(g, q, stride, run_budget_ms)
            if lv is None:  # too expensive to log within the run budget
                continue
            out.append(Sample(qi, list(o), lv, ms, j == 0))
    return out


def features(g: "cb.Graph", queries, samples: Sequence[Sample]):
    """Teacher-forced rows: X (sum_k x FEATURES), y = log(1 + |L_i|), query id per row."""
    X, y, qid = [], [], []
    cache = {}
    for s in samples:
        if s.query not in cache:
            k, arcs = queries[s.query]
            cache[s.query] = cb.Query.from_arcs(k, arcs)
        q = cache[s.query]
        n = len(s.levels)  # a prefix run logs the first n levels only
        lv = list(s.levels) + [0] * (q.k - n)
        F = q.features(g, s.order, lv)[:n]
        X.append(F)
        y.append(np.log1p(np.array(s.levels, np.float64)).astype(np.float32))
        qid += [s.query] * n
    return np.concatenate(X), np.concatenate(y), np.array(qid)


def train(X: np.ndarray, y: np.ndarray, epochs: int = 400, batch: int = 4096, lr: float = 2e-3,
          seed: int = 0, device: int = 0) -> "cb.Mlp":
    m = cb.Mlp(X.shape[1], seed=seed, device=device)
    m.train(X, y, epochs=epochs, batch=batch, lr=lr)
    return m


def prediction_error(m: "cb.Mlp", X: np.ndarray, y: np.ndarray) -> float:
    """Mean absolute error in log space (nats), teacher-forced."""
    return float(np.mean(np.abs(m.predict(X) - y)))


CLOSED_FORM_COST = 0.1  # per parent, a closed-form last level (as the order search)


def work(levels: Sequence[int], k: int, joins: Sequence[int]) -> float:
    """Measured work of an order: sum over levels of |L_i| x the next level's
    per-parent cost (1 + its joined lists; CLOSED_FORM_COST for a last level
    with one joined list, which the engine counts by list arithmetic)."""
    def cost(i):
        if i + 2 == k and joins[i + 1] == 1:
            return CLOSED_FORM_COST
        return 1 + joins[i + 1]
    return float(sum(levels[i] * cost(i) for i in range(k - 1)))


def joins_of(q: "cb.Query") -> List[int]:
    P, C = q.joins()
    return [len(set(P[i]) | set(C[i])) for i in range(q.k)]


def choose_order(g: "cb.Graph", q: "cb.Query", model: "cb.Mlp", proposals: int = 3, beam: int = 256,
                 stride: int = 1 << 16, budget_ms: float = 50.0, flags: int = 0):
    """Learned proposals, measured choice: the model's `proposals` best orders
    and the score order are each timed on the same root stripe
    (u % stride == 0, under budget_ms); the fastest is set on q.  The score
    order wins ties and stays when no proposal finishes its stripe faster.
    Returns (order, {order tuple: stripe ms or None})."""
    score = list(q.order)
    cands = [score] + [o for o, _ in q.candidates(g, model, proposals, beam) if o != score]
    times = {}
    best, best_ms = score, None
    for o in cands:
        q.set_order(o)
        r, done = g.count_sample(q, 0, stride, budget_ms, flags)
        times[tuple(o)] = r.ms if done else None
        if done and (best_ms is None or r.ms < best_ms * (0.9 if o != score else 1.0)):
            best, best_ms = o, r.ms
    q.set_order(best)
    return best, times
