"""Autotuners for the engine's work sizes.

tune_batch: the batched engine's launch shape -- (grain: level-1 candidates
per task, i.e. the work-stealing grain; tasks per work-counter grab; blocks
per SM) on a sample of the batch, replaying each candidate's captured CUDA
graph a few times.

tune_count: the level engine's chunk and tile sizes for one query -- the
number of root slices (the reference's trunks), the level capacity that
cuts the stored levels into memory chunks, and the fused count's tile (the
candidate-set size above which a parent is split over all warps).

Both keep the fastest configuration whose counts agree with the first one
tried (a count never depends on these sizes; disagreement would be a bug and
raises).  Results can be stored per GPU model and graph in a small JSON file.
"""
from __future__ import annotations

import json
import os
import statistics
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import cuts_b200 as cb

GRAINS = (16, 32, 64, 128, 256)
CHUNKS = (1, 2, 4, 8)
SPLITS = (64, 128, 256)
LEVEL_CAPS = (0,)
GRABS = (1, 4)
BLOCKS = (0, 4)


def tune_batch(g: "cb.Graph", queries: Sequence["cb.Query"], flags: int = 0,
               grains: Iterable[int] = GRAINS, grabs: Iterable[int] = GRABS,
               blocks: Iterable[int] = BLOCKS, reps: int = 3, budget_ms: float = 0.0,
               query_budget_ms: float = 0.0):
    """Returns (best (grain, grab, blocks), {config: median ms})."""
    times: Dict[Tuple[int, int, int], float] = {}
    ref: Optional[List[int]] = None
    if budget_ms > 0 or query_budget_ms > 0:
        # tune on the queries that finish within the budgets in the default shape
        b = g.batch(queries, flags=flags)
        b.set_query_budget(query_budget_ms)
        _, status, _ = b.run(budget_ms)
        b.close()
        queries = [q for q, s in zip(queries, status) if s == 0]
        budget_ms = 0.0
        if not queries:
            return (64, 1, 0), times
    for gr in grains:
        for tg in grabs:
            for bl in blocks:
                b = g.batch(queries, flags=flags, grain=gr, tasks_per_grab=tg, blocks_per_sm=bl)
                ms = []
                for _ in range(reps):
                    counts, status, t = b.run(budget_ms)
                    if any(s != 0 for s in status):
                        break
                    if ref is None:
                        ref = counts
                    elif counts != ref:
                        raise RuntimeError(f"batch counts depend on the launch shape {gr, tg, bl}")
                    ms.append(t)
                b.close()
                if len(ms) == reps:
                    times[(gr, tg, bl)] = statistics.median(ms)
    if not times:
        return (64, 1, 0), times
    best = min(times, key=times.get)
    return best, times


def tune_count(g: "cb.Graph", q: "cb.Query", flags: int = 0, chunks: Iterable[int] = CHUNKS,
               splits: Iterable[int] = SPLITS, level_caps: Iterable[int] = LEVEL_CAPS, reps: int = 3,
               apply: bool = True):
    """Returns (best (chunks, split, level cap), {config: median device ms}).
    With apply, the graph keeps the best split and level cap afterwards
    (chunks is an argument of each count); otherwise both return to their
    defaults."""
    times: Dict[Tuple[int, int, int], float] = {}
    ref: Optional[int] = None
    try:
        for ch in chunks:
            for sp in splits:
                for cap in level_caps:
                    g.set_fuse_split(sp)
                    g.set_level_cap(cap)
                    ms = []
                    for _ in range(reps):
                        r = g.count(q, chunks=ch, flags=flags)
                        if ref is None:
                            ref = r.count
                        elif r.count != ref:
                            raise RuntimeError(f"count depends on the work sizes {ch, sp, cap}")
                        ms.append(r.ms)
                    times[(ch, sp, cap)] = statistics.median(ms)
    finally:
        g.set_fuse_split(0)
        g.set_level_cap(0)
    best = min(times, key=times.get)
    if apply:
        g.set_fuse_split(best[1])
        g.set_level_cap(best[2])
    return best, times


def gpu_key(g: "cb.Graph") -> str:
    n, arcs, sym, maxd = g.info()
    try:
        import torch
        name = torch.cuda.get_device_name(0)
    except Exception:
        name = "gpu"
    return f"{name}|n={n}|arcs={arcs}|maxd={maxd}"


def load(path: str, key: str) -> Optional[Tuple[int, int, int]]:
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    v = d.get(key)
    return tuple(v) if v else None


def store(path: str, key: str, cfg: Tuple[int, int, int]) -> None:
    d = {}
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
    d[key] = list(cfg)
    with open(path, "w") as f:
        json.dump(d, f, indent=1)
