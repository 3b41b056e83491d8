"""Shared test helpers: build the same seeded input for the engine and the oracle."""
import numpy as np

import cuts_b200 as cb
from oracle import oracle as O


def oracle_graph_from_host(h: "cb.HostGraph") -> "O.Graph":
    oo, oa, io, ia = h.csr()
    n = h.n
    return O.Graph.from_csr(n, oo, oa)


def directed_er(n: int, mean_deg: float, seed: int, keep: float = 0.6):
    """Directed graph: each arc of a seeded ER graph kept with probability keep."""
    h = cb.HostGraph.erdos_renyi(n, mean_deg / max(n - 1, 1), seed)
    oo, oa, _, _ = h.csr()
    rng = np.random.default_rng(seed + 1000)
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(oo.astype(np.int64)))
    m = rng.random(len(oa)) < keep
    return n, src[m], oa[m]


def csr_from_arcs(n: int, src: np.ndarray, dst: np.ndarray):
    """Sorted duplicate-free out- and in-CSR of an arc list."""
    key = src.astype(np.uint64) << np.uint64(32) | dst.astype(np.uint64)
    key = np.unique(key)
    s = (key >> np.uint64(32)).astype(np.uint32)
    d = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    out_off = np.zeros(n + 1, np.uint64)
    np.add.at(out_off, s.astype(np.int64) + 1, 1)
    out_off = np.cumsum(out_off).astype(np.uint64)
    key2 = np.unique(d.astype(np.uint64) << np.uint64(32) | s.astype(np.uint64))
    s2 = (key2 >> np.uint64(32)).astype(np.uint32)
    d2 = (key2 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    in_off = np.zeros(n + 1, np.uint64)
    np.add.at(in_off, s2.astype(np.int64) + 1, 1)
    in_off = np.cumsum(in_off).astype(np.uint64)
    return out_off, d, in_off, d2, s, d
