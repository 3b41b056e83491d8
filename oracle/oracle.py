"""ctypes binding of the CPU oracle (oracle/cuts_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, always as the checker or the
CPU baseline, never by the cuts_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcuts_oracle.so")
REF_ORDER = os.path.join(HERE, "_ref", "ref_order")
REF_CUTS = os.path.join(HERE, "_ref", "cuts_ref")
MAX_QUERY = 32


class OrGraph(C.Structure):
    _fields_ = [("n", C.c_uint32), ("arcs", C.c_uint64),
                ("out_off", C.POINTER(C.c_uint64)), ("out_adj", C.POINTER(C.c_uint32)),
                ("in_off", C.POINTER(C.c_uint64)), ("in_adj", C.POINTER(C.c_uint32))]


_lib = None
_CB = C.CFUNCTYPE(None, C.POINTER(C.c_uint32), C.c_uint32, C.c_void_p)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        gp = C.POINTER(OrGraph)
        u32p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
        L.or_load_graph.argtypes = [C.c_char_p, gp]
        L.or_graph_from_arcs.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, gp]
        L.or_free_graph.argtypes = [gp]
        L.or_free_graph.restype = None
        L.or_is_symmetric.argtypes = [gp]
        L.or_order.argtypes = [gp, u32p, u32p, u32p, u32p, u32p]
        L.or_joins_for_order.argtypes = [gp, u32p, u32p, u32p, u32p, u32p]
        L.or_count.argtypes = [gp, gp, u32p, C.c_uint32, C.c_uint32, C.c_int, u64p, u64p, u64p]
        L.or_enumerate.argtypes = [gp, gp, u32p, _CB, C.c_void_p]
        L.or_count_striped.argtypes = [gp, gp, u32p, C.c_uint32, C.c_uint32, C.c_int, u64p, u64p]
        L.or_count_ex.argtypes = [gp, gp, u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.c_int, u64p, u64p]
        L.or_gen_chung_lu.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                      C.c_uint64, gp]
        L.or_relabel_by_degree.argtypes = [gp, gp, u32p]
        _lib = L
    return _lib


class Graph:
    """Oracle-side graph (its own loader and CSR)."""

    def __init__(self):
        self.g = OrGraph()

    @classmethod
    def load(cls, path: str) -> "Graph":
        o = cls()
        rc = lib().or_load_graph(path.encode(), C.byref(o.g))
        if rc:
            raise ValueError(f"oracle load failed ({rc}): {path}")
        return o

    @classmethod
    def from_arcs(cls, n: int, arcs: Sequence[Tuple[int, int]]) -> "Graph":
        src = np.array([a for a, _ in arcs] or [0], np.uint32)
        dst = np.array([b for _, b in arcs] or [0], np.uint32)
        return cls.from_arrays(n, src[:len(arcs)], dst[:len(arcs)])

    @classmethod
    def from_arrays(cls, n: int, src: np.ndarray, dst: np.ndarray) -> "Graph":
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        o = cls()
        u32p = C.POINTER(C.c_uint32)
        rc = lib().or_graph_from_arcs(n, len(src), src.ctypes.data_as(u32p),
                                      dst.ctypes.data_as(u32p), C.byref(o.g))
        if rc:
            raise ValueError(f"oracle graph build failed ({rc})")
        return o

    @classmethod
    def from_csr(cls, n: int, off: np.ndarray, adj: np.ndarray) -> "Graph":
        """Graph with arcs u -> adj[off[u]:off[u+1]]."""
        deg = np.diff(off.astype(np.int64))
        src = np.repeat(np.arange(n, dtype=np.uint32), deg)
        return cls.from_arrays(n, src, adj)

    @classmethod
    def chung_lu(cls, n: int, m: int, gamma: float, wmin: float, cap: float, seed: int) -> "Graph":
        """The seeded Chung-Lu graph of the engine's generator, built here."""
        o = cls()
        rc = lib().or_gen_chung_lu(n, m, gamma, wmin, cap, seed, C.byref(o.g))
        if rc:
            raise ValueError(f"oracle generator failed ({rc})")
        return o

    def relabel_by_degree(self) -> "Tuple[Graph, np.ndarray]":
        """(the graph with ids renamed to their (degree, id) rank, orig[rank])."""
        o = Graph()
        orig = np.zeros(max(self.n, 1), np.uint32)
        rc = lib().or_relabel_by_degree(C.byref(self.g), C.byref(o.g),
                                        orig.ctypes.data_as(C.POINTER(C.c_uint32)))
        if rc:
            raise ValueError(f"oracle relabel failed ({rc})")
        return o, orig[:self.n]

    @property
    def n(self) -> int:
        return self.g.n

    @property
    def arcs(self) -> int:
        return self.g.arcs

    def csr(self):
        n, a = self.g.n, self.g.arcs
        oo = np.ctypeslib.as_array(self.g.out_off, (n + 1,)).copy()
        oa = np.ctypeslib.as_array(self.g.out_adj, (max(a, 1),))[:a].copy()
        io = np.ctypeslib.as_array(self.g.in_off, (n + 1,)).copy()
        ia = np.ctypeslib.as_array(self.g.in_adj, (max(a, 1),))[:a].copy()
        return oo, oa, io, ia

    def symmetric(self) -> bool:
        return bool(lib().or_is_symmetric(C.byref(self.g)))

    def __del__(self):
        try:
            lib().or_free_graph(C.byref(self.g))
        except Exception:
            pass


def order(q: Graph):
    """Score order and P/C lists of graph.cpp:62-134."""
    k = q.n
    u32 = lambda m: (C.c_uint32 * m)()
    o, po, p, co, c = u32(k), u32(k + 1), u32(k * k + 1), u32(k + 1), u32(k * k + 1)
    rc = lib().or_order(C.byref(q.g), o, po, p, co, c)
    if rc:
        raise ValueError(f"oracle order failed ({rc})")
    P = [list(p[po[i]:po[i + 1]]) for i in range(k)]
    Cl = [list(c[co[i]:co[i + 1]]) for i in range(k)]
    return list(o), P, Cl


def count(d: Graph, q: Graph, order_: Optional[Sequence[int]] = None, root_begin: int = 0,
          root_end: int = 0xFFFFFFFF, nthreads: int = 0):
    """(count, level_sizes, alg_bytes) with the reference semantics."""
    k = q.n
    cnt = C.c_uint64()
    lv = (C.c_uint64 * k)()
    by = C.c_uint64()
    op = None
    if order_ is not None:
        op = (C.c_uint32 * k)(*order_)
    rc = lib().or_count(C.byref(d.g), C.byref(q.g), op, root_begin, root_end, nthreads,
                        C.byref(cnt), lv, C.byref(by))
    if rc:
        raise ValueError(f"oracle count failed ({rc})")
    return cnt.value, list(lv), by.value


def count_striped(d: Graph, q: Graph, shard: int, nshards: int, order_: Optional[Sequence[int]] = None,
                  nthreads: int = 0):
    """(count, level_sizes) over the roots u with u % nshards == shard."""
    k = q.n
    cnt = C.c_uint64()
    lv = (C.c_uint64 * k)()
    op = (C.c_uint32 * k)(*order_) if order_ is not None else None
    rc = lib().or_count_striped(C.byref(d.g), C.byref(q.g), op, shard, nshards, nthreads,
                                C.byref(cnt), lv)
    if rc:
        raise ValueError(f"oracle striped count failed ({rc})")
    return cnt.value, list(lv)


OPT_CLOSED_LAST = 1


def count_ex(d: Graph, q: Graph, order_: Optional[Sequence[int]] = None,
             conds: Sequence[Tuple[int, int]] = (), shard: int = 0, nshards: int = 1,
             opts: int = 0, nthreads: int = 0):
    """(count, level_sizes) over the roots u % nshards == shard, with
    ordering conditions conds = [(a, b)]: the vertex matched at position a is
    below the one at position b."""
    k = q.n
    cnt = C.c_uint64()
    lv = (C.c_uint64 * k)()
    op = (C.c_uint32 * k)(*order_) if order_ is not None else None
    flat = [x for ab in conds for x in ab]
    cp = (C.c_uint32 * max(len(flat), 1))(*flat)
    rc = lib().or_count_ex(C.byref(d.g), C.byref(q.g), op, cp, len(conds), shard, nshards, opts,
                           nthreads, C.byref(cnt), lv)
    if rc:
        raise ValueError(f"oracle count_ex failed ({rc})")
    return cnt.value, list(lv)


def enumerate_matches(d: Graph, q: Graph, order_: Optional[Sequence[int]] = None) -> List[tuple]:
    """Every embedding as a tuple indexed by query vertex."""
    out = []

    def cb(m, k, _u):
        out.append(tuple(m[i] for i in range(k)))

    f = _CB(cb)
    op = None
    if order_ is not None:
        op = (C.c_uint32 * q.n)(*order_)
    rc = lib().or_enumerate(C.byref(d.g), C.byref(q.g), op, f, None)
    if rc:
        raise ValueError(f"oracle enumerate failed ({rc})")
    return out
