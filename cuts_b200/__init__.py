"""cuts_b200 -- B200 subgraph-isomorphism counting engine (Python host mirror).

The engine is C++ host code and hand-written sm_100a CUDA kernels behind the
C ABI in ``include/cuts_b200.h`` (``cuts_b200/lib/libcuts_b200.so``).  This
module binds that ABI with ctypes and mirrors the reference's in-process API:

* ``search(query_file, data_file, write_to_disk)``           -- host_funcs.cu:115
* ``search_dfs_bfs_strategy(query_file, data_file, write_to_disk, trunks)``
                                                              -- host_funcs.cu:39

Both print the reference's progress lines and its result line
``<data>,<query>,<ms>ms,<count>`` and return the count.  There is no CPU
fallback: without the built library every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcuts_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "cuts")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "cuts_b200.h")

OK = 0
ERR_ARG, ERR_IO, ERR_PARSE, ERR_CUDA, ERR_NOMEM, ERR_QUERY, ERR_CAPACITY, ERR_LIMIT, ERR_BUDGET = \
    range(1, 10)
MAX_QUERY = 16
FLAG_SYMMETRY_BREAK = 1
FLAG_NO_CLOSED_FORM = 2
FLAG_NO_FUSE = 4
FLAG_NO_ORBIT_FOLD = 8
FLAG_NO_PAIR_FOLD = 16
ORDER_SCORE = 0
ORDER_LEARNED = 1


class CutsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cuts error {code}: {msg}")
        self.code = code


_lib: Optional[C.CDLL] = None

_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p
FEATURES = 16

_SIGS = {
    "cuts_last_error": (C.c_char_p, []),
    "cuts_version": (C.c_char_p, []),
    "cuts_hgraph_load": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "cuts_hgraph_gen_er": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, C.POINTER(_vp)]),
    "cuts_hgraph_gen_chung_lu": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_double,
                                           C.c_double, C.c_uint64, C.POINTER(_vp)]),
    "cuts_hgraph_info": (C.c_int, [_vp, _u32p, _u64p, C.POINTER(C.c_int), _u32p]),
    "cuts_hgraph_csr": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cuts_hgraph_write": (C.c_int, [_vp, C.c_char_p]),
    "cuts_graph_upload": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "cuts_hgraph_save_binary": (C.c_int, [_vp, C.c_char_p]),
    "cuts_hgraph_load_binary": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "cuts_hgraph_free": (None, [_vp]),
    "cuts_gen_random_query": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, _u32p, _u32p, _u32p]),
    "cuts_graph_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    "cuts_graph_from_csr": (C.c_int, [C.c_uint32, _vp, _vp, _vp, _vp, C.c_int, C.POINTER(_vp)]),
    "cuts_graph_info": (C.c_int, [_vp, _u32p, _u64p, C.POINTER(C.c_int), _u32p]),
    "cuts_graph_set_level_cap": (C.c_int, [_vp, C.c_uint64]),
    "cuts_graph_set_fuse_split": (C.c_int, [_vp, C.c_uint32]),
    "cuts_graph_set_arena_bytes": (C.c_int, [_vp, C.c_uint64]),
    "cuts_graph_free": (None, [_vp]),
    "cuts_query_load": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "cuts_query_from_arcs": (C.c_int, [C.c_uint32, C.c_uint32, _u32p, _u32p, C.POINTER(_vp)]),
    "cuts_query_info": (C.c_int, [_vp, _u32p, _u32p]),
    "cuts_query_joins": (C.c_int, [_vp, _u32p, _u32p, _u32p, _u32p]),
    "cuts_query_set_order": (C.c_int, [_vp, _u32p]),
    "cuts_query_automorphisms": (C.c_int, [_vp, _u64p]),
    "cuts_query_plan_levels": (C.c_int, [_vp, C.c_int, C.c_uint32, _u32p, _u64p]),
    "cuts_query_prefix": (C.c_int, [_vp, C.c_uint32, C.POINTER(_vp)]),
    "cuts_query_free": (None, [_vp]),
    "cuts_count": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, _u64p, C.POINTER(C.c_float)]),
    "cuts_count_ex": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, _u64p, C.POINTER(C.c_float),
                                _u64p, _u64p]),
    "cuts_count_sharded": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                     _u64p, C.POINTER(C.c_float), _u64p]),
    "cuts_count_sharded_ex": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                        _u64p, _fp, _u64p, _u64p]),
    "cuts_dump_sharded": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_char_p, _u64p]),
    "cuts_dump": (C.c_int, [_vp, _vp, C.c_char_p, _u64p]),
    "cuts_search": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_uint32, _u64p,
                              C.POINTER(C.c_float)]),
    "cuts_count_batch": (C.c_int, [_vp, C.POINTER(_vp), C.c_uint32, C.c_uint32, _u64p,
                                   C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "cuts_count_budget": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_double, _u64p,
                                    C.POINTER(C.c_float), _u64p]),
    "cuts_count_sample": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                    _u64p, C.POINTER(C.c_float), _u64p]),
    "cuts_batch_create": (C.c_int, [_vp, C.POINTER(_vp), C.c_uint32, C.c_uint32, _u32p,
                                    C.POINTER(_vp)]),
    "cuts_batch_run": (C.c_int, [_vp, C.c_double, _u64p, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "cuts_batch_info": (C.c_int, [_vp, _u64p, _u32p]),
    "cuts_batch_set_query_budget": (C.c_int, [_vp, C.c_double]),
    "cuts_batch_set_shard": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "cuts_plan_candidates": (C.c_int, [_vp, _vp, _vp, C.c_uint32, C.c_uint32, _u32p,
                                       C.POINTER(C.c_double), _u32p]),
    "cuts_batch_free": (None, [_vp]),
    "cuts_count_noalloc": (C.c_int, [_vp, _vp, _vp, C.c_uint32, C.POINTER(_vp), C.c_uint32,
                                     C.c_uint32, _vp, _vp]),
    "cuts_mlp_create": (C.c_int, [C.c_uint32, C.c_uint64, C.c_int, C.POINTER(_vp)]),
    "cuts_mlp_param_count": (C.c_int, [_vp, _u32p]),
    "cuts_mlp_get_params": (C.c_int, [_vp, _fp]),
    "cuts_mlp_set_params": (C.c_int, [_vp, _fp]),
    "cuts_mlp_loss_grad": (C.c_int, [_vp, _fp, _fp, C.c_uint32, _fp, _fp]),
    "cuts_mlp_train": (C.c_int, [_vp, _fp, _fp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, _fp]),
    "cuts_mlp_predict": (C.c_int, [_vp, _fp, C.c_uint32, _fp]),
    "cuts_mlp_free": (None, [_vp]),
    "cuts_query_features": (C.c_int, [_vp, _vp, _u32p, _u64p, _fp]),
    "cuts_plan": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_uint32, C.c_double, _u32p,
                            C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}


def lib() -> C.CDLL:
    """The loaded engine library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CutsError(ERR_IO, f"engine library missing: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != OK:
        raise CutsError(rc, lib().cuts_last_error().decode())


def _ptr(a: Optional[np.ndarray], t=_vp):
    if a is None:
        return None
    return a.ctypes.data_as(t) if t is not _vp else C.c_void_p(a.ctypes.data)


# --------------------------------------------------------------------------
# host graphs
# --------------------------------------------------------------------------

class HostGraph:
    """Data graph in host memory (CSR built by the engine's loader)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str) -> "HostGraph":
        h = _vp()
        _check(lib().cuts_hgraph_load(path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def erdos_renyi(cls, n: int, p: float, seed: int = 0) -> "HostGraph":
        h = _vp()
        _check(lib().cuts_hgraph_gen_er(n, p, seed, C.byref(h)))
        return cls(h)

    @classmethod
    def chung_lu(cls, n: int, m: int, gamma: float, wmin: float = 2.0, cap: float = 2e4,
                 seed: int = 0) -> "HostGraph":
        h = _vp()
        _check(lib().cuts_hgraph_gen_chung_lu(n, m, gamma, wmin, cap, seed, C.byref(h)))
        return cls(h)

    def info(self) -> Tuple[int, int, bool, int]:
        n, a, s, d = C.c_uint32(), C.c_uint64(), C.c_int(), C.c_uint32()
        _check(lib().cuts_hgraph_info(self._h, C.byref(n), C.byref(a), C.byref(s), C.byref(d)))
        return n.value, a.value, bool(s.value), d.value

    @property
    def n(self) -> int:
        return self.info()[0]

    def csr(self):
        """(out_off, out_adj, in_off, in_adj); in_* are None when symmetric."""
        n, arcs, sym, _ = self.info()
        oo = np.zeros(n + 1, np.uint64)
        oa = np.zeros(max(arcs, 1), np.uint32)
        io = None if sym else np.zeros(n + 1, np.uint64)
        ia = None if sym else np.zeros(max(arcs, 1), np.uint32)
        _check(lib().cuts_hgraph_csr(self._h, _ptr(oo), _ptr(oa), _ptr(io), _ptr(ia)))
        return oo, oa[:arcs], io, (ia[:arcs] if ia is not None else None)

    def write(self, path: str) -> None:
        _check(lib().cuts_hgraph_write(self._h, path.encode()))

    def save_binary(self, path: str) -> None:
        _check(lib().cuts_hgraph_save_binary(self._h, path.encode()))

    @classmethod
    def load_binary(cls, path: str) -> "HostGraph":
        h = _vp()
        _check(lib().cuts_hgraph_load_binary(path.encode(), C.byref(h)))
        return cls(h)

    def upload(self, device: int = 0) -> "Graph":
        g = _vp()
        _check(lib().cuts_graph_upload(self._h, device, C.byref(g)))
        return Graph(g)

    def close(self):
        if self._h:
            lib().cuts_hgraph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# queries
# --------------------------------------------------------------------------

class Query:
    """Query graph with its matching order (score.cpp order by default)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str) -> "Query":
        h = _vp()
        _check(lib().cuts_query_load(path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_arcs(cls, k: int, arcs: Sequence[Tuple[int, int]]) -> "Query":
        src = np.array([a for a, _ in arcs], np.uint32)
        dst = np.array([b for _, b in arcs], np.uint32)
        h = _vp()
        _check(lib().cuts_query_from_arcs(k, len(arcs), _ptr(src, _u32p), _ptr(dst, _u32p),
                                          C.byref(h)))
        return cls(h)

    @classmethod
    def from_edges(cls, k: int, edges: Sequence[Tuple[int, int]]) -> "Query":
        """Undirected edges: both arcs of each edge."""
        arcs = []
        for a, b in edges:
            arcs.append((a, b))
            arcs.append((b, a))
        return cls.from_arcs(k, arcs)

    @property
    def k(self) -> int:
        k = C.c_uint32()
        _check(lib().cuts_query_info(self._h, C.byref(k), None))
        return k.value

    @property
    def order(self) -> List[int]:
        k = self.k
        o = np.zeros(k, np.uint32)
        _check(lib().cuts_query_info(self._h, None, _ptr(o, _u32p)))
        return [int(x) for x in o]

    def set_order(self, order: Sequence[int]) -> None:
        o = np.array(order, np.uint32)
        _check(lib().cuts_query_set_order(self._h, _ptr(o, _u32p)))

    def joins(self):
        """P and C join lists per level position (graph.cpp:94-133)."""
        k = self.k
        po, co = np.zeros(k + 1, np.uint32), np.zeros(k + 1, np.uint32)
        p, c = np.zeros(k * k + 1, np.uint32), np.zeros(k * k + 1, np.uint32)
        _check(lib().cuts_query_joins(self._h, _ptr(po, _u32p), _ptr(p, _u32p), _ptr(co, _u32p),
                                      _ptr(c, _u32p)))
        P = [[int(x) for x in p[po[i]:po[i + 1]]] for i in range(k)]
        Cl = [[int(x) for x in c[co[i]:co[i + 1]]] for i in range(k)]
        return P, Cl

    def features(self, graph: "Graph", order: Sequence[int], level_sizes: Sequence[int]) -> np.ndarray:
        """k x FEATURES rows of `order`, parent-level feature from level_sizes."""
        k = self.k
        o = np.array(order, np.uint32)
        lv = np.array(level_sizes, np.uint64)
        out = np.zeros((k, FEATURES), np.float32)
        _check(lib().cuts_query_features(self._h, graph._h, _ptr(o, _u32p), _ptr(lv, _u64p),
                                         _ptr(out, _fp)))
        return out

    def plan(self, graph: "Graph", mode: int = ORDER_SCORE, model: "Mlp" = None, beam: int = 0,
             margin: float = 1.25):
        """Choose and set the order; returns (order, predicted work, score-order work)."""
        k = self.k
        o = np.zeros(k, np.uint32)
        pw, sw = C.c_double(), C.c_double()
        _check(lib().cuts_plan(self._h, graph._h, mode, model._h if model else None, beam, margin,
                               _ptr(o, _u32p), C.byref(pw), C.byref(sw)))
        return [int(x) for x in o], pw.value, sw.value

    def prefix(self, j: int) -> "Query":
        """The first j positions of the order as a query whose level sizes are
        this query's first j level sizes (signatures kept, plain counting)."""
        h = _vp()
        _check(lib().cuts_query_prefix(self._h, j, C.byref(h)))
        return Query(h)

    def candidates(self, graph: "Graph", model: "Mlp", count: int = 4, beam: int = 256):
        """The `count` orders with the least predicted work under `model`
        (least first) as [(order, predicted work)]; the query's order is kept."""
        k = self.k
        o = np.zeros(max(count, 1) * k, np.uint32)
        w = (C.c_double * max(count, 1))()
        n = C.c_uint32()
        _check(lib().cuts_plan_candidates(self._h, graph._h, model._h, beam, count, _ptr(o, _u32p), w,
                                          C.byref(n)))
        return [([int(x) for x in o[r * k:(r + 1) * k]], w[r]) for r in range(n.value)]

    def plan_levels(self, data_symmetric: bool = True, flags: int = 0):
        """Per-level plan dicts (joins, sig, closed, fold, guar, gt, lt, fuse,
        ofold, qin, qout) and the count multiplier used."""
        k = self.k
        out = np.zeros(12 * k, np.uint32)
        aut = C.c_uint64()
        _check(lib().cuts_query_plan_levels(self._h, int(data_symmetric), flags, _ptr(out, _u32p),
                                            C.byref(aut)))
        keys = ["joins", "sig", "closed", "fold", "guar", "gt", "lt", "fuse", "ofold", "qin", "qout",
                "fold2"]
        return [dict(zip(keys, (int(x) for x in out[12 * i:12 * i + 12]))) for i in range(k)], aut.value

    def automorphisms(self) -> int:
        a = C.c_uint64()
        _check(lib().cuts_query_automorphisms(self._h, C.byref(a)))
        return a.value

    def close(self):
        if self._h:
            lib().cuts_query_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# device graphs and counting
# --------------------------------------------------------------------------

@dataclass
class CountResult:
    count: int
    ms: float
    level_sizes: List[int] = field(default_factory=list)
    launches: int = 0
    chunks: int = 0
    last_level_bytes: int = 0
    last_level_ms: float = 0.0
    expand_ms: float = 0.0
    last_level_launches: int = 0
    expand_launches: int = 0


class Graph:
    """Data graph resident on one GPU."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Graph":
        h = _vp()
        _check(lib().cuts_graph_load(path.encode(), device, C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, n: int, out_off: np.ndarray, out_adj: np.ndarray,
                 in_off: Optional[np.ndarray] = None, in_adj: Optional[np.ndarray] = None,
                 device: int = 0) -> "Graph":
        out_off = np.ascontiguousarray(out_off, np.uint64)
        out_adj = np.ascontiguousarray(out_adj, np.uint32)
        if in_off is not None:
            in_off = np.ascontiguousarray(in_off, np.uint64)
            in_adj = np.ascontiguousarray(in_adj, np.uint32)
        h = _vp()
        _check(lib().cuts_graph_from_csr(n, _ptr(out_off), _ptr(out_adj), _ptr(in_off),
                                         _ptr(in_adj), device, C.byref(h)))
        return cls(h)

    def info(self) -> Tuple[int, int, bool, int]:
        n, a, s, d = C.c_uint32(), C.c_uint64(), C.c_int(), C.c_uint32()
        _check(lib().cuts_graph_info(self._h, C.byref(n), C.byref(a), C.byref(s), C.byref(d)))
        return n.value, a.value, bool(s.value), d.value

    def set_level_cap(self, entries: int) -> None:
        _check(lib().cuts_graph_set_level_cap(self._h, entries))

    def set_arena_bytes(self, nbytes: int) -> None:
        _check(lib().cuts_graph_set_arena_bytes(self._h, nbytes))

    def set_fuse_split(self, split: int) -> None:
        """|S| above which the fused count splits a parent over all warps (0 = default)."""
        _check(lib().cuts_graph_set_fuse_split(self._h, split))

    def count(self, q: Query, chunks: int = 1, flags: int = 0, stats: bool = False,
              alg_bytes: bool = False, profile: bool = False) -> CountResult:
        cnt, ms = C.c_uint64(), C.c_float()
        if not stats and not alg_bytes and not profile:
            _check(lib().cuts_count(self._h, q._h, chunks, flags, C.byref(cnt), C.byref(ms)))
            return CountResult(cnt.value, ms.value)
        k = q.k
        lv = np.zeros(k, np.uint64)
        st = np.zeros(8, np.uint64)
        st[2] = 1 if alg_bytes else 0
        st[3] = 1 if profile else 0
        _check(lib().cuts_count_ex(self._h, q._h, chunks, flags, C.byref(cnt), C.byref(ms),
                                   _ptr(lv, _u64p), _ptr(st, _u64p)))
        return CountResult(cnt.value, ms.value, [int(x) for x in lv], int(st[0]), int(st[1]),
                           int(st[2]), st[3] / 1e6, st[4] / 1e6, int(st[5]), int(st[6]))

    def count_sharded(self, q: Query, shard: int, nshards: int, chunks: int = 1,
                      flags: int = 0, alg_bytes: bool = False, profile: bool = False) -> CountResult:
        """The roots u with u % nshards == shard only (device ids)."""
        cnt, ms = C.c_uint64(), C.c_float()
        lv = np.zeros(q.k, np.uint64)
        st = np.zeros(8, np.uint64)
        st[2] = 1 if alg_bytes else 0
        st[3] = 1 if profile else 0
        _check(lib().cuts_count_sharded_ex(self._h, q._h, chunks, flags, shard, nshards,
                                           C.byref(cnt), C.byref(ms), _ptr(lv, _u64p), _ptr(st, _u64p)))
        return CountResult(cnt.value, ms.value, [int(x) for x in lv], int(st[0]), int(st[1]),
                           int(st[2]), st[3] / 1e6, st[4] / 1e6, int(st[5]), int(st[6]))

    def count_budget(self, q: Query, budget_ms: float, chunks: int = 1, flags: int = 0):
        """(CountResult, finished): stops once budget_ms has passed (the host
        checks between chunks; the kernels take no more work after budget_ms
        of device time)."""
        cnt, ms = C.c_uint64(), C.c_float()
        lv = np.zeros(q.k, np.uint64)
        rc = lib().cuts_count_budget(self._h, q._h, chunks, flags, budget_ms, C.byref(cnt),
                                     C.byref(ms), _ptr(lv, _u64p))
        if rc == ERR_BUDGET:
            return CountResult(0, budget_ms, [int(x) for x in lv]), False
        _check(rc)
        return CountResult(cnt.value, ms.value, [int(x) for x in lv]), True

    def count_sample(self, q: Query, shard: int, nshards: int, budget_ms: float = 0.0,
                     flags: int = 0):
        """(CountResult, finished) of the root stripe u % nshards == shard."""
        cnt, ms = C.c_uint64(), C.c_float()
        lv = np.zeros(q.k, np.uint64)
        rc = lib().cuts_count_sample(self._h, q._h, shard, nshards, flags, budget_ms, C.byref(cnt),
                                     C.byref(ms), _ptr(lv, _u64p))
        if rc == ERR_BUDGET:
            return CountResult(0, budget_ms, [int(x) for x in lv]), False
        _check(rc)
        return CountResult(cnt.value, ms.value, [int(x) for x in lv]), True

    def dump(self, q: Query, path: str, shard: int = 0, nshards: int = 1) -> int:
        """Write ans.txt lines (the matches whose root is in the stripe
        u % nshards == shard); returns the number of lines."""
        n = C.c_uint64()
        if nshards == 1:
            _check(lib().cuts_dump(self._h, q._h, path.encode(), C.byref(n)))
        else:
            _check(lib().cuts_dump_sharded(self._h, q._h, shard, nshards, path.encode(), C.byref(n)))
        return n.value

    def count_batch(self, queries: Sequence[Query], flags: int = 0):
        nq = len(queries)
        arr = (_vp * nq)(*[q._h for q in queries])
        counts = np.zeros(max(nq, 1), np.uint64)
        status = (C.c_int * max(nq, 1))()
        ms = C.c_float()
        _check(lib().cuts_count_batch(self._h, arr, nq, flags, _ptr(counts, _u64p), status,
                                      C.byref(ms)))
        return [int(x) for x in counts[:nq]], list(status)[:nq], ms.value

    def batch(self, queries: Sequence[Query], flags: int = 0, grain: int = 0,
              tasks_per_grab: int = 0, blocks_per_sm: int = 0) -> "Batch":
        return Batch(self, queries, flags, (grain, tasks_per_grab, blocks_per_sm))

    def close(self):
        if self._h:
            lib().cuts_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """FP32 MLP cost model (in -> 64 -> 64 -> 1) resident on one GPU."""

    def __init__(self, in_dim: int = FEATURES, seed: int = 0, device: int = 0):
        h = _vp()
        _check(lib().cuts_mlp_create(in_dim, seed, device, C.byref(h)))
        self._h = h
        self.in_dim = in_dim

    @property
    def n_params(self) -> int:
        n = C.c_uint32()
        _check(lib().cuts_mlp_param_count(self._h, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        _check(lib().cuts_mlp_get_params(self._h, _ptr(p, _fp)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        _check(lib().cuts_mlp_set_params(self._h, _ptr(p, _fp)))

    def loss_grad(self, X: np.ndarray, y: np.ndarray):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32)
        _check(lib().cuts_mlp_loss_grad(self._h, _ptr(X, _fp), _ptr(y, _fp), len(y), C.byref(loss),
                                        _ptr(g, _fp)))
        return loss.value, g

    def train(self, X: np.ndarray, y: np.ndarray, epochs: int, batch: int = 0,
              lr: float = 1e-3) -> float:
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float()
        _check(lib().cuts_mlp_train(self._h, _ptr(X, _fp), _ptr(y, _fp), len(y), epochs, batch, lr,
                                    C.byref(loss)))
        return loss.value

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(X.shape[0], np.float32)
        _check(lib().cuts_mlp_predict(self._h, _ptr(X, _fp), X.shape[0], _ptr(y, _fp)))
        return y

    def save(self, path: str) -> None:
        np.save(path, self.get_params())

    def load(self, path: str) -> None:
        self.set_params(np.load(path))

    def close(self):
        if self._h:
            lib().cuts_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many queries against one resident graph in one persistent launch,
    captured once in a CUDA graph and replayed by run()."""

    def __init__(self, graph: Graph, queries: Sequence[Query], flags: int = 0,
                 tune: Tuple[int, int, int] = (0, 0, 0)):
        self.graph = graph
        self.queries = list(queries)  # keep the handles alive
        nq = len(self.queries)
        arr = (_vp * max(nq, 1))(*[q._h for q in self.queries])
        t = np.array(tune, np.uint32)
        h = _vp()
        _check(lib().cuts_batch_create(graph._h, arr, nq, flags, _ptr(t, _u32p), C.byref(h)))
        self._h = h
        self.nq = nq

    def run(self, budget_ms: float = 0.0):
        """(counts, status, device ms); status ERR_BUDGET marks unfinished queries."""
        counts = np.zeros(max(self.nq, 1), np.uint64)
        status = (C.c_int * max(self.nq, 1))()
        ms = C.c_float()
        _check(lib().cuts_batch_run(self._h, budget_ms, _ptr(counts, _u64p), status, C.byref(ms)))
        return [int(x) for x in counts[:self.nq]], list(status)[:self.nq], ms.value

    def set_query_budget(self, ms: float) -> None:
        """Each query may use `ms` of the whole GPU in later runs; a query past
        it reports ERR_BUDGET while the others carry on (0 = no limit)."""
        _check(lib().cuts_batch_set_query_budget(self._h, ms))

    def set_shard(self, shard: int, nshards: int) -> None:
        """Later runs take the tasks t % nshards == shard only (one GPU's part)."""
        _check(lib().cuts_batch_set_shard(self._h, shard, nshards))

    def info(self):
        t, b = C.c_uint64(), C.c_uint32()
        _check(lib().cuts_batch_info(self._h, C.byref(t), C.byref(b)))
        return t.value, b.value

    def close(self):
        if self._h:
            lib().cuts_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def count_noalloc(info_out_ptr: int, info_in_ptr: Optional[int], adj_ptr: int, n: int,
                  queries: Sequence[Query], counts_ptr: int, flags: int = 0,
                  stream: Optional[int] = None) -> None:
    """cuts_count_noalloc: count with caller-owned device buffers only (device
    addresses as ints, e.g. tensor.data_ptr()).  Asynchronous on `stream`."""
    nq = len(queries)
    arr = (_vp * max(nq, 1))(*[q._h for q in queries])
    _check(lib().cuts_count_noalloc(info_out_ptr, info_in_ptr, adj_ptr, n, arr, nq, flags,
                                    counts_ptr, stream))


def search(query_file: str, data_file: str, write_to_disk: bool = False) -> int:
    """Reference ``search()`` (host_funcs.cu:115-171)."""
    cnt, ms = C.c_uint64(), C.c_float()
    _check(lib().cuts_search(query_file.encode(), data_file.encode(), int(write_to_disk), 0,
                             C.byref(cnt), C.byref(ms)))
    return cnt.value


def search_dfs_bfs_strategy(query_file: str, data_file: str, write_to_disk: bool,
                            trunks: int) -> int:
    """Reference ``search_dfs_bfs_strategy()`` (host_funcs.cu:39-114)."""
    if trunks <= 0:
        raise CutsError(ERR_ARG, "trunks must be >= 1")
    cnt, ms = C.c_uint64(), C.c_float()
    _check(lib().cuts_search(query_file.encode(), data_file.encode(), int(write_to_disk), trunks,
                             C.byref(cnt), C.byref(ms)))
    return cnt.value


def random_query_arcs(k: int, p: float, seed: int) -> List[Tuple[int, int]]:
    """Seeded random connected undirected query (both arcs per edge)."""
    src = np.zeros(k * k, np.uint32)
    dst = np.zeros(k * k, np.uint32)
    na = C.c_uint32()
    _check(lib().cuts_gen_random_query(k, p, seed, C.byref(na), _ptr(src, _u32p), _ptr(dst, _u32p)))
    return [(int(src[i]), int(dst[i])) for i in range(na.value)]


def write_query(path: str, k: int, arcs: Sequence[Tuple[int, int]]) -> None:
    """Write a query in the reference text format."""
    with open(path, "w") as f:
        f.write(f"{k}\n")
        for a, b in arcs:
            f.write(f"{a}\t{b}\n")


from .queries import NAMED_QUERIES, named_query_arcs  # noqa: E402
