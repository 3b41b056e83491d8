"""Named query graphs used by the workloads (undirected; both arcs per edge)."""
from typing import Dict, List, Tuple


def _sym(edges):
    arcs = []
    for a, b in edges:
        arcs.append((a, b))
        arcs.append((b, a))
    return arcs


def cycle(n: int) -> List[Tuple[int, int]]:
    return _sym([(i, (i + 1) % n) for i in range(n)])


# house: square 0-1-2-3 with roof vertex 4 on edge 0-1 (5 vertices, 6 edges)
HOUSE = _sym([(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4)])
# 4-clique 0..3 plus pendant vertex 4 on vertex 0 (5 vertices, 7 edges)
CLIQUE4_PENDANT = _sym([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (0, 4)])
# triangular prism: triangles 0-1-2 and 3-4-5 joined by 0-3, 1-4, 2-5 (6 vertices, 9 edges)
PRISM3 = _sym([(0, 1), (1, 2), (2, 0), (3, 4), (4, 5), (5, 3), (0, 3), (1, 4), (2, 5)])


def path(n: int) -> List[Tuple[int, int]]:
    return _sym([(i, i + 1) for i in range(n - 1)])


def star(leaves: int) -> List[Tuple[int, int]]:
    return _sym([(0, i) for i in range(1, leaves + 1)])


NAMED_QUERIES: Dict[str, Tuple[int, List[Tuple[int, int]]]] = {
    "triangle": (3, cycle(3)),
    "4-cycle": (4, cycle(4)),
    "5-cycle": (5, cycle(5)),
    "6-cycle": (6, cycle(6)),
    "house": (5, HOUSE),
    "4-clique+pendant": (5, CLIQUE4_PENDANT),
    "3-prism": (6, PRISM3),
    # trees: the queries with matches on graphs of mean degree below 2
    "3-path": (3, path(3)),
    "4-path": (4, path(4)),
    "5-path": (5, path(5)),
    "3-star": (4, star(3)),
}


def named_query_arcs(name: str) -> Tuple[int, List[Tuple[int, int]]]:
    return NAMED_QUERIES[name]
