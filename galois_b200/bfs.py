"""python/galois/_bfs.pyx:171-191 on the B200 path.

``bfs(numThreads, source, filename)`` reads the .gr file, runs BFS from
``source`` on GPU 0 and prints the same report lines as the Cython binding.
Like the binding (``Initialize``, _bfs.pyx:29-42), unreached vertices hold
``numNodes``.  numThreads is accepted for signature compatibility (the work
runs on the GPU).  Returns the level array (the binding returns None).
"""
from __future__ import annotations

import numpy as np

from ._lib import GB_DIST_INFINITY
from .device import DeviceGraph
from .graph import read_gr


def bfs(numThreads: int, source: int, filename: str) -> np.ndarray:  # noqa: N803 (reference names)
    print(f"Using {numThreads} thread(s).")
    g = read_gr(filename, 0)
    print(f"Number of Nodes: {g.n}, Number of Edges: {g.m}")
    print(f"Using Source Node: {source}")
    if source >= g.n:
        raise ValueError(f"source {source} >= numNodes {g.n}")
    with DeviceGraph(g, symmetric=False) as dg:
        level = dg.bfs(source)
    level = level.astype(np.uint32)
    level[level == GB_DIST_INFINITY] = g.n  # binding's infinity (_bfs.pyx:42)
    not_visited = int((level >= g.n).sum())
    if level[source] != 0:
        print(f"ERROR: source has non-zero dist value == {level[source]}")
    if not_visited:
        print(f"{not_visited} unvisited nodes; this is an error if graph is strongly connected")
    reached = level[level < g.n]
    print(f"Max distance : {int(reached.max()) if reached.size else 0}")
    if g.n > 1:
        print(f"Node 1 has dist : {int(level[1])}")
    return level
