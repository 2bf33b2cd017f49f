"""python/galois/_sssp.pyx:154-174 on the B200 path.

``sssp(numThreads, shift, source, filename)`` reads a .gr file with uint32 edge
data, runs delta-stepping with bucket index dist >> shift from ``source`` and
prints the binding's report.  Unreached vertices hold ``numNodes`` as in the
binding's Initialize (_sssp.pyx:33-44).  Returns the distance array.
"""
from __future__ import annotations

import numpy as np

from ._lib import GB_DIST_INFINITY
from .device import DeviceGraph
from .graph import read_gr


def sssp(numThreads: int, shift: int, source: int, filename: str) -> np.ndarray:  # noqa: N803
    print(f"Using {numThreads} thread(s).")
    g = read_gr(filename, 4)
    print(f"Number of Nodes: {g.n}, Number of Edges: {g.m}")
    print(f"Using Source Node: {source}")
    if source >= g.n:
        raise ValueError(f"source {source} >= numNodes {g.n}")
    with DeviceGraph(g, symmetric=False) as dg:
        dist = dg.sssp(source, shift)
    dist = dist.astype(np.uint32)
    dist[dist == GB_DIST_INFINITY] = g.n
    if g.n > 1:
        print(f"Node 1 has dist : {int(dist[1])}")
    return dist
