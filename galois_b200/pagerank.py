"""python/galois/_pagerank.pyx:157-175 on the B200 path.

``pagerank(numThreads, max_iterations, filename)``: the binding's variant of
pull-topological PageRank over the graph as stored -- rank starts at
INIT_RESIDUAL = 1-alpha, the base score is 1-alpha (not divided by n), nout is
the in-degree of the stored graph (computeOutDeg, :80-102) and iteration stops
when the MAX per-vertex change is <= TOLERANCE = 1e-3 (:120-139).  Runs on
GPU 0 through gb_pagerank_pull_ex.  Returns the rank array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import GB_ERR_NOT_CONVERGED, Stats, check, lib
from .device import DeviceGraph
from .graph import read_gr

ALPHA = 0.85
INIT_RESIDUAL = 1 - ALPHA
TOLERANCE = 1.0e-3
MAX_ITER = 1000


def pagerank(numThreads: int, max_iterations: int, filename: str) -> np.ndarray:  # noqa: N803
    print(f"Running Pagerank on : {filename}")
    print(f"Using {numThreads} thread(s).")
    g = read_gr(filename, 0)
    print(f"Number of Nodes: {g.n}, Number of Edges: {g.m}")
    rank = np.empty(g.n, dtype=np.float32)
    it = C.c_uint32(0)
    s = Stats()
    with DeviceGraph(g, symmetric=False) as dg:
        st = lib.gb_pagerank_pull_ex(dg.handle, ALPHA, TOLERANCE, max_iterations, INIT_RESIDUAL, 1 - ALPHA, 1,
                                     C.c_void_p(rank.ctypes.data), C.byref(it), C.byref(s), None)
    check(st, "gb_pagerank_pull_ex", allow=(GB_ERR_NOT_CONVERGED,))
    if it.value >= max_iterations:
        print(f"WARNING : failed to converge in {it.value} iterations")
    return rank
