"""python/galois/_connected_components.pyx:87-104 on the B200 path.

``connectedComponents(numThreads, filename)`` runs label propagation with
pointer jumping on GPU 0; labels converge to the minimum vertex id of each
component, exactly what the binding's labelProp (:62-84) converges to.
Returns the label array.
"""
from __future__ import annotations

import numpy as np

from ._lib import GB_CC_LABELPROP
from .device import DeviceGraph
from .graph import read_gr


def connectedComponents(numThreads: int, filename: str) -> np.ndarray:  # noqa: N802,N803
    print(f"Running Pagerank on : {filename}")  # the binding prints this banner (:93)
    print(f"Using {numThreads} thread(s).")
    g = read_gr(filename, 0)
    print(f"Number of Nodes: {g.n}, Number of Edges: {g.m}")
    with DeviceGraph(g, symmetric=False) as dg:
        labels = dg.cc(GB_CC_LABELPROP)
    return labels
