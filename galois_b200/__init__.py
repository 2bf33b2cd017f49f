"""galois_b200: B200-native CSR edge-map kernels behind Galois' interfaces.

Python surface:
  * galois_b200.bfs.bfs / sssp.sssp / pagerank.pagerank /
    connected_components.connectedComponents mirror python/galois
    (_bfs.pyx:171, _sssp.pyx:154, _pagerank.pyx:157,
    _connected_components.pyx:87) with the same arguments;
  * graph.HostCSR + generators + .gr I/O, device.DeviceGraph (gb_graph*);
  * ppr.PersonalizedPageRank, a torch.autograd.Function over the hand-written
    forward and adjoint kernels.
All compute goes through libgb.so (include/gb.h); importing this package
without the built library raises ImportError.
"""
from . import _lib  # noqa: F401  (loads libgb.so or fails loudly)
from ._lib import (GB_CC_AFFOREST, GB_CC_LABELPROP, GB_CC_UNIONFIND, GB_DIST_INFINITY, GB_ORDER_AUTO,
                   GB_ORDER_DEGREE, GB_ORDER_DEGREE_UNSORTED, GB_ORDER_LOCALITY, GB_ORDER_NONE, GbError)
from .device import DeviceGraph
from .graph import (HostCSR, assign_weights_f32, assign_weights_reference, assign_weights_u32, csr_to_edgelist,
                    edgelist_to_csr, erdos_renyi, grid2d, read_gr, rmat, transpose, write_gr)

__all__ = [
    "DeviceGraph", "HostCSR", "GbError", "GB_DIST_INFINITY", "GB_CC_LABELPROP", "GB_CC_UNIONFIND",
    "GB_CC_AFFOREST", "GB_ORDER_NONE", "GB_ORDER_DEGREE", "GB_ORDER_DEGREE_UNSORTED",
    "GB_ORDER_LOCALITY", "GB_ORDER_AUTO", "read_gr", "write_gr",
    "rmat", "grid2d", "erdos_renyi", "assign_weights_u32", "assign_weights_reference", "assign_weights_f32", "transpose", "edgelist_to_csr", "csr_to_edgelist",
]
