"""ctypes binding of libgb.so (include/gb.h).

The library is the product: if it is missing this module raises ImportError
instead of falling back to anything else.  Build it with
``python -m galois_b200.build``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgb.so"

GB_OK = 0
GB_ERR_ARG = -1
GB_ERR_OOM = -2
GB_ERR_CUDA = -3
GB_ERR_TIMEOUT = -4
GB_ERR_FILE = -5
GB_ERR_FORMAT = -6
GB_ERR_NOT_CONVERGED = -7
GB_ERR_UNSUPPORTED = -8
GB_ERR_CAPACITY = -9
GB_DIST_INFINITY = 2147483646

GB_CC_LABELPROP = 0
GB_CC_UNIONFIND = 1
GB_CC_AFFOREST = 2
GB_ORDER_NONE = 0
GB_ORDER_DEGREE = 1
GB_ORDER_DEGREE_UNSORTED = 2
GB_ORDER_LOCALITY = 3
GB_ORDER_AUTO = 4
GB_PR_PUSH_ASYNC = 0
GB_PR_PUSH_SYNC = 1

_STATUS_NAMES = {
    GB_ERR_ARG: "GB_ERR_ARG", GB_ERR_OOM: "GB_ERR_OOM", GB_ERR_CUDA: "GB_ERR_CUDA",
    GB_ERR_TIMEOUT: "GB_ERR_TIMEOUT", GB_ERR_FILE: "GB_ERR_FILE", GB_ERR_FORMAT: "GB_ERR_FORMAT",
    GB_ERR_NOT_CONVERGED: "GB_ERR_NOT_CONVERGED", GB_ERR_UNSUPPORTED: "GB_ERR_UNSUPPORTED",
    GB_ERR_CAPACITY: "GB_ERR_CAPACITY",
}


class GbError(RuntimeError):
    """A libgb call returned a non-zero status."""

    def __init__(self, status: int, func: str, message: str):
        self.status = status
        super().__init__(f"{func}: {_STATUS_NAMES.get(status, status)}: {message}")


class HostCsrC(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("end_offs", C.POINTER(C.c_uint64)),
                ("col", C.POINTER(C.c_uint32)), ("w_u32", C.POINTER(C.c_uint32)),
                ("w_f32", C.POINTER(C.c_float))]


class Stats(C.Structure):
    _fields_ = [("vertices_reached", C.c_uint64), ("edges_reached", C.c_uint64),
                ("edges_scanned", C.c_uint64), ("relaxations", C.c_uint64), ("rounds", C.c_uint32),
                ("pull_rounds", C.c_uint32), ("buckets", C.c_uint32), ("launches", C.c_uint32),
                ("residual", C.c_double), ("kernel_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("heavy_degree", C.c_uint32), ("tile_edges", C.c_uint32), ("block_threads", C.c_uint32),
                ("blocks_per_sm", C.c_uint32), ("do_alpha", C.c_float), ("do_beta", C.c_float),
                ("direction_opt", C.c_int), ("local_depth", C.c_int),
                ("sssp_async", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python galois_b200/build.py` "
                          "(the CUDA library is required; there is no CPU fallback)")
    return C.CDLL(str(LIB_PATH), mode=C.RTLD_GLOBAL)


lib = _load()

_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_f32p = C.POINTER(C.c_float)
_vp = C.c_void_p
_csrp = C.POINTER(HostCsrC)
_gp = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/gb.h
SIGNATURES: dict[str, tuple] = {
    "gb_last_error": (C.c_char_p, []),
    "gb_version": (C.c_int, []),
    "gb_host_csr_init": (None, [_csrp]),
    "gb_host_csr_free": (None, [_csrp]),
    "gb_gr_read": (C.c_int, [C.c_char_p, C.c_int, _csrp]),
    "gb_gr_write": (C.c_int, [C.c_char_p, _csrp, C.c_int]),
    "gb_edgelist_to_csr": (C.c_int, [C.c_char_p, C.c_int, C.c_char, _csrp]),
    "gb_csr_to_edgelist": (C.c_int, [C.c_char_p, _csrp]),
    "gb_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                              C.c_int, C.c_int, _u32p, _csrp]),
    "gb_gen_grid2d": (C.c_int, [C.c_uint32, C.c_uint32, _csrp]),
    "gb_gen_er": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, _csrp]),
    "gb_assign_weights_u32": (C.c_int, [_csrp, C.c_uint32, C.c_uint32, C.c_uint64]),
    "gb_assign_weights_f32": (C.c_int, [_csrp, C.c_uint64]),
    "gb_assign_weights_reference": (C.c_int, [_csrp, C.c_int, C.c_int, C.c_int]),
    "gb_transpose_host": (C.c_int, [_csrp, _csrp, _u64p]),
    "gb_graph_upload": (C.c_int, [_vp, _vp, _vp, _vp, C.c_uint32, C.c_uint64, C.c_int, C.c_int,
                                  C.POINTER(_gp)]),
    "gb_graph_load_gr": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(_gp)]),
    "gb_graph_free": (C.c_int, [_gp]),
    "gb_graph_info": (C.c_int, [_gp, _u32p, _u64p, C.POINTER(C.c_int)]),
    "gb_graph_device_arrays": (C.c_int, [_gp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                         C.POINTER(_vp)]),
    "gb_graph_build_transpose": (C.c_int, [_gp, _vp]),
    "gb_graph_symmetrize": (C.c_int, [_gp, C.c_int, _vp]),
    "gb_graph_assign_weights_u32": (C.c_int, [_gp, C.c_uint32, C.c_uint32, C.c_uint64, _vp]),
    "gb_graph_assign_weights_f32": (C.c_int, [_gp, C.c_uint64, _vp]),
    "gb_graph_assign_weights_reference": (C.c_int, [_gp, C.c_int, C.c_int, C.c_int, _vp]),
    "gb_graph_reorder": (C.c_int, [_gp, C.c_int, _vp]),
    "gb_pool_trim": (C.c_int, []),
    "gb_graph_permutation": (C.c_int, [_gp, C.POINTER(_vp), C.POINTER(_vp)]),
    "gb_graph_order": (C.c_int, [_gp, C.POINTER(C.c_int)]),
    "gb_graph_set_tuning": (C.c_int, [_gp, C.POINTER(Tuning)]),
    "gb_graph_get_tuning": (C.c_int, [_gp, C.POINTER(Tuning)]),
    "gb_bfs": (C.c_int, [_gp, C.c_uint32, _vp, C.POINTER(Stats), _vp]),
    "gb_bfs_parent": (C.c_int, [_gp, C.c_uint32, _vp, _vp, C.POINTER(Stats), _vp]),
    "gb_bfs_noalloc": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint64, C.c_int, C.c_uint32, _vp, _vp]),
    "gb_sssp_delta": (C.c_int, [_gp, C.c_uint32, C.c_uint32, _vp, C.POINTER(Stats), _vp]),
    "gb_cc": (C.c_int, [_gp, C.c_int, _vp, C.POINTER(Stats), _vp]),
    "gb_pagerank_pull": (C.c_int, [_gp, C.c_float, C.c_float, C.c_uint32, _vp, _u32p, C.POINTER(Stats), _vp]),
    "gb_pagerank_pull_ex": (C.c_int, [_gp, C.c_float, C.c_float, C.c_uint32, C.c_float, C.c_float, C.c_int,
                                      _vp, _u32p, C.POINTER(Stats), _vp]),
    "gb_pagerank_push": (C.c_int, [_gp, C.c_float, C.c_float, C.c_uint32, _vp, _u32p, C.POINTER(Stats), _vp]),
    "gb_pagerank_push_ex": (C.c_int, [_gp, C.c_int, C.c_float, C.c_float, C.c_uint32, _vp, _u32p, C.POINTER(Stats),
                                      _vp]),
    "gb_pagerank_pull_residual": (C.c_int, [_gp, C.c_float, C.c_float, C.c_uint32, _vp, _u32p,
                                            C.POINTER(Stats), _vp]),
    "gb_bc": (C.c_int, [_gp, _vp, C.c_uint32, C.c_uint32, _vp, C.POINTER(Stats), _vp]),
    "gb_multi_graph_bfs_cc": (C.c_int, [_gp, _vp, C.c_uint32, _vp, _vp, _vp, C.POINTER(Stats), _vp]),
    "gb_ppr_forward": (C.c_int, [_gp, C.c_uint32, _vp, _vp, C.c_float, C.c_float, C.c_uint32, _vp, _u32p,
                                 C.POINTER(Stats), _vp]),
    "gb_ppr_backward": (C.c_int, [_gp, C.c_uint32, _vp, _vp, _vp, C.c_float, C.c_float, C.c_uint32, _vp,
                                  _vp, _u32p, C.POINTER(Stats), _vp]),
    "gb_autotune": (C.c_int, [_gp, C.c_char_p, C.c_uint32, C.c_char_p, C.POINTER(Tuning), _vp]),
    "gb_probe_bounded_waits": (C.c_int, [C.c_int, C.c_uint32, _vp]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error() -> str:
    return lib.gb_last_error().decode(errors="replace")


def check(status: int, func: str, allow: tuple[int, ...] = ()) -> int:
    if status != GB_OK and status not in allow:
        raise GbError(status, func, last_error())
    return status
