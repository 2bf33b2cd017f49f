"""Host CSR graphs (numpy) and the device mirror handle over libgb.

HostCSR mirrors Galois' on-disk/in-memory CSR (LC_CSR_Graph end offsets,
uint32 destinations, optional uint32 or float edge data).  DeviceGraph owns a
``gb_graph*`` and exposes every algorithm of include/gb.h; outputs may be numpy
arrays (host) or CUDA torch tensors (device, asynchronous on the current torch
stream).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import HostCsrC, Stats, Tuning, check, lib


def _np_from(ptr, count: int, dtype) -> np.ndarray:
    if not ptr or count == 0:
        return np.empty(count, dtype=dtype)
    ct = np.ctypeslib.as_ctypes_type(dtype)
    buf = C.cast(ptr, C.POINTER(ct))
    return np.ctypeslib.as_array(buf, shape=(count,)).copy()


@dataclass
class HostCSR:
    """CSR with LC_CSR_Graph end offsets (``end_offs[v]`` = end of v's arcs)."""

    end_offs: np.ndarray  # uint64 [n]
    col: np.ndarray  # uint32 [m]
    w_u32: Optional[np.ndarray] = None
    w_f32: Optional[np.ndarray] = None

    def __post_init__(self):
        self.end_offs = np.ascontiguousarray(self.end_offs, dtype=np.uint64)
        self.col = np.ascontiguousarray(self.col, dtype=np.uint32)
        if self.w_u32 is not None:
            self.w_u32 = np.ascontiguousarray(self.w_u32, dtype=np.uint32)
        if self.w_f32 is not None:
            self.w_f32 = np.ascontiguousarray(self.w_f32, dtype=np.float32)

    @property
    def n(self) -> int:
        return int(self.end_offs.shape[0])

    @property
    def m(self) -> int:
        return int(self.col.shape[0])

    @property
    def offs(self) -> np.ndarray:
        """Begin offsets, n+1 entries (offs[0] = 0)."""
        return np.concatenate([np.zeros(1, np.uint64), self.end_offs])

    def degrees(self) -> np.ndarray:
        return np.diff(self.offs).astype(np.int64)

    @classmethod
    def from_offsets(cls, offs, col, w_u32=None, w_f32=None) -> "HostCSR":
        offs = np.asarray(offs, dtype=np.uint64)
        return cls(offs[1:].copy(), col, w_u32, w_f32)

    @classmethod
    def from_edges(cls, n: int, src, dst, w_u32=None, w_f32=None) -> "HostCSR":
        """Arcs in the given order, grouped by source (stable)."""
        src = np.asarray(src, dtype=np.int64)
        dst = np.asarray(dst, dtype=np.uint32)
        order = np.argsort(src, kind="stable")
        counts = np.bincount(src, minlength=n).astype(np.uint64)
        end = np.cumsum(counts).astype(np.uint64)
        wu = None if w_u32 is None else np.asarray(w_u32, np.uint32)[order]
        wf = None if w_f32 is None else np.asarray(w_f32, np.float32)[order]
        return cls(end, dst[order], wu, wf)

    # -- C interop ---------------------------------------------------------
    def _as_c(self) -> HostCsrC:
        c = HostCsrC()
        c.n = self.n
        c.m = self.m
        c.end_offs = self.end_offs.ctypes.data_as(C.POINTER(C.c_uint64))
        c.col = self.col.ctypes.data_as(C.POINTER(C.c_uint32))
        c.w_u32 = (self.w_u32.ctypes.data_as(C.POINTER(C.c_uint32)) if self.w_u32 is not None
                   else C.POINTER(C.c_uint32)())
        c.w_f32 = (self.w_f32.ctypes.data_as(C.POINTER(C.c_float)) if self.w_f32 is not None
                   else C.POINTER(C.c_float)())
        return c

    @classmethod
    def _take(cls, c: HostCsrC) -> "HostCSR":
        """Copy a library-allocated gb_host_csr into numpy and free it."""
        try:
            g = cls(_np_from(c.end_offs, c.n, np.uint64), _np_from(c.col, c.m, np.uint32),
                    _np_from(c.w_u32, c.m, np.uint32) if c.w_u32 else None,
                    _np_from(c.w_f32, c.m, np.float32) if c.w_f32 else None)
        finally:
            lib.gb_host_csr_free(C.byref(c))
        return g


def _call_out(fn_name: str, *args) -> HostCSR:
    c = HostCsrC()
    lib.gb_host_csr_init(C.byref(c))
    st = getattr(lib, fn_name)(*args, C.byref(c))
    if st != _lib.GB_OK:
        lib.gb_host_csr_free(C.byref(c))
        check(st, fn_name)
    return HostCSR._take(c)


def read_gr(path: str, edge_bytes: int = 0) -> HostCSR:
    """Read a Galois .gr file (v1/v2).  edge_bytes: 0, 4 (uint32), -4 (float)."""
    return _call_out("gb_gr_read", str(path).encode(), edge_bytes)


def write_gr(path: str, g: HostCSR, edge_bytes: int = 0) -> None:
    c = g._as_c()
    check(lib.gb_gr_write(str(path).encode(), C.byref(c), edge_bytes), "gb_gr_write")


def edgelist_to_csr(path: str, skip_first_line: bool = False, delim: str = "") -> HostCSR:
    d = delim.encode() if delim else b"\0"
    return _call_out("gb_edgelist_to_csr", str(path).encode(), int(skip_first_line), d)


def csr_to_edgelist(path: str, g: HostCSR) -> None:
    c = g._as_c()
    check(lib.gb_csr_to_edgelist(str(path).encode(), C.byref(c)), "gb_csr_to_edgelist")


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, symmetrize: bool = True, permute: bool = True) -> tuple[HostCSR, np.ndarray]:
    """Seeded RMAT graph; returns (graph, perm) with perm[i] = id of generator vertex i."""
    perm = np.empty(1 << scale, dtype=np.uint32)
    g = _call_out("gb_gen_rmat", scale, edge_factor, a, b, c, seed, int(symmetrize), int(permute),
                  perm.ctypes.data_as(C.POINTER(C.c_uint32)))
    return g, perm


def grid2d(rows: int, cols: int) -> HostCSR:
    return _call_out("gb_gen_grid2d", rows, cols)


def erdos_renyi(n: int, mean_degree: float = 8.0, seed: int = 1) -> HostCSR:
    return _call_out("gb_gen_er", n, mean_degree, seed)


def assign_weights_u32(g: HostCSR, lo: int = 1, hi: int = 255, seed: int = 1) -> HostCSR:
    c = g._as_c()
    c.w_u32 = C.POINTER(C.c_uint32)()
    c.w_f32 = C.POINTER(C.c_float)()
    st = lib.gb_assign_weights_u32(C.byref(c), lo, hi, seed)
    check(st, "gb_assign_weights_u32")
    g.w_u32 = _np_from(c.w_u32, g.m, np.uint32)
    _free_ptr(c.w_u32)
    return g


def assign_weights_f32(g: HostCSR, seed: int = 1) -> HostCSR:
    c = g._as_c()
    c.w_u32 = C.POINTER(C.c_uint32)()
    c.w_f32 = C.POINTER(C.c_float)()
    check(lib.gb_assign_weights_f32(C.byref(c), seed), "gb_assign_weights_f32")
    g.w_f32 = _np_from(c.w_f32, g.m, np.float32)
    _free_ptr(c.w_f32)
    return g


def assign_weights_reference(g: HostCSR, min_value: int = 1, max_value: int = 100, dtype: str = "u32") -> HostCSR:
    """Weights as the reference's gr2randomweightgr draws them: a default
    std::mt19937 with a uniform int (dtype "u32") or float ("f32")
    distribution over [min_value, max_value], one draw per arc in arc order
    (graph-convert.cpp:1145-1190; the converter's defaults are 1 and 100)."""
    if dtype not in ("u32", "f32"):
        raise ValueError("dtype must be 'u32' or 'f32'")
    c = g._as_c()
    c.w_u32 = C.POINTER(C.c_uint32)()
    c.w_f32 = C.POINTER(C.c_float)()
    eb = 4 if dtype == "u32" else -4
    check(lib.gb_assign_weights_reference(C.byref(c), min_value, max_value, eb), "gb_assign_weights_reference")
    if dtype == "u32":
        g.w_u32 = _np_from(c.w_u32, g.m, np.uint32)
        _free_ptr(c.w_u32)
    else:
        g.w_f32 = _np_from(c.w_f32, g.m, np.float32)
        _free_ptr(c.w_f32)
    return g


def _free_ptr(p) -> None:
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(p, C.c_void_p))


def pack_graphs(graphs: list) -> tuple[HostCSR, np.ndarray]:
    """Block-diagonal packing of disjoint graphs; returns (graph, graph_first)
    with graph_first[k] the first vertex of graph k and graph_first[-1] = n."""
    first = np.zeros(len(graphs) + 1, dtype=np.uint32)
    ends, cols = [], []
    vbase, ebase = 0, 0
    for k, g in enumerate(graphs):
        first[k] = vbase
        ends.append(g.end_offs.astype(np.uint64) + np.uint64(ebase))
        cols.append(g.col.astype(np.uint32) + np.uint32(vbase))
        vbase += g.n
        ebase += g.m
    first[-1] = vbase
    return HostCSR(np.concatenate(ends), np.concatenate(cols)), first


def transpose(g: HostCSR) -> tuple[HostCSR, np.ndarray]:
    """Transposed graph and, per transposed arc, its index in g."""
    emap = np.empty(g.m, dtype=np.uint64)
    c = g._as_c()
    out = HostCsrC()
    lib.gb_host_csr_init(C.byref(out))
    st = lib.gb_transpose_host(C.byref(c), C.byref(out), emap.ctypes.data_as(C.POINTER(C.c_uint64)))
    if st != _lib.GB_OK:
        lib.gb_host_csr_free(C.byref(out))
        check(st, "gb_transpose_host")
    return HostCSR._take(out), emap
