"""ORACLE -- test infrastructure only.

ctypes wrapper of oracle/liboracle.so, the CPU (C++17/OpenMP) restatement of
the Galois lonestar algorithms on the CSR edge-map path (see oracle.cpp for the
reference lines each function follows and how the restatement is pinned).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this package; the product never does.

Parity status: the reference cannot be built or run here (Boost, LLVM
CommandLine and fmt are absent; the GPU apps need the un-vendored moderngpu
submodule) and ships no golden outputs for this path, so there are no
reference-run outputs.  The restatement is pinned by the reference's own
verifiers (restated and run on every output), the graph-convert fixtures
(tools/graph-convert/test-inputs) for the .gr path, and closed-form known
answers.  PageRank and BC beyond closed-form cases are unpinned against the
reference itself.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        build()
    return C.CDLL(str(LIB_PATH))


_lib = _load()
_u32 = C.c_uint32
_vp = C.c_void_p

_SIG = {
    "orc_num_threads": (C.c_int, []),
    "orc_set_threads": (None, [C.c_int]),
    "orc_bfs_serial": (None, [_u32, _vp, _vp, _u32, _vp]),
    "orc_bfs_sync_tile": (None, [_u32, _vp, _vp, _u32, _vp]),
    "orc_verify_bfs": (C.c_int, [_u32, _vp, _vp, _u32, _vp]),
    "orc_bfs_do_parent": (None, [_u32, _vp, _vp, _vp, _vp, _u32, C.c_int, C.c_int, _vp]),
    "orc_bfs_parent_min": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_verify_bfs_parent": (C.c_int, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_sssp_dijkstra": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_sssp_delta_serial": (None, [_u32, _vp, _vp, _vp, _u32, _u32, _vp]),
    "orc_sssp_delta_parallel": (None, [_u32, _vp, _vp, _vp, _u32, _u32, _vp]),
    "orc_verify_sssp": (C.c_int, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_cc_union_find": (None, [_u32, _vp, _vp, _vp]),
    "orc_cc_labelprop": (_u32, [_u32, _vp, _vp, _vp]),
    "orc_verify_cc": (C.c_int, [_u32, _vp, _vp, _vp]),
    "orc_pr_pull_topo_f64": (_u32, [_u32, _vp, _vp, C.c_uint64, C.c_double, C.c_double, _u32, _vp]),
    "orc_pr_pull_topo_f32_inplace": (_u32, [_u32, _vp, _vp, C.c_uint64, C.c_float, C.c_float, _u32, _vp]),
    "orc_pr_pull_topo_par": (_u32, [_u32, _vp, _vp, C.c_uint64, C.c_float, C.c_float, _u32, _vp]),
    "orc_pr_pull_residual_f32": (_u32, [_u32, _vp, _vp, C.c_uint64, C.c_float, C.c_float, _u32, _vp]),
    "orc_pr_pull_residual_f64": (_u32, [_u32, _vp, _vp, C.c_uint64, C.c_double, C.c_double, _u32, _vp]),
    "orc_pr_push_sync_f32": (_u32, [_u32, _vp, _vp, C.c_float, C.c_float, _u32, _vp]),
    "orc_pr_push_sync_f64": (_u32, [_u32, _vp, _vp, C.c_double, C.c_double, _u32, _vp]),
    "orc_bc_level": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_bc_level_f64": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_bc_level_par": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_bc_level_f64_par_sources": (None, [_u32, _vp, _vp, _vp, _u32, _vp]),
    "orc_gr2randomweight": (None, [C.c_uint64, C.c_int, C.c_int, C.c_int, _vp]),
    "orc_mt19937_raw": (None, [C.c_uint64, _vp]),
    "orc_ppr_solve_f64": (_u32, [_u32, _vp, _vp, _vp, _vp, C.c_double, C.c_double, _u32, C.c_int, _vp]),
}
for _n, (_r, _a) in _SIG.items():
    _f = getattr(_lib, _n)
    _f.restype = _r
    _f.argtypes = _a

INF = 2147483646


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _g(g):
    """(n, end_offs, col) of a HostCSR-like object (end_offs LC layout)."""
    end = np.ascontiguousarray(g.end_offs, dtype=np.uint64)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    return g.n, end, col


def threads() -> int:
    return _lib.orc_num_threads()


def set_threads(t: int) -> None:
    _lib.orc_set_threads(t)


def bfs_serial(g, src: int) -> np.ndarray:
    n, end, col = _g(g)
    out = np.empty(n, np.uint32)
    _lib.orc_bfs_serial(n, _p(end), _p(col), src, _p(out))
    return out


def bfs_sync_tile(g, src: int) -> np.ndarray:
    n, end, col = _g(g)
    out = np.empty(n, np.uint32)
    _lib.orc_bfs_sync_tile(n, _p(end), _p(col), src, _p(out))
    return out


def verify_bfs(g, src: int, level) -> int:
    n, end, col = _g(g)
    lv = np.ascontiguousarray(level, np.uint32)
    return _lib.orc_verify_bfs(n, _p(end), _p(col), src, _p(lv))


def _in_edges(g):
    """(in_end, in_col): the transposed graph in the same end-offset layout
    (a symmetric graph is its own transpose)."""
    n, end, col = _g(g)
    deg = np.diff(np.concatenate(([0], end.astype(np.int64))))
    rows = np.repeat(np.arange(n, dtype=np.uint32), deg)
    order = np.lexsort((rows, col))  # by target, then source
    in_col = np.ascontiguousarray(rows[order], dtype=np.uint32)
    in_end = np.cumsum(np.bincount(col, minlength=n), dtype=np.uint64)
    return in_end, in_col


def bfs_do_parent(g, src: int, alpha: int = 15, beta: int = 18) -> np.ndarray:
    """Serial restatement of bfsDirectionOpt's SyncDO parents."""
    n, end, col = _g(g)
    in_end, in_col = _in_edges(g)
    out = np.empty(n, np.uint32)
    _lib.orc_bfs_do_parent(n, _p(end), _p(col), _p(in_end), _p(in_col), src, alpha, beta, _p(out))
    return out


def bfs_parent_min(g, src: int, level) -> np.ndarray:
    """Smallest-id in-neighbour one level closer, per reached vertex."""
    n, _, _ = _g(g)
    in_end, in_col = _in_edges(g)
    lv = np.ascontiguousarray(level, np.uint32)
    out = np.empty(n, np.uint32)
    _lib.orc_bfs_parent_min(n, _p(in_end), _p(in_col), _p(lv), src, _p(out))
    return out


def verify_bfs_parent(g, src: int, level, parent) -> int:
    n, _, _ = _g(g)
    in_end, in_col = _in_edges(g)
    lv = np.ascontiguousarray(level, np.uint32)
    pa = np.ascontiguousarray(parent, np.uint32)
    return _lib.orc_verify_bfs_parent(n, _p(in_end), _p(in_col), _p(lv), src, _p(pa))


def make_symmetric_file_order(g):
    """makeSymmetric (libgalois/include/galois/graphs/FileGraph.h:764-826) as
    the reference writes it: sources ascending, each arc (u, v) appended to
    u's row and, when u != v, (v, u) with the same edge data appended to v's
    row, rows filled in that append order.  Returns (end_offs, col, w_u32)."""
    n, end, col = _g(g)
    w = None if g.w_u32 is None else np.asarray(g.w_u32, np.uint32)
    rows = [[] for _ in range(n)]
    b = 0
    for u in range(n):
        e = int(end[u])
        for i in range(b, e):
            v = int(col[i])
            data = None if w is None else int(w[i])
            rows[u].append((v, data))
            if u != v:
                rows[v].append((u, data))
        b = e
    out_col = np.array([v for r in rows for v, _ in r], np.uint32)
    out_w = None if w is None else np.array([d for r in rows for _, d in r], np.uint32)
    out_end = np.cumsum([len(r) for r in rows], dtype=np.uint64)
    return out_end, out_col, out_w


def make_symmetric(g, cleanup: bool):
    """The device form of gr2sgr (and gr2cgr with cleanup): the arcs of
    make_symmetric_file_order with every row sorted by destination, forward
    copies before reverse ones and earlier arcs first among equal
    destinations; with cleanup (Cleanup, tools/graph-convert/
    graph-convert.cpp:1902-2024) self-loops dropped and, of repeated arcs,
    the first kept.  Returns (end_offs, col, w_u32)."""
    n, end, col = _g(g)
    m = col.size
    deg = np.diff(np.concatenate(([0], end.astype(np.int64))))
    src = np.repeat(np.arange(n, dtype=np.uint64), deg)
    dst = col.astype(np.uint64)
    idx = np.arange(m, dtype=np.int64)
    rev = dst != src
    s_all = np.concatenate([src, dst[rev]])
    d_all = np.concatenate([dst, src[rev]])
    i_all = np.concatenate([idx, idx[rev]])
    order = np.argsort((s_all << np.uint64(32)) | d_all, kind="stable")
    s_all, d_all, i_all = s_all[order], d_all[order], i_all[order]
    if cleanup and s_all.size:
        keep = s_all != d_all
        keep[1:] &= (s_all[1:] != s_all[:-1]) | (d_all[1:] != d_all[:-1])
        s_all, d_all, i_all = s_all[keep], d_all[keep], i_all[keep]
    out_end = np.cumsum(np.bincount(s_all.astype(np.int64), minlength=n), dtype=np.uint64)
    out_w = None if g.w_u32 is None else np.asarray(g.w_u32, np.uint32)[i_all]
    return out_end, d_all.astype(np.uint32), out_w


def sssp_dijkstra(g, src: int) -> np.ndarray:
    n, end, col = _g(g)
    w = np.ascontiguousarray(g.w_u32, np.uint32)
    out = np.empty(n, np.uint32)
    _lib.orc_sssp_dijkstra(n, _p(end), _p(col), _p(w), src, _p(out))
    return out


def sssp_delta_serial(g, src: int, shift: int = 13) -> np.ndarray:
    n, end, col = _g(g)
    w = np.ascontiguousarray(g.w_u32, np.uint32)
    out = np.empty(n, np.uint32)
    _lib.orc_sssp_delta_serial(n, _p(end), _p(col), _p(w), src, shift, _p(out))
    return out


def sssp_delta_parallel(g, src: int, shift: int = 13) -> np.ndarray:
    n, end, col = _g(g)
    w = np.ascontiguousarray(g.w_u32, np.uint32)
    out = np.empty(n, np.uint32)
    _lib.orc_sssp_delta_parallel(n, _p(end), _p(col), _p(w), src, shift, _p(out))
    return out


def verify_sssp(g, src: int, dist) -> int:
    n, end, col = _g(g)
    w = np.ascontiguousarray(g.w_u32, np.uint32)
    d = np.ascontiguousarray(dist, np.uint32)
    return _lib.orc_verify_sssp(n, _p(end), _p(col), _p(w), src, _p(d))


def cc_union_find(g) -> np.ndarray:
    n, end, col = _g(g)
    out = np.empty(n, np.uint32)
    _lib.orc_cc_union_find(n, _p(end), _p(col), _p(out))
    return out


def cc_labelprop(g) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.uint32)
    r = _lib.orc_cc_labelprop(n, _p(end), _p(col), _p(out))
    return out, int(r)


def verify_cc(g, label) -> int:
    n, end, col = _g(g)
    lb = np.ascontiguousarray(label, np.uint32)
    return _lib.orc_verify_cc(n, _p(end), _p(col), _p(lb))


def pr_pull_topo_f64(g, alpha=0.85, tol=1e-6, max_iter=1000) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.float64)
    it = _lib.orc_pr_pull_topo_f64(n, _p(end), _p(col), col.size, alpha, tol, max_iter, _p(out))
    return out, int(it)


def pr_pull_topo_f32_inplace(g, alpha=0.85, tol=1e-6, max_iter=1000) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.float32)
    it = _lib.orc_pr_pull_topo_f32_inplace(n, _p(end), _p(col), col.size, alpha, tol, max_iter, _p(out))
    return out, int(it)


def pr_pull_topo_par(g, alpha=0.85, tol=1e-6, max_iter=1000) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.float32)
    it = _lib.orc_pr_pull_topo_par(n, _p(end), _p(col), col.size, alpha, tol, max_iter, _p(out))
    return out, int(it)


def pr_pull_residual(g, alpha=0.85, tol=1e-3, max_iter=1000, f64=True) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.float64 if f64 else np.float32)
    fn = _lib.orc_pr_pull_residual_f64 if f64 else _lib.orc_pr_pull_residual_f32
    it = fn(n, _p(end), _p(col), col.size, alpha, tol, max_iter, _p(out))
    return out, int(it)


def pr_push_sync(g, alpha=0.85, tol=1e-3, max_iter=1000, f64=True) -> tuple[np.ndarray, int]:
    n, end, col = _g(g)
    out = np.empty(n, np.float64 if f64 else np.float32)
    fn = _lib.orc_pr_push_sync_f64 if f64 else _lib.orc_pr_push_sync_f32
    it = fn(n, _p(end), _p(col), alpha, tol, max_iter, _p(out))
    return out, int(it)


def bc_level(g, sources, f64: bool = False, parallel: bool = False) -> np.ndarray:
    """Level BC summed over `sources`.  f64: FP64 sigma, dependency and bc
    (parallel: sources spread over the threads); else the reference's types
    (fp64 sigma, fp32 dependency; parallel: all threads on one source)."""
    n, end, col = _g(g)
    src = np.ascontiguousarray(np.asarray(sources, np.uint32))
    if f64 and parallel:
        out = np.empty(n, np.float64)
        _lib.orc_bc_level_f64_par_sources(n, _p(end), _p(col), _p(src), src.size, _p(out))
    elif f64:
        out = np.empty(n, np.float64)
        _lib.orc_bc_level_f64(n, _p(end), _p(col), _p(src), src.size, _p(out))
    else:
        out = np.empty(n, np.float32)
        fn = _lib.orc_bc_level_par if parallel else _lib.orc_bc_level
        fn(n, _p(end), _p(col), _p(src), src.size, _p(out))
    return out


def ppr_solve_f64(g, w, rhs, alpha=0.85, tol=1e-13, max_iter=10000, adjoint=False) -> tuple[np.ndarray, int]:
    """FP64 Jacobi solve of one PPR column: x = rhs + alpha W~ x, or with
    adjoint the transposed system lam = rhs + alpha W~^T lam (the conventions
    of oracle/ppr.py), stopped at an L1 change <= tol * max(1, |rhs|_1)."""
    n, end, col = _g(g)
    wf = np.ascontiguousarray(w, np.float32)
    r = np.ascontiguousarray(rhs, np.float64)
    out = np.empty(n, np.float64)
    it = _lib.orc_ppr_solve_f64(n, _p(end), _p(col), _p(wf), _p(r), alpha, tol, max_iter, 1 if adjoint else 0,
                                _p(out))
    return out, int(it)


def gr2randomweight(m: int, lo: int = 1, hi: int = 100, dtype: str = "u32") -> np.ndarray:
    """The weights graph-convert's gr2randomweightgr writes for m arcs
    (graph-convert.cpp:1145-1190), from the C++ standard library."""
    out = np.empty(m, np.uint32)
    _lib.orc_gr2randomweight(m, lo, hi, 1 if dtype == "f32" else 0, _p(out))
    return out.view(np.float32) if dtype == "f32" else out


def mt19937_raw(count: int) -> np.ndarray:
    """The first `count` outputs of a default-constructed std::mt19937."""
    out = np.empty(count, np.uint32)
    _lib.orc_mt19937_raw(count, _p(out))
    return out
