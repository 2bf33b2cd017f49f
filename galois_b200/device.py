"""DeviceGraph: the gb_graph handle (device mirror of an LC_CSR_Graph).

Every method calls one C-ABI entry point of libgb.so.  `out` buffers may be
numpy arrays (the call copies back and synchronises) or contiguous CUDA torch
tensors (the call stays asynchronous on torch's current stream unless stats
are requested).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import Stats, Tuning, check, lib
from .graph import HostCSR


def _torch():
    import torch  # noqa: PLC0415  (only needed for device buffers)

    return torch


def _is_tensor(x) -> bool:
    return type(x).__module__.startswith("torch")


def _buf(x, count: int, np_dtype, what: str):
    """Return (pointer, stream, obj) for an input/output buffer."""
    if _is_tensor(x):
        torch = _torch()
        want = {np.uint32: torch.int32, np.float32: torch.float32, np.uint64: torch.int64,
                np.float64: torch.float64}[np_dtype]
        if x.dtype not in (want, getattr(torch, "uint32", want)) and not (
                np_dtype == np.uint32 and x.dtype == torch.int32):
            raise TypeError(f"{what}: expected dtype {want}, got {x.dtype}")
        if not x.is_contiguous() or x.numel() < count:
            raise ValueError(f"{what}: need a contiguous tensor with >= {count} elements")
        stream = torch.cuda.current_stream(x.device).cuda_stream if x.is_cuda else None
        return C.c_void_p(x.data_ptr()), stream, x
    arr = np.asarray(x)
    if arr.dtype != np_dtype or not arr.flags.c_contiguous or arr.size < count:
        raise ValueError(f"{what}: need a C-contiguous {np.dtype(np_dtype).name} array of >= {count}")
    return C.c_void_p(arr.ctypes.data), None, arr


class DeviceGraph:
    """Device-resident CSR (gb_graph*)."""

    def __init__(self, g: HostCSR, symmetric: bool = False, device: int = 0, reorder: int = 0):
        """reorder: 0 keeps file order, 1 (GB_ORDER_DEGREE) relabels by
        descending degree with sorted rows, 2 without the row sort.  Results
        are in original ids either way."""
        handle = C.c_void_p()
        wu = C.c_void_p(g.w_u32.ctypes.data) if g.w_u32 is not None else None
        wf = C.c_void_p(g.w_f32.ctypes.data) if g.w_f32 is not None else None
        check(lib.gb_graph_upload(C.c_void_p(g.end_offs.ctypes.data), C.c_void_p(g.col.ctypes.data), wu, wf,
                                  g.n, g.m, int(symmetric), device, C.byref(handle)), "gb_graph_upload")
        self._h = handle
        self.n = g.n
        self.m = g.m
        self.symmetric = bool(symmetric)
        self.device = device
        if reorder:
            self.reorder(reorder)

    def reorder(self, order: int = _lib.GB_ORDER_DEGREE) -> None:
        check(lib.gb_graph_reorder(self.handle, int(order), None), "gb_graph_reorder")

    @property
    def order(self) -> int:
        """The order the graph was relabelled with (GB_ORDER_NONE if never;
        GB_ORDER_AUTO reports the order it chose)."""
        o = C.c_int()
        check(lib.gb_graph_order(self.handle, C.byref(o)), "gb_graph_order")
        return o.value

    def permutation(self) -> dict:
        """Device pointers of the relabelling (None when in file order)."""
        p = [C.c_void_p() for _ in range(2)]
        check(lib.gb_graph_permutation(self.handle, *[C.byref(x) for x in p]), "gb_graph_permutation")
        return {"new_to_old": p[0].value, "old_to_new": p[1].value}

    @classmethod
    def from_handle(cls, handle: C.c_void_p) -> "DeviceGraph":
        self = cls.__new__(cls)
        self._h = handle
        n = C.c_uint32()
        m = C.c_uint64()
        s = C.c_int()
        check(lib.gb_graph_info(handle, C.byref(n), C.byref(m), C.byref(s)), "gb_graph_info")
        self.n, self.m, self.symmetric, self.device = n.value, m.value, bool(s.value), 0
        return self

    @classmethod
    def load_gr(cls, path: str, edge_bytes: int = 0, symmetric: bool = False, device: int = 0,
                reorder: int = 0) -> "DeviceGraph":
        h = C.c_void_p()
        check(lib.gb_graph_load_gr(str(path).encode(), edge_bytes, int(symmetric), device, C.byref(h)),
              "gb_graph_load_gr")
        g = cls.from_handle(h)
        g.device = device
        if reorder:
            g.reorder(reorder)
        return g

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise RuntimeError("DeviceGraph has been freed")
        return self._h

    def free(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib.gb_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    # -- tuning ------------------------------------------------------------
    def set_tuning(self, **kw) -> None:
        t = Tuning()
        check(lib.gb_graph_get_tuning(self.handle, C.byref(t)), "gb_graph_get_tuning")
        for k, v in kw.items():
            setattr(t, k, v)
        check(lib.gb_graph_set_tuning(self.handle, C.byref(t)), "gb_graph_set_tuning")

    def get_tuning(self) -> dict:
        t = Tuning()
        check(lib.gb_graph_get_tuning(self.handle, C.byref(t)), "gb_graph_get_tuning")
        return t.as_dict()

    def build_transpose(self) -> None:
        check(lib.gb_graph_build_transpose(self.handle, None), "gb_graph_build_transpose")

    def symmetrize(self, cleanup: bool = True) -> None:
        """Add every reverse arc on the device (gr2sgr); with cleanup also
        drop self-loops and repeated arcs (gr2cgr)."""
        check(lib.gb_graph_symmetrize(self.handle, int(cleanup), None), "gb_graph_symmetrize")
        self._refresh()

    def assign_weights_u32(self, lo: int, hi: int, seed: int) -> None:
        """Uniform integer arc weights in [lo, hi], drawn on the device; equal
        to graph.assign_weights_u32 on the host for the same arcs and seed."""
        check(lib.gb_graph_assign_weights_u32(self.handle, lo, hi, seed, None), "gb_graph_assign_weights_u32")

    def assign_weights_reference(self, min_value: int = 1, max_value: int = 100, dtype: str = "u32") -> None:
        """gr2randomweightgr's weights (a default std::mt19937, arc order) on
        the device mirror; see galois_b200.graph.assign_weights_reference."""
        if dtype not in ("u32", "f32"):
            raise ValueError("dtype must be 'u32' or 'f32'")
        check(lib.gb_graph_assign_weights_reference(self.handle, min_value, max_value, 4 if dtype == "u32" else -4,
                                                    None), "gb_graph_assign_weights_reference")

    def assign_weights_f32(self, seed: int) -> None:
        check(lib.gb_graph_assign_weights_f32(self.handle, seed, None), "gb_graph_assign_weights_f32")

    def _refresh(self) -> None:
        n = C.c_uint32()
        m = C.c_uint64()
        s = C.c_int()
        check(lib.gb_graph_info(self.handle, C.byref(n), C.byref(m), C.byref(s)), "gb_graph_info")
        self.n, self.m, self.symmetric = n.value, m.value, bool(s.value)

    def to_host(self):
        """(end_offs, col, w_u32 or None, w_f32 or None) copied back from the
        device mirror, in its current (possibly relabelled) numbering."""
        import torch

        a = self.device_arrays()
        self._refresh()

        class _View:  # a device array seen through __cuda_array_interface__
            def __init__(self, ptr, count, typestr):
                self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                                 "version": 3}

        def grab(ptr, count, dtype):
            if not ptr:
                return None
            if count == 0:
                return np.empty(0, dtype)
            signed = {np.uint64: "<i8", np.uint32: "<i4", np.float32: "<f4"}[dtype]
            t = torch.as_tensor(_View(ptr, count, signed), device=f"cuda:{self.device}")
            return t.cpu().numpy().view(dtype)

        offs = grab(a["offs"], self.n + 1, np.uint64)
        return offs[1:].copy(), grab(a["col"], self.m, np.uint32), grab(a["w_u32"], self.m, np.uint32), \
            grab(a["w_f32"], self.m, np.float32)

    def device_arrays(self) -> dict:
        p = [C.c_void_p() for _ in range(4)]
        check(lib.gb_graph_device_arrays(self.handle, *[C.byref(x) for x in p]), "gb_graph_device_arrays")
        return dict(zip(("offs", "col", "w_u32", "w_f32"), (x.value for x in p)))

    # -- helpers -------------------------------------------------------------
    def _out(self, out, count, dtype, what):
        if out is None:
            out = np.empty(count, dtype=dtype)
        return _buf(out, count, dtype, what)

    @staticmethod
    def _stats(want: bool):
        return Stats() if want else None

    # -- algorithms ----------------------------------------------------------
    def bfs(self, src: int, out=None, stats: bool = False):
        ptr, stream, obj = self._out(out, self.n, np.uint32, "level_out")
        s = self._stats(stats)
        check(lib.gb_bfs(self.handle, src, ptr, C.byref(s) if s else None, stream), "gb_bfs")
        return (obj, s.as_dict()) if stats else obj

    def bfs_parent(self, src: int, out=None, level_out=None, stats: bool = False):
        """Parents of a BFS tree from src (bfsDirectionOpt's output): the
        smallest-id in-neighbour one level closer; 0 at src, INF unreached."""
        ptr, stream, obj = self._out(out, self.n, np.uint32, "parent_out")
        lptr = None
        if level_out is not None:
            lptr, _, _ = self._out(level_out, self.n, np.uint32, "level_out")
        s = self._stats(stats)
        check(lib.gb_bfs_parent(self.handle, src, ptr, lptr, C.byref(s) if s else None, stream), "gb_bfs_parent")
        return (obj, s.as_dict()) if stats else obj

    def sssp(self, src: int, delta_shift: int = 13, out=None, stats: bool = False):
        ptr, stream, obj = self._out(out, self.n, np.uint32, "dist_out")
        s = self._stats(stats)
        check(lib.gb_sssp_delta(self.handle, src, delta_shift, ptr, C.byref(s) if s else None, stream),
              "gb_sssp_delta")
        return (obj, s.as_dict()) if stats else obj

    def cc(self, algo: int = _lib.GB_CC_LABELPROP, out=None, stats: bool = False):
        ptr, stream, obj = self._out(out, self.n, np.uint32, "label_out")
        s = self._stats(stats)
        check(lib.gb_cc(self.handle, algo, ptr, C.byref(s) if s else None, stream), "gb_cc")
        return (obj, s.as_dict()) if stats else obj

    def _pr(self, fn, alpha, tol, max_iter, out, stats, allow_not_converged):
        ptr, stream, obj = self._out(out, self.n, np.float32, "rank_out")
        it = C.c_uint32(0)
        s = Stats()
        st = getattr(lib, fn)(self.handle, alpha, tol, max_iter, ptr, C.byref(it), C.byref(s), stream)
        check(st, fn, allow=(_lib.GB_ERR_NOT_CONVERGED,) if allow_not_converged else ())
        info = s.as_dict()
        info["iterations"] = it.value
        info["converged"] = st == _lib.GB_OK
        return (obj, info) if stats else obj

    def pagerank_pull(self, alpha=0.85, tol=1e-3, max_iter=1000, out=None, stats=False,
                      allow_not_converged=True):
        return self._pr("gb_pagerank_pull", alpha, tol, max_iter, out, stats, allow_not_converged)

    def pagerank_pull_residual(self, alpha=0.85, tol=1e-3, max_iter=1000, out=None, stats=False,
                               allow_not_converged=True):
        return self._pr("gb_pagerank_pull_residual", alpha, tol, max_iter, out, stats, allow_not_converged)

    def pagerank_push(self, alpha=0.85, tol=1e-3, max_iter=1000, out=None, stats=False,
                      allow_not_converged=True, algo: str = "sync"):
        """Residual push (PageRank-push.cpp): algo "sync" (rounds, :103-188)
        or "async" (one worklist pass, :68-101, the lonestar app's default;
        max_iter does not apply and one iteration is reported)."""
        if algo == "sync":
            return self._pr("gb_pagerank_push", alpha, tol, max_iter, out, stats, allow_not_converged)
        if algo != "async":
            raise ValueError("algo must be 'sync' or 'async'")
        ptr, stream, obj = self._out(out, self.n, np.float32, "rank_out")
        it = C.c_uint32(0)
        s = Stats()
        st = lib.gb_pagerank_push_ex(self.handle, _lib.GB_PR_PUSH_ASYNC, alpha, tol, max_iter, ptr, C.byref(it),
                                     C.byref(s), stream)
        check(st, "gb_pagerank_push_ex")
        info = s.as_dict()
        info["iterations"] = it.value
        info["converged"] = True
        return (obj, info) if stats else obj

    def bc(self, sources, batch: int = 64, out=None, stats: bool = False):
        src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32))
        ptr, stream, obj = self._out(out, self.n, np.float32, "bc_out")
        s = self._stats(stats)
        check(lib.gb_bc(self.handle, C.c_void_p(src.ctypes.data), src.size, batch, ptr,
                        C.byref(s) if s else None, stream), "gb_bc")
        return (obj, s.as_dict()) if stats else obj

    def multi_graph_bfs_cc(self, graph_first, local_src, level_out=None, label_out=None, stats=False):
        gf = np.ascontiguousarray(np.asarray(graph_first, dtype=np.uint32))
        ls = np.ascontiguousarray(np.asarray(local_src, dtype=np.uint32))
        lp, stream, lobj = self._out(level_out, self.n, np.uint32, "level_out")
        cp, _, cobj = self._out(label_out, self.n, np.uint32, "label_out")
        s = self._stats(stats)
        check(lib.gb_multi_graph_bfs_cc(self.handle, C.c_void_p(gf.ctypes.data), ls.size,
                                        C.c_void_p(ls.ctypes.data), lp, cp, C.byref(s) if s else None, stream),
              "gb_multi_graph_bfs_cc")
        return (lobj, cobj, s.as_dict()) if stats else (lobj, cobj)

    def autotune(self, kernel: str, src: int = 0, cache_path: Optional[str] = None) -> dict:
        t = Tuning()
        check(lib.gb_autotune(self.handle, kernel.encode(), src, cache_path.encode() if cache_path else None,
                              C.byref(t), None), "gb_autotune")
        return t.as_dict()
