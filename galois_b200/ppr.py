"""Differentiable personalised PageRank over the B200 kernels.

``ppr(graph, teleport, w)`` solves x = (1-alpha) T + alpha W~ x for a batch of
teleport columns (T: [n, B] CUDA float32, B = 1 or a multiple of 4 <= 128)
with W~_ij = w_ji / s_j (arc weights w in the graph's CSR order, s_j the
out-weight sum of j).  Gradients with respect to T and w come from the
hand-written adjoint kernel (gb_ppr_backward): one transposed solve
lam = dL/dx + alpha W~^T lam, then dL/dT = (1-alpha) lam and
dL/dw_ji = alpha/s_j * sum_b x_j^b (lam_i^b - mu_j^b), mu_j = (lam_j - dL/dx_j)/alpha.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import Stats, check, lib
from .device import DeviceGraph


def _ptr(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(t: torch.Tensor):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


class PersonalizedPageRank(torch.autograd.Function):
    @staticmethod
    def forward(ctx, graph: DeviceGraph, teleport: torch.Tensor, w: torch.Tensor | None, alpha: float, tol: float,
                max_iter: int):
        if not teleport.is_cuda or teleport.dtype != torch.float32:
            raise TypeError("teleport must be a CUDA float32 tensor [n, B]")
        teleport = teleport.contiguous()
        n, B = teleport.shape
        if n != graph.n:
            raise ValueError(f"teleport has {n} rows, graph has {graph.n} vertices")
        if w is not None:
            if not w.is_cuda or w.dtype != torch.float32 or w.numel() != graph.m:
                raise TypeError("w must be a CUDA float32 tensor with one weight per arc")
            w = w.contiguous()
        x = torch.empty_like(teleport)
        it = C.c_uint32(0)
        st = Stats()
        check(lib.gb_ppr_forward(graph.handle, B, _ptr(teleport), _ptr(w), alpha, tol, max_iter, _ptr(x),
                                 C.byref(it), C.byref(st), _stream(teleport)), "gb_ppr_forward",
              allow=(_lib.GB_ERR_NOT_CONVERGED,))
        ctx.graph = graph
        ctx.params = (alpha, tol, max_iter)
        ctx.iters = it.value
        ctx.save_for_backward(x, w if w is not None else torch.empty(0, device=x.device))
        ctx.has_w = w is not None
        return x

    @staticmethod
    def backward(ctx, gx: torch.Tensor):
        x, w = ctx.saved_tensors
        alpha, tol, max_iter = ctx.params
        gx = gx.contiguous().to(torch.float32)
        n, B = x.shape
        grad_t = torch.empty_like(x) if ctx.needs_input_grad[1] else None
        grad_w = torch.empty(ctx.graph.m, dtype=torch.float32, device=x.device) if (
            ctx.has_w and ctx.needs_input_grad[2]) else None
        it = C.c_uint32(0)
        check(lib.gb_ppr_backward(ctx.graph.handle, B, _ptr(x), _ptr(gx), _ptr(w) if ctx.has_w else None, alpha, tol,
                                  max_iter, _ptr(grad_t), _ptr(grad_w), C.byref(it), None, _stream(x)),
              "gb_ppr_backward", allow=(_lib.GB_ERR_NOT_CONVERGED,))
        return None, grad_t, grad_w, None, None, None


def ppr(graph: DeviceGraph, teleport: torch.Tensor, w: torch.Tensor | None = None, alpha: float = 0.85,
        tol: float = 1e-7, max_iter: int = 1000) -> torch.Tensor:
    """Batched personalised PageRank with autograd support (see module doc)."""
    return PersonalizedPageRank.apply(graph, teleport, w, alpha, tol, max_iter)
