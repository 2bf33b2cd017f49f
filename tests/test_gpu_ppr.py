"""GPU parity for batched personalised PageRank, its adjoint and the autograd
wrapper, against the FP64 oracle (oracle/ppr.py).

Tolerances: the fp32 Jacobi solve stops at a per-column L1 change <= tol
(1e-7 here); the remaining error is about tol * alpha / (1 - alpha) in L1, so
forward values are compared with atol 1e-6 + rtol 1e-4.  Gradients are
compared to the FP64 adjoint with rtol 1e-3 relative to the largest entry."""
import numpy as np
import pytest

from galois_b200 import DeviceGraph, HostCSR, assign_weights_f32, rmat
from oracle import ppr as oppr

pytestmark = pytest.mark.gpu
ALPHA = 0.85


def setup(scale=10, B=4, seed=5, nnz=8):
    g, _ = rmat(scale, 8, seed=seed, symmetrize=False)
    assign_weights_f32(g, seed=seed)
    rng = np.random.default_rng(seed)
    T = np.zeros((g.n, B), np.float32)
    for b in range(B):
        T[rng.choice(g.n, nnz, replace=False), b] = 1.0 / nnz
    c = rng.standard_normal((g.n, B)).astype(np.float32)
    return g, T, c


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("B", [1, 4, 128])
def test_forward_backward_vs_fp64(cuda_device, B):
    import torch

    from galois_b200 import _lib

    g, T, c = setup(B=B)
    w64 = g.w_f32.astype(np.float64)
    x_ref = oppr.forward(g, T.astype(np.float64), w64, ALPHA)
    gT_ref, gw_ref = oppr.backward(g, x_ref, c.astype(np.float64), w64, ALPHA)
    with DeviceGraph(g) as dg:
        Tt = torch.from_numpy(T).cuda()
        x = torch.empty_like(Tt)
        import ctypes as C

        st = _lib.lib.gb_ppr_forward(dg.handle, B, C.c_void_p(Tt.data_ptr()), None, ALPHA, 1e-7, 1000,
                                     C.c_void_p(x.data_ptr()), None, None, None)
        assert st == 0, _lib.last_error()
        xh = x.cpu().numpy().astype(np.float64)
        assert np.allclose(xh, x_ref, atol=1e-6, rtol=1e-4)
        ct = torch.from_numpy(c).cuda()
        gT = torch.empty_like(Tt)
        gw = torch.empty(g.m, dtype=torch.float32, device="cuda")
        st = _lib.lib.gb_ppr_backward(dg.handle, B, C.c_void_p(x.data_ptr()), C.c_void_p(ct.data_ptr()), None,
                                      ALPHA, 1e-7, 1000, C.c_void_p(gT.data_ptr()), C.c_void_p(gw.data_ptr()),
                                      None, None, None)
        assert st == 0, _lib.last_error()
        assert rel(gT.cpu().numpy(), gT_ref) < 1e-3
        assert rel(gw.cpu().numpy(), gw_ref) < 1e-3


def test_heavy_rows_tiled(cuda_device):
    import torch

    from galois_b200.ppr import ppr

    # a hub with in- and out-degree above the tiling threshold
    n = 3000
    src = [0] * (n - 1) + list(range(1, n)) + list(range(1, n - 1))
    dst = list(range(1, n)) + [0] * (n - 1) + list(range(2, n))
    g = HostCSR.from_edges(n, src, dst)
    assign_weights_f32(g, seed=2)
    rng = np.random.default_rng(1)
    B = 8
    T = np.zeros((n, B), np.float32)
    for b in range(B):
        T[rng.choice(n, 4, replace=False), b] = 0.25
    x_ref = oppr.forward(g, T.astype(np.float64), g.w_f32.astype(np.float64), ALPHA)
    with DeviceGraph(g) as dg:
        x = ppr(dg, torch.from_numpy(T).cuda(), torch.from_numpy(g.w_f32).cuda())
        assert np.allclose(x.cpu().numpy(), x_ref, atol=1e-6, rtol=1e-4)


def test_autograd_matches_fp64_and_finite_differences(cuda_device):
    import torch

    from galois_b200.ppr import ppr

    g, T, c = setup(scale=9, B=8)
    w = torch.from_numpy(g.w_f32.copy()).cuda().requires_grad_(True)
    Tt = torch.from_numpy(T).cuda().requires_grad_(True)
    ct = torch.from_numpy(c).cuda()
    with DeviceGraph(g) as dg:
        x = ppr(dg, Tt, w, ALPHA, 1e-7)
        loss = (ct * x).sum()
        loss.backward()
        w64 = g.w_f32.astype(np.float64)
        x_ref = oppr.forward(g, T.astype(np.float64), w64, ALPHA)
        gT_ref, gw_ref = oppr.backward(g, x_ref, c.astype(np.float64), w64, ALPHA)
        assert rel(Tt.grad.cpu().numpy(), gT_ref) < 1e-3
        assert rel(w.grad.cpu().numpy(), gw_ref) < 1e-3
        # central finite differences of the fp32 GPU forward on a few weights
        rng = np.random.default_rng(4)
        for e in rng.choice(np.flatnonzero(np.abs(gw_ref) > 0.05 * np.abs(gw_ref).max()), 4, replace=False):
            h = 1e-2 * float(g.w_f32[e])
            with torch.no_grad():
                wp = w.detach().clone()
                wp[e] += h
                wm = w.detach().clone()
                wm[e] -= h
                lp = float((ct * ppr(dg, Tt.detach(), wp, ALPHA, 1e-7)).sum())
                lm = float((ct * ppr(dg, Tt.detach(), wm, ALPHA, 1e-7)).sum())
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gw_ref[e]) <= 5e-2 * abs(gw_ref[e]) + 1e-4


def test_ppr_sharded_single_rank_matches_autograd(cuda_device):
    """galois_b200.distributed.ppr_sharded over a one-rank NCCL group gives
    the plain autograd result (the multi-rank split and the all-reduce of
    grad_w are covered by the gloo tests)."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    from galois_b200.distributed import ppr_sharded
    from galois_b200.ppr import ppr

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        g, T, c = setup(scale=10, B=8)
        with DeviceGraph(g) as dg:
            Tt = torch.from_numpy(T).cuda()
            ct = torch.from_numpy(c).cuda()
            w = torch.from_numpy(g.w_f32).cuda()
            x, cols, gt, gw, loss = ppr_sharded(dg, Tt, w, ct, ALPHA, 1e-7)
            wr = w.clone().requires_grad_(True)
            Tr = Tt.clone().requires_grad_(True)
            xr = ppr(dg, Tr, wr, ALPHA, 1e-7)
            lr = (ct * xr).sum()
            lr.backward()
        assert cols == (0, 8)
        assert torch.allclose(x, xr.detach())
        assert torch.allclose(gt, Tr.grad)
        assert torch.allclose(gw, wr.grad)
        assert abs(float(loss) - float(lr.detach())) <= 1e-5 * max(1.0, abs(float(lr.detach())))
    finally:
        dist.destroy_process_group()
