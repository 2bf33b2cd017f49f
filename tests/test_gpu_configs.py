"""GPU parity at the benchmark configurations themselves (full size), through
the C ABI, against the CPU oracle on the same seeded inputs.

Configurations (seeds as bench.py generates them):
  * BFS, RMAT-20 symmetric ef16, source = max-degree vertex; also RMAT-24.
  * SSSP delta-stepping, delta = 2^13, w ~ U[1,255]: RMAT-22 directed ef16
    (source = generator vertex 0) and the 4096x4096 grid (source 0).
  * CC (label propagation, Afforest) and PageRank pull-topological on RMAT-24
    symmetric ef16 (alpha 0.85, tol 1e-6, max 1000).
  * Brandes BC on RMAT-20 symmetric from 1024 seeded sources, 64 per launch.
  * 512 Erdos-Renyi graphs (n log-uniform in [1k, 200k], mean degree 8), BFS
    + CC in one launch, autotuned, replayed from a CUDA graph.
  * Batched personalised PageRank + adjoint, RMAT-22 directed, B = 128.

Tolerances: BFS levels, SSSP distances and CC labels are integers and must be
bit-exact.  PageRank: L-inf <= 1e-5 against the FP64 Jacobi oracle and the
iteration count within 2 of the oracle's.  BC: |gpu - fp64| <= 1e-6 *
max(|fp64|, 1) per vertex.  PPR: forward columns within atol 1e-6 + rtol 1e-4
of an FP64 solve (the fp32 solve stops at an L1 change of 1e-7, whose tail is
about 1e-7 * alpha / (1 - alpha) in L1), teleport gradients within 1e-3 of
the largest entry, and the edge-weight gradient equal (rtol 1e-4 of the
largest entry) to its defining sum evaluated in FP64 from the GPU's own x and
lambda on 20000 sampled arcs.

Both vertex orders are run where bench.py times the degree-ordered graph
(gb_graph_reorder) and the end-to-end leg the file order.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from galois_b200 import (GB_CC_AFFOREST, GB_CC_LABELPROP, DeviceGraph, assign_weights_f32, assign_weights_u32,
                         erdos_renyi, grid2d, rmat)
from galois_b200 import _lib

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
ALPHA = 0.85


@pytest.fixture(scope="module")
def rmat24():
    g, _ = rmat(24, 16, seed=24, symmetrize=True)
    return g


@pytest.fixture(scope="module")
def rmat20():
    g, _ = rmat(20, 16, seed=20, symmetrize=True)
    return g


# ---- BFS ------------------------------------------------------------------------

@pytest.mark.parametrize("order", [0, 1])
def test_bfs_rmat20_config(cuda_device, rmat20, order):
    g = rmat20
    src = int(np.argmax(g.degrees()))
    want = oracle.bfs_serial(g, src)
    with DeviceGraph(g, symmetric=True, reorder=order) as dg:
        got, st = dg.bfs(src, stats=True)
    assert np.array_equal(got, want)
    assert st["vertices_reached"] == int((want != oracle.INF).sum())


def test_bfs_rmat24_config(cuda_device, rmat24):
    g = rmat24
    src = int(np.argmax(g.degrees()))
    want = oracle.bfs_serial(g, src)
    with DeviceGraph(g, symmetric=True, reorder=1) as dg:
        assert np.array_equal(dg.bfs(src), want)


# ---- SSSP -----------------------------------------------------------------------

@pytest.mark.parametrize("order", [0, 1])
def test_sssp_rmat22_config(cuda_device, order):
    g, perm = rmat(22, 16, seed=22, symmetrize=False)
    assign_weights_u32(g, 1, 255, seed=22)
    src = int(perm[0])
    want = oracle.sssp_dijkstra(g, src)
    with DeviceGraph(g, symmetric=False, reorder=order) as dg:
        got = dg.sssp(src, 13)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("order", [0, 1])
def test_sssp_grid4096_config(cuda_device, order):
    g = grid2d(4096, 4096)
    assign_weights_u32(g, 1, 255, seed=4096)
    want = oracle.sssp_dijkstra(g, 0)
    with DeviceGraph(g, symmetric=True, reorder=order) as dg:
        got = dg.sssp(0, 13)
    assert np.array_equal(got, want)


# ---- CC and PageRank on RMAT-24 ---------------------------------------------------

def test_cc_rmat24_config(cuda_device, rmat24):
    g = rmat24
    want = oracle.cc_union_find(g)
    for order in (0, 1):
        with DeviceGraph(g, symmetric=True, reorder=order) as dg:
            assert np.array_equal(dg.cc(GB_CC_LABELPROP), want), f"label propagation, order {order}"
            assert np.array_equal(dg.cc(GB_CC_AFFOREST), want), f"Afforest, order {order}"


def test_pagerank_pull_rmat24_config(cuda_device, rmat24):
    g = rmat24
    want, it64 = oracle.pr_pull_topo_f64(g, ALPHA, 1e-6, 1000)
    for order in (0, 1):
        with DeviceGraph(g, symmetric=True, reorder=order) as dg:
            got, st = dg.pagerank_pull(ALPHA, 1e-6, 1000, stats=True)
        assert np.abs(got - want).max() <= 1e-5, f"order {order}"
        assert abs(st["iterations"] - it64) <= 2, f"order {order}: {st['iterations']} vs {it64}"


def test_pagerank_pull_residual_rmat24_app_default(cuda_device, rmat24):
    """Pull-residual, the pull app's default (PageRank-pull.cpp:34-37), at its
    default tolerance 1e-3 on RMAT-24 against the FP64 restatement of the
    same rounds: every vertex within 1e-5 relative (absolute below 1) except
    rare threshold flips, which stay within 2 tol (the bound and its reason
    are check_residual_parity's in test_gpu_core.py), and the same number of
    rounds within 2; both vertex orders."""
    from test_gpu_core import check_residual_parity

    g = rmat24
    want, it64 = oracle.pr_pull_residual(g, ALPHA, 1e-3, 1000, f64=True)
    for order in (0, 1):
        with DeviceGraph(g, symmetric=True, reorder=order) as dg:
            got, st = dg.pagerank_pull_residual(ALPHA, 1e-3, 1000, stats=True)
        check_residual_parity(got, want, 1e-3, f"order {order}")
        assert abs(st["iterations"] - it64) <= 2, f"order {order}: {st['iterations']} vs {it64}"


# ---- Brandes BC -------------------------------------------------------------------

def test_bc_rmat20_1024_sources_config(cuda_device, rmat20):
    g = rmat20
    rng = np.random.default_rng(1024)
    srcs = rng.choice(np.flatnonzero(g.degrees() > 0), 1024, replace=False).astype(np.uint32)
    want = oracle.bc_level(g, srcs, f64=True, parallel=True)
    with DeviceGraph(g, symmetric=True) as dg:
        got = dg.bc(srcs, batch=64)
    err = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1.0)
    assert err.max() <= 1e-6, f"max relative error {err.max():.3e}"


# ---- many graphs in one launch ------------------------------------------------------

def test_multigraph_512_er_config(cuda_device):
    import torch

    from galois_b200.graph import pack_graphs

    rng = np.random.default_rng(512)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(200000), 512)).astype(int)
    graphs = [erdos_renyi(int(n), 8.0, seed=100 + i) for i, n in enumerate(sizes)]
    packed, first = pack_graphs(graphs)
    local = np.zeros(len(graphs), np.uint32)
    want_lv = np.concatenate([oracle.bfs_serial(gk, 0) for gk in graphs])
    want_lb = np.concatenate([oracle.cc_union_find(gk) for gk in graphs])
    with DeviceGraph(packed, symmetric=True) as dg:
        dg.autotune("bfs", int(first[0]))
        lv = torch.full((packed.n,), -1, dtype=torch.int32, device="cuda")
        lb = torch.full((packed.n,), -1, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            dg.multi_graph_bfs_cc(first, local, lv, lb)
            torch.cuda.synchronize()
            assert np.array_equal(lv.cpu().numpy().view(np.uint32), want_lv)
            assert np.array_equal(lb.cpu().numpy().view(np.uint32), want_lb)
            lv.fill_(-1)
            lb.fill_(-1)
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=s):
                dg.multi_graph_bfs_cc(first, local, lv, lb)
            cg.replay()
            torch.cuda.synchronize()
        assert np.array_equal(lv.cpu().numpy().view(np.uint32), want_lv)
        assert np.array_equal(lb.cpu().numpy().view(np.uint32), want_lb)
        del cg


# ---- personalised PageRank + adjoint ------------------------------------------------

def test_ppr_rmat22_batch128_config(cuda_device):
    import torch

    g, _ = rmat(22, 16, seed=22, symmetrize=False)
    assign_weights_f32(g, seed=22)
    B = 128
    rng = np.random.default_rng(128)
    T = torch.zeros((g.n, B), dtype=torch.float32, device="cuda")
    for b in range(B):
        T[torch.from_numpy(rng.choice(g.n, 32, replace=False)).cuda(), b] = 1.0 / 32
    c = torch.from_numpy(rng.standard_normal((g.n, B)).astype(np.float32)).cuda()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    with DeviceGraph(g) as dg:
        x = torch.empty_like(T)
        st = _lib.lib.gb_ppr_forward(dg.handle, B, C.c_void_p(T.data_ptr()), None, ALPHA, 1e-7, 1000,
                                     C.c_void_p(x.data_ptr()), None, None, s)
        assert st == _lib.GB_OK, _lib.last_error()
        gT = torch.empty_like(T)
        gw = torch.empty(g.m, dtype=torch.float32, device="cuda")
        st = _lib.lib.gb_ppr_backward(dg.handle, B, C.c_void_p(x.data_ptr()), C.c_void_p(c.data_ptr()), None,
                                      ALPHA, 1e-7, 1000, C.c_void_p(gT.data_ptr()), C.c_void_p(gw.data_ptr()),
                                      None, None, s)
        assert st == _lib.GB_OK, _lib.last_error()
        torch.cuda.synchronize()
    # two columns: forward and adjoint against FP64 solves of the same systems
    for b in (0, 77):
        rhs = (1 - ALPHA) * T[:, b].double().cpu().numpy()
        x_ref, _ = oracle.ppr_solve_f64(g, g.w_f32, rhs, ALPHA)
        xb = x[:, b].double().cpu().numpy()
        assert np.allclose(xb, x_ref, atol=1e-6, rtol=1e-4), f"forward column {b}"
        lam_ref, _ = oracle.ppr_solve_f64(g, g.w_f32, c[:, b].double().cpu().numpy(), ALPHA, adjoint=True)
        gt_ref = (1 - ALPHA) * lam_ref
        gtb = gT[:, b].double().cpu().numpy()
        assert np.abs(gtb - gt_ref).max() <= 1e-3 * np.abs(gt_ref).max(), f"teleport gradient column {b}"
    # edge-weight gradient: dL/dw_ji = alpha/s_j * sum_b x_j^b (lam_i^b - mu_j^b),
    # mu_j = (lam_j - gx_j)/alpha, from the GPU's own x and lam, in FP64
    srcs = np.repeat(np.arange(g.n, dtype=np.int64), g.degrees())
    arcs = rng.choice(g.m, 20000, replace=False)
    j = torch.from_numpy(srcs[arcs]).cuda()
    i = torch.from_numpy(g.col[arcs].astype(np.int64)).cuda()
    lam = gT.double() / (1 - ALPHA)
    mu_j = (lam[j] - c[j].double()) / ALPHA
    dots = (x[j].double() * (lam[i] - mu_j)).sum(dim=1).cpu().numpy()
    s_out = np.bincount(srcs, weights=g.w_f32.astype(np.float64), minlength=g.n)
    want = ALPHA / s_out[srcs[arcs]] * dots
    got = gw.cpu().numpy()[arcs].astype(np.float64)
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()
