"""Relabelling (gb_graph_reorder: degree order, and the locality order of
landmark distances): every algorithm keeps taking and returning original
vertex ids, so the results match the oracle exactly (BFS/SSSP/CC) or within
the stated tolerance (PageRank, BC), for host and device outputs, sorted and
unsorted rows, symmetric and directed graphs."""
import numpy as np
import pytest
import torch

import oracle
from galois_b200 import (GB_CC_AFFOREST, GB_CC_LABELPROP, GB_CC_UNIONFIND, GB_ORDER_DEGREE,
                         GB_ORDER_DEGREE_UNSORTED, GB_ORDER_NONE, DeviceGraph, GbError, HostCSR,
                         assign_weights_f32, assign_weights_u32, grid2d, rmat)
from galois_b200 import _lib
from galois_b200._lib import GB_ORDER_LOCALITY
from galois_b200.graph import pack_graphs

pytestmark = pytest.mark.gpu
INF = oracle.INF
ORDERS = [GB_ORDER_DEGREE, GB_ORDER_DEGREE_UNSORTED]


def _dev(n, dtype=torch.int32):
    return torch.full((n,), -7, dtype=dtype, device="cuda")


@pytest.mark.parametrize("order", ORDERS)
def test_bfs_reordered(cuda_device, order):
    g, perm = rmat(14, 16, seed=31)
    deg = g.degrees()
    srcs = [int(np.argmax(deg)), int(perm[5]), int(np.flatnonzero(deg == 0)[0]) if (deg == 0).any() else 3]
    with DeviceGraph(g, symmetric=True, reorder=order) as dg:
        for src in srcs:
            want = oracle.bfs_serial(g, src)
            assert (dg.bfs(src) == want).all()
            out = _dev(g.n)
            dg.bfs(src, out=out)
            assert (out.cpu().numpy().view(np.uint32) == want).all()
        dg.set_tuning(direction_opt=2)
        assert (dg.bfs(srcs[0]) == oracle.bfs_serial(g, srcs[0])).all()


@pytest.mark.parametrize("order", ORDERS)
def test_sssp_reordered_directed(cuda_device, order):
    g, perm = rmat(14, 8, seed=32, symmetrize=False)
    assign_weights_u32(g, 1, 255, seed=5)
    src = int(perm[0])
    want = oracle.sssp_dijkstra(g, src)
    with DeviceGraph(g, reorder=order) as dg:
        got, st = dg.sssp(src, 13, stats=True)
        assert (got == want).all()
        assert st["vertices_reached"] == int((want != INF).sum())
        out = _dev(g.n)
        dg.sssp(src, 4, out=out)
        assert (out.cpu().numpy().view(np.uint32) == want).all()


def test_sssp_reordered_grid(cuda_device):
    g = grid2d(64, 80)
    assign_weights_u32(g, 1, 255, seed=9)
    want = oracle.sssp_dijkstra(g, 77)
    with DeviceGraph(g, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        assert (dg.sssp(77, 6) == want).all()


@pytest.mark.parametrize("algo", [GB_CC_LABELPROP, GB_CC_UNIONFIND, GB_CC_AFFOREST])
@pytest.mark.parametrize("order", ORDERS)
def test_cc_reordered_min_original_label(cuda_device, algo, order):
    # RMAT plus a few isolated / small pieces: labels must be the min ORIGINAL id
    g, _ = rmat(13, 4, seed=33)
    want = oracle.cc_union_find(g)
    with DeviceGraph(g, symmetric=True, reorder=order) as dg:
        assert (dg.cc(algo) == want).all()
        out = _dev(g.n)
        dg.cc(algo, out=out)
        assert (out.cpu().numpy().view(np.uint32) == want).all()


@pytest.mark.parametrize("order", ORDERS)
def test_pagerank_reordered(cuda_device, order):
    g, _ = rmat(13, 16, seed=34)
    want, _ = oracle.pr_pull_topo_f64(g, 0.85, 1e-6, 1000)
    with DeviceGraph(g, symmetric=True, reorder=order) as dg:
        got, info = dg.pagerank_pull(0.85, 1e-6, 1000, stats=True)
        assert np.max(np.abs(got.astype(np.float64) - want)) <= 1e-5
        out = _dev(g.n, torch.float32)
        dg.pagerank_pull(0.85, 1e-6, 1000, out=out)
        assert np.max(np.abs(out.cpu().numpy().astype(np.float64) - want)) <= 1e-5
        # residual variants against their own oracles; leftover residuals below
        # tol 1e-4 flow onward with gain alpha/(1-alpha): 2e-3 absolute
        r, _ = oracle.pr_pull_residual(g, 0.85, 1e-4, 1000)
        assert np.max(np.abs(dg.pagerank_pull_residual(0.85, 1e-4, 1000).astype(np.float64) - r)) < 2e-3
        p, _ = oracle.pr_push_sync(g, 0.85, 1e-4, 1000)
        assert np.max(np.abs(dg.pagerank_push(0.85, 1e-4, 1000).astype(np.float64) - p)) < 2e-3


def test_pagerank_reordered_not_converged_still_maps(cuda_device):
    g, _ = rmat(12, 8, seed=35)
    with DeviceGraph(g, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        got, info = dg.pagerank_pull(0.85, 0.0, 3, stats=True)
        assert not info["converged"] and info["iterations"] == 3
        with DeviceGraph(g, symmetric=True) as plain:
            ref = plain.pagerank_pull(0.85, 0.0, 3)
        assert np.max(np.abs(got - ref)) <= 1e-6


@pytest.mark.parametrize("batch", [1, 64])
def test_bc_reordered(cuda_device, batch):
    g, _ = rmat(11, 8, seed=36)
    srcs = [int(s) for s in np.random.default_rng(3).choice(g.n, 70, replace=False)]
    want = oracle.bc_level(g, srcs, f64=True)
    with DeviceGraph(g, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        got = dg.bc(srcs, batch=batch).astype(np.float64)
    assert np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))) <= 1e-5


def test_reorder_edge_cases(cuda_device):
    # single vertex, no arcs
    g1 = HostCSR.from_edges(1, [], [])
    with DeviceGraph(g1, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        assert dg.bfs(0).tolist() == [0]
        assert dg.cc().tolist() == [0]
    # path whose ids run against degree order
    n = 50
    s = list(range(n - 1)) + list(range(1, n))
    d = list(range(1, n)) + list(range(n - 1))
    gp = HostCSR.from_edges(n, s, d)
    with DeviceGraph(gp, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        assert (dg.bfs(0) == np.arange(n)).all()
        assert (dg.cc() == 0).all()


def test_reorder_api_contract(cuda_device):
    g, _ = rmat(10, 8, seed=37)
    assign_weights_f32(g, seed=1)
    packed, first = pack_graphs([g, g])
    with DeviceGraph(g, symmetric=True) as dg:
        assert dg.permutation() == {"new_to_old": None, "old_to_new": None}
        dg.reorder(GB_ORDER_NONE)  # no-op on file order
        dg.reorder(GB_ORDER_DEGREE)
        p = dg.permutation()
        assert p["new_to_old"] and p["old_to_new"]
        dg.reorder(GB_ORDER_DEGREE)  # same order again: no-op
        for bad in (GB_ORDER_NONE, GB_ORDER_DEGREE_UNSORTED):
            with pytest.raises(GbError) as e:
                dg.reorder(bad)
            assert e.value.status == _lib.GB_ERR_UNSUPPORTED
        with pytest.raises(GbError) as e:
            dg.reorder(7)
        # PPR needs file order
        from galois_b200.ppr import ppr

        T = torch.zeros((g.n, 4), dtype=torch.float32, device="cuda")
        T[0] = 1.0
        with pytest.raises(GbError) as e:
            ppr(dg, T, torch.from_numpy(g.w_f32).cuda())
        assert e.value.status == _lib.GB_ERR_UNSUPPORTED
    with DeviceGraph(packed, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        with pytest.raises(GbError) as e:
            dg.multi_graph_bfs_cc(first, np.zeros(2, np.uint32))
        assert e.value.status == _lib.GB_ERR_UNSUPPORTED


def test_autotune_on_reordered(cuda_device, tmp_path):
    g, perm = rmat(12, 16, seed=38)
    src = int(perm[0])
    with DeviceGraph(g, symmetric=True, reorder=GB_ORDER_DEGREE) as dg:
        dg.autotune("bfs", src, str(tmp_path / "tune.jsonl"))
        assert (dg.bfs(src) == oracle.bfs_serial(g, src)).all()


def _perm_host(dg):
    """new_to_old of a relabelled graph, copied to the host."""
    ptr = dg.permutation()["new_to_old"]

    class _View:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (dg.n,), "typestr": "<i4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_View(), device="cuda").cpu().numpy().view(np.uint32)


def test_locality_order_all_algorithms(cuda_device):
    """GB_ORDER_LOCALITY on a grid with a detached path (a second component,
    out of the landmarks' reach) and on an RMAT graph: BFS, SSSP (both
    kernels), CC, PageRank pull and residual push in original ids, and the
    permutation a bijection that keeps grid neighbours close."""
    grid = grid2d(60, 70)
    path_s = list(range(4199 + 1, 4199 + 30)) + list(range(4199 + 2, 4199 + 31))
    path_d = list(range(4199 + 2, 4199 + 31)) + list(range(4199 + 1, 4199 + 30))
    ends = np.concatenate([grid.end_offs, np.full(31, grid.m, np.uint64)])
    g = HostCSR(ends, grid.col)
    extra = HostCSR.from_edges(g.n, path_s, path_d)
    s_all = np.concatenate([np.repeat(np.arange(g.n), g.degrees()), np.repeat(np.arange(g.n), extra.degrees())])
    d_all = np.concatenate([g.col, extra.col])
    g = HostCSR.from_edges(g.n, s_all, d_all)
    assign_weights_u32(g, 1, 255, seed=11)
    r, _ = rmat(12, 8, seed=13)
    assign_weights_u32(r, 1, 255, seed=13)
    for h in (g, r):
        srcs = [0, int(np.argmax(h.degrees()))]
        with DeviceGraph(h, symmetric=True, reorder=GB_ORDER_LOCALITY) as dg:
            new_to_old = _perm_host(dg)
            assert np.array_equal(np.sort(new_to_old), np.arange(h.n))
            for src in srcs:
                assert (dg.bfs(src) == oracle.bfs_serial(h, src)).all()
                want = oracle.sssp_dijkstra(h, src)
                for mode in (0, 1, -1):
                    dg.set_tuning(sssp_async=mode)
                    assert (dg.sssp(src, 13) == want).all(), (h.n, src, mode)
            assert (dg.cc(GB_CC_LABELPROP) == oracle.cc_union_find(h)).all()
            want_pr, it64 = oracle.pr_pull_topo_f64(h, 0.85, 1e-6, 1000)
            got_pr, st = dg.pagerank_pull(0.85, 1e-6, 1000, stats=True)
            assert np.abs(got_pr - want_pr).max() < 1e-5 and abs(st["iterations"] - it64) <= 2
    # on the grid, ids that are consecutive in the new order are close on the grid
    with DeviceGraph(grid, symmetric=True, reorder=GB_ORDER_LOCALITY) as dg:
        old = _perm_host(dg).astype(np.int64)
    rows, cols = old // 70, old % 70
    hop = np.abs(np.diff(rows)) + np.abs(np.diff(cols))
    assert np.median(hop) <= 2


def test_auto_order_and_default_region_kernel(cuda_device):
    """GB_ORDER_AUTO numbers a bounded-degree grid by locality and an RMAT
    graph by degree; on the locality-ordered grid the default SSSP takes the
    shared-memory region kernel (its statistics report shared-memory rounds),
    sssp_async = -1 the phase-synchronous one; both exact, several sources,
    a bucket width of 1 and of 2^13."""
    from galois_b200 import GB_ORDER_AUTO
    g = grid2d(180, 200)
    assign_weights_u32(g, 1, 255, seed=5)
    r, _ = rmat(12, 8, seed=3)
    with DeviceGraph(r, symmetric=True, reorder=GB_ORDER_AUTO) as dg:
        assert dg.order == GB_ORDER_DEGREE
    with DeviceGraph(g, symmetric=True) as dg:
        assert dg.order == GB_ORDER_NONE
        dg.reorder(GB_ORDER_AUTO)
        assert dg.order == GB_ORDER_LOCALITY
        for src in (0, 17999, 35999):
            for shift in (13, 0):
                want = oracle.sssp_dijkstra(g, src)
                got, st = dg.sssp(src, shift, stats=True)
                assert (got == want).all() and st["pull_rounds"] > 0, (src, shift)
                dg.set_tuning(sssp_async=-1)
                got, st = dg.sssp(src, shift, stats=True)
                assert (got == want).all() and st["pull_rounds"] == 0, (src, shift)
                dg.set_tuning(sssp_async=0)
