"""GPU: the python/galois-mirroring entry points over .gr files, the
autotuner, and the reference-facing .gr load path."""
import numpy as np
import pytest

import oracle
from galois_b200 import DeviceGraph, assign_weights_u32, rmat, write_gr

pytestmark = pytest.mark.gpu


@pytest.fixture()
def gr_files(tmp_path):
    g, perm = rmat(12, 8, seed=13, symmetrize=True)
    assign_weights_u32(g, 1, 255, seed=13)
    p_void = tmp_path / "g.sgr"
    p_w = tmp_path / "g_w.gr"
    write_gr(p_void, g, 0)
    write_gr(p_w, g, 4)
    return g, p_void, p_w


def test_python_bfs_sssp_cc(cuda_device, gr_files, capsys):
    from galois_b200.bfs import bfs
    from galois_b200.connected_components import connectedComponents
    from galois_b200.sssp import sssp

    g, p_void, p_w = gr_files
    src = int(np.argmax(g.degrees()))
    lv = bfs(4, src, str(p_void))
    want = oracle.bfs_serial(g, src)
    want[want == oracle.INF] = g.n  # the binding's infinity is numNodes (_bfs.pyx:42)
    assert np.array_equal(lv, want)
    assert "Node 1 has dist" in capsys.readouterr().out
    d = sssp(4, 13, src, str(p_w))
    wd = oracle.sssp_dijkstra(g, src)
    wd[wd == oracle.INF] = g.n
    assert np.array_equal(d, wd)
    assert np.array_equal(connectedComponents(4, str(p_void)), oracle.cc_union_find(g))


def test_python_pagerank_variant(cuda_device, gr_files):
    """_pagerank.pyx:86-139: rank starts at 1-alpha, base 1-alpha, stop when
    the MAX change <= 1e-3; compare with the converged fixed point of that
    iteration (unnormalised PageRank) within the stopping tolerance."""
    from galois_b200.pagerank import pagerank

    g, p_void, _ = gr_files
    r = pagerank(2, 1000, str(p_void)).astype(np.float64)
    nout = np.bincount(g.col, minlength=g.n).astype(np.float64)
    x = np.full(g.n, 0.15)
    offs = g.offs
    src = np.repeat(np.arange(g.n), g.degrees())
    for _ in range(300):
        c = np.where(nout > 0, x / np.maximum(nout, 1), 0.0)
        x = 0.15 + 0.85 * np.bincount(src, weights=c[g.col], minlength=g.n)
    assert np.abs(r - x).max() < 1e-2 * max(1.0, x.max())


def test_load_gr_and_autotune(cuda_device, gr_files, tmp_path):
    g, _, p_w = gr_files
    src = int(np.argmax(g.degrees()))
    dg = DeviceGraph.load_gr(str(p_w), edge_bytes=4, symmetric=True)
    try:
        cache = tmp_path / "tune.jsonl"
        best = dg.autotune("sssp", src, str(cache))
        assert cache.exists() and "sssp" in cache.read_text()
        assert (dg.sssp(src) == oracle.sssp_dijkstra(g, src)).all()
        best2 = dg.autotune("sssp", src, str(cache))  # served from the cache
        assert best2["heavy_degree"] == best["heavy_degree"] and best2["local_depth"] == best["local_depth"]
        for k in ("bfs", "cc", "pr"):
            dg.autotune(k, src, None)
        assert (dg.bfs(src) == oracle.bfs_serial(g, src)).all()
        assert (dg.cc() == oracle.cc_union_find(g)).all()
    finally:
        dg.free()


def test_pool_reuses_blocks_and_trims(cuda_device):
    """gb_graph_free caches the graph's device blocks for the next upload of
    the same shape; results stay right across reuse, and gb_pool_trim frees
    the cache."""
    from galois_b200 import _lib, rmat

    g, perm = rmat(12, 8, seed=91)
    want = oracle.bfs_serial(g, int(perm[0]))
    first = None
    for _ in range(3):
        with DeviceGraph(g, symmetric=True) as dg:
            ptrs = dg.device_arrays()
            if first is None:
                first = ptrs["col"]
            else:
                assert ptrs["col"] == first  # served from the cache
            assert (dg.bfs(int(perm[0])) == want).all()
    _lib.check(_lib.lib.gb_pool_trim(), "gb_pool_trim")
    with DeviceGraph(g, symmetric=True) as dg:  # a fresh allocation after the trim
        assert (dg.bfs(int(perm[0])) == want).all()


def test_upload_overlaps_another_graphs_kernel(cuda_device):
    """gb_graph_upload copies host arrays on a stream of the library's own, so
    a graph can be uploaded while another graph's kernel runs asynchronously
    into a device buffer; both results stay exact."""
    import torch

    from galois_b200 import grid2d

    ga = grid2d(512, 512)
    assign_weights_u32(ga, 1, 255, seed=5)
    want_a = oracle.sssp_dijkstra(ga, 0)
    gb, perm = rmat(14, 8, seed=6, symmetrize=True)
    src = int(perm[0])
    want_b = oracle.bfs_serial(gb, src)
    with DeviceGraph(ga, symmetric=True) as da:
        out_a = torch.empty(ga.n, dtype=torch.int32, device="cuda")
        da.sssp(0, 13, out=out_a)  # queued on torch's stream, not waited for
        with DeviceGraph(gb, symmetric=True) as db:  # uploaded meanwhile
            lev_b = db.bfs(src)
        torch.cuda.current_stream().synchronize()
        assert (out_a.cpu().numpy().view(np.uint32) == want_a).all()
        assert (lev_b == want_b).all()


def test_upload_from_device_arrays_waits_for_queued_writes(cuda_device):
    """Device inputs are copied on the default stream, after the work queued
    before the call: arrays whose writes are still queued behind a long
    kernel on torch's stream upload complete."""
    import ctypes as C

    import torch

    from galois_b200 import _lib

    g, perm = rmat(14, 8, seed=7, symmetrize=True)
    src = int(perm[0])
    want = oracle.bfs_serial(g, src)
    end_h = torch.from_numpy(g.end_offs.astype(np.int64)).pin_memory()
    col_h = torch.from_numpy(g.col.view(np.int32).copy()).pin_memory()
    end_d = torch.zeros(g.n, dtype=torch.int64, device="cuda")
    col_d = torch.zeros(g.m, dtype=torch.int32, device="cuda")
    x = torch.randn(2048, 2048, device="cuda")
    for _ in range(8):  # keep torch's stream busy before the writes
        x = torch.tanh(x @ x)
    end_d.copy_(end_h, non_blocking=True)
    col_d.copy_(col_h, non_blocking=True)
    handle = C.c_void_p()
    _lib.check(_lib.lib.gb_graph_upload(C.c_void_p(end_d.data_ptr()), C.c_void_p(col_d.data_ptr()), None, None,
                                        g.n, g.m, 1, 0, C.byref(handle)), "gb_graph_upload")
    try:
        lev = np.empty(g.n, np.uint32)
        _lib.check(_lib.lib.gb_bfs(handle, src, C.c_void_p(lev.ctypes.data), None, None), "gb_bfs")
        assert (lev == want).all()
    finally:
        _lib.lib.gb_graph_free(handle)
    assert torch.isfinite(x).all()
