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
