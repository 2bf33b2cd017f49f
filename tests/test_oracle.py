"""Pins the CPU oracle: closed-form known answers, the reference's verifiers,
and agreement between independent restatements.  CPU only."""
import numpy as np
import pytest

import oracle
from galois_b200 import HostCSR, assign_weights_u32, erdos_renyi, grid2d, rmat

INF = oracle.INF


def path_graph(n, directed=False):
    src = list(range(n - 1))
    dst = list(range(1, n))
    if not directed:
        src, dst = src + dst, dst + src
    return HostCSR.from_edges(n, src, dst)


def star_graph(k):
    src = [0] * k + list(range(1, k + 1))
    dst = list(range(1, k + 1)) + [0] * k
    return HostCSR.from_edges(k + 1, src, dst)


def clique(k, offset=0, n=None):
    s, d = [], []
    for i in range(k):
        for j in range(k):
            if i != j:
                s.append(offset + i)
                d.append(offset + j)
    return s, d


def test_bfs_path_levels():
    g = path_graph(50)
    lv = oracle.bfs_serial(g, 0)
    assert lv.tolist() == list(range(50))
    assert oracle.bfs_sync_tile(g, 0).tolist() == list(range(50))
    assert oracle.verify_bfs(g, 0, lv) == 0


def test_bfs_directed_unreachable():
    g = path_graph(10, directed=True)
    lv = oracle.bfs_serial(g, 5)
    assert lv[:5].tolist() == [INF] * 5
    assert lv[5:].tolist() == list(range(5))


def test_bfs_star_and_isolated():
    g = star_graph(300)  # centre degree 300 > edge tile 256
    lv = oracle.bfs_sync_tile(g, 0)
    assert lv[0] == 0 and (lv[1:] == 1).all()
    lv = oracle.bfs_sync_tile(g, 7)
    assert lv[7] == 0 and lv[0] == 1 and lv[1] == 2


def test_bfs_parents_known_answers():
    # path: every vertex's parent is its predecessor, the source's datum is 0
    g = path_graph(40)
    lv = oracle.bfs_serial(g, 10)
    want = [v + 1 for v in range(10)] + [0] + [v - 1 for v in range(11, 40)]
    assert oracle.bfs_parent_min(g, 10, lv).tolist() == want
    assert oracle.bfs_do_parent(g, 10).tolist() == want
    # star from a leaf: the centre's parent is the leaf, other leaves' the centre
    g = star_graph(300)
    lv = oracle.bfs_serial(g, 7)
    for pa in (oracle.bfs_parent_min(g, 7, lv), oracle.bfs_do_parent(g, 7)):
        assert pa[7] == 0 and pa[0] == 7
        assert (np.delete(pa, [0, 7]) == 0).all()
    # directed path: vertices before the source stay unreached
    g = path_graph(10, directed=True)
    pa = oracle.bfs_do_parent(g, 4)
    assert pa[:4].tolist() == [INF] * 4 and pa[4] == 0 and pa[5:].tolist() == [4, 5, 6, 7, 8]


@pytest.mark.parametrize("sym", [True, False])
def test_bfs_parents_restatements_are_trees(sym):
    g, perm = rmat(12, 8, seed=5, symmetrize=sym)
    src = int(perm[0])
    lv = oracle.bfs_serial(g, src)
    do = oracle.bfs_do_parent(g, src)
    pm = oracle.bfs_parent_min(g, src, lv)
    assert oracle.verify_bfs_parent(g, src, lv, do) == 0
    assert oracle.verify_bfs_parent(g, src, lv, pm) == 0
    assert ((do == INF) == (lv == INF)).all()
    # the min rule is a lower bound of every valid choice
    reached = (lv != INF) & (np.arange(g.n) != src)
    assert (pm[reached] <= do[reached]).all()


def test_bfs_parent_verifier_catches_planted_mistakes():
    g, perm = rmat(10, 8, seed=6)
    src = int(perm[0])
    lv = oracle.bfs_serial(g, src)
    pa = oracle.bfs_parent_min(g, src, lv)
    v = int(np.flatnonzero((lv != INF) & (lv >= 2))[0])
    bad = pa.copy(); bad[src] = 1
    assert oracle.verify_bfs_parent(g, src, lv, bad) == 1
    unreached = np.flatnonzero(lv == INF)
    if unreached.size:
        bad = pa.copy(); bad[unreached[0]] = src
        assert oracle.verify_bfs_parent(g, src, lv, bad) == 2
    bad = pa.copy(); bad[v] = src  # the source is two or more levels up
    assert oracle.verify_bfs_parent(g, src, lv, bad) == 3


def _rows(end, col, w):
    out, b = [], 0
    for e in end:
        out.append(sorted(zip(col[b:e].tolist(), [] if w is None else w[b:e].tolist()) if w is not None
                          else col[b:e].tolist()))
        b = int(e)
    return out


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_make_symmetric_rows_match_reference_order(seed):
    # random multigraph with self-loops: the sorted device form holds, row by
    # row, the same arcs and weights as makeSymmetric's append order
    rng = np.random.default_rng(seed)
    n, m = 40, 300
    g = HostCSR.from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m), w_u32=rng.integers(1, 9, m))
    ref = oracle.make_symmetric_file_order(g)
    got = oracle.make_symmetric(g, cleanup=False)
    assert np.array_equal(ref[0], got[0])
    assert _rows(*ref) == _rows(*got)
    loops = int((np.repeat(np.arange(n), g.degrees()) == g.col).sum())
    assert got[1].size == 2 * m - loops


def test_make_symmetric_cleanup_known_answers():
    g = HostCSR.from_edges(4, [0, 0, 1, 2, 3, 3], [1, 1, 1, 3, 2, 0], w_u32=[5, 6, 7, 8, 9, 4])
    end, col, w = oracle.make_symmetric(g, cleanup=True)
    # 0-1 once (first copy, weight 5), self-loop 1-1 gone, 3-0 once (weight
    # 4); 2-3 and 3-2 are both stored arcs, so each row keeps its own
    # forward copy (8 in row 2, 9 in row 3) over the other's reverse copy
    assert end.tolist() == [2, 3, 4, 6]
    assert col.tolist() == [1, 3, 0, 3, 0, 2]
    assert w.tolist() == [5, 4, 5, 8, 4, 9]
    # symmetrising the directed generator output gives the symmetric one
    gd, _ = rmat(10, 8, seed=4, symmetrize=False)
    gs, _ = rmat(10, 8, seed=4, symmetrize=True)
    end, col, _ = oracle.make_symmetric(gd, cleanup=True)
    assert np.array_equal(end, gs.end_offs) and np.array_equal(col, gs.col)


def test_grid_unit_distances_are_manhattan():
    r, c = 17, 23
    g = grid2d(r, c)
    g.w_u32 = np.ones(g.m, np.uint32)
    d = oracle.sssp_dijkstra(g, 0).reshape(r, c)
    ii, jj = np.meshgrid(np.arange(r), np.arange(c), indexing="ij")
    assert (d == ii + jj).all()
    assert (oracle.bfs_serial(g, 0).reshape(r, c) == ii + jj).all()


def test_sssp_formulations_agree():
    g, perm = rmat(11, 8, seed=5, symmetrize=False)
    assign_weights_u32(g, 1, 255, seed=9)
    src = int(perm[0])  # the generator's vertex 0 (the RMAT hub) after relabelling
    ref = oracle.sssp_dijkstra(g, src)
    assert (ref != INF).sum() > g.n // 4
    for shift in (0, 4, 13):
        assert (oracle.sssp_delta_serial(g, src, shift) == ref).all()
        assert (oracle.sssp_delta_parallel(g, src, shift) == ref).all()
    assert oracle.verify_sssp(g, src, ref) == 0
    bad = ref.copy()
    reached = np.flatnonzero((bad != INF) & (np.arange(g.n) != src))
    bad[reached[0]] += 1  # not tight any more
    assert oracle.verify_sssp(g, src, bad) != 0


def test_bfs_formulations_agree_rmat():
    g, _ = rmat(12, 16, seed=2)
    src = int(np.argmax(g.degrees()))
    a = oracle.bfs_serial(g, src)
    assert (oracle.bfs_sync_tile(g, src) == a).all()
    assert oracle.verify_bfs(g, src, a) == 0


def test_cc_min_labels_cliques():
    s, d = [], []
    for off, k in ((0, 5), (5, 3), (9, 7)):
        a, b = clique(k, off)
        s += a
        d += b
    g = HostCSR.from_edges(20, s, d)  # vertices 8 and 16..19 isolated
    lab = oracle.cc_union_find(g)
    want = [0] * 5 + [5] * 3 + [8] + [9] * 7 + [16, 17, 18, 19]
    assert lab.tolist() == want
    lp, rounds = oracle.cc_labelprop(g)
    assert lp.tolist() == want and rounds >= 2
    assert oracle.verify_cc(g, lab) == 0


def test_cc_formulations_agree_er():
    g = erdos_renyi(5000, 1.2, seed=4)  # many components near the threshold
    a = oracle.cc_union_find(g)
    b, _ = oracle.cc_labelprop(g)
    assert (a == b).all()
    assert (a <= np.arange(g.n)).all()


def test_pagerank_cycle_uniform():
    n = 64
    g = HostCSR.from_edges(n, list(range(n)), [(i + 1) % n for i in range(n)])
    r, it = oracle.pr_pull_topo_f64(g, 0.85, 1e-12, 1000)
    assert np.allclose(r, 1.0 / n, atol=1e-15) and it == 1


def test_pagerank_f32_inplace_close_to_f64():
    g, _ = rmat(11, 8, seed=7)
    r64, it64 = oracle.pr_pull_topo_f64(g, 0.85, 1e-6, 1000)
    r32, it32 = oracle.pr_pull_topo_f32_inplace(g, 0.85, 1e-6, 1000)
    assert np.abs(r32 - r64).max() < 1e-5
    rp, _ = oracle.pr_pull_topo_par(g, 0.85, 1e-6, 1000)
    assert np.abs(rp - r64).max() < 1e-5


def test_pagerank_push_and_residual_close_to_solution():
    g, _ = rmat(10, 8, seed=11)
    # unnormalised fixed point x = (1-a) + a * A^T (x / outdeg), dense solve
    n = g.n
    A = np.zeros((n, n))
    deg = g.degrees()
    offs = g.offs
    for v in range(n):
        for i in range(offs[v], offs[v + 1]):
            A[g.col[i], v] += 0.85 / deg[v]
    x = np.linalg.solve(np.eye(n) - A, np.full(n, 0.15))
    xp, _ = oracle.pr_push_sync(g, 0.85, 1e-6, 1000)
    assert np.abs(xp - x).max() < 1e-3
    # pull-residual over the transpose computes the same fixed point
    xr, _ = oracle.pr_pull_residual(g, 0.85, 1e-6, 1000)  # g symmetric: its own transpose
    assert np.abs(xr - x).max() < 1e-3


def test_bc_path_closed_form():
    n = 12
    g = path_graph(n)
    bc = oracle.bc_level(g, [0])
    want = [0.0] + [float(n - 1 - v) for v in range(1, n - 1)] + [0.0]
    assert np.allclose(bc, want)
    allsrc = oracle.bc_level_f64_all = oracle.bc_level(g, range(n), f64=True)
    want_all = [2.0 * v * (n - 1 - v) for v in range(n)]
    assert np.allclose(allsrc, want_all)


def test_bc_star_closed_form():
    k = 9
    g = star_graph(k)
    bc = oracle.bc_level(g, range(k + 1), f64=True)
    assert bc[0] == pytest.approx(k * (k - 1))
    assert np.allclose(bc[1:], 0)


def test_bc_variants_agree():
    g, _ = rmat(10, 8, seed=13)
    rng = np.random.default_rng(0)
    srcs = rng.choice(np.flatnonzero(g.degrees() > 0), 16, replace=False)
    b64 = oracle.bc_level(g, srcs, f64=True)
    b32 = oracle.bc_level(g, srcs)
    bp = oracle.bc_level(g, srcs, parallel=True)
    scale = np.maximum(np.abs(b64), 1.0)
    assert (np.abs(b32 - b64) / scale).max() < 1e-5
    assert (np.abs(bp - b64) / scale).max() < 1e-5
