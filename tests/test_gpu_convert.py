"""GPU: the graph-convert steps on the device mirror (gb_graph_symmetrize,
gb_graph_assign_weights_u32 / _f32) against the oracle's restatement of
makeSymmetric / Cleanup and against the host generators, bit-exact."""
import numpy as np
import pytest

import oracle
from galois_b200 import (GB_CC_LABELPROP, DeviceGraph, GbError, HostCSR, assign_weights_f32, assign_weights_u32,
                         rmat)
from galois_b200 import _lib

pytestmark = pytest.mark.gpu


def _multigraph(seed, n=300, m=4000):
    rng = np.random.default_rng(seed)
    return HostCSR.from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m), w_u32=rng.integers(1, 255, m))


@pytest.mark.parametrize("cleanup", [False, True])
@pytest.mark.parametrize("seed", [1, 2])
def test_symmetrize_matches_oracle(cuda_device, cleanup, seed):
    g = _multigraph(seed)
    want = oracle.make_symmetric(g, cleanup)
    with DeviceGraph(g) as dg:
        dg.symmetrize(cleanup=cleanup)
        assert dg.symmetric and dg.m == want[1].size
        end, col, w, wf = dg.to_host()
    assert np.array_equal(end, want[0])
    assert np.array_equal(col, want[1])
    assert np.array_equal(w, want[2])
    assert wf is None


def test_symmetrize_directed_rmat_then_run(cuda_device):
    gd, perm = rmat(13, 16, seed=21, symmetrize=False)
    gs, _ = rmat(13, 16, seed=21, symmetrize=True)
    src = int(perm[0])
    with DeviceGraph(gd) as dg:
        dg.symmetrize(cleanup=True)
        end, col, _, _ = dg.to_host()
        assert np.array_equal(end, gs.end_offs) and np.array_equal(col, gs.col)
        # the kernels see a symmetric graph: bottom-up BFS steps, LP CC
        assert (dg.bfs(src) == oracle.bfs_serial(gs, src)).all()
        assert (dg.cc(GB_CC_LABELPROP) == oracle.cc_union_find(gs)).all()
        dg.reorder()
        assert (dg.bfs(src) == oracle.bfs_serial(gs, src)).all()
        with pytest.raises(GbError) as e:
            dg.symmetrize()
        assert e.value.status == _lib.GB_ERR_UNSUPPORTED


def test_symmetrize_empty_and_self_loops_only(cuda_device):
    with DeviceGraph(HostCSR(np.zeros(3, np.uint64), np.zeros(0, np.uint32))) as dg:
        dg.symmetrize()
        end, col, _, _ = dg.to_host()
        assert end.tolist() == [0, 0, 0] and col.size == 0
    g = HostCSR.from_edges(3, [0, 1, 1], [0, 1, 1])
    for cleanup, m in ((False, 3), (True, 0)):
        with DeviceGraph(g) as dg:
            dg.symmetrize(cleanup=cleanup)
            assert dg.m == m


def test_device_weights_equal_host_generator(cuda_device):
    g, perm = rmat(12, 8, seed=3, symmetrize=False)
    src = int(perm[0])
    host = assign_weights_f32(assign_weights_u32(HostCSR(g.end_offs, g.col), 1, 255, seed=77), seed=78)
    with DeviceGraph(HostCSR(g.end_offs, g.col)) as dg:
        dg.assign_weights_u32(1, 255, 77)
        dg.assign_weights_f32(78)
        _, _, w, wf = dg.to_host()
        assert np.array_equal(w, host.w_u32)
        assert np.array_equal(wf.view(np.uint32), host.w_f32.view(np.uint32))
        # SSSP over the device-drawn weights
        assert (dg.sssp(src, 13) == oracle.sssp_dijkstra(host, src)).all()
        with pytest.raises(GbError):
            dg.assign_weights_u32(9, 3, 1)


def test_device_reference_weights_equal_converter_draws(cuda_device):
    """gb_graph_assign_weights_reference: the draws of gr2randomweightgr (a
    default std::mt19937 in arc order, graph-convert.cpp:1145-1190) on the
    device mirror, equal to the oracle's restatement; SSSP then runs on them."""
    g, perm = rmat(11, 8, seed=5, symmetrize=False)
    src = int(perm[0])
    with DeviceGraph(HostCSR(g.end_offs, g.col)) as dg:
        dg.assign_weights_reference(1, 100, "u32")
        dg.assign_weights_reference(1, 100, "f32")
        _, _, w, wf = dg.to_host()
        assert np.array_equal(w, oracle.gr2randomweight(g.m, 1, 100, "u32"))
        assert np.array_equal(wf.view(np.uint32), oracle.gr2randomweight(g.m, 1, 100, "f32").view(np.uint32))
        host = HostCSR(g.end_offs, g.col, w_u32=w)
        assert (dg.sssp(src, 13) == oracle.sssp_dijkstra(host, src)).all()
        dg.reorder()
        with pytest.raises(GbError) as e:
            dg.assign_weights_reference(1, 100)
        assert e.value.status == _lib.GB_ERR_UNSUPPORTED
