"""Many disjoint graphs in one launch (gb_multi_graph_bfs_cc) against per-graph
CPU oracles, bit-exact; plus CUDA-graph capture and replay of the call."""
import numpy as np
import pytest

import oracle
from galois_b200 import DeviceGraph, GbError, erdos_renyi
from galois_b200 import _lib
from galois_b200.graph import pack_graphs

pytestmark = pytest.mark.gpu


def make_graphs(k, seed=0, lo=50, hi=3000):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), k)).astype(int)
    return [erdos_renyi(int(n), 8.0 if i % 3 else 1.5, seed=seed * 1000 + i) for i, n in enumerate(sizes)]


def expected(graphs, local_src):
    levels, labels = [], []
    for g, s in zip(graphs, local_src):
        levels.append(oracle.bfs_serial(g, int(s)))
        labels.append(oracle.cc_union_find(g))
    return np.concatenate(levels), np.concatenate(labels)


def test_multigraph_matches_per_graph_oracle(cuda_device):
    graphs = make_graphs(64, seed=3)
    packed, first = pack_graphs(graphs)
    rng = np.random.default_rng(5)
    local = np.array([rng.integers(0, g.n) for g in graphs], np.uint32)
    want_lv, want_lb = expected(graphs, local)
    with DeviceGraph(packed, symmetric=True) as dg:
        lv, lb = dg.multi_graph_bfs_cc(first, local)
        assert np.array_equal(lv, want_lv)
        assert np.array_equal(lb, want_lb)
        # a second layout on the same handle (validation cache refresh)
        local2 = np.zeros(len(graphs), np.uint32)
        lv2, _ = dg.multi_graph_bfs_cc(first, local2)
        assert np.array_equal(lv2, expected(graphs, local2)[0])


def test_multigraph_rejects_crossing_arcs_and_bad_sources(cuda_device):
    graphs = make_graphs(4, seed=1)
    packed, first = pack_graphs(graphs)
    bad_first = first.copy()
    bad_first[1] += 1  # vertex ranges no longer match the packing
    with DeviceGraph(packed, symmetric=True) as dg:
        with pytest.raises(GbError) as e:
            dg.multi_graph_bfs_cc(bad_first, np.zeros(4, np.uint32))
        assert e.value.status == _lib.GB_ERR_FORMAT
        with pytest.raises(GbError):
            dg.multi_graph_bfs_cc(first, np.array([0, 0, 0, graphs[3].n], np.uint32))


def test_multigraph_cuda_graph_replay(cuda_device):
    import torch

    graphs = make_graphs(32, seed=7)
    packed, first = pack_graphs(graphs)
    local = np.zeros(len(graphs), np.uint32)
    want_lv, want_lb = expected(graphs, local)
    with DeviceGraph(packed, symmetric=True) as dg:
        lv = torch.empty(packed.n, dtype=torch.int32, device="cuda")
        lb = torch.empty(packed.n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            dg.multi_graph_bfs_cc(first, local, lv, lb)  # warm-up: layout, workspace, schedule
            torch.cuda.synchronize()
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=s):
                dg.multi_graph_bfs_cc(first, local, lv, lb)
        lv.fill_(-1)
        lb.fill_(-1)
        for _ in range(3):
            cg.replay()
        torch.cuda.synchronize()
        assert np.array_equal(lv.cpu().numpy().view(np.uint32), want_lv)
        assert np.array_equal(lb.cpu().numpy().view(np.uint32), want_lb)
        del cg
