"""gb_bfs_noalloc: the allocation-free BFS entry point.

Callers that cannot call cudaMalloc (a host that owns and budgets all device
memory itself) pass their own device arrays; the library's scratch lives in a
fixed device array inside libgb.  This checks, through the C ABI, that two
calls in a row give exactly the levels of the regular gb_bfs entry point and
of the oracle's serial BFS (BFS levels are integers: the tolerance is zero),
that a directed graph run push-only matches the oracle, that an invalid CSR is
refused with GB_ERR_FORMAT before the levels are written, that host memory is
refused with GB_ERR_ARG, and that graphs beyond the array's limit are refused
with GB_ERR_CAPACITY before any device work.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from galois_b200 import DeviceGraph, rmat
from galois_b200 import _lib

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch

    offs = torch.from_numpy(g.offs.view(np.int64)).cuda()
    col = torch.from_numpy(g.col.view(np.int32)).cuda()
    return offs, col


def _noalloc(offs, col, n, m, symmetric, src, out):
    import torch

    st = _lib.lib.gb_bfs_noalloc(C.c_void_p(offs.data_ptr()), C.c_void_p(col.data_ptr()), n, m, symmetric, src,
                                 C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st


def test_noalloc_matches_gb_bfs_twice(cuda_device):
    import torch

    g, _ = rmat(15, 16, seed=5)
    deg = g.degrees()
    srcs = [int(np.argmax(deg)), int(np.flatnonzero(deg > 0)[-1])]
    offs, col = _device_csr(g)
    with DeviceGraph(g, symmetric=True) as dg:
        want = [dg.bfs(s) for s in srcs]
    for s, w in zip(srcs, want):
        assert np.array_equal(w, oracle.bfs_serial(g, s))
    out = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
    for s, w in zip(srcs, want):  # two calls in a row share the scratch array
        st = _noalloc(offs, col, g.n, g.m, 1, s, out)
        assert st == _lib.GB_OK, _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), w)
    # push-only (directed declaration) gives the same levels
    st = _noalloc(offs, col, g.n, g.m, 0, srcs[0], out)
    assert st == _lib.GB_OK, _lib.last_error()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want[0])


def test_noalloc_directed_push_only(cuda_device):
    import torch

    g, perm = rmat(14, 16, seed=6, symmetrize=False)
    offs, col = _device_csr(g)
    out = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
    for src in (int(perm[0]), int(np.argmax(g.degrees()))):
        st = _noalloc(offs, col, g.n, g.m, 0, src, out)
        assert st == _lib.GB_OK, _lib.last_error()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), oracle.bfs_serial(g, src))


def test_noalloc_rejects_invalid_csr_and_host_memory(cuda_device):
    import torch

    g, _ = rmat(10, 8, seed=2)
    offs, col = _device_csr(g)
    bad_col = col.clone()
    bad_col[g.m // 2] = g.n  # an id >= n
    out = torch.full((g.n,), -7, dtype=torch.int32, device="cuda")
    st = _noalloc(offs, bad_col, g.n, g.m, 1, 0, out)
    assert st == _lib.GB_ERR_FORMAT
    assert "invalid CSR" in _lib.last_error()
    assert (out.cpu() == -7).all()  # levels untouched
    bad_offs = offs.clone()
    bad_offs[5] = bad_offs[6] + 1  # offsets not monotone
    st = _noalloc(bad_offs, col, g.n, g.m, 1, 0, out)
    assert st == _lib.GB_ERR_FORMAT
    assert (out.cpu() == -7).all()
    host_out = torch.zeros(g.n, dtype=torch.int32)
    st = _noalloc(offs, col, g.n, g.m, 1, 0, host_out)
    assert st == _lib.GB_ERR_ARG
    assert "device memory" in _lib.last_error()


def test_noalloc_rejects_oversize_graph(cuda_device):
    import torch

    tiny = torch.zeros(4, dtype=torch.int64, device="cuda")
    st = _noalloc(tiny, tiny, (1 << 20) + 1, 8, 1, 0, tiny)
    assert st == _lib.GB_ERR_CAPACITY
    assert "exceeds the fixed scratch" in _lib.last_error()
