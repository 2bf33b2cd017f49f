"""Failure detection on the GPU without faulting it: the device waits the
persistent kernels rely on (the software grid barrier, a worklist ticket) are
run with a wait that nothing satisfies -- a CTA that never arrives, a chunk
that is never published -- and a short limit.  The wait must give up within
its limit, the call must return GB_ERR_TIMEOUT, and the context must stay
usable for the next computation."""
import time

import numpy as np
import pytest

import oracle
from galois_b200 import DeviceGraph, rmat
from galois_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_gives_up_and_context_survives(cuda_device, which):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = _lib.lib.gb_probe_bounded_waits(which, 20000, None)  # 20 ms limit
    elapsed = time.perf_counter() - t0
    assert st == _lib.GB_ERR_TIMEOUT, _lib.last_error()
    assert "gave up" in _lib.last_error()
    assert elapsed < 5.0
    # the context still computes correctly afterwards
    g, _ = rmat(10, 8, seed=3)
    src = int(np.argmax(g.degrees()))
    with DeviceGraph(g, symmetric=True) as dg:
        assert np.array_equal(dg.bfs(src), oracle.bfs_serial(g, src))


def test_bounded_wait_rejects_bad_arguments(cuda_device):
    assert _lib.lib.gb_probe_bounded_waits(2, 1000, None) == _lib.GB_ERR_ARG
    assert _lib.lib.gb_probe_bounded_waits(0, 0, None) == _lib.GB_ERR_ARG
    assert _lib.lib.gb_probe_bounded_waits(1, 3000000, None) == _lib.GB_ERR_ARG
