"""GPU parity for Brandes BC (single-source looped and multi-source batched)
against the CPU restatement of LevelStructs.h in FP64.

Tolerance: |gpu - fp64| <= 1e-6 * max(|fp64|, 1) per vertex.  The GPU keeps
sigma in fp64 and accumulates bc in fp64 but stores dependencies in fp32 as the
reference does, so each source contributes ~1e-7 relative rounding."""
import numpy as np
import pytest

import oracle
from galois_b200 import DeviceGraph, GbError, HostCSR, rmat
from galois_b200 import _lib

pytestmark = pytest.mark.gpu


def path_graph(n):
    s = list(range(n - 1)) + list(range(1, n))
    d = list(range(1, n)) + list(range(n - 1))
    return HostCSR.from_edges(n, s, d)


def close(got, want):
    scale = np.maximum(np.abs(want), 1.0)
    return float((np.abs(got.astype(np.float64) - want) / scale).max())


@pytest.mark.parametrize("batch", [1, 7, 64])
def test_bc_rmat_matches_fp64(cuda_device, batch):
    g, _ = rmat(12, 8, seed=9)
    rng = np.random.default_rng(1)
    srcs = rng.choice(np.flatnonzero(g.degrees() > 0), 70, replace=False).astype(np.uint32)
    want = oracle.bc_level(g, srcs, f64=True)
    with DeviceGraph(g, symmetric=True) as dg:
        got = dg.bc(srcs, batch=batch)
    assert close(got, want) < 1e-6


def test_bc_heavy_tiles_and_duplicates(cuda_device):
    g, _ = rmat(11, 16, seed=4)
    deg = g.degrees()
    hub = int(np.argmax(deg))
    srcs = np.array([hub, hub, 3, int(np.flatnonzero(deg == 0)[0]) if (deg == 0).any() else 5, 17], np.uint32)
    want = oracle.bc_level(g, srcs, f64=True)
    with DeviceGraph(g, symmetric=True) as dg:
        dg.set_tuning(heavy_degree=16, tile_edges=32)
        for batch in (1, 5):
            assert close(dg.bc(srcs, batch=batch), want) < 1e-6


def test_bc_path_closed_form(cuda_device):
    n = 40
    g = path_graph(n)
    with DeviceGraph(g, symmetric=True) as dg:
        for batch in (1, 40):
            got = dg.bc(np.arange(n), batch=batch)
            assert np.allclose(got, [2.0 * v * (n - 1 - v) for v in range(n)], rtol=1e-6)


def test_bc_directed_single_source_and_errors(cuda_device):
    g, perm = rmat(10, 8, seed=2, symmetrize=False)
    srcs = np.array([perm[0], perm[1], perm[2]], np.uint32)
    want = oracle.bc_level(g, srcs, f64=True)
    with DeviceGraph(g, symmetric=False) as dg:
        assert close(dg.bc(srcs, batch=1), want) < 1e-6
        with pytest.raises(GbError) as e:
            dg.bc(srcs, batch=3)
        assert e.value.status == _lib.GB_ERR_UNSUPPORTED
        with pytest.raises(GbError):
            dg.bc([g.n], batch=1)


def test_bc_sharded_single_rank_matches_plain(cuda_device):
    """galois_b200.distributed over a one-rank NCCL group equals plain gb_bc
    (the multi-rank split and sum are covered by the gloo tests)."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    from galois_b200.distributed import bc_sharded

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        g, _ = rmat(11, 8, seed=44)
        srcs = np.random.default_rng(5).choice(g.n, 100, replace=False).astype(np.uint32)
        with DeviceGraph(g, symmetric=True) as dg:
            want = dg.bc(srcs, batch=64)
            out = torch.empty(g.n, dtype=torch.float32, device="cuda")
            bc_sharded(dg, srcs, out, batch=64)
            assert np.abs(out.cpu().numpy() - want).max() <= 1e-6 * max(1.0, float(np.abs(want).max()))
    finally:
        dist.destroy_process_group()
