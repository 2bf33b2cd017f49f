"""Multi-process plumbing on CPU: two gloo ranks run the same barrier /
max-over-ranks timing path the NCCL ranks of bench.py take (the whole-job
rate is the units of all ranks over the slowest rank's time), and the
source-sharded BC (galois_b200.distributed) splits the sources without gaps
or overlap and sums the partial centralities with one all-reduce.  Every
other kernel runs one replica per GPU, with no data exchange."""
import importlib.util
import os
import socket
import time
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    bench = _bench()
    d = bench.Dist(want_pg=True, backend="gloo", timeout_s=60)
    try:
        # rank r "takes" 10*(r+1) ms; everyone must report the slowest
        t0 = time.perf_counter()
        d.barrier()
        time.sleep(0.01 * (rank + 1))
        d.barrier()
        local = (time.perf_counter() - t0) * 1e3
        got = d.max(float(10 * (rank + 1)))
        wall = d.max(local)
        total = d.sum(float(rank + 1))
        q.put((rank, d.world, got, wall, local, total))
    finally:
        d.close()


def test_dist_gloo_world2_max_and_barrier():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2, 2]
    assert all(r[2] == 20.0 for r in res)  # max over ranks, on every rank
    assert all(r[5] == 3.0 for r in res)  # sum over ranks, on every rank
    walls = {round(r[3], 9) for r in res}
    assert len(walls) == 1  # both ranks agree on one job time
    assert res[0][3] >= max(r[4] for r in res) - 1e-9
    # the second barrier holds the fast rank until the slow one arrives
    assert min(r[4] for r in res) >= 15.0


def test_dist_single_process_is_noop(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    d = _bench().Dist(want_pg=True, backend="gloo")
    assert (d.rank, d.world, d.pg) == (0, 1, False)
    d.barrier()
    assert d.max(3.5) == 3.5
    d.close()


class _FakeBcGraph:
    """Stands in for a DeviceGraph: source s contributes (1 + s) at vertex s
    and 1 at vertex 0, so the reduced vector identifies every source."""

    def __init__(self, n):
        self.n = n
        self.calls = []

    def bc(self, sources, batch, out):
        self.calls.append(list(map(int, sources)))
        out.zero_()
        for s in sources:
            out[int(s)] += 1.0 + float(s)
            out[0] += 1.0


def _bc_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    from galois_b200.distributed import bc_sharded

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 40
        sources = [3, 7, 11, 12, 20, 31, 33]
        g = _FakeBcGraph(n)
        out = torch.empty(n, dtype=torch.float32)
        bc_sharded(g, sources, out, batch=64)
        q.put((rank, g.calls, out.tolist()))
    finally:
        dist.destroy_process_group()


def test_bc_sources_sharded_and_reduced():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bc_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sources = [3, 7, 11, 12, 20, 31, 33]
    owned = [c for r in res for call in r[1] for c in call]
    assert sorted(owned) == sources  # every source exactly once
    assert all(len(r[1]) == 1 for r in res)  # one bc call per rank
    want = [0.0] * 40
    for s in sources:
        want[s] += 1.0 + s
    want[0] += len(sources)
    for r in res:
        assert r[2] == want  # every rank holds the full sum


def test_shard_sources_edges():
    from galois_b200.distributed import shard_sources

    src = list(range(10))
    parts = [shard_sources(src, r, 3).tolist() for r in range(3)]
    assert sorted(sum(parts, [])) == src
    assert shard_sources([], 0, 4).size == 0
    assert shard_sources(src, 3, 4).tolist() == [3, 7]  # more ranks than sources in a stride
    with pytest.raises(ValueError):
        shard_sources(src, 2, 2)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_aggregate_rate_is_whole_job(world):
    bench = _bench()
    # 1e9 units per rank per step, 4 steps, slowest rank 2 s -> world*2 G/s
    assert bench.aggregate_rate(world, 1e9, 4, 2000.0) == pytest.approx(2.0 * world)


def test_clock_sampler_merges_fast_samples():
    """Timed regions shorter than nvidia-smi's 200 ms period still get clock
    samples from the 1 ms NVML thread; idle-clock samples are left out of the
    median and any throttle reason seen is reported."""
    c = _bench().ClockSampler(0)
    c.start()
    c._nvml_rows += [(1965.0, 1965.0, (False, False, False, True)),
                     (1900.0, 1965.0, (False,) * 4), (210.0, 1965.0, (False,) * 4)]
    got = c.stop()
    assert got["sm_mhz"] == pytest.approx(1932.5)
    assert got["sm_max_mhz"] == 1965.0
    assert got["reasons"] == ["sw_power_cap"]
    assert got["samples_nvml"] >= 3


def test_shard_columns_blocks_of_four():
    from galois_b200.distributed import shard_columns

    for B in (4, 8, 128, 12):
        for world in (1, 2, 3, 4, 8):
            parts = [shard_columns(B, r, world) for r in range(world)]
            cols = [c for a, b in parts for c in range(a, b)]
            assert cols == list(range(B))  # contiguous, no gap, no overlap
            assert all((b - a) % 4 == 0 for a, b in parts)
    assert shard_columns(1, 0, 2) == (0, 1) and shard_columns(1, 1, 2) == (0, 0)
    assert shard_columns(128, 1, 2) == (64, 128)
    with pytest.raises(ValueError):
        shard_columns(6, 0, 2)


def _dense_ppr(graph, T, w, alpha, tol, max_iter):
    """Stand-in for the GPU solve on the host: the same system
    x = (1-alpha) T + alpha W~ x with W~_ij = w_ji / s_j, solved densely in
    FP64 by torch (differentiable in T and w)."""
    import torch

    src, dst = graph
    n = T.shape[0]
    s = torch.zeros(n, dtype=w.dtype).index_add(0, src, w)
    vals = w / s[src]
    W = torch.zeros((n, n), dtype=w.dtype).index_put((dst, src), vals, accumulate=True)
    A = torch.eye(n, dtype=w.dtype) - alpha * W
    return torch.linalg.solve(A, (1 - alpha) * T)


def _ppr_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    from galois_b200.distributed import ppr_sharded

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(3)
        n, m, B = 30, 120, 12
        src = torch.randint(0, n, (m,), generator=g)
        dst = torch.randint(0, n, (m,), generator=g)
        w = torch.rand(m, generator=g, dtype=torch.float64) + 0.1
        T = torch.rand((n, B), generator=g, dtype=torch.float64)
        c = torch.randn((n, B), generator=g, dtype=torch.float64)
        x, cols, gt, gw, loss = ppr_sharded((src, dst), T, w, c, solve=_dense_ppr)
        q.put((rank, cols, x.tolist(), gt.tolist(), gw.tolist(), float(loss)))
    finally:
        dist.destroy_process_group()


def test_ppr_columns_sharded_and_grad_w_reduced():
    """Two gloo ranks each solve half of the teleport columns; the all-reduced
    edge-weight gradient and the summed loss equal one process solving all
    columns, and the per-rank columns equal the matching columns of the
    whole solve."""
    import torch

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ppr_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = torch.Generator().manual_seed(3)
    n, m, B = 30, 120, 12
    src = torch.randint(0, n, (m,), generator=g)
    dst = torch.randint(0, n, (m,), generator=g)
    w = (torch.rand(m, generator=g, dtype=torch.float64) + 0.1).requires_grad_(True)
    T = torch.rand((n, B), generator=g, dtype=torch.float64).requires_grad_(True)
    c = torch.randn((n, B), generator=g, dtype=torch.float64)
    x = _dense_ppr((src, dst), T, w, 0.85, 0, 0)
    loss = (c * x).sum()
    loss.backward()
    assert [r[1] for r in res] == [(0, 4), (4, 12)] or [r[1] for r in res] == [(0, 8), (8, 12)]
    for rank, (b0, b1), xl, gtl, gw, tot in res:
        assert torch.allclose(torch.tensor(xl, dtype=torch.float64), x.detach()[:, b0:b1])
        assert torch.allclose(torch.tensor(gtl, dtype=torch.float64), T.grad[:, b0:b1])
        assert torch.allclose(torch.tensor(gw, dtype=torch.float64), w.grad)
        assert abs(tot - float(loss)) < 1e-9 * max(1.0, abs(float(loss)))
