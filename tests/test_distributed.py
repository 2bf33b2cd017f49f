"""Multi-process plumbing of bench.py on CPU: two gloo ranks run the same
barrier / max-over-ranks timing path the NCCL ranks take, and the whole-job
rate is the units of all ranks over the slowest rank's time.  The multi-GPU
path has no data exchange (every rank runs its own replica of the workload),
so these host-side steps are all of it."""
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
        q.put((rank, d.world, got, wall, local))
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


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_aggregate_rate_is_whole_job(world):
    bench = _bench()
    # 1e9 units per rank per step, 4 steps, slowest rank 2 s -> world*2 G/s
    assert bench.aggregate_rate(world, 1e9, 4, 2000.0) == pytest.approx(2.0 * world)
