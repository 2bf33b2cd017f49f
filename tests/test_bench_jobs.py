"""CPU: the bench jobs' CPU-side hooks, which the CPU baseline and the
`--impl reference` arm time (no GPU needed)."""
import importlib.util
from pathlib import Path

import numpy as np

import oracle

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_app_has_a_job_or_batched_runner():
    b = _bench()
    assert set(b.JOBS) == {"sssp", "bfs", "bfs-parent", "cc", "pr", "pr-residual"}
    assert set(b.BATCHED) == {"bc", "multigraph", "ppr"}


def test_cpu_run_units():
    from galois_b200 import rmat

    b = _bench()
    g, _ = rmat(10, 8, seed=3, symmetrize=True)
    # PageRank units are whole sweeps of the arcs (the parallel restatements
    # update in place, so their round count depends on the thread count)
    for cls in (b.PrJob, b.PrResidualJob):
        x, units = cls.__new__(cls).cpu_run(g)
        assert units > 0 and units % g.m == 0 and x.shape == (g.n,)
    lab, units = b.CcJob.__new__(b.CcJob).cpu_run(g)
    assert units == g.m and np.array_equal(lab, oracle.cc_union_find(g))


def test_bfs_parent_job_baseline_is_a_valid_tree():
    b = _bench()
    job = b.BfsParentJob("small")
    g = job.graphs[0]
    parents = job.cpu_call(0)
    lv = oracle.bfs_serial(g["host"], g["src"])
    assert oracle.verify_bfs_parent(g["host"], g["src"], lv, parents) == 0
    assert job.cpu_serial
