#!/usr/bin/env python3
"""Benchmark of the CSR edge-map path on B200.

Default workload (no --app): delta-stepping SSSP, delta = 2^13, uint32 weights
uniform in [1,255], on (a) a directed RMAT scale-22 graph (edge factor 16,
a/b/c = 0.57/0.19/0.19, seeded relabelling; source = the generator's vertex 0)
and (b) the 4096x4096 4-neighbour grid (source 0).  One step = one full SSSP
on each graph.  Metric: GTEPS = (m_r(a) + m_r(b)) / step time, m_r = arcs out
of reached vertices.  Other --app values run the other hot-path kernels on
their configurations (bfs: RMAT-20 sym; cc, pr: RMAT-24 sym).

Prints ONE JSON line (rank 0).  `--impl reference` times the CPU restatement of
the reference algorithm (oracle/, OpenMP on all host cores) on the same
workload instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--app", choices=["sssp", "bfs", "cc", "pr"], default="sssp")
    ap.add_argument("--small", action="store_true", help="reduced sizes (profiling / smoke only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------- plumbing --
class Dist:
    """torch.distributed over NCCL when launched by torchrun, else a no-op."""

    def __init__(self, want_pg: bool):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1 and want_pg:
            import datetime

            import torch
            import torch.distributed as dist

            torch.cuda.set_device(self.local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", self.local_rank))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi samples (200 ms) of the SM clock and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def traffic_from_profiles(key: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(p.read_text()).get(key)
    except Exception:
        return None


def pinned_copy(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory (for the end-to-end leg)."""
    import torch

    tdt = {np.dtype(np.uint32): torch.int32, np.dtype(np.uint64): torch.int64,
           np.dtype(np.float32): torch.float32}[a.dtype]
    t = torch.empty(a.size, dtype=tdt, pin_memory=True)
    _PINNED.append(t)  # keep the page-locked buffer alive
    out = t.numpy().view(a.dtype)
    out[:] = a
    return out


_PINNED: list = []


def emit(line: dict) -> None:
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- jobs --
class Job:
    """One hot-path workload: graphs, the device call, units and bytes."""

    metric = "GTEPS"
    unit = "GTEPS"
    dtype = "u32"
    kernel = ""
    workload = ""

    def __init__(self, small: bool):
        self.small = small
        self.graphs = []  # dicts: name, host (HostCSR), symmetric, src

    def device_call(self, dg, gi, out):
        raise NotImplementedError

    def stats_call(self, dg, gi, out) -> dict:
        raise NotImplementedError

    def units(self, st: dict, gi: int) -> float:  # traversed edges per call
        return float(st["edges_reached"])

    def algo_bytes(self, st: dict, gi: int) -> float:
        raise NotImplementedError

    def cpu_call(self, gi):
        raise NotImplementedError

    def out_kind(self):
        return ("int32", np.uint32)

    def parity(self, gpu_out: np.ndarray, cpu_out, gi: int) -> str:
        return "bit-exact" if np.array_equal(gpu_out.view(np.uint32), np.asarray(cpu_out)) else "MISMATCH"

    def config(self) -> dict:
        return {"workload": self.workload,
                "graphs": [{"name": g["name"], "n": g["host"].n, "m": g["host"].m} for g in self.graphs],
                "l2": "inputs larger than L2 (CSR arrays >= 0.26 GB per graph vs 126 MB L2); no flush",
                "parallelism": "replicas"}


class SsspJob(Job):
    kernel = "sssp_persistent"
    workload = "SSSP delta-stepping, delta=2^13, w~U[1,255]: RMAT-22 directed ef16 (src = generator vertex 0) + grid 4096x4096 (src 0)"

    def __init__(self, small):
        super().__init__(small)
        from galois_b200 import assign_weights_u32, grid2d, rmat

        scale, side = (16, 512) if small else (22, 4096)
        g, perm = rmat(scale, 16, seed=22, symmetrize=False)
        assign_weights_u32(g, 1, 255, seed=22)
        self.graphs.append({"name": f"rmat{scale}-directed", "host": g, "symmetric": False, "src": int(perm[0])})
        gr = grid2d(side, side)
        assign_weights_u32(gr, 1, 255, seed=4096)
        self.graphs.append({"name": f"grid{side}x{side}", "host": gr, "symmetric": True, "src": 0})

    def device_call(self, dg, gi, out):
        dg.sssp(self.graphs[gi]["src"], 13, out=out)

    def stats_call(self, dg, gi, out):
        return dg.sssp(self.graphs[gi]["src"], 13, out=out, stats=True)[1]

    def algo_bytes(self, st, gi):
        # col + weight + dist per arc; offsets (16), dist write, queue push/pop per vertex
        return 12.0 * st["edges_reached"] + 28.0 * st["vertices_reached"]

    def cpu_call(self, gi):
        import oracle

        g = self.graphs[gi]
        return oracle.sssp_delta_parallel(g["host"], g["src"], 13)


class BfsJob(Job):
    kernel = "bfs_persistent"
    workload = "BFS from the max-degree vertex, RMAT-20 symmetric ef16"

    def __init__(self, small):
        super().__init__(small)
        from galois_b200 import rmat

        scale = 16 if small else 20
        g, _ = rmat(scale, 16, seed=20, symmetrize=True)
        self.graphs.append({"name": f"rmat{scale}-sym", "host": g, "symmetric": True,
                            "src": int(np.argmax(g.degrees()))})

    def device_call(self, dg, gi, out):
        dg.bfs(self.graphs[gi]["src"], out=out)

    def stats_call(self, dg, gi, out):
        return dg.bfs(self.graphs[gi]["src"], out=out, stats=True)[1]

    def algo_bytes(self, st, gi):
        return 8.0 * st["edges_reached"] + 28.0 * st["vertices_reached"]

    def cpu_call(self, gi):
        import oracle

        g = self.graphs[gi]
        return oracle.bfs_sync_tile(g["host"], g["src"])


class CcJob(Job):
    kernel = "cc_labelprop"
    workload = "CC label propagation + pointer jumping, RMAT-24 symmetric ef16, min-id labels"

    def __init__(self, small):
        super().__init__(small)
        from galois_b200 import rmat

        scale = 18 if small else 24
        g, _ = rmat(scale, 16, seed=24, symmetrize=True)
        self.graphs.append({"name": f"rmat{scale}-sym", "host": g, "symmetric": True, "src": 0})

    def device_call(self, dg, gi, out):
        dg.cc(0, out=out)

    def stats_call(self, dg, gi, out):
        return dg.cc(0, out=out, stats=True)[1]

    def units(self, st, gi):
        return float(self.graphs[gi]["host"].m)

    def algo_bytes(self, st, gi):
        g = self.graphs[gi]["host"]
        return st["rounds"] * (8.0 * g.m + 16.0 * g.n)

    def cpu_call(self, gi):
        import oracle

        return oracle.cc_labelprop(self.graphs[gi]["host"])[0]


class PrJob(Job):
    kernel = "pr_pull_persistent"
    dtype = "f32"
    workload = "PageRank pull-topological, alpha 0.85, tol 1e-6 (L1), max 1000, RMAT-24 symmetric ef16"

    def __init__(self, small):
        super().__init__(small)
        from galois_b200 import rmat

        scale = 18 if small else 24
        g, _ = rmat(scale, 16, seed=24, symmetrize=True)
        self.graphs.append({"name": f"rmat{scale}-sym", "host": g, "symmetric": True, "src": 0})
        self.iters = {}

    def out_kind(self):
        return ("float32", np.float32)

    def device_call(self, dg, gi, out):
        dg.pagerank_pull(0.85, 1e-6, 1000, out=out)

    def stats_call(self, dg, gi, out):
        st = dg.pagerank_pull(0.85, 1e-6, 1000, out=out, stats=True)[1]
        self.iters[gi] = st["iterations"]
        return st

    def units(self, st, gi):
        return float(st["iterations"]) * self.graphs[gi]["host"].m

    def algo_bytes(self, st, gi):
        g = self.graphs[gi]["host"]
        return st["iterations"] * (8.0 * g.m + 24.0 * g.n)

    def cpu_call(self, gi):
        import oracle

        return oracle.pr_pull_topo_par(self.graphs[gi]["host"], 0.85, 1e-6, 1000)[0]

    def parity(self, gpu_out, cpu_out, gi):
        err = float(np.abs(gpu_out.view(np.float32).astype(np.float64) - cpu_out).max())
        return f"max abs diff vs CPU fp32 in-place {err:.2e}"


JOBS = {"sssp": SsspJob, "bfs": BfsJob, "cc": CcJob, "pr": PrJob}


def cpu_units(job: Job, gpu_stats: list) -> float:
    return sum(job.units(st, gi) for gi, st in enumerate(gpu_stats))


def run_reference(args, job_cls) -> None:
    """CPU restatement of the reference algorithm on all host cores (rank 0 only)."""
    import oracle

    job = job_cls(args.small)
    # units per step: the same traversed-edge count the GPU arm reports,
    # computed on the host from the CPU result (reached vertices' degrees)
    t0 = time.perf_counter()
    outs = [job.cpu_call(gi) for gi in range(len(job.graphs))]
    first = time.perf_counter() - t0
    units = 0.0
    for gi, out in enumerate(outs):
        g = job.graphs[gi]["host"]
        if isinstance(job, (SsspJob, BfsJob)):
            units += float(g.degrees()[np.asarray(out) != oracle.INF].sum())
        elif isinstance(job, CcJob):
            units += float(g.m)
        else:
            _, it = oracle.pr_pull_topo_par(g, 0.85, 1e-6, 1000)
            units += float(it) * g.m
    steps, warm = args.steps, args.warmup
    if first * (steps + warm) > 240.0:  # keep the whole arm within a few minutes
        steps, warm = max(1, int(240.0 / max(first, 1e-3)) - 1), 1
    for _ in range(max(0, warm - 1)):
        for gi in range(len(job.graphs)):
            job.cpu_call(gi)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        for gi in range(len(job.graphs)):
            job.cpu_call(gi)
        times.append(time.perf_counter() - t0)
    t = sum(times)
    value = units * steps / t / 1e9
    cores = oracle.threads()
    sample = f"full workload per step ({steps} timed steps, {warm} warm-up)"
    emit({"impl": "reference", "metric": job.metric, "value": value, "unit": job.unit, "n_gpus": args.gpus,
          "steps": steps, "warmup": warm, "ms_per_step": 1e3 * t / steps, "higher_is_better": True,
          "scaling": "weak", "vs_baseline": None, "dtype": job.dtype, "data": "synthetic", "config": job.config(),
          "cpu_baseline": {"value": value, "unit": job.unit, "cores": cores, "kind": "port", "sample": sample},
          "e2e": {"value": value, "unit": job.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
          "note": "CPU restatement of the reference algorithm (oracle/, OpenMP); the reference itself "
                  "cannot be built here (Boost/LLVM/fmt absent)"})


def main() -> None:
    args = parse_args()
    job_cls = JOBS[args.app]
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, job_cls)
        return

    import torch

    from galois_b200 import DeviceGraph

    dist = Dist(want_pg=True)
    dev = dist.local_rank
    torch.cuda.set_device(dev)
    job = job_cls(args.small)
    tname, npdt = job.out_kind()
    dgs, outs = [], []
    for g in job.graphs:
        dgs.append(DeviceGraph(g["host"], symmetric=g["symmetric"], device=dev))
        outs.append(torch.empty(g["host"].n, dtype=getattr(torch, tname), device=f"cuda:{dev}"))
    # stats runs: warm the workspaces, collect units, bytes and kernel time
    st_runs = [[job.stats_call(dg, gi, outs[gi]) for gi, dg in enumerate(dgs)] for _ in range(3)]
    stats = st_runs[-1]
    units_step = sum(job.units(st, gi) for gi, st in enumerate(stats))
    bytes_step = sum(job.algo_bytes(st, gi) for gi, st in enumerate(stats))
    kms = [sum(r[gi]["kernel_ms"] for r in st_runs) / len(st_runs) for gi in range(len(dgs))]
    for _ in range(args.warmup):
        for gi, dg in enumerate(dgs):
            job.device_call(dg, gi, outs[gi])
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        for gi, dg in enumerate(dgs):
            job.device_call(dg, gi, outs[gi])
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_ms = dist.max(e0.elapsed_time(e1))
    value = dist.world * units_step * args.steps / (t_ms / 1e3) / 1e9
    peak, peak_src = measured_peak_hbm()
    achieved = bytes_step / (sum(kms) / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_src, "kernel": job.kernel,
                "algorithmic_bytes_per_step": bytes_step, "kernel_ms_per_step": sum(kms),
                "traffic": traffic_from_profiles(f"{args.app}{'-small' if args.small else ''}")}
    line = {"metric": job.metric, "value": value, "unit": job.unit, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": job.dtype, "data": "synthetic (seeded generators)",
            "config": job.config(), "roofline": roofline, "clocks": clk,
            "gpu_launches": 2 * len(dgs) * args.steps,
            "detail": [{"graph": job.graphs[gi]["name"], **{k: stats[gi][k] for k in stats[gi]}}
                       for gi in range(len(dgs))]}
    # ---- CPU baseline (rank 0, one GPU only) -----------------------------------
    if dist.world == 1 and not args.no_cpu_baseline:
        import oracle

        t0 = time.perf_counter()
        cpu_outs = [job.cpu_call(gi) for gi in range(len(job.graphs))]
        t_cpu = time.perf_counter() - t0
        gpu_host = [o.cpu().numpy() for o in outs]
        line["cpu_baseline"] = {"value": units_step / t_cpu / 1e9, "unit": job.unit, "cores": oracle.threads(),
                                "kind": "port", "sample": "one full run of every graph of the workload",
                                "parity": [job.parity(gpu_host[gi], cpu_outs[gi], gi)
                                           for gi in range(len(job.graphs))]}
    # ---- end to end through the public API with host buffers -----------------
    if not args.no_e2e:
        pinned = []
        for g in job.graphs:
            h = g["host"]
            pinned.append((pinned_copy(h.end_offs), pinned_copy(h.col),
                           pinned_copy(h.w_u32) if h.w_u32 is not None else None))
        host_out = [pinned_copy(np.zeros(g["host"].n, npdt)) for g in job.graphs]
        h2d = sum(a.nbytes + b.nbytes + (c.nbytes if c is not None else 0) for a, b, c in pinned)
        d2h = sum(o.nbytes for o in host_out)
        from galois_b200.graph import HostCSR

        def e2e_step():
            for gi, g in enumerate(job.graphs):
                a, b, c = pinned[gi]
                with DeviceGraph(HostCSR(a, b, c), symmetric=g["symmetric"], device=dev) as dg:
                    job.device_call(dg, gi, host_out[gi])

        e2e_step()
        ke = max(1, min(args.steps, 5))
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            e2e_step()
        te = dist.max(time.perf_counter() - t0)
        line["e2e"] = {"value": dist.world * units_step * ke / te / 1e9, "unit": job.unit,
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": ke,
                       "path": "gb_graph_upload (pinned host CSR) + kernel + host output copy + gb_graph_free"}
    for dg in dgs:
        dg.free()
    if dist.rank == 0:
        emit(line)
    dist.close()


if __name__ == "__main__":
    main()
