#!/usr/bin/env python3
"""Benchmark of the CSR edge-map path on B200.

Default workload (no --app): delta-stepping SSSP, delta = 2^13, uint32 weights
uniform in [1,255], on (a) a directed RMAT scale-22 graph (edge factor 16,
a/b/c = 0.57/0.19/0.19, seeded relabelling; source = the generator's vertex 0)
and (b) the 4096x4096 4-neighbour grid (source 0).  One step = one full SSSP
on each graph.  Metric: GTEPS = (m_r(a) + m_r(b)) / step time, m_r = arcs out
of reached vertices.  Other --app values run the other hot-path kernels on
their configurations (bfs: RMAT-20 sym; cc, pr: RMAT-24 sym).

On one GPU the default run also measures BFS (RMAT-20 and RMAT-24), CC and
PageRank pull-topological (RMAT-24) and reports them under "apps", each with
its parity against the oracle.

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
    ap.add_argument("--app", choices=["sssp", "bfs", "bfs-parent", "cc", "pr", "pr-residual", "bc", "multigraph", "ppr"], default="sssp")
    ap.add_argument("--size", choices=["small", "medium", "full", "s24"], default="full",
                    help="graph sizes: full = the benchmark configuration; s24 = RMAT scale 24 for every "
                         "app; medium/small for profiling")
    ap.add_argument("--order", type=int, choices=[0, 1, 2, 3, 4], default=4,
                    help="vertex order of the resident graphs (gb_graph_reorder, done once before timing): "
                         "0 file order, 1 degree-ordered with sorted rows, 2 degree-ordered unsorted rows, "
                         "3 locality (Morton order of landmark BFS distances), 4 auto (3 when no vertex has "
                         "more than 16 arcs, else 1)")
    ap.add_argument("--small", action="store_true", help="same as --size small")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-apps", action="store_true",
                    help="skip the BFS / CC / PageRank configurations that the default run adds under 'apps'")
    args = ap.parse_args()
    if args.small:
        args.size = "small"
    return args


# ---------------------------------------------------------------- plumbing --
class Dist:
    """torch.distributed when launched by torchrun (WORLD_SIZE > 1), else a
    no-op.  NCCL on GPUs; `backend="gloo"` keeps everything on the host (the
    CPU tests of the barrier / max-over-ranks timing use it)."""

    def __init__(self, want_pg: bool, backend: str = "nccl", timeout_s: float = 600.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False
        if self.world > 1 and want_pg:
            import datetime

            import torch
            import torch.distributed as dist

            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                kw["device_id"] = torch.device("cuda", self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
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

        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()
            self.pg = False


def aggregate_rate(world: int, units_per_step: float, steps: int, t_ms_max: float) -> float:
    """Whole-job throughput in G-units/s: every rank processes units_per_step
    per step (replicas / weak scaling), timed as the slowest rank."""
    return world * units_per_step * steps / (t_ms_max / 1e3) / 1e9


class ClockSampler:
    """SM clock and throttle reasons during a timed region: nvidia-smi at its
    200 ms period plus an NVML thread at 1 ms, so that timed regions shorter
    than nvidia-smi's period still get samples.  The GPU is named by its UUID
    (CUDA and NVML number devices differently under CUDA_VISIBLE_DEVICES)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu: int, period_s: float = 0.001):
        self.gpu = gpu
        self.period_s = period_s
        self.proc = None
        self.thread = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.uuid = None
        try:
            import torch

            self.uuid = "GPU-" + str(torch.cuda.get_device_properties(gpu).uuid)
        except Exception:
            pass

    def _nvml_loop(self, stop, rows, ready):
        try:
            import pynvml as nv

            nv.nvmlInit()
        except Exception:
            ready.set()
            return
        try:
            h = nv.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else nv.nvmlDeviceGetHandleByIndex(self.gpu)
            smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            while not stop.is_set():
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                rows.append((sm, smax, tuple(bool(mask & b) for b in bits)))
                ready.set()
                stop.wait(self.period_s)
        except Exception:
            pass
        finally:
            ready.set()
            try:
                nv.nvmlShutdown()
            except Exception:
                pass

    def start(self):
        import threading

        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.uuid or str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        self._stop = threading.Event()
        self._nvml_rows = []
        ready = threading.Event()
        self.thread = threading.Thread(target=self._nvml_loop, args=(self._stop, self._nvml_rows, ready), daemon=True)
        self.thread.start()
        # the timed region starts only once NVML is sampling (bounded wait);
        # the samples taken before it are dropped
        ready.wait(2.0)
        self._t0 = len(self._nvml_rows)

    def stop(self) -> dict:
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
        rows = []  # (sm MHz, max MHz, (reason active,) * 4)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.file.flush()
            for line in Path(self.file.name).read_text().splitlines():
                r = [x.strip() for x in line.split(",")]
                if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                    rows.append((float(r[1]), float(r[2]), tuple(r[5 + i].lower() == "active" for i in range(4))))
        os.unlink(self.file.name)
        n_smi = len(rows)
        if self.thread is not None:
            # a region shorter than one period keeps the sample taken as it began
            rows += self._nvml_rows[self._t0:] or self._nvml_rows[-1:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [] if self.proc else ["nvidia-smi unavailable"],
                    "samples": 0}
        smax = max(r[1] for r in rows)
        reasons = sorted({self.REASONS[i] for r in rows for i in range(4) if r[2][i]})
        loaded = [r[0] for r in rows if r[0] > 0.5 * smax] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "samples_nvidia_smi": n_smi, "samples_nvml": len(rows) - n_smi}


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


def pick(size: str, small, medium, full, s24=None):
    return {"small": small, "medium": medium, "full": full, "s24": full if s24 is None else s24}[size]


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

    def __init__(self, size: str):
        self.size = size
        self.graphs = []  # dicts: name, host (HostCSR), symmetric, src

    def check(self, gpu_out: np.ndarray, gi: int) -> str:
        """Parity of one GPU output against the oracle's ground truth."""
        raise NotImplementedError

    def device_call(self, dg, gi, out):
        raise NotImplementedError

    def stats_call(self, dg, gi, out) -> dict:
        raise NotImplementedError

    def units(self, st: dict, gi: int) -> float:  # traversed edges per call
        return float(st["edges_reached"])

    def algo_bytes(self, st: dict, gi: int) -> float:
        raise NotImplementedError

    def work_bytes(self, st: dict, gi: int) -> float:
        """Bytes of the arcs the kernel actually scanned (the algorithmic model
        counts every reached arc once; direction-optimised BFS and the giant
        skip of CC read fewer, label-correcting SSSP reads more)."""
        return self.algo_bytes(st, gi)

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
    # the oracle's delta-stepping drains the current bucket in parallel rounds
    # before it opens the next one
    CPU_SCHEDULE = ("bucket-synchronous delta-stepping (OBIM with a barrier between buckets): the schedule the "
                    "reference's Auto choice runs on the grid (deltaStepBarrier, SSSP.cpp:410-416,453); on the "
                    "power-law RMAT graph the reference picks barrier-free OBIM (deltaStep), which this "
                    "restatement does not model")
    kernel = "sssp_persistent"
    workload = "SSSP delta-stepping, delta=2^13, w~U[1,255]: RMAT-22 directed ef16 (src = generator vertex 0) + grid 4096x4096 (src 0)"

    def __init__(self, size):
        super().__init__(size)
        from galois_b200 import assign_weights_u32, grid2d, rmat

        scale, side = pick(size, (16, 512), (20, 2048), (22, 4096), (24, 4096))
        self.workload = self.workload.replace("RMAT-22", f"RMAT-{scale}").replace("4096x4096", f"{side}x{side}")
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

    def work_bytes(self, st, gi):
        return 12.0 * st["edges_scanned"] + 28.0 * st["vertices_reached"]

    def cpu_call(self, gi):
        import oracle

        g = self.graphs[gi]
        return oracle.sssp_delta_parallel(g["host"], g["src"], 13)


class BfsJob(Job):
    kernel = "bfs_persistent"
    workload = "BFS from the max-degree vertex, RMAT-20 symmetric ef16"

    def __init__(self, size, graph=None, name=None):
        super().__init__(size)
        from galois_b200 import rmat

        if graph is None:
            scale = pick(size, 16, 21, 20, 24)
            graph, _ = rmat(scale, 16, seed=20, symmetrize=True)
            name = f"rmat{scale}-sym"
        self.workload = self.workload.replace("RMAT-20", name.split("-")[0].upper().replace("RMAT", "RMAT-"))
        self.graphs.append({"name": name, "host": graph, "symmetric": True,
                            "src": int(np.argmax(graph.degrees()))})

    def check(self, gpu_out, gi):
        import oracle

        g = self.graphs[gi]
        same = np.array_equal(gpu_out.view(np.uint32), oracle.bfs_serial(g["host"], g["src"]))
        return "bit-exact vs the oracle's serial BFS" if same else "MISMATCH vs the oracle's serial BFS"

    def device_call(self, dg, gi, out):
        dg.bfs(self.graphs[gi]["src"], out=out)

    def stats_call(self, dg, gi, out):
        return dg.bfs(self.graphs[gi]["src"], out=out, stats=True)[1]

    def algo_bytes(self, st, gi):
        return 8.0 * st["edges_reached"] + 28.0 * st["vertices_reached"]

    def work_bytes(self, st, gi):
        return 8.0 * st["edges_scanned"] + 28.0 * st["vertices_reached"]

    def cpu_call(self, gi):
        import oracle

        g = self.graphs[gi]
        return oracle.bfs_sync_tile(g["host"], g["src"])


class BfsParentJob(BfsJob):
    """BFS with parents (bfsDirectionOpt's output): the BFS kernel, then the
    parent pass over every in-arc (gb_bfs_parent)."""

    kernel = "bfs_persistent + parent_rows/parent_tiles"
    workload = "BFS parents (smallest-id valid parent) from the max-degree vertex, RMAT-20 symmetric ef16"
    cpu_serial = True  # the restatement of SyncDO is serial

    def __init__(self, size):
        super().__init__(size)

    def device_call(self, dg, gi, out):
        dg.bfs_parent(self.graphs[gi]["src"], out=out)

    def stats_call(self, dg, gi, out):
        return dg.bfs_parent(self.graphs[gi]["src"], out=out, stats=True)[1]

    def algo_bytes(self, st, gi):
        # the BFS push model, then column + level per in-arc and offsets, level
        # and parent per vertex for the parent pass
        g = self.graphs[gi]["host"]
        return super().algo_bytes(st, gi) + 8.0 * g.m + 24.0 * g.n

    def work_bytes(self, st, gi):
        g = self.graphs[gi]["host"]
        return super().work_bytes(st, gi) + 8.0 * g.m + 24.0 * g.n

    def cpu_call(self, gi):
        import oracle

        g = self.graphs[gi]
        return oracle.bfs_do_parent(g["host"], g["src"])

    def parity(self, gpu_out, cpu_out, gi):
        import oracle

        g = self.graphs[gi]
        lv = oracle.bfs_serial(g["host"], g["src"])
        got = gpu_out.view(np.uint32)
        same = np.array_equal(got, oracle.bfs_parent_min(g["host"], g["src"], lv))
        ok = oracle.verify_bfs_parent(g["host"], g["src"], lv, got) == 0
        return f"{'bit-exact' if same else 'MISMATCH'} vs the min-id rule; BFS tree {'valid' if ok else 'INVALID'}"

    def check(self, gpu_out, gi):
        return self.parity(gpu_out, None, gi)


class CcJob(Job):
    kernel = "cc_labelprop"
    workload = "CC label propagation + pointer jumping, RMAT-24 symmetric ef16, min-id labels"

    def __init__(self, size, graph=None, name=None):
        super().__init__(size)
        from galois_b200 import rmat

        if graph is None:
            scale = pick(size, 18, 21, 24)
            graph, _ = rmat(scale, 16, seed=24, symmetrize=True)
            name = f"rmat{scale}-sym"
        self.graphs.append({"name": name, "host": graph, "symmetric": True, "src": 0})

    def check(self, gpu_out, gi):
        import oracle

        same = np.array_equal(gpu_out.view(np.uint32), oracle.cc_union_find(self.graphs[gi]["host"]))
        return "bit-exact vs the oracle's union-find min-id labels" if same else "MISMATCH vs union-find labels"

    def cpu_run(self, g):
        """(output, units) of the CPU restatement on host graph g."""
        import oracle

        return oracle.cc_labelprop(g)[0], float(g.m)

    def device_call(self, dg, gi, out):
        dg.cc(0, out=out)

    def stats_call(self, dg, gi, out):
        return dg.cc(0, out=out, stats=True)[1]

    def units(self, st, gi):
        return float(self.graphs[gi]["host"].m)

    def algo_bytes(self, st, gi):
        # one sweep = column + label per arc, offsets + label per vertex; counted per round
        g = self.graphs[gi]["host"]
        return st["rounds"] * (8.0 * g.m + 16.0 * g.n)

    def work_bytes(self, st, gi):
        # a round after the first scans only the rows outside the giant component
        g = self.graphs[gi]["host"]
        return 8.0 * st["edges_scanned"] + 16.0 * g.n * st["rounds"]

    def cpu_call(self, gi):
        import oracle

        return oracle.cc_labelprop(self.graphs[gi]["host"])[0]


class PrJob(Job):
    kernel = "pr_pull_persistent"
    dtype = "f32"
    workload = "PageRank pull-topological, alpha 0.85, tol 1e-6 (L1), max 1000, RMAT-24 symmetric ef16"

    def __init__(self, size, graph=None, name=None):
        super().__init__(size)
        from galois_b200 import rmat

        if graph is None:
            scale = pick(size, 18, 21, 24)
            graph, _ = rmat(scale, 16, seed=24, symmetrize=True)
            name = f"rmat{scale}-sym"
        self.graphs.append({"name": name, "host": graph, "symmetric": True, "src": 0})
        self.iters = {}

    def check(self, gpu_out, gi):
        import oracle

        want, it64 = oracle.pr_pull_topo_f64(self.graphs[gi]["host"], 0.85, 1e-6, 1000)
        err = float(np.abs(gpu_out.view(np.float32).astype(np.float64) - want).max())
        ok = err <= 1e-5 and abs(self.iters.get(gi, -99) - it64) <= 2
        return (f"{'within' if ok else 'OUTSIDE'} tolerance: L-inf {err:.2e} vs the FP64 Jacobi oracle (<= 1e-5), "
                f"{self.iters.get(gi)} iterations vs {it64} (within 2)")

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

    def cpu_run(self, g):
        """(output, units) of the CPU restatement on host graph g."""
        import oracle

        x, it = oracle.pr_pull_topo_par(g, 0.85, 1e-6, 1000)
        return x, float(it) * g.m

    def cpu_call(self, gi):
        return self.cpu_run(self.graphs[gi]["host"])[0]

    def parity(self, gpu_out, cpu_out, gi):
        err = float(np.abs(gpu_out.view(np.float32).astype(np.float64) - cpu_out).max())
        return f"max abs diff vs CPU fp32 in-place {err:.2e}"


class PrResidualJob(PrJob):
    """PageRank pull-residual (PageRank-pull.cpp:132-190), the app's default
    -algo, at its default tolerance 1e-3 (PageRank-constants.h)."""

    kernel = "pr_pull_residual_persistent"
    workload = "PageRank pull-residual, alpha 0.85, tol 1e-3 (per vertex), max 1000, RMAT-24 symmetric ef16"
    tol = 1e-3

    def device_call(self, dg, gi, out):
        dg.pagerank_pull_residual(0.85, self.tol, 1000, out=out)

    def stats_call(self, dg, gi, out):
        st = dg.pagerank_pull_residual(0.85, self.tol, 1000, out=out, stats=True)[1]
        self.iters[gi] = st["iterations"]
        return st

    def cpu_run(self, g):
        import oracle

        x, it = oracle.pr_pull_residual(g, 0.85, self.tol, 1000, f64=False)
        return x, float(it) * g.m

    def parity(self, gpu_out, cpu_out, gi):
        err = float(np.abs(gpu_out.view(np.float32).astype(np.float64) - cpu_out).max())
        return f"max abs diff vs CPU fp32 restatement {err:.2e}"

    def check(self, gpu_out, gi):
        import oracle

        want, _ = oracle.pr_pull_residual(self.graphs[gi]["host"], 0.85, self.tol, 1000, f64=True)
        err = float(np.abs(gpu_out.view(np.float32).astype(np.float64) - want).max())
        return f"L-inf {err:.2e} vs the FP64 restatement at the same tolerance"


JOBS = {"sssp": SsspJob, "bfs": BfsJob, "bfs-parent": BfsParentJob, "cc": CcJob, "pr": PrJob, "pr-residual": PrResidualJob}
ORDER_NAMES = {0: "file order", 1: "degree-ordered (gb_graph_reorder, sorted rows)",
               2: "degree-ordered (gb_graph_reorder, unsorted rows)",
               3: "locality (gb_graph_reorder: Morton order of landmark BFS distances, sorted rows)",
               4: "auto (gb_graph_reorder: locality for degree <= 16, else degree-ordered)"}
BATCHED = ("bc", "multigraph", "ppr")


def _time_gpu(fn, steps: int) -> float:
    """Device time (ms) of `steps` calls of fn on torch's current stream."""
    import torch

    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(steps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_batched(args) -> None:
    """Batched kernels against looping the plain kernels on the same GPU."""
    import torch

    import oracle
    from galois_b200 import DeviceGraph, erdos_renyi, rmat

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    steps, warm = args.steps, args.warmup
    line = {"n_gpus": 1, "steps": steps, "warmup": warm, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic (seeded generators)"}
    clocks = ClockSampler(dev)
    if args.app == "bc":
        scale = pick(args.size, 14, 17, 20)
        g, _ = rmat(scale, 16, seed=20, symmetrize=True)
        rng = np.random.default_rng(1024)
        srcs = rng.choice(np.flatnonzero(g.degrees() > 0), 1024, replace=False).astype(np.uint32)
        dg = DeviceGraph(g, symmetric=True, device=dev)
        # traversed edges: forward + backward over the arcs of reached vertices, per source
        lv = torch.empty(g.n, dtype=torch.int32, device="cuda")
        m_r = sum(dg.bfs(int(s), out=lv, stats=True)[1]["edges_reached"] for s in srcs)
        units = 2.0 * m_r
        out = torch.empty(g.n, dtype=torch.float32, device="cuda")
        dg.bc(srcs, batch=64, out=out)
        for _ in range(warm):
            dg.bc(srcs, batch=64, out=out)
        clocks.start()
        t_b = _time_gpu(lambda: dg.bc(srcs, batch=64, out=out), steps)
        dg.bc(srcs, batch=1, out=out)
        t_l = _time_gpu(lambda: dg.bc(srcs, batch=1, out=out), 1)
        clk = clocks.stop()
        bc_gpu = out.cpu().numpy()
        sample = srcs[:8]
        with DeviceGraph(g, symmetric=True, device=dev) as dg8:
            got8 = dg8.bc(sample, batch=8)
        ref8 = oracle.bc_level(g, sample, f64=True)
        rel = float((np.abs(got8 - ref8) / np.maximum(np.abs(ref8), 1.0)).max())
        t0 = time.perf_counter()
        oracle.bc_level(g, srcs[:16], parallel=True)
        t_cpu = time.perf_counter() - t0
        m_r16 = units * 16 / len(srcs)
        line.update({"metric": "BC aggregate GTEPS (fwd+bwd arcs of reached vertices, 1024 sources)",
                     "unit": "GTEPS", "dtype": "f64 sigma / f32 dependency", "value": units * steps / (t_b / 1e3) / 1e9,
                     "ms_per_step": t_b / steps,
                     "config": {"workload": f"Brandes BC, RMAT-{scale} sym ef16, 1024 seeded sources, 64 per launch",
                                "n": g.n, "m": g.m},
                     "looped": {"value": units / (t_l / 1e3) / 1e9, "ms_per_step": t_l,
                                "how": "gb_bc batch=1: one persistent single-source launch per source"},
                     "speedup_vs_looped": (t_l) / (t_b / steps),
                     "parity": f"max rel err vs FP64 oracle on 8 sources: {rel:.2e}",
                     "cpu_baseline": {"value": m_r16 / t_cpu / 1e9, "unit": "GTEPS", "cores": oracle.threads(),
                                      "kind": "port", "sample": "16 of the 1024 sources, Level BC, OpenMP"},
                     "clocks": clk, "gpu_launches": 3 * (len(srcs) // 64) + 1})
        dg.free()
    elif args.app == "multigraph":
        from galois_b200.graph import pack_graphs

        k = pick(args.size, 64, 128, 512)
        hi = pick(args.size, 20000, 50000, 200000)
        rng = np.random.default_rng(512)
        sizes = np.exp(rng.uniform(np.log(1000), np.log(hi), k)).astype(int)
        graphs = [erdos_renyi(int(n), 8.0, seed=100 + i) for i, n in enumerate(sizes)]
        packed, first = pack_graphs(graphs)
        local = np.zeros(k, np.uint32)
        dg = DeviceGraph(packed, symmetric=True, device=dev)
        dg.autotune("bfs", int(first[0]))
        lv = torch.empty(packed.n, dtype=torch.int32, device="cuda")
        lb = torch.empty(packed.n, dtype=torch.int32, device="cuda")
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            dg.multi_graph_bfs_cc(first, local, lv, lb)
            torch.cuda.synchronize()
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=s):
                dg.multi_graph_bfs_cc(first, local, lv, lb)
        for _ in range(warm):
            cg.replay()
        clocks.start()
        t_b = _time_gpu(cg.replay, steps)
        # looped: one handle per graph, gb_bfs + gb_cc each
        dgs = [DeviceGraph(gk, symmetric=True, device=dev) for gk in graphs]
        outs = [(torch.empty(gk.n, dtype=torch.int32, device="cuda"), torch.empty(gk.n, dtype=torch.int32, device="cuda"))
                for gk in graphs]

        def loop():
            for d, (a, b) in zip(dgs, outs):
                d.bfs(0, out=a)
                d.cc(1, out=b)

        loop()
        t_l = _time_gpu(loop, 1)
        clk = clocks.stop()
        lvh = lv.cpu().numpy().view(np.uint32)
        lbh = lb.cpu().numpy().view(np.uint32)
        ok = all(np.array_equal(lvh[first[i]:first[i + 1]], oracle.bfs_serial(graphs[i], 0)) and
                 np.array_equal(lbh[first[i]:first[i + 1]], oracle.cc_union_find(graphs[i]))
                 for i in range(0, k, max(1, k // 16)))
        units = 2.0 * packed.m  # BFS over the reached arcs (giant components) + CC over every arc
        t0 = time.perf_counter()
        for i in range(0, k, max(1, k // 16)):
            oracle.bfs_sync_tile(graphs[i], 0)
            oracle.cc_labelprop(graphs[i])
        t_cpu = time.perf_counter() - t0
        cpu_units = 2.0 * sum(graphs[i].m for i in range(0, k, max(1, k // 16)))
        line.update({"metric": "multi-graph BFS+CC throughput (graphs per second)", "unit": "graphs/s", "dtype": "u32",
                     "value": k * steps / (t_b / 1e3), "ms_per_step": t_b / steps,
                     "aggregate_gteps": units * steps / (t_b / 1e3) / 1e9,
                     "config": {"workload": f"{k} Erdos-Renyi graphs, n log-uniform in [1000, {hi}], mean degree 8, "
                                            "BFS from local vertex 0 + CC, one CUDA-graph replay per step",
                                "n": packed.n, "m": packed.m},
                     "looped": {"value": k / (t_l / 1e3), "ms_per_step": t_l,
                                "how": "one handle per graph: gb_bfs + gb_cc per graph"},
                     "speedup_vs_looped": t_l / (t_b / steps),
                     "parity": "bit-exact on sampled graphs" if ok else "MISMATCH",
                     "cpu_baseline": {"value": cpu_units / t_cpu / 1e9, "unit": "GTEPS", "cores": oracle.threads(),
                                      "kind": "port", "sample": "every k/16-th graph: SyncTile BFS + LabelProp CC"},
                     "clocks": clk, "gpu_launches": 9 * steps})
        del cg
        for d in dgs:
            d.free()
        dg.free()
    else:  # ppr
        from galois_b200 import assign_weights_f32
        from galois_b200.ppr import ppr

        scale = pick(args.size, 16, 19, 22)
        g, _ = rmat(scale, 16, seed=22, symmetrize=False)
        assign_weights_f32(g, seed=22)
        B = 128
        rng = np.random.default_rng(128)
        T = torch.zeros((g.n, B), dtype=torch.float32, device="cuda")
        for b in range(B):
            T[torch.from_numpy(rng.choice(g.n, 32, replace=False)).cuda(), b] = 1.0 / 32
        c = torch.from_numpy(rng.standard_normal((g.n, B)).astype(np.float32)).cuda()
        dg = DeviceGraph(g, device=dev)
        w = torch.from_numpy(g.w_f32).cuda().requires_grad_(True)

        def batched():
            w.grad = None
            x = ppr(dg, T, w, 0.85, 1e-7)
            (c * x).sum().backward()

        def looped():
            w.grad = None
            for b in range(B):
                x = ppr(dg, T[:, b:b + 1].contiguous(), w, 0.85, 1e-7)
                (c[:, b:b + 1] * x).sum().backward()

        batched()
        for _ in range(warm):
            batched()
        clocks.start()
        t_b = _time_gpu(batched, steps)
        looped()
        t_l = _time_gpu(looped, 1)
        clk = clocks.stop()
        line.update({"metric": "PPR forward+adjoint columns per second (batch 128, tol 1e-7)", "unit": "columns/s",
                     "dtype": "f32", "value": B * steps / (t_b / 1e3), "ms_per_step": t_b / steps,
                     "config": {"workload": f"personalised PageRank + adjoint, RMAT-{scale} directed ef16, w~U(0,1], "
                                            "128 teleports x 32 nonzeros, alpha 0.85, tol 1e-7, loss sum(c*x)",
                                "n": g.n, "m": g.m},
                     "looped": {"value": B / (t_l / 1e3), "ms_per_step": t_l,
                                "how": "128 single-column solves (B=1 kernels), forward+adjoint each"},
                     "speedup_vs_looped": t_l / (t_b / steps), "clocks": clk, "gpu_launches": 12 * steps})
        dg.free()
    emit(line)


def run_bc_sharded(args) -> None:
    """--app bc on N GPUs: the 1024 sources are sharded over the ranks and one
    NCCL all-reduce sums the partial centralities (strong scaling: the total
    work is fixed)."""
    import torch

    from galois_b200 import DeviceGraph, rmat
    from galois_b200.distributed import bc_sharded, shard_sources

    dist = Dist(want_pg=True)
    dev = dist.local_rank
    torch.cuda.set_device(dev)
    scale = pick(args.size, 14, 17, 20)
    g, _ = rmat(scale, 16, seed=20, symmetrize=True)
    rng = np.random.default_rng(1024)
    srcs = rng.choice(np.flatnonzero(g.degrees() > 0), 1024, replace=False).astype(np.uint32)
    dg = DeviceGraph(g, symmetric=True, device=dev)
    lv = torch.empty(g.n, dtype=torch.int32, device=f"cuda:{dev}")
    mine = shard_sources(srcs, dist.rank, dist.world)
    m_r_mine = float(sum(dg.bfs(int(s), out=lv, stats=True)[1]["edges_reached"] for s in mine))
    units = 2.0 * dist.sum(m_r_mine)  # forward + backward arcs of all sources, whole job
    out = torch.empty(g.n, dtype=torch.float32, device=f"cuda:{dev}")
    for _ in range(max(args.warmup, 1)):
        bc_sharded(dg, srcs, out, 64)
    clocks = ClockSampler(dev)
    clocks.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        bc_sharded(dg, srcs, out, 64)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_ms = dist.max(e0.elapsed_time(e1))
    if dist.rank == 0:
        emit({"metric": "BC aggregate GTEPS (fwd+bwd arcs of reached vertices, 1024 sources)", "unit": "GTEPS",
              "value": units * args.steps / (t_ms / 1e3) / 1e9, "n_gpus": dist.world, "steps": args.steps,
              "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
              "scaling": "strong", "vs_baseline": None, "dtype": "f64 sigma / f32 dependency",
              "data": "synthetic (seeded generators)",
              "config": {"workload": f"Brandes BC, RMAT-{scale} sym ef16, 1024 seeded sources sharded over "
                                     f"{dist.world} GPUs, 64 per launch, one all-reduce of bc per step",
                         "n": g.n, "m": g.m, "parallelism": f"sources/{dist.world}"},
              "clocks": clk, "gpu_launches": (3 * (len(mine) // 64) + 2) * args.steps})
    dg.free()
    dist.close()


def measure_resident(job: Job, dev: int, dist: Dist, steps: int, warmup: int, order: int) -> dict:
    """Upload (and reorder) the job's graphs, collect per-call statistics,
    then time `steps` steps with inputs resident in HBM: CUDA events on the
    launching stream, barrier + synchronize on both sides, max over ranks."""
    import torch

    from galois_b200 import DeviceGraph

    tname, _ = job.out_kind()
    dgs, outs, reorder_ms = [], [], []
    for g in job.graphs:
        dg = DeviceGraph(g["host"], symmetric=g["symmetric"], device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if order:
            dg.reorder(order)  # graph preparation, once, outside the timed region
        torch.cuda.synchronize()
        reorder_ms.append((time.perf_counter() - t0) * 1e3)
        dgs.append(dg)
        outs.append(torch.empty(g["host"].n, dtype=getattr(torch, tname), device=f"cuda:{dev}"))
    # stats runs: warm the workspaces, collect units, bytes and kernel time
    st_runs = [[job.stats_call(dg, gi, outs[gi]) for gi, dg in enumerate(dgs)] for _ in range(3)]
    stats = st_runs[-1]
    # the first call of a kernel also pays its lazy module load: average the later runs
    kms = [sum(r[gi]["kernel_ms"] for r in st_runs[1:]) / (len(st_runs) - 1) for gi in range(len(dgs))]
    for _ in range(warmup):
        for gi, dg in enumerate(dgs):
            job.device_call(dg, gi, outs[gi])
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        for gi, dg in enumerate(dgs):
            job.device_call(dg, gi, outs[gi])
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_ms = dist.max(e0.elapsed_time(e1))
    return {"dgs": dgs, "outs": outs, "stats": stats, "kms": kms, "t_ms": t_ms, "clocks": clk,
            "reorder_ms": reorder_ms, "orders": [dg.order for dg in dgs],
            "units_step": sum(job.units(st, gi) for gi, st in enumerate(stats)),
            "bytes_step": sum(job.algo_bytes(st, gi) for gi, st in enumerate(stats)),
            "work_step": sum(job.work_bytes(st, gi) for gi, st in enumerate(stats))}


def roofline_of(job: Job, r: dict, order: int, traffic) -> dict:
    """Roofline of the dominant kernel from its event-timed duration.  `frac`
    counts the bytes the kernel both had to read and did read: the smaller of
    the algorithmic model (every reached arc once) and the arcs it actually
    scanned (direction-optimised BFS and CC's giant skip read fewer arcs than
    the model, label-correcting SSSP more); both are kept beside it."""
    peak, peak_src = measured_peak_hbm()
    sec = sum(r["kms"]) / 1e3
    kernel = job.kernel
    if isinstance(job, PrJob) and 1 in r["orders"]:
        # a degree-ordered PageRank runs the binned kernels
        kernel = "pr_resid_binned" if isinstance(job, PrResidualJob) else "pr_pull_binned"
    elif type(job) is SsspJob:
        # the region kernel reports its shared-memory rounds in pull_rounds
        kernel = " + ".join(f"{'sssp_region' if st.get('pull_rounds') else 'sssp_persistent'} ({g['name']})"
                            for g, st in zip(job.graphs, r["stats"]))
    need = min(r["bytes_step"], r["work_step"])
    return {"bound": "hbm", "achieved": need / sec / 1e9, "peak": peak, "unit": "GB/s",
            "frac": need / sec / 1e9 / peak, "peak_source": peak_src,
            "kernel": kernel,
            "bytes_counted_per_step": need,
            "algorithmic_bytes_per_step": r["bytes_step"], "kernel_ms_per_step": sum(r["kms"]),
            "model_frac": r["bytes_step"] / sec / 1e9 / peak,
            "work_bytes_per_step": r["work_step"],
            "frac_of_work": r["work_step"] / sec / 1e9 / peak,
            "traffic": traffic}


def run_apps(args, dev: int) -> dict:
    """The other plain kernels on their configurations, measured in the same
    run as the headline: BFS on RMAT-20 and RMAT-24, CC and PageRank
    pull-topological on RMAT-24 (all symmetric ef16, degree-ordered as the
    headline).  Each entry: device-timed throughput, kernel time, roofline,
    clocks and parity against the oracle."""
    import oracle
    from galois_b200 import rmat

    single = Dist(want_pg=False)
    g24, _ = rmat(24, 16, seed=24, symmetrize=True)
    # (key, job, its DRAM traffic entry in profiles/traffic.json)
    jobs = [("bfs-rmat20", BfsJob("full"), "bfs-full"),
            ("bfs-rmat24", BfsJob("full", graph=g24, name="rmat24-sym"), "bfs-s24"),
            ("cc-rmat24", CcJob("full", graph=g24, name="rmat24-sym"), "cc-full"),
            ("pr-rmat24", PrJob("full", graph=g24, name="rmat24-sym"), "pr-full")]
    out = {}
    for key, job, traffic_key in jobs:
        r = measure_resident(job, dev, single, args.steps, args.warmup, args.order)
        gpu_host = r["outs"][0].cpu().numpy()
        for dg in r["dgs"]:
            dg.free()
        st = r["stats"][0]
        # the CPU restatement on the same graph: PageRank counts its own
        # iterations, the others traverse the same arcs as the GPU
        t0 = time.perf_counter()
        if hasattr(job, "cpu_run"):
            cpu_units = job.cpu_run(job.graphs[0]["host"])[1]
        else:
            job.cpu_call(0)
            cpu_units = r["units_step"]
        t_cpu = time.perf_counter() - t0
        out[key] = {"workload": job.workload, "graph": job.graphs[0]["name"], "n": job.graphs[0]["host"].n,
                    "m": job.graphs[0]["host"].m, "metric": job.metric,
                    "value": r["units_step"] * args.steps / (r["t_ms"] / 1e3) / 1e9, "unit": job.unit,
                    "ms_per_step": r["t_ms"] / args.steps, "kernel_ms": sum(r["kms"]),
                    "roofline": roofline_of(job, r, args.order, traffic_from_profiles(traffic_key)),
                    "clocks": r["clocks"],
                    "parity": job.check(gpu_host, 0),
                    "stats": {k: st[k] for k in ("vertices_reached", "edges_reached", "edges_scanned", "rounds",
                                                 "pull_rounds", "iterations") if k in st},
                    "cpu_baseline": {"value": cpu_units / t_cpu / 1e9, "unit": job.unit, "cores": oracle.threads(),
                                     "kind": "port", "sample": "one full run of the same workload"}}
    return out


def run_ppr_sharded(args) -> None:
    """--app ppr on N GPUs: the 128 teleport columns are sharded over the
    ranks (blocks of multiples of 4) and one NCCL all-reduce sums the
    edge-weight gradient (strong scaling: the total work is fixed)."""
    import torch

    from galois_b200 import DeviceGraph, assign_weights_f32, rmat
    from galois_b200.distributed import ppr_sharded

    dist = Dist(want_pg=True)
    dev = dist.local_rank
    torch.cuda.set_device(dev)
    scale = pick(args.size, 16, 19, 22)
    g, _ = rmat(scale, 16, seed=22, symmetrize=False)
    assign_weights_f32(g, seed=22)
    B = 128
    rng = np.random.default_rng(128)
    T = torch.zeros((g.n, B), dtype=torch.float32, device=f"cuda:{dev}")
    for b in range(B):
        T[torch.from_numpy(rng.choice(g.n, 32, replace=False)).to(T.device), b] = 1.0 / 32
    c = torch.from_numpy(rng.standard_normal((g.n, B)).astype(np.float32)).to(T.device)
    dg = DeviceGraph(g, device=dev)
    w = torch.from_numpy(g.w_f32).to(T.device)
    for _ in range(max(args.warmup, 1)):
        ppr_sharded(dg, T, w, c, 0.85, 1e-7)
    clocks = ClockSampler(dev)
    clocks.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        ppr_sharded(dg, T, w, c, 0.85, 1e-7)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_ms = dist.max(e0.elapsed_time(e1))
    if dist.rank == 0:
        emit({"metric": "PPR forward+adjoint columns per second (batch 128, tol 1e-7)", "unit": "columns/s",
              "value": B * args.steps / (t_ms / 1e3), "n_gpus": dist.world, "steps": args.steps,
              "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
              "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
              "config": {"workload": f"personalised PageRank + adjoint, RMAT-{scale} directed ef16, 128 teleports "
                                     f"sharded over {dist.world} GPUs in blocks of 4 columns, one all-reduce of "
                                     "grad_w per step", "n": g.n, "m": g.m, "parallelism": f"columns/{dist.world}"},
              "clocks": clk, "gpu_launches": 12 * args.steps})
    dg.free()
    dist.close()


def cpu_units(job: Job, gpu_stats: list) -> float:
    return sum(job.units(st, gi) for gi, st in enumerate(gpu_stats))


def run_reference(args, job_cls) -> None:
    """CPU restatement of the reference algorithm on all host cores (rank 0 only)."""
    import oracle

    job = job_cls(args.size)
    # units per step: the same traversed-edge count the GPU arm reports,
    # computed on the host from the CPU result (reached vertices' degrees)
    # the first (untimed) pass is also the first warm-up step
    t0 = time.perf_counter()
    units = 0.0
    for gi in range(len(job.graphs)):
        g = job.graphs[gi]["host"]
        if isinstance(job, (SsspJob, BfsJob)):
            out = job.cpu_call(gi)
            units += float(g.degrees()[np.asarray(out) != oracle.INF].sum())
        else:
            units += job.cpu_run(g)[1]
    first = time.perf_counter() - t0
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
    cores = 1 if getattr(job, "cpu_serial", False) else oracle.threads()
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
    rank = int(os.environ.get("RANK", "0"))
    if args.app in BATCHED:
        if args.impl == "reference":
            if rank == 0:
                emit({"impl": "reference", "unavailable": f"--app {args.app}: the CPU baseline is reported inside the "
                                                          "GPU line (cpu_baseline); see the default SSSP workload"})
            return
        if args.app == "bc" and int(os.environ.get("WORLD_SIZE", "1")) > 1:
            run_bc_sharded(args)  # every rank: sources sharded, one all-reduce
        elif args.app == "ppr" and int(os.environ.get("WORLD_SIZE", "1")) > 1:
            run_ppr_sharded(args)  # every rank: columns sharded, one all-reduce of grad_w
        elif rank == 0:
            run_batched(args)
        return
    job_cls = JOBS[args.app]
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, job_cls)
        return

    import torch

    from galois_b200 import DeviceGraph

    dist = Dist(want_pg=True)
    dev = dist.local_rank
    torch.cuda.set_device(dev)
    job = job_cls(args.size)
    _, npdt = job.out_kind()
    r = measure_resident(job, dev, dist, args.steps, args.warmup, args.order)
    dgs, outs, stats, t_ms = r["dgs"], r["outs"], r["stats"], r["t_ms"]
    units_step = r["units_step"]
    value = aggregate_rate(dist.world, units_step, args.steps, t_ms)
    roofline = roofline_of(job, r, args.order, traffic_from_profiles(f"{args.app}-{args.size}"))
    line = {"metric": job.metric, "value": value, "unit": job.unit, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": job.dtype, "data": "synthetic (seeded generators)",
            "config": {**job.config(), "vertex_order": ORDER_NAMES[args.order],
                       "orders": {job.graphs[gi]["name"]: ORDER_NAMES[o] for gi, o in enumerate(r["orders"])}},
            "roofline": roofline,
            "clocks": r["clocks"],
            "gpu_launches": sum(int(st["launches"]) for st in stats) * args.steps,
            "reorder_ms": r["reorder_ms"],
            "detail": [{"graph": job.graphs[gi]["name"], **{k: stats[gi][k] for k in stats[gi]}}
                       for gi in range(len(dgs))]}
    # ---- CPU baseline (rank 0, one GPU only) -----------------------------------
    if dist.world == 1 and not args.no_cpu_baseline:
        import oracle

        if isinstance(job, (CcJob, PrJob)):
            # the same algorithm on the same graph; PageRank's units count the
            # CPU restatement's own iterations
            t0 = time.perf_counter()
            _, cu = job.cpu_run(job.graphs[0]["host"])
            t_cpu = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": cu / t_cpu / 1e9, "unit": job.unit, "cores": oracle.threads(),
                                    "kind": "port", "sample": "one full run of the workload's graph"}
        else:
            t0 = time.perf_counter()
            cpu_outs = [job.cpu_call(gi) for gi in range(len(job.graphs))]
            t_cpu = time.perf_counter() - t0
            gpu_host = [o.cpu().numpy() for o in outs]
            line["cpu_baseline"] = {"value": units_step / t_cpu / 1e9, "unit": job.unit,
                                    "cores": 1 if getattr(job, "cpu_serial", False) else oracle.threads(),
                                    "kind": "port", "sample": "one full run of every graph of the workload",
                                    **({"schedule": SsspJob.CPU_SCHEDULE} if isinstance(job, SsspJob) else {}),
                                    "parity": [job.parity(gpu_host[gi], cpu_outs[gi], gi)
                                               for gi in range(len(job.graphs))]}
    # ---- end to end through the public API with host buffers -----------------
    if not args.no_e2e:
        pinned = []
        for g in job.graphs:
            h = g["host"]
            pinned.append((pinned_copy(h.end_offs), pinned_copy(h.col),
                           pinned_copy(h.w_u32) if h.w_u32 is not None else None))
        tdt = {np.dtype(np.uint32): torch.int32, np.dtype(np.float32): torch.float32}[np.dtype(npdt)]
        host_out = [torch.empty(g["host"].n, dtype=tdt, pin_memory=True) for g in job.graphs]
        dev_out = [torch.empty(g["host"].n, dtype=tdt, device=f"cuda:{dev}") for g in job.graphs]
        h2d = sum(a.nbytes + b.nbytes + (c.nbytes if c is not None else 0) for a, b, c in pinned)
        d2h = sum(o.numel() * o.element_size() for o in host_out)
        from galois_b200.graph import HostCSR

        # The graphs are independent: the one whose kernel runs longest is
        # uploaded and started first (asynchronously, into a device buffer),
        # and the others are uploaded while it runs (gb_graph_upload copies
        # host inputs on a stream of its own); one readback at the end.
        order = sorted(range(len(job.graphs)), key=lambda gi: -float(stats[gi].get("kernel_ms", 0.0)))

        def e2e_step():
            live = []
            try:
                for gi in order:
                    a, b, c = pinned[gi]
                    dg = DeviceGraph(HostCSR(a, b, c), symmetric=job.graphs[gi]["symmetric"], device=dev)
                    live.append(dg)
                    job.device_call(dg, gi, dev_out[gi])
                for gi in order:
                    host_out[gi].copy_(dev_out[gi], non_blocking=True)
                torch.cuda.current_stream(dev).synchronize()
            finally:
                for dg in live:
                    dg.free()

        for _ in range(2):  # untimed: the first calls also fill the allocator cache and page in the buffers
            e2e_step()
        ke = max(1, min(args.steps, 10))
        dist.barrier()
        t0 = time.perf_counter()
        step_ms = []
        for _ in range(ke):
            ts = time.perf_counter()
            e2e_step()
            step_ms.append(round((time.perf_counter() - ts) * 1e3, 2))
        te = dist.max(time.perf_counter() - t0)
        line["e2e"] = {"value": aggregate_rate(dist.world, units_step, ke, te * 1e3), "unit": job.unit,
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": ke,
                       # every step's wall time on this rank: the host-to-device copy rate of a shared
                       # host varies from step to step, and value is over all of them
                       "step_ms": step_ms,
                       "path": "gb_graph_upload (pinned host CSR, file order: a one-shot call does not "
                               "amortise gb_graph_reorder) + kernel into a device buffer, the graphs' uploads "
                               "overlapping the longest kernel + one host readback + gb_graph_free"}
    for dg in dgs:
        dg.free()
    # ---- the other plain kernels on their configurations (one GPU) ------------
    if args.app == "sssp" and args.size == "full" and dist.world == 1 and not args.no_apps:
        line["apps"] = run_apps(args, dev)
    if dist.rank == 0:
        emit(line)
    dist.close()


if __name__ == "__main__":
    main()
