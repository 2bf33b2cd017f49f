"""The lonestar-style command-line programs (galois_b200/apps/bin/*-gpu) and
the operator-layer example.  CPU tests cover the flag surface and error
paths; GPU tests run each program on a written .gr and compare its report
lines with the oracle."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from galois_b200 import assign_weights_u32, rmat, transpose, write_gr

BIN = Path(__file__).resolve().parents[1] / "galois_b200" / "apps" / "bin"
APPS = ["bfs-gpu", "bfs-directionopt-gpu", "sssp-gpu", "cc-gpu", "pagerank-gpu", "pagerank-push-gpu", "bc-gpu",
        "operator-example"]


def run(app, *args, check=True):
    p = subprocess.run([str(BIN / app), *map(str, args)], capture_output=True, text=True, timeout=300)
    if check and p.returncode != 0:
        raise AssertionError(f"{app} exited {p.returncode}\n{p.stdout}\n{p.stderr}")
    return p


def stats(out: str) -> dict:
    """STAT lines -> {(region, category): value}."""
    lines = out.splitlines()
    assert "STAT_TYPE, REGION, CATEGORY, TOTAL_TYPE, TOTAL" in lines
    d = {}
    for ln in lines:
        if ln.startswith("STAT, "):
            _, region, cat, total_type, val = [x.strip() for x in ln.split(",")]
            assert total_type == "TMAX"
            d[(region, cat)] = float(val)
    return d


@pytest.mark.parametrize("app", APPS[:-1])
def test_app_help(app):
    p = run(app, "-help")
    assert p.stdout.startswith(app)


@pytest.mark.parametrize("app", APPS)
def test_app_missing_file(app, tmp_path):
    p = run(app, tmp_path / "absent.gr", check=False)
    assert p.returncode == 1
    assert "ERROR" in p.stderr


def test_app_flag_contracts(tmp_path):
    # cc needs -symmetricGraph, pull PageRank needs -transposedGraph (as the reference apps)
    p = run("cc-gpu", tmp_path / "x.gr", check=False)
    assert p.returncode == 1 and "symmetric" in p.stderr
    p = run("pagerank-gpu", tmp_path / "x.gr", check=False)
    assert p.returncode == 1 and "transposed" in p.stderr
    # -algo values each app accepts (the pull app's Residual/Topo, the push app's Async/Sync)
    p = run("pagerank-gpu", tmp_path / "x.gr", "-transposedGraph", "-algo=Async", check=False)
    assert p.returncode == 1 and "unknown -algo" in p.stderr
    p = run("pagerank-push-gpu", tmp_path / "x.gr", "-algo=Topo", check=False)
    assert p.returncode == 1 and "unknown -algo" in p.stderr


# ---- GPU --------------------------------------------------------------------------


@pytest.fixture(scope="module")
def graphs(tmp_path_factory):
    d = tmp_path_factory.mktemp("apps")
    g, perm = rmat(12, 8, seed=5)
    g = assign_weights_u32(g, 1, 100, seed=3)
    write_gr(str(d / "g.gr"), g, 4)
    gt, _ = transpose(g)
    write_gr(str(d / "gt.gr"), gt, 0)
    return d, g, gt, int(perm[0])


def _node_line(out, report):
    m = re.search(rf"Node {report} has distance (\d+)", out)
    assert m, out
    return int(m.group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("reorder", [0, 1])
def test_bfs_gpu_app(cuda_device, graphs, reorder):
    d, g, _, src = graphs
    report = int(np.argmax(g.degrees()))
    p = run("bfs-gpu", d / "g.gr", f"-startNode={src}", "-reportNode", report, "-symmetricGraph",
            f"-reorder={reorder}")
    want = oracle.bfs_serial(g, src)
    assert _node_line(p.stdout, report) == int(want[report])
    assert f"# visited nodes is {int((want != oracle.INF).sum())}" in p.stdout
    assert "Verification successful." in p.stdout
    st = stats(p.stdout)
    assert st[("BFS", "Rounds")] >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("sym", [True, False])
def test_bfs_directionopt_gpu_app(cuda_device, graphs, tmp_path, sym):
    d, g, _, src = graphs
    path = d / "g.gr"
    if not sym:
        g, perm = rmat(12, 8, seed=11, symmetrize=False)
        src = int(perm[0])
        path = tmp_path / "dir.gr"
        write_gr(str(path), g, 0)
    report = int(np.argmax(g.degrees()))
    args = [path, f"-startNode={src}", f"-reportNode={report}", "-numPrint=5", "-alpha=15", "-beta=18"]
    p = run("bfs-directionopt-gpu", *args, *(["-symmetricGraph"] if sym else []))
    want = oracle.bfs_parent_min(g, src, oracle.bfs_serial(g, src))
    m = re.search(rf"Node {report} has parent (\d+)", p.stdout)
    assert m and int(m.group(1)) == int(want[report]), p.stdout
    for v in range(5):
        assert f"parent[{v}] : {int(want[v])}" in p.stdout
    assert "Verification successful." in p.stdout


@pytest.mark.gpu
def test_sssp_gpu_app(cuda_device, graphs, tmp_path):
    d, g, _, src = graphs
    p = run("sssp-gpu", d / "g.gr", f"-startNode={src}", "-reportNode=7", "-delta=4",
            f"-statFile={tmp_path / 'st.txt'}")
    want = oracle.sssp_dijkstra(g, src)
    assert _node_line(p.stdout, 7) == int(want[7])
    reached = want != oracle.INF
    assert f"Sum of visited distances is {int(want[reached].astype(np.uint64).sum())}" in p.stdout
    assert "Verification successful." in p.stdout
    st = stats((tmp_path / "st.txt").read_text())
    assert st[("SSSP", "Buckets")] >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("algo,reorder", [("LabelProp", 0), ("Afforest", 0), ("EdgetiledAsync", 0),
                                          ("LabelProp", 1), ("Afforest", 2)])
def test_cc_gpu_app(cuda_device, graphs, algo, reorder):
    d, g, _, _ = graphs
    p = run("cc-gpu", d / "g.gr", "-symmetricGraph", f"-algo={algo}", f"-reorder={reorder}")
    lab = oracle.cc_union_find(g)
    assert f"Total components: {len(np.unique(lab))}" in p.stdout
    assert "Verification successful." in p.stdout


@pytest.mark.gpu
def test_pagerank_gpu_app(cuda_device, graphs):
    d, _, gt, _ = graphs
    p = run("pagerank-gpu", d / "gt.gr", "-transposedGraph", "-tolerance=1e-6", "-algo=Topo")
    want, _ = oracle.pr_pull_topo_f64(gt, 0.85, 1e-6, 1000)
    top = [ln.split() for ln in p.stdout.split("Rank PageRank Id\n")[1].splitlines()[:5]]
    for _, val, vid in top:
        assert abs(float(val) - want[int(vid)]) <= 1e-5
    assert int(top[0][2]) == int(np.argmax(want))
    assert stats(p.stdout)[("PageRank", "Iterations")] >= 1


@pytest.mark.gpu
def test_pagerank_apps_default_algorithms(cuda_device, graphs):
    """The defaults of the reference apps: pull runs Residual
    (PageRank-pull.cpp:34-37), push runs Async (PageRank-push.cpp:42-47).
    At tolerance 1e-7 both list the top vertices of the FP64 fixed point
    x = (1 - alpha) + alpha * sum x[u] / nout[u] within 1e-5 relative."""
    d, _, gt, _ = graphs
    xstar, _ = oracle.pr_pull_topo_f64(gt, 0.85, 1e-15, 5000)
    xstar *= gt.n
    for app, args, algo in (("pagerank-gpu", ["-transposedGraph"], "Residual"), ("pagerank-push-gpu", [], "Async")):
        # the push app reads the graph itself: on this symmetric graph, the same file
        p = run(app, d / "gt.gr", *args, "-tolerance=1e-7")
        assert f"Running {algo} version" in p.stdout, p.stdout
        top = [ln.split() for ln in p.stdout.split("Rank PageRank Id\n")[1].splitlines()[:5]]
        for _, val, vid in top:
            want = xstar[int(vid)]
            assert abs(float(val) - want) <= 1e-5 * max(1.0, want), (app, vid)


@pytest.mark.gpu
def test_bc_gpu_app(cuda_device, graphs, tmp_path):
    d, g, _, _ = graphs
    srcs = [int(x) for x in np.argsort(-g.degrees(), kind="stable")[:40]]
    (tmp_path / "srcs.txt").write_text(" ".join(map(str, srcs)))
    p = run("bc-gpu", d / "g.gr", f"-sourcesToUse={tmp_path / 'srcs.txt'}", "-numOfSources=40", "-output",
            "-symmetricGraph")
    want = oracle.bc_level(g, srcs, f64=True)
    got = np.zeros(g.n)
    for ln in p.stdout.splitlines():
        parts = ln.split()
        if len(parts) == 2 and parts[0].isdigit():
            got[int(parts[0])] = float(parts[1])
    # per vertex, relative to max(|fp64|, 1): the -output lines carry 9 decimals
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1.0)) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("delta", [13, 4])
def test_operator_example(cuda_device, graphs, tmp_path, delta):
    """The operator layer (gb::for_each_edge with gb::wl<gb::FIFO>() for the
    asynchronous BFS operator and gb::wl<gb::DeltaBuckets>(delta) for the
    SSSP operator of SSSP.cpp:134-161) against the oracle, bit-exact: the
    RMAT graph of the other app tests, and a star of 5000 leaves (its hub's
    arcs run as 1024-arc tiles) joined to a path."""
    from galois_b200 import HostCSR

    d, g, _, src = graphs
    k = 5000
    s_ = [0] * k + list(range(1, k + 1)) + list(range(k, k + 99)) + list(range(k + 1, k + 100))
    t_ = list(range(1, k + 1)) + [0] * k + list(range(k + 1, k + 100)) + list(range(k, k + 99))
    star = HostCSR.from_edges(k + 100, s_, t_)
    star = assign_weights_u32(star, 1, 255, seed=9)
    write_gr(str(tmp_path / "star.gr"), star, 4)
    for path, gg, source in ((d / "g.gr", g, src), (tmp_path / "star.gr", star, 0), (tmp_path / "star.gr", star, k + 50)):
        out = tmp_path / "res.bin"
        p = run("operator-example", path, f"-startNode={source}", f"-delta={delta}", f"-output={out}")
        assert "Verification successful." in p.stdout
        res = np.fromfile(out, dtype=np.uint32)
        assert np.array_equal(res[:gg.n], oracle.bfs_serial(gg, source)), path
        assert np.array_equal(res[gg.n:], oracle.sssp_dijkstra(gg, source)), path
