// bfs-directionopt-gpu: lonestar/analytics/cpu/bfs/bfsDirectionOpt.cpp on the
// device.  Options as bfsDirectionOpt.cpp:42-108 (-startNode, -reportNode,
// -alpha, -beta, -numPrint, -numRuns; -exec, -algo and -preAlloc accepted and
// reported), plus -symmetricGraph (in-edges are then the stored arcs; a
// directed input gets its transpose built on the device).  Like the
// reference it prints "Node r has parent p" and, unless -noverify, the
// parents of the first numPrint nodes (:507-517); it also checks that the
// parents form a BFS tree of the source.
#include <algorithm>

#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {});
  if (f.has("help")) {
    std::printf("bfs-directionopt-gpu <input.gr> [-startNode=N] [-reportNode=N] [-alpha=15] [-beta=18] "
                "[-numPrint=10] [-numRuns=1] [-symmetricGraph] [-noverify] [-statFile=F] [-t=N]\n");
    return 0;
  }
  Timer total;
  Loaded L;
  load(f, 0, L);
  const uint32_t n = L.h.n;
  const uint64_t start = f.u64("startNode", 0), report = f.u64("reportNode", 1);
  if (start >= n || report >= n) {
    std::fprintf(stderr, "failed to set report: %llu or failed to set source: %llu\n",
                 (unsigned long long)report, (unsigned long long)start);
    return 1;
  }
  gb_tuning t{};
  check(gb_graph_get_tuning(L.g, &t), "gb_graph_get_tuning");
  t.do_alpha = (float)f.u64("alpha", 15);  // bfsDirectionOpt.cpp:68-72
  t.do_beta = (float)f.u64("beta", 18);    // :73-77
  check(gb_graph_set_tuning(L.g, &t), "gb_graph_set_tuning");
  std::printf("Running %s algorithm with PARALLEL execution on the GPU\n", f.str("algo", "SyncDO").c_str());
  std::printf("WARNING: This bfs version assigns parent instead of the shortest distance from source\n");
  const uint64_t runs = std::max<uint64_t>(1, f.u64("numRuns", 1));
  std::vector<uint32_t> parent(n), level(n);
  gb_stats st{};
  Timer exec;
  for (uint64_t r = 0; r < runs; ++r)
    check(gb_bfs_parent(L.g, (uint32_t)start, parent.data(), level.data(), &st, nullptr), "gb_bfs_parent");
  const unsigned long long exec_ms = exec.ms();
  std::printf("Node %llu has parent %u\n", (unsigned long long)report, parent[report]);
  if (!f.flag("noverify")) {
    const uint64_t np = std::min<uint64_t>(f.u64("numPrint", 10), n);
    for (uint64_t v = 0; v < np; ++v) std::printf("parent[%llu] : %u\n", (unsigned long long)v, parent[v]);
    // a BFS tree: levels exact, every reached non-source vertex hangs off an
    // arc from a vertex one level closer
    if (!verify_paths(L, (uint32_t)start, level, true)) die("verification failed: levels");
    for (uint32_t v = 0; v < n; ++v) {
      if (v == start) {
        if (parent[v] != 0) die("verification failed: source parent");
        continue;
      }
      if (level[v] == GB_DIST_INFINITY) {
        if (parent[v] != GB_DIST_INFINITY) die("verification failed: unreached vertex has a parent");
        continue;
      }
      const uint32_t p = parent[v];
      bool ok = p < n && level[p] + 1 == level[v];
      bool arc = false;
      for (uint64_t i = ok ? L.begin(p) : 0; ok && i < L.end(p) && !arc; ++i) arc = L.h.col[i] == v;
      if (!(ok && arc)) die("verification failed: parent of " + std::to_string(v));
    }
    std::printf("Verification successful.\n");
  }
  Stats s;
  s.add("BFS", "Time", exec_ms);
  s.add("BFS", "KernelTimeMs", st.kernel_ms);
  s.add("BFS", "Rounds", (unsigned long long)st.rounds);
  s.add("BFS", "PullRounds", (unsigned long long)st.pull_rounds);
  s.add("BFS", "EdgesScanned", (unsigned long long)st.edges_scanned);
  s.add("(NULL)", "Time", total.ms());
  s.print(f.str("statFile"));
  return 0;
}
