// bfs-gpu: lonestar/analytics/cpu/bfs/bfs.cpp on the device.
// Options as bfs.cpp:37-62 (-startNode, -reportNode, -algo accepted and
// reported; the device path is the direction-optimizing kernel of gb_bfs),
// plus -symmetricGraph for bottom-up steps without a transpose.
#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {"pushOnly"});
  if (f.has("help")) {
    std::printf("bfs-gpu <input.gr> [-startNode=N] [-reportNode=N] [-symmetricGraph] [-pushOnly] "
                "[-noverify] [-statFile=F] [-t=N]\n");
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
  if (f.flag("pushOnly")) {
    gb_tuning t{};
    check(gb_graph_get_tuning(L.g, &t), "gb_graph_get_tuning");
    t.direction_opt = 2;
    check(gb_graph_set_tuning(L.g, &t), "gb_graph_set_tuning");
  }
  std::printf("Running %s algorithm on the GPU\n", f.str("algo", "DirectionOpt").c_str());
  std::vector<uint32_t> level(n);
  gb_stats st{};
  Timer exec;
  check(gb_bfs(L.g, (uint32_t)start, level.data(), &st, nullptr), "gb_bfs");
  const unsigned long long exec_ms = exec.ms();
  std::printf("Node %llu has distance %u\n", (unsigned long long)report, level[report]);
  report_distances(level);
  if (!f.flag("noverify")) {
    if (verify_paths(L, (uint32_t)start, level, true)) std::printf("Verification successful.\n");
    else die("verification failed");
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
