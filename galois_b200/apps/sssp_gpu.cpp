// sssp-gpu: lonestar/analytics/cpu/sssp/SSSP.cpp on the device.
// Options as SSSP.cpp:40-70: -startNode, -reportNode, -delta (a shift:
// bucket = dist >> delta, default 13), -algo accepted and reported.  The
// graph's edge data is read as uint32 weights (the .gr must carry 4-byte
// edge data, as the reference requires).
#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {});
  if (f.has("help")) {
    std::printf("sssp-gpu <input.gr> [-startNode=N] [-reportNode=N] [-delta=S] "
                "[-noverify] [-statFile=F] [-t=N]\n");
    return 0;
  }
  Timer total;
  Loaded L;
  load(f, 4, L);
  const uint32_t n = L.h.n;
  const uint64_t start = f.u64("startNode", 0), report = f.u64("reportNode", 1);
  if (start >= n || report >= n) {
    std::fprintf(stderr, "failed to set report: %llu or failed to set source: %llu\n",
                 (unsigned long long)report, (unsigned long long)start);
    return 1;
  }
  const uint32_t shift = (uint32_t)f.u64("delta", 13);
  std::printf("INFO: Using delta-step of %u\n", 1u << shift);
  std::printf("Running %s algorithm on the GPU\n", f.str("algo", "deltaStep").c_str());
  std::vector<uint32_t> dist(n);
  gb_stats st{};
  Timer exec;
  check(gb_sssp_delta(L.g, (uint32_t)start, shift, dist.data(), &st, nullptr), "gb_sssp_delta");
  const unsigned long long exec_ms = exec.ms();
  std::printf("Node %llu has distance %u\n", (unsigned long long)report, dist[report]);
  report_distances(dist);
  if (!f.flag("noverify")) {
    if (verify_paths(L, (uint32_t)start, dist, false)) std::printf("Verification successful.\n");
    else die("verification failed");
  }
  Stats s;
  s.add("SSSP", "Time", exec_ms);
  s.add("SSSP", "KernelTimeMs", st.kernel_ms);
  s.add("SSSP", "Buckets", (unsigned long long)st.buckets);
  s.add("SSSP", "Rounds", (unsigned long long)st.rounds);
  s.add("SSSP", "Relaxations", (unsigned long long)st.relaxations);
  s.add("(NULL)", "Time", total.ms());
  s.print(f.str("statFile"));
  return 0;
}
