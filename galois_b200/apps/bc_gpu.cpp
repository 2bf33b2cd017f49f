// bc-gpu: lonestar/analytics/cpu/betweennesscentrality (-algo=Level,
// LevelStructs.h:224-326) on the device.  Sources as the reference picks them
// (LevelStructs.h:253-297): -sourcesToUse=<file of ids>, else 0..numOfSources-1
// (-numOfSources=0 means every vertex), or just -startNode with
// -singleSource.  -batch sets the sources per multi-source launch (1..64,
// default 64; batches need -symmetricGraph, else one source per launch).  Sanity lines and -output as LevelStructs.h:195-217, 314-323.
#include <algorithm>
#include <fstream>
#include <iterator>

#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {"singleSource", "output"});
  if (f.has("help")) {
    std::printf("bc-gpu <input.gr> [-numOfSources=N] [-sourcesToUse=F] [-singleSource -startNode=N] "
                "[-batch=B] [-output] [-statFile=F] [-t=N]\n");
    return 0;
  }
  Timer total;
  Loaded L;
  load(f, 0, L);
  const uint32_t n = L.h.n;
  std::vector<uint32_t> srcs;
  if (f.flag("singleSource")) {
    srcs.push_back((uint32_t)f.u64("startNode", 0));
  } else {
    uint64_t loop_end = f.u64("numOfSources", 0);
    if (loop_end == 0) loop_end = n;
    std::vector<uint64_t> file_srcs;
    if (f.has("sourcesToUse")) {
      std::ifstream in(f.str("sourcesToUse"));
      if (!in) die("cannot open sourcesToUse file " + f.str("sourcesToUse"));
      file_srcs.assign(std::istream_iterator<uint64_t>{in}, std::istream_iterator<uint64_t>{});
    }
    if (!file_srcs.empty()) {
      loop_end = std::min<uint64_t>(loop_end, file_srcs.size());
      for (uint64_t i = 0; i < loop_end; ++i) srcs.push_back((uint32_t)file_srcs[i]);
    } else {
      loop_end = std::min<uint64_t>(loop_end, n);
      for (uint64_t i = 0; i < loop_end; ++i) srcs.push_back((uint32_t)i);
    }
  }
  for (uint32_t s : srcs)
    if (s >= n) die("source " + std::to_string(s) + " is not a vertex");
  uint32_t batch = (uint32_t)f.u64("batch", 64);
  if (batch > 1 && !f.flag("symmetricGraph")) {
    // the multi-source kernels pull over in-edges, which only a symmetric graph has without a transpose
    info("multi-source batches need -symmetricGraph; running one source per launch");
    batch = 1;
  }
  info("Running level BC on the GPU with " + std::to_string(srcs.size()) + " sources, batch " +
       std::to_string(batch));
  std::vector<float> bc(n);
  gb_stats st{};
  Timer exec;
  check(gb_bc(L.g, srcs.data(), (uint32_t)srcs.size(), batch, bc.data(), &st, nullptr), "gb_bc");
  const unsigned long long exec_ms = exec.ms();
  float mx = n ? bc[0] : 0.f, mn = mx, sum = 0.f;
  for (float x : bc) {
    mx = std::max(mx, x);
    mn = std::min(mn, x);
    sum += x;
  }
  std::printf("Max BC is %g\nMin BC is %g\nBC sum is %g\n", mx, mn, sum);
  if (f.flag("output"))
    for (uint32_t v = 0; v < n; ++v) std::printf("%u %.9f\n", v, bc[v]);
  Stats s;
  s.add("BC", "Timer_0", exec_ms);
  s.add("BC", "KernelTimeMs", st.kernel_ms);
  s.add("BC", "Launches", (unsigned long long)st.launches);
  s.add("(NULL)", "Time", total.ms());
  s.print(f.str("statFile"));
  return 0;
}
