// cc-gpu: lonestar/analytics/cpu/connected-components/ConnectedComponents.cpp
// on the device.  -algo maps the reference's families onto the device
// kernels: LabelProp -> label propagation with pointer jumping; Afforest,
// EdgeAfforest, EdgetiledAfforest -> Afforest sampling + hooking; every other
// name (Serial, Sync, Async, EdgeAsync, EdgetiledAsync (default),
// BlockedAsync) -> union-find hooking.  Requires -symmetricGraph, as the
// reference does.  The component report and the per-edge check follow
// ConnectedComponents.cpp:1100-1155 and 1046-1075.
#include <unordered_map>

#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {});
  if (f.has("help")) {
    std::printf("cc-gpu <input.gr> -symmetricGraph [-algo=LabelProp|Afforest|...] [-noverify] "
                "[-statFile=F] [-t=N]\n");
    return 0;
  }
  if (!f.flag("symmetricGraph")) die("This application requires a symmetric graph input; please use the -symmetricGraph flag to indicate the input is a symmetric graph.");
  const std::string algo = f.str("algo", "EdgetiledAsync");
  int code = GB_CC_UNIONFIND;
  if (algo == "LabelProp") code = GB_CC_LABELPROP;
  else if (algo.find("fforest") != std::string::npos) code = GB_CC_AFFOREST;
  Timer total;
  Loaded L;
  load(f, 0, L);
  const uint32_t n = L.h.n;
  std::printf("Running %s algorithm on the GPU\n", algo.c_str());
  std::vector<uint32_t> label(n);
  gb_stats st{};
  Timer exec;
  check(gb_cc(L.g, code, label.data(), &st, nullptr), "gb_cc");
  const unsigned long long exec_ms = exec.ms();

  // Component report: a representative is a vertex labelled with itself.
  std::unordered_map<uint32_t, uint64_t> sizes;
  uint64_t reps = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (label[v] == v) ++reps;
    else ++sizes[label[v]];
  }
  uint32_t largest_id = 0;
  uint64_t largest = 0;
  for (auto& kv : sizes)
    if (kv.second > largest || (kv.second == largest && kv.first < largest_id)) {
      largest = kv.second;
      largest_id = kv.first;
    }
  const uint64_t largest_size = sizes.empty() ? 1 : largest + 1;
  double ratio = (double)n - (double)reps + (double)sizes.size();
  if (ratio != 0) ratio = (double)largest_size / ratio;
  std::printf("Total components: %llu\n", (unsigned long long)reps);
  std::printf("Number of non-trivial components: %llu (largest size: %llu [%g])\n",
              (unsigned long long)sizes.size(), (unsigned long long)largest_size, ratio);

  if (!f.flag("noverify")) {
    bool ok = true;
    for (uint32_t u = 0; u < n && ok; ++u)
      for (uint64_t e = L.begin(u); e < L.end(u); ++e)
        if (label[L.h.col[e]] != label[u]) {
          std::fprintf(stderr, "not in same component: %u (%u) and %u (%u)\n", u, label[u], L.h.col[e],
                       label[L.h.col[e]]);
          ok = false;
          break;
        }
    if (ok) std::printf("Verification successful.\n");
    else die("verification failed");
  }
  Stats s;
  s.add("CC", "Time", exec_ms);
  s.add("CC", "KernelTimeMs", st.kernel_ms);
  s.add("CC", "Rounds", (unsigned long long)st.rounds);
  s.add("(NULL)", "Time", total.ms());
  s.print(f.str("statFile"));
  return 0;
}
