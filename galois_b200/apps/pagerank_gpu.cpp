// pagerank-gpu: lonestar/analytics/cpu/pagerank/PageRank-pull.cpp (-algo=Topo,
// the default here, or Residual) and PageRank-push.cpp (-algo=Sync) on the
// device.  Pull variants take the TRANSPOSED graph (-transposedGraph, as
// PageRank-pull.cpp:285-296 requires); Sync takes the graph itself.
// Constants as PageRank-constants.h:31-37: alpha 0.85, -tolerance 1e-3,
// -maxIterations 1000; top-20 listing as printTop (PageRank-constants.h:78-108).
#include <algorithm>

#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {"transposedGraph"});
  if (f.has("help")) {
    std::printf("pagerank-gpu <input.gr> [-algo=Topo|Residual|Sync] [-transposedGraph] "
                "[-tolerance=T] [-maxIterations=N] [-noverify] [-statFile=F] [-t=N]\n");
    return 0;
  }
  const std::string algo = f.str("algo", "Topo");
  const bool pull = algo != "Sync";
  if (pull && !f.flag("transposedGraph"))
    die("This application requires a transposed graph input; please use the -transposedGraph flag to indicate the input is a transposed graph.");
  const float tol = (float)f.f64("tolerance", 1.0e-3);
  const uint32_t max_iter = (uint32_t)f.u64("maxIterations", 1000);
  Timer total;
  Loaded L;
  load(f, 0, L);
  const uint32_t n = L.h.n;
  std::printf("Running %s version, tolerance:%g, maxIterations:%u\n", algo.c_str(), tol, max_iter);
  std::vector<float> rank(n);
  uint32_t iters = 0;
  gb_stats st{};
  Timer exec;
  int rc;
  if (algo == "Topo") rc = gb_pagerank_pull(L.g, 0.85f, tol, max_iter, rank.data(), &iters, &st, nullptr);
  else if (algo == "Residual")
    rc = gb_pagerank_pull_residual(L.g, 0.85f, tol, max_iter, rank.data(), &iters, &st, nullptr);
  else if (algo == "Sync") rc = gb_pagerank_push(L.g, 0.85f, tol, max_iter, rank.data(), &iters, &st, nullptr);
  else die("unknown -algo " + algo);
  check(rc, "gb_pagerank");
  const unsigned long long exec_ms = exec.ms();
  if (rc == GB_ERR_NOT_CONVERGED) std::printf("ERROR: failed to converge in %u iterations\n", iters);

  float mx = n ? rank[0] : 0.f, mn = mx;
  float sum = 0.f;
  for (float r : rank) {
    mx = std::max(mx, r);
    mn = std::min(mn, r);
    sum += r;
  }
  info("Max rank is " + std::to_string(mx));
  info("Min rank is " + std::to_string(mn));
  info("Sum is " + std::to_string(sum));
  if (!f.flag("noverify")) {
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    const uint32_t top = std::min<uint32_t>(20, n);
    std::partial_sort(idx.begin(), idx.begin() + top, idx.end(), [&](uint32_t a, uint32_t b) {
      return rank[a] != rank[b] ? rank[a] > rank[b] : a < b;
    });
    std::printf("Rank PageRank Id\n");
    for (uint32_t i = 0; i < top; ++i) std::printf("%u: %g %u\n", i + 1, rank[idx[i]], idx[i]);
  }
  Stats s;
  s.add("PageRank", "Time", exec_ms);
  s.add("PageRank", "KernelTimeMs", st.kernel_ms);
  s.add("PageRank", "Iterations", (unsigned long long)iters);
  s.add("PageRank", "Residual", st.residual);
  s.add("(NULL)", "Time", total.ms());
  s.print(f.str("statFile"));
  return 0;
}
