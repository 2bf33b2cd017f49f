// The lonestar PageRank apps on the device, shared by pagerank-gpu (the pull
// app, lonestar/analytics/cpu/pagerank/PageRank-pull.cpp: -algo=Residual,
// the default, or Topo; TRANSPOSED input, -transposedGraph, as
// PageRank-pull.cpp:285-296 requires) and pagerank-push-gpu (the push app,
// PageRank-push.cpp: -algo=Async, the default, or Sync; the graph itself).
// Constants as PageRank-constants.h:31-37: alpha 0.85, -tolerance 1e-3,
// -maxIterations 1000 (round-based variants only); top-20 listing as printTop
// (PageRank-constants.h:78-108).
#pragma once

#include <algorithm>

#include "lonestar_cli.h"

inline int pagerank_app(int argc, char** argv, bool push_app) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {"transposedGraph"});
  if (f.has("help")) {
    if (push_app)
      std::printf("pagerank-push-gpu <input.gr> [-algo=Async|Sync] [-tolerance=T] [-maxIterations=N] "
                  "[-noverify] [-statFile=F] [-t=N]\n");
    else
      std::printf("pagerank-gpu <input.gr> [-algo=Residual|Topo] [-transposedGraph] [-tolerance=T] "
                  "[-maxIterations=N] [-noverify] [-statFile=F] [-t=N]\n");
    return 0;
  }
  // defaults as the reference apps: pull Residual (PageRank-pull.cpp:34-37),
  // push Async (PageRank-push.cpp:42-47)
  const std::string algo = f.str("algo", push_app ? "Async" : "Residual");
  if (push_app ? (algo != "Async" && algo != "Sync") : (algo != "Residual" && algo != "Topo"))
    die("unknown -algo " + algo);
  const bool pull = !push_app;
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
  else
    rc = gb_pagerank_push_ex(L.g, algo == "Async" ? GB_PR_PUSH_ASYNC : GB_PR_PUSH_SYNC, 0.85f, tol, max_iter,
                             rank.data(), &iters, &st, nullptr);
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
