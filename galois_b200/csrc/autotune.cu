// Autotuner for the frontier and sweep kernels.
//
// The reference leaves CHUNK_SIZE / EDGE_TILE_SIZE as compile-time constants
// to be tuned per machine and input (lonestar/analytics/cpu/bfs/bfs.cpp:85-86,
// sssp/SSSP.cpp:97-98, PageRank-pull.cpp:46; bfs/README.md asks the user to
// tune them).  gb_autotune times a small grid of candidates for one kernel on
// the caller's graph -- degree-bin threshold (heavy_degree), tile size,
// persistent CTA shape, SSSP local relaxation rounds and the BFS push/pull
// switch point -- keeps the fastest in the handle and optionally records it
// in a JSON-lines cache keyed by a coarse graph class, so later runs on the
// same class of graph reuse the choice without timing.

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "device_graph.cuh"

namespace gb {

int run_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats, cudaStream_t s, void* scratch,
            size_t scratch_bytes);
int run_sssp(gb_graph* g, uint32_t src, uint32_t shift, uint32_t* dist_out, gb_stats* stats, cudaStream_t s);
int run_cc(gb_graph* g, int algo, uint32_t* label_out, gb_stats* stats, cudaStream_t s);

namespace {

std::string graph_class(const gb_graph* g) {
  const int lg_n = (int)std::lround(std::log2((double)std::max<uint32_t>(g->n, 1)));
  const int avg = (int)std::lround((double)g->m / std::max<uint32_t>(g->n, 1));
  const int lg_maxd = (int)std::lround(std::log2((double)std::max<uint32_t>(g->max_degree, 1)));
  char buf[128];
  std::snprintf(buf, sizeof(buf), "lgn%d-avg%d-lgmaxd%d-sym%d", lg_n, avg, lg_maxd, g->symmetric);
  return buf;
}

std::string tuning_json(const gb_tuning& t) {
  char buf[256];
  std::snprintf(buf, sizeof(buf),
                "{\"heavy_degree\": %u, \"tile_edges\": %u, \"block_threads\": %u, \"blocks_per_sm\": %u, "
                "\"do_alpha\": %g, \"do_beta\": %g, \"direction_opt\": %d, \"local_depth\": %d, "
                "\"sssp_async\": %d}",
                t.heavy_degree, t.tile_edges, t.block_threads, t.blocks_per_sm, t.do_alpha, t.do_beta,
                t.direction_opt, t.local_depth, t.sssp_async);
  return buf;
}

bool parse_field(const std::string& line, const char* key, double* out) {
  const std::string k = std::string("\"") + key + "\": ";
  const size_t p = line.find(k);
  if (p == std::string::npos) return false;
  *out = std::strtod(line.c_str() + p + k.size(), nullptr);
  return true;
}

bool cache_lookup(const char* path, const std::string& cls, const std::string& kernel, gb_tuning* t) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  bool found = false;
  const std::string want = "\"class\": \"" + cls + "\", \"kernel\": \"" + kernel + "\"";
  while (std::getline(in, line)) {
    if (line.find(want) == std::string::npos) continue;
    double v;
    gb_tuning r{};
    if (parse_field(line, "heavy_degree", &v)) r.heavy_degree = (uint32_t)v;
    if (parse_field(line, "tile_edges", &v)) r.tile_edges = (uint32_t)v;
    if (parse_field(line, "block_threads", &v)) r.block_threads = (uint32_t)v;
    if (parse_field(line, "blocks_per_sm", &v)) r.blocks_per_sm = (uint32_t)v;
    if (parse_field(line, "do_alpha", &v)) r.do_alpha = (float)v;
    if (parse_field(line, "do_beta", &v)) r.do_beta = (float)v;
    if (parse_field(line, "direction_opt", &v)) r.direction_opt = (int)v;
    if (parse_field(line, "local_depth", &v)) r.local_depth = (int)v;
    if (parse_field(line, "sssp_async", &v)) r.sssp_async = (int)v;
    *t = r;
    found = true;  // the last matching line wins
  }
  return found;
}

}  // namespace
}  // namespace gb

extern "C" int gb_autotune(gb_graph* g, const char* kernel, uint32_t src, const char* cache_path, gb_tuning* best_out,
                           void* stream) {
  using namespace gb;
  clear_error();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g || !kernel) GB_FAIL(GB_ERR_ARG, "gb_autotune: null argument");
  const std::string k(kernel);
  if (k != "bfs" && k != "sssp" && k != "cc" && k != "pr")
    GB_FAIL(GB_ERR_ARG, "gb_autotune: kernel must be bfs, sssp, cc or pr");
  if ((k == "bfs" || k == "sssp") && src >= g->n) GB_FAIL(GB_ERR_ARG, "gb_autotune: source %u >= n", src);
  if (k == "sssp" && !g->w) GB_FAIL(GB_ERR_ARG, "gb_autotune: sssp needs uint32 weights");
  if (g->perm && (k == "bfs" || k == "sssp")) src = g->h_iperm[src];  // relabelled graph: internal id
  GB_CUDA(cudaSetDevice(g->device));
  const std::string cls = graph_class(g);
  gb_tuning cached{};
  if (cache_path && cache_lookup(cache_path, cls, k, &cached)) {
    g->tuning = cached;
    if (best_out) *best_out = effective_tuning(g);
    return GB_OK;
  }
  // candidate grid
  std::vector<gb_tuning> cands;
  const gb_tuning base = g->tuning;
  for (uint32_t heavy : {32u, 128u, 512u})
    for (uint32_t tile : {128u, 256u, 512u}) {
      if (tile < heavy / 2) continue;
      gb_tuning t = base;
      t.heavy_degree = heavy;
      t.tile_edges = tile;
      if (k == "sssp") {
        for (int depth : {-1, 2, 8, 16}) {
          t.local_depth = depth;
          t.sssp_async = 0;
          cands.push_back(t);
          if (depth > 0) {  // asynchronous buckets (taken only when every vertex is light),
            t.sssp_async = 1;  // then over fixed-width rows (degree <= 8)
            cands.push_back(t);
            t.sssp_async = 2;
            cands.push_back(t);
            if (g->order == GB_ORDER_LOCALITY) {  // 0 took the regions: also without them
              t.sssp_async = -1;
              cands.push_back(t);
            }
          }
        }
      } else if (k == "bfs") {
        for (float alpha : {5.f, 15.f, 40.f}) {
          t.do_alpha = alpha;
          cands.push_back(t);
        }
      } else {
        cands.push_back(t);
      }
    }
  uint32_t* out = nullptr;
  GB_CUDA(cudaMalloc(&out, sizeof(float) * g->n));
  double best_ms = 1e300;
  gb_tuning best = base;
  int rc = GB_OK;
  for (const gb_tuning& t : cands) {
    g->tuning = t;
    double ms = 1e300;
    for (int rep = 0; rep < 3 && rc == GB_OK; ++rep) {  // first run warms workspaces
      gb_stats st{};
      if (k == "bfs") rc = run_bfs(g, src, out, &st, s, nullptr, 0);
      else if (k == "sssp") rc = run_sssp(g, src, 13, out, &st, s);
      else if (k == "cc") rc = run_cc(g, GB_CC_LABELPROP, out, &st, s);
      else rc = gb_pagerank_pull(g, 0.85f, 1e-6f, 1000, reinterpret_cast<float*>(out), nullptr, &st, s);
      if (rc == GB_ERR_NOT_CONVERGED) rc = GB_OK;
      if (rep > 0) ms = std::min(ms, st.kernel_ms);
    }
    if (rc != GB_OK) break;
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  cudaFree(out);
  g->tuning = rc == GB_OK ? best : base;
  if (rc != GB_OK) return rc;
  if (cache_path) {
    FILE* f = std::fopen(cache_path, "a");
    if (!f) GB_FAIL(GB_ERR_FILE, "gb_autotune: cannot append to %s", cache_path);
    std::fprintf(f, "{\"class\": \"%s\", \"kernel\": \"%s\", \"ms\": %.4f, \"tuning\": %s}\n", cls.c_str(), k.c_str(),
                 best_ms, tuning_json(best).c_str());
    std::fclose(f);
  }
  if (best_out) *best_out = effective_tuning(g);
  return GB_OK;
}
