// lonestar_cli.h -- command-line surface shared by the *-gpu programs.
//
// Mirrors the lonestar boilerplate (lonestar/liblonestar/src/BoilerPlate.cpp:25-41):
// a positional input file, -t, -noverify, -statFile, -symmetricGraph, plus
// each app's own options, written "-name=value", "-name value" or "--name".
// Statistics are printed in the StatManager layout
// (libgalois/src/Statistics.cpp:90-95): a "STAT_TYPE, REGION, CATEGORY,
// TOTAL_TYPE, TOTAL" header, then one "STAT, <region>, <category>, TMAX,
// <value>" line per statistic, to stdout or to -statFile.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "gb.h"

namespace lsapp {

struct Flags {
  std::map<std::string, std::string> kv;
  std::vector<std::string> positional;
  std::vector<std::string> bools;  // names that take no value

  bool has(const std::string& k) const { return kv.count(k) != 0; }
  std::string str(const std::string& k, const std::string& d = "") const {
    auto it = kv.find(k);
    return it == kv.end() ? d : it->second;
  }
  unsigned long long u64(const std::string& k, unsigned long long d) const {
    auto it = kv.find(k);
    return it == kv.end() ? d : std::strtoull(it->second.c_str(), nullptr, 0);
  }
  double f64(const std::string& k, double d) const {
    auto it = kv.find(k);
    return it == kv.end() ? d : std::strtod(it->second.c_str(), nullptr);
  }
  bool flag(const std::string& k) const {
    auto it = kv.find(k);
    return it != kv.end() && it->second != "0" && it->second != "false";
  }
};

// Parse argv.  `bool_names` lists the options that take no value.
inline Flags parse(int argc, char** argv, std::vector<std::string> bool_names) {
  Flags f;
  bool_names.insert(bool_names.end(), {"noverify", "symmetricGraph", "help"});
  f.bools = bool_names;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.size() > 1 && a[0] == '-') {
      a = a.substr(a[1] == '-' ? 2 : 1);
      const size_t eq = a.find('=');
      if (eq != std::string::npos) {
        f.kv[a.substr(0, eq)] = a.substr(eq + 1);
        continue;
      }
      bool is_bool = false;
      for (auto& b : bool_names) is_bool |= (b == a);
      if (is_bool || i + 1 >= argc) f.kv[a] = "1";
      else f.kv[a] = argv[++i];
    } else {
      f.positional.push_back(a);
    }
  }
  return f;
}

[[noreturn]] inline void die(const std::string& what) {
  std::fprintf(stderr, "ERROR: %s\n", what.c_str());
  std::exit(1);
}

inline void check(int st, const char* call) {
  if (st != GB_OK && st != GB_ERR_NOT_CONVERGED) die(std::string(call) + ": " + gb_last_error());
}

inline void info(const std::string& s) { std::printf("INFO: %s\n", s.c_str()); }

// StatManager-style report.
struct Stats {
  struct Row {
    std::string region, category, value;
  };
  std::vector<Row> rows;
  void add(const std::string& region, const std::string& cat, unsigned long long v) {
    rows.push_back({region, cat, std::to_string(v)});
  }
  void add(const std::string& region, const std::string& cat, double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.6g", v);
    rows.push_back({region, cat, b});
  }
  void print(const std::string& stat_file) const {
    FILE* out = stdout;
    if (!stat_file.empty()) {
      out = std::fopen(stat_file.c_str(), "w");
      if (!out) die("cannot open statFile " + stat_file);
    }
    std::fprintf(out, "STAT_TYPE, REGION, CATEGORY, TOTAL_TYPE, TOTAL\n");
    for (auto& r : rows)
      std::fprintf(out, "STAT, %s, %s, TMAX, %s\n", r.region.c_str(), r.category.c_str(), r.value.c_str());
    if (out != stdout) std::fclose(out);
  }
};

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  unsigned long long ms() const {
    return (unsigned long long)std::chrono::duration_cast<std::chrono::milliseconds>(
               std::chrono::steady_clock::now() - t0)
        .count();
  }
};

// Host graph plus its device mirror.
struct Loaded {
  gb_host_csr h;
  gb_graph* g = nullptr;
  Loaded() { gb_host_csr_init(&h); }
  Loaded(const Loaded&) = delete;
  Loaded& operator=(const Loaded&) = delete;
  uint64_t begin(uint32_t v) const { return v ? h.end_offs[v - 1] : 0; }
  uint64_t end(uint32_t v) const { return h.end_offs[v]; }
  ~Loaded() {
    if (g) gb_graph_free(g);
    gb_host_csr_free(&h);
  }
};

inline void load(const Flags& f, int edge_bytes, Loaded& L) {
  if (f.positional.empty()) die("missing <input file>");
  const std::string& path = f.positional[0];
  std::printf("Reading from file: %s\n", path.c_str());
  check(gb_gr_read(path.c_str(), edge_bytes, &L.h), "gb_gr_read");
  std::printf("Read %u nodes, %llu edges\n", L.h.n, (unsigned long long)L.h.m);
  check(gb_graph_upload(L.h.end_offs, L.h.col, L.h.w_u32, L.h.w_f32, L.h.n, L.h.m,
                        f.flag("symmetricGraph") ? 1 : 0, (int)f.u64("device", 0), &L.g),
        "gb_graph_upload");
  // -reorder=1|2|3|4: relabel the device mirror (degree, degree without the row
  // sort, locality, auto); results stay in file ids
  const int order = (int)f.u64("reorder", 0);
  if (order) check(gb_graph_reorder(L.g, order, nullptr), "gb_graph_reorder");
}

// Shortest-path verifier (the check of lonestar's BFS/SSSP verify,
// BFS_SSSP.h:231-263): dist[src] = 0, no arc can still improve a
// distance, and every reached vertex other than src has a tight in-arc.
inline bool verify_paths(const Loaded& L, uint32_t src, const std::vector<uint32_t>& dist, bool unit) {
  const uint32_t n = L.h.n;
  if (dist[src] != 0) return false;
  std::vector<char> tight(n, 0);
  tight[src] = 1;
  for (uint32_t u = 0; u < n; ++u) {
    if (dist[u] == GB_DIST_INFINITY) continue;
    for (uint64_t e = L.begin(u); e < L.end(u); ++e) {
      const uint32_t v = L.h.col[e];
      const uint64_t nd = (uint64_t)dist[u] + (unit ? 1u : L.h.w_u32[e]);
      if ((uint64_t)dist[v] > nd) return false;
      if ((uint64_t)dist[v] == nd) tight[v] = 1;
    }
  }
  for (uint32_t v = 0; v < n; ++v)
    if (dist[v] != GB_DIST_INFINITY && !tight[v]) return false;
  return true;
}

// Sanity lines shared by bfs/sssp (bfs.cpp:380-407).
inline void report_distances(const std::vector<uint32_t>& dist) {
  unsigned long long visited = 0, maxd = 0, sum = 0;
  for (uint32_t d : dist)
    if (d != GB_DIST_INFINITY) {
      ++visited;
      sum += d;
      if (d > maxd) maxd = d;
    }
  info("# visited nodes is " + std::to_string(visited));
  info("Max distance is " + std::to_string(maxd));
  info("Sum of visited distances is " + std::to_string(sum));
}

}  // namespace lsapp
