// ORACLE -- test infrastructure only.  Nothing in the product links or calls
// this file; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// use it as the checker and as the timed CPU restatement of the reference.
//
// CPU restatement (C++17 + OpenMP) of the Galois lonestar algorithms on the
// CSR edge-map path.  Every function takes the LC_CSR_Graph layout: n END
// offsets (begin(v) = v ? end[v-1] : 0, LC_CSR_Graph.h:142,172-178), uint32
// destinations and optional uint32 weights.
//
// Pinning: the reference cannot be compiled here (Boost, LLVM CommandLine and
// fmt are absent; the GPU apps need the un-vendored moderngpu submodule) and
// its tests hold no golden outputs for this path (only in-app verifiers), so
// this restatement is pinned by (a) the reference's own verifiers, restated
// below (BFS_SSSP.h:231-263, ConnectedComponents.cpp:1046-1072) and run on
// every output, (b) closed-form known answers (paths, stars, grids, cliques)
// in tests/test_oracle.py, (c) agreement between independent formulations
// (serial queue BFS vs SyncTile, Dijkstra vs serial delta-step vs bucketed
// delta-step, union-find vs label propagation, FP64 vs FP32 PageRank).
// BFS levels, SSSP distances and min-id CC labels are unique, so any correct
// algorithm is an exact oracle for them; PageRank and BC are tolerance-checked.

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <queue>
#include <random>
#include <vector>

namespace {

constexpr uint32_t kInf = 2147483646u;  // BFS_SSSP.h:31-32

struct Csr {
  uint32_t n;
  const uint64_t* end;
  const uint32_t* col;
  uint64_t b(uint32_t v) const { return v ? end[v - 1] : 0; }
  uint64_t e(uint32_t v) const { return end[v]; }
};

inline uint32_t atomic_min_u32(uint32_t* p, uint32_t v) {
  uint32_t old = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v < old && !__atomic_compare_exchange_n(p, &old, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
  return old;
}

inline float atomic_add_f32(float* p, float d) {
  // CAS-loop float add, as PageRank-constants.h:70-76
  uint32_t* q = reinterpret_cast<uint32_t*>(p);
  uint32_t old = __atomic_load_n(q, __ATOMIC_RELAXED);
  for (;;) {
    float of;
    std::memcpy(&of, &old, 4);
    const float nf = of + d;
    uint32_t nu;
    std::memcpy(&nu, &nf, 4);
    if (__atomic_compare_exchange_n(q, &old, nu, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return of;
  }
}

inline void atomic_add_f64(double* p, double d) {
  uint64_t* q = reinterpret_cast<uint64_t*>(p);
  uint64_t old = __atomic_load_n(q, __ATOMIC_RELAXED);
  for (;;) {
    double of;
    std::memcpy(&of, &old, 8);
    const double nf = of + d;
    uint64_t nu;
    std::memcpy(&nu, &nf, 8);
    if (__atomic_compare_exchange_n(q, &old, nu, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
  }
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int t) {
  if (t > 0) omp_set_num_threads(t);
}

// ---- BFS --------------------------------------------------------------------

// Serial queue BFS: ground truth for levels.
void orc_bfs_serial(uint32_t n, const uint64_t* end, const uint32_t* col, uint32_t src, uint32_t* level) {
  Csr g{n, end, col};
  for (uint32_t v = 0; v < n; ++v) level[v] = kInf;
  std::vector<uint32_t> q;
  q.reserve(n);
  level[src] = 0;
  q.push_back(src);
  for (size_t h = 0; h < q.size(); ++h) {
    const uint32_t v = q[h];
    for (uint64_t i = g.b(v); i < g.e(v); ++i) {
      const uint32_t u = col[i];
      if (level[u] == kInf) {
        level[u] = level[v] + 1;
        q.push_back(u);
      }
    }
  }
}

// SyncTile BFS (bfs.cpp:244-293 with EDGE_TILE_SIZE 256 :86, tiles from
// BFS_SSSP.h:81-101): level-synchronous; the next frontier is a bag of edge
// tiles of newly reached vertices.  Parallel with OpenMP (timed baseline).
void orc_bfs_sync_tile(uint32_t n, const uint64_t* end, const uint32_t* col, uint32_t src, uint32_t* level) {
  Csr g{n, end, col};
  constexpr uint64_t kTile = 256;
  struct Tile {
    uint64_t beg, end;
  };
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) level[v] = kInf;
  level[src] = 0;
  auto push_tiles = [&](std::vector<Tile>& out, uint32_t v) {
    uint64_t b = g.b(v);
    const uint64_t e = g.e(v);
    if (e - b > kTile)
      for (; b + kTile < e; b += kTile) out.push_back({b, b + kTile});
    if (e > b) out.push_back({b, e});
  };
  std::vector<Tile> curr, next;
  push_tiles(next, src);
  uint32_t next_level = 0;
  const int nt = omp_get_max_threads();
  std::vector<std::vector<Tile>> local(nt);
  while (!next.empty()) {
    std::swap(curr, next);
    next.clear();
    ++next_level;
#pragma omp parallel
    {
      auto& out = local[omp_get_thread_num()];
      out.clear();
#pragma omp for schedule(dynamic, 256)
      for (int64_t t = 0; t < (int64_t)curr.size(); ++t) {
        for (uint64_t i = curr[t].beg; i < curr[t].end; ++i) {
          const uint32_t u = col[i];
          uint32_t expect = kInf;
          // dstData == INF -> dstData = nextLevel; push (bfs.cpp:280-288); the
          // CAS keeps one pusher per vertex
          if (__atomic_load_n(&level[u], __ATOMIC_RELAXED) == kInf &&
              __atomic_compare_exchange_n(&level[u], &expect, next_level, false, __ATOMIC_RELAXED,
                                          __ATOMIC_RELAXED))
            push_tiles(out, u);
        }
      }
    }
    for (auto& l : local) next.insert(next.end(), l.begin(), l.end());
  }
}

// BFS_SSSP::verify (BFS_SSSP.h:231-263) for unit weights plus the converse
// (every reached vertex other than the source has a tight predecessor).
// Returns 0 when the levels are the exact BFS levels.
int orc_verify_bfs(uint32_t n, const uint64_t* end, const uint32_t* col, uint32_t src, const uint32_t* level) {
  Csr g{n, end, col};
  if (level[src] != 0) return 1;
  std::vector<uint8_t> tight(n, 0);
  tight[src] = 1;
  for (uint32_t v = 0; v < n; ++v) {
    if (level[v] == kInf) continue;
    for (uint64_t i = g.b(v); i < g.e(v); ++i) {
      const uint32_t u = col[i];
      if (level[u] > level[v] + 1) return 2;
      if (level[u] == level[v] + 1) tight[u] = 1;
    }
  }
  for (uint32_t v = 0; v < n; ++v)
    if (level[v] != kInf && !tight[v]) return 3;
  return 0;
}

// ---- BFS parents (bfsDirectionOpt.cpp) ---------------------------------------

// Direction-optimising BFS storing parents, serial: syncDOAlgo
// (bfsDirectionOpt.cpp:204-342) with CONCURRENT = false.  The source's datum
// is 0 (:229, :448), unreached vertices keep DIST_INFINITY.  One work counter
// runs through both kinds of step as in the reference: it starts at 1 (:237);
// a push step (:303-337) resets it and adds the out-degree of every vertex
// it reaches, giving each unvisited target the scanning vertex as parent
// (the compare-and-swap of :325 always wins serially), and scout_count takes
// its value; a pull step (:262-300) saves it, resets it and counts the
// vertices it reaches, each unvisited vertex taking its first in-neighbour
// (in in-arc order) that is in the frontier bitset (:276-290).  Pull steps
// repeat while the count does not shrink or stays above n / beta (:299-300);
// the switch to pull is scout_count > edges_to_check / alpha (:259).  alpha
// and beta are ints (:68-77), so both tests divide as integers.
void orc_bfs_do_parent(uint32_t n, const uint64_t* end, const uint32_t* col, const uint64_t* in_end,
                       const uint32_t* in_col, uint32_t src, int alpha, int beta, uint32_t* parent) {
  Csr g{n, end, col}, t{n, in_end, in_col};
  for (uint32_t v = 0; v < n; ++v) parent[v] = kInf;
  parent[src] = 0;
  std::vector<uint32_t> curr, next{src};
  std::vector<uint8_t> front(n, 0), nextb(n, 0);
  uint64_t work_items = 1;
  int64_t edges_to_check = (int64_t)(n ? end[n - 1] : 0);
  int64_t scout = (int64_t)(g.e(src) - g.b(src));
  while (!next.empty()) {
    std::swap(curr, next);
    next.clear();
    if (scout > edges_to_check / alpha) {
      std::fill(front.begin(), front.end(), 0);
      for (uint32_t v : curr) front[v] = 1;
      uint64_t old_items = 0;
      do {
        old_items = work_items;
        work_items = 0;
        for (uint32_t v = 0; v < n; ++v) {
          if (parent[v] != kInf) continue;
          for (uint64_t i = t.b(v); i < t.e(v); ++i) {
            const uint32_t u = in_col[i];
            if (front[u]) {
              parent[v] = u;
              nextb[v] = 1;
              ++work_items;
              break;
            }
          }
        }
        std::swap(front, nextb);
        std::fill(nextb.begin(), nextb.end(), 0);
      } while (work_items >= old_items || work_items > (uint64_t)n / (uint64_t)beta);
      for (uint32_t v = 0; v < n; ++v)
        if (front[v]) next.push_back(v);
      scout = 1;
    } else {
      edges_to_check -= scout;
      work_items = 0;
      for (uint32_t v : curr) {
        for (uint64_t i = g.b(v); i < g.e(v); ++i) {
          const uint32_t u = col[i];
          if (parent[u] == kInf) {
            parent[u] = v;
            next.push_back(u);
            work_items += g.e(u) - g.b(u);
          }
        }
      }
      scout = (int64_t)work_items;
    }
  }
}

// The canonical parent tree of a BFS: every reached v other than src gets
// the smallest id u over its in-neighbours with level[u] == level[v] - 1;
// src gets 0, unreached vertices INF.
void orc_bfs_parent_min(uint32_t n, const uint64_t* in_end, const uint32_t* in_col, const uint32_t* level,
                        uint32_t src, uint32_t* parent) {
  Csr t{n, in_end, in_col};
  for (uint32_t v = 0; v < n; ++v) {
    if (v == src) {
      parent[v] = 0;
      continue;
    }
    uint32_t best = kInf;
    if (level[v] != kInf)
      for (uint64_t i = t.b(v); i < t.e(v); ++i) {
        const uint32_t u = in_col[i];
        if (level[u] + 1 == level[v] && u < best) best = u;
      }
    parent[v] = best;
  }
}

// A parent array is a BFS tree of src when parent[src] == 0, every other
// vertex reached by the levels names an in-neighbour one level closer, and
// unreached vertices hold INF.  Returns 0 when valid.
int orc_verify_bfs_parent(uint32_t n, const uint64_t* in_end, const uint32_t* in_col, const uint32_t* level,
                          uint32_t src, const uint32_t* parent) {
  Csr t{n, in_end, in_col};
  if (parent[src] != 0) return 1;
  for (uint32_t v = 0; v < n; ++v) {
    if (v == src) continue;
    if (level[v] == kInf) {
      if (parent[v] != kInf) return 2;
      continue;
    }
    const uint32_t p = parent[v];
    if (p >= n || level[p] + 1 != level[v]) return 3;
    bool arc = false;
    for (uint64_t i = t.b(v); i < t.e(v) && !arc; ++i) arc = in_col[i] == p;
    if (!arc) return 4;
  }
  return 0;
}

// ---- SSSP -------------------------------------------------------------------

// Dijkstra (SSSP.cpp:223-261): ground truth.
void orc_sssp_dijkstra(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* w, uint32_t src,
                       uint32_t* dist) {
  Csr g{n, end, col};
  for (uint32_t v = 0; v < n; ++v) dist[v] = kInf;
  using Item = std::pair<uint32_t, uint32_t>;  // (dist, node): UpdateRequest order, BFS_SSSP.h:37-48
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> pq;
  dist[src] = 0;
  pq.push({0, src});
  while (!pq.empty()) {
    auto [d, v] = pq.top();
    pq.pop();
    if (dist[v] < d) continue;  // empty work
    for (uint64_t i = g.b(v); i < g.e(v); ++i) {
      const uint32_t u = col[i];
      const uint32_t nd = d + w[i];
      if (nd < dist[u]) {
        dist[u] = nd;
        pq.push({nd, u});
      }
    }
  }
}

// Serial delta-stepping (serDeltaAlgo, SSSP.cpp:175-221): buckets dist>>shift.
void orc_sssp_delta_serial(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* w,
                           uint32_t src, uint32_t shift, uint32_t* dist) {
  Csr g{n, end, col};
  for (uint32_t v = 0; v < n; ++v) dist[v] = kInf;
  std::vector<std::deque<std::pair<uint32_t, uint32_t>>> buckets(1);
  dist[src] = 0;
  buckets[0].push_back({src, 0});
  for (size_t k = 0; k < buckets.size(); ++k) {
    while (!buckets[k].empty()) {
      auto [v, d] = buckets[k].front();
      buckets[k].pop_front();
      if (dist[v] < d) continue;
      for (uint64_t i = g.b(v); i < g.e(v); ++i) {
        const uint32_t u = col[i];
        const uint32_t nd = d + w[i];
        if (nd < dist[u]) {
          dist[u] = nd;
          const size_t b = nd >> shift;
          if (b >= buckets.size()) buckets.resize(b + 1);
          buckets[b].push_back({u, nd});
        }
      }
    }
  }
}

// Bucketed parallel delta-stepping (deltaStepAlgo, SSSP.cpp:118-173, OBIM
// indexer dist >> shift, BFS_SSSP.h:50-58): the current bucket is drained in
// parallel rounds; improvements inside the bucket join the next round, others
// are filed into their bucket.  Timed CPU baseline.
void orc_sssp_delta_parallel(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* w,
                             uint32_t src, uint32_t shift, uint32_t* dist) {
  Csr g{n, end, col};
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) dist[v] = kInf;
  dist[src] = 0;
  std::vector<std::vector<uint32_t>> buckets(1, std::vector<uint32_t>{src});
  const int nt = omp_get_max_threads();
  std::vector<std::vector<uint32_t>> near_local(nt);
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> far_local(nt);
  for (size_t k = 0; k < buckets.size(); ++k) {
    std::vector<uint32_t> cur;
    cur.swap(buckets[k]);
    while (!cur.empty()) {
#pragma omp parallel
      {
        const int t = omp_get_thread_num();
        near_local[t].clear();
        far_local[t].clear();
#pragma omp for schedule(dynamic, 64)
        for (int64_t j = 0; j < (int64_t)cur.size(); ++j) {
          const uint32_t v = cur[j];
          const uint32_t d = __atomic_load_n(&dist[v], __ATOMIC_RELAXED);
          if ((d >> shift) != k) continue;  // stale: settled in an earlier bucket
          for (uint64_t i = g.b(v); i < g.e(v); ++i) {
            const uint32_t u = col[i];
            const uint32_t nd = d + w[i];
            const uint32_t old = atomic_min_u32(&dist[u], nd);
            if (nd < old) {
              if ((nd >> shift) == k) near_local[t].push_back(u);
              else far_local[t].push_back({u, nd >> shift});
            }
          }
        }
      }
      cur.clear();
      for (auto& l : near_local) cur.insert(cur.end(), l.begin(), l.end());
      for (auto& l : far_local)
        for (auto& [u, b] : l) {
          if (b >= buckets.size()) buckets.resize(b + 1);
          buckets[b].push_back(u);
        }
    }
  }
}

// BFS_SSSP::verify (BFS_SSSP.h:231-263) for weighted graphs plus tightness:
// 0 iff dist holds exact shortest distances.
int orc_verify_sssp(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* w, uint32_t src,
                    const uint32_t* dist) {
  Csr g{n, end, col};
  if (dist[src] != 0) return 1;
  std::vector<uint8_t> tight(n, 0);
  tight[src] = 1;
  for (uint32_t v = 0; v < n; ++v) {
    if (dist[v] == kInf) continue;
    for (uint64_t i = g.b(v); i < g.e(v); ++i) {
      const uint32_t u = col[i];
      const uint64_t nd = (uint64_t)dist[v] + w[i];
      if ((uint64_t)dist[u] > nd) return 2;
      if ((uint64_t)dist[u] == nd) tight[u] = 1;
    }
  }
  for (uint32_t v = 0; v < n; ++v)
    if (dist[v] != kInf && !tight[v]) return 3;
  return 0;
}

// ---- connected components -----------------------------------------------------

// Serial union-find (SerialAlgo, ConnectedComponents.cpp:156-181) with the
// component labelled by its minimum vertex id (what LabelProp converges to).
void orc_cc_union_find(uint32_t n, const uint64_t* end, const uint32_t* col, uint32_t* label) {
  Csr g{n, end, col};
  std::vector<uint32_t> p(n);
  for (uint32_t v = 0; v < n; ++v) p[v] = v;
  auto find = [&](uint32_t x) {
    while (p[x] != x) {
      p[x] = p[p[x]];
      x = p[x];
    }
    return x;
  };
  for (uint32_t v = 0; v < n; ++v)
    for (uint64_t i = g.b(v); i < g.e(v); ++i) {
      uint32_t a = find(v), b = find(col[i]);
      if (a == b) continue;
      if (a < b) p[b] = a;  // smaller id becomes the root
      else p[a] = b;
    }
  for (uint32_t v = 0; v < n; ++v) label[v] = find(v);
}

// LabelPropAlgo (ConnectedComponents.cpp:183-230; init :1162-1172):
// comp_current = id, comp_old = INF; a vertex whose comp_old > comp_current
// pushes comp_current to its neighbours with atomicMin; repeat until no
// change.  Parallel (timed baseline).  Returns the number of rounds.
uint32_t orc_cc_labelprop(uint32_t n, const uint64_t* end, const uint32_t* col, uint32_t* label) {
  Csr g{n, end, col};
  std::vector<uint32_t> old(n, 0xFFFFFFFFu);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) label[v] = (uint32_t)v;
  uint32_t rounds = 0;
  bool changed = true;
  while (changed) {
    changed = false;
    ++rounds;
#pragma omp parallel for schedule(dynamic, 1024) reduction(|| : changed)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      const uint32_t cur = __atomic_load_n(&label[v], __ATOMIC_RELAXED);
      if (old[v] > cur) {
        old[v] = cur;
        changed = true;
        for (uint64_t i = g.b((uint32_t)v); i < g.e((uint32_t)v); ++i) atomic_min_u32(&label[col[i]], cur);
      }
    }
  }
  return rounds;
}

// ConnectedComponents.cpp:1046-1072: both endpoints of every arc share a label.
int orc_verify_cc(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* label) {
  Csr g{n, end, col};
  for (uint32_t v = 0; v < n; ++v)
    for (uint64_t i = g.b(v); i < g.e(v); ++i)
      if (label[col[i]] != label[v]) return 1;
  return 0;
}

// RandomizeEdgeWeights (tools/graph-convert/graph-convert.cpp:1145-1190):
// a default-constructed std::mt19937, one uniform draw per arc in arc order,
// std::uniform_int_distribution<uint32_t>(lo, hi) or, with is_float,
// std::uniform_real_distribution<float>(lo, hi) written as float bits.
void orc_gr2randomweight(uint64_t m, int lo, int hi, int is_float, uint32_t* out) {
  std::mt19937 gen;
  if (is_float) {
    std::uniform_real_distribution<float> dist((float)lo, (float)hi);
    for (uint64_t e = 0; e < m; ++e) {
      const float x = dist(gen);
      std::memcpy(out + e, &x, 4);
    }
  } else {
    std::uniform_int_distribution<uint32_t> dist((uint32_t)lo, (uint32_t)hi);
    for (uint64_t e = 0; e < m; ++e) out[e] = dist(gen);
  }
}

// The raw output of a default-constructed std::mt19937 (the C++ standard,
// [rand.predef], fixes its 10000th value at 4123659995).
void orc_mt19937_raw(uint64_t count, uint32_t* out) {
  std::mt19937 gen;
  for (uint64_t i = 0; i < count; ++i) out[i] = (uint32_t)gen();
}

}  // extern "C"
