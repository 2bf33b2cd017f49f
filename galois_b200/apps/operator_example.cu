// operator-example: a lonestar-style operator written with the header-only
// operator layer (include/gb_operator.cuh) over the libgb device mirror.
//
// Restates the BFS operator of lonestar/analytics/cpu/bfs/bfs.cpp:280-288
// (for every out-edge of the current item, lower the destination's level to
// level+1 and push the destination if it changed) with gb::do_all for the
// initialisation and gb::for_each for the worklist, then checks the result
// against gb_bfs on the same graph.
//
//   operator-example <input.gr> [-startNode=N] [-symmetricGraph]
#include <vector>

#include "gb_operator.cuh"
#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {});
  Loaded L;
  load(f, 0, L);
  const uint32_t n = L.h.n;
  const uint32_t src = (uint32_t)f.u64("startNode", 0);
  if (src >= n) die("startNode is not a vertex");

  gb::DeviceCSR g;
  check(gb::DeviceCSR::from(L.g, &g), "DeviceCSR::from");
  uint32_t* level = nullptr;
  uint32_t* seed = nullptr;
  if (cudaMalloc(&level, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&seed, sizeof(uint32_t)) != cudaSuccess)
    die("cudaMalloc failed");

  // do_all: level[v] = INF, level[src] = 0
  check(gb::do_all(gb::iterate(g),
                   [=] __device__(uint32_t v) { level[v] = v == src ? 0u : (uint32_t)GB_DIST_INFINITY; }),
        "gb::do_all");
  cudaMemcpy(seed, &src, sizeof(uint32_t), cudaMemcpyHostToDevice);

  // for_each: the BFS operator; every vertex is pushed at most once, so n
  // entries bound one round.
  uint32_t rounds = 0;
  check(gb::for_each(
            seed, 1,
            [=] __device__(uint32_t v, const gb::Context& ctx) {
              const uint32_t next = level[v] + 1;
              for (uint64_t e = g.edge_begin(v); e < g.edge_end(v); ++e) {
                const uint32_t dst = g.getEdgeDst(e);
                if (atomicCAS(&level[dst], (uint32_t)GB_DIST_INFINITY, next) == (uint32_t)GB_DIST_INFINITY)
                  ctx.push(dst);
              }
            },
            n, nullptr, n + 1, &rounds),
        "gb::for_each");

  std::vector<uint32_t> mine(n), lib(n);
  cudaMemcpy(mine.data(), level, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  check(gb_bfs(L.g, src, lib.data(), nullptr, nullptr), "gb_bfs");
  cudaFree(level);
  cudaFree(seed);
  size_t bad = 0;
  for (uint32_t v = 0; v < n; ++v) bad += mine[v] != lib[v];
  std::printf("operator BFS: %u rounds, %zu mismatches against gb_bfs\n", rounds, bad);
  if (bad) die("verification failed");
  std::printf("Verification successful.\n");
  return 0;
}
