// operator-example: lonestar-style operators written with the header-only
// operator layer (include/gb_operator.cuh) over the libgb device mirror.
//
//   * BFS: the operator of lonestar/analytics/cpu/bfs/bfs.cpp:155-242 (the
//     asynchronous variant: for every out-arc, lower the destination's level
//     to level+1 and push it if that lowered it), over the FIFO worklist
//     (gb::wl<gb::FIFO>()), seeded by gb::do_all.
//   * SSSP: the delta-stepping operator of
//     lonestar/analytics/cpu/sssp/SSSP.cpp:134-161 (skip a request whose
//     distance is stale, relax every out-arc with atomicMin, push the
//     destination on improvement) over
//     gb::wl<gb::DeltaBuckets>(-delta), the device form of
//     galois::wl<OBIM>(UpdateRequestIndexer{stepShift}).
// Both run through gb::for_each_edge, which spreads every item's arcs over a
// warp.  The results pass the apps' own path verifier (BFS_SSSP.h:231-263)
// and, with -output=FILE, are written as n uint32 levels followed by n
// uint32 distances for an outside check.
//
//   operator-example <input.gr> [-startNode=N] [-delta=S] [-symmetricGraph] [-output=FILE]
#include <cstdio>
#include <vector>

#include "gb_operator.cuh"
#include "lonestar_cli.h"

int main(int argc, char** argv) {
  using namespace lsapp;
  Flags f = parse(argc, argv, {});
  Loaded L;
  load(f, 4, L);
  const uint32_t n = L.h.n;
  const uint32_t src = (uint32_t)f.u64("startNode", 0);
  const uint32_t shift = (uint32_t)f.u64("delta", 13);
  if (src >= n) die("startNode is not a vertex");
  if (!L.h.w_u32) die("the input needs 4-byte edge weights");

  gb::DeviceCSR g;
  check(gb::DeviceCSR::from(L.g, &g), "DeviceCSR::from");
  uint32_t *level = nullptr, *dist = nullptr, *seed = nullptr;
  if (cudaMalloc(&level, sizeof(uint32_t) * n) != cudaSuccess ||
      cudaMalloc(&dist, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&seed, 2 * sizeof(uint32_t)) != cudaSuccess)
    die("cudaMalloc failed");
  const uint32_t h_seed[2] = {src, 0u};  // the item (vertex) and its key (distance 0)
  cudaMemcpy(seed, h_seed, sizeof(h_seed), cudaMemcpyHostToDevice);

  // one workspace for both loops: every vertex can wait in a later bucket once
  // per improvement, bounded here by the arcs
  gb::Worklist ws;
  check(ws.reserve((uint32_t)std::min<uint64_t>(L.h.m + 1, 0xFFFFFFF0ull), (uint64_t)n / 16 + 4096),
        "Worklist::reserve");
  const uint32_t inf = (uint32_t)GB_DIST_INFINITY;

  // BFS: do_all initialises, for_each_edge relaxes levels asynchronously
  check(gb::do_all(gb::iterate(g), [=] __device__(uint32_t v) { level[v] = v == src ? 0u : inf; }), "gb::do_all");
  gb::ForEachStats bst;
  check(gb::for_each_edge(
            ws, g, seed, seed + 1, 1,
            [=] __device__(uint32_t v, uint32_t lv) { return level[v] == lv; },  // stale request: skip
            [=] __device__(uint32_t v, uint32_t lv, uint64_t e, const gb::Ctx& ctx) {
              const uint32_t dst = g.getEdgeDst(e);
              if (atomicMin(&level[dst], lv + 1) > lv + 1) ctx.push(dst, lv + 1);
            },
            gb::wl<gb::FIFO>(), 0, &bst),
        "gb::for_each_edge (BFS)");

  // SSSP: delta-stepping over OBIM-like buckets of dist >> shift
  check(gb::do_all(gb::iterate(g), [=] __device__(uint32_t v) { dist[v] = v == src ? 0u : inf; }), "gb::do_all");
  gb::ForEachStats sst;
  check(gb::for_each_edge(
            ws, g, seed, seed + 1, 1,
            [=] __device__(uint32_t v, uint32_t d) { return dist[v] >= d; },  // SSSP.cpp:138-142
            [=] __device__(uint32_t v, uint32_t d, uint64_t e, const gb::Ctx& ctx) {
              const uint32_t dst = g.getEdgeDst(e);
              const uint32_t nd = d + g.getEdgeData(e);
              if (nd < atomicMin(&dist[dst], nd)) ctx.push(dst, nd);
            },
            gb::wl<gb::DeltaBuckets>(shift), 0, &sst),
        "gb::for_each_edge (SSSP)");

  std::vector<uint32_t> lv(n), dv(n);
  cudaMemcpy(lv.data(), level, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(dv.data(), dist, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  cudaFree(level);
  cudaFree(dist);
  cudaFree(seed);
  uint64_t reached = 0;
  for (uint32_t v = 0; v < n; ++v) reached += lv[v] != inf;
  std::printf("operator BFS (FIFO): %llu items, %llu arcs, %llu chunks; %llu vertices reached\n",
              (unsigned long long)bst.items, (unsigned long long)bst.edges, (unsigned long long)bst.chunks,
              (unsigned long long)reached);
  std::printf("operator SSSP (DeltaBuckets, shift %u): %llu items, %llu arcs, %u buckets\n", shift,
              (unsigned long long)sst.items, (unsigned long long)sst.edges, sst.buckets);
  const std::string out = f.str("output", "");
  if (!out.empty()) {
    FILE* fo = std::fopen(out.c_str(), "wb");
    if (!fo || std::fwrite(lv.data(), 4, n, fo) != n || std::fwrite(dv.data(), 4, n, fo) != n) die("cannot write " + out);
    std::fclose(fo);
  }
  if (!verify_paths(L, src, lv, true) || !verify_paths(L, src, dv, false)) die("verification failed");
  std::printf("Verification successful.\n");
  return 0;
}
