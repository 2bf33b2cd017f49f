// Device frontier queues: the B200 replacement for Galois' InsertBag of
// vertices / edge tiles (BFS_SSSP.h:81-131, bfs.cpp:244-293) and libgpu's
// Worklist2 (libgpu/include/worklist.h:410-510).
//
// A frontier is two queues: `light` holds vertices whose degree is at most
// `heavy` (expanded 32 at a time by one warp), `tiles` holds (vertex, k) pairs
// naming the k-th run of `tile` arcs of a heavier vertex (one warp per tile).
// Degree binning happens once, when a vertex is discovered.
#pragma once

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

struct FrontierCounters {
  uint32_t light;       // entries in the light queue
  uint32_t tiles;       // entries in the tile queue
  uint32_t vertices;    // vertices discovered into this frontier (any degree)
  uint32_t light_work;  // dynamic work-distribution cursors
  uint32_t tile_work;
  uint32_t pad;
  unsigned long long degree_sum;  // sum of out-degrees of discovered vertices
};

struct FrontierQueues {
  uint32_t* light[2];
  uint2* tiles[2];
  uint32_t light_cap;
  uint32_t tile_cap;
};

struct FrontierLayout {
  uint32_t light_cap;
  uint32_t tile_cap;
  size_t bytes;
};

inline FrontierLayout frontier_layout(uint32_t n, uint64_t m, uint32_t heavy, uint32_t tile) {
  FrontierLayout l;
  l.light_cap = n;
  uint64_t tc = m / tile + m / ((uint64_t)heavy + 1) + 2;
  if (tc > 0xFFFFFFF0ull) tc = 0xFFFFFFF0ull;
  l.tile_cap = (uint32_t)tc;
  l.bytes = 2 * carve_size<uint32_t>(l.light_cap) + 2 * carve_size<uint2>(l.tile_cap);
  return l;
}

inline FrontierQueues carve_frontier(Carver& cv, const FrontierLayout& l) {
  FrontierQueues q;
  q.light[0] = cv.take<uint32_t>(l.light_cap);
  q.light[1] = cv.take<uint32_t>(l.light_cap);
  q.tiles[0] = cv.take<uint2>(l.tile_cap);
  q.tiles[1] = cv.take<uint2>(l.tile_cap);
  q.light_cap = l.light_cap;
  q.tile_cap = l.tile_cap;
  return q;
}

// Single-thread seeding of a source vertex into queue buffer qb.
__device__ __forceinline__ void seed_vertex(const FrontierQueues& q, int qb, FrontierCounters& c,
                                            uint32_t v, uint64_t d, uint32_t heavy, uint32_t tile) {
  if (d <= heavy) {
    q.light[qb][c.light++] = v;
  } else {
    const uint32_t nt = (uint32_t)((d + tile - 1) / tile);
    for (uint32_t k = 0; k < nt && c.tiles < q.tile_cap; ++k) q.tiles[qb][c.tiles++] = make_uint2(v, k);
  }
}

// Warp-collective: append every lane's discovered vertex `u` (disc == true,
// out-degree d) into queue buffer qb, binned by degree; zero-degree vertices
// are counted but not queued (nothing to expand).  kCount also maintains the
// vertex and degree totals the BFS direction heuristic reads.  All 32 lanes
// must call.
template <bool kCount>
__device__ __forceinline__ void push_with_degree(const FrontierQueues& q, int qb, FrontierCounters& c, bool disc,
                                                 uint32_t u, uint64_t d, uint32_t heavy, uint32_t tile, int* err) {
  const bool light = disc && d > 0 && d <= heavy;
  const bool hv = disc && d > heavy;
  warp_push(light, u, q.light[qb], &c.light, q.light_cap, err);
  warp_push_tiles(u, hv ? (uint32_t)((d + tile - 1) / tile) : 0u, q.tiles[qb], &c.tiles, q.tile_cap, err);
  if (kCount) {
    const unsigned dmask = __ballot_sync(kFull, disc);
    if (dmask) {
      const unsigned long long ds = warp_sum((unsigned long long)(disc ? d : 0));
      if (lane_id() == 0) {
        atomicAdd(&c.vertices, (uint32_t)__popc(dmask));
        if (ds) atomicAdd(&c.degree_sum, ds);
      }
    }
  }
}

template <bool kCount = true>
__device__ __forceinline__ void push_discovered(const FrontierQueues& q, int qb, FrontierCounters& c, bool disc,
                                                uint32_t u, const uint64_t* __restrict__ offs, uint32_t heavy,
                                                uint32_t tile, int* err) {
  uint64_t d = 0;
  if (disc) d = __ldg(offs + u + 1) - __ldg(offs + u);
  push_with_degree<kCount>(q, qb, c, disc, u, d, heavy, tile, err);
}

// Per-warp staging of light-queue appends in shared memory.  Appends collect
// in `slots` (K entries owned by one warp) and are published with one
// atomicAdd per flush instead of one per warp step, so a queue counter that
// every warp appends to is touched K/32 times less often.  `n` is
// warp-uniform; every call is warp-collective.
template <int K>
struct WarpStage {
  uint32_t* slots;
  uint32_t n;

  __device__ __forceinline__ void flush(uint32_t* queue, uint32_t* count, uint32_t cap, int* err) {
    if (n == 0) return;
    const uint32_t lane = lane_id();
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(count, n);
    base = __shfl_sync(kFull, base, 0);
    for (uint32_t i = lane; i < n; i += 32) {
      if (base + i < cap) queue[base + i] = slots[i];
      else raise_err(err, kDevOverflow);
    }
    __syncwarp();
    n = 0;
  }

  __device__ __forceinline__ void push(bool pred, uint32_t item, uint32_t* queue, uint32_t* count, uint32_t cap,
                                       int* err) {
    const unsigned mask = __ballot_sync(kFull, pred);
    if (!mask) return;
    const uint32_t k = __popc(mask);
    if (n + k > (uint32_t)K) flush(queue, count, cap, err);
    if (pred) slots[n + __popc(mask & ((1u << lane_id()) - 1u))] = item;
    n += k;
    __syncwarp();
  }
};

// Vertices per light task: 32 when the frontier fills every warp, fewer
// (a power of two) for small frontiers so that more warps share them and the
// per-phase critical path is one expansion step instead of several.
__device__ __forceinline__ uint32_t vertices_per_task(uint32_t q_light, uint64_t nwarps) {
  const uint64_t per = q_light / (nwarps ? nwarps : 1);
  if (per >= 32) return 32;
  uint32_t k = 1;
  while ((uint64_t)(k << 1) <= per) k <<= 1;
  return k;
}

// Static, atomic-free distribution of a frontier over all warps of the grid:
// tasks [0, nchunks) are `vpt`-entry chunks of the light queue (vpt from
// vertices_per_task), the remaining tasks are heavy-vertex tiles; warp w
// takes tasks w, w + nwarps, ...  chunk(base, vpt) / tile(t) are called by
// whole warps; in a chunk, lanes < vpt own entries base + lane.
template <class ChunkFn, class TileFn>
__device__ __forceinline__ void for_each_frontier_task(uint32_t q_light, uint32_t q_tiles, uint64_t gwarp,
                                                       uint64_t nwarps, ChunkFn&& chunk, TileFn&& tile) {
  const uint32_t vpt = vertices_per_task(q_light, nwarps);
  const uint64_t nchunks = ((uint64_t)q_light + vpt - 1) / vpt;
  const uint64_t total = nchunks + q_tiles;
  for (uint64_t t = gwarp; t < total; t += nwarps) {
    if (t < nchunks) chunk((uint32_t)(t * vpt), vpt);
    else tile((uint32_t)(t - nchunks));
  }
}

}  // namespace gb
