// All-vertex sweeps (do_all over every vertex's adjacency): the device form of
// `galois::do_all(galois::iterate(graph), op, steal(), chunk_size<K>)`
// (libgalois/include/galois/Loops.h:70-74) for operators that touch every arc,
// i.e. CC label propagation and PageRank pull.
//
// Work decomposition, computed once per graph and cached in the handle:
//   task t <  nchunks : vertices 32t .. 32t+31, each expanded by warp_expand
//                       unless its degree exceeds `heavy` (then it is skipped
//                       here and covered by its tiles);
//   task t >= nchunks : one tile of `tile` arcs of a heavy vertex.
// Tasks are assigned to warps grid-stride (static), which balances because no
// chunk holds more than 32*heavy arcs and tiles are uniform.
#pragma once

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

struct SweepSched {
  const uint2* tiles;   // (vertex, k) for heavy vertices, ascending by vertex
  uint32_t ntiles;
  const uint32_t* heavy_list;  // heavy vertex ids, ascending
  uint32_t nheavy;
  uint32_t heavy;
  uint32_t tile;
};

// Build (or fetch the cached) schedule for the stored out-edges.
int ensure_sweep_schedule(gb_graph* g, uint32_t heavy, uint32_t tile, cudaStream_t s, SweepSched* out);

// Calls light(valid, v, edge, owner_lane) through warp_expand for light
// vertices, and tile_fn(v, e_begin, e_end) once per heavy tile (by the whole
// warp).  All lanes of every warp must enter.
template <class LightEdgeFn, class ChunkDoneFn, class TileFn>
__device__ __forceinline__ void sweep_all(const uint64_t* __restrict__ offs, uint32_t n,
                                          const SweepSched& s, uint64_t gwarp, uint64_t nwarps,
                                          LightEdgeFn&& light, ChunkDoneFn&& chunk_done, TileFn&& tile_fn) {
  const uint32_t lane = lane_id();
  const uint64_t nchunks = ((uint64_t)n + 31) >> 5;
  const uint64_t total = nchunks + s.ntiles;
  for (uint64_t t = gwarp; t < total; t += nwarps) {
    if (t < nchunks) {
      const uint64_t v = (t << 5) + lane;
      uint64_t b = 0;
      uint32_t d = 0;
      bool heavy = false;
      if (v < n) {
        b = ldg(offs + v);
        const uint64_t dd = ldg(offs + v + 1) - b;
        heavy = dd > s.heavy;
        d = heavy ? 0u : (uint32_t)dd;
      }
      warp_expand(b, d, (uint32_t)v, light);
      chunk_done((uint32_t)v, v < n, heavy);
    } else {
      const uint2 tv = s.tiles[t - nchunks];
      const uint64_t vb = ldg(offs + tv.x), ve = ldg(offs + tv.x + 1);
      const uint64_t b = vb + (uint64_t)tv.y * s.tile;
      const uint64_t e = min(ve, b + s.tile);
      tile_fn(tv.x, b, e);
    }
  }
}

}  // namespace gb
