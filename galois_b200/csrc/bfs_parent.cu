// BFS parents: the output of lonestar's direction-optimising BFS, which
// stores for every reached vertex the frontier vertex whose compare-and-swap
// won (bfsDirectionOpt.cpp:284-285 pull, :325 push) and 0 for the source
// (:229), unreached vertices keeping DIST_INFINITY.
//
// Which in-neighbour wins that race is left open by the reference.  Here
// every reached vertex v other than the source gets the smallest original id
// among its in-neighbours u with level[u] == level[v] - 1: always one of the
// reference's possible outputs, and reproducible, so it is checked exactly.
// Levels come from the BFS kernel (bfs.cu); the parent pass is one sweep of
// the reached vertices' in-arcs:
//   * parent_rows: 32 consecutive vertices per warp task, their in-arcs
//     spread over the lanes by warp_expand, candidates reduced into the
//     owner's shared-memory slot with a block-scope atomicMin; vertices with
//     more than `heavy` in-arcs are set to ~0 here and finished by
//   * parent_tiles: one warp per tile of a heavy row, a warp min, one global
//     atomicMin per tile.
// In-arcs are the stored arcs of a symmetric graph, else the transpose
// (built on first use).  On a relabelled graph the candidates are compared by
// original id (perm) and the result is gathered back to original order.

#include "device_common.cuh"
#include "device_graph.cuh"
#include "sweep.cuh"

namespace gb {

int run_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats, cudaStream_t s, void* scratch,
            size_t scratch_bytes);
int build_row_schedule(const uint64_t* offs, uint32_t n, uint64_t m, uint32_t heavy, uint32_t tile, int sm_count,
                       void* pinned, cudaStream_t s, uint2** tiles, uint32_t** heavy_list, uint32_t* ntiles,
                       uint32_t* nheavy);

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kParentBlock = 256;

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) parent_rows(const uint64_t* __restrict__ offs,
                                                     const uint32_t* __restrict__ col,
                                                     const uint32_t* __restrict__ level,
                                                     const uint32_t* __restrict__ key, uint32_t n, uint32_t heavy,
                                                     uint32_t* __restrict__ par) {
  __shared__ uint32_t s_min[BLOCK / 32][32];
  uint32_t* sm = s_min[threadIdx.x >> 5];
  const uint32_t lane = lane_id();
  const uint64_t gwarp = (blockIdx.x * (uint64_t)BLOCK + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * BLOCK) >> 5;
  const uint64_t nchunks = ((uint64_t)n + 31) >> 5;
  for (uint64_t t = gwarp; t < nchunks; t += nwarps) {
    const uint64_t v = (t << 5) + lane;
    uint32_t lv = kInf, d = 0;
    uint64_t b = 0;
    bool hv = false;
    if (v < n) {
      lv = ldg(level + v);
      b = ldg(offs + v);
      const uint64_t dd = ldg(offs + v + 1) - b;
      hv = dd > heavy;
      if (lv != kInf && lv != 0 && !hv) d = (uint32_t)dd;
    }
    sm[lane] = kNone;
    __syncwarp();
    warp_expand(b, d, lv, [&](bool valid, uint64_t e, uint32_t owner, uint32_t olv) {
      if (valid) {
        const uint32_t u = ldg(col + e);
        if (ldg(level + u) + 1u == olv) atomicMin_block(&sm[owner], key ? ldg(key + u) : u);
      }
    });
    __syncwarp();
    if (v < n) par[v] = lv == 0 ? 0u : (lv == kInf ? kInf : (hv ? kNone : sm[lane]));
    __syncwarp();
  }
}

__global__ void parent_tiles(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col,
                             const uint32_t* __restrict__ level, const uint32_t* __restrict__ key,
                             const uint2* __restrict__ tiles, uint32_t ntiles, uint32_t tile,
                             uint32_t* __restrict__ par) {
  const uint32_t lane = lane_id();
  const uint64_t gwarp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t t = gwarp; t < ntiles; t += nwarps) {
    const uint2 tv = tiles[t];
    const uint32_t lv = ldg(level + tv.x);
    if (lv == kInf || lv == 0) continue;  // warp-uniform
    const uint64_t vb = ldg(offs + tv.x), ve = ldg(offs + tv.x + 1);
    const uint64_t b = vb + (uint64_t)tv.y * tile;
    const uint64_t e_end = min(ve, b + tile);
    uint32_t best = kNone;
#pragma unroll 4
    for (uint64_t e = b + lane; e < e_end; e += 32) {
      const uint32_t u = ldg(col + e);
      if (ldg(level + u) + 1u == lv) best = min(best, key ? ldg(key + u) : u);
    }
    best = __reduce_min_sync(kFull, best);
    if (lane == 0 && best != kNone) atomicMin(&par[tv.x], best);
  }
}

}  // namespace

}  // namespace gb

extern "C" int gb_bfs_parent(gb_graph* g, uint32_t src, uint32_t* parent_out, uint32_t* level_out, gb_stats* stats,
                             void* stream) {
  using namespace gb;
  clear_error();
  if (!g || !parent_out) GB_FAIL(GB_ERR_ARG, "gb_bfs_parent: null argument");
  if (src >= g->n) GB_FAIL(GB_ERR_ARG, "gb_bfs_parent: source %u >= n %u", src, g->n);
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = GB_OK;
  if (!g->symmetric) {
    st = ensure_transpose(g, s);
    if (st != GB_OK) return st;
  }
  st = reserve_result_bufs(g);
  if (st != GB_OK) return st;
  const uint32_t n = g->n;
  const uint32_t isrc = g->perm ? g->h_iperm[src] : src;
  uint32_t* lvl = result_buf(g, 0);  // internal ids
  uint32_t* par = result_buf(g, 2);  // internal ids, original-id values
  gb_stats local{};
  st = run_bfs(g, isrc, lvl, stats ? stats : &local, s, nullptr, 0);
  if (st != GB_OK) return st;
  const uint64_t* in_offs = g->symmetric ? g->offs : g->t_offs;
  const uint32_t* in_col = g->symmetric ? g->col : g->t_col;
  const gb_tuning t = effective_tuning(g);
  uint2* tiles = nullptr;
  uint32_t* heavy_list = nullptr;
  uint32_t ntiles = 0, nheavy = 0;
  SweepSched sched{};
  if (g->symmetric) {
    st = ensure_sweep_schedule(g, t.heavy_degree, t.tile_edges, s, &sched);
    if (st != GB_OK) return st;
  } else {
    // the in-arc rows' tiles: built for this call, freed below
    st = build_row_schedule(in_offs, n, g->m, t.heavy_degree, t.tile_edges, g->sm_count, g->pinned, s, &tiles,
                            &heavy_list, &ntiles, &nheavy);
    if (st != GB_OK) {
      cudaFree(tiles);
      cudaFree(heavy_list);
      return st;
    }
    sched.tiles = tiles;
    sched.ntiles = ntiles;
  }
  const int grid = g->sm_count * 8;
  KernelTimer kt(stats != nullptr, s);  // the parent pass, added to the BFS kernel time
  parent_rows<kParentBlock><<<grid, kParentBlock, 0, s>>>(in_offs, in_col, lvl, g->perm, n, t.heavy_degree, par);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && sched.ntiles)
    parent_tiles<<<grid, 256, 0, s>>>(in_offs, in_col, lvl, g->perm, sched.tiles, sched.ntiles, t.tile_edges, par);
  if (e == cudaSuccess) e = cudaGetLastError();
  kt.stop(s);
  if (tiles) {
    // the tiles must outlive the launch that reads them
    const cudaError_t se = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = se;
    cudaFree(tiles);
    cudaFree(heavy_list);
  }
  if (e != cudaSuccess) return cuda_fail(e, "gb_bfs_parent");
  if (stats) {
    GB_CUDA(cudaStreamSynchronize(s));
    stats->launches += sched.ntiles ? 2 : 1;
    stats->kernel_ms += kt.ms();
  }
  if (g->perm) {
    if (level_out) {
      st = finish_u32(g, lvl, level_out, s);
      if (st != GB_OK) return st;
    }
    if (stats) stats->launches += level_out ? 2 : 1;
    return finish_u32(g, par, parent_out, s);
  }
  if (level_out) {
    st = copy_out(level_out, lvl, sizeof(uint32_t) * n, s);
    if (st != GB_OK) return st;
  }
  return copy_out(parent_out, par, sizeof(uint32_t) * n, s);
}
