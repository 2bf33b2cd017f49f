// Builds the cached all-vertex sweep schedule (see sweep.cuh).

#include <algorithm>

#include "sweep.cuh"

namespace gb {

namespace {

__global__ void sweep_tiles_kernel(const uint64_t* __restrict__ offs, uint32_t n, uint32_t heavy, uint32_t tile,
                                   uint2* tiles, uint32_t tile_cap, uint32_t* heavy_list, uint32_t heavy_cap,
                                   uint32_t* counts, int* err) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = tid - lane_id(); base < n; base += stride) {
    const uint64_t v = base + lane_id();
    uint64_t d = 0;
    if (v < n) d = offs[v + 1] - offs[v];
    const bool hv = v < n && d > heavy;
    warp_push(hv, (uint32_t)v, heavy_list, &counts[1], heavy_cap, err);
    warp_push_tiles((uint32_t)v, hv ? (uint32_t)((d + tile - 1) / tile) : 0u, tiles, &counts[0], tile_cap, err);
  }
}

}  // namespace

int build_row_schedule(const uint64_t* offs, uint32_t n, uint64_t m, uint32_t heavy, uint32_t tile, int sm_count,
                       void* pinned, cudaStream_t s, uint2** tiles, uint32_t** heavy_list, uint32_t* ntiles,
                       uint32_t* nheavy) {
  const uint64_t tc64 = m / tile + m / ((uint64_t)heavy + 1) + 2;
  const uint32_t tile_cap = (uint32_t)std::min<uint64_t>(tc64, 0xFFFFFFF0ull);
  const uint32_t heavy_cap = (uint32_t)std::min<uint64_t>(m / ((uint64_t)heavy + 1) + 2, 0xFFFFFFF0ull);
  *tiles = nullptr;
  *heavy_list = nullptr;
  GB_CUDA(cudaMalloc(tiles, sizeof(uint2) * tile_cap));
  GB_CUDA(cudaMalloc(heavy_list, sizeof(uint32_t) * heavy_cap));
  uint32_t* dcount = nullptr;
  GB_CUDA(cudaMalloc(&dcount, 16));
  GB_CUDA(cudaMemsetAsync(dcount, 0, 16, s));
  sweep_tiles_kernel<<<sm_count * 4, 256, 0, s>>>(offs, n, heavy, tile, *tiles, tile_cap, *heavy_list, heavy_cap,
                                                   dcount, reinterpret_cast<int*>(dcount + 2));
  uint32_t* h = static_cast<uint32_t*>(pinned);
  cudaMemcpyAsync(h, dcount, 16, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(dcount);
  if (e != cudaSuccess) return cuda_fail(e, "row schedule");
  if (h[2]) GB_FAIL(GB_ERR_CAPACITY, "row schedule overflow");
  *ntiles = h[0];
  *nheavy = h[1];
  return GB_OK;
}

int ensure_sweep_schedule(gb_graph* g, uint32_t heavy, uint32_t tile, cudaStream_t s, SweepSched* out) {
  if (!(g->sweep_tiles && g->sweep_heavy == heavy && g->sweep_tile == tile)) {
    // pooled (graph_device.cu): a one-shot graph's upload / query / free
    // cycle then makes no cudaMalloc or cudaFree, whose cost varied from
    // under 1 ms to over 600 ms between calls on a loaded host
    if (g->sweep_tiles) GB_CUDA(cudaStreamSynchronize(s));  // a kernel on s may still read the old schedule
    pool_free(g->sweep_tiles);
    pool_free(g->sweep_heavy_list);
    g->sweep_tiles = nullptr;
    g->sweep_heavy_list = nullptr;
    const uint64_t tc64 = g->m / tile + g->m / ((uint64_t)heavy + 1) + 2;
    const uint32_t tile_cap = (uint32_t)std::min<uint64_t>(tc64, 0xFFFFFFF0ull);
    const uint32_t heavy_cap = (uint32_t)std::min<uint64_t>(g->m / ((uint64_t)heavy + 1) + 2, 0xFFFFFFF0ull);
    GB_CUDA(pool_malloc(reinterpret_cast<void**>(&g->sweep_tiles), sizeof(uint2) * tile_cap));
    GB_CUDA(pool_malloc(reinterpret_cast<void**>(&g->sweep_heavy_list), sizeof(uint32_t) * heavy_cap));
    uint32_t* dcount = nullptr;
    GB_CUDA(pool_malloc(reinterpret_cast<void**>(&dcount), 16));
    GB_CUDA(cudaMemsetAsync(dcount, 0, 16, s));
    sweep_tiles_kernel<<<g->sm_count * 4, 256, 0, s>>>(g->offs, g->n, heavy, tile, g->sweep_tiles, tile_cap,
                                                        g->sweep_heavy_list, heavy_cap, dcount,
                                                        reinterpret_cast<int*>(dcount + 2));
    uint32_t* h = static_cast<uint32_t*>(g->pinned);
    cudaMemcpyAsync(h, dcount, 16, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    pool_free(dcount);
    if (e != cudaSuccess) return cuda_fail(e, "sweep schedule");
    if (h[2]) GB_FAIL(GB_ERR_CAPACITY, "sweep schedule overflow");
    g->sweep_ntiles = h[0];
    g->sweep_nheavy = h[1];
    g->sweep_heavy = heavy;
    g->sweep_tile = tile;
  }
  out->tiles = g->sweep_tiles;
  out->ntiles = g->sweep_ntiles;
  out->heavy_list = g->sweep_heavy_list;
  out->nheavy = g->sweep_nheavy;
  out->heavy = heavy;
  out->tile = tile;
  return GB_OK;
}

}  // namespace gb
