// Many disjoint graphs in one launch: BFS + CC over a block-diagonal packing.
//
// Config of the reference build plan: 512 uneven Erdos-Renyi graphs with BFS
// and CC per graph.  Looping gb_bfs / gb_cc per graph pays two launches and a
// host round trip per small graph; here the graphs share ONE device mirror
// (vertex ranges graph_first[k] .. graph_first[k+1]-1, no arc crossing a
// range) and
//   * BFS runs once from the super-source {graph_first[k] + local_src[k]}:
//     since no arc leaves a graph, every vertex gets exactly the level it has
//     in its own graph's BFS (lonestar/analytics/cpu/bfs/bfs.cpp:244-293);
//   * CC (union-find, larger root under the smaller) labels every vertex with
//     the minimum GLOBAL id of its component, which is graph_first[k] plus the
//     minimum LOCAL id -- the label LabelProp converges to per graph
//     (ConnectedComponents.cpp:183-230) -- so one subtraction localises it.
// After the first call on a layout (validation, buffer set-up) the call
// issues only stream-ordered work when the outputs are device pointers, so it
// can be captured in a CUDA graph and replayed.

#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

int run_bfs_sources(gb_graph* g, const uint32_t* d_srcs, uint32_t k, uint32_t* d_level, cudaStream_t s);
int run_cc(gb_graph* g, int algo, uint32_t* label_out, gb_stats* stats, cudaStream_t s);

namespace {

__device__ __forceinline__ uint32_t graph_of(const uint32_t* __restrict__ gf, uint32_t ng, uint32_t v) {
  uint32_t lo = 0, hi = ng;  // largest k with gf[k] <= v
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (gf[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void mg_validate(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col, uint32_t n,
                            const uint32_t* __restrict__ gf, uint32_t ng, int* bad) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride) {
    const uint32_t k = graph_of(gf, ng, (uint32_t)v);
    const uint32_t lo = gf[k], hi = gf[k + 1];
    for (uint64_t e = offs[v]; e < offs[v + 1]; ++e) {
      const uint32_t u = col[e];
      if (u < lo || u >= hi) {
        atomicOr(bad, 1);
        break;
      }
    }
  }
}

__global__ void mg_localize(uint32_t* __restrict__ label, uint32_t n, const uint32_t* __restrict__ gf, uint32_t ng) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride) label[v] -= gf[graph_of(gf, ng, (uint32_t)v)];
}

uint64_t fnv1a(const uint32_t* p, size_t k) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < k; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Validate and cache the layout (first call for a layout only).
int prepare_layout(gb_graph* g, const uint32_t* gf, uint32_t ng, cudaStream_t s) {
  const uint64_t h = fnv1a(gf, (size_t)ng + 1) ^ ng;
  if (g->mg_first && g->mg_ngraphs == ng && g->mg_hash == h) return GB_OK;
  if (gf[0] != 0 || gf[ng] != g->n) GB_FAIL(GB_ERR_ARG, "multi-graph: graph_first must start at 0 and end at n");
  for (uint32_t k = 0; k < ng; ++k)
    if (gf[k + 1] <= gf[k]) GB_FAIL(GB_ERR_ARG, "multi-graph: graph %u is empty or ranges are not increasing", k);
  cudaFree(g->mg_first);
  cudaFree(g->mg_src);
  cudaFree(g->mg_level);
  cudaFree(g->mg_label);
  if (g->mg_stage) cudaFreeHost(g->mg_stage);
  g->mg_first = g->mg_src = g->mg_level = g->mg_label = g->mg_stage = nullptr;
  g->mg_ngraphs = 0;
  GB_CUDA(cudaMalloc(&g->mg_first, sizeof(uint32_t) * (ng + 1)));
  GB_CUDA(cudaMalloc(&g->mg_src, sizeof(uint32_t) * ng));
  GB_CUDA(cudaMalloc(&g->mg_level, sizeof(uint32_t) * g->n));
  GB_CUDA(cudaMalloc(&g->mg_label, sizeof(uint32_t) * g->n));
  GB_CUDA(cudaMallocHost(&g->mg_stage, sizeof(uint32_t) * (2 * (size_t)ng + 1)));
  GB_CUDA(cudaMemcpyAsync(g->mg_first, gf, sizeof(uint32_t) * (ng + 1), cudaMemcpyHostToDevice, s));
  int* dbad = reinterpret_cast<int*>(g->mg_src);  // scratch before sources are written
  GB_CUDA(cudaMemsetAsync(dbad, 0, sizeof(int), s));
  mg_validate<<<g->sm_count * 4, 256, 0, s>>>(g->offs, g->col, g->n, g->mg_first, ng, dbad);
  int hbad = 0;
  GB_CUDA(cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
  GB_CUDA(cudaStreamSynchronize(s));
  if (hbad) GB_FAIL(GB_ERR_FORMAT, "multi-graph: an arc leaves its graph's vertex range");
  g->mg_ngraphs = ng;
  g->mg_hash = h;
  return GB_OK;
}

}  // namespace
}  // namespace gb

extern "C" int gb_multi_graph_bfs_cc(gb_graph* g, const uint32_t* graph_first, uint32_t ngraphs,
                                     const uint32_t* local_src, uint32_t* level_out, uint32_t* label_out,
                                     gb_stats* stats, void* stream) {
  using namespace gb;
  clear_error();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g || !graph_first || !local_src || (!level_out && !label_out))
    GB_FAIL(GB_ERR_ARG, "gb_multi_graph_bfs_cc: null argument");
  if (ngraphs == 0 || ngraphs > g->n) GB_FAIL(GB_ERR_ARG, "gb_multi_graph_bfs_cc: bad graph count %u", ngraphs);
  if (!g->symmetric) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_multi_graph_bfs_cc: needs symmetric graphs");
  if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_multi_graph_bfs_cc: the block-diagonal layout needs file order (graph was relabelled)");
  if (is_device_ptr(graph_first) || is_device_ptr(local_src))
    GB_FAIL(GB_ERR_ARG, "gb_multi_graph_bfs_cc: graph_first and local_src are host arrays");
  GB_CUDA(cudaSetDevice(g->device));
  int st = prepare_layout(g, graph_first, ngraphs, s);
  if (st != GB_OK) return st;
  for (uint32_t k = 0; k < ngraphs; ++k)
    if (local_src[k] >= graph_first[k + 1] - graph_first[k])
      GB_FAIL(GB_ERR_ARG, "gb_multi_graph_bfs_cc: local source %u of graph %u out of range", local_src[k], k);
  for (uint32_t k = 0; k < ngraphs; ++k) g->mg_stage[k] = graph_first[k] + local_src[k];
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaMemcpyAsync(g->mg_src, g->mg_stage, sizeof(uint32_t) * ngraphs, cudaMemcpyHostToDevice, s));
  const bool lev_dev = level_out && is_device_ptr(level_out);
  const bool lab_dev = label_out && is_device_ptr(label_out);
  uint32_t* d_level = lev_dev ? level_out : g->mg_level;
  uint32_t* d_label = lab_dev ? label_out : g->mg_label;
  if (level_out) {
    st = run_bfs_sources(g, g->mg_src, ngraphs, d_level, s);
    if (st != GB_OK) return st;
  }
  if (label_out) {
    st = run_cc(g, GB_CC_UNIONFIND, d_label, nullptr, s);
    if (st != GB_OK) return st;
    mg_localize<<<g->sm_count * 4, 256, 0, s>>>(d_label, g->n, g->mg_first, ngraphs);
    GB_CUDA(cudaGetLastError());
  }
  kt.stop(s);
  if (level_out && !lev_dev) GB_CUDA(cudaMemcpyAsync(level_out, d_level, sizeof(uint32_t) * g->n, cudaMemcpyDefault, s));
  if (label_out && !lab_dev) GB_CUDA(cudaMemcpyAsync(label_out, d_label, sizeof(uint32_t) * g->n, cudaMemcpyDefault, s));
  if (stats || (level_out && !lev_dev) || (label_out && !lab_dev)) {
    GB_CUDA(cudaStreamSynchronize(s));
    const int err = static_cast<int*>(g->pinned)[8];
    if (level_out && err) return dev_err_status(err, "gb_multi_graph_bfs_cc");
    if (stats) {
      *stats = gb_stats{};
      stats->vertices_reached = g->n;
      stats->edges_reached = g->m;
      stats->launches = 8;
      stats->kernel_ms = kt.ms();
    }
  }
  return GB_OK;
}
