// Graph conversion on the device: the graph-convert steps that sit beside the
// edge-map path, applied to a resident gb_graph instead of a file.
//
//  * gb_graph_symmetrize: gr2sgr (graph-convert.cpp:1350-1364 via
//    FileGraph.h:764-826 makeSymmetric) adds, for every arc (u, v) with
//    u != v, the reverse arc (v, u) carrying the same edge data; self-loops
//    stay single.  With cleanup it continues as gr2cgr (Cleanup,
//    graph-convert.cpp:1902-2024): rows sorted by destination, self-loops
//    and repeated arcs removed.
//    B200 form: the m forward and the non-self reverse arcs become 64-bit
//    keys (source << 32 | destination) with their source arc index as value,
//    one stable radix sort orders them by (source, destination), and a
//    compaction, an offsets pass and a gather of the edge data build the new
//    CSR.  The reference appends arcs in file order; here every row comes
//    out sorted, which no algorithm on the path observes except through
//    floating-point summation order.  Of repeated arcs the one kept is the
//    first in (forward arcs, then reverse arcs) arc order, which decides
//    whose weight survives; the reference's unstable sort leaves that open.
//  * gb_graph_assign_weights_u32 / _f32: gr2randomweightgr
//    (graph-convert.cpp:1169-1190) draws a weight per arc.  The reference
//    uses one sequential mt19937 stream; here arc e takes the e-th value of a
//    counter-based stream (the host generators' stream_key / rand_at), so the
//    device fills every arc in parallel and matches gb_assign_weights_u32 /
//    _f32 on the host bit for bit.
//  * gb_graph_assign_weights_reference: the reference converter's own draws
//    (one sequential std::mt19937 stream), made on the host and uploaded.

#include <algorithm>

#include <cub/cub.cuh>

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

namespace {

constexpr uint64_t kDropKey = ~0ull;

// Forward arcs at [0, m), reverse copies at [m, 2m); a self-loop's reverse
// copy gets kDropKey (sorted past every real key, then cut).  A warp per row.
__global__ void sym_keys_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col, uint32_t n,
                                uint64_t m, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                unsigned long long* self_loops) {
  const uint32_t lane = lane_id();
  const uint64_t gwarp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long loops = 0;
  for (uint64_t v = gwarp; v < n; v += nwarps) {
    const uint64_t b = offs[v], e = offs[v + 1];
    for (uint64_t i = b + lane; i < e; i += 32) {
      const uint32_t d = col[i];
      keys[i] = (v << 32) | d;
      vals[i] = (uint32_t)i;
      keys[m + i] = d == v ? kDropKey : (((uint64_t)d << 32) | v);
      vals[m + i] = (uint32_t)i;
      loops += d == v;
    }
  }
  loops = warp_sum(loops);
  if (lane == 0 && loops) atomicAdd(self_loops, loops);
}

// keep[i]: not a self-loop and not a repeat of the previous key
__global__ void cleanup_flags_kernel(const uint64_t* __restrict__ keys, uint64_t cnt, uint8_t* __restrict__ keep) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < cnt; i += stride) {
    const uint64_t k = keys[i];
    const bool self = (uint32_t)(k >> 32) == (uint32_t)k;
    keep[i] = !self && (i == 0 || keys[i - 1] != k);
  }
}

// offs[v] = first position whose source is >= v, for v in [0, n]
__global__ void offsets_from_keys_kernel(const uint64_t* __restrict__ keys, uint64_t cnt, uint32_t n,
                                         uint64_t* __restrict__ offs) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i <= cnt; i += stride) {
    const uint64_t first = i == 0 ? 0 : (keys[i - 1] >> 32) + 1;
    const uint64_t last = i == cnt ? n : (keys[i] >> 32);
    for (uint64_t v = first; v <= last; ++v) offs[v] = i;
  }
}

__global__ void unpack_arcs_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint64_t cnt,
                                   const uint32_t* __restrict__ w, const float* __restrict__ wf,
                                   uint32_t* __restrict__ ncol, uint32_t* __restrict__ nw, float* __restrict__ nwf) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < cnt; i += stride) {
    ncol[i] = (uint32_t)keys[i];
    if (nw) nw[i] = w[vals[i]];
    if (nwf) nwf[i] = wf[vals[i]];
  }
}

__global__ void max_degree_kernel(const uint64_t* __restrict__ offs, uint32_t n, unsigned* out) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned best = 0;
  for (uint64_t v = tid; v < n; v += stride) {
    const uint64_t d = offs[v + 1] - offs[v];
    best = max(best, (unsigned)(d > 0xFFFFFFFFull ? 0xFFFFFFFFull : d));
  }
  best = __reduce_max_sync(kFull, best);
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void weights_u32_kernel(uint32_t* __restrict__ w, uint64_t m, uint64_t key, uint32_t lo, uint64_t span) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = tid; e < m; e += stride) w[e] = lo + (uint32_t)__umul64hi(rand_at(key, e), span);
}

__global__ void weights_f32_kernel(float* __restrict__ w, uint64_t m, uint64_t key) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = tid; e < m; e += stride) {
    const uint64_t r = (rand_at(key, e) >> 40) + 1;  // 24 random bits -> (0, 1]
    w[e] = (float)r * (1.0f / 16777216.0f);
  }
}

int grid_for(const gb_graph* g, uint64_t work) {
  const uint64_t b = (work + 255) / 256;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)g->sm_count * 8));
}

}  // namespace

}  // namespace gb

extern "C" {

int gb_graph_symmetrize(gb_graph* g, int cleanup, void* stream) {
  using namespace gb;
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_symmetrize: null graph");
  if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_symmetrize: symmetrize before gb_graph_reorder");
  const uint64_t m = g->m;
  if (m >= (1ull << 31)) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_symmetrize: limited to < 2^31 arcs");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t n = g->n;
  const uint64_t m2 = 2 * m;
  uint64_t *keys = nullptr, *keys2 = nullptr, *noffs = nullptr;
  uint32_t *vals = nullptr, *vals2 = nullptr, *ncol = nullptr, *nw = nullptr;
  float* nwf = nullptr;
  uint8_t* keep = nullptr;
  unsigned long long* cnt = nullptr;  // [0] self-loops, [1] kept, [2] max degree
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  int st = GB_OK;
  auto release = [&](bool keep_new) {
    cudaFree(keys);
    cudaFree(keys2);
    cudaFree(vals);
    cudaFree(vals2);
    cudaFree(keep);
    cudaFree(cnt);
    cudaFree(tmp);
    if (!keep_new) {
      pool_free(noffs);
      pool_free(ncol);
      pool_free(nw);
      pool_free(nwf);
    }
  };
#define GB_TRY(call)             \
  do {                           \
    cudaError_t _e = (call);     \
    if (_e != cudaSuccess) {     \
      st = cuda_fail(_e, #call); \
      release(false);            \
      return st;                 \
    }                            \
  } while (0)
  const size_t e1 = std::max<uint64_t>(m2, 1);
  GB_TRY(cudaMalloc(&keys, sizeof(uint64_t) * e1));
  GB_TRY(cudaMalloc(&keys2, sizeof(uint64_t) * e1));
  GB_TRY(cudaMalloc(&vals, sizeof(uint32_t) * e1));
  GB_TRY(cudaMalloc(&vals2, sizeof(uint32_t) * e1));
  GB_TRY(cudaMalloc(&cnt, 4 * sizeof(unsigned long long)));
  GB_TRY(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), s));
  unsigned long long* h = static_cast<unsigned long long*>(g->pinned);
  if (m) {
    sym_keys_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, g->col, n, m, keys, vals, cnt);
    GB_TRY(cudaGetLastError());
    int end_bit = 33;  // keys: 32 destination bits + enough source bits, or all ones
    while (end_bit < 64 && (1ull << (end_bit - 32)) < (uint64_t)n) ++end_bit;
    GB_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, (int64_t)m2, 0, end_bit, s));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
    GB_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, (int64_t)m2, 0, end_bit, s));
  }
  GB_TRY(cudaMemcpyAsync(h, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  GB_TRY(cudaStreamSynchronize(s));
  const uint64_t valid = m2 - h[0];  // drop keys sort last
  uint64_t mm = valid;
  const uint64_t* fkeys = keys2;
  const uint32_t* fvals = vals2;
  if (cleanup && valid) {
    GB_TRY(cudaMalloc(&keep, valid));
    cleanup_flags_kernel<<<grid_for(g, valid), 256, 0, s>>>(keys2, valid, keep);
    GB_TRY(cudaGetLastError());
    cudaFree(tmp);
    tmp = nullptr;
    size_t sb = 0, sb2 = 0;
    GB_TRY(cub::DeviceSelect::Flagged(nullptr, sb, keys2, keep, keys, cnt + 1, (int64_t)valid, s));
    GB_TRY(cub::DeviceSelect::Flagged(nullptr, sb2, vals2, keep, vals, cnt + 1, (int64_t)valid, s));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(std::max(sb, sb2), 16)));
    GB_TRY(cub::DeviceSelect::Flagged(tmp, sb2, vals2, keep, vals, cnt + 1, (int64_t)valid, s));
    GB_TRY(cub::DeviceSelect::Flagged(tmp, sb, keys2, keep, keys, cnt + 1, (int64_t)valid, s));
    GB_TRY(cudaMemcpyAsync(h + 1, cnt + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    GB_TRY(cudaStreamSynchronize(s));
    mm = h[1];
    fkeys = keys;
    fvals = vals;
  }
  const size_t mm1 = std::max<uint64_t>(mm, 1);
  GB_TRY(pool_malloc(reinterpret_cast<void**>(&noffs), sizeof(uint64_t) * (n + 1)));
  GB_TRY(pool_malloc(reinterpret_cast<void**>(&ncol), sizeof(uint32_t) * mm1));
  if (g->w) GB_TRY(pool_malloc(reinterpret_cast<void**>(&nw), sizeof(uint32_t) * mm1));
  if (g->wf) GB_TRY(pool_malloc(reinterpret_cast<void**>(&nwf), sizeof(float) * mm1));
  offsets_from_keys_kernel<<<grid_for(g, mm + 1), 256, 0, s>>>(fkeys, mm, n, noffs);
  if (mm) unpack_arcs_kernel<<<grid_for(g, mm), 256, 0, s>>>(fkeys, fvals, mm, g->w, g->wf, ncol, nw, nwf);
  unsigned* dmax = reinterpret_cast<unsigned*>(cnt + 2);
  max_degree_kernel<<<grid_for(g, n), 256, 0, s>>>(noffs, n, dmax);
  GB_TRY(cudaGetLastError());
  GB_TRY(cudaMemcpyAsync(h + 2, cnt + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  GB_TRY(cudaStreamSynchronize(s));
#undef GB_TRY
  const unsigned maxdeg = (unsigned)(h[2] & 0xFFFFFFFFull);
  drop_derived(g);
  pool_free(g->offs);
  pool_free(g->col);
  pool_free(g->w);
  pool_free(g->wf);
  g->offs = noffs;
  g->col = ncol;
  g->w = nw;
  g->wf = nwf;
  g->m = mm;
  g->symmetric = 1;
  g->max_degree = maxdeg;
  g->zero_from = n;
  release(true);
  return GB_OK;
}

int gb_graph_assign_weights_u32(gb_graph* g, uint32_t lo, uint32_t hi, uint64_t seed, void* stream) {
  using namespace gb;
  clear_error();
  if (!g || hi < lo) GB_FAIL(GB_ERR_ARG, "gb_graph_assign_weights_u32: bad argument");
  if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_assign_weights_u32: assign weights before gb_graph_reorder");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g->w) {
    cudaError_t e = pool_malloc(reinterpret_cast<void**>(&g->w), sizeof(uint32_t) * std::max<uint64_t>(g->m, 1));
    if (e != cudaSuccess) return cuda_fail(e, "gb_graph_assign_weights_u32");
  }
  cudaFree(g->ell);  // its rows carry the weights
  g->ell = nullptr;
  g->ell_d = 0;
  if (g->m)
    weights_u32_kernel<<<grid_for(g, g->m), 256, 0, s>>>(g->w, g->m, stream_key(seed, kTagWeightU32), lo,
                                                         (uint64_t)hi - lo + 1);
  GB_CUDA(cudaGetLastError());
  return GB_OK;
}

int gb_graph_assign_weights_f32(gb_graph* g, uint64_t seed, void* stream) {
  using namespace gb;
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_assign_weights_f32: null graph");
  if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_assign_weights_f32: assign weights before gb_graph_reorder");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  // float weights feed the transpose's copy and the PPR state: rebuilt on use
  drop_derived(g);
  if (!g->wf) {
    cudaError_t e = pool_malloc(reinterpret_cast<void**>(&g->wf), sizeof(float) * std::max<uint64_t>(g->m, 1));
    if (e != cudaSuccess) return cuda_fail(e, "gb_graph_assign_weights_f32");
  }
  if (g->m) weights_f32_kernel<<<grid_for(g, g->m), 256, 0, s>>>(g->wf, g->m, stream_key(seed, kTagWeightF32));
  GB_CUDA(cudaGetLastError());
  return GB_OK;
}

int gb_graph_assign_weights_reference(gb_graph* g, int min_value, int max_value, int edge_bytes, void* stream) {
  using namespace gb;
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_assign_weights_reference: null graph");
  int st = check_reference_weights(min_value, max_value, edge_bytes, "gb_graph_assign_weights_reference");
  if (st != GB_OK) return st;
  if (g->perm)
    GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_assign_weights_reference: assign weights before gb_graph_reorder");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (edge_bytes == -4) drop_derived(g);  // float weights feed the transpose's copy and the PPR state
  cudaFree(g->ell);                       // uint32 weights ride in the fixed-width rows
  g->ell = nullptr;
  g->ell_d = 0;
  void** dst = edge_bytes == 4 ? reinterpret_cast<void**>(&g->w) : reinterpret_cast<void**>(&g->wf);
  const size_t bytes = 4 * std::max<uint64_t>(g->m, 1);
  if (!*dst) {
    cudaError_t e = pool_malloc(dst, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "gb_graph_assign_weights_reference");
  }
  void* h = nullptr;
  cudaError_t e = pool_malloc_host(&h, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "gb_graph_assign_weights_reference");
  draw_reference_weights(g->m, min_value, max_value, edge_bytes, h);
  e = cudaMemcpyAsync(*dst, h, 4 * g->m, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  pool_free_host(h);
  if (e != cudaSuccess) return cuda_fail(e, "gb_graph_assign_weights_reference");
  return GB_OK;
}

}  // extern "C"
