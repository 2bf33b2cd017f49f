// Device mirror management: upload / .gr load / free / transpose / workspace.
//
// Replaces libgpu's CSRGraph::read + copy_to_gpu (libgpu/src/csr_graph.cu:
// 172-315), which kept uint32 offsets and copied edge by edge; here offsets are
// uint64, the upload is a handful of bulk copies, and the arrays are validated
// on the device before any kernel indexes through them.

#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

int cuda_fail(cudaError_t e, const char* what) {
  set_error("CUDA error %s (%d) in %s", cudaGetErrorString(e), (int)e, what);
  cudaGetLastError();  // clear sticky non-fatal state
  if (e == cudaErrorMemoryAllocation) return GB_ERR_OOM;
  return GB_ERR_CUDA;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

namespace {

struct Pool {
  std::mutex mu;
  // (device, rounded size) -> cached blocks; -1 is the pinned-host pool
  std::map<std::pair<int, size_t>, std::vector<void*>> free_blocks;
  std::unordered_map<void*, std::pair<int, size_t>> live;
};

Pool& pool() {
  static Pool* p = new Pool();  // never destroyed: blocks may be freed during process exit
  return *p;
}

size_t pool_round(size_t bytes) {
  const size_t g = bytes > (1u << 20) ? (2u << 20) : 4096;
  return (std::max<size_t>(bytes, 1) + g - 1) / g * g;
}

void pool_trim_locked(Pool& P, int device) {
  for (auto it = P.free_blocks.begin(); it != P.free_blocks.end();) {
    if (device == -2 || it->first.first == device) {
      for (void* b : it->second) {
        if (it->first.first == -1) cudaFreeHost(b);
        else cudaFree(b);
      }
      it = P.free_blocks.erase(it);
    } else {
      ++it;
    }
  }
}

cudaError_t pool_get(void** p, size_t bytes, bool host) {
  int dev = -1;
  if (!host && cudaGetDevice(&dev) != cudaSuccess) return cudaErrorInvalidDevice;
  const size_t sz = pool_round(bytes);
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.free_blocks.find({dev, sz});
  if (it != P.free_blocks.end() && !it->second.empty()) {
    *p = it->second.back();
    it->second.pop_back();
    P.live[*p] = {dev, sz};
    return cudaSuccess;
  }
  cudaError_t e = host ? cudaMallocHost(p, sz) : cudaMalloc(p, sz);
  if (e != cudaSuccess) {  // give the cached blocks of this device back and retry
    cudaGetLastError();
    pool_trim_locked(P, dev);
    e = host ? cudaMallocHost(p, sz) : cudaMalloc(p, sz);
  }
  if (e == cudaSuccess) P.live[*p] = {dev, sz};
  return e;
}

void pool_put(void* p, bool host) {
  if (!p) return;
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.live.find(p);
  if (it == P.live.end()) {  // not from the pool
    if (host) cudaFreeHost(p);
    else cudaFree(p);
    return;
  }
  P.free_blocks[it->second].push_back(p);
  P.live.erase(it);
}

}  // namespace

cudaError_t pool_malloc(void** p, size_t bytes) { return pool_get(p, bytes, false); }
void pool_free(void* p) { pool_put(p, false); }
cudaError_t pool_malloc_host(void** p, size_t bytes) { return pool_get(p, bytes, true); }
void pool_free_host(void* p) { pool_put(p, true); }

int ws_reserve(gb_graph* g, size_t bytes, cudaStream_t stream) {
  if (bytes <= g->ws_bytes) return GB_OK;
  if (g->ws) {
    GB_CUDA(cudaStreamSynchronize(stream));
    pool_free(g->ws);
    g->ws = nullptr;
    g->ws_bytes = 0;
  }
  size_t want = bytes + bytes / 8;  // headroom so repeat calls do not regrow
  void* p = nullptr;
  cudaError_t e = pool_malloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    want = bytes;
    GB_CUDA(pool_malloc(&p, want));
  }
  g->ws = p;
  g->ws_bytes = want;
  return GB_OK;
}

gb_tuning effective_tuning(const gb_graph* g) {
  gb_tuning t = g->tuning;
  if (!t.heavy_degree) t.heavy_degree = 128;
  if (!t.tile_edges) t.tile_edges = 256;
  if (!t.block_threads) t.block_threads = 1024;  // SSSP persistent CTA (1 per SM: cheap barrier)
  if (t.do_alpha <= 0.f) t.do_alpha = 15.f;  // bfsDirectionOpt.cpp:68-72
  if (t.do_beta <= 0.f) t.do_beta = 18.f;    // bfsDirectionOpt.cpp:73-77
  // local relaxation rounds pay off on low-degree, high-diameter graphs
  // (grids, road-like) and cost on power-law graphs
  if (t.local_depth == 0) t.local_depth = g->max_degree <= 32 ? 8 : -1;
  return t;
}

int coop_grid(const gb_graph* g, const void* kernel, int threads, size_t smem,
              uint32_t blocks_per_sm_cap) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (blocks_per_sm_cap && (uint32_t)per_sm > blocks_per_sm_cap) per_sm = (int)blocks_per_sm_cap;
  return per_sm * g->sm_count;
}

int dev_err_status(int code, const char* what) {
  switch (code) {
    case kDevOk: return GB_OK;
    case kDevTimeout:
      set_error("%s: a bounded device wait timed out", what);
      return GB_ERR_TIMEOUT;
    case kDevOverflow:
      set_error("%s: a device queue exceeded its capacity", what);
      return GB_ERR_CAPACITY;
    case kDevMaxRounds:
      set_error("%s: iteration cap reached", what);
      return GB_ERR_TIMEOUT;
    default:
      set_error("%s: device error %d", what, code);
      return GB_ERR_CUDA;
  }
}

int copy_out(void* dst, const void* src_dev, size_t bytes, cudaStream_t stream) {
  if (dst == src_dev || bytes == 0) return GB_OK;
  GB_CUDA(cudaMemcpyAsync(dst, src_dev, bytes, cudaMemcpyDefault, stream));
  if (!is_device_ptr(dst)) GB_CUDA(cudaStreamSynchronize(stream));
  return GB_OK;
}

int copy_in(void* dst_dev, const void* src, size_t bytes, cudaStream_t stream) {
  if (dst_dev == src || bytes == 0) return GB_OK;
  GB_CUDA(cudaMemcpyAsync(dst_dev, src, bytes, cudaMemcpyDefault, stream));
  return GB_OK;
}

namespace {

__global__ void validate_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col,
                                uint32_t n, uint64_t m, int* bad) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride)
    if (offs[v] > offs[v + 1]) atomicOr(bad, 1);
  if (tid == 0 && offs[n] != m) atomicOr(bad, 2);
  for (uint64_t e = tid; e < m; e += stride)
    if (col[e] >= n) atomicOr(bad, 4);
}

__global__ void transpose_keys_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col,
                                      uint32_t n, uint64_t* __restrict__ keys, uint64_t* __restrict__ vals) {
  // one warp per source vertex range (grid-stride over vertices)
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t warp = tid >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  for (uint64_t u = warp; u < n; u += nwarps) {
    const uint64_t b = offs[u], e = offs[u + 1];
    for (uint64_t i = b + lane; i < e; i += 32) {
      keys[i] = ((uint64_t)col[i] << 32) | (uint64_t)u;
      vals[i] = i;
    }
  }
}

__global__ void transpose_finish_kernel(const uint64_t* __restrict__ keys, const uint64_t* __restrict__ vals,
                                        uint64_t m, uint32_t* __restrict__ t_col,
                                        uint64_t* __restrict__ emap, const float* __restrict__ wf,
                                        float* __restrict__ t_wf, uint32_t* __restrict__ indeg) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < m; i += stride) {
    const uint64_t k = keys[i];
    t_col[i] = (uint32_t)(k & 0xFFFFFFFFull);
    emap[i] = vals[i];
    if (wf) t_wf[i] = wf[vals[i]];
    atomicAdd(&indeg[k >> 32], 1u);
  }
}

__global__ void degree_max_kernel(const uint64_t* __restrict__ offs, uint32_t n, unsigned* out) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned best = 0;
  for (uint64_t v = tid; v < n; v += stride) {
    const uint64_t d = offs[v + 1] - offs[v];
    best = max(best, (unsigned)(d > 0xFFFFFFFFull ? 0xFFFFFFFFull : d));
  }
  best = max(best, __reduce_max_sync(kFull, best));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

}  // namespace

int ensure_transpose(gb_graph* g, cudaStream_t stream) {
  if (g->t_offs) return GB_OK;
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  if (m >= (1ull << 32)) GB_FAIL(GB_ERR_UNSUPPORTED, "device transpose limited to < 2^32 arcs");
  uint64_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
  uint32_t* indeg = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  int st = GB_OK;
  auto cleanup = [&]() {
    cudaFree(keys);
    cudaFree(vals);
    cudaFree(keys2);
    cudaFree(vals2);
    cudaFree(indeg);
    cudaFree(tmp);
  };
#define GB_TRY(call)                       \
  do {                                     \
    cudaError_t _e = (call);               \
    if (_e != cudaSuccess) {               \
      st = cuda_fail(_e, #call);           \
      cleanup();                           \
      return st;                           \
    }                                      \
  } while (0)
  GB_TRY(cudaMalloc(&g->t_offs, sizeof(uint64_t) * (n + 1)));
  GB_TRY(cudaMalloc(&g->t_col, sizeof(uint32_t) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&g->t_emap, sizeof(uint64_t) * std::max<uint64_t>(m, 1)));
  if (g->wf) GB_TRY(cudaMalloc(&g->t_wf, sizeof(float) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&keys, sizeof(uint64_t) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&vals, sizeof(uint64_t) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&keys2, sizeof(uint64_t) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&vals2, sizeof(uint64_t) * std::max<uint64_t>(m, 1)));
  GB_TRY(cudaMalloc(&indeg, sizeof(uint32_t) * (n + 1)));
  GB_TRY(cudaMemsetAsync(indeg, 0, sizeof(uint32_t) * (n + 1), stream));
  const int blocks = g->sm_count * 8;
  if (m) transpose_keys_kernel<<<blocks, 256, 0, stream>>>(g->offs, g->col, n, keys, vals);
  int end_bit = 32;
  while (end_bit < 64 && (1ull << (end_bit - 32)) < (uint64_t)n) ++end_bit;
  GB_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, (int64_t)m, 0,
                                         end_bit, stream));
  GB_TRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
  GB_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, (int64_t)m, 0, end_bit,
                                         stream));
  if (m)
    transpose_finish_kernel<<<blocks, 256, 0, stream>>>(keys2, vals2, m, g->t_col, g->t_emap, g->wf,
                                                          g->t_wf, indeg);
  // exclusive scan of in-degrees -> begin offsets (uint32 counts, uint64 sums)
  {
    cudaFree(tmp);
    tmp = nullptr;
    size_t sb = 0;
    auto in_it = cub::TransformInputIterator<uint64_t, cub::CastOp<uint64_t>, const uint32_t*>(
        indeg, cub::CastOp<uint64_t>());
    GB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, sb, in_it, g->t_offs, (int64_t)n + 1, stream));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(sb, 16)));
    GB_TRY(cub::DeviceScan::ExclusiveSum(tmp, sb, in_it, g->t_offs, (int64_t)n + 1, stream));
  }
  GB_TRY(cudaStreamSynchronize(stream));
  cleanup();
#undef GB_TRY
  return GB_OK;
}

}  // namespace gb

using namespace gb;

extern "C" {

// A non-blocking stream per device for uploads, kept for the process: an
// upload's copies then overlap kernels that other streams run on the GPU
// (copies on the legacy default stream would wait for them).  Falls back to
// the default stream if one cannot be created.
static cudaStream_t upload_stream(int device) {
  static std::mutex mu;
  static std::vector<cudaStream_t> streams;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)streams.size() <= device) streams.resize(device + 1, nullptr);
  if (!streams[device] && cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    streams[device] = nullptr;
  }
  return streams[device];
}

int gb_graph_upload(const uint64_t* end_offs, const uint32_t* col, const uint32_t* w_u32,
                    const float* w_f32, uint32_t n, uint64_t m, int symmetric, int device,
                    gb_graph** out) {
  clear_error();
  if (!out) GB_FAIL(GB_ERR_ARG, "gb_graph_upload: null output handle");
  *out = nullptr;
  if (n == 0) GB_FAIL(GB_ERR_ARG, "gb_graph_upload: graph has no nodes");
  if ((!end_offs) || (m && !col)) GB_FAIL(GB_ERR_ARG, "gb_graph_upload: null array");
  int ndev = 0;
  GB_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) GB_FAIL(GB_ERR_ARG, "gb_graph_upload: bad device %d", device);
  GB_CUDA(cudaSetDevice(device));
  gb_graph* g = new (std::nothrow) gb_graph();
  if (!g) GB_FAIL(GB_ERR_OOM, "host allocation failed");
  g->device = device;
  g->n = n;
  g->m = m;
  g->symmetric = symmetric ? 1 : 0;
  cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, device);
  auto fail = [&](int st) {
    gb_graph_free(g);
    return st;
  };
  cudaError_t e;
  auto dalloc = [](auto** p, size_t bytes) { return pool_malloc(reinterpret_cast<void**>(p), bytes); };
  if ((e = dalloc(&g->offs, sizeof(uint64_t) * (n + 1))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc offs"));
  if ((e = dalloc(&g->col, sizeof(uint32_t) * std::max<uint64_t>(m, 1))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc col"));
  if (w_u32 && (e = dalloc(&g->w, sizeof(uint32_t) * std::max<uint64_t>(m, 1))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc w"));
  if (w_f32 && (e = dalloc(&g->wf, sizeof(float) * std::max<uint64_t>(m, 1))) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc wf"));
  if ((e = pool_malloc_host(&g->pinned, 8192)) != cudaSuccess) return fail(cuda_fail(e, "cudaMallocHost"));
  // host inputs are ready now; device inputs may still be written by work
  // queued on other streams, which the default stream waits for
  const bool dev_in = is_device_ptr(end_offs) || (m && is_device_ptr(col)) || (w_u32 && is_device_ptr(w_u32)) ||
                      (w_f32 && is_device_ptr(w_f32));
  cudaStream_t s = dev_in ? cudaStream_t(0) : upload_stream(device);
  if ((e = cudaMemsetAsync(g->offs, 0, sizeof(uint64_t), s)) != cudaSuccess) return fail(cuda_fail(e, "memset"));
  if ((e = cudaMemcpyAsync(g->offs + 1, end_offs, sizeof(uint64_t) * n, cudaMemcpyDefault, s)) != cudaSuccess) return fail(cuda_fail(e, "copy offs"));
  if (m && (e = cudaMemcpyAsync(g->col, col, sizeof(uint32_t) * m, cudaMemcpyDefault, s)) != cudaSuccess) return fail(cuda_fail(e, "copy col"));
  if (w_u32 && m && (e = cudaMemcpyAsync(g->w, w_u32, sizeof(uint32_t) * m, cudaMemcpyDefault, s)) != cudaSuccess) return fail(cuda_fail(e, "copy w"));
  if (w_f32 && m && (e = cudaMemcpyAsync(g->wf, w_f32, sizeof(float) * m, cudaMemcpyDefault, s)) != cudaSuccess) return fail(cuda_fail(e, "copy wf"));
  int* flag = static_cast<int*>(g->pinned);
  unsigned* maxdeg = reinterpret_cast<unsigned*>(static_cast<char*>(g->pinned) + 64);
  int* dflag = nullptr;
  if ((e = pool_malloc(reinterpret_cast<void**>(&dflag), 64)) != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc flag"));
  cudaMemsetAsync(dflag, 0, 64, s);
  validate_kernel<<<g->sm_count * 4, 256, 0, s>>>(g->offs, g->col, n, m, dflag);
  degree_max_kernel<<<g->sm_count * 4, 256, 0, s>>>(g->offs, n, reinterpret_cast<unsigned*>(dflag + 4));
  cudaMemcpyAsync(flag, dflag, 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(maxdeg, dflag + 4, 4, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  pool_free(dflag);
  if (e != cudaSuccess) return fail(cuda_fail(e, "graph validation"));
  if (*flag) {
    gb_graph_free(g);
    GB_FAIL(GB_ERR_FORMAT, "gb_graph_upload: invalid CSR (%s%s%s)", (*flag & 1) ? "non-monotone offsets " : "",
            (*flag & 2) ? "last offset != m " : "", (*flag & 4) ? "destination id >= n" : "");
  }
  g->max_degree = *maxdeg;
  g->zero_from = n;
  *out = g;
  return GB_OK;
}

int gb_graph_load_gr(const char* path, int edge_bytes, int symmetric, int device, gb_graph** out) {
  gb_host_csr h;
  gb_host_csr_init(&h);
  int st = gb_gr_read(path, edge_bytes, &h);
  if (st != GB_OK) return st;
  st = gb_graph_upload(h.end_offs, h.col, h.w_u32, h.w_f32, h.n, h.m, symmetric, device, out);
  gb_host_csr_free(&h);
  return st;
}

int gb_graph_free(gb_graph* g) {
  if (!g) return GB_OK;
  cudaSetDevice(g->device);
  // pooled blocks are reused by the next upload: no kernel may still use them
  cudaDeviceSynchronize();
  pool_free(g->offs);
  pool_free(g->col);
  pool_free(g->w);
  pool_free(g->wf);
  cudaFree(g->t_offs);
  cudaFree(g->t_col);
  cudaFree(g->t_wf);
  cudaFree(g->t_emap);
  cudaFree(g->outdeg_of_stored);
  cudaFree(g->lr_rowid);
  gb::free_pr_bins(g);
  cudaFree(g->colsum);
  cudaFree(g->ell);
  if (g->ppr_free) g->ppr_free(g);
  pool_free(g->sweep_tiles);
  pool_free(g->sweep_heavy_list);
  cudaFree(g->mg_first);
  cudaFree(g->mg_src);
  cudaFree(g->mg_level);
  cudaFree(g->mg_label);
  if (g->mg_stage) cudaFreeHost(g->mg_stage);
  cudaFree(g->perm);
  cudaFree(g->iperm);
  cudaFree(g->ro_buf);
  std::free(g->h_iperm);
  pool_free(g->ws);
  pool_free_host(g->pinned);
  delete g;
  return GB_OK;
}

int gb_pool_trim(void) {
  clear_error();
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  pool_trim_locked(P, -2);
  return GB_OK;
}

int gb_graph_info(const gb_graph* g, uint32_t* n, uint64_t* m, int* symmetric) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_info: null graph");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (symmetric) *symmetric = g->symmetric;
  return GB_OK;
}

int gb_graph_device_arrays(const gb_graph* g, const uint64_t** offs, const uint32_t** col,
                           const uint32_t** w_u32, const float** w_f32) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_device_arrays: null graph");
  if (offs) *offs = g->offs;
  if (col) *col = g->col;
  if (w_u32) *w_u32 = g->w;
  if (w_f32) *w_f32 = g->wf;
  return GB_OK;
}

int gb_graph_build_transpose(gb_graph* g, void* stream) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_build_transpose: null graph");
  GB_CUDA(cudaSetDevice(g->device));
  return ensure_transpose(g, static_cast<cudaStream_t>(stream));
}

int gb_graph_set_tuning(gb_graph* g, const gb_tuning* t) {
  clear_error();
  if (!g || !t) GB_FAIL(GB_ERR_ARG, "gb_graph_set_tuning: null argument");
  if (t->block_threads && (t->block_threads % 32 || t->block_threads > 1024))
    GB_FAIL(GB_ERR_ARG, "block_threads must be a multiple of 32 and <= 1024");
  if (t->tile_edges && t->tile_edges < 32) GB_FAIL(GB_ERR_ARG, "tile_edges must be >= 32");
  g->tuning = *t;
  return GB_OK;
}

int gb_graph_get_tuning(const gb_graph* g, gb_tuning* t) {
  clear_error();
  if (!g || !t) GB_FAIL(GB_ERR_ARG, "gb_graph_get_tuning: null argument");
  *t = effective_tuning(g);
  return GB_OK;
}

}  // extern "C"
