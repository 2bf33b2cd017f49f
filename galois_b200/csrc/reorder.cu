// Degree-ordered relabelling of the device mirror, and the mapping of results
// back to original vertex ids.
//
// On power-law graphs most gathers of a vertex array (PageRank contributions,
// CC parents, BFS visited bits, SSSP distances) hit the few high-degree
// vertices.  Under file order those sit on distinct cache lines shared with
// cold vertices; renumbered by descending degree, the hot entries pack into
// a few lines that stay in L1/L2.  The kernels are unchanged: they run on the
// relabelled CSR, and the entry points translate sources in and results out.
//
// GB_ORDER_LOCALITY (no counterpart in the reference either) serves
// bounded-degree, high-diameter graphs instead (grids, meshes, road-like
// graphs): without coordinates it takes a vertex's BFS distances to two
// far-apart landmarks as coordinates (landmark A: the vertex farthest from
// vertex 0; B: farthest from A; C: farthest from both A and B -- on a grid,
// three corners -- coordinates (d_A, d_C)) and numbers the vertices in the
// Morton (Z) order of those coordinates, so that consecutive ids form compact
// 2-D patches instead of long rows.
//
// Steps (all on the device, one stream):
//   1. deg[v] = offs[v+1] - offs[v]; radix sort (deg desc, id) -> perm
//      (new -> old, stable so equal degrees keep id order); iperm = inverse
//      [locality: radix sort (Morton key, id) -> perm]
//   2. new offsets = exclusive scan of the sorted degrees
//   3. one warp per new row copies the old row with columns mapped through
//      iperm (weights follow their arcs)
//   4. each row sorted ascending (cub segmented sort; weights packed as values)

#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

int run_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats, cudaStream_t s, void* scratch,
            size_t scratch_bytes);

namespace {

__global__ void degree_ids_kernel(const uint64_t* __restrict__ offs, uint32_t n, uint32_t* __restrict__ deg,
                                  uint32_t* __restrict__ ids) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += stride) {
    const uint64_t d = offs[v + 1] - offs[v];
    deg[v] = d > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)d;
    ids[v] = (uint32_t)v;
  }
}

// First index of the (descending) sorted degrees that is zero.
__global__ void first_zero_kernel(const uint32_t* __restrict__ deg_sorted, uint32_t n, uint32_t* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    if (deg_sorted[i] == 0 && (i == 0 || deg_sorted[i - 1] != 0)) atomicMin(out, (uint32_t)i);
}

__global__ void invert_kernel(const uint32_t* __restrict__ perm, uint32_t n, uint32_t* __restrict__ iperm) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) iperm[perm[i]] = (uint32_t)i;
}

// One warp per new row: copy old row perm[i] with ids mapped through iperm.
// packed (optional) receives (w << 32 | float bits of wf) per arc for the
// row sort; otherwise the weights are written directly.
__global__ void relabel_rows_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col,
                                    const uint32_t* __restrict__ w, const float* __restrict__ wf,
                                    const uint32_t* __restrict__ perm, const uint32_t* __restrict__ iperm,
                                    const uint64_t* __restrict__ noffs, uint32_t n, uint32_t* __restrict__ ncol,
                                    uint32_t* __restrict__ nw, float* __restrict__ nwf,
                                    uint64_t* __restrict__ packed) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  for (uint64_t i = warp; i < n; i += nwarps) {
    const uint32_t old = perm[i];
    const uint64_t b = offs[old], len = offs[old + 1] - b, d = noffs[i];
    for (uint64_t k = lane; k < len; k += 32) {
      ncol[d + k] = iperm[col[b + k]];
      if (packed) {
        const uint64_t hi = w ? (uint64_t)w[b + k] << 32 : 0;
        const uint64_t lo = wf ? (uint64_t)__float_as_uint(wf[b + k]) : 0;
        packed[d + k] = hi | lo;
      } else {
        if (nw) nw[d + k] = w[b + k];
        if (nwf) nwf[d + k] = wf[b + k];
      }
    }
  }
}

__global__ void unpack_kernel(const uint64_t* __restrict__ packed, uint64_t m, uint32_t* __restrict__ nw,
                              float* __restrict__ nwf) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint64_t p = packed[e];
    if (nw) nw[e] = (uint32_t)(p >> 32);
    if (nwf) nwf[e] = __uint_as_float((uint32_t)(p & 0xFFFFFFFFull));
  }
}

// out[original v] = res[iperm[v]]
template <class T>
__global__ void gather_out_kernel(const T* __restrict__ res, const uint32_t* __restrict__ iperm, uint32_t n,
                                  T* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += stride) out[v] = res[iperm[v]];
}

// minorig[label of internal v] = min original id over the component.  A giant
// component sends most threads to one word: read it first (from L2) and only
// issue the atomic when it would lower the value, so after the first few
// updates the threads only read.
// over internal ids [0, n): the least original id under each label
__global__ void label_min_kernel(const uint32_t* __restrict__ lab, const uint32_t* __restrict__ perm, uint32_t n,
                                 uint32_t* __restrict__ minorig) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t l = lab[i], o = perm[i];
    if (__ldcg(&minorig[l]) > o) atomicMin(&minorig[l], o);
  }
}

// out[original v] = minorig[lab[iperm[v]]]; a vertex from `single` on (no
// arcs on a symmetric graph: a component of its own) is its own answer
__global__ void label_out_kernel(const uint32_t* __restrict__ lab, const uint32_t* __restrict__ minorig,
                                 const uint32_t* __restrict__ iperm, uint32_t n, uint32_t single,
                                 uint32_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += stride) {
    const uint32_t iv = iperm[v];
    out[v] = iv >= single ? (uint32_t)v : minorig[lab[iv]];
  }
}

// Largest reached level, ties to the smallest id: key = level << 32 | ~v.
__global__ void far_vertex_kernel(const uint32_t* __restrict__ lv, const uint32_t* __restrict__ lv2, uint32_t n,
                                  unsigned long long* best) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long mine = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += stride) {
    uint32_t d = lv[v];
    if (d == kInf) continue;
    if (lv2) {  // farthest from both: the smaller of the two distances
      const uint32_t d2 = lv2[v];
      if (d2 == kInf) continue;
      d = min(d, d2);
    }
    const unsigned long long key = ((unsigned long long)d << 32) | (0xFFFFFFFFu - (uint32_t)v);
    mine = key > mine ? key : mine;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(kFull, mine, o);
    mine = other > mine ? other : mine;
  }
  if ((threadIdx.x & 31) == 0 && mine) atomicMax(best, mine);
}

__device__ __forceinline__ uint32_t spread16(uint32_t x) {  // bit i -> bit 2i
  x &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// Morton key of (dx, dy) >> shift per vertex; unreached vertices go last.
__global__ void morton_kernel(const uint32_t* __restrict__ dx, const uint32_t* __restrict__ dy, uint32_t n,
                              uint32_t shift, uint32_t* __restrict__ key, uint32_t* __restrict__ ids) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += stride) {
    const uint32_t x = dx[v], y = dy[v];
    key[v] = (x == kInf || y == kInf) ? 0xFFFFFFFFu : (spread16(x >> shift) | (spread16(y >> shift) << 1));
    ids[v] = (uint32_t)v;
  }
}

__global__ void gather_deg_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ perm, uint32_t n,
                                  uint32_t* __restrict__ deg_sorted) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t v = perm[i];
    const uint64_t d = offs[v + 1] - offs[v];
    deg_sorted[i] = d > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)d;
  }
}

int blocks_for(const gb_graph* g, uint64_t work) {
  const uint64_t b = (work + 255) / 256;
  const uint64_t cap = (uint64_t)g->sm_count * 8;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, cap));
}

}  // namespace

// Drop every cached array derived from the stored arcs (transpose, sweep
// schedules, PageRank/PPR state, multi-graph layout): used when the arcs or
// their numbering change.
void drop_derived(gb_graph* g) {
  cudaFree(g->t_offs);
  cudaFree(g->t_col);
  cudaFree(g->t_wf);
  cudaFree(g->t_emap);
  g->t_offs = nullptr;
  g->t_col = nullptr;
  g->t_wf = nullptr;
  g->t_emap = nullptr;
  cudaFree(g->outdeg_of_stored);
  cudaFree(g->lr_rowid);
  g->lr_rowid = nullptr;
  free_pr_bins(g);
  cudaFree(g->colsum);
  g->outdeg_of_stored = nullptr;
  g->colsum = nullptr;
  cudaFree(g->ell);
  g->ell = nullptr;
  g->ell_d = 0;
  g->region_arcs = 0;
  pool_free(g->sweep_tiles);
  pool_free(g->sweep_heavy_list);
  g->sweep_tiles = nullptr;
  g->sweep_heavy_list = nullptr;
  g->sweep_ntiles = g->sweep_nheavy = g->sweep_heavy = g->sweep_tile = 0;
  if (g->ppr_free) g->ppr_free(g);
  g->ppr_free = nullptr;
  cudaFree(g->mg_first);
  cudaFree(g->mg_src);
  cudaFree(g->mg_level);
  cudaFree(g->mg_label);
  if (g->mg_stage) cudaFreeHost(g->mg_stage);
  g->mg_first = g->mg_src = g->mg_level = g->mg_label = g->mg_stage = nullptr;
  g->mg_ngraphs = 0;
  g->mg_hash = 0;
}

int reserve_result_bufs(gb_graph* g) {
  if (g->ro_buf) return GB_OK;
  GB_CUDA(cudaMalloc(&g->ro_buf, sizeof(uint32_t) * 3 * (size_t)g->n));
  return GB_OK;
}

uint32_t* result_buf(gb_graph* g, int k) { return g->ro_buf + (size_t)k * g->n; }

template <class T>
static int finish_gather(gb_graph* g, const T* res, T* out, cudaStream_t s) {
  const uint32_t n = g->n;
  if (is_device_ptr(out)) {
    gather_out_kernel<T><<<blocks_for(g, n), 256, 0, s>>>(res, g->iperm, n, out);
    GB_CUDA(cudaGetLastError());
    return GB_OK;
  }
  T* tmp = reinterpret_cast<T*>(result_buf(g, 1));
  gather_out_kernel<T><<<blocks_for(g, n), 256, 0, s>>>(res, g->iperm, n, tmp);
  GB_CUDA(cudaGetLastError());
  return copy_out(out, tmp, sizeof(T) * n, s);
}

int finish_u32(gb_graph* g, const uint32_t* res, uint32_t* out, cudaStream_t s) {
  return finish_gather<uint32_t>(g, res, out, s);
}

int finish_f32(gb_graph* g, const float* res, float* out, cudaStream_t s) {
  return finish_gather<float>(g, res, out, s);
}

int finish_labels(gb_graph* g, const uint32_t* res, uint32_t* out, cudaStream_t s) {
  const uint32_t n = g->n;
  // on a symmetric degree-ordered graph the vertices from zero_from on have
  // no arcs: components of their own, labelled by themselves, which no other
  // label reaches (a component's least id is below zero_from)
  const uint32_t single = g->symmetric ? g->zero_from : n;
  uint32_t* minorig = result_buf(g, 1);
  GB_CUDA(cudaMemsetAsync(minorig, 0xFF, sizeof(uint32_t) * single, s));
  if (single) label_min_kernel<<<blocks_for(g, single), 256, 0, s>>>(res, g->perm, single, minorig);
  const bool dev = is_device_ptr(out);
  uint32_t* dst = dev ? out : result_buf(g, 2);
  label_out_kernel<<<blocks_for(g, n), 256, 0, s>>>(res, minorig, g->iperm, n, single, dst);
  GB_CUDA(cudaGetLastError());
  return dev ? GB_OK : copy_out(out, dst, sizeof(uint32_t) * n, s);
}

int reorder_graph(gb_graph* g, int order, cudaStream_t s) {
  if (order == GB_ORDER_NONE) {
    if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_reorder: a relabelled graph cannot be restored");
    return GB_OK;
  }
  if (order == GB_ORDER_AUTO) order = g->max_degree <= 16 ? GB_ORDER_LOCALITY : GB_ORDER_DEGREE;
  if (order != GB_ORDER_DEGREE && order != GB_ORDER_DEGREE_UNSORTED && order != GB_ORDER_LOCALITY)
    GB_FAIL(GB_ERR_ARG, "gb_graph_reorder: unknown order %d", order);
  if (g->perm) {
    if (g->order == order) return GB_OK;
    GB_FAIL(GB_ERR_UNSUPPORTED, "gb_graph_reorder: graph already relabelled with order %d", g->order);
  }
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const bool sort_rows = order != GB_ORDER_DEGREE_UNSORTED && m < (1ull << 31);
  const bool locality = order == GB_ORDER_LOCALITY;
  const bool weighted = g->w || g->wf;

  uint32_t *deg = nullptr, *deg2 = nullptr, *ids = nullptr, *perm = nullptr, *iperm = nullptr;
  uint64_t* noffs = nullptr;
  uint32_t *ncol = nullptr, *ncol2 = nullptr, *nw = nullptr;
  float* nwf = nullptr;
  uint64_t *packed = nullptr, *packed2 = nullptr;
  uint32_t* h_iperm = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  uint32_t *da = nullptr, *db = nullptr, *dc = nullptr;  // locality: landmark distances
  unsigned long long* best = nullptr;
  auto cleanup = [&](bool keep_new) {
    cudaFree(da);
    cudaFree(db);
    cudaFree(dc);
    cudaFree(best);
    da = db = dc = nullptr;
    best = nullptr;
    cudaFree(deg);
    cudaFree(deg2);
    cudaFree(ids);
    cudaFree(ncol2);
    cudaFree(packed);
    cudaFree(packed2);
    cudaFree(tmp);
    if (!keep_new) {
      cudaFree(perm);
      cudaFree(iperm);
      cudaFree(noffs);
      cudaFree(ncol);
      cudaFree(nw);
      cudaFree(nwf);
      std::free(h_iperm);
    }
  };
  int st = GB_OK;
#define GB_TRY(call)                 \
  do {                               \
    cudaError_t _e = (call);         \
    if (_e != cudaSuccess) {         \
      st = cuda_fail(_e, #call);     \
      cleanup(false);                \
      return st;                     \
    }                                \
  } while (0)
  const size_t m1 = std::max<uint64_t>(m, 1);
  GB_TRY(cudaMalloc(&deg, sizeof(uint32_t) * n));
  GB_TRY(cudaMalloc(&deg2, sizeof(uint32_t) * (n + 1)));
  GB_TRY(cudaMalloc(&ids, sizeof(uint32_t) * n));
  GB_TRY(cudaMalloc(&perm, sizeof(uint32_t) * n));
  GB_TRY(cudaMalloc(&iperm, sizeof(uint32_t) * n));
  GB_TRY(cudaMalloc(&noffs, sizeof(uint64_t) * (n + 1)));
  GB_TRY(cudaMalloc(&ncol, sizeof(uint32_t) * m1));
  if (g->w) GB_TRY(cudaMalloc(&nw, sizeof(uint32_t) * m1));
  if (g->wf) GB_TRY(cudaMalloc(&nwf, sizeof(float) * m1));
  h_iperm = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * n));
  if (!h_iperm) {
    cleanup(false);
    GB_FAIL(GB_ERR_OOM, "gb_graph_reorder: host allocation failed");
  }

  uint32_t zero_from = n;
  GB_TRY(cudaMemsetAsync(deg2 + n, 0, sizeof(uint32_t), s));
  if (!locality) {
    // 1. degree-descending permutation
    degree_ids_kernel<<<blocks_for(g, n), 256, 0, s>>>(g->offs, n, deg, ids);
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) <= (uint64_t)g->max_degree) ++end_bit;
    GB_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, deg, deg2, ids, perm, (int64_t)n, 0, end_bit,
                                                     s));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
    GB_TRY(cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, deg, deg2, ids, perm, (int64_t)n, 0, end_bit, s));
    uint32_t* zf = reinterpret_cast<uint32_t*>(ids);  // ids is free after the sort
    GB_TRY(cudaMemcpyAsync(zf, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    first_zero_kernel<<<blocks_for(g, n), 256, 0, s>>>(deg2, n, zf);
    GB_TRY(cudaMemcpyAsync(&zero_from, zf, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  } else {
    // 1. Morton order of the distances to two far-apart landmarks
    GB_TRY(cudaMalloc(&da, sizeof(uint32_t) * n));
    GB_TRY(cudaMalloc(&db, sizeof(uint32_t) * n));
    GB_TRY(cudaMalloc(&dc, sizeof(uint32_t) * n));
    GB_TRY(cudaMalloc(&best, sizeof(unsigned long long)));
    // the farthest reached vertex from `from` (optionally: from both)
    auto farthest = [&](const uint32_t* lv, const uint32_t* lv2, uint32_t* out) -> int {
      cudaError_t e = cudaMemsetAsync(best, 0, sizeof(unsigned long long), s);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
      far_vertex_kernel<<<blocks_for(g, n), 256, 0, s>>>(lv, lv2, n, best);
      unsigned long long h = 0;
      e = cudaMemcpyAsync(&h, best, sizeof(h), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return cuda_fail(e, "landmark search");
      *out = h ? 0xFFFFFFFFu - (uint32_t)(h & 0xFFFFFFFFull) : 0u;
      return GB_OK;
    };
    uint32_t a0 = 0, la = 0, lb = 0, lc = 0;
    int lst = run_bfs(g, a0, da, nullptr, s, nullptr, 0);
    if (lst == GB_OK) lst = farthest(da, nullptr, &la);
    if (lst == GB_OK) lst = run_bfs(g, la, da, nullptr, s, nullptr, 0);
    if (lst == GB_OK) lst = farthest(da, nullptr, &lb);
    if (lst == GB_OK) lst = run_bfs(g, lb, db, nullptr, s, nullptr, 0);
    if (lst == GB_OK) lst = farthest(da, db, &lc);
    if (lst == GB_OK) lst = run_bfs(g, lc, dc, nullptr, s, nullptr, 0);
    if (lst != GB_OK) {
      cleanup(false);
      return lst;
    }
    // the largest coordinate decides how far the keys are shifted to fit 16 bits
    uint32_t ma = 0, mc = 0;
    {
      int fst = farthest(da, nullptr, &ma);
      if (fst == GB_OK) fst = farthest(dc, nullptr, &mc);
      if (fst != GB_OK) {
        cleanup(false);
        return fst;
      }
    }
    uint32_t hmax[2] = {0, 0};
    GB_TRY(cudaMemcpyAsync(&hmax[0], da + ma, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GB_TRY(cudaMemcpyAsync(&hmax[1], dc + mc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GB_TRY(cudaStreamSynchronize(s));
    uint32_t shift = 0;
    while ((std::max(hmax[0], hmax[1]) >> shift) > 0xFFFFu) ++shift;
    morton_kernel<<<blocks_for(g, n), 256, 0, s>>>(da, dc, n, shift, deg, ids);
    GB_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, deg, db, ids, perm, (int64_t)n, 0, 32, s));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
    GB_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, deg, db, ids, perm, (int64_t)n, 0, 32, s));
    gather_deg_kernel<<<blocks_for(g, n), 256, 0, s>>>(g->offs, perm, n, deg2);
  }
  invert_kernel<<<blocks_for(g, n), 256, 0, s>>>(perm, n, iperm);

  // 2. new offsets
  {
    cudaFree(tmp);
    tmp = nullptr;
    size_t sb = 0;
    auto in_it = cub::TransformInputIterator<uint64_t, cub::CastOp<uint64_t>, const uint32_t*>(
        deg2, cub::CastOp<uint64_t>());
    GB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, sb, in_it, noffs, (int64_t)n + 1, s));
    GB_TRY(cudaMalloc(&tmp, std::max<size_t>(sb, 16)));
    GB_TRY(cub::DeviceScan::ExclusiveSum(tmp, sb, in_it, noffs, (int64_t)n + 1, s));
  }

  // 3. rows copied in the new order, 4. sorted
  if (sort_rows && m) {
    GB_TRY(cudaMalloc(&ncol2, sizeof(uint32_t) * m1));
    if (weighted) {
      GB_TRY(cudaMalloc(&packed, sizeof(uint64_t) * m1));
      GB_TRY(cudaMalloc(&packed2, sizeof(uint64_t) * m1));
    }
    relabel_rows_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, g->col, g->w, g->wf, perm, iperm, noffs, n, ncol2,
                                                        nullptr, nullptr, packed);
    cudaFree(tmp);
    tmp = nullptr;
    size_t sb = 0;
    if (weighted) {
      GB_TRY(cub::DeviceSegmentedSort::SortPairs(nullptr, sb, ncol2, ncol, packed, packed2, (int)m, (int)n, noffs,
                                                 noffs + 1, s));
      GB_TRY(cudaMalloc(&tmp, std::max<size_t>(sb, 16)));
      GB_TRY(cub::DeviceSegmentedSort::SortPairs(tmp, sb, ncol2, ncol, packed, packed2, (int)m, (int)n, noffs,
                                                 noffs + 1, s));
      unpack_kernel<<<g->sm_count * 8, 256, 0, s>>>(packed2, m, nw, nwf);
    } else {
      GB_TRY(cub::DeviceSegmentedSort::SortKeys(nullptr, sb, ncol2, ncol, (int)m, (int)n, noffs, noffs + 1, s));
      GB_TRY(cudaMalloc(&tmp, std::max<size_t>(sb, 16)));
      GB_TRY(cub::DeviceSegmentedSort::SortKeys(tmp, sb, ncol2, ncol, (int)m, (int)n, noffs, noffs + 1, s));
    }
  } else if (m) {
    relabel_rows_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, g->col, g->w, g->wf, perm, iperm, noffs, n, ncol,
                                                        nw, nwf, nullptr);
  }
  GB_TRY(cudaGetLastError());
  GB_TRY(cudaMemcpyAsync(h_iperm, iperm, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  GB_TRY(cudaStreamSynchronize(s));
#undef GB_TRY

  // install
  drop_derived(g);
  pool_free(g->offs);
  pool_free(g->col);
  pool_free(g->w);
  pool_free(g->wf);
  g->offs = noffs;
  g->col = ncol;
  g->w = nw;
  g->wf = nwf;
  g->perm = perm;
  g->iperm = iperm;
  g->h_iperm = h_iperm;
  g->order = order;
  g->zero_from = zero_from;
  cleanup(true);
  return reserve_result_bufs(g);
}

}  // namespace gb

using namespace gb;

extern "C" int gb_graph_reorder(gb_graph* g, int order, void* stream) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_reorder: null graph");
  GB_CUDA(cudaSetDevice(g->device));
  return reorder_graph(g, order, static_cast<cudaStream_t>(stream));
}

extern "C" int gb_graph_order(const gb_graph* g, int* order) {
  clear_error();
  if (!g || !order) GB_FAIL(GB_ERR_ARG, "gb_graph_order: null argument");
  *order = g->perm ? g->order : GB_ORDER_NONE;
  return GB_OK;
}

extern "C" int gb_graph_permutation(const gb_graph* g, const uint32_t** new_to_old, const uint32_t** old_to_new) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_graph_permutation: null graph");
  if (new_to_old) *new_to_old = g->perm;
  if (old_to_new) *old_to_new = g->iperm;
  return GB_OK;
}
