// The device mirror of an LC_CSR_Graph (libgalois/include/galois/graphs/
// LC_CSR_Graph.h:133-178) plus the per-handle scratch workspace.
//
// Layout in HBM (all arrays 256-byte aligned by cudaMalloc):
//   offs   uint64[n+1]  begin offsets (the LC end offsets with a leading 0)
//   col    uint32[m]    destinations, adjacency sorted ascending
//   w      uint32[m]    integer weights (SSSP), optional
//   wf     float[m]     float weights (PPR), optional
//   t_*    the same for the transposed graph (in-edges), built on demand,
//          with t_emap uint64[m] mapping each in-arc to its out-arc index.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "gb_internal.h"

struct gb_graph {
  int device = 0;
  uint32_t n = 0;
  uint64_t m = 0;
  int symmetric = 0;
  int sm_count = 148;
  uint64_t* offs = nullptr;
  uint32_t* col = nullptr;
  uint32_t* w = nullptr;
  float* wf = nullptr;
  // transposed (in-edge) CSR
  uint64_t* t_offs = nullptr;
  uint32_t* t_col = nullptr;
  float* t_wf = nullptr;
  uint64_t* t_emap = nullptr;
  // cached per-graph derived arrays
  uint32_t* outdeg_of_stored = nullptr;  // PageRank nout (in-degree counts of the stored graph)
  // degree-ordered graphs: the rows of the light rows' arcs [lr_arc0,
  // lr_arc1) (rows [lr_row0, zero_from)) for flat pull sweeps, packed as the
  // first row of every 256-arc run (uint32) followed by each arc's row offset
  // from its run's first row (one byte)
  uint32_t* lr_rowid = nullptr;
  uint32_t lr_row0 = 0, lr_heavy = 0;
  uint64_t lr_arc0 = 0, lr_arc1 = 0;
  float* colsum = nullptr;               // PPR column sums of wf by source
  // PageRank pull on degree-ordered graphs: the binned layout of the arcs
  // (opaque, built and freed by pagerank.cu)
  struct PrBins* prb = nullptr;
  // bounded-degree graphs: the arcs as fixed-width rows (ell_d slots per
  // vertex, columns then uint32 weights, empty slots 0xFFFFFFFF), for SSSP
  uint32_t* ell = nullptr;
  uint32_t ell_d = 0;
  // largest arc count of an SSSP region (sssp.cu) + 1 (0: not computed) and the
  // fraction of arcs inside their region, for SSSP
  uint64_t region_arcs = 0;
  double region_local = 0.0;
  uint32_t max_degree = 0;
  // all-vertex sweep schedule (sweep.cuh), cached per (heavy, tile)
  uint2* sweep_tiles = nullptr;
  uint32_t* sweep_heavy_list = nullptr;
  uint32_t sweep_ntiles = 0;
  uint32_t sweep_nheavy = 0;
  uint32_t sweep_heavy = 0;
  uint32_t sweep_tile = 0;
  // multi-graph (block-diagonal) layout, validated once and cached
  uint32_t* mg_first = nullptr;   // device copy of graph_first [ngraphs+1]
  uint32_t* mg_src = nullptr;     // device global sources [ngraphs]
  uint32_t* mg_level = nullptr;   // device outputs used for host-pointer calls
  uint32_t* mg_label = nullptr;
  uint32_t* mg_stage = nullptr;   // pinned staging of host arrays
  uint32_t mg_ngraphs = 0;
  uint64_t mg_hash = 0;
  // personalised-PageRank state (opaque, owned by ppr.cu)
  void* ppr_state = nullptr;
  void (*ppr_free)(gb_graph*) = nullptr;
  // degree-ordered relabelling (reorder.cu): when perm is set, every array
  // above uses internal ids; perm[new] = original id, iperm[original] = new
  // id (device), h_iperm the host copy for mapping sources; ro_buf holds 3n
  // words of result staging for mapping outputs back to original ids
  int order = 0;
  uint32_t zero_from = 0;  // degree-ordered: first vertex with no stored arcs (n if none)
  uint32_t* perm = nullptr;
  uint32_t* iperm = nullptr;
  uint32_t* h_iperm = nullptr;
  uint32_t* ro_buf = nullptr;
  // scratch workspace, grown on demand
  void* ws = nullptr;
  size_t ws_bytes = 0;
  // pinned host staging for small readbacks
  void* pinned = nullptr;
  gb_tuning tuning{};
};

namespace gb {

// status helpers
int cuda_fail(cudaError_t e, const char* what);
#define GB_CUDA(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return ::gb::cuda_fail(_e, #call); \
  } while (0)

bool is_device_ptr(const void* p);

// Caching allocator for the large per-graph arrays (CSR mirror, workspace)
// and the pinned readback buffer: blocks freed by gb_graph_free are kept,
// keyed by device and size rounded to 2 MiB, and handed to the next upload of
// the same shape, so a repeated upload/compute/free cycle makes no
// cudaMalloc / cudaFree (each of which can cost milliseconds and cudaFree
// synchronises the device).  pool_free accepts memory from cudaMalloc too.
// gb_pool_trim (gb.h) releases the cached blocks.
cudaError_t pool_malloc(void** p, size_t bytes);
void pool_free(void* p);
cudaError_t pool_malloc_host(void** p, size_t bytes);
void pool_free_host(void* p);
// Ensure at least `bytes` of workspace; returns GB_OK or an error status.
int ws_reserve(gb_graph* g, size_t bytes, cudaStream_t stream);
// Bump-carve helper over the workspace.
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(static_cast<char*>(b)) {}
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};
template <class T>
inline size_t carve_size(size_t count) {
  return ((count * sizeof(T)) + 255) & ~size_t(255);
}

// Resolved tuning with defaults filled in.
gb_tuning effective_tuning(const gb_graph* g);

// Number of CTAs for a cooperative launch of `kernel` with `threads` threads.
int coop_grid(const gb_graph* g, const void* kernel, int threads, size_t smem,
              uint32_t blocks_per_sm_cap);

// Map a device error word to a status (and message).
int dev_err_status(int code, const char* what);

// Copy `count` elements of device data to a caller buffer (host or device).
int copy_out(void* dst, const void* src_dev, size_t bytes, cudaStream_t stream);
// Upload caller data (host or device) into a device buffer.
int copy_in(void* dst_dev, const void* src, size_t bytes, cudaStream_t stream);

int ensure_transpose(gb_graph* g, cudaStream_t stream);
// Frees every cached array derived from the stored arcs (reorder.cu).
void drop_derived(gb_graph* g);
// Frees the PageRank binned layout (pagerank.cu).
void free_pr_bins(gb_graph* g);

// Relabelled graphs (reorder.cu).  result_buf returns the k-th n-word
// staging buffer (k < 3).  finish_* map a result computed in internal ids
// (device, in result_buf(g, 0)) to original ids in `out` (host or device);
// finish_labels also turns min-internal-id labels into min-original-id labels.
uint32_t* result_buf(gb_graph* g, int k);
int reserve_result_bufs(gb_graph* g);
int finish_u32(gb_graph* g, const uint32_t* res, uint32_t* out, cudaStream_t s);
int finish_f32(gb_graph* g, const float* res, float* out, cudaStream_t s);
int finish_labels(gb_graph* g, const uint32_t* res, uint32_t* out, cudaStream_t s);

// Times one kernel launch with CUDA events on its stream (only when `on`).
struct KernelTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  KernelTimer(bool on, cudaStream_t s) {
    if (on && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) cudaEventRecord(a, s);
  }
  void stop(cudaStream_t s) {
    if (b) cudaEventRecord(b, s);
  }
  double ms() const {
    float t = 0.f;
    if (a && b && cudaEventElapsedTime(&t, a, b) == cudaSuccess) return t;
    return 0.0;
  }
  ~KernelTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace gb
