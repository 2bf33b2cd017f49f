/*
 * gb_operator.cuh -- header-only CUDA C++ operator layer over the libgb
 * device mirror.
 *
 * Restates the shape of Galois' operator API for device code:
 *   galois::do_all(galois::iterate(graph), op, ...)     libgalois/include/galois/Loops.h:70-74
 *   galois::for_each(galois::iterate(bag), op, ...)      Loops.h:51-64
 *   graph.edge_begin/edge_end/getEdgeDst/getEdgeData     LC_CSR_Graph.h:388-460
 * so that lonestar-style operators compile as __device__ lambdas
 * (nvcc --extended-lambda) over the same device arrays the library kernels
 * use.  Semantics:
 *   gb::do_all(range, op)    op(v) once for every v in range, grid-stride,
 *                            no ordering; stream-ordered, asynchronous.
 *   gb::for_each(init, op)   bulk-synchronous worklist: round r applies op
 *                            to every item pushed in round r-1 (items pushed
 *                            in a round run in the next one), until a round
 *                            pushes nothing.  This is the schedule of Galois'
 *                            BulkSynchronous worklist (worklists/BulkSynchronous.h)
 *                            rather than its asynchronous chunked FIFO; an
 *                            operator that is correct under any schedule (as
 *                            the lonestar operators are) gives the same result.
 * Not part of the C ABI.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gb.h"

namespace gb {

// Device view of a gb_graph (begin offsets n+1, destinations, weights).
struct DeviceCSR {
  const uint64_t* offs = nullptr;
  const uint32_t* col = nullptr;
  const uint32_t* w = nullptr;
  const float* wf = nullptr;
  uint32_t n = 0;
  uint64_t m = 0;

  __host__ __device__ uint32_t size() const { return n; }
  __host__ __device__ uint64_t sizeEdges() const { return m; }
  __device__ uint64_t edge_begin(uint32_t v) const { return offs[v]; }
  __device__ uint64_t edge_end(uint32_t v) const { return offs[v + 1]; }
  __device__ uint32_t getEdgeDst(uint64_t e) const { return col[e]; }
  __device__ uint32_t getEdgeData(uint64_t e) const { return w[e]; }
  __device__ float getEdgeDataFloat(uint64_t e) const { return wf[e]; }

  // Fill from a handle made by gb_graph_upload / gb_graph_load_gr.
  static int from(const gb_graph* g, DeviceCSR* out) {
    int sym = 0;
    int st = gb_graph_info(g, &out->n, &out->m, &sym);
    if (st != GB_OK) return st;
    return gb_graph_device_arrays(g, &out->offs, &out->col, &out->w, &out->wf);
  }
};

struct VertexRange {
  uint32_t begin, end;
};
inline VertexRange iterate(const DeviceCSR& g) { return {0u, g.n}; }
inline VertexRange iterate(uint32_t begin, uint32_t end) { return {begin, end}; }

namespace detail {

template <class Op>
__global__ void do_all_kernel(VertexRange r, Op op) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = r.begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < r.end; v += stride)
    op((uint32_t)v);
}

inline int grid_for(uint64_t work) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t blocks = (work + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 8;
  return (int)(blocks < 1 ? 1 : (blocks > cap ? cap : blocks));
}

}  // namespace detail

// op(v) for every v in range.
template <class Op>
int do_all(VertexRange r, Op op, cudaStream_t s = 0) {
  if (r.end <= r.begin) return GB_OK;
  detail::do_all_kernel<<<detail::grid_for(r.end - r.begin), 256, 0, s>>>(r, op);
  return cudaGetLastError() == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

// Push context handed to for_each operators: ctx.push(v) appends v to the
// next round (warp-aggregated: one atomic per warp).
struct Context {
  uint32_t* next;
  uint32_t* count;
  uint32_t cap;
  int* overflow;
  __device__ void push(uint32_t v) const {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    const uint32_t pos = base + __popc(mask & ((1u << lane) - 1u));
    if (pos < cap) next[pos] = v;
    else atomicExch(overflow, 1);
  }
};

namespace detail {
template <class Op>
__global__ void for_each_kernel(const uint32_t* __restrict__ cur, uint32_t ncur, Op op, Context ctx) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncur; i += stride) op(cur[i], ctx);
}
}  // namespace detail

// Bulk-synchronous for_each.  `init` (device array of ninit items) seeds round
// 0; each round's pushes (at most `cap` per round) feed the next round.
// Allocates two item buffers of `cap` entries for the duration of the call.
// Returns GB_ERR_CAPACITY if a round pushed more than `cap` items and
// GB_ERR_TIMEOUT after max_rounds rounds.
template <class Op>
int for_each(const uint32_t* init, uint32_t ninit, Op op, uint32_t cap, cudaStream_t s = 0,
             uint32_t max_rounds = 1u << 30, uint32_t* rounds_out = nullptr) {
  uint32_t* buf[2] = {nullptr, nullptr};
  uint32_t* ctr = nullptr;  // [0] count, [1] overflow flag
  if (cudaMalloc(&buf[0], sizeof(uint32_t) * (cap ? cap : 1)) != cudaSuccess ||
      cudaMalloc(&buf[1], sizeof(uint32_t) * (cap ? cap : 1)) != cudaSuccess ||
      cudaMalloc(&ctr, 2 * sizeof(uint32_t)) != cudaSuccess) {
    cudaFree(buf[0]);
    cudaFree(buf[1]);
    return GB_ERR_OOM;
  }
  int st = GB_OK;
  uint32_t n = ninit < cap ? ninit : cap;
  if (n) cudaMemcpyAsync(buf[0], init, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s);
  uint32_t r = 0;
  for (; n > 0; ++r) {
    if (r >= max_rounds) {
      st = GB_ERR_TIMEOUT;
      break;
    }
    cudaMemsetAsync(ctr, 0, 2 * sizeof(uint32_t), s);
    Context ctx{buf[(r + 1) & 1], &ctr[0], cap, reinterpret_cast<int*>(&ctr[1])};
    detail::for_each_kernel<<<detail::grid_for(n), 256, 0, s>>>(buf[r & 1], n, op, ctx);
    uint32_t h[2] = {0, 0};
    if (cudaMemcpyAsync(h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      st = GB_ERR_CUDA;
      break;
    }
    if (h[1]) {
      st = GB_ERR_CAPACITY;
      break;
    }
    n = h[0];
  }
  if (rounds_out) *rounds_out = r;
  cudaFree(buf[0]);
  cudaFree(buf[1]);
  cudaFree(ctr);
  return st;
}

}  // namespace gb
