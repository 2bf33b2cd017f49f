/*
 * gb_operator.cuh -- header-only CUDA C++ operator layer over the libgb
 * device mirror.
 *
 * Restates the shape of Galois' operator API for device code:
 *   galois::do_all(galois::iterate(graph), op, ...)     libgalois/include/galois/Loops.h:70-74
 *   galois::for_each(galois::iterate(bag), op,
 *                    galois::wl<WL>(...))                Loops.h:51-64
 *   graph.edge_begin/edge_end/getEdgeDst/getEdgeData     LC_CSR_Graph.h:388-460
 * so that lonestar-style operators compile as __device__ lambdas
 * (nvcc --extended-lambda) over the same device arrays the library kernels
 * use.
 *
 *   gb::do_all(range, op)   op(v) once for every v in range, grid-stride,
 *                           no ordering; stream-ordered, asynchronous.
 *   gb::for_each(ws, init, op, gb::wl<Policy>(...))
 *                           op(item, key, ctx) for every work item; ctx.push
 *                           (item, key) adds one.  Work items are (item, key)
 *                           pairs of uint32.  Policies:
 *       gb::FIFO            asynchronous chunked FIFO (the device form of
 *                           worklists/Chunk.h PerSocketChunkFIFO): no rounds;
 *       gb::DeltaBuckets    ordered by integer metric key >> shift (the
 *                           device form of worklists/Obim.h:147-430 with
 *                           galois::wl<OBIM>(Indexer{shift})): every item of
 *                           bucket b is processed before any item of a later
 *                           bucket, asynchronously inside a bucket.
 *   gb::for_each_edge(ws, g, init, filter, edge_op, gb::wl<Policy>(...))
 *                           the edge loop of a lonestar operator spread over
 *                           a warp: for every item with filter(item, key),
 *                           edge_op(item, key, e, ctx) for each out-arc e of
 *                           vertex `item`, degree-balanced (a warp walks the
 *                           concatenated arcs of up to 32 items, an item
 *                           above 1024 arcs is split into 1024-arc tiles
 *                           that run as separate work items).
 * Both for_each forms run as ONE persistent cooperative launch over the
 * device worklist of gb_worklist.cuh (per-warp local queues, a ring of
 * chunks, termination by a work count), allocate nothing (the caller's
 * gb::Worklist holds the device memory and is reused), make no host
 * synchronisation between rounds and return after the launch (the status
 * is read back once).  ctx.push may run in divergent code.  As in Galois, an
 * operator must be correct under any schedule: the lonestar operators skip
 * stale items themselves (e.g. SSSP.cpp:138-142).
 * Not part of the C ABI.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gb.h"
#include "gb_worklist.cuh"

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

// ---- worklist policies: gb::wl<gb::FIFO>(), gb::wl<gb::DeltaBuckets>(shift)
struct FIFO {};
struct DeltaBuckets {
  uint32_t shift;
};
template <class Policy, class... A>
Policy wl(A... a) {
  return Policy{static_cast<uint32_t>(a)...};
}

namespace detail {

template <class Op>
__global__ void do_all_kernel(VertexRange r, Op op) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = r.begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < r.end; v += stride)
    op((uint32_t)v);
}

inline int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

inline int grid_for(uint64_t work) {
  const uint64_t blocks = (work + 255) / 256;
  const uint64_t cap = (uint64_t)sm_count() * 8;
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

// Statistics of one for_each call.
struct ForEachStats {
  unsigned long long items = 0;    // work items taken (stale ones included)
  unsigned long long edges = 0;    // arcs handed to edge_op (for_each_edge)
  unsigned long long chunks = 0;   // ring chunks published
  uint32_t buckets = 0;            // DeltaBuckets: buckets processed
};

namespace detail {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kLQ = 64;        // local-queue entries per warp
constexpr int kStage = 64;     // ctx.push staging per warp
constexpr uint32_t kTile = 1024;  // arcs per tile of a large item (for_each_edge)
constexpr uint64_t kBudgetNs = 60ull * 1000000000ull;

struct Ctl {
  unsigned int bar_count, bar_gen;
  int err;
  uint32_t far_count[2];
  uint32_t min_bucket;
  uint32_t buckets;
  uint32_t pad;
  unsigned long long items, edges;
};

struct Args {
  worklists::Ring ring;
  Ctl* ctl;
  uint2* far[2];  // (item, key) piles of later buckets (DeltaBuckets)
  uint32_t far_cap;
  uint32_t shift;
};

// Bounded grid barrier for the cooperative launch: gives up (error word
// worklists::kErrTimeout) after 2 s or past the deadline; false means leave.
__device__ __forceinline__ bool grid_sync(Ctl* c, uint64_t deadline) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &c->bar_gen;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&c->bar_count, 1u) == gridDim.x - 1) {
      c->bar_count = 0;
      __threadfence();
      atomicAdd(&c->bar_gen, 1u);
    } else {
      const uint64_t t0 = worklists::timer_ns();
      while (*gen == g) {
        const uint64_t now = worklists::timer_ns();
        if (worklists::err_set(&c->err)) { ok = 0; break; }
        if (now - t0 > 2000000000ull || now > deadline) {
          worklists::err_raise(&c->err, worklists::kErrTimeout);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok && !worklists::err_set(&c->err);
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace detail

// The push context handed to operators.  push(item, key) may be called from
// divergent code; items of a later bucket go to the far pile, the others to
// this warp's staging area (drained into the worklist after the operator
// returns) or, when that is full, straight to the ring.
struct Ctx {
  uint4* stage;
  uint32_t* stage_n;
  const detail::Args* a;
  int fp;
  uint32_t hi;   // DeltaBuckets: keys at or above hi belong to a later bucket
  bool buckets;  // false: FIFO, keys only travel with their items
  __device__ void push(uint32_t item, uint32_t key = 0) const {
    if (buckets && key >= hi) {
      const uint32_t pos = atomicAdd(&a->ctl->far_count[fp], 1u);
      if (pos < a->far_cap) a->far[fp][pos] = make_uint2(item, key);
      else worklists::err_raise(&a->ctl->err, worklists::kErrOverflow);
      return;
    }
    const uint4 e = make_uint4(item, key, 0u, 0u);
    const uint32_t pos = atomicAdd(stage_n, 1u);
    if (pos < (uint32_t)detail::kStage) stage[pos] = e;
    else worklists::publish_one(a->ring, e, &a->ctl->err);
  }
};

namespace detail {

// Warp-cooperative walk over the concatenated arcs [beg, beg + deg) of the
// lanes' items (deg = 0: idle lane); fn(item, key, arc) for every arc, on the
// lane holding the arc, with the item and key of the lane that owns it.
template <class Fn>
__device__ __forceinline__ void expand(uint64_t beg, uint32_t deg, uint32_t item, uint32_t key, Fn&& fn) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t incl = deg;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if ((int)lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t e = base + lane;
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, pos + step - 1);
      if (v <= e) pos += step;
    }
    const uint64_t ob = __shfl_sync(0xFFFFFFFFu, beg, pos);
    const uint32_t oex = __shfl_sync(0xFFFFFFFFu, excl, pos);
    const uint32_t oi = __shfl_sync(0xFFFFFFFFu, item, pos);
    const uint32_t ok = __shfl_sync(0xFFFFFFFFu, key, pos);
    if (e < total) fn(oi, ok, ob + (uint64_t)(e - oex));
    __syncwarp();
  }
}

// The persistent for_each.  kBuckets: DeltaBuckets (else FIFO); kEdges: the
// edge form (op is edge_op, filter chooses the items to expand).
template <bool kBuckets, bool kEdges, class Filter, class Op>
__global__ void __launch_bounds__(kBlock, 1) for_each_kernel(Args a, DeviceCSR g, Filter filter, Op op) {
  __shared__ uint4 s_lq[kWarps][kLQ];
  __shared__ uint4 s_stage[kWarps][kStage];
  __shared__ uint32_t s_stage_n[kWarps];
  Ctl* ctl = a.ctl;
  const uint64_t deadline = worklists::timer_ns() + kBudgetNs;
  const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  const uint64_t gtid = blockIdx.x * (uint64_t)kBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kBlock;
  if (lane == 0) s_stage_n[wib] = 0;
  __syncwarp();
  unsigned long long my_items = 0, my_edges = 0;
  int fp = 0;
  uint32_t hi = 0xFFFFFFFFu;
  for (;;) {
    if constexpr (kBuckets) {
      // ---- transition: the smallest bucket left in the far pile becomes
      // the ring's work; the later ones stay
      const uint32_t nfar = min(ctl->far_count[fp], a.far_cap);
      if (nfar == 0) break;
      if (gtid == 0) {
        a.ring.rc->head = a.ring.rc->tail;  // tickets left from the last bucket are void
        ctl->min_bucket = 0xFFFFFFFFu;
        ctl->far_count[fp ^ 1] = 0;
      }
      if (!grid_sync(ctl, deadline)) return;
      uint32_t mb = 0xFFFFFFFFu;
      for (uint64_t i = gtid; i < nfar; i += gthreads) mb = min(mb, a.far[fp][i].y >> a.shift);
      mb = __reduce_min_sync(0xFFFFFFFFu, mb);
      if (lane == 0 && mb != 0xFFFFFFFFu) atomicMin(&ctl->min_bucket, mb);
      if (!grid_sync(ctl, deadline)) return;
      const uint32_t nb = ctl->min_bucket;
      const uint64_t hi64 = ((uint64_t)nb + 1) << a.shift;
      hi = hi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)hi64;
      for (uint64_t base = gtid - lane; base < nfar; base += gthreads) {
        const uint64_t i = base + lane;
        uint2 it = make_uint2(0u, 0u);
        if (i < nfar) it = a.far[fp][i];
        const bool now = i < nfar && (it.y >> a.shift) == nb;
        const bool later = i < nfar && !now;
        worklists::publish(a.ring, now, make_uint4(it.x, it.y, 0u, 0u), &ctl->err);
        const unsigned lm = __ballot_sync(0xFFFFFFFFu, later);
        if (lm) {
          uint32_t b0 = 0;
          if (lane == 0) b0 = atomicAdd(&ctl->far_count[fp ^ 1], (uint32_t)__popc(lm));
          b0 = __shfl_sync(0xFFFFFFFFu, b0, 0);
          if (later) a.far[fp ^ 1][b0 + __popc(lm & ((1u << lane) - 1u))] = it;  // fits: a subset of the pile
        }
      }
      fp ^= 1;
      if (gtid == 0) ctl->buckets += 1;
      if (!grid_sync(ctl, deadline)) return;
    }
    // ---- the work: asynchronous, no barrier ----------------------------------
    worklists::WarpQueue<kLQ> q(s_lq[wib], a.ring, &ctl->err, deadline);
    Ctx ctx{s_stage[wib], &s_stage_n[wib], &a, fp, hi, kBuckets};
    auto drain = [&]() {
      __syncwarp();
      const uint32_t ns = min(s_stage_n[wib], (uint32_t)kStage);
      for (uint32_t b0 = 0; b0 < ns; b0 += 32) {
        const bool p = b0 + lane < ns;
        q.push(p, p ? s_stage[wib][b0 + lane] : make_uint4(0u, 0u, 0u, 0u));
      }
      __syncwarp();
      if (lane == 0) s_stage_n[wib] = 0;
      __syncwarp();
    };
    for (;;) {
      uint4 ent;
      bool has;
      if (q.next(ent, has) <= 0) break;
      if (has) ++my_items;
      if constexpr (!kEdges) {
        if (has) op(ent.x, ent.y, ctx);
      } else {
        // tiles of large items (ent.z = tile + 1): the whole warp, one tile at a time
        unsigned tm = __ballot_sync(0xFFFFFFFFu, has && ent.z != 0);
        while (tm) {
          const int j = __ffs(tm) - 1;
          tm &= tm - 1u;
          const uint32_t v = __shfl_sync(0xFFFFFFFFu, ent.x, j);
          const uint32_t key = __shfl_sync(0xFFFFFFFFu, ent.y, j);
          const uint32_t t = __shfl_sync(0xFFFFFFFFu, ent.z, j) - 1;
          const uint64_t b = g.offs[v] + (uint64_t)t * kTile;
          const uint64_t e_end = min(g.offs[v + 1], b + kTile);
          for (uint64_t e = b + lane; e < e_end; e += 32) {
            op(v, key, e, ctx);
            ++my_edges;
          }
          __syncwarp();
        }
        uint64_t b = 0, deg = 0;
        if (has && ent.z == 0 && filter(ent.x, ent.y)) {
          b = g.offs[ent.x];
          deg = g.offs[ent.x + 1] - b;
        }
        const bool big = deg > kTile;
        expand(b, big ? 0u : (uint32_t)deg, ent.x, ent.y, [&](uint32_t v, uint32_t key, uint64_t e) {
          op(v, key, e, ctx);
          ++my_edges;
        });
        // large items: one work item per tile
        unsigned bm = __ballot_sync(0xFFFFFFFFu, big);
        while (bm) {
          const int j = __ffs(bm) - 1;
          bm &= bm - 1u;
          const uint32_t v = __shfl_sync(0xFFFFFFFFu, ent.x, j);
          const uint32_t key = __shfl_sync(0xFFFFFFFFu, ent.y, j);
          const uint32_t nt = (uint32_t)((__shfl_sync(0xFFFFFFFFu, deg, j) + kTile - 1) / kTile);
          for (uint32_t t0 = 0; t0 < nt; t0 += 32) q.push(t0 + lane < nt, make_uint4(v, key, t0 + lane + 1, 0u));
        }
      }
      drain();
      q.share();
    }
    if (!kBuckets) break;
    if (!grid_sync(ctl, deadline)) return;  // everyone has left the bucket
  }
  my_items += __shfl_xor_sync(0xFFFFFFFFu, my_items, 16);
  my_items += __shfl_xor_sync(0xFFFFFFFFu, my_items, 8);
  my_items += __shfl_xor_sync(0xFFFFFFFFu, my_items, 4);
  my_items += __shfl_xor_sync(0xFFFFFFFFu, my_items, 2);
  my_items += __shfl_xor_sync(0xFFFFFFFFu, my_items, 1);
  my_edges += __shfl_xor_sync(0xFFFFFFFFu, my_edges, 16);
  my_edges += __shfl_xor_sync(0xFFFFFFFFu, my_edges, 8);
  my_edges += __shfl_xor_sync(0xFFFFFFFFu, my_edges, 4);
  my_edges += __shfl_xor_sync(0xFFFFFFFFu, my_edges, 2);
  my_edges += __shfl_xor_sync(0xFFFFFFFFu, my_edges, 1);
  if (lane == 0) {
    if (my_items) atomicAdd(&ctl->items, my_items);
    if (my_edges) atomicAdd(&ctl->edges, my_edges);
  }
}

// Seed the worklist: FIFO publishes the initial items as chunks, DeltaBuckets
// files them into the far pile (the first transition picks the smallest
// bucket).
template <bool kBuckets>
__global__ void for_each_seed(Args a, const uint32_t* items, const uint32_t* keys, uint32_t ninit) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t nch = ((uint64_t)ninit + 31) / 32;
  for (uint64_t i = tid; i <= a.ring.mask; i += stride) {
    if (!kBuckets && i < nch) {
      const uint32_t first = (uint32_t)(i * 32), cnt = min(32u, ninit - first);
      for (uint32_t j = 0; j < cnt; ++j)
        a.ring.ent[i * 32 + j] = make_uint4(items[first + j], keys ? keys[first + j] : 0u, 0u, 0u);
      a.ring.cnt[i] = cnt;
      a.ring.seq[i] = i + 1;
    } else {
      a.ring.seq[i] = i;
    }
  }
  if (kBuckets)
    for (uint64_t i = tid; i < ninit; i += stride) a.far[0][i] = make_uint2(items[i], keys ? keys[i] : 0u);
  if (tid == 0) {
    if (kBuckets) {
      a.ctl->far_count[0] = ninit;
    } else {
      a.ring.rc->tail = nch;
      a.ring.rc->work = (int)nch;
    }
  }
}

struct AlwaysTrue {
  __device__ bool operator()(uint32_t, uint32_t) const { return true; }
};

}  // namespace detail

// Device memory of for_each, allocated once and reused by every call (the
// calls themselves allocate nothing).  far_cap bounds the items waiting in
// later buckets (DeltaBuckets) and the initial items; the ring holds
// ring_chunks chunks of up to 32 items.
class Worklist {
 public:
  Worklist() = default;
  Worklist(const Worklist&) = delete;
  Worklist& operator=(const Worklist&) = delete;
  ~Worklist() { cudaFree(mem_); }

  int reserve(uint32_t far_cap, unsigned long long ring_chunks = 1u << 16) {
    cudaFree(mem_);
    mem_ = nullptr;
    cap_ = worklists::ring_capacity(ring_chunks);
    far_cap_ = far_cap ? far_cap : 1;
    const size_t bytes = worklists::ring_part(sizeof(detail::Ctl)) + 2 * worklists::ring_part(sizeof(uint2) * far_cap_) +
                         worklists::ring_bytes(cap_);
    if (cudaMalloc(&mem_, bytes) != cudaSuccess) {
      mem_ = nullptr;
      return GB_ERR_OOM;
    }
    return GB_OK;
  }
  uint32_t far_capacity() const { return far_cap_; }
  unsigned long long ring_capacity() const { return cap_; }

  detail::Args args(uint32_t shift) const {
    char* p = static_cast<char*>(mem_);
    detail::Args a{};
    a.ctl = reinterpret_cast<detail::Ctl*>(p);
    p += worklists::ring_part(sizeof(detail::Ctl));
    a.far[0] = reinterpret_cast<uint2*>(p);
    p += worklists::ring_part(sizeof(uint2) * far_cap_);
    a.far[1] = reinterpret_cast<uint2*>(p);
    p += worklists::ring_part(sizeof(uint2) * far_cap_);
    a.ring = worklists::ring_layout(p, cap_);
    a.far_cap = far_cap_;
    a.shift = shift;
    return a;
  }
  bool ready() const { return mem_ != nullptr; }

 private:
  void* mem_ = nullptr;
  unsigned long long cap_ = 0;
  uint32_t far_cap_ = 0;
};

namespace detail {

template <bool kBuckets, bool kEdges, class Filter, class Op>
int launch_for_each(Worklist& w, const DeviceCSR& g, const uint32_t* items, const uint32_t* keys, uint32_t ninit,
                    Filter filter, Op op, uint32_t shift, cudaStream_t s, ForEachStats* st) {
  if (!w.ready()) return GB_ERR_ARG;
  if (ninit > w.far_capacity() || ((uint64_t)ninit + 31) / 32 > w.ring_capacity()) return GB_ERR_CAPACITY;
  Args a = w.args(shift);
  if (cudaMemsetAsync(a.ctl, 0, sizeof(Ctl), s) != cudaSuccess ||
      cudaMemsetAsync(a.ring.rc, 0, sizeof(worklists::RingCtl), s) != cudaSuccess)
    return GB_ERR_CUDA;
  for_each_seed<kBuckets><<<grid_for(a.ring.mask + 1), 256, 0, s>>>(a, items, keys, ninit);
  if (cudaGetLastError() != cudaSuccess) return GB_ERR_CUDA;
  const void* kfn = reinterpret_cast<const void*>(&for_each_kernel<kBuckets, kEdges, Filter, Op>);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kBlock, 0) != cudaSuccess || per_sm <= 0)
    return GB_ERR_CUDA;
  void* args[] = {&a, const_cast<DeviceCSR*>(&g), &filter, &op};
  if (cudaLaunchCooperativeKernel(kfn, per_sm * sm_count(), kBlock, args, 0, s) != cudaSuccess) return GB_ERR_CUDA;
  Ctl hc{};
  worklists::RingCtl hr{};
  if (cudaMemcpyAsync(&hc, a.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&hr, a.ring.rc, sizeof(hr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return GB_ERR_CUDA;
  if (st) {
    st->items = hc.items;
    st->edges = hc.edges;
    st->chunks = hr.chunks;
    st->buckets = hc.buckets;
  }
  if (hc.err == worklists::kErrTimeout) return GB_ERR_TIMEOUT;
  if (hc.err == worklists::kErrOverflow) return GB_ERR_CAPACITY;
  return hc.err ? GB_ERR_CUDA : GB_OK;
}

}  // namespace detail

// for_each over work items (item, key): items[0..ninit) with keys (or all
// keys 0 when keys is null), both device arrays; op(item, key, ctx).
template <class Op>
int for_each(Worklist& w, const uint32_t* items, const uint32_t* keys, uint32_t ninit, Op op, FIFO,
             cudaStream_t s = 0, ForEachStats* st = nullptr) {
  return detail::launch_for_each<false, false>(w, DeviceCSR{}, items, keys, ninit, detail::AlwaysTrue{}, op, 0u, s,
                                               st);
}
template <class Op>
int for_each(Worklist& w, const uint32_t* items, const uint32_t* keys, uint32_t ninit, Op op, DeltaBuckets p,
             cudaStream_t s = 0, ForEachStats* st = nullptr) {
  return detail::launch_for_each<true, false>(w, DeviceCSR{}, items, keys, ninit, detail::AlwaysTrue{}, op, p.shift,
                                              s, st);
}

// The edge form: for every item with filter(item, key), edge_op(item, key,
// e, ctx) for each out-arc e of vertex `item` of g.
template <class Filter, class EdgeOp>
int for_each_edge(Worklist& w, const DeviceCSR& g, const uint32_t* items, const uint32_t* keys, uint32_t ninit,
                  Filter filter, EdgeOp edge_op, FIFO, cudaStream_t s = 0, ForEachStats* st = nullptr) {
  return detail::launch_for_each<false, true>(w, g, items, keys, ninit, filter, edge_op, 0u, s, st);
}
template <class Filter, class EdgeOp>
int for_each_edge(Worklist& w, const DeviceCSR& g, const uint32_t* items, const uint32_t* keys, uint32_t ninit,
                  Filter filter, EdgeOp edge_op, DeltaBuckets p, cudaStream_t s = 0, ForEachStats* st = nullptr) {
  return detail::launch_for_each<true, true>(w, g, items, keys, ninit, filter, edge_op, p.shift, s, st);
}

}  // namespace gb
