// Device building blocks shared by the frontier kernels.
//
//  * GridBar / grid_barrier: software grid barrier for persistent cooperative
//    launches.  It replaces libgpu's GlobalBarrier (libgpu/include/gbar.cuh:
//    42-121), which spins forever when a CTA is missing; this one gives up
//    after a wall-clock limit, raises a device error word and returns false,
//    so the host sees GB_ERR_TIMEOUT and the context stays usable.
//  * warp_push_*: warp-aggregated queue appends (one atomic per warp, ballot
//    + popc ranks), the device form of InsertBag::push / libgpu's
//    setup_push_warp_one (libgpu/include/worklist.h:330-349).
//  * warp_expand: warp-cooperative, degree-balanced expansion of up to 32
//    vertices' adjacency lists: lanes walk the concatenated edge list, each
//    edge's owner found by a 5-step shuffle search over the degree prefix sum.
//    Together with edge tiles for high-degree vertices this replaces the IrGL
//    TB/warp/fine-grained schedulers (lonestar/analytics/gpu/bfs/bfs.cu:155-267)
//    and Galois' EDGE_TILE_SIZE splitting (BFS_SSSP.h:81-131).
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

constexpr uint32_t kInf = 2147483646u;  // BFS_SSSP.h:31-32
constexpr unsigned kFull = 0xFFFFFFFFu;

enum DevErr : int {
  kDevOk = 0,
  kDevTimeout = 1,     // a bounded wait gave up
  kDevOverflow = 2,    // a fixed-capacity queue would overflow
  kDevMaxRounds = 3,   // an iteration cap was hit
};

struct GridBar {
  unsigned int count;
  unsigned int gen;
};

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ int read_err(const int* err) {
  return *reinterpret_cast<const volatile int*>(err);
}

__device__ __forceinline__ void raise_err(int* err, int code) { atomicCAS(err, 0, code); }

// Whole-kernel wall-clock budget for persistent kernels: every barrier checks
// it, so even a kernel whose loop never terminates leaves within one phase of
// the deadline with kDevTimeout raised.
constexpr uint64_t kKernelBudgetNs = 60ull * 1000000000ull;

__device__ __forceinline__ uint64_t kernel_deadline() { return globaltimer_ns() + kKernelBudgetNs; }

// Grid-wide barrier for a cooperative launch of `nblocks` CTAs.  Returns false
// (for every thread of the CTA) if the error word is set, the wait exceeded
// `timeout_ns`, or the kernel passed `deadline`; callers then leave the kernel.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned nblocks, int* err,
                                             uint64_t deadline = ~0ull,
                                             uint64_t timeout_ns = 2000000000ull) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0 && globaltimer_ns() > deadline) raise_err(err, kDevTimeout);
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(bar->gen);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(bar->count);
    const unsigned g = gen.load(cuda::memory_order_relaxed);
    __threadfence();
    const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
    int ok = 1;
    if (arrived == nblocks - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.fetch_add(1u, cuda::memory_order_release);
    } else {
      const uint64_t t0 = globaltimer_ns();
      unsigned spins = 0;
      while (gen.load(cuda::memory_order_acquire) == g) {
        if ((++spins & 31u) == 0) {
          if (read_err(err)) { ok = 0; break; }
          if (globaltimer_ns() - t0 > timeout_ns) {
            raise_err(err, kDevTimeout);
            ok = 0;
            break;
          }
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    if (ok && read_err(err)) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// grid_barrier whose last arriving CTA (its thread 0) runs last() before it
// releases the others: a step that must see every CTA arrived and be seen by
// every CTA after the barrier, without a second barrier.
template <class F>
__device__ __forceinline__ bool grid_barrier_last(GridBar* bar, unsigned nblocks, int* err, uint64_t deadline, F&& last,
                                                  uint64_t timeout_ns = 2000000000ull) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0 && globaltimer_ns() > deadline) raise_err(err, kDevTimeout);
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(bar->gen);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(bar->count);
    const unsigned g = gen.load(cuda::memory_order_relaxed);
    __threadfence();
    const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
    int ok = 1;
    if (arrived == nblocks - 1) {
      last();
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.fetch_add(1u, cuda::memory_order_release);
    } else {
      const uint64_t t0 = globaltimer_ns();
      unsigned spins = 0;
      while (gen.load(cuda::memory_order_acquire) == g) {
        if ((++spins & 31u) == 0) {
          if (read_err(err)) { ok = 0; break; }
          if (globaltimer_ns() - t0 > timeout_ns) {
            raise_err(err, kDevTimeout);
            ok = 0;
            break;
          }
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    if (ok && read_err(err)) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Append `item` for every lane with pred set; all 32 lanes must call.
__device__ __forceinline__ void warp_push(bool pred, uint32_t item, uint32_t* queue,
                                          uint32_t* count, uint32_t cap, int* err) {
  const unsigned mask = __ballot_sync(kFull, pred);
  if (!mask) return;
  const unsigned lane = lane_id();
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
  base = __shfl_sync(kFull, base, leader);
  if (pred) {
    const uint32_t pos = base + __popc(mask & ((1u << lane) - 1u));
    if (pos < cap) queue[pos] = item;
    else raise_err(err, kDevOverflow);
  }
}

// Reserve `k` consecutive slots per lane (k may be 0); returns this lane's
// first slot.  All 32 lanes must call.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t k, uint32_t* count) {
  uint32_t incl = k;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if ((int)lane_id() >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  uint32_t base = 0;
  if (total) {
    if (lane_id() == 31) base = atomicAdd(count, total);
    base = __shfl_sync(kFull, base, 31);
  }
  return base + incl - k;
}

// Warp-collective: every lane with nt > 0 appends tiles (v, 0) .. (v, nt-1)
// to `tiles`, reserved with one atomic per warp.  The whole warp writes each
// lane's run in turn (32 coalesced stores per step), so a lane holding a
// vertex of very high degree does not write its run alone.
__device__ __forceinline__ void warp_push_tiles(uint32_t v, uint32_t nt, uint2* tiles, uint32_t* count,
                                                uint32_t cap, int* err) {
  unsigned m = __ballot_sync(kFull, nt != 0);
  if (!m) return;
  const uint32_t first = warp_reserve(nt, count);
  const uint32_t lane = lane_id();
  for (; m; m &= m - 1) {
    const int src = __ffs(m) - 1;
    const uint32_t f = __shfl_sync(kFull, first, src);
    const uint32_t cnt = __shfl_sync(kFull, nt, src);
    const uint32_t vv = __shfl_sync(kFull, v, src);
    for (uint32_t k = lane; k < cnt; k += 32) {
      if (f + k < cap) tiles[f + k] = make_uint2(vv, k);
      else raise_err(err, kDevOverflow);
    }
  }
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Warp-cooperative expansion.  Each lane supplies the edge range of one
// vertex (beg, deg; deg = 0 for an idle lane) and a 32-bit payload.  The warp
// walks the concatenated edge list 32 edges at a time; fn(valid, edge,
// owner_lane, owner_payload) is called by ALL lanes every step (valid says
// whether the lane holds an edge), so fn may use warp collectives.
template <class Fn>
__device__ __forceinline__ void warp_expand(uint64_t beg, uint32_t deg, uint32_t payload, Fn&& fn) {
  const unsigned lane = lane_id();
  uint32_t incl = deg;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if ((int)lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t e = base + lane;
    // owner = number of lanes whose inclusive prefix is <= e
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(kFull, incl, pos + step - 1);
      if (v <= e) pos += step;
    }
    const uint64_t ob = __shfl_sync(kFull, beg, pos);
    const uint32_t oex = __shfl_sync(kFull, excl, pos);
    const uint32_t opl = __shfl_sync(kFull, payload, pos);
    const bool valid = e < total;
    fn(valid, ob + (uint64_t)(e - oex), pos, opl);
  }
}

// warp_expand with U steps in flight: for U consecutive 32-arc steps the
// owners are resolved first, then every step's first load (load1: e.g. the
// column id) is issued, then every step's dependent load (load2: e.g. the
// gathered value), and only then consume() runs per step in order.  Each lane
// keeps U independent memory chains in flight instead of one.
//   load1(valid, edge, owner_payload) -> uint32_t
//   load2(valid, edge, v1, owner_payload) -> T
//   consume(valid, owner_lane, owner_payload, v1, v2)   (all lanes call)
template <int U, class T, class Load1, class Load2, class Consume>
__device__ __forceinline__ void warp_expand_mlp(uint64_t beg, uint32_t deg, uint32_t payload, Load1&& load1,
                                                Load2&& load2, Consume&& consume) {
  const unsigned lane = lane_id();
  uint32_t incl = deg;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if ((int)lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - deg;
  for (uint32_t base = 0; base < total; base += 32 * U) {
    uint32_t pos[U], opl[U], v1[U];
    uint64_t edge[U];
    bool valid[U];
    T v2[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const uint32_t e = base + 32 * k + lane;
      uint32_t p = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t v = __shfl_sync(kFull, incl, p + step - 1);
        if (v <= e) p += step;
      }
      pos[k] = p;
      const uint64_t ob = __shfl_sync(kFull, beg, p);
      const uint32_t oex = __shfl_sync(kFull, excl, p);
      opl[k] = __shfl_sync(kFull, payload, p);
      valid[k] = e < total;
      edge[k] = ob + (uint64_t)(e - oex);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) v1[k] = load1(valid[k], edge[k], opl[k]);
#pragma unroll
    for (int k = 0; k < U; ++k) v2[k] = load2(valid[k], edge[k], v1[k], opl[k]);
#pragma unroll
    for (int k = 0; k < U; ++k) consume(valid[k], pos[k], opl[k], v1[k], v2[k]);
  }
}

// Read-only cached loads for graph arrays that no kernel writes.
template <class T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

}  // namespace gb
