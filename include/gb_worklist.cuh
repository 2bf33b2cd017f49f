/*
 * gb_worklist.cuh -- device worklist for asynchronous (barrier-free)
 * processing inside one persistent cooperative launch.
 *
 * The device counterpart of Galois' chunked worklists and of the for_each
 * executor's termination detection (libgalois/include/galois/worklists/
 * Chunk.h PerSocketChunkFIFO, runtime/Executor_ForEach.h): warps, not
 * threads, are the workers, and work items are 16-byte entries (uint4).
 *
 *   * Every warp keeps a LIFO local queue of LQ entries in shared memory and
 *     keeps relaxing what it pushed itself; the fast path touches no global
 *     counter.
 *   * Entries that do not fit, and a warp's surplus while other warps are
 *     waiting, are published to a ring of chunks (up to 32 entries each).
 *     Ring position p lives in slot p & mask; seq[slot] == p means free for
 *     the producer of p, == p + 1 published for the consumer of p, and the
 *     consumer sets it to p + cap, freeing the slot for the next lap.
 *   * A warp out of work takes the next ring position (a ticket: one atomic
 *     on `head`) and waits for its chunk.
 *   * `work` counts busy warps plus published chunks not yet taken.  A
 *     publisher is busy while it publishes and counts the chunk first, a
 *     warp that receives a chunk takes over the chunk's count, and a warp
 *     gives its own count back only when it runs out of work -- so `work`
 *     reads zero exactly when no entry exists anywhere: the loop is over.
 *     Tickets still waiting then are void; before the ring is reused the
 *     caller sets head = tail (between grid barriers).
 * Every wait is bounded: a producer waits at most 2 s for a free slot (the
 * ring is full: error kErrOverflow), a waiting warp at most until the
 * caller's deadline (error kErrTimeout); either raises the caller's error
 * word and returns, and so does every wait once the word is set.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {
namespace worklists {

// Error codes written into the caller's error word (the library kernels use
// the same values for their own device errors).
constexpr int kErrTimeout = 1;
constexpr int kErrOverflow = 2;
constexpr uint64_t kSlotWaitNs = 2000000000ull;

// Control words, each on its own 128-byte line (every waiting warp polls them).
struct alignas(128) RingCtl {
  unsigned long long head;  // positions taken by waiting warps (tickets)
  unsigned long long pad0[15];
  unsigned long long tail;  // positions published
  unsigned long long pad1[15];
  int work;  // busy warps + published chunks not yet taken
  int pad2[31];
  unsigned long long chunks;  // chunks published (statistics)
  unsigned long long pad3[15];
};

struct Ring {
  uint4* ent;               // [cap][32]
  unsigned long long* seq;  // [cap]
  uint32_t* cnt;            // [cap] entries per chunk
  unsigned long long mask;  // cap - 1, cap a power of two
  RingCtl* rc;
};

// Host helpers: device bytes of a ring of `cap` chunks (cap a power of two)
// and its layout over one allocation of that size (256-byte aligned parts).
inline size_t ring_part(size_t b) { return (b + 255) & ~size_t(255); }
inline size_t ring_bytes(unsigned long long cap) {
  return ring_part(sizeof(RingCtl)) + ring_part(cap * 32 * sizeof(uint4)) + ring_part(cap * 8) + ring_part(cap * 4);
}
inline Ring ring_layout(void* base, unsigned long long cap) {
  char* p = static_cast<char*>(base);
  Ring r;
  r.rc = reinterpret_cast<RingCtl*>(p);
  p += ring_part(sizeof(RingCtl));
  r.ent = reinterpret_cast<uint4*>(p);
  p += ring_part(cap * 32 * sizeof(uint4));
  r.seq = reinterpret_cast<unsigned long long*>(p);
  p += ring_part(cap * 8);
  r.cnt = reinterpret_cast<uint32_t*>(p);
  r.mask = cap - 1;
  return r;
}
// Smallest power-of-two capacity >= want (at least 1024 chunks).
inline unsigned long long ring_capacity(unsigned long long want) {
  unsigned long long c = 1024;
  while (c < want) c <<= 1;
  return c;
}

__device__ __forceinline__ uint64_t timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int err_set(const int* err) { return *reinterpret_cast<const volatile int*>(err); }
__device__ __forceinline__ void err_raise(int* err, int code) { atomicCAS(err, 0, code); }

// Initialise the ring (one thread per slot, grid-stride) with no chunk.  The
// caller zeroes *rc beforehand.
__device__ __forceinline__ void ring_init_slots(const Ring& r, uint64_t tid, uint64_t stride) {
  for (uint64_t i = tid; i <= r.mask; i += stride) r.seq[i] = i;
}

// Publish the entries of the lanes with `pred` as one chunk (warp-collective,
// all 32 lanes call).  Returns false if the error word is (or gets) set.
__device__ __forceinline__ bool publish(const Ring& r, bool pred, uint4 e, int* err) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, pred);
  if (!m) return true;
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long p = 0;
  int ok = 1;
  if (lane == 0) {
    atomicAdd(&r.rc->work, 1);
    p = atomicAdd(&r.rc->tail, 1ull);
    atomicAdd(&r.rc->chunks, 1ull);
    const unsigned long long* sq = r.seq + (p & r.mask);
    uint64_t t0 = 0;
    unsigned spins = 0;
    while (ld_acquire(sq) != p) {  // the previous lap's consumer has not released the slot yet
      if ((++spins & 63u) == 0) {
        const uint64_t now = timer_ns();
        if (!t0) t0 = now;
        if (err_set(err)) { ok = 0; break; }
        if (now - t0 > kSlotWaitNs) { err_raise(err, kErrOverflow); ok = 0; break; }
      }
      __nanosleep(64);
    }
  }
  p = __shfl_sync(0xFFFFFFFFu, p, 0);
  ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
  if (!ok) return false;
  const unsigned long long slot = p & r.mask;
  if (pred) r.ent[slot * 32 + __popc(m & ((1u << lane) - 1u))] = e;
  if (lane == 0) r.cnt[slot] = (uint32_t)__popc(m);
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    st_release(r.seq + slot, p + 1);
  }
  return true;
}

// Publish a single entry from one thread (no warp collective: usable in
// divergent code).  Returns false if the error word is (or gets) set.
__device__ __forceinline__ bool publish_one(const Ring& r, uint4 e, int* err) {
  atomicAdd(&r.rc->work, 1);
  const unsigned long long p = atomicAdd(&r.rc->tail, 1ull);
  atomicAdd(&r.rc->chunks, 1ull);
  const unsigned long long slot = p & r.mask;
  uint64_t t0 = 0;
  unsigned spins = 0;
  while (ld_acquire(r.seq + slot) != p) {
    if ((++spins & 63u) == 0) {
      const uint64_t now = timer_ns();
      if (!t0) t0 = now;
      if (err_set(err)) return false;
      if (now - t0 > kSlotWaitNs) {
        err_raise(err, kErrOverflow);
        return false;
      }
    }
    __nanosleep(64);
  }
  r.ent[slot * 32] = e;
  r.cnt[slot] = 1;
  st_release(r.seq + slot, p + 1);  // orders this thread's two stores before it
  return true;
}

// Lane 0 of a warp out of work: wait for the chunk of ring position p,
// polling with a back-off that doubles from 32 ns up to max_ns.
// 1: published; 0: no work left anywhere; -1: error (or deadline: raised).
__device__ __forceinline__ int wait_chunk(const Ring& r, unsigned long long p, int* err, uint64_t deadline,
                                          unsigned max_ns = 512) {
  const unsigned long long* sq = r.seq + (p & r.mask);
  unsigned spins = 0, ns = 32;
  for (;;) {
    if (ld_acquire(sq) == p + 1) return 1;
    if ((++spins & 7u) == 0) {
      if (*reinterpret_cast<const volatile int*>(&r.rc->work) == 0) return 0;
      if (err_set(err)) return -1;
      if (timer_ns() > deadline) {
        err_raise(err, kErrTimeout);
        return -1;
      }
    }
    __nanosleep(ns);
    if (ns < max_ns) ns <<= 1;
  }
}

// One warp's view of the worklist: its local queue (LQ entries of shared
// memory) and the ring.  Every member is warp-collective (all 32 lanes call,
// converged); `n` and `busy` are warp-uniform.
template <int LQ>
struct WarpQueue {
  static_assert(LQ >= 64, "a full local queue holds at least the 32 entries it spills");
  uint4* lq;
  uint32_t n;
  bool busy;
  Ring ring;
  int* err;
  uint64_t deadline;

  __device__ WarpQueue(uint4* local, const Ring& r, int* e, uint64_t dl)
      : lq(local), n(0), busy(false), ring(r), err(e), deadline(dl) {}

  // The next round: up to 32 entries, one per lane (`has`), the most recent
  // local ones first, else a chunk of the ring.  1: a round; 0: the loop is
  // over (no work anywhere); -1: error.
  __device__ int next(uint4& ent, bool& has) {
    const unsigned lane = threadIdx.x & 31u;
    ent = make_uint4(0u, 0u, 0u, 0u);
    has = false;
    if (n > 0) {
      const uint32_t take = n < 32u ? n : 32u;
      has = lane < take;
      if (has) ent = lq[n - take + lane];
      __syncwarp();
      n -= take;
      return 1;
    }
    if (busy && lane == 0) atomicSub(&ring.rc->work, 1);
    busy = false;
    unsigned long long p = 0;
    int got = 0;
    if (lane == 0) {
      p = atomicAdd(&ring.rc->head, 1ull);
      got = wait_chunk(ring, p, err, deadline);
    }
    got = __shfl_sync(0xFFFFFFFFu, got, 0);
    if (got <= 0) return got;
    p = __shfl_sync(0xFFFFFFFFu, p, 0);
    __syncwarp();  // lane 0's acquire orders the other lanes' reads below
    busy = true;   // the chunk's count is now this warp's
    const unsigned long long slot = p & ring.mask;
    const uint32_t c = __ldcg(ring.cnt + slot);
    has = lane < c;
    if (has) ent = __ldcg(ring.ent + slot * 32 + lane);
    __syncwarp();
    if (lane == 0) st_release(ring.seq + slot, p + ring.mask + 1);  // free for the next lap
    return 1;
  }

  // Append the entries of the lanes with `pred` to the local queue.  When
  // they do not fit, the 32 oldest local entries first leave as one full
  // chunk of the ring (so overflow never publishes a part-filled chunk, and
  // the ring holds at most one chunk per 32 entries in flight).
  __device__ void push(bool pred, uint4 e) {
    const unsigned m = __ballot_sync(0xFFFFFFFFu, pred);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t k = __popc(m);
    if (n + k > (uint32_t)LQ) spill_oldest();
    if (pred) lq[n + __popc(m & ((1u << lane) - 1u))] = e;
    n += k;
    __syncwarp();
  }

  // Publish the 32 oldest local entries as one chunk (n >= 32).
  __device__ void spill_oldest() {
    const unsigned lane = threadIdx.x & 31u;
    const uint4 e = lq[lane];
    __syncwarp();
    for (uint32_t i = 32 + lane; i < n; i += 32) lq[i - 32] = lq[i];
    __syncwarp();
    n -= 32;
    publish(ring, true, e, err);
  }

  // While other warps wait for work (tickets beyond the published tail),
  // hand them this warp's 32 oldest local entries.
  __device__ void share() {
    if (n <= 32) return;
    int want = 0;
    if ((threadIdx.x & 31u) == 0)
      want = *reinterpret_cast<const volatile unsigned long long*>(&ring.rc->head) >
             *reinterpret_cast<const volatile unsigned long long*>(&ring.rc->tail);
    if (__shfl_sync(0xFFFFFFFFu, want, 0)) spill_oldest();
  }
};

}  // namespace worklists
}  // namespace gb
