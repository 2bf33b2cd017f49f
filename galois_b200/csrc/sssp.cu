// Delta-stepping single-source shortest paths over uint32 arc weights.
//
// Reference semantics: lonestar/analytics/cpu/sssp/SSSP.cpp:118-173
// (deltaStepAlgo: OBIM buckets indexed by dist >> stepShift, relax with
// atomicMin(dist[dst], dist[src]+w), push on improvement), default shift 13
// (SSSP.cpp:53-56).  Shortest distances are unique, so the output is
// bit-identical to the CPU app for any schedule.
//
// B200 design: one cooperative persistent launch.  OBIM becomes
//   * a near queue (light vertices + heavy-vertex edge tiles, frontier.cuh)
//     holding vertices whose tentative distance lies in the current bucket;
//     a per-vertex stamp keeps a vertex in at most one queue per phase;
//   * per-warp local queues in shared memory: a warp keeps relaxing light
//     vertices it improved itself for up to `local_depth` rounds inside the
//     same phase (label-correcting inside the bucket), so high-diameter
//     graphs need far fewer grid-wide phases; leftovers go to the near queue.
//     Local entries are (vertex, distance, begin offset, degree), their
//     relaxations skipped when popped stale (as the reference's operator
//     drops a request whose distance is no longer current,
//     SSSP.cpp:136-142), so they need no stamp and no fence, and a local hop
//     costs two dependent memory round trips (arcs, then the atomic with the
//     target's offsets);
//   * a far pile holding vertices relaxed beyond the bucket (membership
//     bitmap, so each vertex is in the pile at most once);
//   * for large frontiers, a bitmap instead of the near queue: a phase whose
//     input frontier is estimated above `bm_min` arcs relaxes with reductions
//     that return nothing (red.min on the distance, red.or on the next
//     phase's bitmap), so a warp step never waits on an atomic's reply, and
//     the next phase sweeps the bitmap in id order (light rows 1024 ids per
//     warp step, heavy rows from the graph's cached tile schedule).  Three
//     bitmaps rotate: phase P reads P%3, sets (P+1)%3 and clears (P+2)%3, so
//     no word is cleared by plain stores in the phase right after atomics
//     updated it.  Queue entries and bitmap bits are two encodings of the
//     same set (vertices whose distance dropped inside the bucket); the
//     distance is read when the vertex is expanded, so either encoding gives
//     the same fixed point.
// Work is spread over warps statically (no work-grabbing atomics).  When the
// near queue drains, the far pile is split: settled entries are dropped, the
// minimum remaining bucket becomes current (empty buckets are skipped), its
// vertices move to the near queue and the rest are compacted.  Phases are
// separated by the bounded grid barrier.

//
// sssp_async (tuning sssp_async > 0) is an alternative schedule for
// bounded-degree graphs (every vertex light, local queues on): no grid
// barrier between the phases of a bucket; each warp keeps relaxing its own
// local queue and shares surplus through the device worklist
// (gb_worklist.cuh); a bucket ends when the worklist's work count reaches
// zero, and only the bucket transitions keep grid barriers -- the schedule
// of the reference's barrier-free OBIM inside a bucket.  On the 4096^2 grid
// it measured 43.8 ms against 40.6 ms for the phase-synchronous kernel
// (more arcs re-relaxed, 9.7x against 6.7x the reached arcs), so the
// phase-synchronous kernel stays the default.  sssp_async_ell (tuning
// sssp_async = 2, degree <= 8) carries each queued vertex's fixed-width row:
// one memory round trip per hop, 0.69 against 1.45 us per hop on a path, but
// a round covers 32 / D vertices instead of 32 and it re-relaxes more
// (13.7x), so on the grid's wide wavefront it is slower (115 ms); the
// autotuner may pick it for narrow, chain-like graphs.

#include "device_common.cuh"
#include "device_graph.cuh"
#include "frontier.cuh"
#include "gb_worklist.cuh"
#include "sweep.cuh"

namespace gb {

namespace {

constexpr int kLocalQ = 64;  // local-queue entries per warp
constexpr int kStage = 64;   // near-queue appends staged per warp before publishing
constexpr uint32_t kNotQueued = 0xFFFFFFFFu;

// Reductions whose result is not needed: the SM issues them and moves on.
__device__ __forceinline__ void red_min_u32(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_or_u32(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct SsspCtl {
  GridBar bar;
  int err;
  uint32_t pad0;
  FrontierCounters fc[3];
  uint32_t far_count[2];
  uint32_t min_bucket;
  uint32_t buckets;
  uint32_t phases;
  uint32_t pad1;
  unsigned long long scanned;
  unsigned long long relax;
  unsigned long long local_rounds;  // region kernel: shared-memory rounds over all visits
  uint32_t far_min[2];              // region kernel: least bucket recorded for each far pile
  uint32_t pad2[2];
};

struct SsspArgs {
  const uint64_t* __restrict__ offs;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ w;
  uint32_t n;
  uint32_t src;
  uint32_t shift;
  uint32_t* dist;
  uint32_t* stamp;  // phase whose queue holds the vertex, kNotQueued if none
  uint32_t* infar;  // bitmap: vertex currently in the far pile
  uint32_t* far[2];
  FrontierQueues fq;
  SsspCtl* ctl;
  uint32_t heavy;
  uint32_t tile;
  uint32_t max_phases;
  int local_depth;
  int all_light;  // max degree <= heavy: skip the degree lookup when queueing
  uint32_t* act[3];      // frontier bitmaps (phase P reads act[P % 3])
  const uint2* sw_tiles;  // cached (vertex, k) tiles of every heavy vertex
  uint32_t sw_ntiles;
  uint32_t bm_min;  // frontier estimate above which the next frontier is a bitmap
  worklists::Ring ring;  // sssp_async only
};

__global__ void sssp_init(SsspArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t words = (a.n + 31) >> 5;
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.dist[v] = (v == a.src) ? 0u : kInf;
    a.stamp[v] = (v == a.src) ? 0u : kNotQueued;
  }
  for (uint64_t w = tid; w < words; w += stride) {
    a.infar[w] = 0;
    a.act[0][w] = 0;
    a.act[1][w] = 0;
    a.act[2][w] = 0;
  }
  if (tid == 0) {
    const uint64_t d = a.offs[a.src + 1] - a.offs[a.src];
    FrontierCounters& c = a.ctl->fc[0];
    c.vertices = 1;
    c.degree_sum = d;
    if (d > 0) seed_vertex(a.fq, 0, c, a.src, d, a.heavy, a.tile);
  }
}

// kBitmap: large frontiers may switch to the bitmap encoding (power-law
// graphs); off, the kernel is the queue-only form that low-degree,
// high-diameter graphs (small frontiers, local queues) run.
template <int BLOCK, bool kBitmap>
__global__ void __launch_bounds__(BLOCK) sssp_persistent(SsspArgs a) {
  __shared__ uint4 s_lq[BLOCK / 32][kLocalQ];
  __shared__ uint32_t s_stage[BLOCK / 32][kStage];
  SsspCtl* ctl = a.ctl;
  const unsigned nblocks = gridDim.x;
  const uint64_t deadline = kernel_deadline();
  const uint32_t lane = lane_id();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  __shared__ uint32_t s_push;
  uint4* lq = s_lq[threadIdx.x >> 5];
  unsigned long long my_scanned = 0, my_relax = 0;
  const uint32_t words = (a.n + 31) >> 5;
  if (threadIdx.x == 0) s_push = 0;

  uint32_t bucket = 0;  // current bucket index; near items have dist < hi
  int fp = 0;           // far pile being appended to
  uint32_t P = 0;       // phase counter (counter set P%3, queue buffer P&1)
  bool bm_in = false;   // this phase's frontier is the bitmap act[P % 3]
  uint32_t dirty = 0;   // bit i: act[i] may hold set bits

  for (;;) {
    if (P >= a.max_phases) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    const int rd = P % 3, wr = (P + 1) % 3, cl = (P + 2) % 3;
    FrontierCounters& cur = ctl->fc[rd];
    FrontierCounters& nxt = ctl->fc[wr];
    const uint32_t q_light = min(cur.light, a.fq.light_cap), q_tiles = min(cur.tiles, a.fq.tile_cap);
    if (gtid == 0) {
      ctl->fc[cl] = FrontierCounters{};
      ctl->far_count[fp ^ 1] = 0;  // previous pile is dead once split
    }
    const uint32_t next_stamp = P + 1;
    const uint64_t hi64 = ((uint64_t)bucket + 1) << a.shift;
    const uint32_t hi = hi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)hi64;
    uint32_t* farq = a.far[fp];
    const int qnext = (P + 1) & 1;
    // the bitmap that phase P+1 sets was read in phase P-1 and last set in
    // phase P-2: cleared now, with no atomics on it in flight
    {
      const int clr = (int)((P + 2) % 3);
      if (dirty & (1u << clr)) {
        uint32_t* c = a.act[clr];
        for (uint64_t i = gtid; i < words; i += gthreads) c[i] = 0;
        dirty &= ~(1u << clr);
      }
    }
    // bitmap input: the count of bit-setting reductions of the last phase
    // (an upper bound on the vertices set; zero means an empty frontier)
    const uint32_t bm_count = bm_in ? cur.vertices : 0u;

    if (kBitmap && bm_in ? bm_count != 0 : (q_light != 0 || q_tiles != 0)) {
      // ---- relaxation phase --------------------------------------------
      // every thread reads the same counters, so the choice is grid-uniform
      // estimated arcs of the input frontier (a light vertex counted as 16
      // arcs, a tile as its width): the arcs bound the vertices it can reach
      const uint64_t est = bm_in ? 16ull * bm_count : 16ull * q_light + (uint64_t)a.tile * q_tiles;
      const bool bm_out = kBitmap && est > a.bm_min;
      uint32_t* const act_next = a.act[(P + 1) % 3];
      uint32_t my_push = 0;  // lane 0: this warp's bit-setting reductions
      uint32_t lq_n = 0;  // warp-uniform local queue length
      WarpStage<kStage> stage{s_stage[threadIdx.x >> 5], 0u};
      uint32_t* const nq = a.fq.light[qnext];
      // Route a vertex u this lane just lowered to nd (near: inside the
      // bucket, far: beyond it; ub/deg: u's begin offset and out-degree, or
      // 0/1 when they were not needed).  A light near u goes to this warp's
      // local queue as (u, nd, begin, degree) while there is room, so the
      // local pop needs no offset loads.  Local entries carry no stamp: when
      // one is popped and dist[u] has moved below nd its relaxations are
      // skipped, because whoever moved it routed u again.  Other near
      // vertices enter the next phase's queue once (the stamp; that entry
      // reads dist when popped, so it also covers later improvements), far
      // ones the far pile once (the bitmap).  All lanes call.
      auto route = [&](bool near, bool far, uint32_t u, uint32_t nd, uint64_t ub, uint64_t deg) {
        if (!__any_sync(kFull, near || far)) return;  // most steps lower nothing
        bool loc = a.local_depth > 0 && near && deg > 0 && deg <= a.heavy && deg < 65536 && ub < (1ull << 48);
        const unsigned lm = __ballot_sync(kFull, loc);
        const uint32_t k = __popc(lm);
        if (k) {
          if (lq_n + k <= (uint32_t)kLocalQ) {
            if (loc)
              lq[lq_n + __popc(lm & lanemask_lt)] =
                  make_uint4(u, nd, (uint32_t)ub, (uint32_t)((ub >> 32) << 16) | (uint32_t)deg);
            lq_n += k;
            __syncwarp();
          } else {
            loc = false;
          }
        }
        bool to_near = false;
        if (near && !loc && a.stamp[u] != next_stamp) to_near = atomicExch(&a.stamp[u], next_stamp) != next_stamp;
        stage.push(to_near && deg > 0 && deg <= a.heavy, u, nq, &nxt.light, a.fq.light_cap, &ctl->err);
        push_with_degree<false>(a.fq, qnext, nxt, to_near && deg > a.heavy, u, deg, a.heavy, a.tile, &ctl->err);
        warp_push(far, u, farq, &ctl->far_count[fp], a.n, &ctl->err);
      };
      const bool need_deg = !a.all_light || a.local_depth > 0;
      // du: dist[u] as loaded with the arc, or ~0 to skip the pre-check (a
      // stale value only costs an extra atomic; the atomicMin decides)
      auto relax = [&](bool valid, uint32_t u, uint32_t nd, uint32_t du) {
        bool near = false, far = false;
        if (bm_out) {
          // no reply awaited: the bit marks u for the next phase, which reads
          // dist[u] when it expands u (a bit set by a candidate that lost to
          // a smaller one only costs that re-expansion)
          if (valid && nd < du) {
            red_min_u32(&a.dist[u], nd);
            const uint32_t bit = 1u << (u & 31);
            if (nd < hi) {
              red_or_u32(&act_next[u >> 5], bit);
              near = true;
            } else if (!(a.infar[u >> 5] & bit)) {
              far = !(atomicOr(&a.infar[u >> 5], bit) & bit);
            }
          }
          const unsigned nm = __ballot_sync(kFull, near);
          const unsigned rm = __ballot_sync(kFull, near || far);
          if (lane == 0) {
            my_push += __popc(nm);
            my_relax += __popc(rm);
          }
          if (__any_sync(kFull, far)) warp_push(far, u, farq, &ctl->far_count[fp], a.n, &ctl->err);
          return;
        }
        uint64_t ub = 0, deg = 1;
        if (valid && nd < du) {
          // the offset loads do not depend on the atomic: issued together
          if (need_deg) {
            ub = ldg(a.offs + u);
            deg = ldg(a.offs + u + 1) - ub;
          }
          const uint32_t old = atomicMin(&a.dist[u], nd);
          if (nd < old) {
            ++my_relax;
            if (nd < hi) {
              near = true;
            } else {
              const uint32_t bit = 1u << (u & 31);
              if (!(a.infar[u >> 5] & bit)) far = !(atomicOr(&a.infar[u >> 5], bit) & bit);
            }
          }
        }
        route(near, far, u, nd, ub, deg);
      };
      // Expand one light vertex per lane: arcs [b, b+d) from distance dv
      // (d == 0: idle lane).  cur: the vertex's current distance, compared
      // only when an arc is relaxed, so its load stays off the critical
      // path; precheck: compare each target's distance before the atomic.
      auto expand = [&](uint64_t b, uint32_t d, uint32_t dv, uint32_t cur, bool precheck) {
        my_scanned += d;
        // four 32-arc steps in flight per lane: ids, then weights (and the
        // targets' distances), then the relaxations
        warp_expand_mlp<4, uint2>(
            b, d, dv, [&](bool valid, uint64_t e, uint32_t) { return valid ? ldg(a.col + e) : 0u; },
            [&](bool valid, uint64_t e, uint32_t u, uint32_t dsrc) {
              // the pre-check may read a stale (cached, never smaller) value
              return valid ? make_uint2(dsrc + ldg(a.w + e), precheck ? a.dist[u] : 0xFFFFFFFFu)
                           : make_uint2(0u, 0u);
            },
            [&](bool valid, uint32_t owner, uint32_t dsrc, uint32_t u, uint2 v2) {
              const bool live = __shfl_sync(kFull, cur, owner) >= dsrc;
              relax(valid && live, u, v2.x, v2.y);
            });
      };
      const uint32_t* qin = a.fq.light[P & 1];
      const uint2* tin = a.fq.tiles[P & 1];
      // one heavy tile: arcs [k*tile, (k+1)*tile) of v, by the whole warp
      auto tile_body = [&](uint32_t v, uint32_t k) {
        const uint64_t vb = ldg(a.offs + v), ve = ldg(a.offs + v + 1);
        const uint64_t b = vb + (uint64_t)k * a.tile;
        const uint64_t e_end = min(ve, b + a.tile);
        const uint32_t dsrc = __ldcg(a.dist + v);
        if (lane == 0) my_scanned += e_end - b;
        constexpr int U = 4;
        for (uint64_t e0 = b; e0 < e_end; e0 += 32 * U) {
          uint32_t u[U], nd[U], du[U];
          bool valid[U];
#pragma unroll
          for (int k = 0; k < U; ++k) {
            const uint64_t e = e0 + 32 * k + lane;
            valid[k] = e < e_end;
            u[k] = valid[k] ? ldg(a.col + e) : 0u;
          }
#pragma unroll
          for (int k = 0; k < U; ++k) {
            const uint64_t e = e0 + 32 * k + lane;
            nd[k] = valid[k] ? dsrc + ldg(a.w + e) : 0u;
            du[k] = valid[k] ? a.dist[u[k]] : 0u;
          }
#pragma unroll
          for (int k = 0; k < U; ++k) relax(valid[k], u[k], nd[k], du[k]);
        }
      };
      if (kBitmap && bm_in) {
        // bitmap frontier: a warp owns words gwarp, gwarp + nwarps, ... (32
        // ids each; strided so that the dense low ids of a degree-ordered
        // graph spread over all warps), loads 32 of them per step and expands
        // the non-zero ones one at a time, one vertex per lane
        const uint32_t* act = a.act[P % 3];
        for (uint64_t base = gwarp; base < words; base += nwarps << 5) {
          const uint64_t wi = base + (uint64_t)lane * nwarps;
          const uint32_t word = wi < words ? __ldcg(act + wi) : 0u;
          unsigned nz = __ballot_sync(kFull, word != 0u);
          while (nz) {
            const int j = __ffs(nz) - 1;
            nz &= nz - 1u;
            const uint32_t bits = __shfl_sync(kFull, word, j);
            const uint32_t v = (uint32_t)((base + (uint64_t)j * nwarps) << 5) + lane;  // < n when its bit is set
            uint64_t b = 0;
            uint32_t d = 0, dv = 0;
            if ((bits >> lane) & 1u) {
              b = ldg(a.offs + v);
              const uint64_t dd = ldg(a.offs + v + 1) - b;
              if (dd <= a.heavy) {
                d = (uint32_t)dd;
                dv = __ldcg(a.dist + v);
              }
            }
            expand(b, d, dv, dv, true);
          }
        }
        // heavy vertices: the cached tile schedule, strided the same way
        for (uint64_t t0 = gwarp; t0 < a.sw_ntiles; t0 += nwarps << 5) {
          const uint64_t ti = t0 + (uint64_t)lane * nwarps;
          uint2 tv = make_uint2(0u, 0u);
          bool on = false;
          if (ti < a.sw_ntiles) {
            tv = a.sw_tiles[ti];
            on = (__ldcg(act + (tv.x >> 5)) >> (tv.x & 31)) & 1u;
          }
          unsigned m = __ballot_sync(kFull, on);
          while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1u;
            tile_body(__shfl_sync(kFull, tv.x, j), __shfl_sync(kFull, tv.y, j));
          }
        }
      } else {
        // A large queue is swept densely: every vertex in id order, active
        // when its stamp names this phase (it was queued for it and not
        // queued again since; a vertex re-queued for the next phase is
        // expanded there with its newer distance).  Consecutive rows keep the
        // column and weight reads contiguous, which the queue's order does not.
        const bool dense = q_light > (a.n >> 4);
        const uint32_t nl = dense ? a.n : q_light;
        for_each_frontier_task(
            nl, q_tiles, gwarp, nwarps,
            [&](uint32_t base, uint32_t vpt) {
              const uint32_t idx = base + lane;
              const bool has = lane < vpt && idx < nl;
              uint64_t b = 0;
              uint32_t d = 0, dv = 0;
              if (has) {
                const uint32_t v = dense ? idx : qin[idx];
                b = ldg(a.offs + v);
                d = (uint32_t)(ldg(a.offs + v + 1) - b);
                dv = __ldcg(a.dist + v);
                if (dense && (a.stamp[v] != P || d > a.heavy)) d = 0;  // not this phase's light vertex
              }
              expand(b, d, dv, dv, true);
            },
            [&](uint32_t t) {
              const uint2 tv = tin[t];
              tile_body(tv.x, tv.y);
            });
      }
      // local rounds: keep relaxing what this warp lowered (LIFO), with no
      // distance pre-check (low-degree targets: the atomic is cheaper than
      // another dependent load)
      for (int r = 0; r < a.local_depth && lq_n > 0; ++r) {
        const uint32_t take = min(32u, lq_n);
        const bool has = lane < take;
        const uint4 ent = has ? lq[lq_n - take + lane] : make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        lq_n -= take;
        const uint64_t b = ((uint64_t)(ent.w >> 16) << 32) | ent.z;
        const uint32_t cur = has ? __ldcg(a.dist + ent.x) : 0u;
        expand(b, ent.w & 0xFFFFu, ent.y, cur, false);
      }
      // leftovers that are still current join the next phase's near queue
      while (lq_n > 0) {
        const uint32_t take = min(32u, lq_n);
        const bool has = lane < take;
        const uint4 ent = has ? lq[lq_n - take + lane] : make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        lq_n -= take;
        bool to_near = false;
        if (has && __ldcg(a.dist + ent.x) >= ent.y && a.stamp[ent.x] != next_stamp)
          to_near = atomicExch(&a.stamp[ent.x], next_stamp) != next_stamp;
        stage.push(to_near, ent.x, nq, &nxt.light, a.fq.light_cap, &ctl->err);  // local entries are light
      }
      stage.flush(nq, &nxt.light, a.fq.light_cap, &ctl->err);
      if (bm_out) {  // grid-uniform branch: the CTA's bit-setting reductions, added once
        if (lane == 0 && my_push) atomicAdd_block(&s_push, my_push);
        __syncthreads();
        if (threadIdx.x == 0) {
          if (s_push) atomicAdd(&nxt.vertices, s_push);
          s_push = 0;
        }
        dirty |= 1u << ((P + 1) % 3);
      }
      bm_in = bm_out;
      if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
      ++P;
      continue;
    }

    // ---- near queue drained: advance to the next non-empty bucket --------
    const uint32_t nfar = min(ctl->far_count[fp], a.n);
    if (nfar == 0) break;  // nothing left anywhere
    if (gtid == 0) {
      ctl->min_bucket = 0xFFFFFFFFu;
      ctl->buckets += 1;
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    // R1: minimum bucket among far entries not yet settled
    {
      uint32_t mb = 0xFFFFFFFFu;
      for (uint64_t i = gtid; i < nfar; i += gthreads) {
        const uint32_t d = a.dist[farq[i]];
        if (d >= hi) mb = min(mb, d >> a.shift);
      }
      mb = __reduce_min_sync(kFull, mb);
      if (lane == 0 && mb != 0xFFFFFFFFu) atomicMin(&ctl->min_bucket, mb);
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    const uint32_t nb = ctl->min_bucket;
    if (nb == 0xFFFFFFFFu) break;  // every far entry was settled
    // R2: split the pile into the near queue (bucket nb) and the other pile
    {
      const uint64_t nhi64 = ((uint64_t)nb + 1) << a.shift;
      const uint32_t nhi = nhi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)nhi64;
      uint32_t* keepq = a.far[fp ^ 1];
      for (uint64_t base = gtid - lane; base < nfar; base += gthreads) {
        const uint64_t i = base + lane;
        bool to_near = false, keep = false;
        uint32_t u = 0;
        if (i < nfar) {
          u = farq[i];
          const uint32_t d = a.dist[u];
          if (d >= hi && d < nhi) {
            to_near = true;
            a.stamp[u] = next_stamp;
          } else if (d >= nhi) {
            keep = true;
          }
          if (!keep) atomicAnd(&a.infar[u >> 5], ~(1u << (u & 31)));
        }
        push_discovered<false>(a.fq, qnext, nxt, to_near, u, a.offs, a.heavy, a.tile, &ctl->err);
        warp_push(keep, u, keepq, &ctl->far_count[fp ^ 1], a.n, &ctl->err);
      }
    }
    bucket = nb;
    fp ^= 1;
    bm_in = false;  // the split filled the near queue
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    ++P;
  }
  my_scanned = warp_sum(my_scanned);
  my_relax = warp_sum(my_relax);
  if (lane == 0) {
    if (my_scanned) atomicAdd(&ctl->scanned, my_scanned);
    if (my_relax) atomicAdd(&ctl->relax, my_relax);
  }
  if (gtid == 0) ctl->phases = P;
}

// ---- asynchronous buckets (bounded-degree graphs) ----------------------------

constexpr int kAsyncLQ = 64;  // local-queue entries per warp

__global__ void sssp_async_init(SsspArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t words = (a.n + 31) >> 5;
  for (uint64_t v = tid; v < a.n; v += stride) a.dist[v] = (v == a.src) ? 0u : kInf;
  for (uint64_t w = tid; w < words; w += stride) a.infar[w] = 0;
  const uint64_t b = a.offs[a.src], d = a.offs[a.src + 1] - b;
  for (uint64_t i = tid; i <= a.ring.mask; i += stride) {
    if (i == 0 && d > 0) {
      // the source, published as the chunk of position 0 (counted in work)
      a.ring.ent[0] = make_uint4(a.src, 0u, (uint32_t)b, (uint32_t)((b >> 32) << 16) | (uint32_t)d);
      a.ring.cnt[0] = 1;
      a.ring.seq[0] = 1;
      a.ring.rc->tail = 1;
      a.ring.rc->work = 1;
    } else {
      a.ring.seq[i] = i;
    }
  }
}

// Delta-stepping with asynchronous buckets.  Needs every vertex light
// (degree <= a.heavy, < 65536) and offsets below 2^48: worklist entries are
// (vertex, distance, begin offset low, begin offset high << 16 | degree).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) sssp_async(SsspArgs a) {
  static_assert(worklists::kErrTimeout == kDevTimeout && worklists::kErrOverflow == kDevOverflow,
                "the worklist raises the library's device error codes");
  __shared__ uint4 s_lq[BLOCK / 32][kAsyncLQ];
  SsspCtl* ctl = a.ctl;
  worklists::RingCtl* rc = a.ring.rc;
  const unsigned nblocks = gridDim.x;
  const uint64_t deadline = kernel_deadline();
  const uint32_t lane = lane_id();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  unsigned long long my_scanned = 0, my_relax = 0;

  uint32_t bucket = 0;
  int fp = 0;
  uint32_t P = 0;  // buckets processed
  for (;;) {
    if (P >= a.max_phases) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    const uint64_t hi64 = ((uint64_t)bucket + 1) << a.shift;
    const uint32_t hi = hi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)hi64;
    uint32_t* farq = a.far[fp];
    // ---- the bucket's work, no grid barrier --------------------------------
    worklists::WarpQueue<kAsyncLQ> q(s_lq[threadIdx.x >> 5], a.ring, &ctl->err, deadline);
    // Relax to nd the arc into u: near improvements join the worklist, far
    // ones the far pile (once, by the bitmap).  The target's offsets load
    // beside the atomic.
    auto relax = [&](bool valid, uint32_t u, uint32_t nd) {
      bool near = false, far = false;
      uint64_t ub = 0, deg = 0;
      if (valid) {
        ub = ldg(a.offs + u);
        deg = ldg(a.offs + u + 1) - ub;
        const uint32_t old = atomicMin(&a.dist[u], nd);
        if (nd < old) {
          ++my_relax;
          if (nd < hi) {
            near = deg > 0;  // nothing to relax from a vertex without arcs
          } else {
            const uint32_t bit = 1u << (u & 31);
            if (!(a.infar[u >> 5] & bit)) far = !(atomicOr(&a.infar[u >> 5], bit) & bit);
          }
        }
      }
      q.push(near, make_uint4(u, nd, (uint32_t)ub, (uint32_t)((ub >> 32) << 16) | (uint32_t)deg));
      warp_push(far, u, farq, &ctl->far_count[fp], a.n, &ctl->err);
    };
    for (;;) {
      uint4 ent;
      bool has;
      if (q.next(ent, has) <= 0) break;  // the bucket is done (or an error was raised)
      // one round: every lane's vertex, its arcs spread over the warp; an
      // entry whose vertex has a smaller distance by now is stale (whoever
      // lowered it queued the vertex again)
      const uint64_t b = ((uint64_t)(ent.w >> 16) << 32) | ent.z;
      const uint32_t d = has ? (ent.w & 0xFFFFu) : 0u;
      const uint32_t cur = has ? __ldcg(a.dist + ent.x) : 0u;
      my_scanned += d;
      warp_expand_mlp<4, uint32_t>(
          b, d, ent.y, [&](bool valid, uint64_t e, uint32_t) { return valid ? ldg(a.col + e) : 0u; },
          [&](bool valid, uint64_t e, uint32_t, uint32_t dsrc) { return valid ? dsrc + ldg(a.w + e) : 0u; },
          [&](bool valid, uint32_t owner, uint32_t dsrc, uint32_t u, uint32_t nd) {
            const bool live = __shfl_sync(kFull, cur, owner) >= dsrc;
            relax(valid && live, u, nd);
          });
      q.share();
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    // ---- bucket transition ---------------------------------------------------
    const uint32_t nfar = min(ctl->far_count[fp], a.n);
    ++P;
    if (nfar == 0) break;  // nothing left anywhere
    if (gtid == 0) {
      rc->head = rc->tail;  // tickets still waiting when the bucket ended are void
      ctl->min_bucket = 0xFFFFFFFFu;
      ctl->buckets += 1;
      ctl->far_count[fp ^ 1] = 0;
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    // R1: minimum bucket among far entries not yet settled
    {
      uint32_t mb = 0xFFFFFFFFu;
      for (uint64_t i = gtid; i < nfar; i += gthreads) {
        const uint32_t dd = a.dist[farq[i]];
        if (dd >= hi) mb = min(mb, dd >> a.shift);
      }
      mb = __reduce_min_sync(kFull, mb);
      if (lane == 0 && mb != 0xFFFFFFFFu) atomicMin(&ctl->min_bucket, mb);
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    const uint32_t nb = ctl->min_bucket;
    if (nb == 0xFFFFFFFFu) break;  // every far entry was settled
    // R2: the entries of bucket nb become chunks, later ones stay in the pile
    {
      const uint64_t nhi64 = ((uint64_t)nb + 1) << a.shift;
      const uint32_t nhi = nhi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)nhi64;
      uint32_t* keepq = a.far[fp ^ 1];
      for (uint64_t base = gtid - lane; base < nfar; base += gthreads) {
        const uint64_t i = base + lane;
        bool to_near = false, keep = false;
        uint32_t u = 0, dd = 0;
        uint64_t ub = 0, deg = 0;
        if (i < nfar) {
          u = farq[i];
          dd = a.dist[u];
          if (dd >= hi && dd < nhi) {
            ub = ldg(a.offs + u);
            deg = ldg(a.offs + u + 1) - ub;
            to_near = deg > 0;
          } else if (dd >= nhi) {
            keep = true;
          }
          if (!keep) atomicAnd(&a.infar[u >> 5], ~(1u << (u & 31)));
        }
        worklists::publish(a.ring, to_near,
                           make_uint4(u, dd, (uint32_t)ub, (uint32_t)((ub >> 32) << 16) | (uint32_t)deg), &ctl->err);
        warp_push(keep, u, keepq, &ctl->far_count[fp ^ 1], a.n, &ctl->err);
      }
    }
    bucket = nb;
    fp ^= 1;
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
  }
  my_scanned = warp_sum(my_scanned);
  my_relax = warp_sum(my_relax);
  if (lane == 0) {
    if (my_scanned) atomicAdd(&ctl->scanned, my_scanned);
    if (my_relax) atomicAdd(&ctl->relax, my_relax);
  }
  if (gtid == 0) ctl->phases = P;
}

// ---- asynchronous buckets over fixed-width rows ------------------------------
// For graphs of degree <= D (D = 4 or 8) the arcs are also kept as
// fixed-width rows: vertex u's D columns at ell[u*D ..], its D weights at
// ell[n*D + u*D ..], empty slots 0xFFFFFFFF.  A row's address follows from
// the vertex id alone, so a relaxation loads the target's row beside its
// atomicMin, and a queued entry carries the row it will expand: one hop of
// the dependent chain is one memory round trip (the atomic and the row load
// in flight together) instead of two (arcs, then atomics).  D lanes work on
// one vertex (lane k on its k-th slot), 32 / D vertices per round.

constexpr uint32_t kNoArc = 0xFFFFFFFFu;

__global__ void ell_build_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col,
                                 const uint32_t* __restrict__ w, uint32_t n, uint32_t D, uint32_t* __restrict__ ell) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)n * D; i += stride) {
    const uint64_t v = i / D, k = i % D;
    const uint64_t b = offs[v], deg = offs[v + 1] - b;
    ell[i] = k < deg ? col[b + k] : kNoArc;
    ell[(uint64_t)n * D + i] = k < deg ? w[b + k] : kNoArc;
  }
}

template <int D>
struct EllRow {
  uint4 c[D / 4];
  uint4 w[D / 4];
};

template <int D>
__device__ __forceinline__ EllRow<D> ell_row(const uint32_t* __restrict__ ell, uint32_t n, uint32_t u) {
  EllRow<D> r;
  const uint4* pc = reinterpret_cast<const uint4*>(ell + (uint64_t)u * D);
  const uint4* pw = reinterpret_cast<const uint4*>(ell + (uint64_t)n * D + (uint64_t)u * D);
#pragma unroll
  for (int j = 0; j < D / 4; ++j) {
    r.c[j] = ldg(pc + j);
    r.w[j] = ldg(pw + j);
  }
  return r;
}

__device__ __forceinline__ uint32_t u4_at(const uint4& v, uint32_t k) {
  return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}

constexpr int kEllLQ = 64;  // local-queue entries per warp

template <int BLOCK, int D>
__global__ void __launch_bounds__(BLOCK) sssp_async_ell(SsspArgs a, const uint32_t* __restrict__ ell) {
  static_assert(D == 4 || D == 8, "rows of 4 or 8 slots");
  constexpr uint32_t kPer = 32 / D;  // vertices per round
  __shared__ uint2 s_meta[BLOCK / 32][kEllLQ];  // (vertex, distance)
  __shared__ EllRow<D> s_row[BLOCK / 32][kEllLQ];
  SsspCtl* ctl = a.ctl;
  worklists::RingCtl* rc = a.ring.rc;
  const unsigned nblocks = gridDim.x;
  const uint64_t deadline = kernel_deadline();
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const uint32_t slot = lane / D, k = lane % D;
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  uint2* meta = s_meta[wib];
  EllRow<D>* rows = s_row[wib];
  unsigned long long my_scanned = 0, my_relax = 0;
  uint32_t bucket = 0;
  int fp = 0;
  uint32_t P = 0;
  for (;;) {
    if (P >= a.max_phases) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    const uint64_t hi64 = ((uint64_t)bucket + 1) << a.shift;
    const uint32_t hi = hi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)hi64;
    uint32_t* farq = a.far[fp];
    uint32_t lq_n = 0;  // warp-uniform
    bool busy = false;  // this warp holds one count of rc->work
    // the 32 oldest local entries leave as one ring chunk of (vertex, distance)
    auto spill_oldest = [&]() {
      const uint2 e = meta[lane];
      __syncwarp();
      for (uint32_t i = 32 + lane; i < lq_n; i += 32) {
        meta[i - 32] = meta[i];
        rows[i - 32] = rows[i];
      }
      __syncwarp();
      lq_n -= 32;
      worklists::publish(a.ring, true, make_uint4(e.x, e.y, 0u, 0u), &ctl->err);
    };
    for (;;) {
      uint32_t v = 0, dv = 0, u = 0, w = 0;
      bool has = false;
      if (lq_n == 0) {
        // out of work: give up this warp's count, take a ticket, wait for a chunk
        if (busy && lane == 0) atomicSub(&rc->work, 1);
        busy = false;
        unsigned long long p = 0;
        int got = 0;
        if (lane == 0) {
          p = atomicAdd(&rc->head, 1ull);
          got = worklists::wait_chunk(a.ring, p, &ctl->err, deadline);
        }
        got = __shfl_sync(kFull, got, 0);
        if (got <= 0) break;  // the bucket is done (or an error was raised)
        p = __shfl_sync(kFull, p, 0);
        __syncwarp();
        busy = true;
        const unsigned long long cs = p & a.ring.mask;
        const uint32_t c = __ldcg(a.ring.cnt + cs);
        if (lane < c) {
          const uint4 e = __ldcg(a.ring.ent + cs * 32 + lane);
          meta[lane] = make_uint2(e.x, e.y);
          rows[lane] = ell_row<D>(ell, a.n, e.x);
        }
        __syncwarp();
        if (lane == 0) worklists::st_release(a.ring.seq + cs, p + a.ring.mask + 1);
        lq_n = c;
      }
      // one round: the kPer most recent entries, lane k on slot k of its vertex
      const uint32_t take = min(kPer, lq_n);
      has = slot < take;
      if (has) {
        const uint32_t idx = lq_n - take + slot;
        const uint2 m = meta[idx];
        v = m.x;
        dv = m.y;
        u = u4_at(rows[idx].c[k >> 2], k & 3);
        w = u4_at(rows[idx].w[k >> 2], k & 3);
      }
      __syncwarp();
      lq_n -= take;
      const bool valid = has && u != kNoArc;
      const uint32_t nd = dv + w;
      // in flight together: the entry's own distance (stale check), the
      // target's atomic and the target's row
      const uint32_t cur = (has && k == 0) ? __ldcg(a.dist + v) : 0u;
      uint32_t old = 0;
      EllRow<D> nr{};
      if (valid) {
        old = atomicMin(&a.dist[u], nd);
        nr = ell_row<D>(ell, a.n, u);
      }
      const bool live = __shfl_sync(kFull, cur, lane & ~(D - 1)) >= dv;
      const bool improved = valid && live && nd < old;
      if (valid && live) ++my_scanned;
      bool near = false, far = false;
      if (improved) {
        ++my_relax;
        if (nd < hi) {
          near = nr.c[0].x != kNoArc;  // nothing to relax from a vertex without arcs
        } else {
          const uint32_t bit = 1u << (u & 31);
          if (!(a.infar[u >> 5] & bit)) far = !(atomicOr(&a.infar[u >> 5], bit) & bit);
        }
      }
      const unsigned nm = __ballot_sync(kFull, near);
      if (nm) {
        const uint32_t kk = __popc(nm);
        if (lq_n + kk > (uint32_t)kEllLQ) spill_oldest();
        if (near) {
          const uint32_t pos = lq_n + __popc(nm & lanemask_lt);
          meta[pos] = make_uint2(u, nd);
          rows[pos] = nr;
        }
        lq_n += kk;
        __syncwarp();
      }
      warp_push(far, u, farq, &ctl->far_count[fp], a.n, &ctl->err);
      // while other warps wait for work, hand them the oldest entries
      if (lq_n > 32) {
        int want = 0;
        if (lane == 0)
          want = *reinterpret_cast<const volatile unsigned long long*>(&rc->head) >
                 *reinterpret_cast<const volatile unsigned long long*>(&rc->tail);
        if (__shfl_sync(kFull, want, 0)) spill_oldest();
      }
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    // ---- bucket transition (as sssp_async) --------------------------------------
    const uint32_t nfar = min(ctl->far_count[fp], a.n);
    ++P;
    if (nfar == 0) break;
    if (gtid == 0) {
      rc->head = rc->tail;
      ctl->min_bucket = 0xFFFFFFFFu;
      ctl->buckets += 1;
      ctl->far_count[fp ^ 1] = 0;
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    {
      uint32_t mb = 0xFFFFFFFFu;
      for (uint64_t i = gtid; i < nfar; i += gthreads) {
        const uint32_t dd = a.dist[farq[i]];
        if (dd >= hi) mb = min(mb, dd >> a.shift);
      }
      mb = __reduce_min_sync(kFull, mb);
      if (lane == 0 && mb != 0xFFFFFFFFu) atomicMin(&ctl->min_bucket, mb);
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    const uint32_t nb = ctl->min_bucket;
    if (nb == 0xFFFFFFFFu) break;
    {
      const uint64_t nhi64 = ((uint64_t)nb + 1) << a.shift;
      const uint32_t nhi = nhi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)nhi64;
      uint32_t* keepq = a.far[fp ^ 1];
      for (uint64_t base = gtid - lane; base < nfar; base += gthreads) {
        const uint64_t i = base + lane;
        bool to_near = false, keep = false;
        uint32_t uu = 0, dd = 0;
        if (i < nfar) {
          uu = farq[i];
          dd = a.dist[uu];
          if (dd >= hi && dd < nhi) to_near = ell[(uint64_t)uu * D] != kNoArc;
          else if (dd >= nhi) keep = true;
          if (!keep) atomicAnd(&a.infar[uu >> 5], ~(1u << (uu & 31)));
        }
        worklists::publish(a.ring, to_near, make_uint4(uu, dd, 0u, 0u), &ctl->err);
        warp_push(keep, uu, keepq, &ctl->far_count[fp ^ 1], a.n, &ctl->err);
      }
    }
    bucket = nb;
    fp ^= 1;
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
  }
  my_scanned = warp_sum(my_scanned);
  my_relax = warp_sum(my_relax);
  if (lane == 0) {
    if (my_scanned) atomicAdd(&ctl->scanned, my_scanned);
    if (my_relax) atomicAdd(&ctl->relax, my_relax);
  }
  if (gtid == 0) ctl->phases = P;
}

// ---- regions in shared memory (bounded-degree graphs numbered by locality) ---
// On a graph numbered so that consecutive ids form compact patches
// (GB_ORDER_LOCALITY), the vertices [r * kRegion, (r + 1) * kRegion) form
// region r and most arcs stay inside their region.  A CTA takes one queued
// region at a time, loads its distances, row offsets and arcs into shared
// memory and relaxes to a local fixed point inside the current bucket: a hop
// inside the region is a shared-memory atomic and a barrier of the relaxing
// warps, not a global round trip.  An arc that leaves the region lowers the global distance and
// then either marks the target pending (one bit per vertex) and queues the
// target's region, or files the target in the far pile.  Global distances
// stay authoritative: the region writes its lowered distances back with
// atomicMin, and pending bits set while it ran queue it again when it is
// released.  Regions travel through the device worklist ring
// (gb_worklist.cuh) as single ids, at most once each (a queued flag per
// region); a bucket ends when no region is queued and no CTA holds one.

// 2048-vertex regions (27.4 ms on the 4096^2 grid against 29.3 for 4096 and
// 28.7 for 1024, measured with two CTAs per SM), one CTA per SM: the CTAs
// mostly wait for queued regions, and 96 registers a thread instead of 64
// shorten a round (733 against 827 cycles per hop of a path; grid 16.9
// against 17.4 ms)
constexpr uint32_t kRegion = 2048;       // vertices per region (a multiple of 32)
constexpr uint32_t kRegionArcs = 8192;   // arcs a region may hold in shared memory
constexpr uint32_t kRegionOut = 128;     // outbox: relaxations of arcs leaving the region, per round
constexpr uint32_t kRegionOutBufs = 8;   // outbox buffers (round k uses buffer k % 8)
constexpr int kRegionBlock = 512;
constexpr int kRegionPerSm = 1;
constexpr int kRegionRelax = 448;        // threads that relax (warps 0-13); warps 14 and 15 are the couriers
static_assert(kRegion % 1024 == 0, "a lane takes kRegion / 1024 pending words");
constexpr int kRegionPer = (kRegion + kRegionBlock - 1) / kRegionBlock;  // vertices of a region per thread

struct RegionArgs {
  uint32_t* pend;  // bitmap: vertex lowered from outside its region, to be expanded
  uint32_t* rq;    // per region: queued or being processed (1) or not (0)
  uint32_t nregions;
};

// D = 0: the region's arcs as CSR (row offsets, columns, weights); D > 0:
// fixed rows of D slots per vertex (graphs of degree <= D: a lane reads its
// arc from the vertex id alone, one dependent load fewer per round).
template <int D>
constexpr size_t region_smem_bytes() {
  return sizeof(uint32_t) * kRegion                                    // distances
         + (D ? 0 : sizeof(uint32_t) * (kRegion + 4))                  // local row offsets
         + 2 * sizeof(uint32_t) * (D ? (size_t)kRegion * D : kRegionArcs)  // columns, weights
         + 2 * sizeof(uint16_t) * kRegion        // the two round worklists
         + 3 * sizeof(uint32_t) * (kRegion / 32) // two listed bitmaps, the inbox bitmap
         + sizeof(uint2) * kRegionOutBufs * kRegionOut;  // outbox buffers
}

// Shared-memory flags between the relaxing warps and the couriers.
__device__ __forceinline__ uint32_t ld_acquire_cta(uint32_t* p) {
  return cuda::atomic_ref<uint32_t, cuda::thread_scope_block>(*p).load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release_cta(uint32_t* p, uint32_t v) {
  cuda::atomic_ref<uint32_t, cuda::thread_scope_block>(*p).store(v, cuda::memory_order_release);
}

// Largest arc count of any region (out[0], the host check that regions fit)
// and the number of arcs whose two ends share a region (out[1]).
__global__ void region_arcs_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col, uint32_t n,
                                   uint32_t nregions, unsigned long long* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  unsigned long long mine = 0, local = 0;
  for (uint64_t r = tid; r < nregions; r += stride) {
    const uint64_t b = r * kRegion, e = b + kRegion < (uint64_t)n ? b + kRegion : (uint64_t)n;
    mine = max(mine, (unsigned long long)(offs[e] - offs[b]));
  }
  // arcs by row: a thread per vertex
  for (uint64_t v = tid; v < n; v += stride) {
    const uint64_t r = v / kRegion;
    for (uint64_t j = offs[v]; j < offs[v + 1]; ++j) local += (uint64_t)col[j] / kRegion == r;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mine = max(mine, __shfl_xor_sync(kFull, mine, o));
    local += __shfl_xor_sync(kFull, local, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, mine);
    atomicAdd(out + 1, local);
  }
}

__global__ void sssp_region_init(SsspArgs a, RegionArgs ra) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t words = (a.n + 31) >> 5;
  for (uint64_t v = tid; v < a.n; v += stride) a.dist[v] = (v == a.src) ? 0u : kInf;
  for (uint64_t w = tid; w < words; w += stride) {
    a.infar[w] = 0;
    ra.pend[w] = (w == (a.src >> 5)) ? (1u << (a.src & 31)) : 0u;
  }
  const uint32_t r0 = a.src / kRegion;
  for (uint64_t r = tid; r < ra.nregions; r += stride) ra.rq[r] = (r == r0) ? 1u : 0u;
  if (tid == 0) a.ctl->far_min[0] = a.ctl->far_min[1] = 0xFFFFFFFFu;
  for (uint64_t i = tid; i <= a.ring.mask; i += stride) {
    if (i == 0) {  // the source's region, published as the chunk of position 0 (counted in work)
      a.ring.ent[0] = make_uint4(r0, 0u, 0u, 0u);
      a.ring.cnt[0] = 1;
      a.ring.seq[0] = 1;
      a.ring.rc->tail = 1;
      a.ring.rc->work = 1;
    } else {
      a.ring.seq[i] = i;
    }
  }
}

// u (outside the caller's region) was lowered to a distance inside the
// bucket (the atomicMin has returned): announce it with its pending bit and
// queue its region unless it is queued.  No fence is needed: every step is an
// atomic whose result is awaited before the next one is issued, and the
// region's release (atomicExch of its flag, then a read of its bits) is built
// the same way, so either this call sees the flag cleared or the release sees
// the bit.  A bit that was set already was announced by its setter, which
// took care of the queue, and the region reads the distance after taking the
// bit.
__device__ __forceinline__ void region_touch(const SsspArgs& a, const RegionArgs& ra, uint32_t u, int* err) {
  const uint32_t bit = 1u << (u & 31);
  if (atomicOr(&ra.pend[u >> 5], bit) & bit) return;
  const uint32_t rg = u / kRegion;
  if (atomicOr(&ra.rq[rg], 1u) == 0u) worklists::publish_one(a.ring, make_uint4(rg, 0u, 0u, 0u), err);
}

// File u (lowered to nd, beyond the bucket) in the far pile once, and record
// nd's bucket in the CTA's least bucket for the pile (s_fmin).
__device__ __forceinline__ void far_file(const SsspArgs& a, uint32_t* farq, uint32_t* count, uint32_t u, uint32_t nd,
                                         uint32_t* s_fmin, int* err) {
  atomicMin(s_fmin, nd >> a.shift);
  const uint32_t bit = 1u << (u & 31);
  if (!(__ldcg(a.infar + (u >> 5)) & bit) && !(atomicOr(&a.infar[u >> 5], bit) & bit)) {
    const uint32_t pos = atomicAdd(count, 1u);
    if (pos < a.n) farq[pos] = u;
    else raise_err(err, kDevOverflow);
  }
}

// Load a region into shared memory with 16-byte loads: its distances (base
// is a multiple of kRegion, so 16-byte aligned), its nv + 1 offsets relative
// to o0, and its na arcs from o0 (any alignment: the unaligned head and tail
// are loaded one by one).  Only elements inside the arrays are read.
__device__ __forceinline__ void region_load(const SsspArgs& a, uint32_t base, uint32_t nv, uint64_t o0, uint32_t na,
                                            uint32_t* s_dist, uint32_t* s_loff, uint32_t* s_col, uint32_t* s_w) {
  const uint32_t tid = threadIdx.x;
  const uint4* d4 = reinterpret_cast<const uint4*>(a.dist + base);
#pragma unroll 4
  for (uint32_t q = tid; q < nv / 4; q += kRegionBlock) reinterpret_cast<uint4*>(s_dist)[q] = __ldcg(d4 + q);
  for (uint32_t i = (nv & ~3u) + tid; i < nv; i += kRegionBlock) s_dist[i] = __ldcg(a.dist + base + i);
  const ulonglong2* o2 = reinterpret_cast<const ulonglong2*>(a.offs + base);
  const uint32_t npairs = (nv + 1) / 2;  // offsets [0, 2 * npairs) lie within [0, nv]
#pragma unroll 4
  for (uint32_t q = tid; q < npairs; q += kRegionBlock) {
    const ulonglong2 x = ldg(o2 + q);
    s_loff[2 * q] = (uint32_t)(x.x - o0);
    s_loff[2 * q + 1] = (uint32_t)(x.y - o0);
  }
  if (tid == 0 && 2 * npairs == nv) s_loff[nv] = (uint32_t)(ldg(a.offs + base + nv) - o0);
  // arcs: [o0, q0 * 4) and [q1 * 4, o0 + na) one by one, [q0, q1) as 16-byte words
  const uint64_t e = o0 + na;
  const uint64_t q0 = (o0 + 3) / 4, q1 = e / 4;
  if (q0 < q1) {
    const uint4* c4 = reinterpret_cast<const uint4*>(a.col);
    const uint4* w4 = reinterpret_cast<const uint4*>(a.w);
    const uint32_t nq = (uint32_t)(q1 - q0);
    const uint32_t off = (uint32_t)(q0 * 4 - o0);
#pragma unroll 4
    for (uint32_t q = tid; q < nq; q += kRegionBlock) {
      const uint4 c = ldg(c4 + q0 + q), w = ldg(w4 + q0 + q);
      const uint32_t j = off + 4 * q;
      s_col[j] = c.x, s_col[j + 1] = c.y, s_col[j + 2] = c.z, s_col[j + 3] = c.w;
      s_w[j] = w.x, s_w[j + 1] = w.y, s_w[j + 2] = w.z, s_w[j + 3] = w.w;
    }
    for (uint32_t t = tid; t < off; t += kRegionBlock) {
      s_col[t] = ldg(a.col + o0 + t);
      s_w[t] = ldg(a.w + o0 + t);
    }
    for (uint64_t g = q1 * 4 + tid; g < e; g += kRegionBlock) {
      s_col[g - o0] = ldg(a.col + g);
      s_w[g - o0] = ldg(a.w + g);
    }
  } else {
    for (uint32_t t = tid; t < na; t += kRegionBlock) {
      s_col[t] = ldg(a.col + o0 + t);
      s_w[t] = ldg(a.w + o0 + t);
    }
  }
}

// The region's distances, and its arcs as rows of D slots (empty slots
// kNoArc; every vertex has at most D arcs, checked on the host).
template <int D>
__device__ __forceinline__ void region_load_rows(const SsspArgs& a, uint32_t base, uint32_t nv, uint32_t* s_dist,
                                                 uint32_t* s_col, uint32_t* s_w) {
  const uint32_t tid = threadIdx.x;
  const uint4* d4 = reinterpret_cast<const uint4*>(a.dist + base);
#pragma unroll 4
  for (uint32_t q = tid; q < nv / 4; q += kRegionBlock) reinterpret_cast<uint4*>(s_dist)[q] = __ldcg(d4 + q);
  for (uint32_t i = (nv & ~3u) + tid; i < nv; i += kRegionBlock) s_dist[i] = __ldcg(a.dist + base + i);
  // a thread's vertices all at once: their offsets, then their arcs (two
  // dependent loads in all, not two per vertex)
  constexpr int kPer = kRegionPer;
  uint64_t b[kPer], e[kPer];
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const uint32_t lv = tid + t * kRegionBlock;
    b[t] = e[t] = 0;
    if (lv < nv) b[t] = ldg(a.offs + base + lv), e[t] = ldg(a.offs + base + lv + 1);
  }
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const uint32_t lv = tid + t * kRegionBlock;
    if (lv < nv) {
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const bool ok = b[t] + k < e[t];
        s_col[lv * D + k] = ok ? ldg(a.col + b[t] + k) : kNoArc;
        s_w[lv * D + k] = ok ? ldg(a.w + b[t] + k) : 0u;
      }
    }
  }
}

// Needs every region's arcs to fit (at most kRegionArcs; checked on the host).
template <int D>
__global__ void __launch_bounds__(kRegionBlock, kRegionPerSm) sssp_region(SsspArgs a, RegionArgs ra) {
  static_assert(worklists::kErrTimeout == kDevTimeout && worklists::kErrOverflow == kDevOverflow,
                "the worklist raises the library's device error codes");
  extern __shared__ __align__(16) unsigned char s_raw[];
  constexpr uint32_t kArcSlots = D ? kRegion * D : kRegionArcs;
  uint32_t* s_dist = reinterpret_cast<uint32_t*>(s_raw);
  uint32_t* s_loff = s_dist + kRegion;  // D == 0 only
  uint32_t* s_col = D ? s_dist + kRegion : s_loff + kRegion + 4;
  uint32_t* s_w = s_col + kArcSlots;
  uint2* s_out = reinterpret_cast<uint2*>(s_w + kArcSlots);  // [kRegionOutBufs][kRegionOut] outbox
  uint32_t* s_bm = reinterpret_cast<uint32_t*>(s_out + kRegionOutBufs * kRegionOut);  // [2][kRegion / 32] listed bitmaps
  uint32_t* s_inbm = s_bm + 2 * (kRegion / 32);                         // inbox: taken pending vertices
  uint16_t* s_wl = reinterpret_cast<uint16_t*>(s_inbm + kRegion / 32);  // [2][kRegion] round lists
  // s_on: entries in each outbox buffer; s_obok[k & 1]: round k may use its
  // buffer; s_opub: rounds published to the outbox courier; s_odone: rounds
  // it has taken; s_qreq: the relaxers' latest request to finish; s_in_any:
  // the inbox has vertices
  __shared__ uint32_t s_region, s_go, s_n[3], s_on[kRegionOutBufs], s_obok[2], s_opub, s_odone, s_qreq, s_in_any;
  // least bucket of the distances this CTA filed in the current far pile
  // since it last added them to ctl->far_min
  __shared__ uint32_t s_fmin;
  if (threadIdx.x == 0) s_fmin = 0xFFFFFFFFu;  // the first barrier below orders it
  SsspCtl* ctl = a.ctl;
  worklists::RingCtl* rc = a.ring.rc;
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kRegionBlock + tid;
  const uint64_t gthreads = (uint64_t)gridDim.x * kRegionBlock;
  unsigned long long my_scanned = 0, my_relax = 0, my_rounds = 0;
  uint32_t bucket = 0;
  int fp = 0;
  uint32_t P = 0;
  bool busy = false;  // thread 0: this CTA holds one count of rc->work
  for (;;) {
    if (P >= a.max_phases) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    const uint64_t hi64 = ((uint64_t)bucket + 1) << a.shift;
    const uint32_t hi = hi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)hi64;
    uint32_t* farq = a.far[fp];
    uint32_t* far_count = &ctl->far_count[fp];
    // ---- the bucket's regions, no grid barrier ---------------------------------
    for (;;) {
      if (tid == 0) {
        if (busy) atomicSub(&rc->work, 1);
        busy = false;
        const unsigned long long p = atomicAdd(&rc->head, 1ull);
        // a queued region is on the path of the bucket's wave: poll often
        const int got = worklists::wait_chunk(a.ring, p, &ctl->err, deadline, 128);
        s_go = got > 0 ? 1u : 0u;
        if (got > 0) {
          busy = true;  // the chunk's count is now this CTA's
          const unsigned long long cs = p & a.ring.mask;
          s_region = __ldcg(&a.ring.ent[cs * 32].x);
          worklists::st_release(a.ring.seq + cs, p + a.ring.mask + 1);
        }
      }
      __syncthreads();
      if (!s_go) break;  // the bucket is done (or an error was raised)
      const uint32_t r = s_region;
      const uint32_t base = r * kRegion;
      const uint32_t nv = min(kRegion, a.n - base);
      const uint32_t nw = (nv + 31) >> 5;
      const uint64_t o0 = ldg(a.offs + base);
      const uint32_t na = (uint32_t)(ldg(a.offs + base + nv) - o0);
      if (tid == 0) s_n[0] = s_n[1] = s_n[2] = s_opub = s_odone = s_qreq = s_in_any = 0;
      if (tid < kRegionOutBufs) s_on[tid] = 0;
      if (tid == 0) s_obok[0] = 1;
      for (uint32_t j = tid; j < kRegion / 32; j += kRegionBlock) s_bm[kRegion / 32 + j] = s_inbm[j] = 0u;
      __syncthreads();
      // the pending vertices start the worklist; they are taken before the
      // distances are read, so a lowering after this point sets its bit again
      for (uint32_t j = tid; j < kRegion / 32; j += kRegionBlock) {
        uint32_t bits = j < nw ? atomicExch(&ra.pend[(base >> 5) + j], 0u) : 0u;
        s_bm[j] = bits;
        if (bits) {
          const uint32_t pos = atomicAdd(&s_n[0], (uint32_t)__popc(bits));
          for (uint32_t k = 0; bits; ++k, bits &= bits - 1) s_wl[pos + k] = (uint16_t)(j * 32 + __ffs(bits) - 1);
        }
      }
      // no fence: the exchanges above have returned, and a writer's
      // atomicMin on a distance had returned before it set the pending bit
      // (region_touch), so the L2 reads below (ldcg) see it
      __syncthreads();
      if constexpr (D == 0) region_load(a, base, nv, o0, na, s_dist, s_loff, s_col, s_w);
      else region_load_rows<D>(a, base, nv, s_dist, s_col, s_w);
      __syncthreads();
      // Warps 0-13 relax in rounds.  Round k relaxes list k & 1 (count
      // s_n[k % 3]) into list (k + 1) & 1 (count s_n[(k + 1) % 3], listed
      // bitmap (k + 1) & 1) and clears bitmap k & 1 and s_n[(k + 2) % 3],
      // which no thread uses in round k, so one barrier of the relaxing
      // threads per round suffices.  A vertex lowered while its entry is
      // being expanded is listed again for the next round, so the expansion
      // may read its distance at any time.  Four lanes share an entry, one arc
      // each; each lane appends what it lists.  An arc that leaves the region
      // goes to outbox buffer k % 8, which warp 15 (a courier) applies to the
      // global distances once the round is published (queueing the targets'
      // regions or filing them far) while the rounds go on; when the courier
      // has not yet taken the buffer's previous round, the arc is applied on
      // the spot.  Warp 14 polls the region's pending bits: it takes them,
      // lowers the shared distances to the global ones (atomicMin) and marks
      // the vertices in the inbox bitmap.  Warps 12 and 13, which relax only
      // in rounds of more than 96 entries, keep the books: warp 12 publishes
      // the last round (a release), warp 13 clears the bitmap, moves the
      // inbox into the next round's list and decides whether the next round
      // may use its buffer (an acquire), so the fences (about 400 cycles
      // each) stay off the other warps' path.  When a round lists nothing,
      // the relaxers ask the couriers to finish (the outbox drained, one more
      // poll) and all 512 threads meet; the visit goes on if the inbox holds
      // vertices.
      constexpr uint32_t kBooks = kRegionRelax / 32 - 1;  // the book-keeping warp
      uint32_t k = 0, jo = 0;
      for (uint32_t q = 1;; ++q) {
        if (warp < kRegionRelax / 32) {
          for (;; ++k) {
            const uint32_t cnt = s_n[k % 3];
            const uint16_t* wl = s_wl + (k & 1) * kRegion;
            uint16_t* wl_next = s_wl + ((k + 1) & 1) * kRegion;
            uint32_t* bm_next = s_bm + ((k + 1) & 1) * (kRegion / 32);
            uint32_t* n_next = &s_n[(k + 1) % 3];
            if (warp == kBooks - 1 && lane == 0) {
              if (k > 0) st_release_cta(&s_opub, k);  // rounds < k are complete
              s_n[(k + 2) % 3] = 0;
            }
            if (warp == kBooks) {
              if (lane == 0) {
                // round k + 1's buffer was last used by round k + 1 - 8 (none
                // for k < 7); the courier clears its count when it takes it.
                // (A count of zero is no sign: the courier may not have taken
                // that empty round yet, and would read this round's count.)
                const uint32_t nb = k + 1 - kRegionOutBufs;
                const bool ok = k + 1 < kRegionOutBufs || ld_acquire_cta(&s_odone) > nb;
                s_obok[(k + 1) & 1] = ok ? 1u : 0u;
              }
#pragma unroll
              for (uint32_t t = 0; t < kRegion / 1024; ++t) s_bm[(k & 1) * (kRegion / 32) + lane + 32 * t] = 0u;
              // the inbox flag is cleared before the bits are taken (the
              // courier sets bits, then the flag)
              uint32_t f = 0;
              if (lane == 0 && *reinterpret_cast<volatile uint32_t*>(&s_in_any) != 0u) f = atomicExch(&s_in_any, 0u);
              if (__shfl_sync(kFull, f, 0) != 0u) {
                __threadfence_block();
                for (uint32_t w = lane; w < nw; w += 32) {
                  uint32_t bits = atomicExch(&s_inbm[w], 0u);
                  for (; bits; bits &= bits - 1) {
                    const uint32_t b = __ffs(bits) - 1, i = w * 32 + b;
                    if (*reinterpret_cast<volatile uint32_t*>(&s_dist[i]) < hi &&
                        !(atomicOr(&bm_next[w], 1u << b) & (1u << b)))
                      wl_next[atomicAdd(n_next, 1u)] = (uint16_t)i;
                  }
                }
              }
            }
            const bool ob_ok = *reinterpret_cast<volatile uint32_t*>(&s_obok[k & 1]) != 0u;
            uint32_t* on = &s_on[k % kRegionOutBufs];
            uint2* ob = s_out + (k % kRegionOutBufs) * kRegionOut;
            for (uint32_t i0 = warp * 8; i0 < cnt; i0 += kRegionRelax / 4) {  // warp-uniform
              const uint32_t i = i0 + (lane >> 2), sub = lane & 3u;
              const bool has = i < cnt;
              const uint32_t v = has ? (uint32_t)wl[i] : 0u;
              const uint32_t d = has ? *reinterpret_cast<volatile uint32_t*>(&s_dist[v]) : hi;
              const bool live = d < hi;
              // relax one arc per lane (valid lanes) and append what it lists
              auto relax = [&](bool valid, uint32_t u, uint32_t nd, bool precheck) {
                if (!valid) return;
                ++my_scanned;
                const uint32_t lu = u - base;
                if (lu < nv) {
                  if ((!precheck || nd < *reinterpret_cast<volatile uint32_t*>(&s_dist[lu])) &&
                      nd < atomicMin(&s_dist[lu], nd)) {
                    ++my_relax;
                    const uint32_t bit = 1u << (lu & 31);
                    // each lane appends on its own: a shared-memory atomic on
                    // the count is one dependent step, a warp-aggregated append
                    // (vote, leader's atomic, shuffle) three
                    if (nd < hi && !(atomicOr(&bm_next[lu >> 5], bit) & bit))
                      wl_next[atomicAdd(n_next, 1u)] = (uint16_t)lu;
                  }
                  return;
                }
                if (ob_ok) {
                  const uint32_t pos = atomicAdd(on, 1u);
                  if (pos < kRegionOut) {
                    ob[pos] = make_uint2(u, nd);
                    return;
                  }
                }
                if (nd < atomicMin(&a.dist[u], nd)) {  // no room: applied here
                  ++my_relax;
                  if (nd < hi) region_touch(a, ra, u, &ctl->err);
                  else far_file(a, farq, far_count, u, nd, &s_fmin, &ctl->err);
                }
              };
              if constexpr (D == 0) {
                uint32_t j = live ? s_loff[v] + sub : 0u;
                const uint32_t e1 = live ? s_loff[v + 1] : 0u;
                for (; j < e1; j += 4) relax(true, s_col[j], d + s_w[j], true);
              } else {
                // lane sub takes slot sub of the vertex's row (D == 4: one each)
                static_assert(D == 4, "rows of 4 slots: one per lane of the group");
                const uint32_t u = s_col[v * D + sub];
                relax(live && u != kNoArc, u, d + s_w[v * D + sub], false);
              }
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kRegionRelax) : "memory");
            // uniform: s_n[(k + 1) % 3] changes only after the next barrier
            if (*n_next == 0) break;
          }
          if (warp == kBooks && lane == 0) {
            st_release_cta(&s_opub, k + 1);
            st_release_cta(&s_qreq, q);
          }
          ++k;  // the next round (if the visit goes on) starts from an empty list
        } else if (warp == kRegionRelax / 32) {
          // pending courier: a pass that starts after the request is the last
          const uint32_t pw0 = base >> 5;
          for (uint32_t pass = 1;; ++pass) {
            uint32_t qr = 0;
            if (lane == 0) qr = ld_acquire_cta(&s_qreq);
            qr = __shfl_sync(kFull, qr, 0);
            // a lane takes pending words lane, lane + 32, ...
            uint32_t bw[kRegion / 1024];
#pragma unroll
            for (uint32_t t = 0; t < kRegion / 1024; ++t) {
              const uint32_t w = lane + 32 * t;
              bw[t] = 0u;
              if (w < nw) {
                bw[t] = *reinterpret_cast<volatile uint32_t*>(&ra.pend[pw0 + w]);
                if (bw[t]) bw[t] = atomicExch(&ra.pend[pw0 + w], 0u);
              }
            }
            // no fence: the exchanges have returned, and a writer's atomicMin
            // had returned before it set the bit (region_touch)
            bool any = false;
            auto take_word = [&](uint32_t w, uint32_t bits) {
              bool want = false;
              if ((bits >> lane) & 1u) {
                const uint32_t i = w * 32 + lane;
                const uint32_t gd = __ldcg(a.dist + base + i);
                // a bit asks for an expansion at the global distance: also
                // when it equals the local one (read at the visit's start
                // after the bit was set); a smaller local one is expanded
                want = gd <= atomicMin(&s_dist[i], gd) && gd < hi;
              }
              const unsigned mk = __ballot_sync(kFull, want);
              if (mk) {
                any = true;
                if (lane == 0) atomicOr(&s_inbm[w], mk);
              }
            };
#pragma unroll
            for (uint32_t t = 0; t < kRegion / 1024; ++t)
              for (unsigned m = __ballot_sync(kFull, bw[t] != 0u); m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                take_word((uint32_t)src + 32 * t, __shfl_sync(kFull, bw[t], src));
              }
            if (any && lane == 0) st_release_cta(&s_in_any, 1u);
            if (qr == q) break;
            if ((pass & 63u) == 0 && globaltimer_ns() > deadline) {
              if (lane == 0) raise_err(&ctl->err, kDevTimeout);
              break;
            }
          }
        } else {
          // outbox courier: every published round at once, then the request
          for (uint32_t spins = 1;; ++spins) {
            uint32_t qr = 0, pub = 0;
            if (lane == 0) {
              qr = ld_acquire_cta(&s_qreq);
              pub = ld_acquire_cta(&s_opub);
            }
            qr = __shfl_sync(kFull, qr, 0);
            pub = __shfl_sync(kFull, pub, 0);
            if (jo < pub) {
              // rounds [jo, pub): at most kRegionOutBufs of them are unread
              // (a round uses its buffer only once the courier took it)
              uint32_t total = 0;
              uint32_t cum[kRegionOutBufs];
#pragma unroll
              for (uint32_t t = 0; t < kRegionOutBufs; ++t) {
                const uint32_t r = jo + t;
                const uint32_t c = r < pub ? min(*reinterpret_cast<volatile uint32_t*>(&s_on[r % kRegionOutBufs]), kRegionOut) : 0u;
                total += c;
                cum[t] = total;
              }
              for (uint32_t g = lane; g < total; g += 32) {
                uint32_t t = 0, first = 0;
#pragma unroll
                for (uint32_t x = 0; x + 1 < kRegionOutBufs; ++x)
                  if (g >= cum[x]) t = x + 1, first = cum[x];
                const uint2 o = s_out[((jo + t) % kRegionOutBufs) * kRegionOut + (g - first)];
                if (o.y < atomicMin(&a.dist[o.x], o.y)) {
                  ++my_relax;
                  if (o.y < hi) region_touch(a, ra, o.x, &ctl->err);
                  else far_file(a, farq, far_count, o.x, o.y, &s_fmin, &ctl->err);
                }
              }
              __syncwarp();
              const uint32_t nr = min(pub - jo, kRegionOutBufs);
              if (lane < nr) s_on[(jo + lane) % kRegionOutBufs] = 0;
              __syncwarp();
              jo += nr;
              if (lane == 0) st_release_cta(&s_odone, jo);
              continue;
            }
            if (qr == q) break;  // read before pub: every round published before the request is taken
            __nanosleep(32);
            if ((spins & 255u) == 0 && globaltimer_ns() > deadline) {
              if (lane == 0) raise_err(&ctl->err, kDevTimeout);
              break;
            }
          }
        }
        __syncthreads();
        const bool go = *reinterpret_cast<volatile uint32_t*>(&s_in_any) != 0u;
        __syncthreads();
        if (!go) break;
      }
      if (tid == 0) my_rounds += k;
      // write the lowered distances back (a thread's global distances read
      // at once); those beyond the bucket join the far pile
      {
        constexpr int kPer = kRegionPer;
        uint32_t gd[kPer];
#pragma unroll
        for (int t = 0; t < kPer; ++t) {
          const uint32_t i = tid + t * kRegionBlock;
          gd[t] = i < nv ? __ldcg(a.dist + base + i) : 0u;
        }
#pragma unroll
        for (int t = 0; t < kPer; ++t) {
          const uint32_t i = tid + t * kRegionBlock;
          const uint32_t d = i < nv ? s_dist[i] : 0u;
          if (d < gd[t] && d < atomicMin(&a.dist[base + i], d) && d >= hi)
            far_file(a, farq, far_count, base + i, d, &s_fmin, &ctl->err);
        }
      }
      __syncthreads();
      // release: vertices lowered from outside meanwhile queue the region again
      // the write-back atomics above have returned: the next visit's loads see them
      if (tid == 0) atomicExch(&ra.rq[r], 0u);
      __syncthreads();
      if (tid < 32) {
        bool any = false;
        for (uint32_t j = tid; j < nw; j += 32)
          any |= *reinterpret_cast<volatile uint32_t*>(&ra.pend[(base >> 5) + j]) != 0u;
        if (__any_sync(kFull, any) && tid == 0 && atomicCAS(&ra.rq[r], 0u, 1u) == 0u)
          worklists::publish_one(a.ring, make_uint4(r, 0u, 0u, 0u), &ctl->err);
      }
      __syncthreads();
    }
    // ---- bucket transition: two grid barriers -------------------------------------
    // The least bucket of the pile is recorded as entries are filed (and as
    // R2 keeps them): every entry's distance was recorded when it was set,
    // so the record is at most the least bucket still in the pile (a bucket
    // emptied since by lowerings only costs an empty bucket).
    if (tid == 0 && s_fmin != 0xFFFFFFFFu) {
      atomicMin(&ctl->far_min[fp], s_fmin);
      s_fmin = 0xFFFFFFFFu;
    }
    // the last CTA to arrive voids the tickets still waiting: no CTA waits any more
    if (!grid_barrier_last(&ctl->bar, gridDim.x, &ctl->err, deadline, [&] { rc->head = rc->tail; })) return;
    const uint32_t nfar = min(__ldcg(&ctl->far_count[fp]), a.n);
    ++P;
    if (nfar == 0) break;  // nothing left anywhere
    const uint32_t nb = __ldcg(&ctl->far_min[fp]);
    if (nb == 0xFFFFFFFFu) break;  // nothing recorded: every far entry was settled
    if (gtid == 0) ctl->buckets += 1;
    // R2: the entries of bucket nb become pending (their regions queued),
    // later ones stay in the pile (their buckets recorded for the next one)
    {
      const uint64_t nhi64 = ((uint64_t)nb + 1) << a.shift;
      const uint32_t nhi = nhi64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)nhi64;
      uint32_t* keepq = a.far[fp ^ 1];
      uint32_t kmin = 0xFFFFFFFFu;
      for (uint64_t b0 = gtid - lane; b0 < nfar; b0 += gthreads) {
        const uint64_t i = b0 + lane;
        bool keep = false;
        uint32_t u = 0;
        if (i < nfar) {
          u = farq[i];
          const uint32_t dd = __ldcg(a.dist + u);
          if (dd >= hi && dd < nhi) region_touch(a, ra, u, &ctl->err);
          else if (dd >= nhi) keep = true, kmin = min(kmin, dd >> a.shift);
          if (!keep) atomicAnd(&a.infar[u >> 5], ~(1u << (u & 31)));
        }
        warp_push(keep, u, keepq, &ctl->far_count[fp ^ 1], a.n, &ctl->err);
      }
      kmin = __reduce_min_sync(kFull, kmin);
      if (lane == 0 && kmin != 0xFFFFFFFFu) atomicMin(&s_fmin, kmin);
    }
    // the last CTA to arrive empties the pile just split
    const int done_pile = fp;
    if (!grid_barrier_last(&ctl->bar, gridDim.x, &ctl->err, deadline, [&] {
          ctl->far_count[done_pile] = 0;
          ctl->far_min[done_pile] = 0xFFFFFFFFu;
        }))
      return;
    bucket = nb;
    fp ^= 1;
  }
  my_scanned = warp_sum(my_scanned);
  my_relax = warp_sum(my_relax);
  if (lane == 0) {
    if (my_scanned) atomicAdd(&ctl->scanned, my_scanned);
    if (my_relax) atomicAdd(&ctl->relax, my_relax);
  }
  if (tid == 0 && my_rounds) atomicAdd(&ctl->local_rounds, my_rounds);
  if (gtid == 0) ctl->phases = (uint32_t)min(rc->chunks + 1, 0xFFFFFFFFull);  // region visits
}

__global__ void sssp_reach_kernel(const uint32_t* __restrict__ dist, const uint64_t* __restrict__ offs,
                                  uint32_t n, unsigned long long* out) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long nr = 0, mr = 0;
  for (uint64_t v = tid; v < n; v += stride) {
    if (dist[v] != kInf) {
      nr += 1;
      mr += offs[v + 1] - offs[v];
    }
  }
  nr = warp_sum(nr);
  mr = warp_sum(mr);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, nr);
    atomicAdd(out + 1, mr);
  }
}

}  // namespace

// Error word, statistics and the host copy of the distances after the
// persistent kernel.
static int finish_sssp(gb_graph* g, const SsspArgs& a, unsigned long long* reach, const KernelTimer& kt, uint32_t launches,
                uint32_t* dist_out, bool out_dev, gb_stats* stats, cudaStream_t s) {
  const uint32_t n = g->n;
  int* pin = static_cast<int*>(g->pinned);
  GB_CUDA(cudaMemcpyAsync(pin, &a.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (stats) {
    GB_CUDA(cudaMemsetAsync(reach, 0, 16, s));
    sssp_reach_kernel<<<g->sm_count * 4, 256, 0, s>>>(a.dist, g->offs, n, reach);
    SsspCtl* hc = reinterpret_cast<SsspCtl*>(static_cast<char*>(g->pinned) + 256);
    unsigned long long* hr = reinterpret_cast<unsigned long long*>(static_cast<char*>(g->pinned) + 2048);
    GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(SsspCtl), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(hr, reach, 16, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    *stats = gb_stats{};
    stats->vertices_reached = hr[0];
    stats->edges_reached = hr[1];
    stats->edges_scanned = hc->scanned;
    stats->relaxations = hc->relax;
    stats->rounds = hc->phases;
    stats->pull_rounds = (uint32_t)min(hc->local_rounds, 0xFFFFFFFFull);
    stats->buckets = hc->buckets + 1;
    stats->launches = launches;
    stats->kernel_ms = kt.ms();
  }
  if (!out_dev) {
    int st = copy_out(dist_out, a.dist, sizeof(uint32_t) * n, s);
    if (st != GB_OK) return st;
  }
  if (stats || !out_dev) {
    GB_CUDA(cudaStreamSynchronize(s));
    if (*pin) return dev_err_status(*pin, "gb_sssp_delta");
  }
  return GB_OK;
}

// The region kernel (every region's arcs fit in shared memory).
static int run_sssp_region(gb_graph* g, uint32_t src, uint32_t shift, uint32_t nregions,
                           uint32_t* dist_out, bool out_dev, gb_stats* stats, cudaStream_t s) {
  const uint32_t n = g->n;
  const uint32_t words = (n + 31) / 32;
  // each region is queued at most once at a time
  const unsigned long long cap = worklists::ring_capacity((uint64_t)nregions + 1024);
  const size_t need = carve_size<SsspCtl>(1) + 2 * carve_size<uint32_t>(words) + 2 * carve_size<uint32_t>(n) +
                      (out_dev ? 0 : carve_size<uint32_t>(n)) + carve_size<unsigned long long>(2) +
                      carve_size<uint32_t>(nregions) + carve_size<char>(worklists::ring_bytes(cap));
  int st = ws_reserve(g, need, s);
  if (st != GB_OK) return st;
  Carver cv(g->ws);
  SsspArgs a{};
  RegionArgs ra{};
  a.ctl = cv.take<SsspCtl>(1);
  a.infar = cv.take<uint32_t>(words);
  a.far[0] = cv.take<uint32_t>(n);
  a.far[1] = cv.take<uint32_t>(n);
  unsigned long long* reach = cv.take<unsigned long long>(2);
  a.dist = out_dev ? dist_out : cv.take<uint32_t>(n);
  ra.pend = cv.take<uint32_t>(words);
  ra.rq = cv.take<uint32_t>(nregions);
  ra.nregions = nregions;
  a.ring = worklists::ring_layout(cv.take<char>(worklists::ring_bytes(cap)), cap);
  a.offs = g->offs;
  a.col = g->col;
  a.w = g->w;
  a.n = n;
  a.src = src;
  a.shift = shift;
  a.max_phases = 0x7FFFFFFFu;
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(SsspCtl), s));
  GB_CUDA(cudaMemsetAsync(a.ring.rc, 0, sizeof(worklists::RingCtl), s));
  sssp_region_init<<<g->sm_count * 4, 256, 0, s>>>(a, ra);
  GB_CUDA(cudaGetLastError());
  // graphs of degree <= 4 keep their arcs as 4-slot rows in shared memory
  const bool rows = g->max_degree <= 4;
  const void* kfn = rows ? reinterpret_cast<const void*>(&sssp_region<4>) : reinterpret_cast<const void*>(&sssp_region<0>);
  const size_t smem = rows ? region_smem_bytes<4>() : region_smem_bytes<0>();
  GB_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = coop_grid(g, kfn, kRegionBlock, smem, kRegionPerSm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_sssp_delta: cannot size cooperative grid");
  void* args[] = {&a, &ra};
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, kRegionBlock, args, smem, s));
  kt.stop(s);
  return finish_sssp(g, a, reach, kt, 2, dist_out, out_dev, stats, s);
}

int run_sssp(gb_graph* g, uint32_t src, uint32_t shift, uint32_t* dist_out, gb_stats* stats,
             cudaStream_t s) {
  if (!g->w) GB_FAIL(GB_ERR_ARG, "gb_sssp_delta: graph has no uint32 edge weights");
  if (shift > 31) GB_FAIL(GB_ERR_ARG, "gb_sssp_delta: delta shift %u > 31", shift);
  const gb_tuning t = effective_tuning(g);
  const uint32_t n = g->n;
  const uint32_t words = (n + 31) / 32;
  const bool out_dev = is_device_ptr(dist_out);
  const int local_depth = t.local_depth < 0 ? 0 : t.local_depth;
  // asynchronous buckets (asked for): local queues on and every vertex
  // light (entries pack the degree in 16 bits and the begin offset in 48)
  const bool async = t.sssp_async > 0 && local_depth > 0 && g->max_degree <= t.heavy_degree &&
                     g->max_degree < 65536 && g->m < (1ull << 48);
  // regions in shared memory: asked for (sssp_async 3: whenever every
  // region's arcs fit), or by default on a graph numbered by locality whose
  // regions fit and keep at least 90 % of the arcs inside (measured on the
  // 4096^2 grid: 29.3 ms against 38.5 ms for the phase-synchronous kernel)
  bool region = false;
  const uint32_t nregions = (uint32_t)(((uint64_t)n + kRegion - 1) / kRegion);
  if (t.sssp_async == 3 || (t.sssp_async == 0 && g->order == GB_ORDER_LOCALITY)) {
    if (!g->region_arcs) {  // once per graph (and after a relabelling)
      int rst = ws_reserve(g, 256, s);
      if (rst != GB_OK) return rst;
      unsigned long long* dout = static_cast<unsigned long long*>(g->ws);
      unsigned long long* hout = static_cast<unsigned long long*>(g->pinned);
      GB_CUDA(cudaMemsetAsync(dout, 0, 2 * sizeof(unsigned long long), s));
      region_arcs_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, g->col, n, nregions, dout);
      GB_CUDA(cudaGetLastError());
      GB_CUDA(cudaMemcpyAsync(hout, dout, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
      GB_CUDA(cudaStreamSynchronize(s));
      g->region_arcs = hout[0] + 1;
      g->region_local = g->m ? (double)hout[1] / (double)g->m : 1.0;
    }
    const bool fits = g->region_arcs - 1 <= kRegionArcs;
    region = t.sssp_async == 3 ? fits : fits && g->region_local >= 0.9;
  }
  if (region) return run_sssp_region(g, src, shift, nregions, dist_out, out_dev, stats, s);
  FrontierLayout fl = frontier_layout(n, g->m, t.heavy_degree, t.tile_edges);
  SweepSched sched{};
  if (!async && g->max_degree > t.heavy_degree) {  // heavy rows of a bitmap frontier come from the tile schedule
    int sst = ensure_sweep_schedule(g, t.heavy_degree, t.tile_edges, s, &sched);
    if (sst != GB_OK) return sst;
  }
  // worklist ring: a bucket's split fills at most one chunk per 32 far
  // entries, the warps' overflow only full chunks
  const unsigned long long cap = worklists::ring_capacity((uint64_t)n / 16 + 8192);
  size_t need = carve_size<SsspCtl>(1) + carve_size<uint32_t>(words) + 2 * carve_size<uint32_t>(n) +
                (out_dev ? 0 : carve_size<uint32_t>(n)) + carve_size<unsigned long long>(2);
  if (async) need += carve_size<char>(worklists::ring_bytes(cap));
  else
    need += carve_size<uint32_t>(n) + 3 * carve_size<uint32_t>(words) + fl.bytes;
  int st = ws_reserve(g, need, s);
  if (st != GB_OK) return st;
  Carver cv(g->ws);
  SsspArgs a{};
  a.ctl = cv.take<SsspCtl>(1);
  a.infar = cv.take<uint32_t>(words);
  a.far[0] = cv.take<uint32_t>(n);
  a.far[1] = cv.take<uint32_t>(n);
  unsigned long long* reach = cv.take<unsigned long long>(2);
  a.dist = out_dev ? dist_out : cv.take<uint32_t>(n);
  if (async) {
    a.ring = worklists::ring_layout(cv.take<char>(worklists::ring_bytes(cap)), cap);
  } else {
    a.stamp = cv.take<uint32_t>(n);
    for (int i = 0; i < 3; ++i) a.act[i] = cv.take<uint32_t>(words);
    a.fq = carve_frontier(cv, fl);
  }
  a.offs = g->offs;
  a.col = g->col;
  a.w = g->w;
  a.n = n;
  a.src = src;
  a.shift = shift;
  a.heavy = t.heavy_degree;
  a.tile = t.tile_edges;
  a.max_phases = 0x7FFFFFFFu;
  a.local_depth = local_depth;
  a.all_light = g->max_degree <= t.heavy_degree ? 1 : 0;
  a.sw_tiles = sched.tiles;
  a.sw_ntiles = sched.ntiles;
  // a frontier estimated at more than n/256 arcs writes the next one as a
  // bitmap: its sweep reads n/8 bytes of bitmap and the tile schedule, small
  // beside what such a frontier relaxes (n/64 and n/1024 measured slower on
  // RMAT-22/24)
  a.bm_min = n >> 8;
  if (async) {
    GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(SsspCtl), s));
    GB_CUDA(cudaMemsetAsync(a.ring.rc, 0, sizeof(worklists::RingCtl), s));
    sssp_async_init<<<g->sm_count * 4, 256, 0, s>>>(a);
    GB_CUDA(cudaGetLastError());
    // sssp_async 2: fixed-width rows on a graph of degree <= 8
    const uint32_t D = t.sssp_async == 2 && g->max_degree <= 8 ? (g->max_degree <= 4 ? 4u : 8u) : 0u;
    const uint32_t* ell = nullptr;
    if (D) {
      if (!g->ell || g->ell_d != D) {
        cudaFree(g->ell);
        g->ell = nullptr;
        g->ell_d = 0;
        GB_CUDA(cudaMalloc(&g->ell, sizeof(uint32_t) * 2 * (uint64_t)n * D));
        ell_build_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, g->col, g->w, n, D, g->ell);
        GB_CUDA(cudaGetLastError());
        g->ell_d = D;
      }
      ell = g->ell;
    }
    const void* kfn = D == 4   ? reinterpret_cast<const void*>(&sssp_async_ell<256, 4>)
                      : D == 8 ? reinterpret_cast<const void*>(&sssp_async_ell<256, 8>)
                               : reinterpret_cast<const void*>(&sssp_async<256>);
    const int grid = coop_grid(g, kfn, 256, 0, t.blocks_per_sm);
    if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_sssp_delta: cannot size cooperative grid");
    void* args[] = {&a, &ell};
    KernelTimer kt(stats != nullptr, s);
    GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, 256, args, 0, s));
    kt.stop(s);
    return finish_sssp(g, a, reach, kt, 2, dist_out, out_dev, stats, s);
  }
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(SsspCtl), s));
  sssp_init<<<g->sm_count * 4, 256, 0, s>>>(a);
  GB_CUDA(cudaGetLastError());
  // local queues serve small frontiers; only without them can a frontier
  // grow large enough for the bitmap
  const bool bm = a.local_depth == 0;
  // CTA size: as tuned, else 1024 threads for the bitmap kernel (at 256 it
  // needs 117 registers, two CTAs per SM) and 256 for the queue-only one
  // (4096^2 grid 1.5-2 % faster than with 1024 at every local depth)
  const bool big = g->tuning.block_threads ? t.block_threads >= 1024 : bm;
  const int block = big ? 1024 : 256;
  const void* kfn = big ? (bm ? reinterpret_cast<const void*>(&sssp_persistent<1024, true>)
                              : reinterpret_cast<const void*>(&sssp_persistent<1024, false>))
                        : (bm ? reinterpret_cast<const void*>(&sssp_persistent<256, true>)
                              : reinterpret_cast<const void*>(&sssp_persistent<256, false>));
  const int grid = coop_grid(g, kfn, block, 0, t.blocks_per_sm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_sssp_delta: cannot size cooperative grid");
  void* args[] = {&a};
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, block, args, 0, s));
  kt.stop(s);
  return finish_sssp(g, a, reach, kt, 2, dist_out, out_dev, stats, s);
}

}  // namespace gb

extern "C" int gb_sssp_delta(gb_graph* g, uint32_t src, uint32_t delta_shift, uint32_t* dist_out,
                             gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !dist_out) GB_FAIL(GB_ERR_ARG, "gb_sssp_delta: null argument");
  if (src >= g->n) GB_FAIL(GB_ERR_ARG, "gb_sssp_delta: source %u >= n %u", src, g->n);
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g->perm) {
    gb_stats local{};
    uint32_t* res = gb::result_buf(g, 0);
    int st = gb::run_sssp(g, g->h_iperm[src], delta_shift, res,
                          stats ? stats : (gb::is_device_ptr(dist_out) ? nullptr : &local), s);
    if (st != GB_OK) return st;
    if (stats) stats->launches += 1;  // the mapping gather
    return gb::finish_u32(g, res, dist_out, s);
  }
  return gb::run_sssp(g, src, delta_shift, dist_out, stats, s);
}
