// PageRank: pull-topological, pull-residual and residual-push.
//
// Reference semantics (lonestar/analytics/cpu/pagerank):
//   pull-topological  PageRank-pull.cpp:196-251 over the TRANSPOSED graph:
//                     value = 1/n; nout = in-degree of the stored graph
//                     (computeOutDeg :90-122); per iteration
//                     value[v] = alpha * sum_{u in edges(v)} value[u]/nout[u]
//                                + (1-alpha)/n,
//                     stop when sum |delta| <= tol or at maxIterations.
//                     The CPU code updates in place (schedule-dependent); the
//                     device runs the Jacobi form, which the FP64 oracle
//                     restates.
//   pull-residual     PageRank-pull.cpp:132-190 (delta/residual rounds).
//   residual push     PageRank-push.cpp:103-188 (Sync): value 0, residual
//                     1-alpha; active vertices over tol absorb their residual
//                     and push residual*alpha/outdeg along out-edges; a
//                     vertex is activated when its residual crosses tol.
//                     PageRank-push.cpp:68-101 (Async, the app's default):
//                     the same operator over a worklist with no rounds -- a
//                     vertex is processed when it is taken, absorbing the
//                     residual accumulated until then (exchange with 0), and
//                     pushed again when an add lifts its residual from below
//                     tol to tol or above.
//
// B200 design: one cooperative persistent launch per solve.  Pull iterations
// use the cached all-vertex sweep schedule (sweep.cuh): 32 consecutive
// vertices per warp with a segmented shuffle reduction per owner vertex,
// heavy vertices as tiles whose partial sums meet in an accumulator, a
// contribution array c[u] = value[u]/nout[u] (SoA, double-buffered) so each
// arc costs one 4-byte column read and one 4-byte gather, and the L1 change
// reduced in fp64.  On a degree-ordered graph pull-topological runs over a
// binned layout instead (pr_pull_binned, below).  Residual push (Sync) reuses the frontier queues
// (frontier.cuh); Async runs over the device worklist (gb_worklist.cuh): a
// warp keeps working on the vertices it activated itself, surplus goes to
// the ring, and the launch ends when the worklist's work count reaches zero.

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "device_common.cuh"
#include "device_graph.cuh"
#include "frontier.cuh"
#include "gb_worklist.cuh"
#include "sweep.cuh"

#include <cstring>

// The binned layout of a degree-ordered graph's arcs for the PageRank pull
// (pr_pull_binned): one device allocation, cached in the graph handle.
struct PrBins {
  void* mem = nullptr;
  uint16_t* dst = nullptr;
  uint8_t* roff = nullptr;
  uint32_t* crun = nullptr;
  uint32_t* rsrc = nullptr;  // per run: its source
  uint4* tasks = nullptr;
  uint32_t ntasks = 0;
  uint64_t npairs = 0, nchunks = 0;
};

namespace gb {

void free_pr_bins(gb_graph* g) {
  if (!g->prb) return;
  cudaFree(g->prb->mem);
  delete g->prb;
  g->prb = nullptr;
}

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kL1Slots = 32;  // the per-iteration L1 sum is spread over this many words

struct PrCtl {
  GridBar bar;
  int err;
  uint32_t iters;
  double l1[3][kL1Slots];  // per-iteration L1 change, one slot per (CTA % kL1Slots)
  uint32_t linf[3];        // max |delta| as float bits (non-negative floats order as uints)
  uint32_t active[3];
  uint32_t pad;
  FrontierCounters fc[3];
  unsigned long long pushes;
  unsigned long long absorbs;  // Async push: residuals taken
  uint32_t task_next[2];       // binned pull: next gather task (iteration parity)
};

struct PrArgs {
  const uint64_t* __restrict__ offs;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ nout;
  uint32_t n;
  float alpha;
  float base;
  float tol;
  uint32_t max_iter;
  float init;  // initial rank (1/n for the lonestar app)
  int linf;    // 1: stop on max |delta| (python/galois/_pagerank.pyx:114-139)
  float* value;
  float* c[2];
  float* acc;   // per-row partial sums of heavy rows (and flat-swept light rows)
  float* acc2;  // the alternate accumulator (pull kernels): iteration it adds into
                // (it & 1 ? acc2 : acc) and zeroes the other; a plain store to a
                // word the same iteration's atomics just updated stalled (~0.4 ms
                // for 9 M words at RMAT-24), one iteration later it does not
  SweepSched sched;
  PrCtl* ctl;
  // residual variants
  float* residual;
  float* delta;
  uint32_t* active[2];
  uint32_t* stamp;
  FrontierQueues fq;
  uint32_t heavy, tile;
  worklists::Ring ring;  // Async push: the worklist ring
  uint32_t zero_from;  // first vertex of the no-in-arc suffix (degree-ordered graphs), else n
  // flat sweep of the light rows (degree-ordered graphs): arcs [lr_arc0,
  // lr_arc1) in runs of kLightRun; an arc's row is lr_runrow[run] +
  // lr_rowd[arc - lr_arc0] (a run spans at most kLightRun rows, so the
  // offset fits a byte: a quarter of the bytes of a row id per arc)
  const uint32_t* __restrict__ lr_runrow;
  const uint8_t* __restrict__ lr_rowd;
  uint64_t lr_arc0, lr_arc1;
  // binned pull (degree-ordered graphs, pr_pull_binned)
  const uint16_t* __restrict__ b_dst;   // per padded arc: destination - partition base (0xFFFF: padding)
  const uint8_t* __restrict__ b_roff;   // per padded arc: its run - the chunk's first run
  const uint32_t* __restrict__ b_crun;  // per 256-arc chunk: its first run
  const uint32_t* __restrict__ b_rsrc;  // per run: its source
  const uint4* __restrict__ b_tasks;    // (partition base, vertices | multi << 31, chunk begin, chunk end)
  uint32_t b_ntasks;
};

constexpr int kLightRun = 256;  // arcs per light-row run of pr_pull_flat (32 lanes x 8)

__global__ void count_nout(const uint32_t* __restrict__ col, uint64_t m, uint32_t* nout) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = tid; e < m; e += stride) atomicAdd(&nout[col[e]], 1u);
}

__global__ void pr_pull_init(PrArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const float init = a.init;  // 1/n: PageRank-pull.cpp:62
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.value[v] = init;
    const uint32_t k = a.nout[v];
    a.c[0][v] = k ? init / (float)k : 0.f;
    a.acc[v] = 0.f;
    a.acc2[v] = 0.f;
  }
}

// Segmented (by owner lane) warp reduction of x; returns true on the lane
// that heads its segment, which then holds the segment's sum.
__device__ __forceinline__ bool seg_reduce(bool valid, uint32_t owner, float& x) {
  const uint32_t lane = lane_id();
  const uint32_t key = valid ? owner : 0xFFFFFFFFu;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const float y = __shfl_down_sync(kFull, x, off);
    const uint32_t k2 = __shfl_down_sync(kFull, key, off);
    if (lane + off < 32 && k2 == key) x += y;
  }
  const uint32_t kprev = __shfl_up_sync(kFull, key, 1);
  return valid && (lane == 0 || kprev != key);
}

// Jacobi pull iterations, one cooperative persistent launch.  Shared memory
// is kept small (one float per lane) so that the SM's unified L1/shared array
// serves as L1 for the gathers; on a degree-ordered graph the hot
// contributions sit on few lines and stay there.  On such a graph the
// vertices from zero_from on have no in-arcs, so after two iterations their
// rank and contribution are constants and their chunks are skipped.
// Publish this thread's share of the iteration's L1 / max change: summed per
// CTA in shared memory, then one atomic per CTA into one of kL1Slots words
// (an atomic per warp on one word serialised ~7 K atomics per iteration), the
// max with a read before the atomic.  All threads of the CTA call.
__device__ __forceinline__ void publish_change(PrCtl* ctl, uint32_t slot_set, double my_l1, float my_max,
                                               double* s_l1, uint32_t* s_max) {
  my_l1 = warp_sum(my_l1);
  const uint32_t mbits = __reduce_max_sync(kFull, __float_as_uint(my_max));
  if (lane_id() == 0) {
    if (my_l1 != 0.0) atomicAdd(s_l1, my_l1);
    if (mbits != 0u) atomicMax(s_max, mbits);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (*s_l1 != 0.0) atomicAdd(&ctl->l1[slot_set][blockIdx.x % kL1Slots], *s_l1);
    if (*s_max > *reinterpret_cast<volatile uint32_t*>(&ctl->linf[slot_set])) atomicMax(&ctl->linf[slot_set], *s_max);
    *s_l1 = 0.0;
    *s_max = 0u;
  }
}

// The iteration's change after the barrier that follows publish_change: one
// thread per CTA reads the slots and shares the total through shared memory
// (every thread reading them would hammer the same L2 lines).  All threads
// of the CTA call.
__device__ __forceinline__ double read_change(const PrCtl* ctl, uint32_t slot_set, int linf, double* s_total) {
  if (threadIdx.x == 0) {
    double v = 0.0;
    if (linf) {
      v = (double)__uint_as_float(*reinterpret_cast<const volatile uint32_t*>(&ctl->linf[slot_set]));
    } else {
      for (int k = 0; k < kL1Slots; ++k) v += *reinterpret_cast<const volatile double*>(&ctl->l1[slot_set][k]);
    }
    *s_total = v;
  }
  __syncthreads();
  const double v = *s_total;
  __syncthreads();  // s_total is rewritten next iteration
  return v;
}

// Zero the slots of iteration it+1 (by one thread, before that iteration's barrier).
__device__ __forceinline__ void clear_change(PrCtl* ctl, uint32_t slot_set) {
  for (int k = 0; k < kL1Slots; ++k) ctl->l1[slot_set][k] = 0.0;
  ctl->linf[slot_set] = 0u;
}

template <int BLOCK, int U, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) pr_pull_persistent(PrArgs a) {
  constexpr int kW = BLOCK / 32;
  __shared__ float s_acc[kW][32];
  __shared__ double s_l1, s_total;
  __shared__ uint32_t s_max;
  if (threadIdx.x == 0) {
    s_l1 = 0.0;
    s_max = 0u;
  }
  __syncthreads();
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  s_acc[wib][lane] = 0.f;
  __syncwarp();
  for (uint32_t it = 0;; ++it) {
    const float* __restrict__ c_in = a.c[it & 1];
    float* __restrict__ c_out = a.c[(it + 1) & 1];
    float* const acc_cur = (it & 1) ? a.acc2 : a.acc;
    float* const acc_nxt = (it & 1) ? a.acc : a.acc2;
    if (gtid == 0) clear_change(ctl, (it + 1) % 3);
    auto gather = [&](uint32_t u) -> float { return c_in[u]; };
    double my_l1 = 0.0;
    float my_max = 0.f;
    auto finish = [&](uint32_t v, float sum) {
      const float value = sum * a.alpha + a.base;  // PageRank-pull.cpp:222
      const float old = a.value[v];
      a.value[v] = value;
      const uint32_t k = a.nout[v];
      c_out[v] = k ? value / (float)k : 0.f;
      my_l1 += (double)fabsf(value - old);
      my_max = fmaxf(my_max, fabsf(value - old));
    };
    // Tasks: 32-vertex chunks (warp expansion, U steps of loads in flight;
    // a chunk without arcs only finishes its vertices), then heavy-vertex
    // tiles (sweep.cuh's decomposition).
    const uint64_t nchunks = ((uint64_t)(it >= 2 ? a.zero_from : a.n) + 31) >> 5;  // constant tail skipped
    const uint64_t total = nchunks + a.sched.ntiles;
    for (uint64_t t = gwarp; t < total; t += nwarps) {
      if (t < nchunks) {
        const uint64_t v = (t << 5) + lane;
        uint64_t b = 0;
        uint32_t d = 0;
        bool heavy = false;
        if (v < a.n) {
          b = ldg(a.offs + v);
          const uint64_t dd = ldg(a.offs + v + 1) - b;
          heavy = dd > a.sched.heavy;
          d = heavy ? 0u : (uint32_t)dd;
        }
        const uint32_t dmax = __reduce_max_sync(kFull, d);
        if (dmax == 0) {
          if (v < a.n && !heavy) finish((uint32_t)v, 0.f);
        } else {
          // U steps of (column id, contribution) loads in flight per lane
          warp_expand_mlp<U, float>(
              b, d, (uint32_t)v, [&](bool valid, uint64_t e, uint32_t) { return valid ? ldg(a.col + e) : 0u; },
              [&](bool valid, uint64_t, uint32_t u, uint32_t) { return valid ? gather(u) : 0.f; },
              [&](bool valid, uint32_t owner, uint32_t, uint32_t, float x) {
                if (seg_reduce(valid, owner, x)) s_acc[wib][owner] += x;
                __syncwarp();
              });
          const float sum = s_acc[wib][lane];
          s_acc[wib][lane] = 0.f;
          __syncwarp();
          if (v < a.n && !heavy) finish((uint32_t)v, sum);
        }
      } else {
        // one tile of a heavy row: 8 column loads per lane per round, the
        // next round's loads issued before this round's gathers are summed
        const uint2 tv = a.sched.tiles[t - nchunks];
        const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
        const uint64_t b = vb + (uint64_t)tv.y * a.sched.tile;
        const uint64_t e = min(ve, b + a.sched.tile);
        constexpr int UT = 8;
        uint32_t u[UT];
#pragma unroll
        for (int k = 0; k < UT; ++k) {
          const uint64_t i = b + lane + 32 * k;
          u[k] = i < e ? ldg(a.col + i) : 0xFFFFFFFFu;
        }
        float sum = 0.f;
        for (uint64_t i0 = b; i0 < e; i0 += 32 * UT) {
          uint32_t un[UT];
#pragma unroll
          for (int k = 0; k < UT; ++k) {
            const uint64_t i = i0 + 32 * UT + lane + 32 * k;
            un[k] = i < e ? ldg(a.col + i) : 0xFFFFFFFFu;
          }
#pragma unroll
          for (int k = 0; k < UT; ++k) sum += u[k] != 0xFFFFFFFFu ? gather(u[k]) : 0.f;
#pragma unroll
          for (int k = 0; k < UT; ++k) u[k] = un[k];
        }
        sum = warp_sum(sum);
        if (lane == 0) atomicAdd(&acc_cur[tv.x], sum);
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    for (uint64_t i = gtid; i < a.sched.nheavy; i += gthreads) {
      const uint32_t v = a.sched.heavy_list[i];
      const float sum = acc_cur[v];
      acc_nxt[v] = 0.f;
      finish(v, sum);
    }
    publish_change(ctl, it % 3, my_l1, my_max, &s_l1, &s_max);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    const double l1 = read_change(ctl, it % 3, a.linf, &s_total);
    if (gtid == 0) ctl->iters = it + 1;
    if (l1 <= (double)a.tol || it + 1 >= a.max_iter) break;  // PageRank-pull.cpp:238-243
  }
}

// Jacobi pull iterations for a degree-ordered graph.  Its heavy rows are the
// ids [0, nheavy) and its light rows follow with falling degree, so the light
// rows' arcs form one contiguous range.  That range is swept flat, like a
// tile: 256 arcs per warp task, 8 column ids and 8 row ids per lane loaded
// together, 8 gathers in flight, a segmented warp sum per 32 arcs and one
// atomicAdd per row segment into acc.  Heavy rows keep their tiles.  A
// coalesced pass over the vertices then finishes every row from acc (rows
// from zero_from on have no in-arcs: constant after two iterations, skipped).
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) pr_pull_flat(PrArgs a) {
  __shared__ double s_l1, s_total;
  __shared__ uint32_t s_max;
  if (threadIdx.x == 0) {
    s_l1 = 0.0;
    s_max = 0u;
  }
  __syncthreads();
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  constexpr int UT = 8;
  const uint64_t nruns = (a.lr_arc1 - a.lr_arc0 + 32 * UT - 1) / (32 * UT);
  const uint64_t total = (uint64_t)a.sched.ntiles + nruns;
  for (uint32_t it = 0;; ++it) {
    const float* __restrict__ c_in = a.c[it & 1];
    float* __restrict__ c_out = a.c[(it + 1) & 1];
    float* const acc_cur = (it & 1) ? a.acc2 : a.acc;
    float* const acc_nxt = (it & 1) ? a.acc : a.acc2;
    if (gtid == 0) clear_change(ctl, (it + 1) % 3);
    for (uint64_t t = gwarp; t < total; t += nwarps) {
      if (t < a.sched.ntiles) {
        // one tile of a heavy row (as in pr_pull_persistent)
        const uint2 tv = a.sched.tiles[t];
        const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
        const uint64_t b = vb + (uint64_t)tv.y * a.sched.tile;
        const uint64_t e = min(ve, b + a.sched.tile);
        uint32_t u[UT];
#pragma unroll
        for (int k = 0; k < UT; ++k) {
          const uint64_t i = b + lane + 32 * k;
          u[k] = i < e ? ldg(a.col + i) : 0xFFFFFFFFu;
        }
        float sum = 0.f;
        for (uint64_t i0 = b; i0 < e; i0 += 32 * UT) {
          uint32_t un[UT];
#pragma unroll
          for (int k = 0; k < UT; ++k) {
            const uint64_t i = i0 + 32 * UT + lane + 32 * k;
            un[k] = i < e ? ldg(a.col + i) : 0xFFFFFFFFu;
          }
#pragma unroll
          for (int k = 0; k < UT; ++k) sum += u[k] != 0xFFFFFFFFu ? c_in[u[k]] : 0.f;
#pragma unroll
          for (int k = 0; k < UT; ++k) u[k] = un[k];
        }
        sum = warp_sum(sum);
        if (lane == 0) atomicAdd(&acc_cur[tv.x], sum);
      } else {
        // one run of 256 arcs of the light rows
        static_assert(32 * UT == kLightRun, "a light run is one warp step of UT arcs per lane");
        const uint64_t run = t - a.sched.ntiles;
        const uint64_t r0 = a.lr_arc0 + run * kLightRun;
        const uint32_t row0 = ldg(a.lr_runrow + run);
        uint32_t u[UT], row[UT];
#pragma unroll
        for (int k = 0; k < UT; ++k) {
          const uint64_t i = r0 + lane + 32 * k;
          const bool ok = i < a.lr_arc1;
          u[k] = ok ? ldg(a.col + i) : 0u;
          row[k] = ok ? row0 + (uint32_t)__ldg(a.lr_rowd + (i - a.lr_arc0)) : 0xFFFFFFFFu;
        }
        float x[UT];
#pragma unroll
        for (int k = 0; k < UT; ++k) x[k] = row[k] != 0xFFFFFFFFu ? c_in[u[k]] : 0.f;
#pragma unroll
        for (int k = 0; k < UT; ++k) {
          if (seg_reduce(row[k] != 0xFFFFFFFFu, row[k], x[k])) atomicAdd(&acc_cur[row[k]], x[k]);
        }
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    double my_l1 = 0.0;
    float my_max = 0.f;
    const uint32_t vend = it >= 2 ? a.zero_from : a.n;  // constant tail skipped
    for (uint64_t v = gtid; v < vend; v += gthreads) {
      const float sum = acc_cur[v];
      acc_nxt[v] = 0.f;
      const float value = sum * a.alpha + a.base;  // PageRank-pull.cpp:222
      const float old = a.value[v];
      a.value[v] = value;
      const uint32_t k = a.nout[v];
      c_out[v] = k ? value / (float)k : 0.f;
      my_l1 += (double)fabsf(value - old);
      my_max = fmaxf(my_max, fabsf(value - old));
    }
    publish_change(ctl, it % 3, my_l1, my_max, &s_l1, &s_max);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    const double l1 = read_change(ctl, it % 3, a.linf, &s_total);
    if (gtid == 0) ctl->iters = it + 1;
    if (l1 <= (double)a.tol || it + 1 >= a.max_iter) break;  // PageRank-pull.cpp:238-243
  }
}

// ---- binned pull (degree-ordered graphs) --------------------------------------
// The destinations are cut into partitions of kBinPart consecutive ids, few
// enough that a partition's sums fit in shared memory.  Inside a partition
// the in-arcs are ordered by source, so the arcs from one source form a run;
// the arcs are stored in 256-arc chunks (per arc a 2-byte local destination
// and a 1-byte offset of its run from the chunk's first run, the chunk's arcs
// sorted by destination), and per run its source.  Per iteration
//   gather: a CTA takes a task (a range of chunks of one partition), streams
//     the chunks, reads each run's source and that source's contribution
//     (the contributions, 4 bytes per vertex, stay mostly in L2), sums equal
//     destinations of a lane's 8 arcs in registers and adds them into the
//     partition's sums in shared memory, then writes the sums out (added
//     with atomics when the partition has several tasks);
//   finish: per vertex the new rank and its contribution (coalesced).
// Against the row sweep, an arc costs 3 streamed bytes instead of a 4-byte
// column and a 4-byte random gather, and one contribution is gathered per
// run instead of per arc (0.16 runs per arc on RMAT graphs in degree order
// at 4 M vertices).  Measured on RMAT-24: 18.9 ms for 15 iterations against
// 29.3 ms for pr_pull_flat.  Variants that wrote each contribution into the
// slots of its runs (so the gather read them sequentially) were slower
// (23-35 ms): the scattered 4-byte writes into a 0.5 GB array cost more than
// the gathers from the L2-resident contributions.

constexpr uint32_t kBinPart = 32768;  // destinations per partition (a local id fits 15 bits)
constexpr uint32_t kBinChunk = 256;   // arcs per chunk (a run offset fits a byte)
constexpr int kBinBlock = 1024;
constexpr uint16_t kBinPad = 0xFFFFu;

// A lane's 8 arcs of chunk c (all padding past the task's end).
__device__ __forceinline__ void bin_load_chunk(const PrArgs& a, uint64_t c, uint64_t cend, uint32_t lane, uint4& dd,
                                               uint2& rr, uint32_t& r0) {
  if (c < cend) {
    dd = ldg(reinterpret_cast<const uint4*>(a.b_dst + c * kBinChunk) + lane);
    rr = ldg(reinterpret_cast<const uint2*>(a.b_roff + c * kBinChunk) + lane);
    r0 = ldg(a.b_crun + c);
  } else {
    dd = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
    rr = make_uint2(0u, 0u);
    r0 = 0u;
  }
}

__device__ __forceinline__ uint32_t bin_dst(const uint4& dd, int k) {
  const uint32_t w = k < 2 ? dd.x : k < 4 ? dd.y : k < 6 ? dd.z : dd.w;
  return (w >> (16 * (k & 1))) & 0xFFFFu;
}

// The contributions of a lane's 8 arcs: each run's source, then its
// contribution (written by the finish pass: a plain load, not ldg; the
// 64 MB of contributions at 16 M vertices stay mostly in L2).
__device__ __forceinline__ void bin_load_vals(const PrArgs& a, const float* c_in, const uint4& dd, const uint2& rr,
                                              uint32_t r0, float (&x)[8]) {
  uint32_t u[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t off = ((k < 4 ? rr.x : rr.y) >> (8 * (k & 3))) & 0xFFu;
    u[k] = bin_dst(dd, k) != kBinPad ? ldg(a.b_rsrc + r0 + off) : 0xFFFFFFFFu;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = u[k] != 0xFFFFFFFFu ? c_in[u[k]] : 0.f;
}

// Add a lane's 8 arcs into the partition sums, one atomic per distinct
// destination (the 8 are sorted by destination, padding last).  A lane's
// last destination may continue in the next lanes (the chunk is sorted), so
// those last runs are first summed over the warp by destination: a chunk of
// 256 arcs into one hub makes one atomic, not 32, and the hub's sum is built
// from tree-summed parts (32 sequential float adds per chunk lost 8e-5 of a
// hub's rank over 150 K in-arcs).  All lanes call.
__device__ __forceinline__ void bin_add(float* s_sum, const uint4& dd, const float (&x)[8]) {
  uint32_t cur = bin_dst(dd, 0);
  float run = x[0];
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    const uint32_t d = bin_dst(dd, k);
    if (d != cur) {
      if (cur != kBinPad && run != 0.f) atomicAdd(&s_sum[cur], run);
      cur = d;
      run = x[k];
    } else {
      run += x[k];
    }
  }
  // only when some lane's last destination continues in the next lane
  const uint32_t next_first = __shfl_down_sync(kFull, bin_dst(dd, 0), 1);
  const bool cont = (threadIdx.x & 31u) < 31u && cur != kBinPad && next_first == cur;
  if (__any_sync(kFull, cont)) {
    if (seg_reduce(cur != kBinPad, cur, run) && run != 0.f) atomicAdd(&s_sum[cur], run);
  } else if (cur != kBinPad && run != 0.f) {
    atomicAdd(&s_sum[cur], run);
  }
}

// The gather phase of a binned iteration: the CTA takes tasks until none is
// left and leaves in every destination's sum slot of acc_cur the sum of
// c_in over its in-arcs.  All threads of the CTA call.
template <int BLOCK>
__device__ __forceinline__ void bin_gather(const PrArgs& a, const float* c_in, float* acc_cur, uint32_t it, float* s_sum,
                                           uint32_t* s_task) {
  const uint32_t tid = threadIdx.x, lane = lane_id(), wib = tid >> 5;
  constexpr uint32_t kW = BLOCK / 32;
    for (;;) {
      if (tid == 0) *s_task = atomicAdd(&a.ctl->task_next[it & 1], 1u);
      __syncthreads();
      const uint32_t t = *s_task;
      if (t >= a.b_ntasks) break;  // uniform
      const uint4 tk = ldg(a.b_tasks + t);
      const uint32_t v0 = tk.x, nv = tk.y & 0x7FFFFFFFu;
      const bool multi = (tk.y >> 31) != 0u;
      for (uint32_t d = tid; d < nv; d += BLOCK) s_sum[d] = 0.f;
      __syncthreads();
      // a lane takes 8 consecutive arcs of a chunk (sorted by destination
      // inside the chunk, so equal destinations are summed in registers
      // before one shared-memory atomic); the next chunk's words load while
      // this chunk's contributions are read and added (a second chunk ahead
      // measured slower: 29.6 against 23.0 ms on RMAT-24)
      uint64_t c = tk.z + wib;
      uint4 dd;
      uint2 rr;
      uint32_t r0;
      bin_load_chunk(a, c, tk.w, lane, dd, rr, r0);
      for (; c < tk.w; c += kW) {
        uint4 ddn;
        uint2 rrn;
        uint32_t r0n;
        bin_load_chunk(a, c + kW, tk.w, lane, ddn, rrn, r0n);
        float x[8];
        bin_load_vals(a, c_in, dd, rr, r0, x);
        bin_add(s_sum, dd, x);
        dd = ddn;
        rr = rrn;
        r0 = r0n;
      }
      __syncthreads();
      for (uint32_t d = tid; d < nv; d += BLOCK) {
        const float x = s_sum[d];
        if (!multi) acc_cur[v0 + d] = x;
        else if (x != 0.f) atomicAdd(&acc_cur[v0 + d], x);
      }
      __syncthreads();  // s_sum and s_task are reused by the next task
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) pr_pull_binned(PrArgs a) {
  extern __shared__ float s_sum[];  // kBinPart floats
  __shared__ double s_l1, s_total;
  __shared__ uint32_t s_max, s_task;
  if (threadIdx.x == 0) {
    s_l1 = 0.0;
    s_max = 0u;
  }
  __syncthreads();
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint32_t tid = threadIdx.x, lane = lane_id(), wib = tid >> 5;
  constexpr uint32_t kW = BLOCK / 32;
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + tid;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  float* const c_io = a.c[0];  // gathered, then rewritten after the barrier
  for (uint32_t it = 0;; ++it) {
    float* const acc_cur = (it & 1) ? a.acc2 : a.acc;
    float* const acc_nxt = (it & 1) ? a.acc : a.acc2;
    if (gtid == 0) {
      clear_change(ctl, (it + 1) % 3);
      ctl->task_next[(it + 1) & 1] = 0u;  // the counter iteration it + 1 takes (it - 1's is done)
    }
    bin_gather<BLOCK>(a, c_io, acc_cur, it, s_sum, &s_task);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    // ---- finish: ranks and contributions for the next gather
    double my_l1 = 0.0;
    float my_max = 0.f;
    const uint32_t vend = it >= 2 ? a.zero_from : a.n;  // constant tail skipped (its values stay)
    for (uint64_t v = gtid; v < vend; v += gthreads) {
      const float sum = acc_cur[v];
      acc_nxt[v] = 0.f;
      const float value = sum * a.alpha + a.base;  // PageRank-pull.cpp:222
      const float old = a.value[v];
      a.value[v] = value;
      const uint32_t k = a.nout[v];
      c_io[v] = k ? value / (float)k : 0.f;
      my_l1 += (double)fabsf(value - old);
      my_max = fmaxf(my_max, fabsf(value - old));
    }
    publish_change(ctl, it % 3, my_l1, my_max, &s_l1, &s_max);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    const double l1 = read_change(ctl, it % 3, a.linf, &s_total);
    if (gtid == 0) ctl->iters = it + 1;
    if (l1 <= (double)a.tol || it + 1 >= a.max_iter) break;  // PageRank-pull.cpp:238-243
  }
}

// Layout build, once per graph.  key = partition << 32 | source, value = destination.
__global__ void bin_keys_kernel(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col, uint32_t n,
                                uint64_t* __restrict__ key, uint32_t* __restrict__ row) {
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
    const uint64_t p = v / kBinPart;
    for (uint64_t j = offs[v] + lane; j < offs[v + 1]; j += 32) {
      key[j] = (p << 32) | col[j];
      row[j] = (uint32_t)v;
    }
  }
}

// runs: 1 where a (partition, source) pair starts
__global__ void bin_flags_kernel(const uint64_t* __restrict__ key, uint64_t m, uint32_t* __restrict__ flag) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride)
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// Sorted arc i of partition p goes to padded position pad[p] + i - first[p].
__global__ void bin_place_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ row,
                                 const uint32_t* __restrict__ runp1, uint64_t m, const uint64_t* __restrict__ first,
                                 const uint64_t* __restrict__ pad, uint16_t* __restrict__ dst,
                                 uint32_t* __restrict__ crun, uint32_t* __restrict__ run_src) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t p = (uint32_t)(key[i] >> 32);
    const uint64_t q = pad[p] + (i - first[p]);
    dst[q] = (uint16_t)(row[i] % kBinPart);
    const uint32_t r = runp1[i] - 1;
    if (q % kBinChunk == 0) crun[q / kBinChunk] = r;
    if (i == 0 || runp1[i] != runp1[i - 1]) run_src[r] = (uint32_t)key[i];
  }
}

__global__ void bin_roff_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ runp1, uint64_t m,
                                const uint64_t* __restrict__ first, const uint64_t* __restrict__ pad,
                                const uint32_t* __restrict__ crun, uint8_t* __restrict__ roff) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t p = (uint32_t)(key[i] >> 32);
    const uint64_t q = pad[p] + (i - first[p]);
    roff[q] = (uint8_t)(runp1[i] - 1 - crun[q / kBinChunk]);
  }
}

// Sort each chunk's arcs by destination (padding last): equal destinations
// become neighbours, so a lane sums them before its atomic.
__global__ void __launch_bounds__(kBinChunk) bin_chunk_sort_kernel(uint16_t* __restrict__ dst, uint8_t* __restrict__ roff,
                                                                   uint64_t nchunks) {
  using Sort = cub::BlockRadixSort<uint32_t, kBinChunk, 1>;
  __shared__ typename Sort::TempStorage tmp;
  for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint64_t i = c * kBinChunk + threadIdx.x;
    uint32_t key[1] = {((uint32_t)dst[i] << 8) | roff[i]};
    Sort(tmp).Sort(key, 0, 24);
    dst[i] = (uint16_t)(key[0] >> 8);
    roff[i] = (uint8_t)(key[0] & 0xFFu);
    __syncthreads();  // the temp storage is reused by the next chunk
  }
}

// The light rows' run table, in two passes: the row holding each run's first
// arc, then every arc's offset from it.
__global__ void light_runrow_kernel(const uint64_t* __restrict__ offs, uint32_t row0, uint32_t row1, uint64_t arc0,
                                    uint32_t* __restrict__ runrow) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = row0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < row1; v += stride) {
    const uint64_t b = offs[v] - arc0, e = offs[v + 1] - arc0;
    // the runs whose first arc lies in [b, e)
    for (uint64_t r = (b + kLightRun - 1) / kLightRun; r * kLightRun < e; ++r) runrow[r] = (uint32_t)v;
  }
}

__global__ void light_rowd_kernel(const uint64_t* __restrict__ offs, uint32_t row0, uint32_t row1, uint64_t arc0,
                                  const uint32_t* __restrict__ runrow, uint8_t* __restrict__ rowd) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = row0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < row1; v += stride)
    for (uint64_t e = offs[v] - arc0; e < offs[v + 1] - arc0; ++e)
      rowd[e] = (uint8_t)((uint32_t)v - runrow[e / kLightRun]);
}

// ---- pull-residual (PageRank-pull.cpp:132-190) ------------------------------
__global__ void pr_resid_init(PrArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.value[v] = 0.f;
    a.delta[v] = 0.f;
    a.residual[v] = 1.0f - a.alpha;  // INIT_RESIDUAL, PageRank-constants.h:33
  }
}

__global__ void __launch_bounds__(kBlock) pr_pull_residual_persistent(PrArgs a) {
  __shared__ float s_acc[kWarps][32];
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kBlock;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  s_acc[wib][lane] = 0.f;
  __syncwarp();
  for (uint32_t it = 0;; ++it) {
    if (gtid == 0) ctl->active[(it + 1) % 3] = 0;
    uint32_t my_accum = 0;
    for (uint64_t v = gtid; v < a.n; v += gthreads) {
      a.delta[v] = 0.f;
      const float r = a.residual[v];
      if (r > a.tol) {
        a.residual[v] = 0.f;
        a.value[v] += r;
        const uint32_t k = a.nout[v];
        if (k > 0) {
          a.delta[v] = r * a.alpha / (float)k;
          ++my_accum;
        }
      }
    }
    my_accum = __reduce_add_sync(kFull, my_accum);
    if (lane == 0 && my_accum) atomicAdd(&ctl->active[it % 3], my_accum);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    auto finish = [&](uint32_t v, float sum) {
      if (sum > 0.f) a.residual[v] = sum;
    };
    sweep_all(
        a.offs, a.n, a.sched, gwarp, nwarps,
        [&](bool valid, uint64_t e, uint32_t owner, uint32_t) {
          float x = 0.f;
          if (valid) {
            const float d = a.delta[ldg(a.col + e)];
            x = d > 0.f ? d : 0.f;
          }
          if (seg_reduce(valid, owner, x)) s_acc[wib][owner] += x;
          __syncwarp();
        },
        [&](uint32_t v, bool valid, bool heavy) {
          const float sum = s_acc[wib][lane];
          s_acc[wib][lane] = 0.f;
          __syncwarp();
          if (valid && !heavy) finish(v, sum);
        },
        [&](uint32_t v, uint64_t b, uint64_t e) {
          float s = 0.f;
          for (uint64_t i = b + lane; i < e; i += 32) {
            const float d = a.delta[ldg(a.col + i)];
            s += d > 0.f ? d : 0.f;
          }
          s = warp_sum(s);
          if (lane == 0) atomicAdd(&a.acc[v], s);
        });
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    for (uint64_t i = gtid; i < a.sched.nheavy; i += gthreads) {
      const uint32_t v = a.sched.heavy_list[i];
      const float sum = a.acc[v];
      a.acc[v] = 0.f;
      finish(v, sum);
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    const uint32_t accum = *reinterpret_cast<volatile uint32_t*>(&ctl->active[it % 3]);
    if (gtid == 0) ctl->iters = it + 1;
    if (it + 1 >= a.max_iter || accum == 0) break;
  }
}

// Pull-residual rounds over the binned layout (degree-ordered graphs): the
// vertex pass of round it first closes round it - 1 (a positive sum becomes
// the residual), then takes the residuals above tol (value += residual,
// delta = residual * alpha / outdeg), and the gather sums the deltas over
// the in-arcs.  The rounds, their deltas and the stopping rule are those of
// pr_pull_residual_persistent; a round ends in two grid barriers, not three.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) pr_resid_binned(PrArgs a) {
  extern __shared__ float s_sum[];  // kBinPart floats
  __shared__ uint32_t s_task;
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  for (uint32_t it = 0;; ++it) {
    float* const acc_prev = (it & 1) ? a.acc : a.acc2;  // round it - 1's sums
    float* const acc_cur = (it & 1) ? a.acc2 : a.acc;
    if (gtid == 0) {
      ctl->active[(it + 1) % 3] = 0;
      ctl->task_next[(it + 1) & 1] = 0u;
    }
    uint32_t my_accum = 0;
    for (uint64_t v = gtid; v < a.n; v += gthreads) {
      float r = a.residual[v];
      if (it > 0) {
        const float sum = acc_prev[v];
        if (sum > 0.f) r = sum;
      }
      // the sums of round it - 2, read by round it - 1: zeroed for this
      // round's gather (zeroing the slots the last gather's atomics just
      // updated stalls)
      acc_cur[v] = 0.f;
      float d = 0.f;
      if (r > a.tol) {
        a.value[v] += r;
        const uint32_t k = a.nout[v];
        if (k > 0) {
          d = r * a.alpha / (float)k;
          ++my_accum;
        }
        r = 0.f;
      }
      a.residual[v] = r;
      a.delta[v] = d;
    }
    my_accum = __reduce_add_sync(kFull, my_accum);
    if (lane_id() == 0 && my_accum) atomicAdd(&ctl->active[it % 3], my_accum);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    bin_gather<BLOCK>(a, a.delta, acc_cur, it, s_sum, &s_task);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    const uint32_t accum = *reinterpret_cast<volatile uint32_t*>(&ctl->active[it % 3]);
    if (gtid == 0) ctl->iters = it + 1;
    if (it + 1 >= a.max_iter || accum == 0) break;
  }
}

// ---- residual push, Sync (PageRank-push.cpp:103-188) ------------------------
__global__ void pr_push_init(PrArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.value[v] = 0.f;
    a.residual[v] = 1.0f - a.alpha;
    a.active[0][v] = (uint32_t)v;
    a.stamp[v] = 0xFFFFFFFFu;
  }
  if (tid == 0) a.ctl->active[0] = a.n;
}

__global__ void __launch_bounds__(kBlock) pr_push_persistent(PrArgs a) {
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kBlock;
  const uint32_t lane = lane_id();
  unsigned long long my_push = 0;
  for (uint32_t it = 0;; ++it) {
    const uint32_t na = min(ctl->active[it % 3], a.n);
    if (na == 0 || it >= a.max_iter) break;
    const int fset = it % 3;
    if (gtid == 0) {
      ctl->active[(it + 2) % 3] = 0;
      ctl->fc[(it + 1) % 3] = FrontierCounters{};
    }
    FrontierCounters& fc = ctl->fc[fset];
    const uint32_t* act = a.active[it & 1];
    uint32_t* act_next = a.active[(it + 1) & 1];
    // phase A: absorb residual, compute delta, queue vertices with out-arcs
    for (uint64_t base = gtid - lane; base < na; base += gthreads) {
      const uint64_t i = base + lane;
      bool q = false;
      uint32_t v = 0;
      if (i < na) {
        v = act[i];
        const float r = a.residual[v];
        if (r > a.tol) {
          const float old = atomicExch(&a.residual[v], 0.f);
          if (old > 0.f) {
            a.value[v] += old;
            const uint64_t deg = ldg(a.offs + v + 1) - ldg(a.offs + v);
            if (deg > 0) {
              a.delta[v] = old * a.alpha / (float)deg;
              q = true;
            }
          }
        }
      }
      push_discovered(a.fq, it & 1, fc, q, v, a.offs, a.heavy, a.tile, &ctl->err);
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    // phase B: push deltas along out-arcs, activate on crossing tol
    const uint32_t q_light = min(fc.light, a.fq.light_cap), q_tiles = min(fc.tiles, a.fq.tile_cap);
    auto apply = [&](bool valid, uint32_t u, float d) {
      bool act_u = false;
      if (valid) {
        const float old = atomicAdd(&a.residual[u], d);
        ++my_push;
        if (old <= a.tol && old + d >= a.tol) {
          if (a.stamp[u] != it) act_u = atomicExch(&a.stamp[u], it) != it;
        }
      }
      warp_push(act_u, u, act_next, &ctl->active[(it + 1) % 3], a.n, &ctl->err);
    };
    const uint32_t* qin = a.fq.light[it & 1];
    const uint2* tin = a.fq.tiles[it & 1];
    for (;;) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&fc.light_work, 32u);
      base = __shfl_sync(kFull, base, 0);
      if (base >= q_light) break;
      const uint32_t idx = base + lane;
      uint64_t b = 0;
      uint32_t d = 0;
      float dl = 0.f;
      if (idx < q_light) {
        const uint32_t v = qin[idx];
        b = ldg(a.offs + v);
        d = (uint32_t)(ldg(a.offs + v + 1) - b);
        dl = a.delta[v];
      }
      warp_expand(b, d, __float_as_uint(dl), [&](bool valid, uint64_t e, uint32_t, uint32_t pl) {
        apply(valid, valid ? ldg(a.col + e) : 0u, __uint_as_float(pl));
      });
    }
    for (;;) {
      uint32_t t = 0;
      if (lane == 0) t = atomicAdd(&fc.tile_work, 1u);
      t = __shfl_sync(kFull, t, 0);
      if (t >= q_tiles) break;
      const uint2 tv = tin[t];
      const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
      const uint64_t b = vb + (uint64_t)tv.y * a.tile;
      const uint64_t e_end = min(ve, b + a.tile);
      const float dl = a.delta[tv.x];
      for (uint64_t e0 = b; e0 < e_end; e0 += 32) {
        const uint64_t e = e0 + lane;
        apply(e < e_end, e < e_end ? ldg(a.col + e) : 0u, dl);
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    if (gtid == 0) ctl->iters = it + 1;
  }
  my_push = warp_sum(my_push);
  if (lane == 0 && my_push) atomicAdd(&ctl->pushes, my_push);
}

// ---- residual push, Async (PageRank-push.cpp:68-101) -------------------------
// Worklist entries: (v, kAbsorb, 0, 0) "take v's residual if it is above
// tol" -- every vertex once at the start (the reference iterates the whole
// graph), then each vertex whose residual an add lifts across tol -- and
// (v, k, delta bits, 0): "add delta along the k-th tile of v's arcs", made
// when a heavy vertex is absorbed.
constexpr uint32_t kAbsorb = 0xFFFFFFFFu;
constexpr int kPushLQ = 64;

__global__ void pr_push_async_init(PrArgs a, uint32_t nchunks) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.value[v] = 0.f;
    a.residual[v] = 1.0f - a.alpha;  // INIT_RESIDUAL, PageRank-constants.h:33
  }
  // the initial worklist: every vertex, 32 per chunk, published
  for (uint64_t i = tid; i <= a.ring.mask; i += stride) {
    if (i < nchunks) {
      const uint32_t first = (uint32_t)(i * 32);
      const uint32_t cnt = min(32u, a.n - first);
      for (uint32_t j = 0; j < cnt; ++j) a.ring.ent[i * 32 + j] = make_uint4(first + j, kAbsorb, 0u, 0u);
      a.ring.cnt[i] = cnt;
      a.ring.seq[i] = i + 1;
    } else {
      a.ring.seq[i] = i;
    }
  }
  if (tid == 0) {
    a.ring.rc->tail = nchunks;
    a.ring.rc->work = (int)nchunks;
  }
}

__global__ void __launch_bounds__(kBlock, 1) pr_push_async(PrArgs a) {
  __shared__ uint4 s_lq[kWarps][kPushLQ];
  PrCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint32_t lane = lane_id();
  unsigned long long my_push = 0, my_absorb = 0;
  worklists::WarpQueue<kPushLQ> q(s_lq[threadIdx.x >> 5], a.ring, &ctl->err, deadline);
  const float tol = a.tol;
  // add d to u's residual; activate u when the add lifts it across tol
  // (old < tol <= old + d, PageRank-push.cpp:92-94)
  auto add = [&](bool valid, uint32_t u, float d) {
    bool act = false;
    if (valid && d > 0.f) {
      const float old = atomicAdd(&a.residual[u], d);
      ++my_push;
      act = old < tol && old + d >= tol;
    }
    q.push(act, make_uint4(u, kAbsorb, 0u, 0u));
  };
  for (;;) {
    uint4 ent;
    bool has;
    const int got = q.next(ent, has);
    if (got <= 0) break;
    // tiles of heavy vertices: the whole warp adds along each in turn
    unsigned tm = __ballot_sync(kFull, has && ent.y != kAbsorb);
    while (tm) {
      const int j = __ffs(tm) - 1;
      tm &= tm - 1u;
      const uint32_t v = __shfl_sync(kFull, ent.x, j);
      const uint32_t k = __shfl_sync(kFull, ent.y, j);
      const float d = __uint_as_float(__shfl_sync(kFull, ent.z, j));
      const uint64_t vb = ldg(a.offs + v), ve = ldg(a.offs + v + 1);
      const uint64_t b = vb + (uint64_t)k * a.tile, e_end = min(ve, b + a.tile);
      for (uint64_t e0 = b; e0 < e_end; e0 += 32) {
        const uint64_t e = e0 + lane;
        add(e < e_end, e < e_end ? ldg(a.col + e) : 0u, d);
      }
    }
    // absorb: exchange the residual with 0 if it is above tol
    const bool absorb = has && ent.y == kAbsorb;
    uint64_t b = 0, deg = 0;
    float delta = 0.f;
    if (absorb && __ldcg(a.residual + ent.x) > tol) {
      const float old = atomicExch(&a.residual[ent.x], 0.f);
      atomicAdd(&a.value[ent.x], old);  // a vertex may be queued twice when tol >= 1 - alpha
      ++my_absorb;
      b = ldg(a.offs + ent.x);
      deg = ldg(a.offs + ent.x + 1) - b;
      if (deg > 0) delta = old * a.alpha / (float)deg;
    }
    const bool light = deg > 0 && deg <= a.heavy;
    // light rows: their arcs spread over the warp
    warp_expand(b, light ? (uint32_t)deg : 0u, __float_as_uint(delta), [&](bool valid, uint64_t e, uint32_t, uint32_t pl) {
      add(valid, valid ? ldg(a.col + e) : 0u, __uint_as_float(pl));
    });
    // heavy rows: one worklist entry per tile
    unsigned hm = __ballot_sync(kFull, deg > a.heavy && delta > 0.f);
    while (hm) {
      const int j = __ffs(hm) - 1;
      hm &= hm - 1u;
      const uint32_t v = __shfl_sync(kFull, ent.x, j);
      const uint32_t nt = (uint32_t)((__shfl_sync(kFull, deg, j) + a.tile - 1) / a.tile);
      const uint32_t dbits = __shfl_sync(kFull, __float_as_uint(delta), j);
      for (uint32_t t0 = 0; t0 < nt; t0 += 32) q.push(t0 + lane < nt, make_uint4(v, t0 + lane, dbits, 0u));
    }
    q.share();
  }
  my_push = warp_sum(my_push);
  my_absorb = warp_sum(my_absorb);
  if (lane == 0) {
    if (my_push) atomicAdd(&ctl->pushes, my_push);
    if (my_absorb) atomicAdd(&ctl->absorbs, my_absorb);
  }
}

int ensure_nout(gb_graph* g, cudaStream_t s) {
  if (g->outdeg_of_stored) return GB_OK;
  GB_CUDA(cudaMalloc(&g->outdeg_of_stored, sizeof(uint32_t) * g->n));
  GB_CUDA(cudaMemsetAsync(g->outdeg_of_stored, 0, sizeof(uint32_t) * g->n, s));
  if (g->m) count_nout<<<g->sm_count * 8, 256, 0, s>>>(g->col, g->m, g->outdeg_of_stored);
  GB_CUDA(cudaGetLastError());
  return GB_OK;
}

enum class PrKind { Pull, PullResidual, Push, PushAsync };

// Build (once) the binned layout of the stored arcs for pr_pull_binned.
// GB_ERR_UNSUPPORTED when it does not apply (no arcs, 2^32 arcs or more);
// on any failure nothing is cached and the caller keeps the row sweep.
int ensure_pr_bins(gb_graph* g, cudaStream_t s) {
  if (g->prb) return GB_OK;
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  if (m == 0 || m >= 0xFFFFFFF0ull) return GB_ERR_UNSUPPORTED;  // run ids and run offsets are 32-bit
  const uint32_t P = (uint32_t)(((uint64_t)n + kBinPart - 1) / kBinPart);
  std::vector<uint64_t> ho((size_t)n + 1);
  GB_CUDA(cudaMemcpyAsync(ho.data(), g->offs, sizeof(uint64_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, s));
  GB_CUDA(cudaStreamSynchronize(s));
  // partitions: their arcs, padded to whole chunks; tasks of about
  // m / (6 per SM) arcs, the largest first
  std::vector<uint64_t> first((size_t)P + 1), pad((size_t)P + 1);
  uint64_t mpad = 0;
  for (uint32_t p = 0; p < P; ++p) {
    const uint64_t v0 = (uint64_t)p * kBinPart, v1 = std::min<uint64_t>(v0 + kBinPart, n);
    first[p] = ho[v0];
    pad[p] = mpad;
    mpad += (ho[v1] - ho[v0] + kBinChunk - 1) / kBinChunk * kBinChunk;
  }
  first[P] = m;
  pad[P] = mpad;
  const uint64_t nchunks = mpad / kBinChunk;
  const uint64_t target_chunks = std::max<uint64_t>(64, m / ((uint64_t)g->sm_count * 6 * kBinChunk));
  std::vector<uint4> tasks;
  for (uint32_t p = 0; p < P; ++p) {
    const uint64_t c0 = pad[p] / kBinChunk, c1 = pad[p + 1] / kBinChunk;
    if (c0 == c1) continue;  // no in-arcs: the finish pass keeps those sums at zero
    const uint64_t nt = (c1 - c0 + target_chunks - 1) / target_chunks;
    const uint64_t per = (c1 - c0 + nt - 1) / nt;
    const uint32_t v0 = p * kBinPart;
    const uint32_t nv = (uint32_t)std::min<uint64_t>(kBinPart, (uint64_t)n - v0);
    for (uint64_t c = c0; c < c1; c += per)
      tasks.push_back(make_uint4(v0, nv | (nt > 1 ? 0x80000000u : 0u), (uint32_t)c, (uint32_t)std::min(c1, c + per)));
  }
  std::stable_sort(tasks.begin(), tasks.end(), [](const uint4& x, const uint4& y) { return x.w - x.z > y.w - y.z; });
  if (nchunks >= 0xFFFFFFFFull) return GB_ERR_UNSUPPORTED;  // chunk ids are 32-bit in the tasks

  // temporaries
  uint64_t *key0 = nullptr, *key1 = nullptr, *dfirst = nullptr;
  uint32_t *row0 = nullptr, *row1 = nullptr, *runp1 = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  PrBins* b = new PrBins;
  auto cleanup = [&](bool keep) {
    cudaFree(key0);
    cudaFree(key1);
    cudaFree(row0);
    cudaFree(row1);
    cudaFree(runp1);
    cudaFree(dfirst);
    cudaFree(tmp);
    if (!keep) {
      cudaFree(b->mem);
      delete b;
    }
  };
#define GB_BTRY(call)                       \
  do {                                      \
    cudaError_t _e = (call);                \
    if (_e != cudaSuccess) {                \
      const int _st = cuda_fail(_e, #call); \
      cleanup(false);                       \
      return _st;                           \
    }                                       \
  } while (0)
  GB_BTRY(cudaMalloc(&key0, sizeof(uint64_t) * m));
  GB_BTRY(cudaMalloc(&key1, sizeof(uint64_t) * m));
  GB_BTRY(cudaMalloc(&row0, sizeof(uint32_t) * m));
  GB_BTRY(cudaMalloc(&row1, sizeof(uint32_t) * m));
  GB_BTRY(cudaMalloc(&runp1, sizeof(uint32_t) * m));
  GB_BTRY(cudaMalloc(&dfirst, sizeof(uint64_t) * 2 * ((size_t)P + 1)));
  uint64_t* dpad = dfirst + P + 1;
  GB_BTRY(cudaMemcpyAsync(dfirst, first.data(), sizeof(uint64_t) * ((size_t)P + 1), cudaMemcpyHostToDevice, s));
  GB_BTRY(cudaMemcpyAsync(dpad, pad.data(), sizeof(uint64_t) * ((size_t)P + 1), cudaMemcpyHostToDevice, s));
  const int grid = g->sm_count * 8;
  bin_keys_kernel<<<grid, 256, 0, s>>>(g->offs, g->col, n, key0, row0);
  GB_BTRY(cudaGetLastError());
  int end_bit = 33;  // partition ids above the 32 source bits
  while ((1ull << (end_bit - 32)) < (uint64_t)P) ++end_bit;
  cub::DoubleBuffer<uint64_t> dk(key0, key1);
  cub::DoubleBuffer<uint32_t> dv(row0, row1);
  GB_BTRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dv, (int64_t)m, 0, end_bit, s));
  size_t scan_bytes = 0;
  GB_BTRY(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, runp1, runp1, (int64_t)m, s));
  tmp_bytes = std::max(tmp_bytes, scan_bytes);
  GB_BTRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
  GB_BTRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, dk, dv, (int64_t)m, 0, end_bit, s));
  bin_flags_kernel<<<grid, 256, 0, s>>>(dk.Current(), m, runp1);
  GB_BTRY(cudaGetLastError());
  GB_BTRY(cub::DeviceScan::InclusiveSum(tmp, scan_bytes, runp1, runp1, (int64_t)m, s));
  uint32_t np32 = 0;
  GB_BTRY(cudaMemcpyAsync(&np32, runp1 + (m - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GB_BTRY(cudaStreamSynchronize(s));
  const uint64_t npairs = np32;
  // the cached layout, one allocation (parts 256-byte aligned)
  auto part = [](uint64_t bytes) { return (bytes + 255) & ~uint64_t(255); };
  const uint64_t sz_dst = part(2 * mpad), sz_roff = part(mpad), sz_crun = part(4 * nchunks), sz_rsrc = part(4 * npairs),
                 sz_tasks = part(16 * tasks.size());
  GB_BTRY(cudaMalloc(&b->mem, sz_dst + sz_roff + sz_crun + sz_rsrc + sz_tasks));
  char* q = static_cast<char*>(b->mem);
  b->dst = reinterpret_cast<uint16_t*>(q);
  q += sz_dst;
  b->roff = reinterpret_cast<uint8_t*>(q);
  q += sz_roff;
  b->crun = reinterpret_cast<uint32_t*>(q);
  q += sz_crun;
  b->rsrc = reinterpret_cast<uint32_t*>(q);
  q += sz_rsrc;
  b->tasks = reinterpret_cast<uint4*>(q);
  b->ntasks = (uint32_t)tasks.size();
  b->npairs = npairs;
  b->nchunks = nchunks;
  GB_BTRY(cudaMemsetAsync(b->dst, 0xFF, 2 * mpad, s));  // padding: kBinPad
  GB_BTRY(cudaMemsetAsync(b->roff, 0, mpad, s));
  GB_BTRY(cudaMemcpyAsync(b->tasks, tasks.data(), 16 * tasks.size(), cudaMemcpyHostToDevice, s));
  bin_place_kernel<<<grid, 256, 0, s>>>(dk.Current(), dv.Current(), runp1, m, dfirst, dpad, b->dst, b->crun, b->rsrc);
  GB_BTRY(cudaGetLastError());
  bin_roff_kernel<<<grid, 256, 0, s>>>(dk.Current(), runp1, m, dfirst, dpad, b->crun, b->roff);
  GB_BTRY(cudaGetLastError());
  bin_chunk_sort_kernel<<<g->sm_count * 16, kBinChunk, 0, s>>>(b->dst, b->roff, nchunks);
  GB_BTRY(cudaGetLastError());
  GB_BTRY(cudaStreamSynchronize(s));
#undef GB_BTRY
  cleanup(true);
  g->prb = b;
  return GB_OK;
}


inline float bits_to_float(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// The flat sweeps' run table of a degree-ordered graph (its heavy rows are
// [0, nheavy), the light rows' arcs one contiguous range): built once per
// heavy threshold and cached in the handle, then wired into `a`.
int light_run_table(gb_graph* g, const SweepSched& sched, PrArgs* a, cudaStream_t s) {
  if (!g->lr_rowid || g->lr_heavy != sched.heavy) {
    cudaFree(g->lr_rowid);
    g->lr_rowid = nullptr;
    uint64_t ends[2] = {0, 0};
    GB_CUDA(cudaMemcpyAsync(&ends[0], g->offs + sched.nheavy, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(&ends[1], g->offs + g->zero_from, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    if (ends[1] < ends[0]) GB_FAIL(GB_ERR_CUDA, "pagerank: light rows out of order");
    // one allocation: the run rows (uint32 per run), then a byte per arc
    const uint64_t narcs = ends[1] - ends[0];
    const uint64_t nruns = (narcs + kLightRun - 1) / kLightRun;
    GB_CUDA(cudaMalloc(&g->lr_rowid, sizeof(uint32_t) * std::max<uint64_t>(nruns, 1) + narcs + 16));
    if (g->zero_from > sched.nheavy) {
      uint32_t* runrow = g->lr_rowid;
      uint8_t* rowd = reinterpret_cast<uint8_t*>(g->lr_rowid + std::max<uint64_t>(nruns, 1));
      light_runrow_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, sched.nheavy, g->zero_from, ends[0], runrow);
      light_rowd_kernel<<<g->sm_count * 8, 256, 0, s>>>(g->offs, sched.nheavy, g->zero_from, ends[0], runrow, rowd);
    }
    GB_CUDA(cudaGetLastError());
    g->lr_row0 = sched.nheavy;
    g->lr_heavy = sched.heavy;
    g->lr_arc0 = ends[0];
    g->lr_arc1 = ends[1];
  }
  a->lr_runrow = g->lr_rowid;
  a->lr_rowd = reinterpret_cast<const uint8_t*>(
      g->lr_rowid + std::max<uint64_t>((g->lr_arc1 - g->lr_arc0 + kLightRun - 1) / kLightRun, 1));
  a->lr_arc0 = g->lr_arc0;
  a->lr_arc1 = g->lr_arc1;
  return GB_OK;
}

int run_pagerank(gb_graph* g, PrKind kind, float alpha, float tol, uint32_t max_iter, float* rank_out,
                 uint32_t* iters_out, gb_stats* stats, cudaStream_t s, float init = -1.f, float base = -1.f,
                 int linf = 0) {
  static_assert(sizeof(PrCtl) <= 4096, "PrCtl must fit the pinned readback area");
  if (!(alpha > 0.f && alpha < 1.f)) GB_FAIL(GB_ERR_ARG, "pagerank: alpha must be in (0,1)");
  if (!(tol >= 0.f)) GB_FAIL(GB_ERR_ARG, "pagerank: tolerance must be >= 0");
  if (max_iter == 0) GB_FAIL(GB_ERR_ARG, "pagerank: max_iter must be > 0");
  const gb_tuning t = effective_tuning(g);
  const uint32_t n = g->n;
  const bool out_dev = is_device_ptr(rank_out);
  int st = GB_OK;
  SweepSched sched{};
  if (kind == PrKind::Pull || kind == PrKind::PullResidual) {
    st = ensure_sweep_schedule(g, t.heavy_degree, t.tile_edges, s, &sched);
    if (st != GB_OK) return st;
    st = ensure_nout(g, s);
    if (st != GB_OK) return st;
  }
  FrontierLayout fl = frontier_layout(n, g->m, t.heavy_degree, t.tile_edges);
  // Async: the initial worklist (every vertex, 32 per chunk) plus room for
  // as many chunks again and the tiles of the heavy vertices
  const uint32_t nchunks = (uint32_t)(((uint64_t)n + 31) / 32);
  const unsigned long long cap = worklists::ring_capacity(2ull * nchunks + g->m / ((uint64_t)t.tile_edges * 32) + 8192);
  size_t need = carve_size<PrCtl>(1) + 5 * carve_size<float>(n) + (out_dev ? 0 : carve_size<float>(n));
  if (kind != PrKind::Pull) need += 2 * carve_size<float>(n);
  if (kind == PrKind::Push) need += 3 * carve_size<uint32_t>(n) + fl.bytes;
  if (kind == PrKind::PushAsync) need += carve_size<char>(worklists::ring_bytes(cap));
  st = ws_reserve(g, need, s);
  if (st != GB_OK) return st;
  Carver cv(g->ws);
  PrArgs a{};
  a.ctl = cv.take<PrCtl>(1);
  a.c[0] = cv.take<float>(n);
  a.c[1] = cv.take<float>(n);
  a.acc = cv.take<float>(n);
  a.acc2 = cv.take<float>(n);
  if (kind != PrKind::Pull) {
    a.residual = cv.take<float>(n);
    a.delta = cv.take<float>(n);
  }
  if (kind == PrKind::Push) {
    a.active[0] = cv.take<uint32_t>(n);
    a.active[1] = cv.take<uint32_t>(n);
    a.stamp = cv.take<uint32_t>(n);
    a.fq = carve_frontier(cv, fl);
  }
  if (kind == PrKind::PushAsync) a.ring = worklists::ring_layout(cv.take<char>(worklists::ring_bytes(cap)), cap);
  a.value = out_dev ? rank_out : cv.take<float>(n);
  a.offs = g->offs;
  a.col = g->col;
  a.nout = g->outdeg_of_stored;
  a.n = n;
  a.alpha = alpha;
  a.base = base >= 0.f ? base : (1.0f - alpha) / (float)n;  // PageRank-pull.cpp:200
  a.init = init >= 0.f ? init : 1.0f / (float)n;
  a.linf = linf;
  a.tol = tol;
  a.max_iter = max_iter;
  a.sched = sched;
  a.heavy = t.heavy_degree;
  a.tile = t.tile_edges;
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(PrCtl), s));
  const void* kfn = nullptr;
  int block = kBlock;
  size_t smem = 0;
  if (kind == PrKind::Pull) {
    pr_pull_init<<<g->sm_count * 4, 256, 0, s>>>(a);
    a.zero_from = g->perm ? g->zero_from : n;
    kfn = reinterpret_cast<const void*>(&pr_pull_persistent<kBlock, 2, 6>);
    // the flat sweep needs the degree order: heavy rows first, the light rows' arcs one range
    if (g->perm && (g->order == GB_ORDER_DEGREE || g->order == GB_ORDER_DEGREE_UNSORTED)) {
      // degree-ordered: the binned layout (sequential streams, few
      // (source, partition) pairs per arc); where it cannot be built, the
      // flat sweep (heavy rows are [0, nheavy), the light rows' arcs one
      // contiguous range)
      if (ensure_pr_bins(g, s) == GB_OK) {
        const PrBins* b = g->prb;
        a.b_dst = b->dst;
        a.b_roff = b->roff;
        a.b_crun = b->crun;
        a.b_rsrc = b->rsrc;
        a.b_tasks = b->tasks;
        a.b_ntasks = b->ntasks;
        kfn = reinterpret_cast<const void*>(&pr_pull_binned<kBinBlock>);
        block = kBinBlock;
        smem = sizeof(float) * kBinPart;
        GB_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      } else {
        clear_error();
        st = light_run_table(g, sched, &a, s);
        if (st != GB_OK) return st;
        kfn = reinterpret_cast<const void*>(&pr_pull_flat<kBlock, 6>);
      }
    }
  } else if (kind == PrKind::PullResidual) {
    pr_resid_init<<<g->sm_count * 4, 256, 0, s>>>(a);
    GB_CUDA(cudaMemsetAsync(a.acc, 0, sizeof(float) * n, s));
    kfn = reinterpret_cast<const void*>(&pr_pull_residual_persistent);
    if (g->perm && (g->order == GB_ORDER_DEGREE || g->order == GB_ORDER_DEGREE_UNSORTED)) {
      if (ensure_pr_bins(g, s) == GB_OK) {  // else the row sweep
        const PrBins* b = g->prb;
        a.b_dst = b->dst;
        a.b_roff = b->roff;
        a.b_crun = b->crun;
        a.b_rsrc = b->rsrc;
        a.b_tasks = b->tasks;
        a.b_ntasks = b->ntasks;
        GB_CUDA(cudaMemsetAsync(a.acc2, 0, sizeof(float) * n, s));
        kfn = reinterpret_cast<const void*>(&pr_resid_binned<kBinBlock>);
        block = kBinBlock;
        smem = sizeof(float) * kBinPart;
        GB_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      } else {
        clear_error();
      }
    }
  } else if (kind == PrKind::Push) {
    pr_push_init<<<g->sm_count * 4, 256, 0, s>>>(a);
    kfn = reinterpret_cast<const void*>(&pr_push_persistent);
  } else {
    GB_CUDA(cudaMemsetAsync(a.ring.rc, 0, sizeof(worklists::RingCtl), s));
    pr_push_async_init<<<g->sm_count * 4, 256, 0, s>>>(a, nchunks);
    kfn = reinterpret_cast<const void*>(&pr_push_async);
  }
  GB_CUDA(cudaGetLastError());
  const int grid = coop_grid(g, kfn, block, smem, t.blocks_per_sm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "pagerank: cannot size cooperative grid");
  void* args[] = {&a};
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, block, args, smem, s));
  kt.stop(s);
  PrCtl* hc = reinterpret_cast<PrCtl*>(static_cast<char*>(g->pinned) + 4096);  // PrCtl is ~1 KB
  GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(PrCtl), cudaMemcpyDeviceToHost, s));
  if (!out_dev) {
    st = copy_out(rank_out, a.value, sizeof(float) * n, s);
    if (st != GB_OK) return st;
  }
  if (stats || iters_out || !out_dev) {
    GB_CUDA(cudaStreamSynchronize(s));
    if (hc->err) return dev_err_status(hc->err, "pagerank");
    // Async has no rounds: one pass over the worklist
    if (kind == PrKind::PushAsync) hc->iters = 1;
    if (iters_out) *iters_out = hc->iters;
    if (stats) {
      *stats = gb_stats{};
      stats->vertices_reached = n;
      stats->edges_reached = g->m;
      stats->rounds = hc->iters;
      stats->relaxations = hc->pushes;
      if (kind == PrKind::PushAsync) stats->vertices_reached = hc->absorbs;  // residuals taken
      stats->launches = 2;
      stats->kernel_ms = kt.ms();
      double l1sum = 0.0;
      for (int k = 0; k < kL1Slots; ++k) l1sum += hc->l1[(hc->iters + 2) % 3][k];
      stats->residual = kind == PrKind::Pull ? (linf ? (double)bits_to_float(hc->linf[(hc->iters + 2) % 3]) : l1sum)
                                             : 0.0;
    }
    if (kind != PrKind::Push && kind != PrKind::PushAsync && hc->iters >= max_iter) {
      // the ranks are set; the status tells the caller the cap was hit
      gb::set_error("pagerank: failed to converge in %u iterations", hc->iters);
      return GB_ERR_NOT_CONVERGED;
    }
  }
  return GB_OK;
}

}  // namespace

// Entry wrapper: on a relabelled graph the ranks are computed in internal ids
// and mapped back (also when the iteration cap was hit: the ranks are set).
int pagerank_entry(gb_graph* g, PrKind kind, float alpha, float tol, uint32_t max_iter, float* rank_out,
                   uint32_t* iters_out, gb_stats* stats, cudaStream_t s, float init = -1.f, float base = -1.f,
                   int linf = 0) {
  if (!g->perm) return run_pagerank(g, kind, alpha, tol, max_iter, rank_out, iters_out, stats, s, init, base, linf);
  gb_stats local{};
  float* res = reinterpret_cast<float*>(result_buf(g, 0));
  int st = run_pagerank(g, kind, alpha, tol, max_iter, res, iters_out,
                        stats ? stats : (is_device_ptr(rank_out) ? nullptr : &local), s, init, base, linf);
  if (st != GB_OK && st != GB_ERR_NOT_CONVERGED) return st;
  if (stats) stats->launches += 1;  // the mapping gather
  const int fs = finish_f32(g, res, rank_out, s);
  return fs != GB_OK ? fs : st;
}

}  // namespace gb

extern "C" {

int gb_pagerank_pull(gb_graph* g, float alpha, float tol, uint32_t max_iter, float* rank_out,
                     uint32_t* iters_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !rank_out) GB_FAIL(GB_ERR_ARG, "gb_pagerank_pull: null argument");
  GB_CUDA(cudaSetDevice(g->device));
  return gb::pagerank_entry(g, gb::PrKind::Pull, alpha, tol, max_iter, rank_out, iters_out, stats,
                            static_cast<cudaStream_t>(stream));
}

int gb_pagerank_pull_ex(gb_graph* g, float alpha, float tol, uint32_t max_iter, float init, float base,
                        int norm_linf, float* rank_out, uint32_t* iters_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !rank_out) GB_FAIL(GB_ERR_ARG, "gb_pagerank_pull_ex: null argument");
  if (!(init >= 0.f) || !(base >= 0.f)) GB_FAIL(GB_ERR_ARG, "gb_pagerank_pull_ex: init and base must be >= 0");
  GB_CUDA(cudaSetDevice(g->device));
  return gb::pagerank_entry(g, gb::PrKind::Pull, alpha, tol, max_iter, rank_out, iters_out, stats,
                            static_cast<cudaStream_t>(stream), init, base, norm_linf ? 1 : 0);
}

int gb_pagerank_pull_residual(gb_graph* g, float alpha, float tol, uint32_t max_iter, float* rank_out,
                              uint32_t* iters_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !rank_out) GB_FAIL(GB_ERR_ARG, "gb_pagerank_pull_residual: null argument");
  GB_CUDA(cudaSetDevice(g->device));
  return gb::pagerank_entry(g, gb::PrKind::PullResidual, alpha, tol, max_iter, rank_out, iters_out, stats,
                            static_cast<cudaStream_t>(stream));
}

int gb_pagerank_push(gb_graph* g, float alpha, float tol, uint32_t max_iter, float* rank_out,
                     uint32_t* iters_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !rank_out) GB_FAIL(GB_ERR_ARG, "gb_pagerank_push: null argument");
  GB_CUDA(cudaSetDevice(g->device));
  return gb::pagerank_entry(g, gb::PrKind::Push, alpha, tol, max_iter, rank_out, iters_out, stats,
                            static_cast<cudaStream_t>(stream));
}

int gb_pagerank_push_ex(gb_graph* g, int algo, float alpha, float tol, uint32_t max_iter, float* rank_out,
                        uint32_t* iters_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !rank_out) GB_FAIL(GB_ERR_ARG, "gb_pagerank_push_ex: null argument");
  if (algo != GB_PR_PUSH_ASYNC && algo != GB_PR_PUSH_SYNC) GB_FAIL(GB_ERR_ARG, "gb_pagerank_push_ex: unknown algo %d", algo);
  GB_CUDA(cudaSetDevice(g->device));
  return gb::pagerank_entry(g, algo == GB_PR_PUSH_ASYNC ? gb::PrKind::PushAsync : gb::PrKind::Push, alpha, tol,
                            max_iter, rank_out, iters_out, stats, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
