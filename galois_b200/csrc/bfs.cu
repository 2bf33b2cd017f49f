// Breadth-first search, level output.
//
// Reference semantics: lonestar/analytics/cpu/bfs/bfs.cpp:244-293 (SyncTile:
// level-synchronous, `if level[dst]==INF {level[dst]=nextLevel; push}`), with
// the push/pull switch of bfsDirectionOpt.cpp:204-342 (alpha=15, beta=18).
// Levels are unique, so the result is bit-identical to the CPU app whatever
// the schedule.
//
// B200 design: ONE cooperative persistent launch runs every level.  A level is
// either
//   push (top-down): warps grab 32 frontier vertices at a time from the light
//        queue and expand them cooperatively (degree prefix sum + shuffle
//        owner search, coalesced column reads); vertices above heavy_degree
//        were queued as edge tiles of tile_edges arcs, which any warp can take;
//        discovery = check-before-atomicOr on a visited bitmap (2 MB for 16M
//        vertices, L2 resident), warp-aggregated queue appends;
//   pull (bottom-up): every unvisited vertex scans its in-edges until it finds
//        a parent in the frontier bitmap; a warp owns one bitmap word, so the
//        visited and next-frontier words are written with plain stores.
// Every level writes the next frontier bitmap; push levels also fill the
// next queue, and a push level that follows a pull level first converts the
// bitmap into the queue.  The frontier totals that drive the direction switch
// are summed per CTA and added to the global counters once per CTA, so no
// counter is hit by every warp.  Levels are separated by a bounded software
// grid barrier.

#include "device_common.cuh"
#include "device_graph.cuh"
#include "frontier.cuh"

namespace gb {

namespace {

struct BfsCtl {
  GridBar bar;
  int err;
  uint32_t pad0;
  FrontierCounters fc[3];
  unsigned long long scanned;
  uint32_t levels;
  uint32_t pull_levels;
  unsigned long long reached;
  unsigned long long reached_deg;
};

struct BfsArgs {
  const uint64_t* __restrict__ offs;
  const uint32_t* __restrict__ col;
  const uint64_t* __restrict__ in_offs;  // nullptr: push only
  const uint32_t* __restrict__ in_col;
  uint32_t n;
  uint32_t pull_end;  // bottom-up steps scan vertices below it (vertices from it on have no in-arcs)
  uint64_t m;
  uint32_t src;
  uint32_t* level;
  uint32_t* visited;
  uint32_t* fbits[3];
  FrontierQueues fq;
  BfsCtl* ctl;
  uint32_t heavy;
  uint32_t tile;
  float alpha, beta;
  uint32_t max_levels;
};

__global__ void bfs_init(BfsArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t words = (a.n + 31) >> 5;
  for (uint64_t v = tid; v < a.n; v += stride) a.level[v] = (v == a.src) ? 0u : kInf;
  for (uint64_t w = tid; w < words; w += stride) {
    const uint32_t bit = (w == (a.src >> 5)) ? (1u << (a.src & 31)) : 0u;
    a.visited[w] = bit;
    a.fbits[0][w] = bit;
    a.fbits[1][w] = 0;
    a.fbits[2][w] = 0;
  }
  if (tid == 0 && a.src < a.n) {  // src == ~0u: seeded by bfs_seed_many
    const uint64_t b = a.offs[a.src], d = a.offs[a.src + 1] - b;
    FrontierCounters& c = a.ctl->fc[0];
    c.vertices = 1;
    c.degree_sum = d;
    if (d > 0) seed_vertex(a.fq, 0, c, a.src, d, a.heavy, a.tile);
    a.ctl->reached = 1;
    a.ctl->reached_deg = d;
  }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) bfs_persistent(BfsArgs a) {
  BfsCtl* ctl = a.ctl;
  const unsigned nblocks = gridDim.x;
  const uint64_t deadline = kernel_deadline();
  const uint32_t lane = lane_id();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint32_t words = (a.n + 31) >> 5;
  const bool can_pull = a.in_offs != nullptr;

  // direction-optimisation state (bfsDirectionOpt.cpp:247-337), replicated
  // identically in every thread
  int64_t edges_to_check = (int64_t)a.m;
  int pull = 0;
  uint32_t old_items = 0;
  unsigned long long my_scanned = 0;

  // per-level totals of the next frontier, summed per CTA in shared memory
  // and added to the global counters once per CTA
  __shared__ unsigned long long s_cnt[2];
  __shared__ uint32_t s_stage[BLOCK / 32][64];
  if (threadIdx.x == 0) s_cnt[0] = s_cnt[1] = 0;
  __syncthreads();

  for (uint32_t L = 0;; ++L) {
    const int rd = L % 3, wr = (L + 1) % 3, cl = (L + 2) % 3;
    FrontierCounters& cur = ctl->fc[rd];
    FrontierCounters& nxt = ctl->fc[wr];
    const uint32_t items = cur.vertices;
    const unsigned long long scout = cur.degree_sum;
    if (scout == 0) break;  // no frontier vertex has an arc: nothing left to find
    if (L >= a.max_levels) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    // choose the direction for this level
    const int prev_pull = pull;
    if (can_pull) {
      if (!pull) {
        if ((double)scout > (double)edges_to_check / a.alpha) { pull = 1; old_items = 0; }
      } else {
        if (!(items >= old_items || items > a.n / a.beta)) pull = 0;
      }
    }
    if (pull) old_items = items;
    else edges_to_check -= (int64_t)scout;

    if (gtid == 0) {
      ctl->fc[cl] = FrontierCounters{};
      ctl->levels = L + 1;
      if (pull) ctl->pull_levels += 1;
    }
    uint32_t* fb_rd = a.fbits[rd];
    uint32_t* fb_wr = a.fbits[wr];
    uint32_t* fb_cl = a.fbits[cl];
    for (uint64_t w = gtid; w < words; w += gthreads) fb_cl[w] = 0;
    const uint32_t next_level = L + 1;
    uint32_t my_items = 0;
    unsigned long long my_deg = 0;

    if (!pull) {
      // A pull level leaves only the frontier bitmap; a push level after it
      // first turns the bitmap into the queue.
      if (prev_pull) {
        for (uint64_t base = gtid - lane; base < words; base += gthreads) {
          const uint64_t w = base + lane;
          uint32_t bits = w < words ? fb_rd[w] : 0u;
          while (__any_sync(kFull, bits != 0)) {
            const bool has = bits != 0;
            const uint32_t v = has ? (uint32_t)(w << 5) + (uint32_t)(__ffs(bits) - 1) : 0u;
            bits &= bits - 1;
            push_discovered<false>(a.fq, L & 1, cur, has, v, a.offs, a.heavy, a.tile, &ctl->err);
          }
        }
        if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
      }
      const uint32_t q_light = min(cur.light, a.fq.light_cap);
      const uint32_t q_tiles = min(cur.tiles, a.fq.tile_cap);
      WarpStage<64> stage{s_stage[threadIdx.x >> 5], 0u};  // light appends, published per 64
      uint32_t* const nq = a.fq.light[(L + 1) & 1];
      // discovery: all lanes call with their candidate and its visited word
      // as loaded earlier (a stale word only costs an extra atomicOr)
      auto discover = [&](bool cand, uint32_t u, uint32_t vw) {
        bool disc = false;
        if (cand) {
          const uint32_t bit = 1u << (u & 31);
          if (!(vw & bit)) {
            const uint32_t old = atomicOr(&a.visited[u >> 5], bit);
            disc = !(old & bit);
          }
          if (disc) {
            a.level[u] = next_level;
            atomicOr(&fb_wr[u >> 5], bit);
          }
        }
        if (__any_sync(kFull, disc)) {  // most steps discover nothing
          uint64_t d = 0;
          if (disc) d = ldg(a.offs + u + 1) - ldg(a.offs + u);
          my_items += disc ? 1u : 0u;
          my_deg += d;
          stage.push(disc && d > 0 && d <= a.heavy, u, nq, &nxt.light, a.fq.light_cap, &ctl->err);
          push_with_degree<false>(a.fq, (L + 1) & 1, nxt, disc && d > a.heavy, u, d, a.heavy, a.tile, &ctl->err);
        }
      };
      const uint32_t* qin = a.fq.light[L & 1];
      const uint2* tin = a.fq.tiles[L & 1];
      // light vertices 32 per task, heavy vertices' edge tiles one per task,
      // spread statically over all warps (no work-grabbing atomics)
      for_each_frontier_task(
          q_light, q_tiles, gtid >> 5, gthreads >> 5,
          [&](uint32_t base, uint32_t vpt) {
            const uint32_t idx = base + lane;
            uint64_t b = 0;
            uint32_t d = 0;
            if (lane < vpt && idx < q_light) {
              const uint32_t v = qin[idx];
              b = ldg(a.offs + v);
              d = (uint32_t)(ldg(a.offs + v + 1) - b);
            }
            my_scanned += d;
            warp_expand_mlp<4, uint32_t>(
                b, d, 0u, [&](bool valid, uint64_t e, uint32_t) { return valid ? ldg(a.col + e) : 0u; },
                [&](bool valid, uint64_t, uint32_t u, uint32_t) { return valid ? a.visited[u >> 5] : ~0u; },
                [&](bool valid, uint32_t, uint32_t, uint32_t u, uint32_t vw) { discover(valid, u, vw); });
          },
          [&](uint32_t t) {
            const uint2 tv = tin[t];
            const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
            const uint64_t b = vb + (uint64_t)tv.y * a.tile;
            const uint64_t e_end = min(ve, b + a.tile);
            if (lane == 0) my_scanned += e_end - b;
            constexpr int U = 4;
            for (uint64_t e0 = b; e0 < e_end; e0 += 32 * U) {
              uint32_t u[U], vw[U];
              bool valid[U];
#pragma unroll
              for (int k = 0; k < U; ++k) {
                const uint64_t e = e0 + 32 * k + lane;
                valid[k] = e < e_end;
                u[k] = valid[k] ? ldg(a.col + e) : 0u;
              }
#pragma unroll
              for (int k = 0; k < U; ++k) vw[k] = valid[k] ? a.visited[u[k] >> 5] : ~0u;
#pragma unroll
              for (int k = 0; k < U; ++k) discover(valid[k], u[k], vw[k]);
            }
          });
      stage.flush(nq, &nxt.light, a.fq.light_cap, &ctl->err);
    } else {
      // Bottom-up over all vertices; warp-uniform trip count.  A warp owns
      // the 32 vertices of one bitmap word and is the only writer of that
      // word of `visited` and of the next frontier in a pull level, so both
      // are written with plain stores of the warp's ballot.  The next
      // frontier is left as a bitmap (no queue).
      for (uint64_t base = gtid - lane; base < a.pull_end; base += gthreads) {
        const uint64_t u64 = base + lane;
        bool found = false;
        const uint32_t u = (uint32_t)u64;
        const uint32_t vword = base < a.n ? a.visited[base >> 5] : ~0u;
        if (u64 < a.pull_end && !(vword & (1u << lane))) {
          const uint64_t b = ldg(a.in_offs + u), e = ldg(a.in_offs + u + 1);
          uint64_t i = b;
          for (; i < e; ++i) {
            const uint32_t p = ldg(a.in_col + i);
            if (fb_rd[p >> 5] & (1u << (p & 31))) { found = true; ++i; break; }
          }
          my_scanned += i - b;
        }
        const uint32_t m = __ballot_sync(kFull, found);
        if (m) {
          if (lane == 0) {
            a.visited[base >> 5] = vword | m;
            fb_wr[base >> 5] = m;
          }
          if (found) {
            a.level[u] = next_level;
            my_items += 1;
            my_deg += ldg(a.offs + u + 1) - ldg(a.offs + u);
          }
        }
      }
    }
    my_items = warp_sum(my_items);
    my_deg = warp_sum(my_deg);
    if (lane == 0 && my_items) {
      atomicAdd(&s_cnt[0], (unsigned long long)my_items);
      atomicAdd(&s_cnt[1], my_deg);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_cnt[0]) {
        atomicAdd(&nxt.vertices, (uint32_t)s_cnt[0]);
        atomicAdd(&nxt.degree_sum, s_cnt[1]);
      }
      s_cnt[0] = s_cnt[1] = 0;
    }
    if (!grid_barrier(&ctl->bar, nblocks, &ctl->err, deadline)) return;
    if (gtid == 0) {
      ctl->reached += nxt.vertices;
      ctl->reached_deg += nxt.degree_sum;
    }
  }
  my_scanned = warp_sum(my_scanned);
  if (lane == 0 && my_scanned) atomicAdd(&ctl->scanned, my_scanned);
}

}  // namespace

int run_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats, cudaStream_t s,
            void* scratch, size_t scratch_bytes) {
  const gb_tuning t = effective_tuning(g);
  const uint32_t n = g->n;
  const uint32_t words = (n + 31) / 32;
  const bool out_dev = is_device_ptr(level_out);
  FrontierLayout fl = frontier_layout(n, g->m, t.heavy_degree, t.tile_edges);
  size_t need = carve_size<BfsCtl>(1) + 4 * carve_size<uint32_t>(words) + fl.bytes +
                (out_dev ? 0 : carve_size<uint32_t>(n));
  void* base = scratch;
  if (!base) {
    int st = ws_reserve(g, need, s);
    if (st != GB_OK) return st;
    base = g->ws;
  } else if (scratch_bytes < need) {
    GB_FAIL(GB_ERR_CAPACITY, "gb_bfs: scratch of %zu bytes, need %zu", scratch_bytes, need);
  }
  Carver cv(base);
  BfsArgs a{};
  a.ctl = cv.take<BfsCtl>(1);
  a.visited = cv.take<uint32_t>(words);
  for (int i = 0; i < 3; ++i) a.fbits[i] = cv.take<uint32_t>(words);
  a.fq = carve_frontier(cv, fl);
  a.level = out_dev ? level_out : cv.take<uint32_t>(n);
  a.offs = g->offs;
  a.col = g->col;
  const bool allow_pull = t.direction_opt != 2;
  if (allow_pull && g->symmetric) {
    a.in_offs = g->offs;
    a.in_col = g->col;
  } else if (allow_pull && g->t_offs) {
    a.in_offs = g->t_offs;
    a.in_col = g->t_col;
  }
  a.n = n;
  // a symmetric graph's in-arcs are its arcs: on a degree-ordered one the
  // vertices from zero_from on have none, and no bottom-up step finds them
  a.pull_end = g->symmetric && g->perm ? g->zero_from : n;
  a.m = g->m;
  a.src = src;
  a.heavy = t.heavy_degree;
  a.tile = t.tile_edges;
  a.alpha = t.do_alpha;
  a.beta = t.do_beta;
  a.max_levels = n + 1;
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(BfsCtl), s));
  bfs_init<<<g->sm_count * 4, 256, 0, s>>>(a);
  GB_CUDA(cudaGetLastError());
  const void* kfn = reinterpret_cast<const void*>(&bfs_persistent<256>);
  const int grid = coop_grid(g, kfn, 256, 0, t.blocks_per_sm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_bfs: cannot size cooperative grid");
  void* args[] = {&a};
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, 256, args, 0, s));
  kt.stop(s);
  int* pin = static_cast<int*>(g->pinned);
  GB_CUDA(cudaMemcpyAsync(pin, &a.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (stats) {
    BfsCtl* hc = reinterpret_cast<BfsCtl*>(static_cast<char*>(g->pinned) + 256);
    GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    stats->vertices_reached = hc->reached;
    stats->edges_reached = hc->reached_deg;
    stats->edges_scanned = hc->scanned;
    stats->relaxations = hc->reached;
    stats->rounds = hc->levels;
    stats->pull_rounds = hc->pull_levels;
    stats->buckets = 0;
    stats->launches = 2;
    stats->residual = 0;
    stats->kernel_ms = kt.ms();
  }
  if (!out_dev) {
    int st = copy_out(level_out, a.level, sizeof(uint32_t) * n, s);
    if (st != GB_OK) return st;
  }
  if (stats || !out_dev) {
    GB_CUDA(cudaStreamSynchronize(s));
    if (*pin) return dev_err_status(*pin, "gb_bfs");
  }
  return GB_OK;
}

namespace {

// Seeds level 0 with k sources at once (a BFS from a virtual super-source):
// for disjoint graphs packed block-diagonally this gives every graph its own
// BFS levels in one traversal.  Repeated sources are queued once.
__global__ void bfs_seed_many(BfsArgs a, const uint32_t* __restrict__ srcs, uint32_t k) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  FrontierCounters& c = a.ctl->fc[0];
  for (uint64_t base = tid - lane_id(); base < k; base += stride) {
    const uint64_t i = base + lane_id();
    bool first = false;
    uint32_t s = 0;
    if (i < k) {
      s = srcs[i];
      const uint32_t bit = 1u << (s & 31);
      first = !(atomicOr(&a.visited[s >> 5], bit) & bit);
      if (first) {
        a.level[s] = 0;
        atomicOr(&a.fbits[0][s >> 5], bit);
      }
    }
    push_discovered<true>(a.fq, 0, c, first, s, a.offs, a.heavy, a.tile, &a.ctl->err);
  }
}

}  // namespace

// BFS from k sources (device array) into a device level array, asynchronous
// on `s` (no host synchronisation, so it can be captured in a CUDA graph once
// the workspace exists).  Errors raised on the device are returned by the
// next synchronous call on the handle.
int run_bfs_sources(gb_graph* g, const uint32_t* d_srcs, uint32_t k, uint32_t* d_level, cudaStream_t s) {
  const gb_tuning t = effective_tuning(g);
  const uint32_t n = g->n;
  const uint32_t words = (n + 31) / 32;
  FrontierLayout fl = frontier_layout(n, g->m, t.heavy_degree, t.tile_edges);
  const size_t need = carve_size<BfsCtl>(1) + 4 * carve_size<uint32_t>(words) + fl.bytes;
  int st = ws_reserve(g, need, s);
  if (st != GB_OK) return st;
  Carver cv(g->ws);
  BfsArgs a{};
  a.ctl = cv.take<BfsCtl>(1);
  a.visited = cv.take<uint32_t>(words);
  for (int i = 0; i < 3; ++i) a.fbits[i] = cv.take<uint32_t>(words);
  a.fq = carve_frontier(cv, fl);
  a.level = d_level;
  a.offs = g->offs;
  a.col = g->col;
  if (t.direction_opt != 2 && g->symmetric) {
    a.in_offs = g->offs;
    a.in_col = g->col;
  }
  a.n = n;
  a.pull_end = g->symmetric && g->perm ? g->zero_from : n;
  a.m = g->m;
  a.src = 0xFFFFFFFFu;
  a.heavy = t.heavy_degree;
  a.tile = t.tile_edges;
  a.alpha = t.do_alpha;
  a.beta = t.do_beta;
  a.max_levels = n + 1;
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(BfsCtl), s));
  bfs_init<<<g->sm_count * 4, 256, 0, s>>>(a);
  bfs_seed_many<<<std::max<uint32_t>(1, std::min<uint32_t>((k + 255) / 256, g->sm_count * 4)), 256, 0, s>>>(a, d_srcs, k);
  GB_CUDA(cudaGetLastError());
  const void* kfn = reinterpret_cast<const void*>(&bfs_persistent<256>);
  const int grid = coop_grid(g, kfn, 256, 0, t.blocks_per_sm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "bfs: cannot size cooperative grid");
  void* args[] = {&a};
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, 256, args, 0, s));
  // keep the device error word where the caller can read it
  GB_CUDA(cudaMemcpyAsync(static_cast<int*>(g->pinned) + 8, &a.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  return GB_OK;
}

}  // namespace gb

extern "C" int gb_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !level_out) GB_FAIL(GB_ERR_ARG, "gb_bfs: null argument");
  if (src >= g->n) GB_FAIL(GB_ERR_ARG, "gb_bfs: source %u >= n %u", src, g->n);
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g->perm) {
    // relabelled graph: run on internal ids, map the levels back (a stats
    // struct makes run_bfs check the device status before host copies)
    gb_stats local{};
    uint32_t* res = gb::result_buf(g, 0);
    int st = gb::run_bfs(g, g->h_iperm[src], res, stats ? stats : (gb::is_device_ptr(level_out) ? nullptr : &local),
                         s, nullptr, 0);
    if (st != GB_OK) return st;
    if (stats) stats->launches += 1;  // the mapping gather
    return gb::finish_u32(g, res, level_out, s);
  }
  return gb::run_bfs(g, src, level_out, stats, s, nullptr, 0);
}

// ---------------------------------------------------------------------------
// Allocation-free BFS.
//
// Some callers cannot call cudaMalloc: a host application that owns and
// budgets every byte of device memory itself and forbids libraries from
// allocating behind its back, or code that must not take the allocator's
// implicit device synchronisation in the middle of its work.  For them,
// gb_bfs_noalloc runs the same BFS kernels as gb_bfs, but takes the graph as
// caller-owned device arrays (no gb_graph handle, which allocates) and keeps
// its frontier queues, bitmaps and control words in the fixed-size file-scope
// array below.  Every GPU that loads libgb holds that array until the process
// exits.
//
// Limits: n <= kNoAllocMaxNodes (2^20) vertices and m <= kNoAllocMaxArcs
// (2^26) arcs; larger graphs are rejected with GB_ERR_CAPACITY.
// All calls on a device share the one array and it keeps the previous call's
// contents, so each call clears what must start at zero (the control block;
// bitmaps and levels are rewritten by the init kernel).  Calls that overlap
// on the GPU (other streams, other host threads) race on the array and must
// be serialised by the caller.
// Every call looks up the array's device address on the current device with
// cudaGetSymbolAddress (cheap), so no address is kept across calls, devices or
// a cudaDeviceReset.  The call is synchronous: it waits for `stream` to finish
// the validation and the BFS before it returns.
// ---------------------------------------------------------------------------

namespace gb {
namespace {

constexpr uint32_t kNoAllocMaxNodes = 1u << 20;
constexpr uint64_t kNoAllocMaxArcs = 1ull << 26;
constexpr uint32_t kNoAllocHeavy = 512;
constexpr uint32_t kNoAllocTile = 512;

constexpr size_t na_round(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t na_tile_cap() {
  return kNoAllocMaxArcs / kNoAllocTile + kNoAllocMaxArcs / (kNoAllocHeavy + 1) + 2;
}
// control block + validation flag + visited + 3 frontier bitmaps + 2 light
// queues + 2 tile queues, each rounded to 256 bytes like Carver does
constexpr size_t kNoAllocScratchBytes =
    na_round(sizeof(BfsCtl)) + na_round(sizeof(int)) + 4 * na_round(sizeof(uint32_t) * (kNoAllocMaxNodes / 32)) +
    2 * na_round(sizeof(uint32_t) * kNoAllocMaxNodes) + 2 * na_round(sizeof(uint2) * na_tile_cap());

static __device__ __align__(256) unsigned char g_bfs_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array on the current device.  Host code sees
// only a host-side stand-in under the array's name, never the device address,
// so the symbol itself must never be passed to a kernel.
int noalloc_scratch(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_bfs_noalloc_scratch);
  if (e != cudaSuccess || !p) return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
  *out = p;
  return GB_OK;
}

// GB_OK if p is device (or managed) memory that the current device `dev` can
// address as its own; a pointer into another GPU's memory would make the
// kernels fault instead of returning an error.
int noalloc_check_ptr(const void* p, const char* what, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    GB_FAIL(GB_ERR_ARG, "gb_bfs_noalloc: %s is not device memory", what);
  }
  if (at.type == cudaMemoryTypeManaged) return GB_OK;
  if (at.type != cudaMemoryTypeDevice) GB_FAIL(GB_ERR_ARG, "gb_bfs_noalloc: %s is not device memory", what);
  if (at.device != dev)
    GB_FAIL(GB_ERR_ARG, "gb_bfs_noalloc: %s lives on device %d, the current device is %d", what, at.device, dev);
  return GB_OK;
}

__global__ void noalloc_validate(const uint64_t* __restrict__ offs, const uint32_t* __restrict__ col, uint32_t n,
                                 uint64_t m, int* bad) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if (tid == 0 && (offs[0] != 0 || offs[n] != m)) atomicOr(bad, 1);
  for (uint64_t v = tid; v < n; v += stride)
    if (offs[v] > offs[v + 1]) atomicOr(bad, 1);
  for (uint64_t e = tid; e < m; e += stride)
    if (col[e] >= n) atomicOr(bad, 2);
}

}  // namespace
}  // namespace gb

extern "C" int gb_bfs_noalloc(const uint64_t* offs, const uint32_t* col, uint32_t n, uint64_t m, int symmetric,
                              uint32_t src, uint32_t* level_out, void* stream) {
  using namespace gb;
  clear_error();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!offs || !col || !level_out) GB_FAIL(GB_ERR_ARG, "gb_bfs_noalloc: null argument");
  if (n == 0 || src >= n) GB_FAIL(GB_ERR_ARG, "gb_bfs_noalloc: source %u not below n %u", src, n);
  if (n > kNoAllocMaxNodes || m > kNoAllocMaxArcs)
    GB_FAIL(GB_ERR_CAPACITY, "gb_bfs_noalloc: graph of %u vertices / %llu arcs exceeds the fixed scratch "
            "(at most %u vertices and %llu arcs); use gb_bfs", n, (unsigned long long)m, kNoAllocMaxNodes,
            (unsigned long long)kNoAllocMaxArcs);
  int dev = 0, sms = 0;
  GB_CUDA(cudaGetDevice(&dev));
  int st = noalloc_check_ptr(offs, "offs", dev);
  if (st == GB_OK) st = noalloc_check_ptr(col, "col", dev);
  if (st == GB_OK) st = noalloc_check_ptr(level_out, "level_out", dev);
  if (st != GB_OK) return st;
  void* base = nullptr;
  st = noalloc_scratch(&base);
  if (st != GB_OK) return st;
  const uint32_t words = (n + 31) / 32;
  const FrontierLayout fl = frontier_layout(n, m, kNoAllocHeavy, kNoAllocTile);
  const size_t need = carve_size<BfsCtl>(1) + carve_size<int>(1) + 4 * carve_size<uint32_t>(words) + fl.bytes;
  if (need > kNoAllocScratchBytes) GB_FAIL(GB_ERR_CAPACITY, "gb_bfs_noalloc: scratch too small (%zu > %zu)", need,
                                           kNoAllocScratchBytes);
  Carver cv(base);
  BfsArgs a{};
  a.ctl = cv.take<BfsCtl>(1);
  int* bad = cv.take<int>(1);
  a.visited = cv.take<uint32_t>(words);
  for (int i = 0; i < 3; ++i) a.fbits[i] = cv.take<uint32_t>(words);
  a.fq = carve_frontier(cv, fl);
  a.level = level_out;
  a.offs = offs;
  a.col = col;
  if (symmetric) {
    a.in_offs = offs;
    a.in_col = col;
  }
  a.n = n;
  a.pull_end = n;
  a.m = m;
  a.src = src;
  a.heavy = kNoAllocHeavy;
  a.tile = kNoAllocTile;
  a.alpha = 15.f;
  a.beta = 18.f;
  a.max_levels = n + 1;
  GB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // the array keeps the previous call's contents: clear the control block and
  // the validation flag (bitmaps and levels are rewritten by bfs_init)
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(BfsCtl), s));
  GB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
  noalloc_validate<<<sms * 4, 256, 0, s>>>(offs, col, n, m, bad);
  GB_CUDA(cudaGetLastError());
  int hbad = 0;
  GB_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  GB_CUDA(cudaStreamSynchronize(s));
  if (hbad) GB_FAIL(GB_ERR_FORMAT, "gb_bfs_noalloc: invalid CSR (offsets not monotone / not ending at m, or id >= n)");
  bfs_init<<<sms * 4, 256, 0, s>>>(a);
  GB_CUDA(cudaGetLastError());
  const void* kfn = reinterpret_cast<const void*>(&bfs_persistent<256>);
  int per_sm = 0;
  GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, 256, 0));
  if (per_sm <= 0) GB_FAIL(GB_ERR_CUDA, "gb_bfs_noalloc: cannot size cooperative grid");
  void* args[] = {&a};
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, per_sm * sms, 256, args, 0, s));
  int herr = 0;
  GB_CUDA(cudaMemcpyAsync(&herr, &a.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  GB_CUDA(cudaStreamSynchronize(s));
  if (herr) return dev_err_status(herr, "gb_bfs_noalloc");
  return GB_OK;
}
