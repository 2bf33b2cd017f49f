// Connected components with minimum-id labels.
//
// Reference semantics: lonestar/analytics/cpu/connected-components/
// ConnectedComponents.cpp:183-230 (LabelPropAlgo: comp_current starts at the
// vertex id, min-labels propagate over edges until nothing changes), init
// :1162-1172, verify :1046-1072.  LabelProp converges to the minimum vertex id
// of each component; every algorithm here produces exactly that labelling.
//
// Algorithms (one cooperative persistent launch each, rounds separated by the
// bounded grid barrier):
//   GB_CC_LABELPROP  label propagation with pointer jumping: per round, every
//                    edge (v,u) hooks the larger of (p[v], p[u]) under the
//                    smaller with atomicMin, then every vertex jumps to its
//                    root.  p[x] <= x always holds and sum(p) strictly drops
//                    while anything changes, so it terminates with p = min id.
//                    On a symmetric graph rounds after the first scan only
//                    the vertices outside the sampled giant component.
//   GB_CC_UNIONFIND  one sweep of lock-free union-find (larger root linked
//                    under the smaller with atomicCAS, path halving), then a
//                    compression sweep.  Same labels.
//   GB_CC_AFFOREST   neighbour sampling (first 2 arcs of every vertex), a
//                    compression, detection of the most frequent root, then
//                    union-find only over vertices outside that component.
// On a symmetric graph each undirected edge is processed once (u > v) in a
// full sweep; on a directed graph every arc is processed, giving weakly
// connected components.

#include "device_common.cuh"
#include "device_graph.cuh"
#include "sweep.cuh"

namespace gb {

namespace {

struct CcCtl {
  GridBar bar;
  int err;
  uint32_t changed[3];
  uint32_t rounds;
  uint32_t giant;
  uint32_t pad;
  unsigned long long scanned;
};

struct CcArgs {
  const uint64_t* __restrict__ offs;
  const uint32_t* __restrict__ col;
  uint32_t n;
  int half;    // process only u < v (symmetric graph)
  int sorted;  // rows sorted ascending (relabelled graphs): a row's u < v arcs are its prefix
  uint32_t vend;  // rows from vend on are empty (degree-ordered graphs; else n)
  uint32_t* p;
  SweepSched sched;
  CcCtl* ctl;
  uint32_t* hist;  // Afforest root histogram sample
  uint32_t max_rounds;
};

__global__ void cc_init(uint32_t* p, uint32_t n) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride) p[v] = (uint32_t)v;
}

__device__ __forceinline__ uint32_t find_root(uint32_t* p, uint32_t x) {
  uint32_t px = p[x];
  while (px != x) {
    const uint32_t ppx = p[px];
    if (ppx != px) p[x] = ppx;  // path halving (benign race: ancestors only)
    x = px;
    px = ppx;
  }
  return x;
}

// Link the trees of a and b: larger root goes under the smaller (ECL-CC style).
__device__ __forceinline__ void link(uint32_t* p, uint32_t a, uint32_t b) {
  uint32_t ra = find_root(p, a), rb = find_root(p, b);
  for (int guard = 0; ra != rb && guard < (1 << 20); ++guard) {
    if (ra < rb) {
      const uint32_t ret = atomicCAS(&p[rb], rb, ra);
      if (ret == rb) break;
      rb = find_root(p, ret);
    } else {
      const uint32_t ret = atomicCAS(&p[ra], ra, rb);
      if (ret == ra) break;
      ra = find_root(p, ret);
    }
  }
}

__device__ __forceinline__ void compress_all(CcArgs& a, uint64_t gtid, uint64_t gthreads) {
  // on a symmetric graph a vertex without arcs keeps its own label
  const uint32_t vn = a.half ? a.vend : a.n;
  for (uint64_t v = gtid; v < vn; v += gthreads) {
    uint32_t x = a.p[v];
    while (x != a.p[x]) x = a.p[x];
    a.p[v] = x;
  }
}

// Most frequent label among BLOCK evenly spaced vertices (Afforest's estimate
// of the giant component), written to ctl->giant.  Called by every thread of
// one CTA, one sample each (1024 samples with 1024 comparisons per sample
// kept the other CTAs waiting 75 us on RMAT-24; any label is correct, the
// estimate only decides which rows the next round may skip).
template <int BLOCK>
__device__ void sample_giant(const CcArgs& a, CcCtl* ctl) {
  __shared__ uint32_t s_root[BLOCK];
  __shared__ uint32_t s_best[2];
  const uint32_t i = threadIdx.x;
  s_root[i] = a.p[(uint32_t)(((uint64_t)i * a.vend) / BLOCK)];  // vertices with arcs
  if (i == 0) s_best[0] = s_best[1] = 0;
  __syncthreads();
  uint32_t c = 0;
  for (uint32_t j = 0; j < BLOCK; ++j) c += s_root[j] == s_root[i];
  // the count in the high bits, the sample's index in the low: one atomicMax
  atomicMax(&s_best[0], (c << 16) | (BLOCK - 1 - i));
  __syncthreads();
  if (i == 0) ctl->giant = s_root[BLOCK - 1 - (s_best[0] & 0xFFFFu)];
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) cc_labelprop(CcArgs a) {
  CcCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  unsigned long long my_scanned = 0;
  // After the first round (and its compression) every label is a root.  On a
  // symmetric graph a later round then scans only the rows of vertices whose
  // label is not the sampled giant label, each in full (both arc directions):
  // an arc whose ends disagree has at least one end outside the giant
  // component, and that end's row holds it (the skip Afforest makes,
  // applied to label propagation).  Most vertices join the giant component
  // in the first round, so the confirming round reads few arcs.
  uint32_t giant = 0xFFFFFFFFu;
  for (uint32_t r = 0;; ++r) {
    if (r >= a.max_rounds) {
      if (gtid == 0) raise_err(&ctl->err, kDevMaxRounds);
      break;
    }
    const bool skip_giant = a.half && r >= 1;
    // the first sweep of a symmetric graph takes each edge once, as its arc
    // u < v: on a degree-ordered graph that is a prefix of a hub's row (its
    // neighbours of higher degree), and the gathered labels are the hubs'
    const bool all_dirs = !a.half || skip_giant;  // arcs u > v too
    uint32_t* changed = &ctl->changed[r % 3];
    if (gtid == 0) ctl->changed[(r + 1) % 3] = 0;
    bool my_change = false;
    // Hook labels pv (of v, read once per vertex; a stale value is still a
    // label of v's component, so the union stays valid) and pu: the larger
    // goes under the smaller, checked before the atomic.
    // When hi already hangs under another label c (p[hi] = c, read first,
    // or returned by the atomic), the arc also joins c and lo, so the hook
    // goes on with that pair: a label read once per row may be stale, and
    // without this a vertex between two hubs would leave their trees apart
    // for another round.  The larger of the pair falls every step (p[x] <= x);
    // a pair still apart after 4 steps marks the round changed, and the next
    // round scans a row of it (its two labels differ after the compression,
    // so at most one is the giant one).
    auto hook = [&](bool valid, uint32_t pv, uint32_t pu) {
      if (!valid) return;
      uint32_t x = pv, y = pu;
      for (int step = 0; x != y; ++step) {
        if (step == 4) {
          my_change = true;
          return;
        }
        const uint32_t hi = max(x, y), lo = min(x, y);
        const uint32_t c = a.p[hi];
        if (c == lo) return;
        if (c < lo) {
          x = c, y = lo;  // hi is under c already: join c and lo
          continue;
        }
        const uint32_t old = atomicMin(&a.p[hi], lo);
        if (old > lo) my_change = true;
        if (old == hi || old == lo) return;  // hi was a root, or is under lo already
        x = old, y = lo;                     // hi hung under old: join old and lo
      }
    };
    // Tasks as in sweep.cuh: 32-vertex chunks, then heavy-vertex tiles.  In
    // a chunk each lane reads its vertex's label once; the expansion (4 steps
    // of column and label loads in flight) takes the owner's label by shuffle.
    const uint64_t nchunks = ((uint64_t)a.vend + 31) >> 5;  // rows from vend on are empty
    const uint64_t total = nchunks + a.sched.ntiles;
    // one tile of a heavy row: 8 column loads, then 8 label loads, per lane
    auto tile_fn = [&](uint32_t v, uint64_t b, uint64_t e) {
      // a sorted row's u < v arcs end before the first u >= v
      if (!all_dirs && a.sorted && ldg(a.col + b) >= v) return;  // warp-uniform
      const uint32_t pv = a.p[v];
      if (skip_giant && pv == giant) return;  // warp-uniform
      constexpr int UT = 8;
      for (uint64_t i0 = b; i0 < e; i0 += 32 * UT) {
        if (i0 > b && !all_dirs && a.sorted && ldg(a.col + i0) >= v) break;  // warp-uniform
        if (lane == 0) my_scanned += e - i0 < 32 * UT ? e - i0 : (uint64_t)(32 * UT);  // the arcs read
        uint32_t u[UT], pu[UT];
#pragma unroll
        for (int k = 0; k < UT; ++k) {
          const uint64_t i = i0 + lane + 32 * k;
          const uint32_t x = i < e ? ldg(a.col + i) : 0u;
          u[k] = (i < e && (all_dirs || x < v)) ? x : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int k = 0; k < UT; ++k) pu[k] = u[k] != 0xFFFFFFFFu ? a.p[u[k]] : 0u;
#pragma unroll
        for (int k = 0; k < UT; ++k) hook(u[k] != 0xFFFFFFFFu, pv, pu[k]);
      }
    };
    for (uint64_t t = gwarp; t < total; t += nwarps) {
      if (t < nchunks) {
        const uint64_t v64 = (t << 5) + lane;
        uint64_t b = 0;
        uint32_t d = 0, pv = 0;
        bool mine = false;
        if (v64 < a.vend) {
          pv = a.p[v64];
          mine = !(skip_giant && pv == giant);
        }
        // a later round reads a chunk's labels first: most chunks lie inside
        // the giant label and need no offsets
        if (skip_giant && !__any_sync(kFull, mine)) continue;  // warp-uniform
        if (mine) {
          b = ldg(a.offs + v64);
          const uint64_t dd = ldg(a.offs + v64 + 1) - b;
          d = dd > a.sched.heavy ? 0u : (uint32_t)dd;
        }
        my_scanned += d;
        warp_expand_mlp<4, uint32_t>(
            b, d, (uint32_t)v64,
            [&](bool valid, uint64_t e, uint32_t v) {
              const uint32_t u = valid ? ldg(a.col + e) : 0u;
              return (valid && (all_dirs || u < v)) ? u : 0xFFFFFFFFu;
            },
            [&](bool, uint64_t, uint32_t u, uint32_t) { return u != 0xFFFFFFFFu ? a.p[u] : 0u; },
            [&](bool, uint32_t owner, uint32_t, uint32_t u, uint32_t pu) {
              const uint32_t opv = __shfl_sync(kFull, pv, owner);
              hook(u != 0xFFFFFFFFu, opv, pu);
            });
      } else {
        const uint2 tv = a.sched.tiles[t - nchunks];
        const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
        const uint64_t tb = vb + (uint64_t)tv.y * a.sched.tile;
        tile_fn(tv.x, tb, min(ve, tb + a.sched.tile));
      }
    }
    // read before the atomic: every warp changes something in the first sweep
    if (__any_sync(kFull, my_change) && lane == 0 && *reinterpret_cast<volatile uint32_t*>(changed) == 0)
      atomicOr(changed, 1u);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    if (gtid == 0) ctl->rounds = r + 1;
    // a round that hooked nothing leaves every label a root already
    if (*reinterpret_cast<volatile uint32_t*>(changed) == 0) break;
    compress_all(a, gtid, gthreads);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    if (r == 0 && a.half) {
      if (blockIdx.x == 0) sample_giant<BLOCK>(a, ctl);
      if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
      giant = *reinterpret_cast<volatile uint32_t*>(&ctl->giant);
    }
  }
  my_scanned = warp_sum(my_scanned);
  if (lane == 0 && my_scanned) atomicAdd(&ctl->scanned, my_scanned);
}

// Union-find: mode 0 = all arcs; mode 1 = Afforest (sample, then the rest).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) cc_unionfind(CcArgs a, int afforest) {
  CcCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)BLOCK + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * BLOCK;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  constexpr uint32_t kSamples = 2;
  uint32_t giant = 0xFFFFFFFFu;
  if (afforest) {
    // 1. neighbour sampling: link every vertex with its first kSamples arcs
    for (uint64_t v = gtid; v < a.n; v += gthreads) {
      const uint64_t b = ldg(a.offs + v), e = ldg(a.offs + v + 1);
      for (uint64_t i = b; i < e && i < b + kSamples; ++i) link(a.p, (uint32_t)v, ldg(a.col + i));
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    compress_all(a, gtid, gthreads);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    // 2. most frequent root among 1024 evenly spaced vertices
    if (blockIdx.x == 0) sample_giant<BLOCK>(a, ctl);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    giant = *reinterpret_cast<volatile uint32_t*>(&ctl->giant);
  }
  unsigned long long my_scanned = 0;
  // 3. union-find over all remaining arcs (Afforest: skip vertices already in
  //    the giant component and the arcs already sampled)
  auto skip_vertex = [&](uint32_t v) { return afforest && a.p[v] == giant; };
  sweep_all(
      a.offs, a.n, a.sched, gwarp, nwarps,
      [&](bool valid, uint64_t e, uint32_t, uint32_t v) {
        if (!valid) return;
        const uint32_t u = ldg(a.col + e);
        if (a.half && !afforest && u < v) return;
        if (afforest && (skip_vertex(v) || e < ldg(a.offs + v) + kSamples)) return;
        link(a.p, v, u);
      },
      [&](uint32_t, bool, bool) {},
      [&](uint32_t v, uint64_t b, uint64_t e) {
        if (afforest && skip_vertex(v)) return;
        if (lane == 0) my_scanned += e - b;
        const uint64_t b0 = ldg(a.offs + v);
        for (uint64_t i = b + lane; i < e; i += 32) {
          const uint32_t u = ldg(a.col + i);
          if (a.half && !afforest && u < v) continue;
          if (afforest && i < b0 + kSamples) continue;
          link(a.p, v, u);
        }
      });
  if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
  compress_all(a, gtid, gthreads);
  if (gtid == 0) ctl->rounds = 1;
  my_scanned = warp_sum(my_scanned);
  if (lane == 0 && my_scanned) atomicAdd(&ctl->scanned, my_scanned);
}

}  // namespace

int run_cc(gb_graph* g, int algo, uint32_t* label_out, gb_stats* stats, cudaStream_t s) {
  if (algo < 0 || algo > 2) GB_FAIL(GB_ERR_ARG, "gb_cc: unknown algo %d", algo);
  if (algo == GB_CC_AFFOREST && !g->symmetric)
    GB_FAIL(GB_ERR_UNSUPPORTED, "gb_cc: Afforest needs a symmetric graph (it skips the giant component's arcs)");
  const gb_tuning t = effective_tuning(g);
  const uint32_t n = g->n;
  const bool out_dev = is_device_ptr(label_out);
  SweepSched sched;
  int st = ensure_sweep_schedule(g, t.heavy_degree, t.tile_edges, s, &sched);
  if (st != GB_OK) return st;
  const size_t need = carve_size<CcCtl>(1) + carve_size<uint32_t>(1024) + (out_dev ? 0 : carve_size<uint32_t>(n));
  st = ws_reserve(g, need, s);
  if (st != GB_OK) return st;
  Carver cv(g->ws);
  CcArgs a{};
  a.ctl = cv.take<CcCtl>(1);
  a.hist = cv.take<uint32_t>(1024);
  a.p = out_dev ? label_out : cv.take<uint32_t>(n);
  a.offs = g->offs;
  a.col = g->col;
  a.n = n;
  a.half = g->symmetric ? 1 : 0;
  a.sorted = (g->perm && g->order != GB_ORDER_DEGREE_UNSORTED && g->m < (1ull << 31)) ? 1 : 0;
  a.vend = g->perm ? std::max<uint32_t>(g->zero_from, 1u) : n;
  a.sched = sched;
  a.max_rounds = 1u << 20;
  GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(CcCtl), s));
  cc_init<<<g->sm_count * 4, 256, 0, s>>>(a.p, n);
  GB_CUDA(cudaGetLastError());
  const void* kfn = algo == GB_CC_LABELPROP ? reinterpret_cast<const void*>(&cc_labelprop<256>)
                                            : reinterpret_cast<const void*>(&cc_unionfind<256>);
  const int grid = coop_grid(g, kfn, 256, 0, t.blocks_per_sm);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_cc: cannot size cooperative grid");
  int aff = algo == GB_CC_AFFOREST ? 1 : 0;
  void* args_lp[] = {&a};
  void* args_uf[] = {&a, &aff};
  KernelTimer kt(stats != nullptr, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, 256, algo == GB_CC_LABELPROP ? args_lp : args_uf, 0, s));
  kt.stop(s);
  int* pin = static_cast<int*>(g->pinned);
  GB_CUDA(cudaMemcpyAsync(pin, &a.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (stats) {
    CcCtl* hc = reinterpret_cast<CcCtl*>(static_cast<char*>(g->pinned) + 256);
    GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(CcCtl), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    *stats = gb_stats{};
    stats->vertices_reached = n;
    stats->edges_reached = g->m;
    stats->edges_scanned = hc->scanned;
    stats->rounds = hc->rounds;
    stats->launches = 2;
    stats->kernel_ms = kt.ms();
  }
  if (!out_dev) {
    st = copy_out(label_out, a.p, sizeof(uint32_t) * n, s);
    if (st != GB_OK) return st;
  }
  if (stats || !out_dev) {
    GB_CUDA(cudaStreamSynchronize(s));
    if (*pin) return dev_err_status(*pin, "gb_cc");
  }
  return GB_OK;
}

}  // namespace gb

extern "C" int gb_cc(gb_graph* g, int algo, uint32_t* label_out, gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !label_out) GB_FAIL(GB_ERR_ARG, "gb_cc: null argument");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g->perm) {
    // labels come back as min internal ids; finish_labels makes them the
    // min ORIGINAL id of each component
    gb_stats local{};
    uint32_t* res = gb::result_buf(g, 0);
    int st = gb::run_cc(g, algo, res, stats ? stats : (gb::is_device_ptr(label_out) ? nullptr : &local), s);
    if (st != GB_OK) return st;
    if (stats) stats->launches += 2;  // component minimum + mapping
    return gb::finish_labels(g, res, label_out, s);
  }
  return gb::run_cc(g, algo, label_out, stats, s);
}
