// Brandes betweenness centrality, Level variant, single- and multi-source.
//
// Reference semantics: lonestar/analytics/cpu/betweennesscentrality/
// LevelStructs.h:87-185 per source: forward level-synchronous BFS counting
// shortest paths (sigma, fp64 -- LevelShortPathType = double, :16), then a
// backward sweep over the levels from the second-to-last down to 1:
// dep[v] = sigma[v] * sum_{w succ of v} (1 + dep[w]) / sigma[w], bc[v] += dep[v]
// (fp32 dependency/bc, :20-25; the source and the last level add nothing).
// Sources are processed one at a time in the reference (doLevelBC :224-326).
//
// B200 design:
//  * batch == 1 ("plain" kernel, looped per source): one persistent launch
//    per source; push-style forward over frontier queues (CAS on the level,
//    fp64 atomicAdd of sigma, as LevelSSSP does), every level's queue kept in
//    an append-only order array (the stack of worklists), backward sweep over
//    those level ranges with per-owner segmented reductions.
//  * batch 2..64 (multi-source, cf. MRBC's source batching in
//    lonestar/analytics/distributed/betweennesscentrality/bc_mr.cpp:84-158):
//    per vertex and level a 64-bit mask of the sources that reach it at that
//    level; sigma (fp64) and dep (fp32) stored vertex-major [n][64] so lane s
//    of a warp owns source s and s+32 and a row is one coalesced load.
//    Forward levels pull: a vertex still missing sources scans its neighbours
//    32 at a time, a ballot keeps the neighbours in the frontier for a needed
//    source, and only those rows of sigma are read.  Backward levels walk the
//    stored masks.  Light vertices are owned by one warp (no atomics); heavy
//    vertices are split into tiles that combine with atomics.
//  bc accumulates in fp64 across sources and batches; the output is fp32.

#include "device_common.cuh"
#include "device_graph.cuh"
#include "frontier.cuh"
#include "sweep.cuh"

#include <algorithm>
#include <vector>

namespace gb {

namespace {

constexpr int kBcBlock = 1024;
constexpr uint32_t kBcInf = 0xFFFFFFFFu / 4;  // BetweennessCentrality.cpp:32

struct BcCtl {
  GridBar bar;
  int err;
  uint32_t levels;
  uint32_t any[4];  // per-level "something reached" flags (ring)
  uint32_t level_needed;
  uint32_t pad;
  unsigned long long scanned;
};

// ---------------------------------------------------------------- batched --
struct MsArgs {
  const uint64_t* __restrict__ offs;  // successors (out-edges)
  const uint32_t* __restrict__ col;
  const uint64_t* __restrict__ in_offs;  // predecessors (in-edges)
  const uint32_t* __restrict__ in_col;
  uint32_t n;
  uint32_t nsrc;  // sources in this batch (<= 64)
  const uint32_t* srcs;
  unsigned long long* lm;  // [lcap][n] level masks
  uint32_t lcap;
  unsigned long long* visit;  // [n]
  double* sigma;              // [n][64]
  float* dep;                 // [n][64]
  double* bc;                 // [n]
  double* hacc;               // [2][nheavy][64] backward partial sums of heavy vertices; level L adds
                              // into half L & 1 and zeroes the other half (a store to a word this
                              // level's atomics just updated stalls)
  uint32_t* hidx;             // [n] heavy-list index of a heavy vertex
  SweepSched fs;              // heavy schedule over in-edges (forward)
  SweepSched bs;              // heavy schedule over out-edges (backward)
  BcCtl* ctl;
};

__device__ __forceinline__ unsigned long long shfl64(unsigned long long x, int k) {
  return __shfl_sync(kFull, x, k);
}

__global__ void ms_init(MsArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < (uint64_t)a.n * 64; i += stride) {
    a.sigma[i] = 0.0;
    a.dep[i] = 0.f;
  }
  for (uint64_t i = tid; i < (uint64_t)a.lcap * a.n; i += stride) a.lm[i] = 0ull;
  for (uint64_t v = tid; v < a.n; v += stride) a.visit[v] = 0ull;
  for (uint64_t i = tid; i < 2ull * a.bs.nheavy * 64; i += stride) a.hacc[i] = 0.0;
  for (uint64_t i = tid; i < a.bs.nheavy; i += stride) a.hidx[a.bs.heavy_list[i]] = (uint32_t)i;
}

__global__ void ms_seed(MsArgs a) {
  // one thread: sources may repeat, each gets its own bit
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (uint32_t b = 0; b < a.nsrc; ++b) {
      const uint32_t s = a.srcs[b];
      a.lm[s] |= 1ull << b;
      a.visit[s] |= 1ull << b;
      a.sigma[(uint64_t)s * 64 + b] = 1.0;
    }
  }
}

// Forward work for one (vertex, arc range) by a whole warp.  Returns the
// newly reached source mask; sA/sB receive the sigma sums for sources lane
// and lane+32.
__device__ __forceinline__ unsigned long long ms_forward_range(const MsArgs& a, const unsigned long long* cur,
                                                               unsigned long long need, uint64_t b, uint64_t e,
                                                               double& sA, double& sB) {
  const uint32_t lane = lane_id();
  unsigned long long acc = 0;
  for (uint64_t base = b; base < e; base += 32) {
    const uint64_t j = base + lane;
    uint32_t v = 0;
    unsigned long long f = 0;
    if (j < e) {
      v = ldg(a.in_col + j);
      f = cur[v] & need;
    }
    unsigned hits = __ballot_sync(kFull, f != 0);
    while (hits) {
      const int k = __ffs(hits) - 1;
      hits &= hits - 1;
      const uint32_t vk = __shfl_sync(kFull, v, k);
      const unsigned long long fk = shfl64(f, k);
      acc |= fk;
      const double* row = a.sigma + (uint64_t)vk * 64;
      if ((fk >> lane) & 1ull) sA += row[lane];
      if ((fk >> (lane + 32)) & 1ull) sB += row[lane + 32];
    }
  }
  return acc;
}

// Backward work for one (vertex, arc range): sums (1+dep[w])/sigma[w] over
// successors w for the sources in cv.
__device__ __forceinline__ void ms_backward_range(const MsArgs& a, const unsigned long long* nextl,
                                                  unsigned long long cv, uint64_t b, uint64_t e, double& dA,
                                                  double& dB) {
  const uint32_t lane = lane_id();
  for (uint64_t base = b; base < e; base += 32) {
    const uint64_t j = base + lane;
    uint32_t w = 0;
    unsigned long long g = 0;
    if (j < e) {
      w = ldg(a.col + j);
      g = nextl[w] & cv;
    }
    unsigned hits = __ballot_sync(kFull, g != 0);
    while (hits) {
      const int k = __ffs(hits) - 1;
      hits &= hits - 1;
      const uint32_t wk = __shfl_sync(kFull, w, k);
      const unsigned long long gk = shfl64(g, k);
      const uint64_t r = (uint64_t)wk * 64;
      if ((gk >> lane) & 1ull) dA += (1.0 + (double)a.dep[r + lane]) / a.sigma[r + lane];
      if ((gk >> (lane + 32)) & 1ull) dB += (1.0 + (double)a.dep[r + lane + 32]) / a.sigma[r + lane + 32];
    }
  }
}

// Lanes filter 32 consecutive vertices; the warp then serves the selected
// ones one by one.  fn(v) is called by the whole warp.
template <class Fn>
__device__ __forceinline__ void ms_for_light(const MsArgs& a, const SweepSched& s, const uint64_t* offs,
                                             uint64_t gwarp, uint64_t nwarps, Fn&& select_and_run) {
  const uint32_t lane = lane_id();
  const uint64_t nchunks = ((uint64_t)a.n + 31) >> 5;
  for (uint64_t c = gwarp; c < nchunks; c += nwarps) {
    const uint64_t v = (c << 5) + lane;
    bool light = false;
    if (v < a.n) light = ldg(offs + v + 1) - ldg(offs + v) <= s.heavy;
    select_and_run((uint32_t)v, v < a.n && light);
  }
}

__global__ void __launch_bounds__(kBcBlock) ms_persistent(MsArgs a) {
  BcCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kBcBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kBcBlock;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  const unsigned long long active = a.nsrc >= 64 ? ~0ull : ((1ull << a.nsrc) - 1ull);
  // ---- forward: level masks and path counts ----------------------------------
  uint32_t L = 0;
  for (;; ++L) {
    if (L + 1 >= a.lcap) {
      if (gtid == 0) {
        ctl->level_needed = L + 2;
        raise_err(&ctl->err, kDevOverflow);
      }
      return;
    }
    const unsigned long long* cur = a.lm + (uint64_t)L * a.n;
    unsigned long long* nxt = a.lm + (uint64_t)(L + 1) * a.n;
    if (gtid == 0) ctl->any[(L + 2) & 3] = 0;
    ms_for_light(a, a.fs, a.in_offs, gwarp, nwarps, [&](uint32_t v, bool light) {
      const unsigned long long need = light ? (~a.visit[v] & active) : 0ull;
      unsigned sel = __ballot_sync(kFull, need != 0);
      while (sel) {
        const int k = __ffs(sel) - 1;
        sel &= sel - 1;
        const uint32_t vk = __shfl_sync(kFull, v, k);
        const unsigned long long nk = shfl64(need, k);
        double sA = 0.0, sB = 0.0;
        const unsigned long long acc =
            ms_forward_range(a, cur, nk, ldg(a.in_offs + vk), ldg(a.in_offs + vk + 1), sA, sB);
        if (acc) {
          if (lane == 0) nxt[vk] = acc;
          double* row = a.sigma + (uint64_t)vk * 64;
          if ((acc >> lane) & 1ull) row[lane] = sA;
          if ((acc >> (lane + 32)) & 1ull) row[lane + 32] = sB;
        }
      }
    });
    for (uint64_t t = gwarp; t < a.fs.ntiles; t += nwarps) {
      const uint2 tv = a.fs.tiles[t];
      const unsigned long long need = ~a.visit[tv.x] & active;
      if (!need) continue;
      const uint64_t vb = ldg(a.in_offs + tv.x), ve = ldg(a.in_offs + tv.x + 1);
      const uint64_t b = vb + (uint64_t)tv.y * a.fs.tile, e = min(ve, b + a.fs.tile);
      double sA = 0.0, sB = 0.0;
      const unsigned long long acc = ms_forward_range(a, cur, need, b, e, sA, sB);
      if (acc) {
        if (lane == 0) atomicOr(&nxt[tv.x], acc);
        double* row = a.sigma + (uint64_t)tv.x * 64;
        if ((acc >> lane) & 1ull) atomicAdd(&row[lane], sA);
        if ((acc >> (lane + 32)) & 1ull) atomicAdd(&row[lane + 32], sB);
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    bool my_any = false;
    for (uint64_t v = gtid; v < a.n; v += gthreads) {
      const unsigned long long x = nxt[v];
      if (x) {
        a.visit[v] |= x;
        my_any = true;
      }
    }
    if (__any_sync(kFull, my_any) && lane == 0) atomicOr(&ctl->any[L & 3], 1u);
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    if (*reinterpret_cast<volatile uint32_t*>(&ctl->any[L & 3]) == 0) break;
  }
  const uint32_t nlev = L + 1;  // levels 0..L are non-empty
  // ---- backward: dependencies, levels nlev-2 .. 1 (LevelStructs.h:147-183) --
  for (int Lb = (int)nlev - 2; Lb >= 1; --Lb) {
    const unsigned long long* cur = a.lm + (uint64_t)Lb * a.n;
    const unsigned long long* nextl = a.lm + (uint64_t)(Lb + 1) * a.n;
    double* const hcur = a.hacc + (uint64_t)(Lb & 1) * a.bs.nheavy * 64;
    double* const hoth = a.hacc + (uint64_t)((Lb + 1) & 1) * a.bs.nheavy * 64;
    ms_for_light(a, a.bs, a.offs, gwarp, nwarps, [&](uint32_t v, bool light) {
      const unsigned long long cv = light ? cur[v] : 0ull;
      unsigned sel = __ballot_sync(kFull, cv != 0);
      while (sel) {
        const int k = __ffs(sel) - 1;
        sel &= sel - 1;
        const uint32_t vk = __shfl_sync(kFull, v, k);
        const unsigned long long ck = shfl64(cv, k);
        double dA = 0.0, dB = 0.0;
        ms_backward_range(a, nextl, ck, ldg(a.offs + vk), ldg(a.offs + vk + 1), dA, dB);
        const uint64_t r = (uint64_t)vk * 64;
        double t = 0.0;
        if ((ck >> lane) & 1ull) {
          const float d = (float)(dA * a.sigma[r + lane]);
          a.dep[r + lane] = d;
          t += d;
        }
        if ((ck >> (lane + 32)) & 1ull) {
          const float d = (float)(dB * a.sigma[r + lane + 32]);
          a.dep[r + lane + 32] = d;
          t += d;
        }
        t = warp_sum(t);
        if (lane == 0) a.bc[vk] += t;
      }
    });
    for (uint64_t t = gwarp; t < a.bs.ntiles; t += nwarps) {
      const uint2 tv = a.bs.tiles[t];
      const unsigned long long cv = cur[tv.x];
      if (!cv) continue;
      const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
      const uint64_t b = vb + (uint64_t)tv.y * a.bs.tile, e = min(ve, b + a.bs.tile);
      double dA = 0.0, dB = 0.0;
      ms_backward_range(a, nextl, cv, b, e, dA, dB);
      double* h = hcur + (uint64_t)a.hidx[tv.x] * 64;
      if ((cv >> lane) & 1ull) atomicAdd(&h[lane], dA);
      if ((cv >> (lane + 32)) & 1ull) atomicAdd(&h[lane + 32], dB);
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    for (uint64_t i = gwarp; i < a.bs.nheavy; i += nwarps) {
      const uint32_t v = a.bs.heavy_list[i];
      // clear what level Lb+1 left in the other half (level Lb-1 adds there)
      const unsigned long long prev = nextl[v];
      if (prev) {
        double* ho = hoth + i * 64;
        if ((prev >> lane) & 1ull) ho[lane] = 0.0;
        if ((prev >> (lane + 32)) & 1ull) ho[lane + 32] = 0.0;
      }
      const unsigned long long cv = cur[v];
      if (!cv) continue;
      const double* h = hcur + i * 64;
      const uint64_t r = (uint64_t)v * 64;
      double t = 0.0;
      if ((cv >> lane) & 1ull) {
        const float d = (float)(h[lane] * a.sigma[r + lane]);
        a.dep[r + lane] = d;
        t += d;
      }
      if ((cv >> (lane + 32)) & 1ull) {
        const float d = (float)(h[lane + 32] * a.sigma[r + lane + 32]);
        a.dep[r + lane + 32] = d;
        t += d;
      }
      t = warp_sum(t);
      if (lane == 0) a.bc[v] += t;
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
  }
  if (gtid == 0) ctl->levels = nlev;
}

// ----------------------------------------------------------- single source --
struct SsArgs {
  const uint64_t* __restrict__ offs;
  const uint32_t* __restrict__ col;
  uint32_t n;
  uint32_t src;
  uint32_t* dist;
  double* sigma;
  float* dep;
  double* bc;
  double* hacc;           // [n] heavy-vertex partial sums (backward)
  uint32_t* order;        // vertices in discovery (level) order
  uint32_t* level_start;  // [n + 2] order index where each level starts
  uint2* tiles;           // heavy-vertex tiles, appended level by level
  uint32_t* tile_start;   // [n + 2]
  uint32_t tile_cap;
  uint32_t heavy, tile;
  uint32_t* tails;  // [0] order tail, [1] tile tail
  BcCtl* ctl;
};

__global__ void ss_init(SsArgs a) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < a.n; v += stride) {
    a.dist[v] = v == a.src ? 0u : kBcInf;  // LevelInitializeIteration :66-80
    a.sigma[v] = v == a.src ? 1.0 : 0.0;
    a.dep[v] = 0.f;
  }
  if (tid == 0) {
    a.order[0] = a.src;
    a.level_start[0] = 0;
    a.level_start[1] = 1;
    a.tile_start[0] = 0;
    const uint64_t d = a.offs[a.src + 1] - a.offs[a.src];
    uint32_t nt = 0;
    if (d > a.heavy)
      for (uint32_t k = 0; k < (d + a.tile - 1) / a.tile && nt < a.tile_cap; ++k) a.tiles[nt++] = make_uint2(a.src, k);
    a.tile_start[1] = nt;
    a.tails[0] = 1;
    a.tails[1] = nt;
  }
}

__device__ __forceinline__ bool seg_reduce_f64(bool valid, uint32_t owner, double& x) {
  const uint32_t lane = lane_id();
  const uint32_t key = valid ? owner : 0xFFFFFFFFu;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double y = __shfl_down_sync(kFull, x, off);
    const uint32_t k2 = __shfl_down_sync(kFull, key, off);
    if (lane + off < 32 && k2 == key) x += y;
  }
  const uint32_t kprev = __shfl_up_sync(kFull, key, 1);
  return valid && (lane == 0 || kprev != key);
}

__global__ void __launch_bounds__(kBcBlock) ss_persistent(SsArgs a) {
  __shared__ double s_acc[kBcBlock / 32][32];
  BcCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kBcBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kBcBlock;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  s_acc[wib][lane] = 0.0;
  __syncwarp();
  // ---- forward: LevelSSSP (LevelStructs.h:87-134) ------------------------
  uint32_t L = 0;
  for (;; ++L) {
    const uint32_t lo = a.level_start[L], hi = a.level_start[L + 1];
    const uint32_t tlo = a.tile_start[L], thi = a.tile_start[L + 1];
    if (lo == hi) break;
    const uint32_t next = L + 1;
    auto visit = [&](bool valid, uint32_t v, uint32_t u) {
      bool disc = false;
      if (valid) {
        uint32_t du = a.dist[u];
        if (du == kBcInf) {
          const uint32_t old = atomicCAS(&a.dist[u], kBcInf, next);
          disc = old == kBcInf;  // one thread adds u to the next level
          du = disc ? next : old;
        }
        if (du == next) atomicAdd(&a.sigma[u], a.sigma[v]);
      }
      // append discovered vertices to the order array, heavy ones as tiles too
      const unsigned dm = __ballot_sync(kFull, disc);
      if (dm) {
        uint32_t base = 0;
        if (lane == __ffs(dm) - 1) base = atomicAdd(&a.tails[0], (uint32_t)__popc(dm));
        base = __shfl_sync(kFull, base, __ffs(dm) - 1);
        if (disc) a.order[base + __popc(dm & lanemask_lt)] = u;
        uint64_t d = 0;
        if (disc) d = ldg(a.offs + u + 1) - ldg(a.offs + u);
        const uint32_t nt = (disc && d > a.heavy) ? (uint32_t)((d + a.tile - 1) / a.tile) : 0u;
        warp_push_tiles(u, nt, a.tiles, &a.tails[1], a.tile_cap, &ctl->err);
      }
    };
    for_each_frontier_task(
        hi - lo, thi - tlo, gwarp, nwarps,
        [&](uint32_t base, uint32_t vpt) {
          const uint32_t idx = lo + base + lane;
          uint64_t b = 0;
          uint32_t d = 0, v = 0;
          if (lane < vpt && idx < hi) {
            v = a.order[idx];
            b = ldg(a.offs + v);
            const uint64_t dd = ldg(a.offs + v + 1) - b;
            d = dd > a.heavy ? 0u : (uint32_t)dd;
          }
          warp_expand(b, d, v, [&](bool valid, uint64_t e, uint32_t, uint32_t ov) {
            visit(valid, ov, valid ? ldg(a.col + e) : 0u);
          });
        },
        [&](uint32_t t) {
          const uint2 tv = a.tiles[tlo + t];
          const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
          const uint64_t b = vb + (uint64_t)tv.y * a.tile, e_end = min(ve, b + a.tile);
          for (uint64_t e0 = b; e0 < e_end; e0 += 32) {
            const uint64_t e = e0 + lane;
            visit(e < e_end, tv.x, e < e_end ? ldg(a.col + e) : 0u);
          }
        });
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    if (gtid == 0) {
      a.level_start[L + 2] = min(a.tails[0], a.n);
      a.tile_start[L + 2] = min(a.tails[1], a.tile_cap);
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
  }
  const uint32_t nlev = L;  // levels 0..L-1 are non-empty
  // ---- backward: LevelBackwardBrandes (LevelStructs.h:142-185) ------------
  for (int Lb = (int)nlev - 2; Lb >= 1; --Lb) {
    const uint32_t lo = a.level_start[Lb], hi = a.level_start[Lb + 1];
    const uint32_t tlo = a.tile_start[Lb], thi = a.tile_start[Lb + 1];
    const uint32_t succ = (uint32_t)Lb + 1;
    auto contrib = [&](bool valid, uint32_t w) -> double {
      if (!valid || a.dist[w] != succ) return 0.0;
      return (1.0 + (double)a.dep[w]) / a.sigma[w];
    };
    auto finish = [&](uint32_t v, double sum) {
      const float d = (float)(sum * a.sigma[v]);
      a.dep[v] = d;
      a.bc[v] += d;
    };
    for_each_frontier_task(
        hi - lo, thi - tlo, gwarp, nwarps,
        [&](uint32_t base, uint32_t vpt) {
          const uint32_t idx = lo + base + lane;
          uint64_t b = 0;
          uint32_t d = 0, v = 0;
          bool mine = false, heavy = false;
          if (lane < vpt && idx < hi) {
            v = a.order[idx];
            b = ldg(a.offs + v);
            const uint64_t dd = ldg(a.offs + v + 1) - b;
            heavy = dd > a.heavy;
            d = heavy ? 0u : (uint32_t)dd;
            mine = !heavy;
          }
          warp_expand(b, d, v, [&](bool valid, uint64_t e, uint32_t owner, uint32_t) {
            double x = contrib(valid, valid ? ldg(a.col + e) : 0u);
            if (seg_reduce_f64(valid, owner, x)) s_acc[wib][owner] += x;
            __syncwarp();
          });
          const double sum = s_acc[wib][lane];
          s_acc[wib][lane] = 0.0;
          __syncwarp();
          if (mine) finish(v, sum);
        },
        [&](uint32_t t) {
          const uint2 tv = a.tiles[tlo + t];
          const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
          const uint64_t b = vb + (uint64_t)tv.y * a.tile, e_end = min(ve, b + a.tile);
          double s = 0.0;
          for (uint64_t e = b + lane; e < e_end; e += 32) s += contrib(true, ldg(a.col + e));
          s = warp_sum(s);
          if (lane == 0) atomicAdd(&a.hacc[tv.x], s);
        });
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    for (uint64_t t = tlo + gtid; t < thi; t += gthreads) {
      const uint2 tv = a.tiles[t];
      if (tv.y == 0) {  // one finisher per heavy vertex
        finish(tv.x, a.hacc[tv.x]);
        a.hacc[tv.x] = 0.0;
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
  }
  if (gtid == 0) ctl->levels = nlev;
}

__global__ void bc_to_f32(const double* __restrict__ bc, float* __restrict__ out, uint32_t n) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride) out[v] = (float)bc[v];
}

}  // namespace

int run_bc(gb_graph* g, const uint32_t* srcs_in, uint32_t nsrc, uint32_t batch, float* bc_out, gb_stats* stats,
           cudaStream_t s) {
  if (batch < 1 || batch > 64) GB_FAIL(GB_ERR_ARG, "gb_bc: batch must be in [1, 64]");
  const uint32_t n = g->n;
  std::vector<uint32_t> srcs(nsrc);
  if (nsrc) GB_CUDA(cudaMemcpy(srcs.data(), srcs_in, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  for (uint32_t i = 0; i < nsrc; ++i)
    if (srcs[i] >= n) GB_FAIL(GB_ERR_ARG, "gb_bc: source %u >= n %u", srcs[i], n);
  if (batch > 1 && !g->symmetric)
    GB_FAIL(GB_ERR_UNSUPPORTED, "gb_bc: batched sources need a symmetric graph (in-edges = out-edges); use batch 1");
  const gb_tuning t = effective_tuning(g);
  const bool out_dev = is_device_ptr(bc_out);
  double total_ms = 0.0;
  uint32_t total_levels = 0;
  int launches = 0;
  BcCtl* hc = reinterpret_cast<BcCtl*>(static_cast<char*>(g->pinned) + 256);
  double* bc64 = nullptr;
  float* out32 = nullptr;
  if (batch == 1) {
    FrontierLayout fl = frontier_layout(n, g->m, t.heavy_degree, t.tile_edges);
    const size_t need = carve_size<BcCtl>(1) + carve_size<double>(n) * 3 + carve_size<float>(n) +
                        carve_size<uint32_t>(n) * 2 + carve_size<uint32_t>(n + 2) * 2 + carve_size<uint2>(fl.tile_cap) +
                        carve_size<uint32_t>(2) + (out_dev ? 0 : carve_size<float>(n));
    int st = ws_reserve(g, need, s);
    if (st != GB_OK) return st;
    Carver cv(g->ws);
    SsArgs a{};
    a.ctl = cv.take<BcCtl>(1);
    bc64 = cv.take<double>(n);
    a.bc = bc64;
    a.sigma = cv.take<double>(n);
    a.hacc = cv.take<double>(n);
    a.dep = cv.take<float>(n);
    a.dist = cv.take<uint32_t>(n);
    a.order = cv.take<uint32_t>(n);
    a.level_start = cv.take<uint32_t>(n + 2);
    a.tile_start = cv.take<uint32_t>(n + 2);
    a.tiles = cv.take<uint2>(fl.tile_cap);
    a.tails = cv.take<uint32_t>(2);
    out32 = out_dev ? bc_out : cv.take<float>(n);
    a.offs = g->offs;
    a.col = g->col;
    a.n = n;
    a.tile_cap = fl.tile_cap;
    a.heavy = t.heavy_degree;
    a.tile = t.tile_edges;
    GB_CUDA(cudaMemsetAsync(bc64, 0, sizeof(double) * n, s));
    GB_CUDA(cudaMemsetAsync(a.hacc, 0, sizeof(double) * n, s));
    const void* kfn = reinterpret_cast<const void*>(&ss_persistent);
    const int grid = coop_grid(g, kfn, kBcBlock, 0, t.blocks_per_sm);
    if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_bc: cannot size cooperative grid");
    for (uint32_t i = 0; i < nsrc; ++i) {
      a.src = srcs[i];
      GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(BcCtl), s));
      ss_init<<<g->sm_count * 4, 256, 0, s>>>(a);
      void* args[] = {&a};
      KernelTimer kt(stats != nullptr, s);
      GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, kBcBlock, args, 0, s));
      kt.stop(s);
      launches += 2;
      if (stats) {
        GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(BcCtl), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        if (hc->err) return dev_err_status(hc->err, "gb_bc");
        total_ms += kt.ms();
        total_levels += hc->levels;
      }
    }
    if (!stats) {
      GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(BcCtl), cudaMemcpyDeviceToHost, s));
      GB_CUDA(cudaStreamSynchronize(s));
      if (hc->err) return dev_err_status(hc->err, "gb_bc");
    }
  } else {
    SweepSched sched;
    int st = ensure_sweep_schedule(g, t.heavy_degree, t.tile_edges, s, &sched);
    if (st != GB_OK) return st;
    uint32_t lcap = 64;
    for (int attempt = 0;; ++attempt) {
      const size_t need = carve_size<BcCtl>(1) + carve_size<double>(n) + carve_size<unsigned long long>((size_t)lcap * n) +
                          carve_size<unsigned long long>(n) + carve_size<double>((size_t)n * 64) +
                          carve_size<float>((size_t)n * 64) + carve_size<double>(2 * (size_t)sched.nheavy * 64 + 1) +
                          carve_size<uint32_t>(n) + carve_size<uint32_t>(64) + (out_dev ? 0 : carve_size<float>(n));
      st = ws_reserve(g, need, s);
      if (st != GB_OK) return st;
      Carver cv(g->ws);
      MsArgs a{};
      a.ctl = cv.take<BcCtl>(1);
      bc64 = cv.take<double>(n);
      a.bc = bc64;
      a.lm = cv.take<unsigned long long>((size_t)lcap * n);
      a.visit = cv.take<unsigned long long>(n);
      a.sigma = cv.take<double>((size_t)n * 64);
      a.dep = cv.take<float>((size_t)n * 64);
      a.hacc = cv.take<double>(2 * (size_t)sched.nheavy * 64 + 1);
      a.hidx = cv.take<uint32_t>(n);
      uint32_t* dsrc = cv.take<uint32_t>(64);
      out32 = out_dev ? bc_out : cv.take<float>(n);
      a.offs = a.in_offs = g->offs;
      a.col = a.in_col = g->col;
      a.n = n;
      a.lcap = lcap;
      a.fs = a.bs = sched;
      a.srcs = dsrc;
      GB_CUDA(cudaMemsetAsync(bc64, 0, sizeof(double) * n, s));
      const void* kfn = reinterpret_cast<const void*>(&ms_persistent);
      const int grid = coop_grid(g, kfn, kBcBlock, 0, t.blocks_per_sm);
      if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "gb_bc: cannot size cooperative grid");
      bool retry = false;
      total_ms = 0.0;
      total_levels = 0;
      launches = 0;
      for (uint32_t b0 = 0; b0 < nsrc && !retry; b0 += batch) {
        a.nsrc = std::min(batch, nsrc - b0);
        GB_CUDA(cudaMemcpyAsync(dsrc, srcs.data() + b0, sizeof(uint32_t) * a.nsrc, cudaMemcpyHostToDevice, s));
        GB_CUDA(cudaMemsetAsync(a.ctl, 0, sizeof(BcCtl), s));
        ms_init<<<g->sm_count * 8, 256, 0, s>>>(a);
        ms_seed<<<1, 32, 0, s>>>(a);
        void* args[] = {&a};
        KernelTimer kt(stats != nullptr, s);
        GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, kBcBlock, args, 0, s));
        kt.stop(s);
        launches += 3;
        GB_CUDA(cudaMemcpyAsync(hc, a.ctl, sizeof(BcCtl), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        if (hc->err == kDevOverflow && hc->level_needed > lcap && attempt < 8) {
          lcap = std::max(lcap * 2, hc->level_needed + 8);
          retry = true;
        } else if (hc->err) {
          return dev_err_status(hc->err, "gb_bc");
        }
        total_ms += kt.ms();
        total_levels += hc->levels;
      }
      if (!retry) break;
    }
  }
  bc_to_f32<<<g->sm_count * 4, 256, 0, s>>>(bc64, out32, n);
  GB_CUDA(cudaGetLastError());
  if (!out_dev) {
    int st = copy_out(bc_out, out32, sizeof(float) * n, s);
    if (st != GB_OK) return st;
  }
  if (stats) {
    GB_CUDA(cudaStreamSynchronize(s));
    *stats = gb_stats{};
    stats->rounds = total_levels;
    stats->launches = launches + 1;
    stats->kernel_ms = total_ms;
    stats->edges_reached = 0;
  }
  return GB_OK;
}

}  // namespace gb

extern "C" int gb_bc(gb_graph* g, const uint32_t* srcs, uint32_t nsrc, uint32_t batch, float* bc_out,
                     gb_stats* stats, void* stream) {
  gb::clear_error();
  if (!g || !bc_out || (nsrc && !srcs)) GB_FAIL(GB_ERR_ARG, "gb_bc: null argument");
  GB_CUDA(cudaSetDevice(g->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g->perm) {
    std::vector<uint32_t> mapped(nsrc);
    for (uint32_t i = 0; i < nsrc; ++i) {
      if (srcs[i] >= g->n) GB_FAIL(GB_ERR_ARG, "gb_bc: source %u >= n %u", srcs[i], g->n);
      mapped[i] = g->h_iperm[srcs[i]];
    }
    float* res = reinterpret_cast<float*>(gb::result_buf(g, 0));
    int st = gb::run_bc(g, mapped.data(), nsrc, batch, res, stats, s);
    if (st != GB_OK) return st;
    if (stats) stats->launches += 1;  // the mapping gather
    return gb::finish_f32(g, res, bc_out, s);
  }
  return gb::run_bc(g, srcs, nsrc, batch, bc_out, stats, s);
}
