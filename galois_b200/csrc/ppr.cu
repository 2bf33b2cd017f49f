// Batched personalised PageRank and its adjoint (differentiable PPR).
//
// No reference counterpart: an addition beside the PageRank kernels
// (lonestar/analytics/cpu/pagerank/PageRank-pull.cpp:196-251 is the
// un-personalised, unweighted pull iteration it generalises).
//
//   forward  x = (1-a) T + a W~ x,      W~_ij = w_ji / s_j,  s_j = sum_i w_ji
//   adjoint  lam = gx + a W~^T lam
//   grads    dL/dT = (1-a) lam
//            dL/dw_ji = a/s_j * sum_b x_j^b (lam_i^b - mu_j^b),
//            mu_j = (W~^T lam)_j = (lam_j - gx_j) / a
//
// B200 design: B right-hand sides stored vertex-major [n][B] so that, for
// B = 128, one arc's gather is a single coalesced 512-byte row (a float4 per
// lane) and the graph (column id + normalised weight, 8 bytes per arc) is
// read once per iteration for all B columns.  One warp owns a row (light
// rows); rows above `heavy` arcs are split into tiles whose partial rows meet
// in a per-heavy-row accumulator.  The forward pulls over the in-arcs of the
// device transpose, the adjoint over the out-arcs of the CSR.  Each solve is
// one cooperative persistent launch; per-column L1 changes are reduced per
// block in shared memory and across blocks with fp64 atomics.  B = 1 (the
// plain single-vector solve) uses lanes over arcs instead of columns.

#include <algorithm>
#include <vector>

#include "device_common.cuh"
#include "device_graph.cuh"

namespace gb {

int build_row_schedule(const uint64_t* offs, uint32_t n, uint64_t m, uint32_t heavy, uint32_t tile, int sm_count,
                       void* pinned, cudaStream_t s, uint2** tiles, uint32_t** heavy_list, uint32_t* ntiles,
                       uint32_t* nheavy);

namespace {

constexpr int kPprBlock = 256;
constexpr int kPprWarps = kPprBlock / 32;
constexpr uint32_t kPprHeavy = 1024;  // arcs per row above which a row is tiled
constexpr uint32_t kPprTile = 512;

struct RowSched {
  uint2* tiles = nullptr;
  uint32_t* heavy = nullptr;
  uint32_t* hidx = nullptr;  // [n] heavy index of a heavy row
  uint32_t ntiles = 0, nheavy = 0;
};

struct PprState {
  RowSched fwd, bwd;      // over the transpose (in-arcs) and the CSR (out-arcs)
  float* s = nullptr;     // [n] out-weight sums
  float* wn = nullptr;    // [m] w / s_src, CSR order
  float* wn_t = nullptr;  // [m] the same, transpose order
  uint32_t* flags = nullptr;  // [n/32] rows with a non-zero source term
  double* l1 = nullptr;       // [3][128] per-column L1 change ring
  double* colnorm = nullptr;  // [128] per-column L1 norm of the adjoint's source term
  float* hacc = nullptr;      // [max(nheavy)][128]
  size_t hacc_rows = 0;
};

void free_state(gb_graph* g) {
  PprState* st = static_cast<PprState*>(g->ppr_state);
  if (!st) return;
  for (RowSched* r : {&st->fwd, &st->bwd}) {
    cudaFree(r->tiles);
    cudaFree(r->heavy);
    cudaFree(r->hidx);
  }
  cudaFree(st->s);
  cudaFree(st->wn);
  cudaFree(st->wn_t);
  cudaFree(st->flags);
  cudaFree(st->l1);
  cudaFree(st->colnorm);
  cudaFree(st->hacc);
  delete st;
  g->ppr_state = nullptr;
  g->ppr_free = nullptr;
}

__global__ void fill_hidx(const uint32_t* __restrict__ heavy, uint32_t nheavy, uint32_t* hidx) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < nheavy; i += stride) hidx[heavy[i]] = (uint32_t)i;
}

// s_j = sum of out-arc weights; wn[e] = w[e] / s_j (one warp per row j)
__global__ void ppr_normalise(const uint64_t* __restrict__ offs, const float* __restrict__ w, uint32_t n,
                              float* __restrict__ s, float* __restrict__ wn) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  for (uint64_t j = gw; j < n; j += nw) {
    const uint64_t b = offs[j], e = offs[j + 1];
    float acc = 0.f;
    for (uint64_t k = b + lane; k < e; k += 32) acc += w[k];
    acc = warp_sum(acc);
    if (lane == 0) s[j] = acc;
    const float inv = acc > 0.f ? 1.0f / acc : 0.f;
    for (uint64_t k = b + lane; k < e; k += 32) wn[k] = w[k] * inv;
  }
}

__global__ void ppr_permute(const float* __restrict__ wn, const uint64_t* __restrict__ emap, uint64_t m,
                            float* __restrict__ wn_t) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = tid; e < m; e += stride) wn_t[e] = wn[emap[e]];
}

// flags[r] = 1 if row r of src has a non-zero entry; dst = scale * src
__global__ void ppr_seed(const float* __restrict__ src, float scale, uint32_t n, uint32_t B, uint32_t* flags,
                         float* __restrict__ dst) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  for (uint64_t r = gw; r < n; r += nw) {
    bool nz = false;
    for (uint32_t b = lane; b < B; b += 32) {
      const float v = src[r * B + b];
      nz |= v != 0.f;
      dst[r * B + b] = scale * v;
    }
    nz = __any_sync(kFull, nz);
    if (lane == 0 && nz) atomicOr(&flags[r >> 5], 1u << (r & 31));
  }
}

struct IterCtl {
  GridBar bar;
  int err;
  uint32_t iters;
};

struct IterArgs {
  const uint64_t* __restrict__ offs;  // rows: in-arcs (forward) or out-arcs (adjoint)
  const uint32_t* __restrict__ col;
  const float* __restrict__ wn;       // normalised weight per arc
  uint32_t n, B;
  const float* __restrict__ src;      // source term, [n][B]
  float src_scale;
  const uint32_t* __restrict__ flags;  // rows with a source term (nullptr: every row)
  float* buf[2];                       // buf[0] holds x0
  float alpha, tol;
  uint32_t max_iter;
  RowSched sched;
  float* hacc;  // [nheavy][128]
  double* l1;   // [3][128]
  const double* col_scale;  // per-column stopping scale (nullptr: 1)
  IterCtl* ctl;
};

__device__ __forceinline__ float4 f4_fma(float a, float4 x, float4 y) {
  return make_float4(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y), fmaf(a, x.z, y.z), fmaf(a, x.w, y.w));
}

// Sum over arcs [b, e) of wn * x[col] for this lane's 4 columns (WIDE) or, in
// narrow mode (B == 1), for the whole warp (lanes over arcs, result in every
// lane after the reduction).
template <bool WIDE>
__device__ __forceinline__ float4 row_sum(const IterArgs& a, const float* __restrict__ x, uint64_t b, uint64_t e) {
  const uint32_t lane = lane_id();
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (WIDE) {
    const bool act = 4 * lane < a.B;
    for (uint64_t k0 = b; k0 < e; k0 += 32) {
      const uint32_t cnt = (uint32_t)(e - k0 < 32 ? e - k0 : 32);
      uint32_t mc = 0;
      float mw = 0.f;
      if (lane < cnt) {
        mc = ldg(a.col + k0 + lane);
        mw = ldg(a.wn + k0 + lane);
      }
      uint32_t u = 0;
      for (; u + 4 <= cnt; u += 4) {
        const uint32_t c0 = __shfl_sync(kFull, mc, u), c1 = __shfl_sync(kFull, mc, u + 1);
        const uint32_t c2 = __shfl_sync(kFull, mc, u + 2), c3 = __shfl_sync(kFull, mc, u + 3);
        const float w0 = __shfl_sync(kFull, mw, u), w1 = __shfl_sync(kFull, mw, u + 1);
        const float w2 = __shfl_sync(kFull, mw, u + 2), w3 = __shfl_sync(kFull, mw, u + 3);
        if (act) {
          const float4 x0 = *reinterpret_cast<const float4*>(x + (uint64_t)c0 * a.B + 4 * lane);
          const float4 x1 = *reinterpret_cast<const float4*>(x + (uint64_t)c1 * a.B + 4 * lane);
          const float4 x2 = *reinterpret_cast<const float4*>(x + (uint64_t)c2 * a.B + 4 * lane);
          const float4 x3 = *reinterpret_cast<const float4*>(x + (uint64_t)c3 * a.B + 4 * lane);
          acc = f4_fma(w0, x0, acc);
          acc = f4_fma(w1, x1, acc);
          acc = f4_fma(w2, x2, acc);
          acc = f4_fma(w3, x3, acc);
        }
      }
      for (; u < cnt; ++u) {
        const uint32_t c0 = __shfl_sync(kFull, mc, u);
        const float w0 = __shfl_sync(kFull, mw, u);
        if (act) acc = f4_fma(w0, *reinterpret_cast<const float4*>(x + (uint64_t)c0 * a.B + 4 * lane), acc);
      }
    }
  } else {
    float s = 0.f;
    for (uint64_t k = b + lane; k < e; k += 32) s = fmaf(ldg(a.wn + k), x[ldg(a.col + k)], s);
    acc.x = warp_sum(s);
  }
  return acc;
}

template <bool WIDE>
__global__ void __launch_bounds__(kPprBlock) ppr_iterate(IterArgs a) {
  __shared__ float s_diff[kPprWarps][128];
  IterCtl* ctl = a.ctl;
  const uint64_t deadline = kernel_deadline();
  const uint64_t gtid = blockIdx.x * (uint64_t)kPprBlock + threadIdx.x;
  const uint64_t gthreads = (uint64_t)gridDim.x * kPprBlock;
  const uint64_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const bool act = WIDE ? 4 * lane < a.B : lane == 0;
  for (uint32_t it = 0;; ++it) {
    const float* __restrict__ x = a.buf[it & 1];
    float* __restrict__ y = a.buf[(it + 1) & 1];
    if (gtid == 0)
      for (int c = 0; c < 128; ++c) a.l1[((it + 1) % 3) * 128 + c] = 0.0;
    float4 dsum = make_float4(0.f, 0.f, 0.f, 0.f);
    auto finish = [&](uint32_t r, float4 acc) {
      if (!act) return;
      const bool has_src = !a.flags || ((a.flags[r >> 5] >> (r & 31)) & 1u);
      const uint64_t base = (uint64_t)r * a.B + (WIDE ? 4 * lane : 0);
      if (WIDE) {
        float4 v = make_float4(a.alpha * acc.x, a.alpha * acc.y, a.alpha * acc.z, a.alpha * acc.w);
        if (has_src) v = f4_fma(a.src_scale, *reinterpret_cast<const float4*>(a.src + base), v);
        const float4 o = *reinterpret_cast<const float4*>(x + base);
        dsum.x += fabsf(v.x - o.x);
        dsum.y += fabsf(v.y - o.y);
        dsum.z += fabsf(v.z - o.z);
        dsum.w += fabsf(v.w - o.w);
        *reinterpret_cast<float4*>(y + base) = v;
      } else {
        float v = a.alpha * acc.x;
        if (has_src) v = fmaf(a.src_scale, a.src[base], v);
        dsum.x += fabsf(v - x[base]);
        y[base] = v;
      }
    };
    // light rows: one warp per row
    for (uint64_t r = gwarp; r < a.n; r += nwarps) {
      const uint64_t b = ldg(a.offs + r), e = ldg(a.offs + r + 1);
      if (e - b > kPprHeavy) continue;
      finish((uint32_t)r, row_sum<WIDE>(a, x, b, e));
    }
    // heavy rows: tiles of kPprTile arcs
    for (uint64_t t = gwarp; t < a.sched.ntiles; t += nwarps) {
      const uint2 tv = a.sched.tiles[t];
      const uint64_t vb = ldg(a.offs + tv.x), ve = ldg(a.offs + tv.x + 1);
      const uint64_t b = vb + (uint64_t)tv.y * kPprTile, e = min(ve, b + kPprTile);
      const float4 acc = row_sum<WIDE>(a, x, b, e);
      float* h = a.hacc + (uint64_t)a.sched.hidx[tv.x] * 128 + (WIDE ? 4 * lane : 0);
      if (act) {
        atomicAdd(h, acc.x);
        if (WIDE) {
          atomicAdd(h + 1, acc.y);
          atomicAdd(h + 2, acc.z);
          atomicAdd(h + 3, acc.w);
        }
      }
    }
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    for (uint64_t i = gwarp; i < a.sched.nheavy; i += nwarps) {
      const uint32_t r = a.sched.heavy[i];
      float* h = a.hacc + i * 128 + (WIDE ? 4 * lane : 0);
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      if (act) {
        acc.x = h[0];
        h[0] = 0.f;
        if (WIDE) {
          acc.y = h[1];
          acc.z = h[2];
          acc.w = h[3];
          h[1] = h[2] = h[3] = 0.f;
        }
      }
      finish(r, acc);
    }
    // per-column L1 change: block reduction, then one fp64 atomic per column
    if (WIDE) {
      s_diff[wib][4 * lane + 0] = dsum.x;
      s_diff[wib][4 * lane + 1] = dsum.y;
      s_diff[wib][4 * lane + 2] = dsum.z;
      s_diff[wib][4 * lane + 3] = dsum.w;
    } else if (lane == 0) {
      s_diff[wib][0] = dsum.x;
    }
    __syncthreads();
    if (threadIdx.x < a.B) {
      float sum = 0.f;
      for (int w = 0; w < kPprWarps; ++w) sum += s_diff[w][threadIdx.x];
      if (sum != 0.f) atomicAdd(&a.l1[(it % 3) * 128 + threadIdx.x], (double)sum);
    }
    __syncthreads();
    if (!grid_barrier(&ctl->bar, gridDim.x, &ctl->err, deadline)) return;
    // converged when every column's L1 change is at most tol (times the
    // column's scale for the adjoint, whose source term is not normalised)
    bool done = true;
    for (uint32_t c = 0; c < a.B; ++c) {
      const double lim = (double)a.tol * (a.col_scale ? a.col_scale[c] : 1.0);
      done &= *reinterpret_cast<volatile double*>(&a.l1[(it % 3) * 128 + c]) <= lim;
    }
    if (gtid == 0) ctl->iters = it + 1;
    if (done || it + 1 >= a.max_iter) break;
  }
}

// dL/dw for every arc of the CSR (rows = sources j):
//   g[e] = alpha/s_j * sum_b x_j^b (lam_i^b - mu_j^b),  mu_j = (lam_j - gx_j)/alpha
template <bool WIDE>
__global__ void __launch_bounds__(kPprBlock) ppr_grad_w(const uint64_t* __restrict__ offs,
                                                         const uint32_t* __restrict__ col, const float* __restrict__ s,
                                                         const float* __restrict__ x, const float* __restrict__ lam,
                                                         const float* __restrict__ gx, uint32_t n, uint32_t B,
                                                         float alpha, RowSched sched, float* __restrict__ grad_w) {
  const uint64_t gtid = blockIdx.x * (uint64_t)kPprBlock + threadIdx.x;
  const uint64_t gwarp = gtid >> 5, nwarps = ((uint64_t)gridDim.x * kPprBlock) >> 5;
  const uint32_t lane = lane_id();
  const float inv_alpha = 1.0f / alpha;
  auto run = [&](uint32_t j, uint64_t b, uint64_t e) {
    const float sj = s[j];
    const float scale = sj > 0.f ? alpha / sj : 0.f;
    if (WIDE) {
      const bool act = 4 * lane < B;
      float4 xj = make_float4(0.f, 0.f, 0.f, 0.f), mj = xj;
      if (act) {
        const uint64_t base = (uint64_t)j * B + 4 * lane;
        xj = *reinterpret_cast<const float4*>(x + base);
        const float4 lj = *reinterpret_cast<const float4*>(lam + base);
        const float4 gj = *reinterpret_cast<const float4*>(gx + base);
        mj = make_float4((lj.x - gj.x) * inv_alpha, (lj.y - gj.y) * inv_alpha, (lj.z - gj.z) * inv_alpha,
                         (lj.w - gj.w) * inv_alpha);
      }
      for (uint64_t k = b; k < e; ++k) {
        const uint32_t i = ldg(col + k);
        float d = 0.f;
        if (act) {
          const float4 li = *reinterpret_cast<const float4*>(lam + (uint64_t)i * B + 4 * lane);
          d = xj.x * (li.x - mj.x) + xj.y * (li.y - mj.y) + xj.z * (li.z - mj.z) + xj.w * (li.w - mj.w);
        }
        d = warp_sum(d);
        if (lane == 0) grad_w[k] = scale * d;
      }
    } else {
      const float xj = x[j];
      const float mj = (lam[j] - gx[j]) * inv_alpha;
      for (uint64_t k = b + lane; k < e; k += 32) grad_w[k] = scale * xj * (lam[ldg(col + k)] - mj);
    }
  };
  for (uint64_t j = gwarp; j < n; j += nwarps) {
    const uint64_t b = ldg(offs + j), e = ldg(offs + j + 1);
    if (e - b > kPprHeavy) continue;
    run((uint32_t)j, b, e);
  }
  for (uint64_t t = gwarp; t < sched.ntiles; t += nwarps) {
    const uint2 tv = sched.tiles[t];
    const uint64_t vb = ldg(offs + tv.x), ve = ldg(offs + tv.x + 1);
    const uint64_t b = vb + (uint64_t)tv.y * kPprTile;
    run(tv.x, b, min(ve, b + kPprTile));
  }
}

// out[c] = sum_r |src[r][c]| for the B columns of a vertex-major [n][B] array.
__global__ void ppr_colnorm(const float* __restrict__ src, uint32_t n, uint32_t B, double* out) {
  __shared__ double s_sum[128];
  for (uint32_t c = threadIdx.x; c < 128; c += blockDim.x) s_sum[c] = 0.0;
  __syncthreads();
  const uint32_t rows_per_pass = blockDim.x / B;  // threads past rows_per_pass * B stay idle
  const uint32_t c = threadIdx.x % B, r0 = threadIdx.x / B;
  double acc = 0.0;
  if (r0 < rows_per_pass)
    for (uint64_t r = (uint64_t)blockIdx.x * rows_per_pass + r0; r < n; r += (uint64_t)gridDim.x * rows_per_pass)
      acc += fabs((double)src[r * B + c]);
  if (r0 < rows_per_pass) atomicAdd(&s_sum[c], acc);
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < B; k += blockDim.x)
    if (s_sum[k] != 0.0) atomicAdd(&out[k], s_sum[k]);
}

__global__ void ppr_scale(const float* __restrict__ src, float scale, uint64_t count, float* __restrict__ dst) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < count; i += stride) dst[i] = scale * src[i];
}

int ensure_state(gb_graph* g, cudaStream_t s, PprState** out) {
  int rc = ensure_transpose(g, s);
  if (rc != GB_OK) return rc;
  if (!g->ppr_state) {
    PprState* st = new (std::nothrow) PprState();
    if (!st) GB_FAIL(GB_ERR_OOM, "ppr: host allocation failed");
    g->ppr_state = st;
    g->ppr_free = free_state;
    const uint32_t n = g->n;
    const uint64_t m = g->m;
    rc = build_row_schedule(g->t_offs, n, m, kPprHeavy, kPprTile, g->sm_count, g->pinned, s, &st->fwd.tiles,
                            &st->fwd.heavy, &st->fwd.ntiles, &st->fwd.nheavy);
    if (rc != GB_OK) return rc;
    rc = build_row_schedule(g->offs, n, m, kPprHeavy, kPprTile, g->sm_count, g->pinned, s, &st->bwd.tiles,
                            &st->bwd.heavy, &st->bwd.ntiles, &st->bwd.nheavy);
    if (rc != GB_OK) return rc;
    for (RowSched* r : {&st->fwd, &st->bwd}) {
      GB_CUDA(cudaMalloc(&r->hidx, sizeof(uint32_t) * n));
      if (r->nheavy) fill_hidx<<<g->sm_count, 256, 0, s>>>(r->heavy, r->nheavy, r->hidx);
    }
    st->hacc_rows = std::max<size_t>(1, std::max(st->fwd.nheavy, st->bwd.nheavy));
    GB_CUDA(cudaMalloc(&st->hacc, sizeof(float) * 128 * st->hacc_rows));
    GB_CUDA(cudaMemsetAsync(st->hacc, 0, sizeof(float) * 128 * st->hacc_rows, s));
    GB_CUDA(cudaMalloc(&st->s, sizeof(float) * n));
    GB_CUDA(cudaMalloc(&st->wn, sizeof(float) * std::max<uint64_t>(m, 1)));
    GB_CUDA(cudaMalloc(&st->wn_t, sizeof(float) * std::max<uint64_t>(m, 1)));
    GB_CUDA(cudaMalloc(&st->flags, sizeof(uint32_t) * ((n + 31) / 32)));
    GB_CUDA(cudaMalloc(&st->l1, sizeof(double) * 3 * 128));
    GB_CUDA(cudaMalloc(&st->colnorm, sizeof(double) * 128));
  }
  *out = static_cast<PprState*>(g->ppr_state);
  return GB_OK;
}

int prepare_weights(gb_graph* g, PprState* st, const float* w, cudaStream_t s) {
  if (!w) w = g->wf;
  if (!w) GB_FAIL(GB_ERR_ARG, "ppr: no arc weights (pass w or upload w_f32)");
  if (w != g->wf && !is_device_ptr(w)) GB_FAIL(GB_ERR_ARG, "ppr: w must be device memory");
  ppr_normalise<<<g->sm_count * 8, 256, 0, s>>>(g->offs, w, g->n, st->s, st->wn);
  ppr_permute<<<g->sm_count * 8, 256, 0, s>>>(st->wn, g->t_emap, g->m, st->wn_t);
  GB_CUDA(cudaGetLastError());
  return GB_OK;
}

// One Jacobi solve x = scale*src + alpha * M x (M = W~ or W~^T) into `out`.
int solve(gb_graph* g, PprState* st, bool adjoint, uint32_t B, const float* src, float scale, float alpha, float tol,
          uint32_t max_iter, float* out, float* tmp, IterCtl* ctl, uint32_t* iters, double* kernel_ms,
          cudaStream_t s) {
  IterArgs a{};
  a.offs = adjoint ? g->offs : g->t_offs;
  a.col = adjoint ? g->col : g->t_col;
  a.wn = adjoint ? st->wn : st->wn_t;
  a.sched = adjoint ? st->bwd : st->fwd;
  a.n = g->n;
  a.B = B;
  a.src = src;
  a.src_scale = scale;
  a.flags = adjoint ? nullptr : st->flags;
  a.buf[0] = out;
  a.buf[1] = tmp;
  a.alpha = alpha;
  a.tol = tol;
  a.max_iter = max_iter;
  a.hacc = st->hacc;
  a.l1 = st->l1;
  a.col_scale = adjoint ? st->colnorm : nullptr;
  a.ctl = ctl;
  if (adjoint) {
    // the adjoint's source term (the loss gradient) has arbitrary scale: stop
    // on the L1 change relative to each column's L1 norm
    GB_CUDA(cudaMemsetAsync(st->colnorm, 0, sizeof(double) * 128, s));
    ppr_colnorm<<<g->sm_count * 4, 256, 0, s>>>(src, g->n, B, st->colnorm);
  }
  GB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(IterCtl), s));
  GB_CUDA(cudaMemsetAsync(st->l1, 0, sizeof(double) * 3 * 128, s));
  GB_CUDA(cudaMemsetAsync(st->flags, 0, sizeof(uint32_t) * ((g->n + 31) / 32), s));
  ppr_seed<<<g->sm_count * 8, 256, 0, s>>>(src, scale, g->n, B, st->flags, out);  // x0 = scale * src
  GB_CUDA(cudaGetLastError());
  const bool wide = B > 1;
  const void* kfn = wide ? reinterpret_cast<const void*>(&ppr_iterate<true>)
                         : reinterpret_cast<const void*>(&ppr_iterate<false>);
  const int grid = coop_grid(g, kfn, kPprBlock, 0, 0);
  if (grid <= 0) GB_FAIL(GB_ERR_CUDA, "ppr: cannot size cooperative grid");
  void* args[] = {&a};
  KernelTimer kt(true, s);
  GB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, kPprBlock, args, 0, s));
  kt.stop(s);
  IterCtl* hc = reinterpret_cast<IterCtl*>(static_cast<char*>(g->pinned) + 1024);
  GB_CUDA(cudaMemcpyAsync(hc, ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, s));
  GB_CUDA(cudaStreamSynchronize(s));
  if (hc->err) return dev_err_status(hc->err, "ppr");
  *iters = hc->iters;
  *kernel_ms += kt.ms();
  if (hc->iters & 1) GB_CUDA(cudaMemcpyAsync(out, tmp, sizeof(float) * (size_t)g->n * B, cudaMemcpyDeviceToDevice, s));
  return GB_OK;
}

int check_common(gb_graph* g, uint32_t B, float alpha, uint32_t max_iter) {
  // teleport / rank / arc-weight arrays are indexed by the caller's ids and arcs
  if (g->perm) GB_FAIL(GB_ERR_UNSUPPORTED, "ppr: graph was relabelled; PPR needs file order");
  if (!(B == 1 || (B % 4 == 0 && B >= 4 && B <= 128))) GB_FAIL(GB_ERR_ARG, "ppr: B must be 1 or a multiple of 4 <= 128");
  if (!(alpha > 0.f && alpha < 1.f)) GB_FAIL(GB_ERR_ARG, "ppr: alpha must be in (0,1)");
  if (max_iter == 0) GB_FAIL(GB_ERR_ARG, "ppr: max_iter must be > 0");
  if (g->m >= (1ull << 32)) GB_FAIL(GB_ERR_UNSUPPORTED, "ppr: limited to < 2^32 arcs");
  return GB_OK;
}

}  // namespace
}  // namespace gb

extern "C" int gb_ppr_forward(gb_graph* g, uint32_t B, const float* teleport, const float* w, float alpha, float tol,
                              uint32_t max_iter, float* x_out, uint32_t* iters_out, gb_stats* stats, void* stream) {
  using namespace gb;
  clear_error();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g || !teleport || !x_out) GB_FAIL(GB_ERR_ARG, "gb_ppr_forward: null argument");
  int rc = check_common(g, B, alpha, max_iter);
  if (rc != GB_OK) return rc;
  GB_CUDA(cudaSetDevice(g->device));
  if (!is_device_ptr(teleport) || !is_device_ptr(x_out)) GB_FAIL(GB_ERR_ARG, "gb_ppr_forward: arrays must be device memory");
  PprState* st = nullptr;
  if ((rc = ensure_state(g, s, &st)) != GB_OK) return rc;
  if ((rc = prepare_weights(g, st, w, s)) != GB_OK) return rc;
  const size_t need = carve_size<IterCtl>(1) + carve_size<float>((size_t)g->n * B);
  if ((rc = ws_reserve(g, need, s)) != GB_OK) return rc;
  Carver cv(g->ws);
  IterCtl* ctl = cv.take<IterCtl>(1);
  float* tmp = cv.take<float>((size_t)g->n * B);
  uint32_t iters = 0;
  double ms = 0.0;
  if ((rc = solve(g, st, false, B, teleport, 1.0f - alpha, alpha, tol, max_iter, x_out, tmp, ctl, &iters, &ms, s)) != GB_OK)
    return rc;
  if (iters_out) *iters_out = iters;
  if (stats) {
    GB_CUDA(cudaStreamSynchronize(s));
    *stats = gb_stats{};
    stats->rounds = iters;
    stats->edges_reached = g->m;
    stats->vertices_reached = g->n;
    stats->launches = 5;
    stats->kernel_ms = ms;
  }
  if (iters >= max_iter) {
    set_error("gb_ppr_forward: failed to converge in %u iterations", iters);
    return GB_ERR_NOT_CONVERGED;
  }
  return GB_OK;
}

extern "C" int gb_ppr_backward(gb_graph* g, uint32_t B, const float* x, const float* gx, const float* w, float alpha,
                               float tol, uint32_t max_iter, float* grad_teleport, float* grad_w, uint32_t* iters_out,
                               gb_stats* stats, void* stream) {
  using namespace gb;
  clear_error();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g || !x || !gx) GB_FAIL(GB_ERR_ARG, "gb_ppr_backward: null argument");
  int rc = check_common(g, B, alpha, max_iter);
  if (rc != GB_OK) return rc;
  GB_CUDA(cudaSetDevice(g->device));
  if (!is_device_ptr(x) || !is_device_ptr(gx) || (grad_teleport && !is_device_ptr(grad_teleport)) ||
      (grad_w && !is_device_ptr(grad_w)))
    GB_FAIL(GB_ERR_ARG, "gb_ppr_backward: arrays must be device memory");
  PprState* st = nullptr;
  if ((rc = ensure_state(g, s, &st)) != GB_OK) return rc;
  if ((rc = prepare_weights(g, st, w, s)) != GB_OK) return rc;
  const size_t nb = (size_t)g->n * B;
  const size_t need = carve_size<IterCtl>(1) + 2 * carve_size<float>(nb);
  if ((rc = ws_reserve(g, need, s)) != GB_OK) return rc;
  Carver cv(g->ws);
  IterCtl* ctl = cv.take<IterCtl>(1);
  float* lam = cv.take<float>(nb);
  float* tmp = cv.take<float>(nb);
  uint32_t iters = 0;
  double ms = 0.0;
  rc = solve(g, st, true, B, gx, 1.0f, alpha, tol, max_iter, lam, tmp, ctl, &iters, &ms, s);
  if (rc != GB_OK) return rc;
  KernelTimer kt(stats != nullptr, s);
  if (grad_teleport) ppr_scale<<<g->sm_count * 8, 256, 0, s>>>(lam, 1.0f - alpha, nb, grad_teleport);
  if (grad_w) {
    if (B > 1)
      ppr_grad_w<true><<<g->sm_count * 8, kPprBlock, 0, s>>>(g->offs, g->col, st->s, x, lam, gx, g->n, B, alpha,
                                                              st->bwd, grad_w);
    else
      ppr_grad_w<false><<<g->sm_count * 8, kPprBlock, 0, s>>>(g->offs, g->col, st->s, x, lam, gx, g->n, B, alpha,
                                                               st->bwd, grad_w);
  }
  kt.stop(s);
  GB_CUDA(cudaGetLastError());
  if (iters_out) *iters_out = iters;
  if (stats) {
    GB_CUDA(cudaStreamSynchronize(s));
    *stats = gb_stats{};
    stats->rounds = iters;
    stats->edges_reached = g->m;
    stats->vertices_reached = g->n;
    stats->launches = 7;
    stats->kernel_ms = ms + kt.ms();
  }
  if (iters >= max_iter) {
    set_error("gb_ppr_backward: failed to converge in %u iterations", iters);
    return GB_ERR_NOT_CONVERGED;
  }
  return GB_OK;
}
