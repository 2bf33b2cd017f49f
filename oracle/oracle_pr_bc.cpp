// ORACLE -- test infrastructure only (see oracle.cpp for the pinning notes).
// PageRank and Brandes BC restatements.

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t kBcInf = 0xFFFFFFFFu / 4;  // BetweennessCentrality.cpp:32

struct Csr {
  uint32_t n;
  const uint64_t* end;
  const uint32_t* col;
  uint64_t b(uint32_t v) const { return v ? end[v - 1] : 0; }
  uint64_t e(uint32_t v) const { return end[v]; }
};

// computeOutDeg (PageRank-pull.cpp:90-122): in-degree of the stored graph.
std::vector<uint32_t> nout_of(const Csr& g, uint64_t m) {
  std::vector<uint32_t> k(g.n, 0);
  for (uint64_t i = 0; i < m; ++i) k[g.col[i]]++;
  return k;
}

template <class T>
uint32_t pr_push_sync(const Csr& g, T alpha, T tol, uint32_t max_iter, T* value) {
  // PageRank-push.cpp:103-188 (Sync) in a deterministic serial order:
  // phase 1 over the active list, then the updates in the same order.
  const uint32_t n = g.n;
  std::vector<T> residual(n, (T)1 - alpha);
  for (uint32_t v = 0; v < n; ++v) value[v] = 0;
  std::vector<uint32_t> active(n), next;
  for (uint32_t v = 0; v < n; ++v) active[v] = v;
  std::vector<uint8_t> queued(n, 0);
  uint32_t iter = 0;
  for (; !active.empty() && iter < max_iter; ++iter) {
    std::vector<std::pair<uint32_t, T>> updates;
    for (uint32_t v : active) {
      if (residual[v] > tol) {
        const T old = residual[v];
        value[v] += old;
        residual[v] = 0;
        const uint64_t deg = g.e(v) - g.b(v);
        if (deg > 0) updates.push_back({v, old * alpha / (T)deg});
      }
    }
    next.clear();
    std::fill(queued.begin(), queued.end(), 0);
    for (auto& [v, d] : updates)
      for (uint64_t i = g.b(v); i < g.e(v); ++i) {
        const uint32_t u = g.col[i];
        const T old = residual[u];
        residual[u] = old + d;
        if (old <= tol && old + d >= tol && !queued[u]) {
          queued[u] = 1;
          next.push_back(u);
        }
      }
    active.swap(next);
  }
  return iter;
}

template <class T>
uint32_t pr_pull_residual(const Csr& g, uint64_t m, T alpha, T tol, uint32_t max_iter, T* value) {
  // PageRank-pull.cpp:132-190 (two sweeps per round; delta read as written
  // by the first sweep)
  const uint32_t n = g.n;
  std::vector<uint32_t> nout = nout_of(g, m);
  std::vector<T> delta(n, 0), residual(n, (T)1 - alpha);
  for (uint32_t v = 0; v < n; ++v) value[v] = 0;
  uint32_t iterations = 0;
  while (true) {
    // both loops are per-vertex and read only what the other loop wrote, so
    // the parallel form gives the serial result
    uint64_t accum = 0;
#pragma omp parallel for schedule(static) reduction(+ : accum)
    for (int64_t vv = 0; vv < (int64_t)n; ++vv) {
      const uint32_t v = (uint32_t)vv;
      delta[v] = 0;
      if (residual[v] > tol) {
        const T old = residual[v];
        residual[v] = 0;
        value[v] += old;
        if (nout[v] > 0) {
          delta[v] = old * alpha / (T)nout[v];
          accum += 1;
        }
      }
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t vv = 0; vv < (int64_t)n; ++vv) {
      const uint32_t v = (uint32_t)vv;
      T sum = 0;
      for (uint64_t i = g.b(v); i < g.e(v); ++i) {
        const T d = delta[g.col[i]];
        if (d > 0) sum += d;
      }
      if (sum > 0) residual[v] = sum;
    }
    iterations++;
    if (iterations >= max_iter || !accum) break;
  }
  return iterations;
}

}  // namespace

extern "C" {

// PageRank pull-topological (PageRank-pull.cpp:196-251) in FP64, Jacobi form:
// value = 1/n; value'[v] = alpha*sum value[u]/nout[u] + (1-alpha)/n; stop when
// sum |delta| <= tol or at max_iter.  Returns the iteration count.
uint32_t orc_pr_pull_topo_f64(uint32_t n, const uint64_t* end, const uint32_t* col, uint64_t m, double alpha,
                              double tol, uint32_t max_iter, double* value) {
  Csr g{n, end, col};
  std::vector<uint32_t> nout = nout_of(g, m);
  std::vector<double> c(n), nv(n);
  for (uint32_t v = 0; v < n; ++v) value[v] = 1.0 / n;
  const double base = (1.0 - alpha) / n;
  uint32_t it = 0;
  while (true) {
    for (uint32_t v = 0; v < n; ++v) c[v] = nout[v] ? value[v] / nout[v] : 0.0;
    double l1 = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : l1)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      double s = 0;
      for (uint64_t i = g.b((uint32_t)v); i < g.e((uint32_t)v); ++i) s += c[col[i]];
      nv[v] = s * alpha + base;
      l1 += std::fabs(nv[v] - value[v]);
    }
    for (uint32_t v = 0; v < n; ++v) value[v] = nv[v];
    ++it;
    if (l1 <= tol || it >= max_iter) break;
  }
  return it;
}

// The reference's own fp32 schedule run serially: in-place update in vertex
// order (PageRank-pull.cpp:206-231), float sums, float base score.
uint32_t orc_pr_pull_topo_f32_inplace(uint32_t n, const uint64_t* end, const uint32_t* col, uint64_t m,
                                      float alpha, float tol, uint32_t max_iter, float* value) {
  Csr g{n, end, col};
  std::vector<uint32_t> nout = nout_of(g, m);
  for (uint32_t v = 0; v < n; ++v) value[v] = 1.0f / n;
  const float base = (1.0f - alpha) / n;
  uint32_t it = 0;
  while (true) {
    float accum = 0;
    for (uint32_t v = 0; v < n; ++v) {
      float sum = 0;
      for (uint64_t i = g.b(v); i < g.e(v); ++i) sum += value[col[i]] / nout[col[i]];
      const float nvv = sum * alpha + base;
      accum += std::fabs(nvv - value[v]);
      value[v] = nvv;
    }
    ++it;
    if (accum <= tol || it >= max_iter) break;
  }
  return it;
}

// Parallel fp32 in-place restatement (the reference's do_all with steal and
// chunk_size 32): the timed CPU baseline.
uint32_t orc_pr_pull_topo_par(uint32_t n, const uint64_t* end, const uint32_t* col, uint64_t m, float alpha,
                              float tol, uint32_t max_iter, float* value) {
  Csr g{n, end, col};
  std::vector<uint32_t> nout(n, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) __atomic_fetch_add(&nout[col[i]], 1u, __ATOMIC_RELAXED);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) value[v] = 1.0f / n;
  const float base = (1.0f - alpha) / n;
  uint32_t it = 0;
  while (true) {
    double accum = 0;
#pragma omp parallel for schedule(dynamic, 32) reduction(+ : accum)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      float sum = 0;
      for (uint64_t i = g.b((uint32_t)v); i < g.e((uint32_t)v); ++i) {
        const uint32_t u = col[i];
        float x;
        __atomic_load(value + u, &x, __ATOMIC_RELAXED);  // in place, as the reference
        sum += x / nout[u];
      }
      const float nvv = sum * alpha + base;
      accum += std::fabs(nvv - value[v]);
      __atomic_store(value + v, &nvv, __ATOMIC_RELAXED);
    }
    ++it;
    if (accum <= tol || it >= max_iter) break;
  }
  return it;
}

uint32_t orc_pr_pull_residual_f32(uint32_t n, const uint64_t* end, const uint32_t* col, uint64_t m, float alpha,
                                  float tol, uint32_t max_iter, float* value) {
  return pr_pull_residual<float>(Csr{n, end, col}, m, alpha, tol, max_iter, value);
}
uint32_t orc_pr_pull_residual_f64(uint32_t n, const uint64_t* end, const uint32_t* col, uint64_t m,
                                  double alpha, double tol, uint32_t max_iter, double* value) {
  return pr_pull_residual<double>(Csr{n, end, col}, m, alpha, tol, max_iter, value);
}
uint32_t orc_pr_push_sync_f32(uint32_t n, const uint64_t* end, const uint32_t* col, float alpha, float tol,
                              uint32_t max_iter, float* value) {
  return pr_push_sync<float>(Csr{n, end, col}, alpha, tol, max_iter, value);
}
uint32_t orc_pr_push_sync_f64(uint32_t n, const uint64_t* end, const uint32_t* col, double alpha, double tol,
                              uint32_t max_iter, double* value) {
  return pr_push_sync<double>(Csr{n, end, col}, alpha, tol, max_iter, value);
}

// Brandes BC, Level variant (LevelStructs.h:42-185, driver :224-326), one
// source at a time.  Sigma in SigmaT, dependency and bc in DepT (the
// reference: double sigma, float dependency and bc).  Level order within a
// level follows the worklist (here: discovery order, serial).
}  // extern "C"

template <class SigmaT, class DepT, class BcT>
static void bc_level(const Csr& g, const uint32_t* srcs, uint32_t nsrc, BcT* bc) {
  const uint32_t n = g.n;
  std::vector<uint32_t> dist(n);
  std::vector<SigmaT> sigma(n);
  std::vector<DepT> dep(n);
  for (uint32_t v = 0; v < n; ++v) bc[v] = 0;
  for (uint32_t s = 0; s < nsrc; ++s) {
    const uint32_t src = srcs[s];
    for (uint32_t v = 0; v < n; ++v) {  // LevelInitializeIteration :61-80
      dist[v] = kBcInf;
      sigma[v] = 0;
      dep[v] = 0;
    }
    dist[src] = 0;
    sigma[src] = 1;
    std::vector<std::vector<uint32_t>> levels(1, std::vector<uint32_t>{src});
    for (uint32_t L = 0; !levels[L].empty(); ++L) {  // LevelSSSP :87-134
      levels.emplace_back();
      for (uint32_t v : levels[L])
        for (uint64_t i = g.b(v); i < g.e(v); ++i) {
          const uint32_t u = g.col[i];
          if (dist[u] == kBcInf) {
            dist[u] = L + 1;
            levels[L + 1].push_back(u);
            sigma[u] += sigma[v];
          } else if (dist[u] == L + 1) {
            sigma[u] += sigma[v];
          }
        }
    }
    // LevelBackwardBrandes :142-185: levels.size()-3 down to 1
    if (levels.size() >= 3) {
      for (uint32_t L = (uint32_t)levels.size() - 3; L > 0; --L) {
        for (uint32_t v : levels[L]) {
          for (uint64_t i = g.b(v); i < g.e(v); ++i) {
            const uint32_t u = g.col[i];
            if (dist[u] == L + 1) dep[v] = (DepT)(dep[v] + ((DepT)1 + dep[u]) / sigma[u]);
          }
          dep[v] = (DepT)(dep[v] * sigma[v]);
          bc[v] = (BcT)(bc[v] + dep[v]);
        }
      }
    }
  }
}

extern "C" {

void orc_bc_level(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* srcs, uint32_t nsrc,
                  float* bc) {
  bc_level<double, float, float>(Csr{n, end, col}, srcs, nsrc, bc);
}
void orc_bc_level_f64(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* srcs, uint32_t nsrc,
                      double* bc) {
  bc_level<double, double, double>(Csr{n, end, col}, srcs, nsrc, bc);
}

// Parallel Level BC (all threads on one source at a time, as the reference):
// the timed CPU baseline.  fp64 sigma via CAS adds, fp32 dependency.
void orc_bc_level_par(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* srcs, uint32_t nsrc,
                      float* bc) {
  Csr g{n, end, col};
  std::vector<uint32_t> dist(n);
  std::vector<double> sigma(n);
  std::vector<float> dep(n);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) bc[v] = 0;
  const int nt = omp_get_max_threads();
  std::vector<std::vector<uint32_t>> local(nt);
  for (uint32_t s = 0; s < nsrc; ++s) {
    const uint32_t src = srcs[s];
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      dist[v] = kBcInf;
      sigma[v] = 0;
      dep[v] = 0;
    }
    dist[src] = 0;
    sigma[src] = 1;
    std::vector<std::vector<uint32_t>> levels(1, std::vector<uint32_t>{src});
    for (uint32_t L = 0; !levels[L].empty(); ++L) {
      const auto& cur = levels[L];
#pragma omp parallel
      {
        auto& out = local[omp_get_thread_num()];
        out.clear();
#pragma omp for schedule(dynamic, 256)
        for (int64_t j = 0; j < (int64_t)cur.size(); ++j) {
          const uint32_t v = cur[j];
          const double sv = sigma[v];
          for (uint64_t i = g.b(v); i < g.e(v); ++i) {
            const uint32_t u = col[i];
            uint32_t du = __atomic_load_n(&dist[u], __ATOMIC_RELAXED);
            if (du == kBcInf) {
              uint32_t expect = kBcInf;
              if (__atomic_compare_exchange_n(&dist[u], &expect, L + 1, false, __ATOMIC_RELAXED,
                                              __ATOMIC_RELAXED))
                out.push_back(u);
              du = L + 1;
            }
            if (du == L + 1) {
              uint64_t* q = reinterpret_cast<uint64_t*>(&sigma[u]);
              uint64_t old = __atomic_load_n(q, __ATOMIC_RELAXED);
              for (;;) {
                double of;
                std::memcpy(&of, &old, 8);
                const double nf = of + sv;
                uint64_t nu;
                std::memcpy(&nu, &nf, 8);
                if (__atomic_compare_exchange_n(q, &old, nu, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
              }
            }
          }
        }
      }
      levels.emplace_back();
      for (auto& l : local) levels[L + 1].insert(levels[L + 1].end(), l.begin(), l.end());
    }
    if (levels.size() >= 3) {
      for (uint32_t L = (uint32_t)levels.size() - 3; L > 0; --L) {
        const auto& cur = levels[L];
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t j = 0; j < (int64_t)cur.size(); ++j) {
          const uint32_t v = cur[j];
          float d = 0;
          for (uint64_t i = g.b(v); i < g.e(v); ++i) {
            const uint32_t u = col[i];
            if (dist[u] == L + 1) d = (float)(d + (1.0f + dep[u]) / sigma[u]);
          }
          d = (float)(d * sigma[v]);
          dep[v] = d;
          bc[v] += d;
        }
      }
    }
  }
}

// Level BC in FP64 with the sources spread over the threads (each thread runs
// whole sources with its own arrays and the per-thread sums are added at the
// end): the FP64 ground truth for batches of many sources on large graphs.
void orc_bc_level_f64_par_sources(uint32_t n, const uint64_t* end, const uint32_t* col, const uint32_t* srcs,
                                  uint32_t nsrc, double* bc) {
  Csr g{n, end, col};
  for (uint32_t v = 0; v < n; ++v) bc[v] = 0;
#pragma omp parallel
  {
    std::vector<double> mine(n, 0.0), one(n);
#pragma omp for schedule(dynamic, 1)
    for (int64_t s = 0; s < (int64_t)nsrc; ++s) {
      bc_level<double, double, double>(g, srcs + s, 1, one.data());
      for (uint32_t v = 0; v < n; ++v) mine[v] += one[v];
    }
#pragma omp critical
    for (uint32_t v = 0; v < n; ++v) bc[v] += mine[v];
  }
}

// FP64 Jacobi solve of one personalised-PageRank column (no reference: the
// PPR addition's ground truth on graphs too large for a sparse LU).  Arcs
// j->i in CSR order with weight w[e]; s_j = out-weight sum of j;
// W~_ij = w_ji / s_j.  adjoint == 0: x = rhs + alpha W~ x (rhs = (1-alpha) T);
// adjoint != 0: lam = rhs + alpha W~^T lam (rhs = dL/dx).  Iterates from
// out = rhs until the L1 change is <= tol * max(1, |rhs|_1) or max_iter;
// returns the iteration count.
uint32_t orc_ppr_solve_f64(uint32_t n, const uint64_t* end, const uint32_t* col, const float* w, const double* rhs,
                           double alpha, double tol, uint32_t max_iter, int adjoint, double* out) {
  Csr g{n, end, col};
  std::vector<double> s(n, 0.0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t j = 0; j < (int64_t)n; ++j) {
    double t = 0;
    for (uint64_t e = g.b((uint32_t)j); e < g.e((uint32_t)j); ++e) t += w[e];
    s[j] = t;
  }
  // in-arcs (forward pulls x_j over arcs j->i): counting sort by target
  std::vector<uint64_t> tb;
  std::vector<uint32_t> tsrc;
  std::vector<double> tcoef;
  const uint64_t m = n ? end[n - 1] : 0;
  if (!adjoint) {
    tb.assign((size_t)n + 1, 0);
    for (uint64_t e = 0; e < m; ++e) tb[col[e] + 1]++;
    for (uint32_t i = 0; i < n; ++i) tb[i + 1] += tb[i];
    std::vector<uint64_t> fill(tb.begin(), tb.end() - 1);
    tsrc.resize(m);
    tcoef.resize(m);
    for (uint32_t j = 0; j < n; ++j)
      for (uint64_t e = g.b(j); e < g.e(j); ++e) {
        const uint64_t k = fill[col[e]]++;
        tsrc[k] = j;
        tcoef[k] = s[j] > 0 ? (double)w[e] / s[j] : 0.0;
      }
  }
  double rn = 0;
  for (uint32_t v = 0; v < n; ++v) rn += std::fabs(rhs[v]);
  const double stop = tol * (rn > 1.0 ? rn : 1.0);
  std::vector<double> nx(n);
  for (uint32_t v = 0; v < n; ++v) out[v] = rhs[v];
  uint32_t it = 0;
  while (it < max_iter) {
    double l1 = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : l1)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      double acc = 0;
      if (adjoint) {
        for (uint64_t e = g.b((uint32_t)v); e < g.e((uint32_t)v); ++e)
          acc += (s[v] > 0 ? (double)w[e] / s[v] : 0.0) * out[col[e]];
      } else {
        for (uint64_t k = tb[v]; k < tb[v + 1]; ++k) acc += tcoef[k] * out[tsrc[k]];
      }
      nx[v] = rhs[v] + alpha * acc;
      l1 += std::fabs(nx[v] - out[v]);
    }
    for (uint32_t v = 0; v < n; ++v) out[v] = nx[v];
    ++it;
    if (l1 <= stop) break;
  }
  return it;
}

}  // extern "C"
