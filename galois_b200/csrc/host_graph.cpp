// Host-side graph substrate of libgb: .gr I/O, text edge lists, seeded
// synthetic generators, per-arc weights and transpose.  Pure C++17/OpenMP;
// no CUDA is needed to call anything in this file.
//
// Formats and semantics follow the Galois sources:
//   .gr layout            libgalois/src/FileGraph.cpp:44-53 (header, end
//                         offsets, uint32/uint64 dsts, 8-byte re-alignment,
//                         edge data), reader FileGraph.cpp:104-135
//   edge-list conversion  tools/graph-convert/graph-convert.cpp:351-530
//   gr2edgelist           tools/graph-convert/graph-convert.cpp:867-900
//   transpose             libgalois/include/galois/graphs/LC_CSR_Graph.h:617-712

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <random>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "gb_internal.h"

namespace gb {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}
void clear_error() { g_last_error.clear(); }

namespace {

inline uint64_t mulhi64(uint64_t a, uint64_t b) {
  return (uint64_t)(((__uint128_t)a * (__uint128_t)b) >> 64);
}

template <class T>
T* xmalloc(size_t count) {
  if (count == 0) count = 1;
  return static_cast<T*>(std::malloc(count * sizeof(T)));
}

// Build a CSR (begin offsets, n+1) from a degree count pass and a scatter
// pass over the same deterministic arc stream, then sort and deduplicate each
// adjacency list.  `emit(i, fn)` must call fn(u, v) for every arc of draw i.
template <class Emit>
int build_csr_from_stream(uint32_t n, uint64_t ndraws, Emit emit,
                          gb_host_csr* out) {
  std::vector<std::atomic<uint64_t>> deg(n);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) deg[v].store(0, std::memory_order_relaxed);

#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)ndraws; ++i) {
    emit((uint64_t)i, [&](uint32_t u, uint32_t) {
      deg[u].fetch_add(1, std::memory_order_relaxed);
    });
  }
  std::vector<uint64_t> offs(n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) offs[v + 1] = offs[v] + deg[v].load(std::memory_order_relaxed);
  const uint64_t mraw = offs[n];
  uint32_t* raw = xmalloc<uint32_t>(mraw);
  if (!raw) GB_FAIL(GB_ERR_OOM, "host allocation of %llu arcs failed", (unsigned long long)mraw);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; ++v) deg[v].store(offs[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)ndraws; ++i) {
    emit((uint64_t)i, [&](uint32_t u, uint32_t v) {
      uint64_t p = deg[u].fetch_add(1, std::memory_order_relaxed);
      raw[p] = v;
    });
  }
  // sort + unique per row
  std::vector<uint64_t> ndeg(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)n; ++v) {
    uint32_t* b = raw + offs[v];
    uint32_t* e = raw + offs[v + 1];
    std::sort(b, e);
    ndeg[v] = (uint64_t)(std::unique(b, e) - b);
  }
  uint64_t* end_offs = xmalloc<uint64_t>(n);
  if (!end_offs) {
    std::free(raw);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
  uint64_t acc = 0;
  for (uint32_t v = 0; v < n; ++v) {
    acc += ndeg[v];
    end_offs[v] = acc;
  }
  const uint64_t m = acc;
  uint32_t* col = xmalloc<uint32_t>(m);
  if (!col) {
    std::free(raw);
    std::free(end_offs);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)n; ++v) {
    uint64_t dst = v ? end_offs[v - 1] : 0;
    std::memcpy(col + dst, raw + offs[v], ndeg[v] * sizeof(uint32_t));
  }
  std::free(raw);
  gb_host_csr_free(out);
  out->n = n;
  out->m = m;
  out->end_offs = end_offs;
  out->col = col;
  return GB_OK;
}

}  // namespace
}  // namespace gb

using namespace gb;

namespace gb {

int check_reference_weights(int min_value, int max_value, int edge_bytes, const char* what) {
  if (edge_bytes != 4 && edge_bytes != -4) GB_FAIL(GB_ERR_ARG, "%s: edge_bytes must be 4 (uint32) or -4 (float)", what);
  if (max_value < min_value) GB_FAIL(GB_ERR_ARG, "%s: max_value < min_value", what);
  if (edge_bytes == 4 && min_value < 0) GB_FAIL(GB_ERR_ARG, "%s: uint32 weights need min_value >= 0", what);
  return GB_OK;
}

// gr2randomweightgr's draws (tools/graph-convert/graph-convert.cpp:1145-1190):
// one default-constructed std::mt19937 and a std::uniform_int_distribution
// <uint32_t>(min, max) (edge_bytes 4) or std::uniform_real_distribution
// <float>(min, max) (edge_bytes -4), evaluated once per arc in arc order.
// The draws come from this build's C++ standard library, so they equal the
// converter's output when both use the same library (the distributions'
// algorithms are implementation-defined).
void draw_reference_weights(uint64_t m, int min_value, int max_value, int edge_bytes, void* out) {
  std::mt19937 gen;
  if (edge_bytes == 4) {
    std::uniform_int_distribution<uint32_t> dist((uint32_t)min_value, (uint32_t)max_value);
    uint32_t* w = static_cast<uint32_t*>(out);
    for (uint64_t e = 0; e < m; ++e) w[e] = dist(gen);
  } else {
    std::uniform_real_distribution<float> dist((float)min_value, (float)max_value);
    float* w = static_cast<float*>(out);
    for (uint64_t e = 0; e < m; ++e) w[e] = dist(gen);
  }
}

}  // namespace gb

extern "C" {

const char* gb_last_error(void) { return g_last_error.c_str(); }
int gb_version(void) { return 10000; }

void gb_host_csr_init(gb_host_csr* g) {
  if (!g) return;
  std::memset(g, 0, sizeof(*g));
}

void gb_host_csr_free(gb_host_csr* g) {
  if (!g) return;
  std::free(g->end_offs);
  std::free(g->col);
  std::free(g->w_u32);
  std::free(g->w_f32);
  std::memset(g, 0, sizeof(*g));
}

int gb_gr_read(const char* path, int edge_bytes, gb_host_csr* out) {
  clear_error();
  if (!path || !out) GB_FAIL(GB_ERR_ARG, "gb_gr_read: null argument");
  if (edge_bytes != 0 && edge_bytes != 4 && edge_bytes != -4)
    GB_FAIL(GB_ERR_ARG, "gb_gr_read: edge_bytes must be 0, 4 or -4");
  FILE* f = std::fopen(path, "rb");
  if (!f) GB_FAIL(GB_ERR_FILE, "cannot open %s: %s", path, std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const uint64_t fsize = (uint64_t)std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  uint64_t hdr[4];
  if (fsize < sizeof(hdr) || std::fread(hdr, sizeof(uint64_t), 4, f) != 4) {
    std::fclose(f);
    GB_FAIL(GB_ERR_FORMAT, "%s: truncated header", path);
  }
  const uint64_t version = hdr[0], sizeof_edge = hdr[1], n64 = hdr[2], m = hdr[3];
  if (version != 1 && version != 2) {
    std::fclose(f);
    GB_FAIL(GB_ERR_FORMAT, "%s: unknown file version %llu", path, (unsigned long long)version);
  }
  if (n64 > 0xFFFFFFFFull) {
    std::fclose(f);
    GB_FAIL(GB_ERR_UNSUPPORTED, "%s: %llu nodes exceed uint32 ids", path, (unsigned long long)n64);
  }
  const uint32_t n = (uint32_t)n64;
  const uint64_t dst_bytes = version == 1 ? 4 : 8;
  // padding: the dst array is re-aligned to 8 bytes (v1 with odd m pads 4
  // bytes; FileGraph.cpp:120-134 applies the numEdges % 2 step to v2 as well)
  const uint64_t pad = (m % 2) ? dst_bytes : 0;
  const uint64_t need = 32 + 8 * n64 + dst_bytes * m + pad;
  if (fsize < need) {
    std::fclose(f);
    GB_FAIL(GB_ERR_FORMAT, "%s: file has %llu bytes, header needs %llu", path,
            (unsigned long long)fsize, (unsigned long long)need);
  }
  if (edge_bytes != 0 && sizeof_edge != (uint64_t)std::abs(edge_bytes)) {
    std::fclose(f);
    GB_FAIL(GB_ERR_FORMAT, "%s: sizeofEdge %llu does not match requested %d", path,
            (unsigned long long)sizeof_edge, std::abs(edge_bytes));
  }
  if (edge_bytes != 0 && fsize < need + sizeof_edge * m) {
    std::fclose(f);
    GB_FAIL(GB_ERR_FORMAT, "%s: edge data section truncated", path);
  }
  gb_host_csr g;
  gb_host_csr_init(&g);
  g.n = n;
  g.m = m;
  g.end_offs = xmalloc<uint64_t>(n);
  g.col = xmalloc<uint32_t>(m);
  if (!g.end_offs || !g.col) {
    std::fclose(f);
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
  bool ok = std::fread(g.end_offs, sizeof(uint64_t), n, f) == n;
  if (ok && version == 1) {
    ok = std::fread(g.col, sizeof(uint32_t), m, f) == m;
  } else if (ok) {
    std::vector<uint64_t> tmp(1 << 20);
    for (uint64_t done = 0; ok && done < m;) {
      uint64_t k = std::min<uint64_t>(tmp.size(), m - done);
      ok = std::fread(tmp.data(), sizeof(uint64_t), k, f) == k;
      for (uint64_t i = 0; ok && i < k; ++i) {
        if (tmp[i] >= n64) ok = false;
        g.col[done + i] = (uint32_t)tmp[i];
      }
      done += k;
    }
  }
  if (ok && pad) ok = std::fseek(f, (long)pad, SEEK_CUR) == 0;
  if (ok && edge_bytes == 4) {
    g.w_u32 = xmalloc<uint32_t>(m);
    ok = g.w_u32 && std::fread(g.w_u32, 4, m, f) == m;
  } else if (ok && edge_bytes == -4) {
    g.w_f32 = xmalloc<float>(m);
    ok = g.w_f32 && std::fread(g.w_f32, 4, m, f) == m;
  }
  std::fclose(f);
  if (!ok) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_FORMAT, "%s: short read or destination id out of range", path);
  }
  // validate offsets and destinations
  uint64_t prev = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (g.end_offs[v] < prev || g.end_offs[v] > m) {
      gb_host_csr_free(&g);
      GB_FAIL(GB_ERR_FORMAT, "%s: edge index of node %u is not monotone", path, v);
    }
    prev = g.end_offs[v];
  }
  if (n > 0 && g.end_offs[n - 1] != m) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_FORMAT, "%s: last edge index %llu != numEdges %llu", path,
            (unsigned long long)g.end_offs[n - 1], (unsigned long long)m);
  }
  if (n == 0 && m != 0) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_FORMAT, "%s: edges without nodes", path);
  }
  bool bad = false;
#pragma omp parallel for reduction(|| : bad)
  for (int64_t e = 0; e < (int64_t)m; ++e) bad = bad || (g.col[e] >= n);
  if (bad) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_FORMAT, "%s: destination id >= numNodes", path);
  }
  gb_host_csr_free(out);
  *out = g;
  return GB_OK;
}

int gb_gr_write(const char* path, const gb_host_csr* g, int edge_bytes) {
  clear_error();
  if (!path || !g) GB_FAIL(GB_ERR_ARG, "gb_gr_write: null argument");
  if (edge_bytes == 4 && !g->w_u32) GB_FAIL(GB_ERR_ARG, "gb_gr_write: no uint32 weights");
  if (edge_bytes == -4 && !g->w_f32) GB_FAIL(GB_ERR_ARG, "gb_gr_write: no float weights");
  if (edge_bytes != 0 && edge_bytes != 4 && edge_bytes != -4)
    GB_FAIL(GB_ERR_ARG, "gb_gr_write: edge_bytes must be 0, 4 or -4");
  FILE* f = std::fopen(path, "wb");
  if (!f) GB_FAIL(GB_ERR_FILE, "cannot create %s: %s", path, std::strerror(errno));
  uint64_t hdr[4] = {1, (uint64_t)std::abs(edge_bytes), g->n, g->m};
  bool ok = std::fwrite(hdr, 8, 4, f) == 4;
  ok = ok && std::fwrite(g->end_offs, 8, g->n, f) == g->n;
  ok = ok && std::fwrite(g->col, 4, g->m, f) == g->m;
  if (ok && (g->m % 2)) {
    uint32_t zero = 0;
    ok = std::fwrite(&zero, 4, 1, f) == 1;
  }
  if (ok && edge_bytes == 4) ok = std::fwrite(g->w_u32, 4, g->m, f) == g->m;
  if (ok && edge_bytes == -4) ok = std::fwrite(g->w_f32, 4, g->m, f) == g->m;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) GB_FAIL(GB_ERR_FILE, "write to %s failed", path);
  return GB_OK;
}

int gb_edgelist_to_csr(const char* path, int skip_first_line, char delim,
                       gb_host_csr* out) {
  clear_error();
  if (!path || !out) GB_FAIL(GB_ERR_ARG, "gb_edgelist_to_csr: null argument");
  std::ifstream in(path);
  if (!in.is_open()) GB_FAIL(GB_ERR_FILE, "cannot open %s", path);
  std::string line;
  if (skip_first_line) std::getline(in, line);
  std::vector<std::pair<uint64_t, uint64_t>> arcs;
  uint64_t maxid = 0;
  bool any = false;
  while (std::getline(in, line)) {
    std::stringstream iss(line);
    uint64_t s, d;
    char rd;
    if (!(iss >> s)) continue;
    if (delim && (!(iss >> rd) || rd != delim)) continue;
    if (!(iss >> d)) continue;
    arcs.emplace_back(s, d);
    maxid = std::max(maxid, std::max(s, d));
    any = true;
  }
  const uint64_t n64 = any ? maxid + 1 : 1;  // graph-convert: numNodes = max id + 1
  if (n64 > 0xFFFFFFFFull) GB_FAIL(GB_ERR_UNSUPPORTED, "%s: node id exceeds uint32", path);
  const uint32_t n = (uint32_t)n64;
  gb_host_csr g;
  gb_host_csr_init(&g);
  g.n = n;
  g.m = arcs.size();
  g.end_offs = xmalloc<uint64_t>(n);
  g.col = xmalloc<uint32_t>(g.m);
  if (!g.end_offs || !g.col) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
  std::vector<uint64_t> deg(n, 0);
  for (auto& a : arcs) deg[a.first]++;
  std::vector<uint64_t> cur(n, 0);
  uint64_t acc = 0;
  for (uint32_t v = 0; v < n; ++v) {
    cur[v] = acc;
    acc += deg[v];
    g.end_offs[v] = acc;
  }
  for (auto& a : arcs) g.col[cur[a.first]++] = (uint32_t)a.second;  // stable per source
  gb_host_csr_free(out);
  *out = g;
  return GB_OK;
}

int gb_csr_to_edgelist(const char* path, const gb_host_csr* g) {
  clear_error();
  if (!path || !g) GB_FAIL(GB_ERR_ARG, "gb_csr_to_edgelist: null argument");
  FILE* f = std::fopen(path, "w");
  if (!f) GB_FAIL(GB_ERR_FILE, "cannot create %s", path);
  uint64_t b = 0;
  for (uint32_t v = 0; v < g->n; ++v) {
    for (uint64_t e = b; e < g->end_offs[v]; ++e) std::fprintf(f, "%u %u\n", v, g->col[e]);
    b = g->end_offs[v];
  }
  if (std::fclose(f) != 0) GB_FAIL(GB_ERR_FILE, "write to %s failed", path);
  return GB_OK;
}

int gb_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                uint64_t seed, int symmetrize, int permute, uint32_t* perm_out,
                gb_host_csr* out) {
  clear_error();
  if (!out) GB_FAIL(GB_ERR_ARG, "gb_gen_rmat: null output");
  if (scale == 0 || scale > 31) GB_FAIL(GB_ERR_ARG, "gb_gen_rmat: scale must be in [1,31]");
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    GB_FAIL(GB_ERR_ARG, "gb_gen_rmat: bad quadrant probabilities");
  const uint32_t n = 1u << scale;
  const uint64_t ndraws = (uint64_t)edge_factor << scale;
  // 32-bit integer thresholds: quadrant choice is exact integer arithmetic
  const uint64_t two32 = 1ull << 32;
  const uint64_t ta = (uint64_t)std::floor(a * (double)two32);
  const uint64_t tab = (uint64_t)std::floor((a + b) * (double)two32);
  const uint64_t tabc = (uint64_t)std::floor((a + b + c) * (double)two32);
  const uint64_t key = stream_key(seed, kTagRmat);
  const uint32_t words = (scale + 1) / 2;  // two 32-bit choices per 64-bit draw

  std::vector<uint32_t> perm;
  if (permute) {
    perm.resize(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    const uint64_t pk = stream_key(seed, kTagPerm);
    for (uint32_t i = n - 1; i > 0; --i) {  // Fisher-Yates
      uint32_t j = (uint32_t)mulhi64(rand_at(pk, i), (uint64_t)i + 1);
      std::swap(perm[i], perm[j]);
    }
    if (perm_out) std::memcpy(perm_out, perm.data(), sizeof(uint32_t) * n);
  } else if (perm_out) {
    for (uint32_t i = 0; i < n; ++i) perm_out[i] = i;
  }
  const uint32_t* P = permute ? perm.data() : nullptr;
  auto emit = [&](uint64_t i, auto&& fn) {
    uint32_t u = 0, v = 0;
    for (uint32_t w = 0; w < words; ++w) {
      const uint64_t r = rand_at(key, i * words + w);
      for (uint32_t h = 0; h < 2 && 2 * w + h < scale; ++h) {
        const uint64_t x = h ? (r >> 32) : (r & 0xFFFFFFFFull);
        uint32_t bu, bv;
        if (x < ta) { bu = 0; bv = 0; }
        else if (x < tab) { bu = 0; bv = 1; }
        else if (x < tabc) { bu = 1; bv = 0; }
        else { bu = 1; bv = 1; }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
    }
    if (u == v) return;  // self-loop removed
    if (P) { u = P[u]; v = P[v]; }
    fn(u, v);
    if (symmetrize) fn(v, u);
  };
  return build_csr_from_stream(n, ndraws, emit, out);
}

int gb_gen_grid2d(uint32_t rows, uint32_t cols, gb_host_csr* out) {
  clear_error();
  if (!out || rows == 0 || cols == 0) GB_FAIL(GB_ERR_ARG, "gb_gen_grid2d: bad argument");
  const uint64_t n64 = (uint64_t)rows * cols;
  if (n64 > 0xFFFFFFFFull) GB_FAIL(GB_ERR_ARG, "gb_gen_grid2d: too many nodes");
  const uint32_t n = (uint32_t)n64;
  gb_host_csr g;
  gb_host_csr_init(&g);
  g.n = n;
  g.end_offs = xmalloc<uint64_t>(n);
  const uint64_t m = 2ull * rows * (cols - 1) + 2ull * cols * (rows - 1);
  g.m = m;
  g.col = xmalloc<uint32_t>(m);
  if (!g.end_offs || !g.col) {
    gb_host_csr_free(&g);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
  // degree of (r,c) = (r>0)+(c>0)+(c<cols-1)+(r<rows-1); offsets by rows
  auto deg = [&](uint32_t r, uint32_t c) -> uint32_t {
    return (r > 0) + (c > 0) + (c + 1 < cols) + (r + 1 < rows);
  };
  std::vector<uint64_t> row_start(rows + 1, 0);
  for (uint32_t r = 0; r < rows; ++r) {
    uint64_t s = 0;
    for (uint32_t c = 0; c < cols; ++c) s += deg(r, c);
    row_start[r + 1] = row_start[r] + s;
  }
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)rows; ++r) {
    uint64_t e = row_start[r];
    for (uint32_t c = 0; c < cols; ++c) {
      const uint32_t v = (uint32_t)r * cols + c;
      if (r > 0) g.col[e++] = v - cols;
      if (c > 0) g.col[e++] = v - 1;
      if (c + 1 < cols) g.col[e++] = v + 1;
      if (r + 1 < (int64_t)rows) g.col[e++] = v + cols;
      g.end_offs[v] = e;
    }
  }
  gb_host_csr_free(out);
  *out = g;
  return GB_OK;
}

int gb_gen_er(uint32_t n, double mean_degree, uint64_t seed, gb_host_csr* out) {
  clear_error();
  if (!out || n < 2 || mean_degree < 0) GB_FAIL(GB_ERR_ARG, "gb_gen_er: bad argument");
  const uint64_t M = (uint64_t)std::llround((double)n * mean_degree / 2.0);
  const uint64_t key = stream_key(seed, kTagEr);
  auto emit = [&](uint64_t i, auto&& fn) {
    const uint32_t u = (uint32_t)mulhi64(rand_at(key, 2 * i), n);
    const uint32_t v = (uint32_t)mulhi64(rand_at(key, 2 * i + 1), n);
    if (u == v) return;
    fn(u, v);
    fn(v, u);
  };
  return build_csr_from_stream(n, M, emit, out);
}

int gb_assign_weights_u32(gb_host_csr* g, uint32_t lo, uint32_t hi, uint64_t seed) {
  clear_error();
  if (!g || hi < lo) GB_FAIL(GB_ERR_ARG, "gb_assign_weights_u32: bad argument");
  std::free(g->w_u32);
  g->w_u32 = xmalloc<uint32_t>(g->m);
  if (!g->w_u32) GB_FAIL(GB_ERR_OOM, "host allocation failed");
  const uint64_t key = stream_key(seed, kTagWeightU32);
  const uint64_t span = (uint64_t)hi - lo + 1;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)g->m; ++e)
    g->w_u32[e] = lo + (uint32_t)mulhi64(rand_at(key, (uint64_t)e), span);
  return GB_OK;
}

int gb_assign_weights_f32(gb_host_csr* g, uint64_t seed) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_assign_weights_f32: null graph");
  std::free(g->w_f32);
  g->w_f32 = xmalloc<float>(g->m);
  if (!g->w_f32) GB_FAIL(GB_ERR_OOM, "host allocation failed");
  const uint64_t key = stream_key(seed, kTagWeightF32);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)g->m; ++e) {
    // 24 random bits -> (0,1], exactly representable in fp32
    const uint64_t r = (rand_at(key, (uint64_t)e) >> 40) + 1;
    g->w_f32[e] = (float)r * (1.0f / 16777216.0f);
  }
  return GB_OK;
}

// gr2randomweightgr exactly as the reference converter draws its weights
// (tools/graph-convert/graph-convert.cpp:1145-1190): one default-constructed
// std::mt19937 and a std::uniform_int_distribution<uint32_t>(min, max) (or
// std::uniform_real_distribution<float>(min, max)) evaluated once per arc in
// arc order.  The draws come from this build's C++ standard library, so they
// equal the converter's output when both use the same library (the
// distributions' algorithms are implementation-defined).
int gb_assign_weights_reference(gb_host_csr* g, int min_value, int max_value, int edge_bytes) {
  clear_error();
  if (!g) GB_FAIL(GB_ERR_ARG, "gb_assign_weights_reference: null graph");
  const int st = check_reference_weights(min_value, max_value, edge_bytes, "gb_assign_weights_reference");
  if (st != GB_OK) return st;
  void** slot = edge_bytes == 4 ? reinterpret_cast<void**>(&g->w_u32) : reinterpret_cast<void**>(&g->w_f32);
  std::free(*slot);
  *slot = xmalloc<uint32_t>(g->m);
  if (!*slot && g->m) GB_FAIL(GB_ERR_OOM, "host allocation failed");
  draw_reference_weights(g->m, min_value, max_value, edge_bytes, *slot);
  return GB_OK;
}

int gb_transpose_host(const gb_host_csr* g, gb_host_csr* out, uint64_t* edge_map) {
  clear_error();
  if (!g || !out) GB_FAIL(GB_ERR_ARG, "gb_transpose_host: null argument");
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  gb_host_csr t;
  gb_host_csr_init(&t);
  t.n = n;
  t.m = m;
  t.end_offs = xmalloc<uint64_t>(n);
  t.col = xmalloc<uint32_t>(m);
  if (g->w_u32) t.w_u32 = xmalloc<uint32_t>(m);
  if (g->w_f32) t.w_f32 = xmalloc<float>(m);
  if (!t.end_offs || !t.col || (g->w_u32 && !t.w_u32) || (g->w_f32 && !t.w_f32)) {
    gb_host_csr_free(&t);
    GB_FAIL(GB_ERR_OOM, "host allocation failed");
  }
  std::vector<uint64_t> cur(n + 1, 0);
  for (uint64_t e = 0; e < m; ++e) cur[g->col[e] + 1]++;
  for (uint32_t v = 0; v < n; ++v) cur[v + 1] += cur[v];
  for (uint32_t v = 0; v < n; ++v) t.end_offs[v] = cur[v + 1];
  uint64_t b = 0;
  for (uint32_t u = 0; u < n; ++u) {  // sources in ascending order -> sorted rows
    for (uint64_t e = b; e < g->end_offs[u]; ++e) {
      const uint64_t p = cur[g->col[e]]++;
      t.col[p] = u;
      if (t.w_u32) t.w_u32[p] = g->w_u32[e];
      if (t.w_f32) t.w_f32[p] = g->w_f32[e];
      if (edge_map) edge_map[p] = e;
    }
    b = g->end_offs[u];
  }
  gb_host_csr_free(out);
  *out = t;
  return GB_OK;
}

}  // extern "C"
