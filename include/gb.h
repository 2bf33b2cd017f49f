/*
 * gb.h -- C ABI of the B200-native CSR edge-map library (libgb.so).
 *
 * This header is the drop-in boundary for the Galois lonestar analytics hot
 * path: BFS, delta-stepping SSSP, label-propagation connected components,
 * PageRank (pull-topological and residual-push), Brandes betweenness
 * centrality, and a differentiable personalised PageRank.  Every entry point
 * takes plain pointers and sizes, returns an int status (GB_OK == 0, negative
 * on error, message in gb_last_error()), and never aborts or exits.
 *
 * Reference interfaces replaced (paths relative to the Galois source tree):
 *   graph + .gr I/O     libgalois/include/galois/graphs/LC_CSR_Graph.h:879-1011
 *                       (readGraphFromGRFile), libgalois/src/FileGraph.cpp:44-53
 *                       (format), libgpu/src/csr_graph.cu:172-315 (device mirror)
 *   per-operator C ABI  lonestar/analytics/distributed/bfs/bfs_push_cuda.h:103-145
 *                       (BFS_cuda / InitializeGraph_allNodes_cuda pattern over
 *                       an opaque struct CUDA_Context*)
 *   algorithms          lonestar/analytics/cpu/bfs/bfs.cpp:244-293,
 *                       lonestar/analytics/cpu/sssp/SSSP.cpp:118-173,
 *                       lonestar/analytics/cpu/connected-components/
 *                       ConnectedComponents.cpp:183-230,
 *                       lonestar/analytics/cpu/pagerank/PageRank-pull.cpp:196-251,
 *                       lonestar/analytics/cpu/pagerank/PageRank-push.cpp:68-188,
 *                       lonestar/analytics/cpu/betweennesscentrality/
 *                       LevelStructs.h:87-185
 *   python entry points python/galois/_bfs.pyx:171, _sssp.pyx:154,
 *                       _pagerank.pyx:157, _connected_components.pyx:87
 *
 * Conventions
 *   - Node ids are uint32; edge offsets are uint64.  Offsets passed IN follow
 *     the LC_CSR_Graph layout: n END offsets, begin(v) = v ? end[v-1] : 0
 *     (LC_CSR_Graph.h:142,172-178).
 *   - Unreached BFS/SSSP vertices hold GB_DIST_INFINITY = UINT_MAX/2-1
 *     (lonestar/liblonestar/include/Lonestar/BFS_SSSP.h:31-32).
 *   - Output buffers may be host or device memory; the library detects which.
 *     Device outputs keep the call asynchronous on `stream` (unless `stats` is
 *     non-NULL, which synchronises the stream to read counters).
 *   - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *     default stream.
 *   - A gb_graph handle is not re-entrant: use one handle per host thread.
 */
#ifndef GB_H
#define GB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GB_OK 0
#define GB_ERR_ARG (-1)           /* bad argument (null pointer, id >= n, ...) */
#define GB_ERR_OOM (-2)           /* host or device allocation failed          */
#define GB_ERR_CUDA (-3)          /* a CUDA runtime call failed                */
#define GB_ERR_TIMEOUT (-4)       /* a bounded device wait or loop gave up     */
#define GB_ERR_FILE (-5)          /* file could not be opened/read/written     */
#define GB_ERR_FORMAT (-6)        /* malformed .gr / edge list                 */
#define GB_ERR_NOT_CONVERGED (-7) /* iteration cap reached (result still set)  */
#define GB_ERR_UNSUPPORTED (-8)   /* valid request this build does not handle  */
#define GB_ERR_CAPACITY (-9)      /* input larger than a fixed-size buffer     */

#define GB_DIST_INFINITY 2147483646u /* std::numeric_limits<uint32_t>::max()/2-1 */

/* Last error message of the calling host thread ("" if none). */
const char* gb_last_error(void);
/* Library version: major*10000 + minor*100 + patch. */
int gb_version(void);

/* ---- host-side CSR (no GPU needed) -------------------------------------- */
/* Arrays are malloc'd by the library and released by gb_host_csr_free.
 * end_offs follows the LC_CSR_Graph end-offset layout (n entries). */
typedef struct gb_host_csr {
  uint32_t n;
  uint64_t m;
  uint64_t* end_offs; /* [n]                         */
  uint32_t* col;      /* [m] destination ids         */
  uint32_t* w_u32;    /* [m] or NULL (integer weights) */
  float* w_f32;       /* [m] or NULL (float weights)   */
} gb_host_csr;

void gb_host_csr_init(gb_host_csr* g);
void gb_host_csr_free(gb_host_csr* g);

/* .gr v1/v2 reader (FileGraph.cpp:44-53, 104-135; LC_CSR_Graph.h:879-1011).
 * edge_bytes selects how the edge-data section is interpreted:
 *   0 = ignore, 4 = uint32 weights into w_u32, -4 = float weights into w_f32.
 * A file whose sizeofEdge differs from |edge_bytes| (when non-zero) is
 * rejected with GB_ERR_FORMAT. */
int gb_gr_read(const char* path, int edge_bytes, gb_host_csr* out);
/* .gr v1 writer: edge_bytes 0 (void), 4 (w_u32) or -4 (w_f32). */
int gb_gr_write(const char* path, const gb_host_csr* g, int edge_bytes);
/* Text edge lists (tools/graph-convert/graph-convert.cpp:351-530):
 * "src dst" per line, or "src<delim>dst" with skip_first_line for CSV.
 * Lines that do not parse are ignored; per-source order is preserved. */
int gb_edgelist_to_csr(const char* path, int skip_first_line, char delim,
                       gb_host_csr* out);
/* gr2edgelist (graph-convert.cpp:867-900): "src dst\n" per edge. */
int gb_csr_to_edgelist(const char* path, const gb_host_csr* g);

/* Seeded synthetic generators (SplitMix64 counter-based streams).
 * RMAT: edge_factor * 2^scale draws with quadrant probabilities a,b,c
 * (d = 1-a-b-c); self-loops and duplicate arcs removed; if symmetrize, every
 * arc gets its reverse; if permute, vertex ids are relabelled by a seeded
 * random permutation (perm_out[i] = new id of generator vertex i, may be
 * NULL).  Adjacency lists are sorted ascending. */
int gb_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                double c, uint64_t seed, int symmetrize, int permute,
                uint32_t* perm_out, gb_host_csr* out);
/* rows x cols 4-neighbour grid, both arc directions, row-major ids. */
int gb_gen_grid2d(uint32_t rows, uint32_t cols, gb_host_csr* out);
/* Erdos-Renyi G(n, M) with M = round(n*mean_degree/2) undirected draws,
 * symmetrised, self-loops and duplicates removed. */
int gb_gen_er(uint32_t n, double mean_degree, uint64_t seed, gb_host_csr* out);
/* Per-arc weights by CSR position: uint32 uniform in [lo,hi], or float
 * uniform in (0,1]. */
int gb_assign_weights_u32(gb_host_csr* g, uint32_t lo, uint32_t hi,
                          uint64_t seed);
int gb_assign_weights_f32(gb_host_csr* g, uint64_t seed);
/* gr2randomweightgr as the reference converter draws it
 * (tools/graph-convert/graph-convert.cpp:1145-1190): a default-constructed
 * std::mt19937 and std::uniform_int_distribution<uint32_t>(min_value,
 * max_value) (edge_bytes 4, into w_u32) or
 * std::uniform_real_distribution<float>(min_value, max_value) (edge_bytes -4,
 * into w_f32), one draw per arc in arc order (the converter's defaults are
 * min 1, max 100).  Serial, from the C++ standard library this library was
 * built with. */
int gb_assign_weights_reference(gb_host_csr* g, int min_value, int max_value,
                                int edge_bytes);
/* Transpose (LC_CSR_Graph.h:617-712 semantics): arcs u->v become v->u, edge
 * data follows its arc, adjacency sorted by source id.  If edge_map is
 * non-NULL it receives, for every transposed arc, its index in g. */
int gb_transpose_host(const gb_host_csr* g, gb_host_csr* out,
                      uint64_t* edge_map);

/* ---- device graph ------------------------------------------------------- */
typedef struct gb_graph gb_graph;

/* Upload a CSR to `device`.  end_offs: LC layout (n entries).  Either weight
 * array may be NULL.  symmetric != 0 declares in-edges == out-edges (the
 * -symmetricGraph flag, BoilerPlate.cpp:38-41), which enables pull/bottom-up
 * steps without a transpose.  Inputs may be host or device pointers.
 * Host inputs are copied on a stream of the library's own that does not wait
 * for kernels running on other streams (an upload can overlap a kernel of
 * another graph); device inputs are copied on the default stream, after the
 * work queued before the call.  The call returns when the graph is on the
 * device. */
int gb_graph_upload(const uint64_t* end_offs, const uint32_t* col,
                    const uint32_t* w_u32, const float* w_f32, uint32_t n,
                    uint64_t m, int symmetric, int device, gb_graph** out);
int gb_graph_load_gr(const char* path, int edge_bytes, int symmetric,
                     int device, gb_graph** out);
int gb_graph_free(gb_graph* g);
/* gb_graph_free keeps the graph's large device blocks (and its pinned
 * readback buffer) in a process-wide cache for the next upload of the same
 * shape; this releases every cached block. */
int gb_pool_trim(void);
int gb_graph_info(const gb_graph* g, uint32_t* n, uint64_t* m,
                  int* symmetric);
/* Device-resident begin offsets (n+1), columns and weights (NULL if absent):
 * lets a caller build operators (include/gb_operator.cuh) over the mirror. */
int gb_graph_device_arrays(const gb_graph* g, const uint64_t** offs,
                           const uint32_t** col, const uint32_t** w_u32,
                           const float** w_f32);
/* Build the in-edge (transposed) CSR on the device, with the map from each
 * transposed arc to its original arc.  Needed for pull/bottom-up steps on
 * directed graphs and for the PPR forward pass. */
int gb_graph_build_transpose(gb_graph* g, void* stream);

/* Conversions applied to the device mirror (tools/graph-convert on a file
 * in the reference).  gb_graph_symmetrize: gr2sgr (graph-convert.cpp:
 * 1350-1364, FileGraph.h:764-826): every arc (u,v) with u != v gains the
 * reverse arc (v,u) with the same weights; with cleanup != 0 it continues as
 * gr2cgr (Cleanup, graph-convert.cpp:1902-2024), dropping self-loops and
 * repeated arcs (the first copy in arc order, forward arcs before reverse
 * ones, keeps its weights).  Rows come out sorted by destination; the graph
 * is marked symmetric; cached derived arrays are dropped.  Not for a
 * relabelled graph (call it before gb_graph_reorder); m < 2^31.
 * gb_graph_assign_weights_u32 / _f32: gr2randomweightgr
 * (graph-convert.cpp:1169-1190) with the counter-based stream of the host
 * generators, so the result equals gb_assign_weights_u32 / _f32 on the same
 * arcs and seed (uniform in [lo, hi]; fp32 in (0, 1]). */
int gb_graph_symmetrize(gb_graph* g, int cleanup, void* stream);
/* gb_assign_weights_reference on the device mirror's arcs (drawn on the host
 * in arc order, then uploaded; synchronous).  Before gb_graph_reorder. */
int gb_graph_assign_weights_reference(gb_graph* g, int min_value, int max_value,
                                      int edge_bytes, void* stream);
int gb_graph_assign_weights_u32(gb_graph* g, uint32_t lo, uint32_t hi,
                                uint64_t seed, void* stream);
int gb_graph_assign_weights_f32(gb_graph* g, uint64_t seed, void* stream);

/* Degree-ordered relabelling of the device mirror (no counterpart in the
 * reference, which keeps file order).  GB_ORDER_DEGREE renumbers vertices by
 * descending out-degree (ties by id) and sorts each adjacency list (when
 * m < 2^31; larger graphs keep the relabelled file order), so that the
 * gathers of high-degree vertices share cache lines.  GB_ORDER_DEGREE_UNSORTED
 * skips the row sort.  Every algorithm call keeps taking and returning
 * ORIGINAL vertex ids (sources are mapped in, results mapped out; CC labels
 * stay the minimum original id of the component), so results are unchanged;
 * gb_graph_device_arrays and gb_graph_build_transpose then describe the
 * relabelled graph.  Cannot be undone; GB_ORDER_NONE is accepted only on a
 * graph that was never reordered.  Multi-graph and PPR calls return
 * GB_ERR_UNSUPPORTED on a reordered graph. */
#define GB_ORDER_NONE 0
#define GB_ORDER_DEGREE 1
#define GB_ORDER_DEGREE_UNSORTED 2
/* GB_ORDER_LOCALITY: for bounded-degree, high-diameter graphs (grids, meshes,
 * road-like graphs).  Vertices are numbered in the Morton order of their BFS
 * distances to two far-apart landmark vertices (found by BFS: the vertex
 * farthest from vertex 0, the one farthest from it, and the one farthest
 * from both), so consecutive ids form compact 2-D patches; rows are sorted. */
#define GB_ORDER_LOCALITY 3
/* GB_ORDER_AUTO: GB_ORDER_LOCALITY when no vertex has more than 16 stored
 * arcs, else GB_ORDER_DEGREE. */
#define GB_ORDER_AUTO 4
int gb_graph_reorder(gb_graph* g, int order, void* stream);
/* The order a graph was relabelled with (GB_ORDER_NONE if it never was;
 * GB_ORDER_AUTO reports the order it chose). */
int gb_graph_order(const gb_graph* g, int* order);
/* Device permutation of a reordered graph: new_to_old[internal id] =
 * original id, old_to_new the inverse; both NULL if not reordered. */
int gb_graph_permutation(const gb_graph* g, const uint32_t** new_to_old,
                         const uint32_t** old_to_new);

/* Per-call statistics (all optional). */
typedef struct gb_stats {
  uint64_t vertices_reached; /* n_r                                          */
  uint64_t edges_reached;    /* m_r = sum of out-degrees of reached vertices  */
  uint64_t edges_scanned;    /* arcs actually read                           */
  uint64_t relaxations;      /* successful atomicMin / pushes                */
  uint32_t rounds;           /* levels / phases / sweeps / iterations        */
  uint32_t pull_rounds;      /* bottom-up rounds (BFS)                       */
  uint32_t buckets;          /* delta buckets processed (SSSP)               */
  uint32_t launches;         /* kernels launched by this call                */
  double residual;           /* final L1 residual (PageRank)                 */
  double kernel_ms;          /* device time of the main (persistent) kernel,
                                CUDA events on the launching stream          */
} gb_stats;

/* Tuning knobs; zero fields mean "library default / autotuned". */
typedef struct gb_tuning {
  uint32_t heavy_degree; /* vertices above this degree are edge-tiled      */
  uint32_t tile_edges;   /* edges per tile for heavy vertices              */
  uint32_t block_threads;/* CTA size for persistent kernels (multiple of 32)*/
  uint32_t blocks_per_sm;/* persistent CTAs per SM (0 = max resident)      */
  float do_alpha;        /* push->pull switch (bfsDirectionOpt.cpp:68-72)  */
  float do_beta;         /* pull->push switch (bfsDirectionOpt.cpp:73-77)  */
  int direction_opt;     /* 0 = pull steps allowed when in-edges exist, 2 = push only */
  int local_depth;       /* SSSP: per-warp local-queue rounds per phase
                            (0 = library default, < 0 = off); the region
                            kernel does not use it */
  int sssp_async;        /* SSSP with local queues on a graph whose every
                            vertex is light: 1 = asynchronous buckets (no
                            grid barrier inside a bucket), 2 = the same over
                            fixed-width rows when the degree is <= 8 (one
                            memory round trip per hop: faster on narrow,
                            chain-like graphs, slower on wide wavefronts);
                            3 = regions of 2048 consecutive ids relaxed in
                            shared memory when every region holds at most
                            8192 arcs (for graphs numbered by locality,
                            GB_ORDER_LOCALITY; otherwise as 1); stats:
                            rounds = region visits, pull_rounds =
                            shared-memory rounds;
                            0 = library default: regions on a
                            GB_ORDER_LOCALITY graph whose regions fit and
                            keep >= 90 % of the arcs inside, else a grid
                            barrier after every phase; < 0 = a grid
                            barrier after every phase */
} gb_tuning;
int gb_graph_set_tuning(gb_graph* g, const gb_tuning* t);
int gb_graph_get_tuning(const gb_graph* g, gb_tuning* t);

/* BFS levels from src (bfs.cpp:244-293; bfsDirectionOpt.cpp:204-342 for
 * the push/pull switch).  level_out[n], unreached = GB_DIST_INFINITY. */
int gb_bfs(gb_graph* g, uint32_t src, uint32_t* level_out, gb_stats* stats,
           void* stream);

/* BFS parents from src, the output of the direction-optimising lonestar BFS
 * (bfsDirectionOpt.cpp:204-342, which stores the parent, not the level:
 * :284-285, :325).  parent_out[src] = 0 as the reference leaves the source's
 * datum (:229); unreached = GB_DIST_INFINITY; every other reached v gets the
 * smallest id among its in-neighbours one level closer to src -- the
 * reference keeps whichever such in-neighbour wins a compare-and-swap, so
 * this is one of its possible outputs, made reproducible.  level_out
 * (nullable) receives the levels as gb_bfs gives them.  A directed graph
 * needs its in-edges: the transpose is built on first use. */
int gb_bfs_parent(gb_graph* g, uint32_t src, uint32_t* parent_out,
                  uint32_t* level_out, gb_stats* stats, void* stream);

/* Allocation-free BFS (no counterpart in the reference).  For callers that
 * cannot call cudaMalloc -- e.g. a host application that owns and budgets all
 * device memory and forbids libraries from allocating -- this runs the gb_bfs
 * kernels over caller-owned device arrays (offs: n+1 begin offsets, col: m
 * ids, level_out: n) with all scratch in a fixed file-scope device array that
 * every GPU loading libgb keeps until exit.  Limits: n <= 2^20, m <= 2^26
 * (GB_ERR_CAPACITY beyond).  Calls share the array: calls that overlap on the
 * GPU race.  The three arrays must live on the current device (GB_ERR_ARG
 * otherwise); an invalid CSR (offsets not monotone or not ending at m, an id
 * >= n) returns GB_ERR_FORMAT before level_out is written.  The call is
 * synchronous (it waits for `stream`).  symmetric != 0 declares that every
 * arc (u,v) has its reverse (v,u), as gb_graph_upload's flag does, and lets
 * bottom-up steps read the out-arcs as in-arcs; a directed graph must pass 0
 * (push-only levels), or its levels come out wrong. */
int gb_bfs_noalloc(const uint64_t* offs, const uint32_t* col, uint32_t n,
                   uint64_t m, int symmetric, uint32_t src,
                   uint32_t* level_out, void* stream);

/* Delta-stepping SSSP over uint32 weights (SSSP.cpp:118-173, -delta is a
 * shift: bucket = dist >> delta_shift).  dist_out[n]. */
int gb_sssp_delta(gb_graph* g, uint32_t src, uint32_t delta_shift,
                  uint32_t* dist_out, gb_stats* stats, void* stream);

/* Connected components of a symmetric graph; label = minimum vertex id of the
 * component, as LabelProp converges to (ConnectedComponents.cpp:183-230).
 * algo: 0 = label propagation with pointer jumping, 1 = union-find hooking
 * (one sweep), 2 = Afforest-style sampling then hooking. */
#define GB_CC_LABELPROP 0
#define GB_CC_UNIONFIND 1
#define GB_CC_AFFOREST 2
int gb_cc(gb_graph* g, int algo, uint32_t* label_out, gb_stats* stats,
          void* stream);

/* PageRank pull-topological over the graph as stored, which must be the
 * TRANSPOSE of the web graph (the -transposedGraph contract,
 * PageRank-pull.cpp:196-251): rank = alpha*sum(rank[u]/nout[u]) +
 * (1-alpha)/n, nout counted from the stored graph, stop when the L1 change
 * <= tol or after max_iter iterations.  rank_out[n] float.  On a
 * degree-ordered graph (gb_graph_reorder) this and gb_pagerank_pull_residual
 * run over a binned copy of the arcs built on the first call and kept with
 * the graph until gb_graph_free (about 3 bytes per arc plus 4 per
 * (source, 32 K-destination partition) pair: 1.6 GB at RMAT-24; building it
 * takes 12 bytes per arc of temporary device memory).  Where it cannot be
 * built the row sweep runs. */
int gb_pagerank_pull(gb_graph* g, float alpha, float tol, uint32_t max_iter,
                     float* rank_out, uint32_t* iters_out, gb_stats* stats,
                     void* stream);
/* The pull-topological kernel with the initial rank, the base score and the
 * stopping norm as parameters.  python/galois/_pagerank.pyx:86-139 uses
 * init = base = 1-alpha and stops on the MAX |delta| (norm_linf = 1);
 * gb_pagerank_pull is init = 1/n, base = (1-alpha)/n, L1 norm. */
int gb_pagerank_pull_ex(gb_graph* g, float alpha, float tol, uint32_t max_iter,
                        float init, float base, int norm_linf,
                        float* rank_out, uint32_t* iters_out, gb_stats* stats,
                        void* stream);
/* PageRank residual push over out-edges (PageRank-push.cpp:103-188, Sync):
 * value starts 0, residual 1-alpha; a vertex whose residual exceeds tol
 * absorbs it and pushes residual*alpha/outdeg to its out-neighbours. */
int gb_pagerank_push(gb_graph* g, float alpha, float tol, uint32_t max_iter,
                     float* rank_out, uint32_t* iters_out, gb_stats* stats,
                     void* stream);
/* Residual push with the algorithm chosen as PageRank-push.cpp:42-47 does:
 * GB_PR_PUSH_ASYNC (the app's default, :68-101) runs the operator over a
 * worklist with no rounds -- every vertex at the start, then each vertex
 * whose residual an add lifts from below tol to tol or above -- and reports
 * one iteration (max_iter is ignored, as the reference ignores it there);
 * GB_PR_PUSH_SYNC is gb_pagerank_push. */
#define GB_PR_PUSH_ASYNC 0
#define GB_PR_PUSH_SYNC 1
int gb_pagerank_push_ex(gb_graph* g, int algo, float alpha, float tol,
                        uint32_t max_iter, float* rank_out, uint32_t* iters_out,
                        gb_stats* stats, void* stream);
/* PageRank pull-residual (PageRank-pull.cpp:132-190): delta/residual rounds
 * over the stored (transposed) graph. */
int gb_pagerank_pull_residual(gb_graph* g, float alpha, float tol,
                              uint32_t max_iter, float* rank_out,
                              uint32_t* iters_out, gb_stats* stats,
                              void* stream);

/* Brandes betweenness centrality (LevelStructs.h:87-185) accumulated over
 * srcs[0..nsrc).  batch = sources per multi-source launch (1..64); batch 1
 * runs the single-source level-synchronous kernels once per source.
 * fp64 path counts, fp32 dependencies; bc_out[n] float. */
int gb_bc(gb_graph* g, const uint32_t* srcs, uint32_t nsrc, uint32_t batch,
          float* bc_out, gb_stats* stats, void* stream);

/* Many disjoint graphs in one launch: the graphs are packed block-diagonally
 * into a symmetric `g` (vertex ranges graph_first[k] .. graph_first[k+1]-1,
 * graph_first has ngraphs+1 HOST entries, graph_first[ngraphs] == n, no arc
 * leaves its range), BFS runs from graph_first[k] + local_src[k] (host array)
 * for every k at once and CC labels every graph.  Labels are local ids (min
 * local id of the component), levels are per-graph BFS levels.
 * level_out/label_out: [n] (either may be NULL).  The first call on a layout
 * validates it; later calls with device outputs issue only stream-ordered
 * work, so they can be captured in a CUDA graph. */
int gb_multi_graph_bfs_cc(gb_graph* g, const uint32_t* graph_first,
                          uint32_t ngraphs, const uint32_t* local_src,
                          uint32_t* level_out, uint32_t* label_out,
                          gb_stats* stats, void* stream);

/* Personalised PageRank (no counterpart in the reference; an addition beside
 * the PageRank kernels), batched over B teleport vectors, on a directed graph
 * with positive float arc weights w (arc j->i, CSR order).  W~_ij = w_ji / s_j
 * with s_j the out-weight sum of j.  Solves x = (1-alpha) T + alpha W~ x by
 * Jacobi iteration from x0 = (1-alpha) T until the largest per-column L1
 * change is <= tol (or max_iter).
 *   B:        1, or a multiple of 4 up to 128
 *   teleport: dense [n][B] row-major float, device memory
 *   w:        [m] device floats, or NULL for the uploaded w_f32
 *   x_out:    [n][B] row-major float, device memory
 * The transpose is built on first use. */
int gb_ppr_forward(gb_graph* g, uint32_t B, const float* teleport,
                   const float* w, float alpha, float tol, uint32_t max_iter,
                   float* x_out, uint32_t* iters_out, gb_stats* stats,
                   void* stream);
/* Adjoint of gb_ppr_forward: given x (forward solution) and gx = dL/dx, solves
 * lam = gx + alpha W~^T lam by Jacobi iteration until every column's L1
 * change is <= tol times that column's L1 norm of gx (a loss gradient has no
 * fixed scale, unlike a teleport distribution), and returns
 *   grad_teleport[n][B] = (1-alpha) lam
 *   grad_w[m]  = dL/dw_ji = alpha/s_j * sum_b x_j^b (lam_i^b - mu_j^b),
 *                mu_j = (lam_j - gx_j)/alpha, summed over the batch
 * Either output may be NULL; all arrays are device memory. */
int gb_ppr_backward(gb_graph* g, uint32_t B, const float* x, const float* gx,
                    const float* w, float alpha, float tol, uint32_t max_iter,
                    float* grad_teleport, float* grad_w, uint32_t* iters_out,
                    gb_stats* stats, void* stream);

/* Failure detection check (no counterpart in the reference): runs one of the
 * device waits the persistent kernels rely on -- which = 0: the software grid
 * barrier with one CTA that never arrives; 1: a worklist ticket whose chunk is
 * never published -- with a limit of limit_us microseconds (1 .. 2e6).  The
 * wait gives up, the kernel returns, and the call returns GB_ERR_TIMEOUT;
 * the context stays usable.  Synchronous on `stream`. */
int gb_probe_bounded_waits(int which, uint32_t limit_us, void* stream);

/* Autotuner: times candidate degree-bin thresholds, tile sizes, CTA shapes
 * and push/pull switch points for `kernel` ("bfs", "sssp", "cc", "pr") on this
 * graph, keeps the fastest in the handle, and (if cache_path is non-NULL)
 * merges it into a JSON-lines cache keyed by graph class and kernel. */
int gb_autotune(gb_graph* g, const char* kernel, uint32_t src,
                const char* cache_path, gb_tuning* best_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GB_H */
