/*
 * grafeo_cuda.h — C ABI of the B200 (sm_100a) graph hot paths.
 *
 * This is the drop-in boundary for the four algorithm paths of grafeo-cuda
 * (triangle counting, BFS, PageRank, k-truss). Every entry point takes plain
 * pointers and sizes; no CUDA or torch types appear in the signatures. Each
 * declaration names the reference interface it replaces (file:line inside the
 * grafeo-cuda project). The reference's host side is Rust; a Rust `-sys` crate,
 * the Python module and the C++ tools all bind to these symbols.
 *
 * Conventions
 *  - Every fallible call returns a gcu_status. On failure the thread-local
 *    message returned by gcu_last_error() holds the same text as the
 *    reference's `CudaError` Display impl (crates/grafeo-cuda-core/src/error.rs:5-38).
 *  - Calls are synchronous, like the reference's (each syncs its stream before
 *    returning). Results are written into caller-owned host buffers unless a
 *    function says otherwise.
 *  - `seconds` out-parameters are host wall time around the whole call,
 *    including allocation and result copies, as the reference's `time_seconds`
 *    (e.g. crates/grafeo-cuda-algos/src/bfs.rs:43,121-123). They may be NULL.
 */
#ifndef GRAFEO_CUDA_H
#define GRAFEO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GCU_API __attribute__((visibility("default")))
#else
#define GCU_API
#endif

/* ---- status / errors: crates/grafeo-cuda-core/src/error.rs:5-38 ---- */

typedef enum gcu_status {
    GCU_OK = 0,
    GCU_ERR_NO_DEVICE = 1,     /* CudaError::NoDevice */
    GCU_ERR_DRIVER = 2,        /* CudaError::Driver */
    GCU_ERR_OUT_OF_MEMORY = 3, /* CudaError::OutOfMemory{required, available} */
    GCU_ERR_KERNEL = 4,        /* CudaError::Kernel (also argument errors) */
    GCU_ERR_EXPORT = 5,        /* CudaError::Export */
    GCU_ERR_INVALID_CSR = 6    /* CudaError::InvalidCsr */
} gcu_status;

/* Message of the last failed call on this thread ("" if none). */
GCU_API const char* gcu_last_error(void);
/* Library version string, e.g. "0.3.0+b200". */
GCU_API const char* gcu_version(void);
/* Number of visible CUDA devices (0 when there is no driver or device). */
GCU_API int gcu_device_count(void);

/* ---- device: crates/grafeo-cuda-core/src/device.rs:9-66 ---- */

typedef struct gcu_device gcu_device;

/* GpuDevice::new(ordinal) (device.rs:30). Creates one stream for the device. */
GCU_API gcu_status gcu_device_create(int ordinal, gcu_device** out);
/* Drops this handle. Graphs created on it keep the device alive. */
GCU_API void gcu_device_destroy(gcu_device* dev);
/* DeviceProperties{name, ordinal, total_memory} (device.rs:9-17,54). */
GCU_API const char* gcu_device_name(const gcu_device* dev);
GCU_API int gcu_device_ordinal(const gcu_device* dev);
GCU_API uint64_t gcu_device_total_memory(const gcu_device* dev);
GCU_API int gcu_device_sm_count(const gcu_device* dev);
/* GpuDevice::stream() (device.rs:64): the cudaStream_t every call runs on. */
GCU_API void* gcu_device_stream(gcu_device* dev);
GCU_API gcu_status gcu_device_synchronize(gcu_device* dev);

/* Device-time measurement on the device stream (CUDA events), for benchmarks:
 * start records an event, stop records a second one, synchronizes and
 * returns the elapsed milliseconds. Replaces the reference's wall-clock
 * best-of-N (crates/grafeo-cuda-algos/src/bin/gpu_bfs.rs:63-83). */
GCU_API gcu_status gcu_device_timer_start(gcu_device* dev);
GCU_API gcu_status gcu_device_timer_stop(gcu_device* dev, float* ms);
/* Number of kernels this library has launched on the device. */
GCU_API uint64_t gcu_device_launch_count(const gcu_device* dev);
/* When on, every kernel launch is bracketed by CUDA events and its device time
 * is accumulated per kernel name. */
GCU_API void gcu_device_set_kernel_timing(gcu_device* dev, int on);
/* BFS level loop on the device (default, on = 1): a search is one CUDA-graph
 * launch whose WHILE node runs decide + step until the frontier is empty, with
 * no host round trip per level. on = 0 (or per-kernel timing on) drives the
 * levels from the host, reading the counters back after each step. Results
 * are the same either way. No reference counterpart (bfs.rs:42-131 syncs
 * every level). */
GCU_API void gcu_device_set_bfs_device_loop(gcu_device* dev, int on);
/* Writes per-kernel statistics as JSON {"name": [launches, total_ms], ...}
 * into buf (always NUL-terminated) and returns the full length needed. */
GCU_API size_t gcu_device_kernel_stats(gcu_device* dev, char* buf, size_t buflen);
GCU_API void gcu_device_reset_stats(gcu_device* dev);

/* ---- host CSR arrays: crates/grafeo-cuda-core/src/csr_export.rs ---- */

typedef struct gcu_csr gcu_csr; /* CsrArrays (csr_export.rs:16-30), host memory */

/* validate_csr(offsets, targets) (csr_export.rs:71-120), on the host. */
GCU_API gcu_status gcu_validate_csr(const uint32_t* offsets, size_t n_offsets,
                                    const uint32_t* targets, size_t n_targets);
/* from_edge_pairs(edges, num_nodes, symmetric) (csr_export.rs:202-239).
 * pairs holds n_pairs (src, dst) pairs interleaved. */
GCU_API gcu_status gcu_csr_from_edge_pairs(const uint32_t* pairs, size_t n_pairs,
                                           uint32_t num_nodes, int symmetric,
                                           gcu_csr** out);
/* from_edge_pairs_oriented(edges, num_nodes) (csr_export.rs:299-350). */
GCU_API gcu_status gcu_csr_from_edge_pairs_oriented(const uint32_t* pairs, size_t n_pairs,
                                                    uint32_t num_nodes, gcu_csr** out);
/* parse_tsv_to_edges(path) (csr_export.rs:246-287). *pairs is freed with
 * gcu_free_pairs. A missing file is GCU_ERR_EXPORT. */
GCU_API gcu_status gcu_parse_tsv_to_edges(const char* path, uint32_t** pairs,
                                          size_t* n_pairs, uint32_t* num_nodes);
GCU_API void gcu_free_pairs(uint32_t* pairs);
/* Synthetic inputs standing in for Graph500/GraphChallenge files (which the
 * reference loads through parse_tsv_to_edges): R-MAT and Erdos-Renyi, built
 * symmetric without self-loops or duplicates, from a counter-based SplitMix64
 * stream so the graph is the same for any thread count. */
GCU_API gcu_status gcu_generate_rmat(uint32_t scale, uint32_t edge_factor, double a,
                                     double b, double c, uint64_t seed, gcu_csr** out);
GCU_API gcu_status gcu_generate_erdos_renyi(uint32_t num_nodes, uint64_t num_pairs,
                                            uint64_t seed, gcu_csr** out);
GCU_API uint32_t gcu_csr_num_nodes(const gcu_csr* csr);
GCU_API uint64_t gcu_csr_num_edges(const gcu_csr* csr);
GCU_API const uint32_t* gcu_csr_offsets(const gcu_csr* csr);
GCU_API const uint32_t* gcu_csr_targets(const gcu_csr* csr);
GCU_API void gcu_csr_free(gcu_csr* csr);

/* ---- device graph: crates/grafeo-cuda-core/src/gpu_graph.rs:15-88 ---- */

typedef struct gcu_graph gcu_graph;

/* GpuGraph::from_csr_slices(offsets, targets, device) (gpu_graph.rs:66-88) and
 * from_csr_arrays (gpu_graph.rs:46-60). Copies the arrays to the device and
 * validates them there with the same rules and messages as validate_csr;
 * an invalid CSR is GCU_ERR_INVALID_CSR and no graph is returned. */
GCU_API gcu_status gcu_graph_from_csr(gcu_device* dev, const uint32_t* offsets,
                                      size_t n_offsets, const uint32_t* targets,
                                      size_t n_targets, gcu_graph** out);
GCU_API uint32_t gcu_graph_num_nodes(const gcu_graph* g);
GCU_API uint32_t gcu_graph_num_edges(const gcu_graph* g);
GCU_API void gcu_graph_destroy(gcu_graph* g);

/* Copies the device CSR back: offsets gets num_nodes + 1 entries, targets
 * num_edges (GpuGraph's public offsets/targets fields, gpu_graph.rs:17-19,
 * read back with the reference's dtoh copies). */
GCU_API gcu_status gcu_graph_copy_csr(const gcu_graph* g, uint32_t* offsets, uint32_t* targets);

/* ---- device CSR construction (the step before the path) ---- */

/* from_edge_pairs(pairs, num_nodes, symmetric) followed by
 * GpuGraph::from_csr_arrays (csr_export.rs:202-239, gpu_graph.rs:46-60), with
 * the sort and deduplication done on the device: `pairs` holds n_pairs
 * interleaved (src, dst) u32 values in host memory. Same CSR and the same
 * errors (GCU_ERR_EXPORT for a node >= num_nodes; GCU_ERR_INVALID_CSR for a
 * directed target >= num_nodes, which the host builder lets through and
 * validate_csr rejects). At most 2^32 - 2 entries before deduplication. */
GCU_API gcu_status gcu_graph_from_edge_pairs(gcu_device* dev, const uint32_t* pairs, size_t n_pairs,
                                             uint32_t num_nodes, int symmetric, gcu_graph** out);
/* from_edge_pairs_oriented (csr_export.rs:299-350) on the device. */
GCU_API gcu_status gcu_graph_from_edge_pairs_oriented(gcu_device* dev, const uint32_t* pairs,
                                                      size_t n_pairs, uint32_t num_nodes,
                                                      gcu_graph** out);

/* Synthetic symmetric graphs generated on the device (loop-free, deduplicated,
 * sorted). R-MAT and Erdos-Renyi draw exactly the pairs of gcu_generate_rmat /
 * gcu_generate_erdos_renyi, so the CSR equals theirs. No reference
 * counterpart: they stand in for the Graph500/GraphChallenge inputs. */
GCU_API gcu_status gcu_graph_generate_rmat(gcu_device* dev, uint32_t scale, uint32_t edge_factor,
                                           double a, double b, double c, uint64_t seed,
                                           gcu_graph** out);
GCU_API gcu_status gcu_graph_generate_erdos_renyi(gcu_device* dev, uint32_t num_nodes,
                                                  uint64_t num_pairs, uint64_t seed, gcu_graph** out);
/* width x height grid (vertex y * width + x); every lattice edge dropped with
 * probability `drop`. */
GCU_API gcu_status gcu_graph_generate_grid(gcu_device* dev, uint32_t width, uint32_t height,
                                           double drop, uint64_t seed, gcu_graph** out);
/* Watts-Strogatz: ring lattice of even degree k, each lattice edge (u, u + j)
 * rewired to (u, w), w uniform, with probability p. */
GCU_API gcu_status gcu_graph_generate_watts_strogatz(gcu_device* dev, uint32_t num_nodes, uint32_t k,
                                                     double p, uint64_t seed, gcu_graph** out);
/* Random geometric graph: num_nodes uniform points in the unit square, an edge
 * between points at distance <= r, (num_nodes - 1) * pi * r^2 = avg_degree. */
GCU_API gcu_status gcu_graph_generate_geometric(gcu_device* dev, uint32_t num_nodes, double avg_degree,
                                                uint64_t seed, gcu_graph** out);

/* ---- algorithms: crates/grafeo-cuda-algos/src ---- */

/* triangle_counting::triangle_count (triangle_counting.rs:40-152): total
 * triangles of the undirected simple graph in a symmetric CSR. */
GCU_API gcu_status gcu_triangle_count(gcu_graph* g, uint64_t* total, double* seconds);
/* triangle_counting::triangle_count_oriented (triangle_counting.rs:162-210):
 * sum over CSR entries u->v of |N(u) ∩ N(v)|, for a degree-oriented CSR. */
GCU_API gcu_status gcu_triangle_count_oriented(gcu_graph* g, uint64_t* total,
                                               double* seconds);

/* Allocation-free oriented triangle count. No counterpart in the reference.
 * For callers that cannot allocate device memory when they need the count
 * (a process whose memory pool owns the whole device, a framework allocator
 * that forbids side allocations, a path where an allocation may block or fail
 * late): the same count as gcu_triangle_count_oriented over a CSR the caller
 * already holds on the device (d_offsets: num_nodes + 1 u32, d_targets:
 * num_edges u32, valid per validate_csr; not checked here), run on `stream`
 * (NULL: the default stream) of the calling thread's current device, result
 * in *total (host). Its only working memory is a fixed 4 MiB array inside the
 * library, present on every device that loads it until exit; it calls no
 * cudaMalloc/cudaFree. At most 1,048,576 nodes (else GCU_ERR_KERNEL). All
 * calls on a device share that array: calls that overlap on the GPU race.
 * The first call on a device looks the array up (cudaGetSymbolAddress); make
 * it before any stream capture. That address is kept for the life of the
 * process, so the device's primary context must not be reset
 * (cudaDeviceReset) between calls. Each call waits for `stream` to finish
 * before it returns. */
GCU_API gcu_status gcu_triangle_count_oriented_noalloc(const uint32_t* d_offsets, const uint32_t* d_targets,
                                                       uint32_t num_nodes, uint32_t num_edges, void* stream,
                                                       uint64_t* total);

/* bfs::bfs(graph, source) (bfs.rs:42-131). distances (num_nodes i32, -1 =
 * unreachable) may be NULL, in which case the distances stay on the device.
 * A source >= num_nodes is GCU_ERR_KERNEL. */
GCU_API gcu_status gcu_bfs(gcu_graph* g, uint32_t source, int32_t* distances,
                           uint32_t* reachable, int32_t* max_depth, double* seconds);

/* pagerank::pagerank(graph, damping, max_iterations, tolerance)
 * (pagerank.rs:46-199). ranks (num_nodes f32) may be NULL, in which case the
 * ranks stay on the device. Convergence: L1 change between iterations below
 * tolerance (pagerank.rs:150-182). */
GCU_API gcu_status gcu_pagerank(gcu_graph* g, float damping, uint32_t max_iterations,
                                float tolerance, float* ranks, uint32_t* iterations,
                                int* converged, double* seconds);

/* Directed PageRank. The reference can only pull over the CSR lists, which is
 * right for symmetric graphs (pagerank.rs:10 notes that directed graphs need a
 * transpose). Here the lists are the out-edges: the library builds the
 * transpose on the device (stable radix sort, cached on the graph), pulls over
 * the in-lists, takes out-degrees from the lists, and treats vertices without
 * out-edges as dangling. Same arguments and results as gcu_pagerank. */
GCU_API gcu_status gcu_pagerank_directed(gcu_graph* g, float damping, uint32_t max_iterations, float tolerance,
                                         float* ranks, uint32_t* iterations, int* converged, double* seconds);

/* Personalised PageRank: the teleport share and the dangling mass go to the
 * n_seeds seed vertices (each seed 1/n_seeds, repeats add up) instead of all
 * vertices uniformly; ranks still start at 1/N. directed = 0 pulls over the
 * lists (symmetric graph), 1 over the transpose as in gcu_pagerank_directed.
 * A seed >= num_nodes, or no seeds, is GCU_ERR_KERNEL. */
GCU_API gcu_status gcu_personalized_pagerank(gcu_graph* g, const uint32_t* seeds, size_t n_seeds, int directed,
                                             float damping, uint32_t max_iterations, float tolerance, float* ranks,
                                             uint32_t* iterations, int* converged, double* seconds);

/* Diagnostic, no reference counterpart: the floor of a pull SpMV on the
 * PageRank plan. Times `passes` launches (after one warm-up) of a kernel that
 * streams the plan's relabelled in-CSR targets and gathers the contribution
 * of each, with nothing else (no row offsets or row structure, no rank
 * update), on the grid and CTA shape of the PageRank row kernel.
 * *ms_per_pass = device time per launch. directed as in
 * gcu_personalized_pagerank; builds the plan if needed. */
GCU_API gcu_status gcu_pagerank_gather_probe(gcu_graph* g, int directed, uint32_t passes, double* ms_per_pass);

typedef struct gcu_edge_list gcu_edge_list; /* Vec<(u32, u32)>, host memory */

/* k_truss::k_truss(graph, k) (k_truss.rs:42-161). Edges (u, v) with u < v in
 * CSR order. k < 3 is GCU_ERR_KERNEL. */
GCU_API gcu_status gcu_k_truss(gcu_graph* g, uint32_t k, gcu_edge_list** edges,
                               uint32_t* iterations, double* seconds);
/* Truss decomposition. No single reference call: the reference's tests sweep
 * k_truss for k = 3..8 (tests/correctness.rs:305-326). For every CSR entry
 * u -> v, trussness[j] = the largest k whose k-truss contains the edge {u, v}
 * (2 for an edge in no triangle, 0 for a self-loop entry), so that
 * gcu_k_truss(g, k) returns exactly the entries with u < v and trussness >= k.
 * trussness (num_edges u32) may be NULL. *max_trussness = the largest k with a
 * non-empty k-truss (0 without edges); *rounds = peeling rounds run.
 * Symmetric CSR only (GCU_ERR_KERNEL otherwise). */
GCU_API gcu_status gcu_truss_decomposition(gcu_graph* g, uint32_t* trussness, uint32_t* max_trussness,
                                           uint32_t* rounds, double* seconds);

GCU_API size_t gcu_edge_list_len(const gcu_edge_list* list);
/* 2 * len values: u0, v0, u1, v1, ... */
GCU_API const uint32_t* gcu_edge_list_data(const gcu_edge_list* list);
GCU_API void gcu_edge_list_free(gcu_edge_list* list);

/* ---- learned schedule (no reference counterpart: the reference has one
 * fixed schedule). A 12-32-32-3 network (BF16 weights as uint16_t bit
 * patterns, FP32 accumulation, ReLU hidden layers) maps the 12 features of a
 * decision to the predicted log2(microseconds) of three variants: for a BFS
 * level {push with a warp per frontier vertex, load-balanced push, pull}, for
 * a DAG out-degree bucket of the triangle count {warp hash table, CTA hash
 * table, CTA binary search}. Parameter layout: W1[32][12], b1[32], W2[32][32],
 * b2[32], W3[3][32], b3[3]. The schedule never changes a result. ---- */

/* ---- batched form (no reference counterpart: the reference runs one graph
 * per call). Many graphs packed into one CSR: graph i owns the vertices
 * [vertex_base[i], vertex_base[i + 1]) of a union CSR whose targets are union
 * ids, and no edge leaves its graph. Triangle counts, BFS from S sources per
 * graph and personalised PageRank from K seeds per graph run as persistent
 * kernels over all graphs at once; gcu_batch_capture records the three into
 * one CUDA graph that gcu_batch_replay launches. Results equal the per-graph
 * calls (gcu_triangle_count, gcu_bfs, gcu_personalized_pagerank with the same
 * seeds), which gcu_batch_member makes possible for comparison. ---- */

typedef struct gcu_batch gcu_batch;

/* The synthetic corpus: graph i is R-MAT (scale U{8..16}, edge factor
 * U{8..32}, a, b, c = 0.57, 0.19, 0.19) or Watts-Strogatz (n U{256..65536},
 * k = 10, p = 0.1) with equal odds, drawn from (seed, i) and generated on the
 * device. */
GCU_API gcu_status gcu_batch_generate(gcu_device* dev, uint32_t num_graphs, uint64_t seed, gcu_batch** out);
/* A union CSR from the host, validated like gcu_graph_from_csr plus the
 * no-edge-leaves-its-graph rule (GCU_ERR_KERNEL). */
GCU_API gcu_status gcu_batch_from_csr(gcu_device* dev, const uint32_t* vertex_base, size_t num_graphs,
                                      const uint32_t* offsets, size_t n_offsets, const uint32_t* targets,
                                      size_t n_targets, gcu_batch** out);
GCU_API void gcu_batch_destroy(gcu_batch* b);
GCU_API uint32_t gcu_batch_num_graphs(const gcu_batch* b);
GCU_API uint32_t gcu_batch_num_nodes(const gcu_batch* b);
GCU_API uint32_t gcu_batch_num_edges(const gcu_batch* b);
/* vertex_base: num_graphs + 1 values. */
GCU_API gcu_status gcu_batch_vertex_base(const gcu_batch* b, uint32_t* vertex_base);
/* The union CSR copied back (num_nodes + 1 offsets, num_edges targets). */
GCU_API gcu_status gcu_batch_copy_csr(const gcu_batch* b, uint32_t* offsets, uint32_t* targets);
/* Member `index` as a separate device graph with local ids. */
GCU_API gcu_status gcu_batch_member(gcu_batch* b, uint32_t index, gcu_graph** out);

/* Triangles of every graph (totals: num_graphs values). */
GCU_API gcu_status gcu_batch_triangle_count(gcu_batch* b, uint64_t* totals, double* seconds);
/* Sets the BFS sources: sources[g * S + k] is source k of graph g (local id),
 * 1 <= S <= 32. keep_distances = 0 skips the per-vertex distances. Drops a
 * captured graph (it reads the buffers this replaces): capture again before
 * the next gcu_batch_replay. */
GCU_API gcu_status gcu_batch_set_bfs_sources(gcu_batch* b, const uint32_t* sources, uint32_t S,
                                             int keep_distances);
/* Runs the BFS; distances (S * num_nodes, source-major: distances[k *
 * num_nodes + v] for union vertex v; may be NULL), reachable and max_depth
 * (num_graphs * S each, graph-major; may be NULL) as gcu_bfs gives them. */
GCU_API gcu_status gcu_batch_bfs(gcu_batch* b, int32_t* distances, uint32_t* reachable, int32_t* max_depth,
                                 double* seconds);
/* Sets the personalised PageRank seeds: seeds[g * K + k] (local ids). Drops a
 * captured graph, as gcu_batch_set_bfs_sources does. */
GCU_API gcu_status gcu_batch_set_pagerank_seeds(gcu_batch* b, const uint32_t* seeds, uint32_t K, float damping,
                                                uint32_t max_iterations, float tolerance);
/* Runs it; ranks (num_nodes, may be NULL), iterations and converged
 * (num_graphs each, may be NULL). */
GCU_API gcu_status gcu_batch_personalized_pagerank(gcu_batch* b, float* ranks, uint32_t* iterations,
                                                   uint8_t* converged, double* seconds);
/* Plans, autotunes and captures triangles + BFS + PageRank into one CUDA
 * graph; gcu_batch_replay enqueues it on the device stream (asynchronous);
 * gcu_batch_results synchronizes and copies any of the results (NULL skips). */
GCU_API gcu_status gcu_batch_capture(gcu_batch* b);
GCU_API gcu_status gcu_batch_replay(gcu_batch* b);
GCU_API gcu_status gcu_batch_results(gcu_batch* b, uint64_t* triangles, int32_t* distances, uint32_t* reachable,
                                     int32_t* max_depth, float* ranks, uint32_t* iterations, uint8_t* converged);
/* JSON of the autotuned choices (variant per bucket, CTA sizes with their
 * timings); returns the length, writes up to buflen bytes. */
GCU_API size_t gcu_batch_tuning(const gcu_batch* b, char* buf, size_t buflen);

#define GCU_SCHEDULE_FEATURES 12
#define GCU_SCHEDULE_OUTPUTS 3
#define GCU_SCHEDULE_PARAMS 1571

/* Installs the network on the device for gcu_bfs and gcu_triangle_count
 * (copied); NULL returns to the fixed rules (the alpha/beta BFS direction
 * rule and the degree-range intersection buckets), which stay the fallback
 * wherever the network's prediction is not finite. */
GCU_API gcu_status gcu_device_set_schedule(gcu_device* dev, const uint16_t* weights);

/* Batched forward pass: out[n][3] for features[n][12]. */
GCU_API gcu_status gcu_schedule_forward(gcu_device* dev, const uint16_t* weights, const float* features,
                                        size_t n, float* out);
/* Masked mean squared error between the predictions and targets[n][3] over
 * the entries with mask[n][3] != 0, and its gradient w.r.t. the parameters
 * (grad: GCU_SCHEDULE_PARAMS floats), computed on the device. */
GCU_API gcu_status gcu_schedule_gradient(gcu_device* dev, const uint16_t* weights, const float* features,
                                         const float* targets, const uint8_t* mask, size_t n, double* loss,
                                         float* grad);
/* Trains on the device: `steps` Adam steps (learning rate lr) on minibatches
 * of `batch` samples drawn with replacement from the seeded stream. master
 * (FP32, GCU_SCHEDULE_PARAMS) holds the initial weights and receives the
 * trained ones; weights receives their BF16 rounding; *final_loss = loss over
 * all n samples. */
GCU_API gcu_status gcu_schedule_train(gcu_device* dev, float* master, uint16_t* weights, const float* features,
                                      const float* targets, const uint8_t* mask, size_t n, uint32_t steps,
                                      uint32_t batch, float lr, uint64_t seed, double* final_loss);

/* BFS trace from `source`: for every level, the decision's features
 * (features[level][12]), the device time of every valid variant run from the
 * same frontier (times_us[level][3], NaN when not valid), the valid-variant
 * mask, the alpha/beta rule's pick and the variant the traced run continued
 * with (the rule's pick, or for 3 levels in 10 chosen by explore_seed a
 * uniformly drawn valid variant). Up to `capacity` levels are written;
 * *levels = the number of levels traced. The variants must label the same
 * vertices (GCU_ERR_KERNEL otherwise). */
GCU_API gcu_status gcu_bfs_trace(gcu_graph* g, uint32_t source, uint64_t explore_seed, float* features,
                                 float* times_us, uint8_t* valid, uint8_t* fixed_rule, uint8_t* taken,
                                 size_t capacity, size_t* levels);

/* Triangle-count trace: for every non-empty out-degree bucket of the DAG
 * (highest first), the features, the device time of every valid
 * intersection variant (NaN when not valid), the valid mask and the fixed
 * rule's pick; *total = the triangle count, which every variant of every
 * bucket must reproduce (GCU_ERR_KERNEL otherwise). At most 33 buckets. */
GCU_API gcu_status gcu_triangle_trace(gcu_graph* g, float* features, float* times_us, uint8_t* valid,
                                      uint8_t* fixed_rule, size_t capacity, size_t* buckets, uint64_t* total);

#ifdef __cplusplus
}
#endif

#endif /* GRAFEO_CUDA_H */
