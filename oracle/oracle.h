/*
 * Oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement, in plain C with OpenMP, of what the reference's four
 * graph paths compute. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; nothing in the product links or calls it.
 *
 * What it restates (paths inside the grafeo-cuda project):
 *  - Grafeo 0.6.3's CPU algorithms (crate grafeo-adapters =0.6.3,
 *    `plugins::algorithms::{total_triangles, bfs_layers, pagerank, k_truss}`,
 *    pinned at Cargo.toml:37 / Cargo.lock:460-470) are the reference's test
 *    oracle (crates/grafeo-cuda-algos/tests/correctness.rs:233-326). That crate
 *    is not vendored and cannot be built here (no Rust toolchain), so its
 *    published semantics are restated from the reference's call sites and
 *    tests, and the reference kernels' own math decides the details:
 *      triangle counts  kernels/triangle_counting.cu:246-315, :331-376
 *      BFS levels       src/bfs.rs:42-131, kernels/bfs.cu:54-83
 *      PageRank         src/pagerank.rs:46-199, kernels/pagerank.cu:19-134
 *      k-truss rounds   src/k_truss.rs:42-161, kernels/k_truss.cu:46-124
 *  - CSR builders from crates/grafeo-cuda-core/src/csr_export.rs:202-239 and
 *    :299-350.
 *
 * Pinning: the literal known answers of the reference's tests
 * (tests/roundtrip.rs, tests/correctness.rs:330-386) and networkx 3.6.1 on
 * the reference's catalog graphs, committed as JSON files under tests/golden/ by
 * tests/golden/make_golden.py, are checked against this oracle by
 * tests/test_oracle.py.
 */
#ifndef GRAFEO_ORACLE_H
#define GRAFEO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* sum_u sum_{v in N(u), v > u} |{w in N(u) ∩ N(v) : w > v}|
 * (triangle_counting.cu:246-315). On a symmetric CSR this is the number of
 * triangles of the undirected simple graph (Grafeo's total_triangles). */
uint64_t orc_triangle_count(const uint32_t* offsets, const uint32_t* targets, uint32_t n);

/* sum over entries u -> v of |N(u) ∩ N(v)| (triangle_counting.cu:331-376). */
uint64_t orc_triangle_count_oriented(const uint32_t* offsets, const uint32_t* targets, uint32_t n);

/* Level-synchronous BFS along the CSR lists (bfs.rs:42-131): dist[v] = level or
 * -1; *reachable = #reached; *max_depth = last non-empty level. */
void orc_bfs(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t source, int32_t* dist,
             uint32_t* reachable, int32_t* max_depth);

/* FP64 power iteration, pull over the CSR lists, with uniform dangling
 * redistribution and teleport (1-d)/N (pagerank.cu:67-94), starting from 1/N.
 * rule 0: stop when the L1 change < tol (the reference GPU rule,
 * pagerank.rs:150-182); rule 1: stop when the largest per-node change < tol
 * (Grafeo's rule, pagerank.rs:40-42). out_degree may be NULL (then the row
 * length is the out-degree: symmetric CSR); otherwise the CSR holds in-lists
 * and out_degree[u] the out-degree of u (directed graphs). */
void orc_pagerank(const uint32_t* offsets, const uint32_t* targets, uint32_t n, const uint32_t* out_degree,
                  double damping, uint32_t max_iterations, double tolerance, int rule, double* ranks,
                  uint32_t* iterations, int* converged);

/* orc_pagerank with a personalisation vector tele (NULL: uniform 1/N) that
 * takes the teleport share and the dangling mass: r'[v] = (1-d) tele[v] +
 * d (sum + dangling tele[v]). Ranks start at 1/N either way. */
void orc_pagerank_tele(const uint32_t* offsets, const uint32_t* targets, uint32_t n, const uint32_t* out_degree,
                       const double* tele, double damping, uint32_t max_iterations, double tolerance, int rule,
                       double* ranks, uint32_t* iterations, int* converged);

/* In-lists of a CSR (each ordered by source); returns the entry count. */
size_t orc_transpose(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* t_offsets,
                     uint32_t* t_targets);

/* Synchronous peeling exactly as k_truss.rs/k_truss.cu: per round, support of
 * each live entry u -> v (v > u) is the merge count of the live lists, copied to
 * the live reverse entry; live entries below k-2 are removed; repeat until a
 * round removes nothing. Writes the surviving (u, v), u < v, in CSR order into
 * out (capacity 2 * n_targets values) and returns their count. */
size_t orc_k_truss(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t k, uint32_t* out,
                   uint32_t* iterations);

/* csr_export.rs:202-239. offsets has n+1 slots, targets 2*n_pairs slots;
 * returns the number of targets written, or SIZE_MAX on a bad node id. */
size_t orc_from_edge_pairs(const uint32_t* pairs, size_t n_pairs, uint32_t n, int symmetric, uint32_t* offsets,
                           uint32_t* targets);
/* csr_export.rs:299-350. */
size_t orc_from_edge_pairs_oriented(const uint32_t* pairs, size_t n_pairs, uint32_t n, uint32_t* offsets,
                                    uint32_t* targets);

/* Number of OpenMP threads the oracle uses. */
int orc_num_threads(void);

/* ---- at scale (oracle_scale.c): parallel restatements for the large
 * configurations; see that file's header for what each restates. */

/* Symmetric, loop-free, deduplicated CSR of an R-MAT graph: edge_factor << scale
 * pairs, pair i choosing one quadrant per level (a, b, c, rest) from SplitMix64
 * draws i * scale + level of the stream seeded by `seed`. `targets` holds at
 * least 2 * (edge_factor << scale) entries; returns the entry count. */
size_t orc_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                         uint32_t* offsets, uint32_t* targets);

/* The same for Erdos-Renyi G(n, num_pairs): pair i = draws 2i and 2i + 1
 * mapped onto [0, n). `targets` holds at least 2 * num_pairs entries. */
size_t orc_generate_erdos_renyi(uint32_t n, uint64_t num_pairs, uint64_t seed, uint32_t* offsets,
                                uint32_t* targets);

/* orc_transpose by a parallel radix sort (same output). */
size_t orc_transpose_sorted(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* t_offsets,
                            uint32_t* t_targets);

/* support[j] = triangles through the edge of entry j; -1 unless the CSR is
 * simple (no self-loops or repeated entries) and symmetric. */
int orc_edge_support(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* support);

/* orc_k_truss on a simple symmetric CSR by incremental peeling (same edges,
 * same round count). support0 (optional) is orc_edge_support's output, to
 * share it across several k. Returns the edge count, or SIZE_MAX when the
 * CSR is not simple and symmetric. */
size_t orc_k_truss_peel(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t k,
                        const uint32_t* support0, uint32_t* out, uint32_t* iterations);

/* Truss decomposition by the same peeling continued level by level: the
 * trussness of every entry's edge (2 for edges in no triangle), the largest
 * k with a non-empty k-truss, and the number of synchronous rounds (a round
 * that removes nothing ends its level and is counted). -1 unless simple and
 * symmetric. */
int orc_truss_decomposition_peel(const uint32_t* offsets, const uint32_t* targets, uint32_t n,
                                 const uint32_t* support0, uint32_t* trussness, uint32_t* max_trussness,
                                 uint32_t* rounds);


#ifdef __cplusplus
}
#endif

#endif
