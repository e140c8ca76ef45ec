/*
 * Oracle — TEST INFRASTRUCTURE ONLY. See oracle.h for what each function
 * restates and where its semantics come from in the reference.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

int orc_num_threads(void) { return omp_get_max_threads(); }

/* First index in a[lo, hi) with a[i] >= x. */
static size_t lower_bound(const uint32_t* a, size_t lo, size_t hi, uint32_t x) {
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* |a ∩ b| for sorted duplicate-free lists: walk the shorter, search the longer. */
static uint64_t intersect(const uint32_t* a, size_t na, const uint32_t* b, size_t nb) {
    if (na > nb) {
        const uint32_t* t = a;
        a = b;
        b = t;
        size_t tn = na;
        na = nb;
        nb = tn;
    }
    uint64_t c = 0;
    size_t lo = 0;
    for (size_t i = 0; i < na; ++i) {
        lo = lower_bound(b, lo, nb, a[i]);
        if (lo == nb) break;
        if (b[lo] == a[i]) ++c;
    }
    return c;
}

uint64_t orc_triangle_count(const uint32_t* offsets, const uint32_t* targets, uint32_t n) {
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        const uint32_t* nu = targets + offsets[u];
        size_t du = offsets[u + 1] - offsets[u];
        size_t first = lower_bound(nu, 0, du, (uint32_t)u + 1); /* v > u */
        for (size_t i = first; i < du; ++i) {
            uint32_t v = nu[i];
            const uint32_t* nv = targets + offsets[v];
            size_t dv = offsets[v + 1] - offsets[v];
            size_t fv = lower_bound(nv, 0, dv, v + 1); /* w > v in N(v) */
            /* w > v in N(u): the entries after v itself */
            total += intersect(nu + i + 1, du - i - 1, nv + fv, dv - fv);
        }
    }
    return total;
}

uint64_t orc_triangle_count_oriented(const uint32_t* offsets, const uint32_t* targets, uint32_t n) {
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        const uint32_t* nu = targets + offsets[u];
        size_t du = offsets[u + 1] - offsets[u];
        for (size_t i = 0; i < du; ++i) {
            uint32_t v = nu[i];
            total += intersect(nu, du, targets + offsets[v], offsets[v + 1] - offsets[v]);
        }
    }
    return total;
}

void orc_bfs(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t source, int32_t* dist,
             uint32_t* reachable, int32_t* max_depth) {
    for (uint32_t v = 0; v < n; ++v) dist[v] = -1;
    uint32_t* frontier = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* next = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    dist[source] = 0;
    frontier[0] = source;
    size_t fsize = 1;
    uint32_t reached = 1;
    int32_t level = 0;
    while (fsize > 0) {
        size_t nsize = 0;
#pragma omp parallel
        {
            /* Each thread collects its discoveries locally, then appends them. */
            size_t cap = 1024, cnt = 0;
            uint32_t* local = (uint32_t*)malloc(sizeof(uint32_t) * cap);
#pragma omp for schedule(dynamic, 64)
            for (int64_t i = 0; i < (int64_t)fsize; ++i) {
                uint32_t u = frontier[i];
                for (uint32_t j = offsets[u]; j < offsets[u + 1]; ++j) {
                    uint32_t v = targets[j];
                    int32_t expected = -1;
                    if (__atomic_load_n(&dist[v], __ATOMIC_RELAXED) == -1 &&
                        __atomic_compare_exchange_n(&dist[v], &expected, level + 1, 0, __ATOMIC_RELAXED,
                                                    __ATOMIC_RELAXED)) {
                        if (cnt == cap) {
                            cap *= 2;
                            local = (uint32_t*)realloc(local, sizeof(uint32_t) * cap);
                        }
                        local[cnt++] = v;
                    }
                }
            }
            size_t at = __atomic_fetch_add(&nsize, cnt, __ATOMIC_RELAXED);
            memcpy(next + at, local, sizeof(uint32_t) * cnt);
            free(local);
        }
        if (nsize == 0) break;
        level += 1;
        reached += (uint32_t)nsize;
        uint32_t* t = frontier;
        frontier = next;
        next = t;
        fsize = nsize;
    }
    free(frontier);
    free(next);
    *reachable = reached;
    *max_depth = level;
}

void orc_pagerank(const uint32_t* offsets, const uint32_t* targets, uint32_t n, const uint32_t* out_degree,
                  double damping, uint32_t max_iterations, double tolerance, int rule, double* ranks,
                  uint32_t* iterations, int* converged) {
    orc_pagerank_tele(offsets, targets, n, out_degree, NULL, damping, max_iterations, tolerance, rule, ranks,
                      iterations, converged);
}

void orc_pagerank_tele(const uint32_t* offsets, const uint32_t* targets, uint32_t n, const uint32_t* out_degree,
                       const double* tele, double damping, uint32_t max_iterations, double tolerance, int rule,
                       double* ranks, uint32_t* iterations, int* converged) {
    *iterations = 0;
    *converged = 0;
    if (n == 0) {
        *converged = 1;
        return;
    }
    double* r = ranks;
    double* next = (double*)malloc(sizeof(double) * n);
    double* contrib = (double*)malloc(sizeof(double) * n);
    uint32_t* deg = (uint32_t*)malloc(sizeof(uint32_t) * n);
    for (uint32_t v = 0; v < n; ++v) {
        deg[v] = out_degree ? out_degree[v] : offsets[v + 1] - offsets[v];
        r[v] = 1.0 / (double)n;
    }
    const double base = (1.0 - damping) / (double)n;
    for (uint32_t it = 0; it < max_iterations; ++it) {
        double dangling = 0.0;
#pragma omp parallel for reduction(+ : dangling)
        for (int64_t v = 0; v < (int64_t)n; ++v) {
            contrib[v] = deg[v] > 0 ? r[v] / (double)deg[v] : 0.0;
            if (deg[v] == 0) dangling += r[v];
        }
        const double spread = dangling / (double)n;
        double l1 = 0.0, linf = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : l1) reduction(max : linf)
        for (int64_t v = 0; v < (int64_t)n; ++v) {
            double s = 0.0;
            for (uint32_t j = offsets[v]; j < offsets[v + 1]; ++j) s += contrib[targets[j]];
            double x = tele ? (1.0 - damping) * tele[v] + damping * (s + dangling * tele[v])
                            : base + damping * (s + spread);
            double d = fabs(x - r[v]);
            l1 += d;
            if (d > linf) linf = d;
            next[v] = x;
        }
        memcpy(r, next, sizeof(double) * n);
        *iterations = it + 1;
        if ((rule == 0 ? l1 : linf) < tolerance) {
            *converged = 1;
            break;
        }
    }
    free(next);
    free(contrib);
    free(deg);
}

size_t orc_k_truss(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t k, uint32_t* out,
                   uint32_t* iterations) {
    const size_t E = offsets[n];
    *iterations = 0;
    if (E == 0) return 0; /* k_truss.rs:53-60: no edges, no rounds */
    uint8_t* removed = (uint8_t*)calloc(E ? E : 1, 1);
    uint32_t* support = (uint32_t*)malloc(sizeof(uint32_t) * (E ? E : 1));
    const uint32_t threshold = k - 2;
    uint32_t rounds = 0;
    for (;;) {
        memset(support, 0, sizeof(uint32_t) * E);
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t u = 0; u < (int64_t)n; ++u) {
            const uint32_t us = offsets[u], ue = offsets[u + 1];
            for (uint32_t idx = us; idx < ue; ++idx) {
                if (removed[idx]) continue;
                const uint32_t v = targets[idx];
                if (v <= (uint32_t)u) continue;
                const uint32_t vs = offsets[v], ve = offsets[v + 1];
                uint32_t j = us, m = vs, count = 0;
                while (j < ue && m < ve) {
                    if (removed[j]) {
                        ++j;
                        continue;
                    }
                    if (removed[m]) {
                        ++m;
                        continue;
                    }
                    uint32_t a = targets[j], b = targets[m];
                    if (a == b) {
                        ++count;
                        ++j;
                        ++m;
                    } else if (a < b) {
                        ++j;
                    } else {
                        ++m;
                    }
                }
                support[idx] = count;
                for (uint32_t r = vs; r < ve; ++r) {
                    if (targets[r] == (uint32_t)u && !removed[r]) {
                        support[r] = count;
                        break;
                    }
                }
            }
        }
        size_t removed_now = 0;
        for (size_t i = 0; i < E; ++i) {
            if (!removed[i] && support[i] < threshold) {
                removed[i] = 1;
                ++removed_now;
            }
        }
        ++rounds;
        if (removed_now == 0) break;
    }
    size_t count = 0;
    for (uint32_t u = 0; u < n; ++u) {
        for (uint32_t idx = offsets[u]; idx < offsets[u + 1]; ++idx) {
            const uint32_t v = targets[idx];
            if (v > u && !removed[idx]) {
                if (out) {
                    out[2 * count] = u;
                    out[2 * count + 1] = v;
                }
                ++count;
            }
        }
    }
    free(removed);
    free(support);
    *iterations = rounds;
    return count;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static size_t csr_from_keys(uint64_t* keys, size_t m, uint32_t n, uint32_t* offsets, uint32_t* targets) {
    memset(offsets, 0, sizeof(uint32_t) * ((size_t)n + 1));
    for (size_t i = 0; i < m; ++i) {
        offsets[(keys[i] >> 32) + 1] += 1;
        targets[i] = (uint32_t)keys[i];
    }
    for (size_t i = 1; i <= n; ++i) offsets[i] += offsets[i - 1];
    return m;
}

size_t orc_from_edge_pairs(const uint32_t* pairs, size_t n_pairs, uint32_t n, int symmetric, uint32_t* offsets,
                           uint32_t* targets) {
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (2 * n_pairs + 1));
    size_t m = 0;
    for (size_t i = 0; i < n_pairs; ++i) {
        uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        if (s >= n || (symmetric && d >= n)) {
            free(keys);
            return (size_t)-1;
        }
        keys[m++] = ((uint64_t)s << 32) | d;
        if (symmetric && s != d) keys[m++] = ((uint64_t)d << 32) | s;
    }
    qsort(keys, m, sizeof(uint64_t), cmp_u64);
    size_t w = 0;
    for (size_t i = 0; i < m; ++i)
        if (w == 0 || keys[i] != keys[w - 1]) keys[w++] = keys[i];
    size_t r = csr_from_keys(keys, w, n, offsets, targets);
    free(keys);
    return r;
}

size_t orc_from_edge_pairs_oriented(const uint32_t* pairs, size_t n_pairs, uint32_t n, uint32_t* offsets,
                                    uint32_t* targets) {
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n_pairs + 1));
    size_t m = 0;
    for (size_t i = 0; i < n_pairs; ++i) {
        uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        if (s >= n || d >= n) {
            free(keys);
            return (size_t)-1;
        }
        if (s == d) continue;
        uint32_t lo = s < d ? s : d, hi = s < d ? d : s;
        keys[m++] = ((uint64_t)lo << 32) | hi;
    }
    qsort(keys, m, sizeof(uint64_t), cmp_u64);
    size_t w = 0;
    for (size_t i = 0; i < m; ++i)
        if (w == 0 || keys[i] != keys[w - 1]) keys[w++] = keys[i];
    uint32_t* degree = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
    for (size_t i = 0; i < w; ++i) {
        degree[keys[i] >> 32] += 1;
        degree[(uint32_t)keys[i]] += 1;
    }
    for (size_t i = 0; i < w; ++i) {
        uint32_t u = (uint32_t)(keys[i] >> 32), v = (uint32_t)keys[i];
        if (!(degree[u] < degree[v] || (degree[u] == degree[v] && u < v))) keys[i] = ((uint64_t)v << 32) | u;
    }
    qsort(keys, w, sizeof(uint64_t), cmp_u64);
    size_t r = csr_from_keys(keys, w, n, offsets, targets);
    free(degree);
    free(keys);
    return r;
}

size_t orc_transpose(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* t_offsets,
                     uint32_t* t_targets) {
    const size_t E = offsets[n];
    memset(t_offsets, 0, sizeof(uint32_t) * ((size_t)n + 1));
    for (size_t j = 0; j < E; ++j) t_offsets[targets[j] + 1] += 1;
    for (size_t v = 1; v <= n; ++v) t_offsets[v] += t_offsets[v - 1];
    uint32_t* cursor = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    memcpy(cursor, t_offsets, sizeof(uint32_t) * ((size_t)n + 1));
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t j = offsets[u]; j < offsets[u + 1]; ++j) t_targets[cursor[targets[j]]++] = u;
    free(cursor);
    return E;
}
