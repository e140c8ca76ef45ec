/*
 * Oracle at scale — TEST INFRASTRUCTURE ONLY (part of liboracle.so; see
 * oracle.h). Only tests/, __graft_entry__.smoke() and bench.py's CPU legs
 * call it; the product never does.
 *
 * The configurations at scale (R-MAT 22 and 24, Erdos-Renyi 2^22) need the
 * oracle to build their graphs and check their results in seconds to
 * minutes on the host cores, which the small-graph restatements in oracle.c
 * (qsort builders, a full support recomputation per k-truss round) do not.
 * This file restates the same things with parallel building blocks:
 *
 *  - the synthetic generators (R-MAT with the recursive quadrant choice of
 *    Chakrabarti, Zhan and Faloutsos, SDM 2004; Erdos-Renyi G(n, m) pairs),
 *    drawn from counter-based SplitMix64 streams (Steele, Lea and Flood,
 *    OOPSLA 2014) and turned into a symmetric, loop-free, deduplicated CSR
 *    by a parallel LSD radix sort of (source, target) keys;
 *  - the transpose of a CSR (in-lists in ascending source order) by the same
 *    sort;
 *  - the k-truss of a simple symmetric CSR and its full truss decomposition
 *    with the reference's synchronous round rule (k_truss.rs:75-151: every
 *    round removes every alive edge with support < k - 2; the round in which
 *    nothing is removed is counted), computed incrementally: the per-edge
 *    support is counted once, and every round only subtracts the triangles
 *    that its removed edges destroy (each destroyed triangle once, credited
 *    to its removed edge with the smallest id). Only edges whose support
 *    fell to below the threshold in a round can be removed in the next one,
 *    so rounds after the first of a level visit those edges only.
 *
 * Pinning: tests/test_oracle.py checks the generators against the
 * library's host generators and the numpy restatements in tests/graphs.py,
 * the transpose against orc_transpose, and the peel against orc_k_truss and
 * the definition-based truss decomposition (oracle.py) on the golden
 * catalog and random graphs.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---------------------------------------------------------------- radix sort */

/* Number of bits that values 0..n-1 need (0 for n <= 1). */
static int bits_for(uint64_t n) {
    int b = 0;
    while (b < 64 && (1ull << b) < n) ++b;
    return b;
}

/* Stable LSD radix sort of keys[0, m) on their low `bits` bits, 12 bits per
 * pass; every thread owns a contiguous slice and a histogram, so equal keys
 * keep their order. Returns the buffer that holds the sorted keys. */
static uint64_t* radix_sort(uint64_t* keys, uint64_t* tmp, size_t m, int bits) {
    enum { kDigit = 12, kBuckets = 1 << kDigit };
    const int T = omp_get_max_threads();
    size_t* hist = (size_t*)malloc(sizeof(size_t) * (size_t)T * kBuckets);
    for (int shift = 0; shift < bits; shift += kDigit) {
#pragma omp parallel num_threads(T)
        {
            const int nt = omp_get_num_threads(), t = omp_get_thread_num();
            const size_t lo = m * (size_t)t / (size_t)nt, hi = m * (size_t)(t + 1) / (size_t)nt;
            size_t* h = hist + (size_t)t * kBuckets;
            memset(h, 0, sizeof(size_t) * kBuckets);
            for (size_t i = lo; i < hi; ++i) ++h[(keys[i] >> shift) & (kBuckets - 1)];
#pragma omp barrier
#pragma omp single
            {
                size_t sum = 0;
                for (int b = 0; b < kBuckets; ++b)
                    for (int u = 0; u < nt; ++u) {
                        const size_t c = hist[(size_t)u * kBuckets + b];
                        hist[(size_t)u * kBuckets + b] = sum;
                        sum += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                const uint64_t k = keys[i];
                tmp[h[(k >> shift) & (kBuckets - 1)]++] = k;
            }
        }
        uint64_t* s = keys;
        keys = tmp;
        tmp = s;
    }
    free(hist);
    return keys;
}

/* CSR from sorted (source << tb | target) keys, duplicates dropped. */
static size_t csr_from_sorted(const uint64_t* keys, size_t m, int tb, uint32_t n, uint32_t* offsets,
                              uint32_t* targets) {
    const uint64_t mask = tb ? ((1ull << tb) - 1) : 0;
    memset(offsets, 0, sizeof(uint32_t) * ((size_t)n + 1));
    size_t w = 0;
    for (size_t i = 0; i < m; ++i) {
        if (i > 0 && keys[i] == keys[i - 1]) continue;
        offsets[(keys[i] >> tb) + 1] += 1;
        targets[w++] = (uint32_t)(keys[i] & mask);
    }
    for (size_t v = 1; v <= n; ++v) offsets[v] += offsets[v - 1];
    return w;
}

/* ---------------------------------------------------------------- generators */

static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
#define GOLDEN_GAMMA 0x9E3779B97F4A7C15ull
/* n-th output of the SplitMix64 generator whose state starts at `state`. */
static inline uint64_t stream_draw(uint64_t state, uint64_t n) { return mix64(state + (n + 1) * GOLDEN_GAMMA); }

typedef struct {
    int kind; /* 0: R-MAT, 1: Erdos-Renyi */
    uint64_t state;
    uint32_t scale, n;
    double a, ab, abc;
} PairSource;

/* Pair i: R-MAT picks one quadrant per level from draw i * scale + level
 * (top bit first); Erdos-Renyi maps draws 2i and 2i + 1 onto [0, n). */
static inline void draw_pair(const PairSource* ps, uint64_t i, uint32_t* s, uint32_t* d) {
    if (ps->kind == 0) {
        uint32_t x = 0, y = 0;
        for (uint32_t l = 0; l < ps->scale; ++l) {
            const double u = (double)(stream_draw(ps->state, i * ps->scale + l) >> 11) * (1.0 / 9007199254740992.0);
            const uint32_t row = u >= ps->ab;                      /* quadrants c and d: lower half */
            const uint32_t col = (u >= ps->a && u < ps->ab) || u >= ps->abc; /* quadrants b and d */
            x = (x << 1) | row;
            y = (y << 1) | col;
        }
        *s = x;
        *d = y;
    } else {
        *s = (uint32_t)(((unsigned __int128)stream_draw(ps->state, 2 * i) * ps->n) >> 64);
        *d = (uint32_t)(((unsigned __int128)stream_draw(ps->state, 2 * i + 1) * ps->n) >> 64);
    }
}

/* Symmetric, loop-free, deduplicated CSR of m drawn pairs: every thread
 * counts its slice's non-loop pairs, then writes both directions of each as
 * keys at its offset; one radix sort; duplicates dropped while writing. */
static size_t symmetric_csr_of_pairs(const PairSource* ps, uint64_t m, uint32_t* offsets, uint32_t* targets) {
    const int T = omp_get_max_threads();
    size_t* base = (size_t*)calloc((size_t)T + 1, sizeof(size_t));
    int used = T;
#pragma omp parallel num_threads(T)
    {
        const int nt = omp_get_num_threads(), t = omp_get_thread_num();
        if (t == 0) used = nt;
        const uint64_t lo = m * (uint64_t)t / (uint64_t)nt, hi = m * (uint64_t)(t + 1) / (uint64_t)nt;
        size_t c = 0;
        for (uint64_t i = lo; i < hi; ++i) {
            uint32_t s, d;
            draw_pair(ps, i, &s, &d);
            c += s != d;
        }
        base[t + 1] = 2 * c;
    }
    for (int t = 0; t < used; ++t) base[t + 1] += base[t];
    const size_t k = base[used];
    const int tb = bits_for(ps->n);
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (k ? k : 1));
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (k ? k : 1));
#pragma omp parallel num_threads(used)
    {
        const int nt = omp_get_num_threads(), t = omp_get_thread_num();
        const uint64_t lo = m * (uint64_t)t / (uint64_t)nt, hi = m * (uint64_t)(t + 1) / (uint64_t)nt;
        size_t w = base[t];
        for (uint64_t i = lo; i < hi; ++i) {
            uint32_t s, d;
            draw_pair(ps, i, &s, &d);
            if (s == d) continue;
            keys[w++] = ((uint64_t)s << tb) | d;
            keys[w++] = ((uint64_t)d << tb) | s;
        }
    }
    const uint64_t* sorted = radix_sort(keys, tmp, k, 2 * tb);
    const size_t e = csr_from_sorted(sorted, k, tb, ps->n, offsets, targets);
    free(keys);
    free(tmp);
    free(base);
    return e;
}

size_t orc_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                         uint32_t* offsets, uint32_t* targets) {
    if (scale == 0 || scale > 31) return (size_t)-1;
    PairSource ps = {0, mix64(seed + GOLDEN_GAMMA), scale, 1u << scale, a, a + b, a + b + c};
    return symmetric_csr_of_pairs(&ps, (uint64_t)edge_factor << scale, offsets, targets);
}

size_t orc_generate_erdos_renyi(uint32_t n, uint64_t num_pairs, uint64_t seed, uint32_t* offsets,
                                uint32_t* targets) {
    PairSource ps = {1, mix64(seed + GOLDEN_GAMMA), 0, n, 0, 0, 0};
    if (n == 0) {
        offsets[0] = 0;
        return 0;
    }
    return symmetric_csr_of_pairs(&ps, num_pairs, offsets, targets);
}

/* ---------------------------------------------------------------- transpose */

size_t orc_transpose_sorted(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* t_offsets,
                            uint32_t* t_targets) {
    const size_t E = offsets[n];
    const int tb = bits_for(n);
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (E ? E : 1));
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (E ? E : 1));
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < (int64_t)n; ++u)
        for (uint32_t j = offsets[u]; j < offsets[u + 1]; ++j) keys[j] = ((uint64_t)targets[j] << tb) | (uint64_t)u;
    const uint64_t* sorted = radix_sort(keys, tmp, E, 2 * tb);
    /* Keys are distinct (one per entry of a CSR without repeated entries) or
     * repeat with their entries; keep every entry. */
    const uint64_t mask = tb ? ((1ull << tb) - 1) : 0;
    memset(t_offsets, 0, sizeof(uint32_t) * ((size_t)n + 1));
    for (size_t i = 0; i < E; ++i) {
        t_offsets[(sorted[i] >> tb) + 1] += 1;
        t_targets[i] = (uint32_t)(sorted[i] & mask);
    }
    for (size_t v = 1; v <= n; ++v) t_offsets[v] += t_offsets[v - 1];
    free(keys);
    free(tmp);
    return E;
}

/* ---------------------------------------------------------------- k-truss peel */

/* A simple symmetric CSR with, per entry, its row and the id of its edge
 * (the index of the entry u -> v with u < v). */
typedef struct {
    uint32_t n;
    size_t E;
    const uint32_t* off;
    const uint32_t* tgt;
    uint32_t* src;
    uint32_t* eid;
} SymCsr;

static size_t find_entry(const uint32_t* tgt, size_t lo, size_t hi, uint32_t x) {
    const size_t end = hi;
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (tgt[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < end && tgt[lo] == x) ? lo : (size_t)-1;
}

/* 0 on success; -1 when the CSR has a self-loop, a repeated entry or an
 * entry without its reverse. */
static int sym_init(SymCsr* g, const uint32_t* offsets, const uint32_t* targets, uint32_t n) {
    g->n = n;
    g->E = offsets[n];
    g->off = offsets;
    g->tgt = targets;
    g->src = (uint32_t*)malloc(sizeof(uint32_t) * (g->E ? g->E : 1));
    g->eid = (uint32_t*)malloc(sizeof(uint32_t) * (g->E ? g->E : 1));
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        for (uint32_t j = offsets[u]; j < offsets[u + 1]; ++j) {
            const uint32_t v = targets[j];
            g->src[j] = (uint32_t)u;
            if (v == (uint32_t)u || v >= n || (j > offsets[u] && targets[j - 1] >= v)) {
                bad = 1;
                continue;
            }
            if (v > (uint32_t)u) {
                g->eid[j] = j;
            } else {
                const size_t r = find_entry(targets, offsets[v], offsets[v + 1], (uint32_t)u);
                if (r == (size_t)-1)
                    bad = 1;
                else
                    g->eid[j] = (uint32_t)r;
            }
        }
    }
    /* every u < v entry needs its reverse too */
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t u = 0; u < (int64_t)n; ++u)
        for (uint32_t j = offsets[u]; j < offsets[u + 1]; ++j)
            if (targets[j] > (uint32_t)u &&
                find_entry(targets, offsets[targets[j]], offsets[targets[j] + 1], (uint32_t)u) == (size_t)-1)
                bad = 1;
    return bad ? -1 : 0;
}

static void sym_free(SymCsr* g) {
    free(g->src);
    free(g->eid);
}

/* support[e] = |N(u) ∩ N(v)| for every edge e = (u < v): each edge is
 * handled by its endpoint of higher (degree, id), which marks its own list
 * in a bitmap once and probes the other endpoint's list against it. */
static void edge_support(const SymCsr* g, uint32_t* support) {
    const uint32_t n = g->n;
    const size_t words = ((size_t)n + 63) / 64;
#pragma omp parallel
    {
        uint64_t* mark = (uint64_t*)calloc(words ? words : 1, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 64)
        for (int64_t h = 0; h < (int64_t)n; ++h) {
            const uint32_t hs = g->off[h], he = g->off[h + 1], dh = he - hs;
            for (uint32_t j = hs; j < he; ++j) mark[g->tgt[j] >> 6] |= 1ull << (g->tgt[j] & 63);
            for (uint32_t j = hs; j < he; ++j) {
                const uint32_t l = g->tgt[j], dl = g->off[l + 1] - g->off[l];
                if (!(dl < dh || (dl == dh && l < (uint32_t)h))) continue;
                uint32_t c = 0;
                for (uint32_t q = g->off[l]; q < g->off[l + 1]; ++q) c += (uint32_t)(mark[g->tgt[q] >> 6] >> (g->tgt[q] & 63)) & 1u;
                support[g->eid[j]] = c;
            }
            for (uint32_t j = hs; j < he; ++j) mark[g->tgt[j] >> 6] = 0;
        }
        free(mark);
    }
}

/* Alive adjacency: per vertex the entries whose edge was alive when the
 * lists were last compacted (in CSR order), each with its edge id. */
typedef struct {
    uint32_t* off;
    uint32_t* tgt;
    uint32_t* eid;
    size_t alive_at_build;
} AliveLists;

static void alive_build(const SymCsr* g, const uint32_t* state, AliveLists* a, size_t alive) {
    const uint32_t n = g->n;
    uint32_t* cnt = a->off; /* n + 1 */
    cnt[0] = 0;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        uint32_t c = 0;
        for (uint32_t j = g->off[u]; j < g->off[u + 1]; ++j) c += state[g->eid[j]] == 0;
        cnt[u + 1] = c;
    }
    for (size_t u = 1; u <= n; ++u) cnt[u] += cnt[u - 1];
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        uint32_t w = a->off[u];
        for (uint32_t j = g->off[u]; j < g->off[u + 1]; ++j)
            if (state[g->eid[j]] == 0) {
                a->tgt[w] = g->tgt[j];
                a->eid[w] = g->eid[j];
                ++w;
            }
    }
    a->alive_at_build = alive;
}

/* Removes the edges of `removed` (already marked state = rnd): every
 * triangle alive at the start of the round that holds a removed edge is
 * destroyed once, by its removed edge with the smallest id, and each of its
 * surviving edges loses one support; an edge whose support falls from
 * `threshold` to below it is appended to `crossed`. Returns its length. */
static size_t peel_round(const SymCsr* g, const AliveLists* a, uint32_t* state, uint32_t* support,
                         const uint32_t* removed, size_t nrem, uint32_t rnd, uint32_t threshold, uint32_t* crossed) {
    size_t ncross = 0;
#pragma omp parallel for schedule(dynamic, 1) if (nrem > 1)
    for (int64_t i = 0; i < (int64_t)nrem; ++i) {
        const uint32_t e = removed[i];
        const uint32_t x = g->src[e], y = g->tgt[e];
        uint32_t ss = a->off[x], se = a->off[x + 1], ls = a->off[y], le = a->off[y + 1];
        if (se - ss > le - ls) {
            uint32_t t0 = ss, t1 = se;
            ss = ls;
            se = le;
            ls = t0;
            le = t1;
        }
        uint32_t pos = ls; /* every target before pos is below the current w */
        for (uint32_t j = ss; j < se && pos < le; ++j) {
            const uint32_t w = a->tgt[j], e1 = a->eid[j];
            const uint32_t s1 = state[e1];
            if (s1 != 0 && s1 != rnd) continue; /* removed in an earlier round */
            /* galloping search forward from pos for the first target >= w */
            uint32_t step = 1, lo = pos, hi = pos;
            while (hi < le && a->tgt[hi] < w) {
                lo = hi + 1;
                hi += step;
                step *= 2;
            }
            if (hi > le) hi = le;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (a->tgt[mid] < w)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            pos = lo;
            if (pos == le || a->tgt[pos] != w) continue;
            const uint32_t e2 = a->eid[pos];
            const uint32_t s2 = state[e2];
            if ((s1 != 0 && s1 != rnd) || (s2 != 0 && s2 != rnd)) continue;
            if ((s1 == rnd && e1 < e) || (s2 == rnd && e2 < e)) continue;
            const uint32_t ex[2] = {e1, e2};
            const uint32_t sx[2] = {s1, s2};
            for (int q = 0; q < 2; ++q) {
                if (sx[q] != 0) continue;
                const uint32_t old = __atomic_fetch_sub(&support[ex[q]], 1u, __ATOMIC_RELAXED);
                if (old == threshold) crossed[__atomic_fetch_add(&ncross, 1, __ATOMIC_RELAXED)] = ex[q];
            }
        }
    }
    return ncross;
}

/* Active list: the u < v entries of the edges that were alive when it was
 * last filtered, ascending. */
typedef struct {
    uint32_t* ids;
    uint32_t* spare;
    size_t n;
} ActiveList;

/* Drops the removed edges from the active list and lists, in ascending
 * order, the alive edges whose support is below t. */
static size_t scan_below(ActiveList* al, const uint32_t* state, const uint32_t* support, uint32_t t, uint32_t* out) {
    const int T = omp_get_max_threads();
    size_t* cnt = (size_t*)calloc(2 * ((size_t)T + 1), sizeof(size_t));
    const size_t na = al->n;
    int used = T;
#pragma omp parallel num_threads(T)
    {
        const int nt = omp_get_num_threads(), th = omp_get_thread_num();
        if (th == 0) used = nt;
        const size_t lo = na * (size_t)th / (size_t)nt, hi = na * (size_t)(th + 1) / (size_t)nt;
        size_t keep = 0, below = 0;
        for (size_t i = lo; i < hi; ++i) {
            const uint32_t e = al->ids[i];
            if (state[e] != 0) continue;
            ++keep;
            below += support[e] < t;
        }
        cnt[2 * (th + 1)] = keep;
        cnt[2 * (th + 1) + 1] = below;
#pragma omp barrier
#pragma omp single
        for (int u = 1; u <= nt; ++u) {
            cnt[2 * u] += cnt[2 * (u - 1)];
            cnt[2 * u + 1] += cnt[2 * (u - 1) + 1];
        }
        size_t wk = cnt[2 * th], wb = cnt[2 * th + 1];
        for (size_t i = lo; i < hi; ++i) {
            const uint32_t e = al->ids[i];
            if (state[e] != 0) continue;
            al->spare[wk++] = e;
            if (support[e] < t) out[wb++] = e;
        }
    }
    uint32_t* x = al->ids;
    al->ids = al->spare;
    al->spare = x;
    al->n = cnt[2 * used];
    const size_t nb = cnt[2 * used + 1];
    free(cnt);
    return nb;
}

typedef struct {
    SymCsr g;
    AliveLists a;
    uint32_t* state;
    uint32_t* support;
    uint32_t* removed;
    uint32_t* crossed;
    ActiveList active;
    size_t alive;
} Peel;

static int peel_init(Peel* p, const uint32_t* offsets, const uint32_t* targets, uint32_t n, const uint32_t* support0) {
    memset(p, 0, sizeof(*p));
    if (sym_init(&p->g, offsets, targets, n) != 0) {
        sym_free(&p->g);
        return -1;
    }
    const size_t E = p->g.E ? p->g.E : 1;
    p->state = (uint32_t*)calloc(E, sizeof(uint32_t));
    p->support = (uint32_t*)malloc(sizeof(uint32_t) * E);
    p->removed = (uint32_t*)malloc(sizeof(uint32_t) * E);
    p->crossed = (uint32_t*)malloc(sizeof(uint32_t) * E);
    p->a.off = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    p->a.tgt = (uint32_t*)malloc(sizeof(uint32_t) * E);
    p->a.eid = (uint32_t*)malloc(sizeof(uint32_t) * E);
    if (support0)
        memcpy(p->support, support0, sizeof(uint32_t) * p->g.E);
    else
        edge_support(&p->g, p->support);
    p->alive = p->g.E / 2;
    alive_build(&p->g, p->state, &p->a, p->alive);
    p->active.ids = (uint32_t*)malloc(sizeof(uint32_t) * (p->alive ? p->alive : 1));
    p->active.spare = (uint32_t*)malloc(sizeof(uint32_t) * (p->alive ? p->alive : 1));
    p->active.n = 0;
    for (size_t j = 0; j < p->g.E; ++j)
        if (p->g.tgt[j] > p->g.src[j]) p->active.ids[p->active.n++] = (uint32_t)j;
    return 0;
}

static void peel_free(Peel* p) {
    sym_free(&p->g);
    free(p->state);
    free(p->support);
    free(p->removed);
    free(p->crossed);
    free(p->a.off);
    free(p->a.tgt);
    free(p->a.eid);
    free(p->active.ids);
    free(p->active.spare);
}

/* Marks `nrem` removals of round rnd, peels them and compacts the alive
 * lists once a quarter of the edges they held are gone; returns the crossed count
 * (the crossed list is left in p->removed for the next round). */
static size_t peel_step(Peel* p, size_t nrem, uint32_t rnd, uint32_t threshold) {
    for (size_t i = 0; i < nrem; ++i) p->state[p->removed[i]] = rnd;
    const size_t nc = peel_round(&p->g, &p->a, p->state, p->support, p->removed, nrem, rnd, threshold, p->crossed);
    p->alive -= nrem;
    if (p->alive * 4 <= p->a.alive_at_build * 3) alive_build(&p->g, p->state, &p->a, p->alive);
    uint32_t* t = p->removed;
    p->removed = p->crossed;
    p->crossed = t;
    return nc;
}

/* Per-edge support of a simple symmetric CSR (both entries of an edge carry
 * it); -1 when the CSR is not simple and symmetric. */
int orc_edge_support(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t* support) {
    SymCsr g;
    if (sym_init(&g, offsets, targets, n) != 0) {
        sym_free(&g);
        return -1;
    }
    edge_support(&g, support);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)g.E; ++j)
        if (g.tgt[j] < g.src[j]) support[j] = support[g.eid[j]];
    sym_free(&g);
    return 0;
}

size_t orc_k_truss_peel(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t k,
                        const uint32_t* support0, uint32_t* out, uint32_t* iterations) {
    *iterations = 0;
    if (offsets[n] == 0) return 0; /* no edges, no rounds (k_truss.rs:53-60) */
    Peel p;
    if (peel_init(&p, offsets, targets, n, support0) != 0) return (size_t)-1;
    const uint32_t threshold = k >= 2 ? k - 2 : 0;
    uint32_t rnd = 1;
    size_t nrem = scan_below(&p.active, p.state, p.support, threshold, p.removed);
    while (nrem > 0) {
        nrem = peel_step(&p, nrem, rnd, threshold);
        ++rnd;
    }
    *iterations = rnd;
    size_t count = 0;
    for (size_t j = 0; j < p.g.E; ++j)
        if (p.g.tgt[j] > p.g.src[j] && p.state[j] == 0) {
            if (out) {
                out[2 * count] = p.g.src[j];
                out[2 * count + 1] = p.g.tgt[j];
            }
            ++count;
        }
    peel_free(&p);
    return count;
}

int orc_truss_decomposition_peel(const uint32_t* offsets, const uint32_t* targets, uint32_t n,
                                 const uint32_t* support0, uint32_t* trussness, uint32_t* max_trussness,
                                 uint32_t* rounds) {
    *max_trussness = 0;
    *rounds = 0;
    if (offsets[n] == 0) return 0;
    Peel p;
    if (peel_init(&p, offsets, targets, n, support0) != 0) return -1;
    uint32_t* level = (uint32_t*)calloc(p.g.E, sizeof(uint32_t)); /* trussness per u < v entry */
    uint32_t rnd = 0, k = 3, top = p.alive ? 2 : 0;
    int level_start = 1;
    size_t nrem = 0;
    while (p.alive > 0) {
        ++rnd;
        if (level_start) nrem = scan_below(&p.active, p.state, p.support, k - 2, p.removed);
        if (nrem == 0) {
            top = k;
            ++k;
            level_start = 1;
            continue;
        }
        for (size_t i = 0; i < nrem; ++i) level[p.removed[i]] = k - 1;
        nrem = peel_step(&p, nrem, rnd, k - 2);
        level_start = 0;
    }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)p.g.E; ++j) trussness[j] = level[p.g.eid[j]];
    *max_trussness = top;
    *rounds = rnd;
    free(level);
    peel_free(&p);
    return 0;
}
