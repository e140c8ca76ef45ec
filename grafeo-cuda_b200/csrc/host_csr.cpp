// Host-side CSR construction and validation.
//
// Restates crates/grafeo-cuda-core/src/csr_export.rs: validate_csr (:71-120),
// from_edge_pairs (:202-239), parse_tsv_to_edges (:246-287) and
// from_edge_pairs_oriented (:299-350), with the same outputs and messages.
// The synthetic generators (R-MAT, Erdos-Renyi) produce the benchmark inputs
// that stand in for the Graph500/GraphChallenge TSV files the reference reads.
#include <omp.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "gcu_internal.h"

namespace gcu {

// ---------------------------------------------------------------- validation

static std::string not_increasing_msg(uint64_t node, uint32_t prev, uint32_t target) {
    // The reference message keeps the 22 spaces of its source literal
    // (csr_export.rs:113).
    return "neighbor list of node " + std::to_string(node) + " is not strictly increasing" +
           std::string(22, ' ') + "(" + std::to_string(prev) + " then " + std::to_string(target) + ")";
}

std::string describe_node_violation(uint32_t node, uint32_t start, uint32_t end, const uint32_t* list,
                                    size_t list_len, uint32_t num_nodes) {
    if (end < start) {
        return "offsets decrease at node " + std::to_string(node) + ": " + std::to_string(start) +
               " then " + std::to_string(end);
    }
    for (size_t p = 0; p < list_len; ++p) {
        uint32_t t = list[p];
        if (t >= num_nodes) {
            return "node " + std::to_string(node) + " has neighbor " + std::to_string(t) +
                   ", but there are only " + std::to_string(num_nodes) + " nodes";
        }
        if (p > 0 && list[p - 1] >= t) return not_increasing_msg(node, list[p - 1], t);
    }
    if (static_cast<size_t>(end) - start > list_len) {
        // The list runs past the targets array (offsets rise above their last
        // value and fall again later); the reference cannot index it either.
        return "offsets at node " + std::to_string(node) + " point past the end of targets (" +
               std::to_string(start) + ".." + std::to_string(end) + ")";
    }
    return "node " + std::to_string(node) + " is malformed";
}

Error validate_csr_host(const uint32_t* offsets, size_t n_offsets, const uint32_t* targets, size_t n_targets) {
    if (n_offsets == 0) {
        return invalid_csr("offsets must have num_nodes + 1 entries, got an empty array");
    }
    if (n_offsets > 0xFFFFFFFFull || n_targets > 0xFFFFFFFFull) {
        return invalid_csr("graph too large for u32 indices: " + std::to_string(n_offsets) + " offsets, " +
                           std::to_string(n_targets) + " targets");
    }
    if (offsets[0] != 0) return invalid_csr("offsets[0] must be 0, got " + std::to_string(offsets[0]));
    const size_t n = n_offsets - 1;
    if (static_cast<size_t>(offsets[n]) != n_targets) {
        return invalid_csr("offsets[" + std::to_string(n) + "] is " + std::to_string(offsets[n]) +
                           " but targets has " + std::to_string(n_targets) + " entries");
    }
    for (size_t node = 0; node < n; ++node) {
        uint32_t start = offsets[node], end = offsets[node + 1];
        bool bad = end < start || static_cast<size_t>(end) > n_targets;
        if (!bad) {
            for (uint32_t j = start; j < end; ++j) {
                uint32_t t = targets[j];
                if (t >= n || (j > start && targets[j - 1] >= t)) {
                    bad = true;
                    break;
                }
            }
        }
        if (bad) {
            size_t lo = std::min<size_t>(start, n_targets);
            size_t hi = std::min<size_t>(std::max(start, end), n_targets);
            return invalid_csr(describe_node_violation(static_cast<uint32_t>(node), start, end, targets + lo,
                                                       hi - lo, static_cast<uint32_t>(n)));
        }
    }
    return ok();
}

// ---------------------------------------------------------------- builders

// Builds a CSR from (src, dst) pairs already sorted and deduplicated.
static void csr_from_sorted_pairs(const std::vector<uint64_t>& keys, uint32_t num_nodes, HostCsr* out) {
    out->num_nodes = num_nodes;
    out->offsets.assign(static_cast<size_t>(num_nodes) + 1, 0);
    out->targets.resize(keys.size());
    for (size_t i = 0; i < keys.size(); ++i) {
        out->offsets[(keys[i] >> 32) + 1] += 1;
        out->targets[i] = static_cast<uint32_t>(keys[i]);
    }
    for (size_t i = 1; i <= num_nodes; ++i) out->offsets[i] += out->offsets[i - 1];
}

Error from_edge_pairs(const uint32_t* pairs, size_t n_pairs, uint32_t num_nodes, bool symmetric, HostCsr* out) {
    std::vector<uint64_t> keys;
    keys.reserve(symmetric ? 2 * n_pairs : n_pairs);
    for (size_t i = 0; i < n_pairs; ++i) {
        uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        if (s >= num_nodes || (symmetric && d >= num_nodes)) {
            return export_error("edge (" + std::to_string(s) + ", " + std::to_string(d) +
                                ") references a node >= num_nodes (" + std::to_string(num_nodes) + ")");
        }
        keys.push_back((static_cast<uint64_t>(s) << 32) | d);
        if (symmetric && s != d) keys.push_back((static_cast<uint64_t>(d) << 32) | s);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if (keys.size() > 0xFFFFFFFFull) return export_error("too many CSR entries for u32 offsets");
    csr_from_sorted_pairs(keys, num_nodes, out);
    return ok();
}

Error from_edge_pairs_oriented(const uint32_t* pairs, size_t n_pairs, uint32_t num_nodes, HostCsr* out) {
    std::vector<uint64_t> und;
    und.reserve(n_pairs);
    for (size_t i = 0; i < n_pairs; ++i) {
        uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        if (s >= num_nodes || d >= num_nodes) {
            return export_error("edge (" + std::to_string(s) + ", " + std::to_string(d) +
                                ") references a node >= num_nodes (" + std::to_string(num_nodes) + ")");
        }
        if (s == d) continue;
        uint32_t lo = std::min(s, d), hi = std::max(s, d);
        und.push_back((static_cast<uint64_t>(lo) << 32) | hi);
    }
    std::sort(und.begin(), und.end());
    und.erase(std::unique(und.begin(), und.end()), und.end());
    std::vector<uint32_t> degree(num_nodes, 0);
    for (uint64_t k : und) {
        degree[k >> 32] += 1;
        degree[static_cast<uint32_t>(k)] += 1;
    }
    for (auto& k : und) {
        uint32_t u = static_cast<uint32_t>(k >> 32), v = static_cast<uint32_t>(k);
        uint32_t du = degree[u], dv = degree[v];
        if (!(du < dv || (du == dv && u < v))) k = (static_cast<uint64_t>(v) << 32) | u;
    }
    std::sort(und.begin(), und.end());
    csr_from_sorted_pairs(und, num_nodes, out);
    return ok();
}

static bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Parses a u64 like Rust's `str::parse::<u64>`: optional '+', digits only.
static bool parse_u64(const std::string& tok, uint64_t* v) {
    size_t i = 0;
    if (i < tok.size() && tok[i] == '+') ++i;
    if (i == tok.size()) return false;
    uint64_t acc = 0;
    for (; i < tok.size(); ++i) {
        char c = tok[i];
        if (c < '0' || c > '9') return false;
        uint64_t d = static_cast<uint64_t>(c - '0');
        if (acc > (UINT64_MAX - d) / 10) return false;
        acc = acc * 10 + d;
    }
    *v = acc;
    return true;
}

Error parse_tsv(const char* path, std::vector<uint32_t>* pairs, uint32_t* num_nodes) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        return export_error(std::string("cannot open ") + path + ": " + std::strerror(errno));
    }
    std::unordered_map<uint64_t, uint32_t> ids;
    uint32_t next = 0;
    std::string line;
    auto id_of = [&](uint64_t raw) {
        auto it = ids.find(raw);
        if (it != ids.end()) return it->second;
        ids.emplace(raw, next);
        return next++;
    };
    while (std::getline(in, line)) {
        size_t b = 0, e = line.size();
        while (b < e && is_ws(line[b])) ++b;
        while (e > b && is_ws(line[e - 1])) --e;
        if (b == e || line[b] == '#' || line[b] == '%') continue;
        std::string tok[2];
        size_t p = b;
        int got = 0;
        while (got < 2 && p < e) {
            while (p < e && is_ws(line[p])) ++p;
            size_t q = p;
            while (q < e && !is_ws(line[q])) ++q;
            if (q > p) tok[got++] = line.substr(p, q - p);
            p = q;
        }
        uint64_t s, d;
        if (got < 1 || !parse_u64(tok[0], &s)) continue;
        if (got < 2 || !parse_u64(tok[1], &d)) continue;
        uint32_t si = id_of(s);
        uint32_t di = id_of(d);
        pairs->push_back(si);
        pairs->push_back(di);
    }
    *num_nodes = next;
    return ok();
}

// ---------------------------------------------------------------- generators

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): the n-th output of the
// generator seeded with `state` is mix(state + (n + 1) * golden gamma), which
// makes it a counter-based stream that any thread can index directly.
static inline uint64_t splitmix_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
static inline uint64_t stream_at(uint64_t state, uint64_t n) { return splitmix_mix(state + (n + 1) * kGamma); }
static inline double unit_double(uint64_t r) { return static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0); }

// Symmetric, loop-free, deduplicated CSR from raw (possibly repeated) pairs:
// counting sort by endpoint, then a sort + unique of each neighbour list.
static Error symmetric_csr_from_pairs(const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst,
                                      uint32_t n, HostCsr* out) {
    const size_t m = src.size();
    std::vector<uint64_t> start(static_cast<size_t>(n) + 1, 0);
    {
        std::vector<uint32_t> cnt(n, 0);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < m; ++i) {
            uint32_t s = src[i], d = dst[i];
            if (s == d) continue;
            __atomic_fetch_add(&cnt[s], 1u, __ATOMIC_RELAXED);
            __atomic_fetch_add(&cnt[d], 1u, __ATOMIC_RELAXED);
        }
        for (size_t v = 0; v < n; ++v) start[v + 1] = start[v] + cnt[v];
    }
    std::vector<uint32_t> bucket(start[n]);
    {
        std::vector<uint64_t> cursor(start.begin(), start.end() - 1);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < m; ++i) {
            uint32_t s = src[i], d = dst[i];
            if (s == d) continue;
            uint64_t ps = __atomic_fetch_add(&cursor[s], 1ull, __ATOMIC_RELAXED);
            uint64_t pd = __atomic_fetch_add(&cursor[d], 1ull, __ATOMIC_RELAXED);
            bucket[ps] = d;
            bucket[pd] = s;
        }
    }
    std::vector<uint32_t> deg(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (size_t v = 0; v < n; ++v) {
        uint32_t* b = bucket.data() + start[v];
        uint32_t* e = bucket.data() + start[v + 1];
        std::sort(b, e);
        deg[v] = static_cast<uint32_t>(std::unique(b, e) - b);
    }
    uint64_t total = 0;
    out->offsets.resize(static_cast<size_t>(n) + 1);
    for (size_t v = 0; v < n; ++v) {
        out->offsets[v] = static_cast<uint32_t>(total);
        total += deg[v];
        if (total > 0xFFFFFFFFull) return export_error("too many CSR entries for u32 offsets");
    }
    out->offsets[n] = static_cast<uint32_t>(total);
    out->targets.resize(total);
#pragma omp parallel for schedule(dynamic, 1024)
    for (size_t v = 0; v < n; ++v) {
        std::memcpy(out->targets.data() + out->offsets[v], bucket.data() + start[v], sizeof(uint32_t) * deg[v]);
    }
    out->num_nodes = n;
    return ok();
}

Error generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                    HostCsr* out) {
    if (scale == 0 || scale > 31) return export_error("R-MAT scale must be in 1..=31");
    if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return export_error("R-MAT probabilities must be >= 0 and sum to <= 1");
    const uint32_t n = 1u << scale;
    const size_t m = static_cast<size_t>(edge_factor) << scale;
    const uint64_t state = splitmix_mix(seed + kGamma);
    std::vector<uint32_t> src(m), dst(m);
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < m; ++i) {
        uint32_t s = 0, d = 0;
        for (uint32_t l = 0; l < scale; ++l) {
            double u = unit_double(stream_at(state, static_cast<uint64_t>(i) * scale + l));
            uint32_t sb = 0, db = 0;
            if (u < a) {
            } else if (u < ab) {
                db = 1;
            } else if (u < abc) {
                sb = 1;
            } else {
                sb = 1;
                db = 1;
            }
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        src[i] = s;
        dst[i] = d;
    }
    return symmetric_csr_from_pairs(src, dst, n, out);
}

Error generate_erdos_renyi(uint32_t n, uint64_t num_pairs, uint64_t seed, HostCsr* out) {
    if (n == 0) {
        out->num_nodes = 0;
        out->offsets.assign(1, 0);
        out->targets.clear();
        return ok();
    }
    const uint64_t state = splitmix_mix(seed + kGamma);
    std::vector<uint32_t> src(num_pairs), dst(num_pairs);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < num_pairs; ++i) {
        uint64_t r1 = stream_at(state, 2 * static_cast<uint64_t>(i));
        uint64_t r2 = stream_at(state, 2 * static_cast<uint64_t>(i) + 1);
        src[i] = static_cast<uint32_t>((static_cast<unsigned __int128>(r1) * n) >> 64);
        dst[i] = static_cast<uint32_t>((static_cast<unsigned __int128>(r2) * n) >> 64);
    }
    return symmetric_csr_from_pairs(src, dst, n, out);
}

}  // namespace gcu

using namespace gcu;

struct gcu_csr {
    HostCsr csr;
};

extern "C" {

GCU_API gcu_status gcu_validate_csr(const uint32_t* offsets, size_t n_offsets, const uint32_t* targets,
                                    size_t n_targets) {
    if (n_offsets && !offsets) return fail(kernel_error("offsets is NULL"));
    if (n_targets && !targets) return fail(kernel_error("targets is NULL"));
    Error e = validate_csr_host(offsets, n_offsets, targets, n_targets);
    return e.ok() ? succeed() : fail(e);
}

GCU_API gcu_status gcu_csr_from_edge_pairs(const uint32_t* pairs, size_t n_pairs, uint32_t num_nodes,
                                           int symmetric, gcu_csr** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    if (n_pairs && !pairs) return fail(kernel_error("pairs is NULL"));
    auto c = std::make_unique<gcu_csr>();
    Error e = from_edge_pairs(pairs, n_pairs, num_nodes, symmetric != 0, &c->csr);
    if (!e.ok()) return fail(e);
    *out = c.release();
    return succeed();
}

GCU_API gcu_status gcu_csr_from_edge_pairs_oriented(const uint32_t* pairs, size_t n_pairs, uint32_t num_nodes,
                                                    gcu_csr** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    if (n_pairs && !pairs) return fail(kernel_error("pairs is NULL"));
    auto c = std::make_unique<gcu_csr>();
    Error e = from_edge_pairs_oriented(pairs, n_pairs, num_nodes, &c->csr);
    if (!e.ok()) return fail(e);
    *out = c.release();
    return succeed();
}

GCU_API gcu_status gcu_parse_tsv_to_edges(const char* path, uint32_t** pairs, size_t* n_pairs,
                                          uint32_t* num_nodes) {
    if (!path || !pairs || !n_pairs || !num_nodes) return fail(kernel_error("NULL argument"));
    *pairs = nullptr;
    *n_pairs = 0;
    *num_nodes = 0;
    std::vector<uint32_t> v;
    uint32_t n = 0;
    Error e = parse_tsv(path, &v, &n);
    if (!e.ok()) return fail(e);
    uint32_t* buf = static_cast<uint32_t*>(std::malloc(std::max<size_t>(v.size(), 1) * sizeof(uint32_t)));
    if (!buf) return fail(export_error("out of host memory"));
    if (!v.empty()) std::memcpy(buf, v.data(), v.size() * sizeof(uint32_t));
    *pairs = buf;
    *n_pairs = v.size() / 2;
    *num_nodes = n;
    return succeed();
}

GCU_API void gcu_free_pairs(uint32_t* pairs) { std::free(pairs); }

GCU_API gcu_status gcu_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                     uint64_t seed, gcu_csr** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    auto r = std::make_unique<gcu_csr>();
    Error e = generate_rmat(scale, edge_factor, a, b, c, seed, &r->csr);
    if (!e.ok()) return fail(e);
    *out = r.release();
    return succeed();
}

GCU_API gcu_status gcu_generate_erdos_renyi(uint32_t num_nodes, uint64_t num_pairs, uint64_t seed, gcu_csr** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    auto r = std::make_unique<gcu_csr>();
    Error e = generate_erdos_renyi(num_nodes, num_pairs, seed, &r->csr);
    if (!e.ok()) return fail(e);
    *out = r.release();
    return succeed();
}

GCU_API uint32_t gcu_csr_num_nodes(const gcu_csr* csr) { return csr ? csr->csr.num_nodes : 0; }
GCU_API uint64_t gcu_csr_num_edges(const gcu_csr* csr) { return csr ? csr->csr.targets.size() : 0; }
GCU_API const uint32_t* gcu_csr_offsets(const gcu_csr* csr) { return csr ? csr->csr.offsets.data() : nullptr; }
GCU_API const uint32_t* gcu_csr_targets(const gcu_csr* csr) {
    return csr && !csr->csr.targets.empty() ? csr->csr.targets.data() : nullptr;
}
GCU_API void gcu_csr_free(gcu_csr* csr) { delete csr; }

}  // extern "C"
