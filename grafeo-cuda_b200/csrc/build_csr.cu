// Device CSR construction: edge pairs (copied from the host or generated on
// the device) -> sorted, deduplicated u32 CSR, built in HBM.
//
// Restates on the device what crates/grafeo-cuda-core/src/csr_export.rs
// builds on the host: from_edge_pairs (:202-239: one (src, dst) key per pair,
// the reverse key too when symmetric, sort, dedup) and
// from_edge_pairs_oriented (:299-350: undirected dedup without self-loops,
// each edge oriented from the lower (degree, id) end, sort). Keys are
// (source << 32) | target; the stable LSD radix sort of sort.cu runs over the
// bits the ids actually use, the target bits first and the source bits second
// (two digit runs of one LSD sort). Deduplication and the row pointers come
// from one scan over "key differs from its predecessor" flags.
//
// The generators (R-MAT, Erdos-Renyi, 2D grid with edge dropout, random
// geometric, Watts-Strogatz) append their keys straight into the key buffer
// from the SplitMix64 streams that host_csr.cpp uses, so a device-generated
// R-MAT or Erdos-Renyi graph equals the host-generated one entry for entry.
// Appends are warp-aggregated atomics: the append order varies from run to
// run, the sorted result does not.
#include <algorithm>
#include <cmath>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

namespace {

constexpr int kBuildThreads = 256;

__device__ __forceinline__ uint64_t sm64_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
__host__ __device__ __forceinline__ uint64_t host_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t stream_at(uint64_t state, uint64_t n) { return sm64_mix(state + (n + 1) * kGamma); }
__device__ __forceinline__ double unit_double(uint64_t r) {
    return static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ uint32_t scale_to(uint64_t r, uint32_t n) {
    return static_cast<uint32_t>(__umul64hi(r, static_cast<uint64_t>(n)));
}

// Warp-aggregated append of `want` keys per lane (all 32 lanes call it);
// returns this lane's first slot.
__device__ __forceinline__ unsigned long long warp_append(unsigned long long* counter, uint32_t want) {
    const uint32_t incl = warp_inclusive_scan(want);
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    unsigned long long base = 0;
    if (lane_id() == 31 && total) base = atomicAdd(counter, static_cast<unsigned long long>(total));
    base = __shfl_sync(kFullMask, base, 31);
    return base + incl - want;
}

__device__ __forceinline__ uint64_t key_of(uint32_t s, uint32_t d) { return (static_cast<uint64_t>(s) << 32) | d; }

// Both directions of an undirected non-loop edge, nothing for a self-loop.
__device__ __forceinline__ void append_undirected(unsigned long long* count, uint64_t* keys, bool valid, uint32_t s,
                                                  uint32_t d) {
    const uint32_t want = (valid && s != d) ? 2u : 0u;
    const unsigned long long slot = warp_append(count, want);
    if (want) {
        keys[slot] = key_of(s, d);
        keys[slot + 1] = key_of(d, s);
    }
}

// Grid-stride loop whose trip count is the same for the 32 lanes of a warp
// (the warp-wide helpers above need every lane).
#define GCU_WARP_UNIFORM_LOOP(i, n)                                                                            \
    for (uint64_t _b = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~uint64_t(31), i = 0; \
         i = _b + lane_id(), _b < (n); _b += static_cast<uint64_t>(gridDim.x) * blockDim.x)

enum PairMode : int { kDirected = 0, kSymmetric = 1, kUndirected = 2 };

// Keys of host pairs (csr_export.rs:211-231 and :306-318): kDirected one key
// per pair, kSymmetric the reverse too (a self-loop once), kUndirected
// (min, max) without self-loops. Records the first pair whose source (or,
// unless kDirected, target) is >= num_nodes, and the largest target.
__global__ void __launch_bounds__(kBuildThreads) pairs_to_keys_kernel(const uint32_t* __restrict__ pairs,
                                                                      uint64_t n_pairs, uint32_t num_nodes, int mode,
                                                                      uint64_t* __restrict__ keys,
                                                                      unsigned long long* __restrict__ count,
                                                                      unsigned long long* __restrict__ first_bad,
                                                                      unsigned* __restrict__ max_target) {
    uint32_t local_max = 0;
    GCU_WARP_UNIFORM_LOOP(i, n_pairs) {
        const bool valid = i < n_pairs;
        uint32_t s = 0, d = 0;
        if (valid) {
            s = pairs[2 * i];
            d = pairs[2 * i + 1];
        }
        const bool bad = valid && (s >= num_nodes || (mode != kDirected && d >= num_nodes));
        if (bad) atomicMin(first_bad, static_cast<unsigned long long>(i));
        uint32_t want = 0;
        if (valid && !bad) {
            if (mode == kDirected)
                want = 1;
            else if (mode == kSymmetric)
                want = s == d ? 1 : 2;
            else
                want = s == d ? 0 : 1;
            local_max = max(local_max, d);
        }
        const unsigned long long slot = warp_append(count, want);
        if (want) {
            if (mode == kUndirected) {
                keys[slot] = key_of(min(s, d), max(s, d));
            } else {
                keys[slot] = key_of(s, d);
                if (want == 2) keys[slot + 1] = key_of(d, s);
            }
        }
    }
    local_max = __reduce_max_sync(kFullMask, local_max);
    if (lane_id() == 0 && local_max) atomicMax(max_target, local_max);
}

// R-MAT pairs as host_csr.cpp generate_rmat draws them: `scale` quadrant
// choices per pair from consecutive stream positions.
__global__ void __launch_bounds__(kBuildThreads) rmat_keys_kernel(uint64_t state, uint32_t scale, uint64_t m,
                                                                  double a, double ab, double abc,
                                                                  uint64_t* __restrict__ keys,
                                                                  unsigned long long* __restrict__ count,
                                                                  uint32_t base) {
    GCU_WARP_UNIFORM_LOOP(i, m) {
        const bool valid = i < m;
        uint32_t s = 0, d = 0;
        if (valid) {
            for (uint32_t l = 0; l < scale; ++l) {
                const double u = unit_double(stream_at(state, i * scale + l));
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
        }
        append_undirected(count, keys, valid, s + base, d + base);
    }
}

// G(n, m) pairs as host_csr.cpp generate_erdos_renyi draws them.
__global__ void __launch_bounds__(kBuildThreads) er_keys_kernel(uint64_t state, uint32_t n, uint64_t m,
                                                                uint64_t* __restrict__ keys,
                                                                unsigned long long* __restrict__ count) {
    GCU_WARP_UNIFORM_LOOP(i, m) {
        const bool valid = i < m;
        uint32_t s = 0, d = 0;
        if (valid) {
            s = scale_to(stream_at(state, 2 * i), n);
            d = scale_to(stream_at(state, 2 * i + 1), n);
        }
        append_undirected(count, keys, valid, s, d);
    }
}

// width x height grid, vertex y * width + x. Lattice edge e (the horizontal
// edges (x, y)-(x + 1, y) first, index y * (width - 1) + x, then the vertical
// ones (x, y)-(x, y + 1), index H + y * width + x) is dropped when stream
// value e is below `drop`.
__global__ void __launch_bounds__(kBuildThreads) grid_keys_kernel(uint64_t state, uint32_t width, uint32_t height,
                                                                  double drop, uint64_t* __restrict__ keys,
                                                                  unsigned long long* __restrict__ count) {
    const uint64_t horizontal = static_cast<uint64_t>(height) * (width - 1);
    const uint64_t total = horizontal + static_cast<uint64_t>(height - 1) * width;
    GCU_WARP_UNIFORM_LOOP(e, total) {
        bool keep = e < total;
        uint32_t s = 0, d = 0;
        if (keep) {
            if (e < horizontal) {
                const uint64_t y = e / (width - 1), x = e - y * (width - 1);
                s = static_cast<uint32_t>(y * width + x);
                d = s + 1;
            } else {
                const uint64_t f = e - horizontal;
                s = static_cast<uint32_t>(f);
                d = s + width;
            }
            keep = unit_double(stream_at(state, e)) >= drop;
        }
        append_undirected(count, keys, keep, s, d);
    }
}

// Watts-Strogatz: ring lattice u -- u + j (j = 1..half), and lattice edge
// idx = u * half + j - 1 rewired to (u, w) when stream value 2 idx is below p,
// w drawn from value 2 idx + 1. Self-loops and repeats fall out in the build.
__global__ void __launch_bounds__(kBuildThreads) ws_keys_kernel(uint64_t state, uint32_t n, uint32_t half, double p,
                                                                uint64_t* __restrict__ keys,
                                                                unsigned long long* __restrict__ count,
                                                                uint32_t base) {
    const uint64_t total = static_cast<uint64_t>(n) * half;
    GCU_WARP_UNIFORM_LOOP(idx, total) {
        const bool valid = idx < total;
        uint32_t s = 0, d = 0;
        if (valid) {
            s = static_cast<uint32_t>(idx / half);
            const uint32_t j = static_cast<uint32_t>(idx - static_cast<uint64_t>(s) * half) + 1;
            d = static_cast<uint32_t>((static_cast<uint64_t>(s) + j) % n);
            if (unit_double(stream_at(state, 2 * idx)) < p) d = scale_to(stream_at(state, 2 * idx + 1), n);
        }
        append_undirected(count, keys, valid, s + base, d + base);
    }
}

// Random geometric graph: point i at (stream 2i, stream 2i + 1) in the unit
// square; cell keys (cell << 32) | i for the bucketing sort.
__global__ void geo_points_kernel(uint64_t state, uint32_t n, uint32_t cells_per_side, double2* __restrict__ pts,
                                  uint64_t* __restrict__ cell_keys) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double x = unit_double(stream_at(state, 2 * i)), y = unit_double(stream_at(state, 2 * i + 1));
        pts[i] = make_double2(x, y);
        const uint32_t cx = min(cells_per_side - 1, static_cast<uint32_t>(x * cells_per_side));
        const uint32_t cy = min(cells_per_side - 1, static_cast<uint32_t>(y * cells_per_side));
        cell_keys[i] = (static_cast<uint64_t>(cy * cells_per_side + cx) << 32) | i;
    }
}

// cell_start[c] = first sorted position whose cell is >= c (c = 0..cells).
__global__ void geo_cell_starts_kernel(const uint64_t* __restrict__ sorted, uint32_t n, uint32_t cells,
                                       uint32_t* __restrict__ cell_start) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int64_t prev = i == 0 ? -1 : static_cast<int64_t>(sorted[i - 1] >> 32);
        const int64_t cur = i < n ? static_cast<int64_t>(sorted[i] >> 32) : static_cast<int64_t>(cells);
        for (int64_t c = prev + 1; c <= cur; ++c) cell_start[c] = static_cast<uint32_t>(i);
    }
}

// Pairs i < j at squared distance <= r2 (products and sums rounded
// separately, no fused multiply-add, so that a CPU restatement in double
// arithmetic draws the same edges). Point at sorted position p either counts
// its keys into counts[p] (emit = false) or writes them from slot base[p].
__global__ void __launch_bounds__(kBuildThreads) geo_pairs_kernel(const double2* __restrict__ pts,
                                                                  const uint64_t* __restrict__ sorted,
                                                                  const uint32_t* __restrict__ cell_start, uint32_t n,
                                                                  uint32_t side, double r2, bool emit,
                                                                  uint32_t* __restrict__ counts_or_base,
                                                                  uint64_t* __restrict__ keys) {
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = static_cast<uint32_t>(sorted[p]);
        const uint32_t cell = static_cast<uint32_t>(sorted[p] >> 32);
        const uint32_t cx = cell % side, cy = cell / side;
        const double2 a = pts[i];
        uint32_t slot = emit ? counts_or_base[p] : 0u;
        for (uint32_t yy = cy > 0 ? cy - 1 : 0; yy <= min(cy + 1, side - 1); ++yy) {
            for (uint32_t xx = cx > 0 ? cx - 1 : 0; xx <= min(cx + 1, side - 1); ++xx) {
                const uint32_t c = yy * side + xx;
                for (uint32_t q = cell_start[c]; q < cell_start[c + 1]; ++q) {
                    const uint32_t j = static_cast<uint32_t>(sorted[q]);
                    if (j <= i) continue;
                    const double2 b = pts[j];
                    const double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y);
                    if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= r2) {
                        if (emit) {
                            keys[slot] = key_of(i, j);
                            keys[slot + 1] = key_of(j, i);
                        }
                        slot += 2;
                    }
                }
            }
        }
        if (!emit) counts_or_base[p] = slot;
    }
}

// flags[i] = key i differs from key i - 1 (the first key always does).
__global__ void mark_first_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ flags) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// Unique keys -> targets at their scanned positions; rows s_prev < r <= s
// (s_prev = source of key i - 1, s = source of key i, or num_nodes past the
// end) start at pos[i]. Every row gets exactly one writer.
__global__ void keys_to_csr_kernel(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ pos,
                                   uint32_t num_nodes, uint32_t* __restrict__ offsets,
                                   uint32_t* __restrict__ targets) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int64_t prev = i == 0 ? -1 : static_cast<int64_t>(keys[i - 1] >> 32);
        const int64_t cur = i < n ? static_cast<int64_t>(keys[i] >> 32) : static_cast<int64_t>(num_nodes);
        const uint32_t p = pos[i];
        if (i < n && (i == 0 || keys[i] != keys[i - 1])) targets[p] = static_cast<uint32_t>(keys[i]);
        for (int64_t r = prev + 1; r <= cur; ++r) offsets[r] = p;
    }
}

// Unique keys -> out[pos[i]] (compaction).
__global__ void compact_unique_kernel(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ pos,
                                      uint64_t* __restrict__ out) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (i == 0 || keys[i] != keys[i - 1]) out[pos[i]] = keys[i];
}

__global__ void undirected_degree_kernel(const uint64_t* __restrict__ keys, uint64_t m, uint32_t* __restrict__ deg) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        atomicAdd(deg + (keys[i] >> 32), 1u);
        atomicAdd(deg + static_cast<uint32_t>(keys[i]), 1u);
    }
}

// u -> v when d(u) < d(v), or equal degrees and u < v (csr_export.rs:327-336).
__global__ void orient_keys_kernel(uint64_t* __restrict__ keys, uint64_t m, const uint32_t* __restrict__ deg) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = static_cast<uint32_t>(keys[i] >> 32), v = static_cast<uint32_t>(keys[i]);
        const uint32_t du = deg[u], dv = deg[v];
        if (!(du < dv || (du == dv && u < v))) keys[i] = key_of(v, u);
    }
}

uint32_t bit_length(uint64_t x) {
    uint32_t b = 0;
    while (b < 64 && (x >> b) != 0) ++b;
    return b;
}

unsigned grid_for(const DeviceImpl& dev, uint64_t n) {
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(n, kBuildThreads), cap)));
}

// Key scratch: keys and tmp of `capacity` entries plus the device append
// counter, first-bad index and largest target.
struct KeyScratch {
    DeviceBuffer<uint64_t> keys, tmp;
    DeviceBuffer<unsigned long long> meta;  // [0] count, [1] first bad pair
    DeviceBuffer<unsigned> max_target;
    Error allocate(DeviceImpl& dev, uint64_t capacity) {
        GCU_TRY(keys.allocate(dev, std::max<uint64_t>(capacity, 1)));
        GCU_TRY(tmp.allocate(dev, std::max<uint64_t>(capacity, 1)));
        GCU_TRY(meta.allocate(dev, 2));
        GCU_TRY(max_target.allocate(dev, 1));
        const unsigned long long init[2] = {0ull, ~0ull};
        GCU_CUDA(cudaMemcpyAsync(meta.ptr, init, sizeof(init), cudaMemcpyHostToDevice, dev.stream), "copy");
        GCU_CUDA(cudaMemsetAsync(max_target.ptr, 0, sizeof(unsigned), dev.stream), "memset");
        return ok();
    }
    Error read_meta(DeviceImpl& dev, uint64_t* count, uint64_t* first_bad, uint32_t* maxt) {
        unsigned long long m[2];
        unsigned mt = 0;
        GCU_CUDA(cudaMemcpyAsync(m, meta.ptr, sizeof(m), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_CUDA(cudaMemcpyAsync(&mt, max_target.ptr, sizeof(mt), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        *count = m[0];
        *first_bad = m[1];
        *maxt = mt;
        return ok();
    }
};

// Sorts keys[0..n) by target bits [0, target_bits) then source bits
// [32, 32 + source_bits); *sorted is whichever buffer holds the result.
Error sort_keys(DeviceImpl& dev, uint64_t* keys, uint64_t* tmp, uint64_t n, uint32_t target_bits,
                uint32_t source_bits, uint64_t** sorted, uint64_t** other) {
    uint64_t* s1 = nullptr;
    GCU_TRY(radix_sort_u64(dev, keys, tmp, n, 0, target_bits, &s1));
    uint64_t* o1 = s1 == keys ? tmp : keys;
    uint64_t* s2 = nullptr;
    GCU_TRY(radix_sort_u64(dev, s1, o1, n, 32, 32 + source_bits, &s2));
    *sorted = s2;
    *other = s2 == s1 ? o1 : s1;
    return ok();
}

// CSR of the sorted keys (repeats dropped) into a new graph's buffers.
Error csr_from_sorted_keys(DeviceImpl& dev, const uint64_t* sorted, uint64_t n, uint32_t num_nodes, GraphImpl& g) {
    DeviceBuffer<uint32_t> pos;
    GCU_TRY(pos.allocate(dev, n + 1));
    GCU_LAUNCH(dev, "build_mark_first", mark_first_kernel, grid_for(dev, n), kBuildThreads, 0, sorted, n, pos.ptr);
    GCU_TRY(exclusive_scan_u32(dev, pos.ptr, pos.ptr, n));
    uint32_t total = 0;
    GCU_CUDA(cudaMemcpyAsync(&total, pos.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    g.num_nodes = num_nodes;
    g.num_edges = total;
    GCU_TRY(g.offsets.allocate(dev, static_cast<uint64_t>(num_nodes) + 1));
    GCU_TRY(g.targets.allocate(dev, total));
    GCU_LAUNCH(dev, "build_keys_to_csr", keys_to_csr_kernel, grid_for(dev, n + 1), kBuildThreads, 0, sorted, n,
               pos.ptr, num_nodes, g.offsets.ptr, g.targets.ptr);
    GCU_TRY(dev.sync());  // scratch is freed on return
    return ok();
}

Error check_capacity(uint64_t keys) {
    if (keys > 0xFFFFFFFEull)
        return export_error("too many edge pairs for the device CSR builder (at most 4294967294 CSR entries "
                            "before deduplication, got " + std::to_string(keys) + ")");
    return ok();
}

}  // namespace

Error build_graph_from_pairs(DeviceImpl& dev, const uint32_t* host_pairs, uint64_t n_pairs, uint32_t num_nodes,
                             int mode, GraphImpl& g) {
    const uint64_t capacity = mode == kSymmetric ? 2 * n_pairs : n_pairs;
    GCU_TRY(check_capacity(capacity));
    DeviceBuffer<uint32_t> d_pairs;
    GCU_TRY(d_pairs.allocate(dev, std::max<uint64_t>(2 * n_pairs, 1)));
    if (n_pairs)
        GCU_CUDA(cudaMemcpyAsync(d_pairs.ptr, host_pairs, 8 * n_pairs, cudaMemcpyHostToDevice, dev.stream),
                 "copy edge pairs to device");
    KeyScratch ks;
    GCU_TRY(ks.allocate(dev, capacity));
    GCU_LAUNCH(dev, "build_pairs_to_keys", pairs_to_keys_kernel, grid_for(dev, n_pairs), kBuildThreads, 0, d_pairs.ptr,
               n_pairs, num_nodes, mode, ks.keys.ptr, ks.meta.ptr, ks.meta.ptr + 1, ks.max_target.ptr);
    uint64_t count = 0, bad = 0;
    uint32_t maxt = 0;
    GCU_TRY(ks.read_meta(dev, &count, &bad, &maxt));
    if (bad != ~0ull) {
        const uint32_t s = host_pairs[2 * bad], d = host_pairs[2 * bad + 1];
        return export_error("edge (" + std::to_string(s) + ", " + std::to_string(d) +
                            ") references a node >= num_nodes (" + std::to_string(num_nodes) + ")");
    }
    d_pairs.reset();
    const uint32_t id_bits = bit_length(num_nodes > 0 ? num_nodes - 1 : 0);
    const uint32_t target_bits = std::max(id_bits, bit_length(maxt));
    uint64_t *sorted = nullptr, *other = nullptr;
    GCU_TRY(sort_keys(dev, ks.keys.ptr, ks.tmp.ptr, count, target_bits, id_bits, &sorted, &other));
    if (mode == kSymmetric) {
        GCU_TRY(csr_from_sorted_keys(dev, sorted, count, num_nodes, g));
        g.symmetric = 1;
        return ok();
    }
    if (mode == kDirected) {
        GCU_TRY(csr_from_sorted_keys(dev, sorted, count, num_nodes, g));
        if (count == 0 || maxt < num_nodes) return ok();
        // A target >= num_nodes passes the builder (csr_export.rs:211-231) and
        // fails validate_csr when the CSR is loaded (gpu_graph.rs:46-63).
        uint32_t bad_node = UINT32_MAX;
        GCU_TRY(validate_csr_device(dev, g.offsets.ptr, g.targets.ptr, g.num_nodes, g.num_edges, &bad_node));
        if (bad_node == UINT32_MAX) return kernel_error("device CSR build: out-of-range target not found");
        uint32_t range[2];
        GCU_CUDA(cudaMemcpy(range, g.offsets.ptr + bad_node, sizeof(range), cudaMemcpyDeviceToHost), "copy");
        std::vector<uint32_t> list(range[1] - range[0]);
        if (!list.empty())
            GCU_CUDA(cudaMemcpy(list.data(), g.targets.ptr + range[0], 4 * list.size(), cudaMemcpyDeviceToHost),
                     "copy");
        return invalid_csr(
            describe_node_violation(bad_node, range[0], range[1], list.data(), list.size(), g.num_nodes));
    }

    // Oriented: unique undirected edges, degrees, orientation, sort again.
    DeviceBuffer<uint32_t> pos;
    GCU_TRY(pos.allocate(dev, count + 1));
    GCU_LAUNCH(dev, "build_mark_first", mark_first_kernel, grid_for(dev, count), kBuildThreads, 0, sorted, count,
               pos.ptr);
    GCU_TRY(exclusive_scan_u32(dev, pos.ptr, pos.ptr, count));
    uint32_t m = 0;
    GCU_CUDA(cudaMemcpyAsync(&m, pos.ptr + count, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_LAUNCH(dev, "build_compact_unique", compact_unique_kernel, grid_for(dev, count), kBuildThreads, 0, sorted,
               count, pos.ptr, other);
    GCU_TRY(dev.sync());
    DeviceBuffer<uint32_t> deg;
    GCU_TRY(deg.allocate(dev, std::max<uint32_t>(num_nodes, 1)));
    GCU_CUDA(cudaMemsetAsync(deg.ptr, 0, sizeof(uint32_t) * std::max<uint32_t>(num_nodes, 1), dev.stream), "memset");
    GCU_LAUNCH(dev, "build_degree", undirected_degree_kernel, grid_for(dev, m), kBuildThreads, 0, other, m, deg.ptr);
    GCU_LAUNCH(dev, "build_orient", orient_keys_kernel, grid_for(dev, m), kBuildThreads, 0, other, m, deg.ptr);
    uint64_t *sorted2 = nullptr, *other2 = nullptr;
    GCU_TRY(sort_keys(dev, other, sorted, m, id_bits, id_bits, &sorted2, &other2));
    return csr_from_sorted_keys(dev, sorted2, m, num_nodes, g);
}

Error generate_graph(DeviceImpl& dev, const GeneratorSpec& spec, GraphImpl& g) {
    uint64_t capacity = 0;
    uint32_t n = 0;
    switch (spec.kind) {
        case GeneratorSpec::kRmat:
            if (spec.scale == 0 || spec.scale > 31) return export_error("R-MAT scale must be in 1..=31");
            if (!(spec.a >= 0 && spec.b >= 0 && spec.c >= 0 && spec.a + spec.b + spec.c <= 1.0))
                return export_error("R-MAT probabilities must be >= 0 and sum to <= 1");
            n = 1u << spec.scale;
            capacity = 2 * (static_cast<uint64_t>(spec.edge_factor) << spec.scale);
            break;
        case GeneratorSpec::kErdosRenyi:
            n = spec.n;
            capacity = n ? 2 * spec.pairs : 0;
            break;
        case GeneratorSpec::kGrid: {
            const uint64_t v = static_cast<uint64_t>(spec.width) * spec.height;
            if (v > 0xFFFFFFFFull) return export_error("grid has more than 2^32 - 1 vertices");
            if (!(spec.p >= 0.0 && spec.p <= 1.0)) return export_error("grid drop probability must be in [0, 1]");
            n = static_cast<uint32_t>(v);
            capacity = n ? 2 * (static_cast<uint64_t>(spec.height) * (spec.width - 1) +
                                static_cast<uint64_t>(spec.height - 1) * spec.width)
                         : 0;
            break;
        }
        case GeneratorSpec::kWattsStrogatz:
            if (spec.k % 2 != 0) return export_error("Watts-Strogatz k must be even");
            if (!(spec.p >= 0.0 && spec.p <= 1.0)) return export_error("Watts-Strogatz p must be in [0, 1]");
            n = spec.n;
            capacity = 2 * static_cast<uint64_t>(n) * (spec.k / 2);
            break;
        case GeneratorSpec::kGeometric:
            if (!(spec.avg_degree > 0.0)) return export_error("geometric graph average degree must be > 0");
            n = spec.n;
            break;
    }
    const uint64_t state = host_mix(spec.seed + kGamma);
    if (n == 0) {
        g.num_nodes = 0;
        g.num_edges = 0;
        GCU_TRY(g.offsets.allocate(dev, 1));
        GCU_TRY(g.targets.allocate(dev, 0));
        GCU_CUDA(cudaMemsetAsync(g.offsets.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
        g.symmetric = 1;
        return dev.sync();
    }
    KeyScratch ks;
    DeviceBuffer<double2> pts;
    DeviceBuffer<uint32_t> cell_start, geo_slots;
    DeviceBuffer<uint64_t> cell_keys, cell_tmp;
    uint64_t* cell_sorted = nullptr;
    uint32_t side = 1;
    double r2 = 0.0;
    if (spec.kind == GeneratorSpec::kGeometric) {
        // Radius for the requested mean degree away from the border:
        // (n - 1) * pi * r^2 = avg_degree; cells of side >= r.
        const double r = n > 1 ? std::sqrt(spec.avg_degree / (M_PI * (n - 1))) : 1.0;
        r2 = r * r;
        // Cells no smaller than r (so a 3 x 3 block of cells holds every
        // neighbour), at most about one per point, side^2 < 2^31.
        side = static_cast<uint32_t>(
            std::max(1.0, std::min({std::floor(1.0 / r), std::floor(std::sqrt(static_cast<double>(n))), 46340.0})));
        const uint64_t cells = static_cast<uint64_t>(side) * side;
        GCU_TRY(pts.allocate(dev, n));
        GCU_TRY(cell_keys.allocate(dev, n));
        GCU_TRY(cell_tmp.allocate(dev, n));
        GCU_TRY(cell_start.allocate(dev, cells + 1));
        GCU_LAUNCH(dev, "gen_geo_points", geo_points_kernel, grid_for(dev, n), kBuildThreads, 0, state, n, side,
                   pts.ptr, cell_keys.ptr);
        GCU_TRY(radix_sort_u64(dev, cell_keys.ptr, cell_tmp.ptr, n, 32, 32 + bit_length(cells - 1), &cell_sorted));
        GCU_LAUNCH(dev, "gen_geo_cells", geo_cell_starts_kernel, grid_for(dev, n + 1), kBuildThreads, 0, cell_sorted,
                   n, static_cast<uint32_t>(cells), cell_start.ptr);
        GCU_TRY(geo_slots.allocate(dev, static_cast<uint64_t>(n) + 1));
        GCU_LAUNCH(dev, "gen_geo_count", geo_pairs_kernel, grid_for(dev, n), kBuildThreads, 0, pts.ptr, cell_sorted,
                   cell_start.ptr, n, side, r2, false, geo_slots.ptr, nullptr);
        GCU_TRY(exclusive_scan_u32(dev, geo_slots.ptr, geo_slots.ptr, n));
        uint32_t c = 0;
        GCU_CUDA(cudaMemcpyAsync(&c, geo_slots.ptr + n, sizeof(c), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        capacity = c;
    }
    GCU_TRY(check_capacity(capacity));
    GCU_TRY(ks.allocate(dev, capacity));
    switch (spec.kind) {
        case GeneratorSpec::kRmat: {
            const uint64_t m = static_cast<uint64_t>(spec.edge_factor) << spec.scale;
            GCU_LAUNCH(dev, "gen_rmat", rmat_keys_kernel, grid_for(dev, m), kBuildThreads, 0, state, spec.scale, m,
                       spec.a, spec.a + spec.b, spec.a + spec.b + spec.c, ks.keys.ptr, ks.meta.ptr, 0u);
            break;
        }
        case GeneratorSpec::kErdosRenyi:
            GCU_LAUNCH(dev, "gen_erdos_renyi", er_keys_kernel, grid_for(dev, spec.pairs), kBuildThreads, 0, state, n,
                       spec.pairs, ks.keys.ptr, ks.meta.ptr);
            break;
        case GeneratorSpec::kGrid:
            GCU_LAUNCH(dev, "gen_grid", grid_keys_kernel, grid_for(dev, capacity / 2), kBuildThreads, 0, state,
                       spec.width, spec.height, spec.p, ks.keys.ptr, ks.meta.ptr);
            break;
        case GeneratorSpec::kWattsStrogatz:
            GCU_LAUNCH(dev, "gen_watts_strogatz", ws_keys_kernel, grid_for(dev, capacity / 2), kBuildThreads, 0,
                       state, n, spec.k / 2, spec.p, ks.keys.ptr, ks.meta.ptr, 0u);
            break;
        case GeneratorSpec::kGeometric:
            GCU_LAUNCH(dev, "gen_geo_pairs", geo_pairs_kernel, grid_for(dev, n), kBuildThreads, 0, pts.ptr,
                       cell_sorted, cell_start.ptr, n, side, r2, true, geo_slots.ptr, ks.keys.ptr);
            GCU_CUDA(cudaMemcpyAsync(ks.meta.ptr, &capacity, sizeof(uint64_t), cudaMemcpyHostToDevice, dev.stream),
                     "copy");
            break;
    }
    uint64_t count = 0, bad = 0;
    uint32_t maxt = 0;
    GCU_TRY(ks.read_meta(dev, &count, &bad, &maxt));
    pts.reset();
    cell_keys.reset();
    cell_tmp.reset();
    cell_start.reset();
    const uint32_t id_bits = bit_length(n - 1);
    uint64_t *sorted = nullptr, *other = nullptr;
    GCU_TRY(sort_keys(dev, ks.keys.ptr, ks.tmp.ptr, count, id_bits, id_bits, &sorted, &other));
    GCU_TRY(csr_from_sorted_keys(dev, sorted, count, n, g));
    g.symmetric = 1;
    return ok();
}

Error generate_union(DeviceImpl& dev, const std::vector<GeneratorSpec>& specs, std::vector<uint32_t>* vbase,
                     GraphImpl& u) {
    vbase->assign(specs.size() + 1, 0);
    uint64_t vertices = 0, capacity = 0;
    for (size_t i = 0; i < specs.size(); ++i) {
        const GeneratorSpec& s = specs[i];
        uint64_t n = 0;
        if (s.kind == GeneratorSpec::kRmat) {
            if (s.scale == 0 || s.scale > 31) return export_error("R-MAT scale must be in 1..=31");
            n = 1ull << s.scale;
            capacity += 2 * (static_cast<uint64_t>(s.edge_factor) << s.scale);
        } else if (s.kind == GeneratorSpec::kWattsStrogatz) {
            if (s.k % 2 != 0) return export_error("Watts-Strogatz k must be even");
            n = s.n;
            capacity += 2 * n * (s.k / 2);
        } else {
            return kernel_error("a packed batch is generated from R-MAT and Watts-Strogatz graphs only");
        }
        (*vbase)[i] = static_cast<uint32_t>(vertices);
        vertices += n;
        if (vertices > 0xFFFFFFFEull) return export_error("packed batch has more than 2^32 - 2 vertices");
    }
    (*vbase)[specs.size()] = static_cast<uint32_t>(vertices);
    GCU_TRY(check_capacity(capacity));
    KeyScratch ks;
    GCU_TRY(ks.allocate(dev, capacity));
    for (size_t i = 0; i < specs.size(); ++i) {
        const GeneratorSpec& s = specs[i];
        const uint64_t state = host_mix(s.seed + kGamma);
        const uint32_t base = (*vbase)[i];
        if (s.kind == GeneratorSpec::kRmat) {
            const uint64_t m = static_cast<uint64_t>(s.edge_factor) << s.scale;
            GCU_LAUNCH(dev, "gen_rmat", rmat_keys_kernel, grid_for(dev, m), kBuildThreads, 0, state, s.scale, m, s.a,
                       s.a + s.b, s.a + s.b + s.c, ks.keys.ptr, ks.meta.ptr, base);
        } else if (s.n) {
            GCU_LAUNCH(dev, "gen_watts_strogatz", ws_keys_kernel, grid_for(dev, static_cast<uint64_t>(s.n) * (s.k / 2)),
                       kBuildThreads, 0, state, s.n, s.k / 2, s.p, ks.keys.ptr, ks.meta.ptr, base);
        }
    }
    uint64_t count = 0, bad = 0;
    uint32_t maxt = 0;
    GCU_TRY(ks.read_meta(dev, &count, &bad, &maxt));
    const uint32_t id_bits = bit_length(vertices > 0 ? vertices - 1 : 0);
    uint64_t *sorted = nullptr, *other = nullptr;
    GCU_TRY(sort_keys(dev, ks.keys.ptr, ks.tmp.ptr, count, id_bits, id_bits, &sorted, &other));
    GCU_TRY(csr_from_sorted_keys(dev, sorted, count, static_cast<uint32_t>(vertices), u));
    u.symmetric = 1;
    return ok();
}

}  // namespace gcu
