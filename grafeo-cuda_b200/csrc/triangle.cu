// Triangle counting over a degree-oriented DAG built on the device.
//
// Reference: crates/grafeo-cuda-algos/src/triangle_counting.rs:40-210 and
// kernels/triangle_counting.cu. The reference's default path maps one warp to
// each forward edge u < v, finds v by a linear walk of N(u) (a sum of d(u)^2
// over hubs), runs a single-thread prefix sum, and refuses graphs with more
// than 134,217,727 forward edges (launch.rs:27-35). Here:
//
//  1. Orientation: each undirected edge is kept once, from the endpoint of
//     lower (degree, id) to the higher one, the same rule as
//     from_edge_pairs_oriented (csr_export.rs:319-329). A flag pass over the
//     flat entry range, a device scan and an order-preserving scatter build
//     the DAG CSR; self-loops drop out because the order is strict. Max out-degree becomes O(sqrt m).
//     A CSR that is not symmetric is oriented by id alone (keep v > u): the
//     count below is then exactly the reference's formula, the sum over
//     entries u -> v, v > u, of |{w in N(u) ∩ N(v) : w > v}|
//     (triangle_counting.cu:246-315), whatever the input.
//  2. Counting: sum over DAG edges u -> v of |N+(u) ∩ N+(v)|, which counts
//     every triangle exactly once. Each edge streams the shorter of the two
//     lists against a shared-memory hash table of the longer one:
//     - tail side (d+(v) <= d+(u)): a warp or CTA hashes N+(u), then walks
//       the wedges (v, w), v in N+(u), w in N+(v), 32 at a time with the
//       (v, w) pairs balanced over the lanes by a warp scan of the d+(v), and
//       probes each w (wedge.cuh). Vertices are bucketed by ceil(log2 d+);
//       each bucket runs one of three variants (warp hash table up to 128
//       entries, CTA hash table up to 2048, CTA binary search beyond), by the
//       fixed degree ranges or by an installed learned schedule (sched.cuh).
//     - head side (2 <= d+(u) < d+(v)): the tails of such edges are gathered
//       into in-lists of their heads; a warp or CTA hashes N+(v) and streams
//       N+(u) for every tail u of a slice of v's in-list. On an R-MAT graph of
//       scale 22 this cuts the probes from 2.9e10 (all edges tail side) to
//       1.2e10.
//  All indices are 64-bit where they can exceed 2^32, so there is no cap on the
//  number of edges.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"
#include "sched.cuh"
#include "wedge.cuh"

namespace gcu {


__device__ __forceinline__ bool dag_keep(uint32_t u, uint32_t du, uint32_t v, uint32_t dv, bool by_degree) {
    return by_degree ? (du < dv || (du == dv && u < v)) : u < v;
}

// The orientation runs over the flat range of CSR entries, so a hub's list is
// shared by many blocks instead of walked by one warp:
//  1. keep[j] for every entry j = u -> v (tc_orient_flag_kernel): a block
//     takes a tile of consecutive entries, finds their rows with a binary
//     search of the row starts staged in shared memory, and evaluates the
//     orientation rule;
//  2. an exclusive scan of keep gives every kept entry its DAG position (the
//     DAG lists are the CSR lists filtered, in the same order);
//  3. the kept entries are scattered to their positions and every row's DAG
//     offset is the scan at the row's first CSR entry.
constexpr int kOrientThreads = 256;
constexpr int kOrientItems = 4;
constexpr int kOrientTile = kOrientThreads * kOrientItems;  // entries per tile

// With `rank`, u -> v is kept when v ranks below u (the orientation is that
// vertex order) and by_degree is ignored.
__global__ void __launch_bounds__(kOrientThreads) tc_orient_flag_kernel(const uint32_t* __restrict__ offsets,
                                                                        const uint32_t* __restrict__ targets,
                                                                        uint32_t V, uint32_t E, bool by_degree,
                                                                        const uint32_t* __restrict__ rank,
                                                                        uint32_t* __restrict__ keep) {
    __shared__ uint32_t s_start[kOrientTile];
    __shared__ uint32_t s_meta[2];
    for (uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kOrientTile; e0 < E;
         e0 += static_cast<uint64_t>(gridDim.x) * kOrientTile) {
        const uint64_t e1 = min_u64(e0 + kOrientTile, E);
        const bool staged = stage_tile_rows<kOrientTile>(offsets, V, e0, e1, s_start, s_meta);
        const uint32_t r0 = s_meta[0], nrows = s_meta[1] - r0 + 1;
#pragma unroll
        for (int q = 0; q < kOrientItems; ++q) {
            const uint64_t j = e0 + q * kOrientThreads + threadIdx.x;
            if (j >= e1) continue;
            const uint32_t u = tile_row(offsets, V, s_start, staged, r0, nrows, static_cast<uint32_t>(j));
            const uint32_t v = ld_stream(targets + j);
            if (rank) {
                keep[j] = __ldg(rank + v) < __ldg(rank + u) ? 1u : 0u;
            } else {
                const uint32_t du = __ldg(offsets + u + 1) - __ldg(offsets + u);
                const uint32_t dv = __ldg(offsets + v + 1) - __ldg(offsets + v);
                keep[j] = dag_keep(u, du, v, dv, by_degree) ? 1u : 0u;
            }
        }
        __syncthreads();  // the staged starts are rewritten for the next tile
    }
}

// Kept entries to their DAG positions; with dag_eid, also the CSR index of
// the edge's u < v entry (the undirected edge id); with dag_rank, the rank of
// each kept target.
__global__ void __launch_bounds__(kOrientThreads) tc_orient_fill_kernel(const uint32_t* __restrict__ offsets,
                                                                        const uint32_t* __restrict__ targets,
                                                                        uint32_t V, uint32_t E,
                                                                        const uint32_t* __restrict__ pos,
                                                                        uint32_t* __restrict__ dag_targets,
                                                                        const uint32_t* __restrict__ rev,
                                                                        uint32_t* __restrict__ dag_eid,
                                                                        const uint32_t* __restrict__ rank,
                                                                        uint32_t* __restrict__ dag_rank) {
    __shared__ uint32_t s_start[kOrientTile];
    __shared__ uint32_t s_meta[2];
    for (uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kOrientTile; e0 < E;
         e0 += static_cast<uint64_t>(gridDim.x) * kOrientTile) {
        const uint64_t e1 = min_u64(e0 + kOrientTile, E);
        const bool staged = dag_eid ? stage_tile_rows<kOrientTile>(offsets, V, e0, e1, s_start, s_meta) : false;
        const uint32_t r0 = dag_eid ? s_meta[0] : 0, nrows = dag_eid ? s_meta[1] - r0 + 1 : 0;
#pragma unroll
        for (int q = 0; q < kOrientItems; ++q) {
            const uint64_t j = e0 + q * kOrientThreads + threadIdx.x;
            if (j >= e1) continue;
            const uint32_t at = pos[j];
            if (pos[j + 1] == at) continue;
            const uint32_t v = ld_stream(targets + j);
            dag_targets[at] = v;
            if (dag_rank) dag_rank[at] = __ldg(rank + v);
            if (dag_eid) {
                const uint32_t u = tile_row(offsets, V, s_start, staged, r0, nrows, static_cast<uint32_t>(j));
                dag_eid[at] = u < v ? static_cast<uint32_t>(j) : rev[j];
            }
        }
        if (dag_eid) __syncthreads();
    }
}

// dag_offsets[u] = pos[offsets[u]] for u = 0..V.
__global__ void tc_orient_offsets_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                         const uint32_t* __restrict__ pos, uint32_t* __restrict__ dag_offsets) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u <= V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        dag_offsets[u] = pos[offsets[u]];
}

// ---------------------------------------------------------------- host

namespace {

// Counts every triangle reported by the wedge kernels.
struct CountSink {
    static constexpr bool kNeedsPos = false;
    unsigned long long* total;
    unsigned long long count;
    __device__ __forceinline__ void hit(uint32_t, uint32_t, uint32_t, uint32_t) { ++count; }
    __device__ __forceinline__ void end_vertex(uint32_t) {}
    __device__ __forceinline__ void finish() {
        unsigned long long c = warp_sum(count);
        if (lane_id() == 0 && c) atomicAdd(total, c);
    }
};

}  // namespace

// With `rank`: oriented by that vertex order, and dag_rank (when given) holds
// the rank of every DAG target.
static Error build_dag_impl(GraphImpl& g, bool by_degree, const uint32_t* rank, const uint32_t* rev,
                            DeviceBuffer<uint32_t>* dag_offsets, DeviceBuffer<uint32_t>* dag_targets,
                            DeviceBuffer<uint32_t>* dag_eid, DeviceBuffer<uint32_t>* dag_rank, uint32_t* m) {
    DeviceImpl& dev = *g.dev;
    const uint32_t V = g.num_nodes, E = g.num_edges;
    GCU_TRY(dag_offsets->allocate(dev, static_cast<uint64_t>(V) + 1));
    *m = 0;
    DeviceBuffer<uint32_t> pos;  // keep flags, then their exclusive scan (E + 1)
    GCU_TRY(pos.allocate(dev, static_cast<uint64_t>(E) + 1));
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned tiles = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(E, kOrientTile), cap)));
    const unsigned vgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(static_cast<uint64_t>(V) + 1, 256), cap));
    if (E > 0)
        GCU_LAUNCH(dev, "tc_orient_flag", tc_orient_flag_kernel, tiles, kOrientThreads, 0, g.offsets.ptr,
                   g.targets.ptr, V, E, by_degree, rank, pos.ptr);
    GCU_TRY(exclusive_scan_u32(dev, pos.ptr, pos.ptr, E));
    GCU_LAUNCH(dev, "tc_orient_offsets", tc_orient_offsets_kernel, vgrid, 256, 0, g.offsets.ptr, V, pos.ptr,
               dag_offsets->ptr);
    GCU_CUDA(cudaMemcpyAsync(m, pos.ptr + E, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    GCU_TRY(dag_targets->allocate(dev, std::max<uint32_t>(*m, 1)));
    if (dag_eid) GCU_TRY(dag_eid->allocate(dev, std::max<uint32_t>(*m, 1)));
    if (dag_rank) GCU_TRY(dag_rank->allocate(dev, std::max<uint32_t>(*m, 1)));
    if (*m == 0) return ok();
    GCU_LAUNCH(dev, "tc_orient_fill", tc_orient_fill_kernel, tiles, kOrientThreads, 0, g.offsets.ptr, g.targets.ptr,
               V, E, pos.ptr, dag_targets->ptr, rev, dag_eid ? dag_eid->ptr : nullptr, rank,
               dag_rank ? dag_rank->ptr : nullptr);
    GCU_TRY(dev.sync());  // pos is freed on return
    return ok();
}

Error build_dag(GraphImpl& g, bool by_degree, const uint32_t* rev, DeviceBuffer<uint32_t>* dag_offsets,
                DeviceBuffer<uint32_t>* dag_targets, DeviceBuffer<uint32_t>* dag_eid, uint32_t* m) {
    return build_dag_impl(g, by_degree, nullptr, rev, dag_offsets, dag_targets, dag_eid, nullptr, m);
}

// ---------------------------------------------------------------- out-degree buckets
//
// Vertices with d+ >= min_deg are grouped by c = ceil(log2 d+) (bucket c holds
// out-degrees in (2^(c-1), 2^c]); each bucket runs one intersection variant:
//   0  warp per vertex, shared hash table  (valid for d+ <= 128, c <= 7)
//   1  CTA per vertex, shared hash table   (valid for d+ <= 2048, c <= 11)
//   2  CTA per vertex, binary search of the out-list in global memory (any d+)
// The fixed rule takes the first valid one; an installed learned schedule
// takes the valid variant with the smallest predicted time. Buckets run from
// the highest out-degrees down.

constexpr int kBuckets = 33;

__device__ __forceinline__ int bucket_of(uint32_t d) { return d <= 1 ? 0 : 32 - __clz(d - 1); }
__host__ __device__ __forceinline__ unsigned bucket_valid(int c) { return c <= 7 ? 7u : (c <= 11 ? 6u : 4u); }
__host__ __device__ __forceinline__ int bucket_fixed(int c) { return c <= 7 ? 0 : (c <= 11 ? 1 : 2); }

__global__ void tc_bucket_count_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t min_deg,
                                       uint32_t* __restrict__ counts, unsigned long long* __restrict__ entries) {
    __shared__ uint32_t s_count[kBuckets];
    __shared__ unsigned long long s_entries[kBuckets];
    if (threadIdx.x < kBuckets) {
        s_count[threadIdx.x] = 0;
        s_entries[threadIdx.x] = 0;
    }
    __syncthreads();
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t d = offsets[u + 1] - offsets[u];
        if (d < min_deg || d == 0) continue;
        const int c = bucket_of(d);
        atomicAdd(&s_count[c], 1u);
        atomicAdd(&s_entries[c], static_cast<unsigned long long>(d));
    }
    __syncthreads();
    if (threadIdx.x < kBuckets && s_count[threadIdx.x]) {
        atomicAdd(counts + threadIdx.x, s_count[threadIdx.x]);
        atomicAdd(entries + threadIdx.x, s_entries[threadIdx.x]);
    }
}

// cursor[c] starts at bucket c's first list slot.
__global__ void tc_bucket_fill_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t min_deg,
                                      uint32_t* __restrict__ cursor, uint32_t* __restrict__ list) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t d = offsets[u + 1] - offsets[u];
        if (d < min_deg || d == 0) continue;
        list[atomicAdd(cursor + bucket_of(d), 1u)] = static_cast<uint32_t>(u);
    }
}

// One warp: features of every non-empty bucket (to features[c][12] when
// given) and, with a network, the chosen variant per bucket (-1: fixed rule).
__global__ void tc_decide_kernel(const __nv_bfloat16* __restrict__ w, const uint32_t* __restrict__ counts,
                                 const unsigned long long* __restrict__ entries, DegreeStats stats, float dag_edges,
                                 int* __restrict__ choices, float* __restrict__ features) {
    for (int c = 0; c < kBuckets; ++c) {
        if (lane_id() == 0) choices[c] = -1;
        if (counts[c] == 0) continue;
        const float hi = static_cast<float>(1ull << c), lo = c == 0 ? 1.f : static_cast<float>((1ull << (c - 1)) + 1);
        float f[kSchedIn];
        bucket_features(f, static_cast<float>(counts[c]), static_cast<float>(entries[c]), dag_edges, stats, lo, hi,
                        stats.num_nodes > 0.f ? dag_edges / stats.num_nodes : 0.f);
        if (features && lane_id() == 0)
            for (int k = 0; k < kSchedIn; ++k) features[c * kSchedIn + k] = f[k];
        if (w) {
            float out[kSchedOut];
            sched_forward_warp(w, f, out);
            if (lane_id() == 0) choices[c] = sched_pick_over(out, bucket_valid(c), bucket_fixed(c));
        }
    }
}

namespace {

struct BucketPlan {
    DeviceBuffer<uint32_t> list, counts, cursor;
    DeviceBuffer<unsigned long long> entries;
    DeviceBuffer<int> choices;
    DeviceBuffer<float> features;
    uint32_t host_counts[kBuckets] = {};
    uint32_t host_starts[kBuckets] = {};
    int host_choices[kBuckets] = {};
    float host_features[kBuckets * kSchedIn] = {};
};

// Buckets the vertices of a DAG and runs the decide kernel.
Error plan_buckets(DeviceImpl& dev, const uint32_t* d_offsets, uint32_t V, uint32_t min_deg, uint32_t m,
                   const DegreeStats& stats, bool want_features, BucketPlan& p) {
    GCU_TRY(p.counts.allocate(dev, kBuckets));
    GCU_TRY(p.cursor.allocate(dev, kBuckets));
    GCU_TRY(p.entries.allocate(dev, kBuckets));
    GCU_TRY(p.choices.allocate(dev, kBuckets));
    GCU_TRY(p.features.allocate(dev, kBuckets * kSchedIn));
    GCU_CUDA(cudaMemsetAsync(p.counts.ptr, 0, sizeof(uint32_t) * kBuckets, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(p.entries.ptr, 0, sizeof(unsigned long long) * kBuckets, dev.stream), "memset");
    const unsigned grid =
        static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(V, 256), dev.sm_count * 4ull)));
    GCU_LAUNCH(dev, "tc_bucket_count", tc_bucket_count_kernel, grid, 256, 0, d_offsets, V, min_deg, p.counts.ptr,
               p.entries.ptr);
    const __nv_bfloat16* net = reinterpret_cast<const __nv_bfloat16*>(dev.schedule);
    if (net || want_features) {
        GCU_LAUNCH(dev, "tc_decide", tc_decide_kernel, 1, 32, 0, net, p.counts.ptr, p.entries.ptr, stats,
                   static_cast<float>(m), p.choices.ptr, want_features ? p.features.ptr : nullptr);
        GCU_CUDA(cudaMemcpyAsync(p.host_choices, p.choices.ptr, sizeof(p.host_choices), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
    } else {
        std::fill(p.host_choices, p.host_choices + kBuckets, -1);
    }
    GCU_CUDA(cudaMemcpyAsync(p.host_counts, p.counts.ptr, sizeof(p.host_counts), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    if (want_features)
        GCU_CUDA(cudaMemcpyAsync(p.host_features, p.features.ptr, sizeof(p.host_features), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
    GCU_TRY(dev.sync());
    uint64_t total = 0;
    for (int c = 0; c < kBuckets; ++c) {
        p.host_starts[c] = static_cast<uint32_t>(total);
        total += p.host_counts[c];
    }
    GCU_TRY(p.list.allocate(dev, std::max<uint64_t>(total, 1)));
    GCU_CUDA(cudaMemcpyAsync(p.cursor.ptr, p.host_starts, sizeof(p.host_starts), cudaMemcpyHostToDevice, dev.stream),
             "copy");
    GCU_LAUNCH(dev, "tc_bucket_fill", tc_bucket_fill_kernel, grid, 256, 0, d_offsets, V, min_deg, p.cursor.ptr,
               p.list.ptr);
    return ok();
}

// One launch of `variant` over bucket c's vertices; next = its handout counter (zeroed).
// rank / vrank (a DAG oriented by a vertex order: the rank of every entry's
// target, of every vertex) let the CTA variants use rank bitmaps; nullptr
// for any other DAG.
template <class Sink>
Error launch_bucket(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, const BucketPlan& p, int c,
                    int variant, uint32_t* next, bool split, const uint32_t* rank, const uint32_t* vrank, Sink sink) {
    const uint32_t n = p.host_counts[c];
    const uint32_t* list = p.list.ptr + p.host_starts[c];
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 8;
    if (variant == 0) {
        const unsigned grid = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(n, kWedgeWarps * kVertexBatch), cap)));
        GCU_LAUNCH(dev, "wedge_warp_bucket", wedge_warp_list_kernel<Sink>, grid, kWedgeThreads, 0, d_offsets,
                   d_targets, list, n, next, split, sink);
    } else {
        const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(n, cap)));
        GCU_LAUNCH(dev, variant == 1 ? "wedge_cta_bucket" : "wedge_search_bucket", wedge_cta_list_kernel<Sink>, grid,
                   kWedgeThreads, 0, d_offsets, d_targets, list, n, next, variant == 2 ? 1 : 0, split, rank, vrank,
                   sink);
    }
    return ok();
}

// ---------------------------------------------------------------- head side

// For every DAG entry u -> v with 2 <= d+(u) < d+(v): counts it for v (pass
// without in_src) or places u in v's in-list (in_src given; counter zeroed).
__global__ void __launch_bounds__(kOrientThreads) tc_head_lists_kernel(const uint32_t* __restrict__ offsets,
                                                                       const uint32_t* __restrict__ targets,
                                                                       uint32_t V, uint32_t m,
                                                                       uint32_t* __restrict__ counter,
                                                                       const uint32_t* __restrict__ in_off,
                                                                       uint32_t* __restrict__ in_src) {
    for_each_entry<kOrientThreads, kOrientItems>(offsets, V, m, [&](uint32_t j, uint32_t u) {
        const uint32_t du = __ldg(offsets + u + 1) - __ldg(offsets + u);
        if (du < 2) return;
        const uint32_t v = ld_stream(targets + j);
        const uint32_t dv = __ldg(offsets + v + 1) - __ldg(offsets + v);
        if (du >= dv) return;
        const uint32_t k = atomicAdd(counter + v, 1u);
        if (in_src) in_src[in_off[v] + k] = u;
    });
}

// Items of a head with `tails` tails in out-degree bucket c: warp items for
// heads within a warp table, CTA items beyond.
__host__ __device__ __forceinline__ uint32_t head_slices(int c, uint32_t tails) {
    const uint32_t slice = bucket_fixed(c) == 0 ? kHeadWarpSlice : kHeadCtaSlice;
    return static_cast<uint32_t>((static_cast<uint64_t>(tails) + slice - 1) / slice);
}

// Items per out-degree bucket of the heads (counts[c]); with `items`, also
// writes every (v, slice) at cursor[c].
__global__ void tc_head_items_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ in_off,
                                     uint32_t V, uint32_t* __restrict__ counts, uint32_t* __restrict__ cursor,
                                     uint2* __restrict__ items) {
    __shared__ uint32_t s_count[kBuckets];
    if (!items && threadIdx.x < kBuckets) s_count[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t tails = in_off[v + 1] - in_off[v];
        if (tails == 0) continue;
        const int c = bucket_of(offsets[v + 1] - offsets[v]);
        const uint32_t n = head_slices(c, tails);
        if (!items) {
            atomicAdd(&s_count[c], n);
        } else {
            const uint32_t at = atomicAdd(cursor + c, n);
            for (uint32_t k = 0; k < n; ++k) items[at + k] = make_uint2(static_cast<uint32_t>(v), k);
        }
    }
    if (items) return;
    __syncthreads();
    if (threadIdx.x < kBuckets && s_count[threadIdx.x]) atomicAdd(counts + threadIdx.x, s_count[threadIdx.x]);
}

struct HeadPlan {
    DeviceBuffer<uint32_t> in_off, in_src, counter, counts;
    DeviceBuffer<uint2> items;
    uint32_t host_counts[kBuckets] = {};
    uint32_t host_starts[kBuckets] = {};
};

// In-lists of the head side and their (head, slice) items, bucketed by the
// head's out-degree.
Error plan_head(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, uint32_t V, uint32_t m,
                HeadPlan& h) {
    GCU_TRY(h.counter.allocate(dev, static_cast<uint64_t>(V) + 1));
    GCU_TRY(h.in_off.allocate(dev, static_cast<uint64_t>(V) + 1));
    GCU_TRY(h.counts.allocate(dev, kBuckets));
    GCU_CUDA(cudaMemsetAsync(h.counter.ptr, 0, sizeof(uint32_t) * (static_cast<uint64_t>(V) + 1), dev.stream),
             "memset");
    GCU_CUDA(cudaMemsetAsync(h.counts.ptr, 0, sizeof(uint32_t) * kBuckets, dev.stream), "memset");
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned tiles =
        static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(m, kOrientTile), cap)));
    const unsigned vgrid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(V, 256), cap)));
    GCU_LAUNCH(dev, "tc_head_count", tc_head_lists_kernel, tiles, kOrientThreads, 0, d_offsets, d_targets, V, m,
               h.counter.ptr, nullptr, nullptr);
    GCU_TRY(exclusive_scan_u32(dev, h.counter.ptr, h.in_off.ptr, V));
    GCU_LAUNCH(dev, "tc_head_items", tc_head_items_kernel, vgrid, 256, 0, d_offsets, h.in_off.ptr, V, h.counts.ptr,
               nullptr, nullptr);
    uint32_t tails = 0;
    GCU_CUDA(cudaMemcpyAsync(&tails, h.in_off.ptr + V, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_CUDA(cudaMemcpyAsync(h.host_counts, h.counts.ptr, sizeof(h.host_counts), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    GCU_TRY(dev.sync());
    if (tails == 0) return ok();
    // Buckets in descending order: the heaviest heads start first, and the
    // items of each variant (c >= 12, 8..11, <= 7) are contiguous.
    uint64_t total = 0;
    for (int c = kBuckets - 1; c >= 0; --c) {
        h.host_starts[c] = static_cast<uint32_t>(total);
        total += h.host_counts[c];
    }
    GCU_TRY(h.in_src.allocate(dev, tails));
    GCU_TRY(h.items.allocate(dev, std::max<uint64_t>(total, 1)));
    GCU_CUDA(cudaMemsetAsync(h.counter.ptr, 0, sizeof(uint32_t) * (static_cast<uint64_t>(V) + 1), dev.stream),
             "memset");
    GCU_LAUNCH(dev, "tc_head_fill", tc_head_lists_kernel, tiles, kOrientThreads, 0, d_offsets, d_targets, V, m,
               h.counter.ptr, h.in_off.ptr, h.in_src.ptr);
    // The counts buffer becomes the item cursors.
    GCU_CUDA(cudaMemcpyAsync(h.counts.ptr, h.host_starts, sizeof(h.host_starts), cudaMemcpyHostToDevice, dev.stream),
             "copy");
    GCU_LAUNCH(dev, "tc_head_items", tc_head_items_kernel, vgrid, 256, 0, d_offsets, h.in_off.ptr, V, nullptr,
               h.counts.ptr, h.items.ptr);
    return ok();
}

// Head-side items, one launch per variant over its contiguous buckets: CTA
// binary search for heads beyond 2048 out-edges, CTA tables down to 129,
// warp tables below.
template <class Sink>
Error launch_head(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, const HeadPlan& h,
                  uint32_t* next, const uint32_t* rank, const uint32_t* vrank, Sink sink) {
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 8;
    const int ranges[3][2] = {{kBuckets - 1, 12}, {11, 8}, {7, 0}};  // [hi, lo] buckets of variants 2, 1, 0
    for (int r = 0; r < 3; ++r) {
        const int hi = ranges[r][0], lo = ranges[r][1];
        uint32_t n = 0;
        for (int c = hi; c >= lo; --c) n += h.host_counts[c];
        if (n == 0) continue;
        const uint2* items = h.items.ptr + h.host_starts[hi];
        const int variant = bucket_fixed(lo);
        if (variant == 0) {
            const unsigned grid = static_cast<unsigned>(
                std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(n, kWedgeWarps * kVertexBatch), cap)));
            GCU_LAUNCH(dev, "wedge_head_warp", wedge_head_warp_kernel<Sink>, grid, kWedgeThreads, 0, d_offsets,
                       d_targets, items, n, h.in_off.ptr, h.in_src.ptr, next + r, sink);
        } else {
            const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(n, cap)));
            GCU_LAUNCH(dev, "wedge_head_cta", wedge_head_cta_kernel<Sink>, grid, kWedgeThreads, 0, d_offsets,
                       d_targets, items, n, h.in_off.ptr, h.in_src.ptr, next + r, variant == 2 ? 1 : 0, rank, vrank,
                       sink);
        }
    }
    return ok();
}

// Sum over DAG edges u -> v of |N+(u) ∩ N+(v)| for vertices with at least
// min_deg out-edges. With `trace`, every valid variant of every bucket runs
// (each into its own counter), is timed, and all must agree.
Error count_dag(GraphImpl& g, const uint32_t* d_offsets, const uint32_t* d_targets, const uint32_t* d_rank,
                const uint32_t* d_vrank, uint32_t m, uint32_t min_deg, uint64_t* total,
                std::vector<TcTraceBucket>* trace) {
    DeviceImpl& dev = *g.dev;
    const uint32_t V = g.num_nodes;
    DegreeStats stats;
    if (dev.schedule || trace) GCU_TRY(degree_stats(g, &stats));
    BucketPlan p;
    GCU_TRY(plan_buckets(dev, d_offsets, V, min_deg, m, stats, trace != nullptr, p));
    HeadPlan head;
    GCU_TRY(plan_head(dev, d_offsets, d_targets, V, m, head));
    const int runs = trace ? kSchedOut : 1;
    // [bucket][variant] with trace, else [0]; then the head side's total
    // (slot kBuckets * runs with trace, else [0] too) and handout counters.
    const int head_slot = trace ? kBuckets * runs : 0;
    const int slots = kBuckets * runs + 1 + kBuckets;
    DeviceBuffer<unsigned long long> totals;
    DeviceBuffer<uint32_t> next;
    GCU_TRY(totals.allocate(dev, slots));
    GCU_TRY(next.allocate(dev, slots));
    GCU_CUDA(cudaMemsetAsync(totals.ptr, 0, sizeof(unsigned long long) * slots, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(next.ptr, 0, sizeof(uint32_t) * slots, dev.stream), "memset");
    std::vector<cudaEvent_t> ev;
    struct Events {
        std::vector<cudaEvent_t>& e;
        ~Events() {
            for (auto x : e) cudaEventDestroy(x);
        }
    } guard{ev};
    if (trace) {
        ev.resize(2 * kBuckets * kSchedOut);
        for (auto& e : ev) GCU_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    }
    for (int c = kBuckets - 1; c >= 0; --c) {
        if (p.host_counts[c] == 0) continue;
        const unsigned valid = bucket_valid(c);
        if (!trace) {
            int variant = bucket_fixed(c);
            const int pick = p.host_choices[c];
            if (pick >= 0 && ((valid >> pick) & 1u)) variant = pick;
            GCU_TRY(launch_bucket(dev, d_offsets, d_targets, p, c, variant, next.ptr + c, true, d_rank, d_vrank,
                                  CountSink{totals.ptr, 0}));
            continue;
        }
        for (int v = 0; v < kSchedOut; ++v) {
            if (!((valid >> v) & 1u)) continue;
            const int slot = c * kSchedOut + v;
            GCU_CUDA(cudaEventRecord(ev[2 * slot], dev.stream), "cudaEventRecord");
            GCU_TRY(launch_bucket(dev, d_offsets, d_targets, p, c, v, next.ptr + slot, true, d_rank, d_vrank,
                                  CountSink{totals.ptr + slot, 0}));
            GCU_CUDA(cudaEventRecord(ev[2 * slot + 1], dev.stream), "cudaEventRecord");
        }
    }
    GCU_TRY(launch_head(dev, d_offsets, d_targets, head, next.ptr + kBuckets * runs + 1, d_rank, d_vrank,
                        CountSink{totals.ptr + head_slot, 0}));
    std::vector<unsigned long long> host(kBuckets * runs + 1);
    GCU_CUDA(cudaMemcpyAsync(host.data(), totals.ptr, sizeof(unsigned long long) * host.size(), cudaMemcpyDeviceToHost,
                             dev.stream),
             "copy");
    GCU_TRY(dev.sync());
    if (!trace) {
        *total = host[0];
        return ok();
    }
    uint64_t sum = host[head_slot];
    trace->clear();
    for (int c = kBuckets - 1; c >= 0; --c) {
        if (p.host_counts[c] == 0) continue;
        TcTraceBucket rec{};
        std::copy(p.host_features + c * kSchedIn, p.host_features + (c + 1) * kSchedIn, rec.features);
        rec.valid = static_cast<uint8_t>(bucket_valid(c));
        rec.fixed_rule = static_cast<uint8_t>(bucket_fixed(c));
        const unsigned long long expect = host[c * kSchedOut + bucket_fixed(c)];
        for (int v = 0; v < kSchedOut; ++v) {
            rec.times_us[v] = __builtin_nanf("");
            if (!((rec.valid >> v) & 1u)) continue;
            const int slot = c * kSchedOut + v;
            if (host[slot] != expect)
                return kernel_error("intersection variants disagree on out-degree bucket " + std::to_string(c));
            float ms = 0.f;
            GCU_CUDA(cudaEventElapsedTime(&ms, ev[2 * slot], ev[2 * slot + 1]), "cudaEventElapsedTime");
            rec.times_us[v] = 1000.f * ms;
        }
        sum += expect;
        trace->push_back(rec);
    }
    *total = sum;
    return ok();
}

Error triangle_count_ex(GraphImpl& g, bool oriented, uint64_t* total, std::vector<TcTraceBucket>* trace) {
    *total = 0;
    if (trace) trace->clear();
    // triangle_counting.rs:44-49: nothing to count.
    if (g.num_edges == 0) return ok();
    if (oriented) {
        // The input is already a DAG: count over its lists as given; a
        // self-loop entry u -> u contributes |N(u)| like in the reference.
        return count_dag(g, g.offsets.ptr, g.targets.ptr, nullptr, nullptr, g.num_edges, 1, total, trace);
    }
    bool symmetric = false;
    GCU_TRY(graph_symmetry(g, &symmetric));
    DeviceBuffer<uint32_t> dag_offsets, dag_targets, rank, dag_rank;
    uint32_t m = 0;
    if (symmetric) {
        // Oriented toward the higher degree class (ties by id): every
        // out-neighbour ranks below its owner, so an owner's table can be a
        // bitmap of the ranks below its own.
        GCU_TRY(degree_class_order(*g.dev, g.offsets.ptr, g.num_nodes, &rank));
        GCU_TRY(build_dag_impl(g, true, rank.ptr, nullptr, &dag_offsets, &dag_targets, nullptr, &dag_rank, &m));
    } else {
        GCU_TRY(build_dag(g, false, nullptr, &dag_offsets, &dag_targets, nullptr, &m));
    }
    if (m == 0) return ok();
    // A DAG vertex needs two out-neighbours to close a triangle.
    return count_dag(g, dag_offsets.ptr, dag_targets.ptr, symmetric ? dag_rank.ptr : nullptr,
                     symmetric ? rank.ptr : nullptr, m, 2, total, trace);
}

}  // namespace

Error triangle_count(GraphImpl& g, bool oriented, uint64_t* total) {
    return triangle_count_ex(g, oriented, total, nullptr);
}

Error triangle_trace(GraphImpl& g, std::vector<TcTraceBucket>* buckets, uint64_t* total) {
    return triangle_count_ex(g, false, total, buckets);
}

// ---------------------------------------------------------------- batched form

namespace {

// Triangles per DAG source vertex: each warp adds its lanes' count for u.
struct VertexCountSink {
    static constexpr bool kNeedsPos = false;
    unsigned long long* per_vertex;
    unsigned long long count;
    __device__ __forceinline__ void hit(uint32_t, uint32_t, uint32_t, uint32_t) { ++count; }
    __device__ __forceinline__ void end_vertex(uint32_t u) {
        const unsigned long long c = warp_sum(count);
        if (lane_id() == 0 && c) atomicAdd(per_vertex + u, c);
        count = 0;
    }
    __device__ __forceinline__ void finish() {}
};

}  // namespace

struct BatchTcPlan {
    DeviceBuffer<uint32_t> dag_offsets, dag_targets;
    uint32_t m = 0;
    BucketPlan buckets;
    int variant[kBuckets] = {};
    DeviceBuffer<uint32_t> next;  // handout counter per bucket
};

void destroy_batch_tc_plan(BatchTcPlan* p) { delete p; }

Error batch_tc_plan(GraphImpl& u, BatchTcPlan** out, std::string* tuning) {
    DeviceImpl& dev = *u.dev;
    auto p = std::make_unique<BatchTcPlan>();
    GCU_TRY(build_dag(u, true, nullptr, &p->dag_offsets, &p->dag_targets, nullptr, &p->m));
    DegreeStats stats;
    if (dev.schedule) GCU_TRY(degree_stats(u, &stats));
    GCU_TRY(plan_buckets(dev, p->dag_offsets.ptr, u.num_nodes, 2, p->m, stats, false, p->buckets));
    GCU_TRY(p->next.allocate(dev, kBuckets * kSchedOut));
    // Variant per bucket: the learned schedule's pick when one is installed,
    // else the fastest valid variant timed once on this batch (autotune).
    DeviceBuffer<unsigned long long> scratch;
    GCU_TRY(scratch.allocate(dev, std::max<uint32_t>(u.num_nodes, 1)));
    GCU_CUDA(cudaMemsetAsync(p->next.ptr, 0, sizeof(uint32_t) * kBuckets * kSchedOut, dev.stream), "memset");
    cudaEvent_t ev[2 * kSchedOut];
    for (auto& e : ev) GCU_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    struct Guard {
        cudaEvent_t* e;
        ~Guard() {
            for (int i = 0; i < 2 * kSchedOut; ++i) cudaEventDestroy(e[i]);
        }
    } guard{ev};
    std::string json = "{";
    for (int c = kBuckets - 1; c >= 0; --c) {
        if (p->buckets.host_counts[c] == 0) continue;
        const unsigned valid = bucket_valid(c);
        int pick = bucket_fixed(c);
        float best = 0.f;
        const int learned = p->buckets.host_choices[c];
        std::string how;
        if (learned >= 0 && ((valid >> learned) & 1u)) {
            pick = learned;
            how = "learned";
        } else {
            bool first = true;
            for (int v = 0; v < kSchedOut; ++v) {
                if (!((valid >> v) & 1u)) continue;
                GCU_CUDA(cudaEventRecord(ev[2 * v], dev.stream), "cudaEventRecord");
                GCU_TRY(launch_bucket(dev, p->dag_offsets.ptr, p->dag_targets.ptr, p->buckets, c, v,
                                      p->next.ptr + c * kSchedOut + v, false, nullptr, nullptr,
                                      VertexCountSink{scratch.ptr, 0}));
                GCU_CUDA(cudaEventRecord(ev[2 * v + 1], dev.stream), "cudaEventRecord");
            }
            GCU_TRY(dev.sync());
            for (int v = 0; v < kSchedOut; ++v) {
                if (!((valid >> v) & 1u)) continue;
                float ms = 0.f;
                GCU_CUDA(cudaEventElapsedTime(&ms, ev[2 * v], ev[2 * v + 1]), "cudaEventElapsedTime");
                if (first || ms < best) {
                    best = ms;
                    pick = v;
                    first = false;
                }
            }
            how = "timed";
        }
        p->variant[c] = pick;
        if (json.size() > 1) json += ", ";
        json += "\"" + std::to_string(c) + "\": {\"vertices\": " + std::to_string(p->buckets.host_counts[c]) +
                ", \"variant\": " + std::to_string(pick) + ", \"by\": \"" + how + "\"}";
    }
    json += "}";
    if (tuning) *tuning = json;
    GCU_TRY(dev.sync());
    *out = p.release();
    return ok();
}

Error batch_tc_launch(DeviceImpl& dev, BatchTcPlan& p, unsigned long long* per_vertex, uint32_t num_nodes) {
    GCU_CUDA(cudaMemsetAsync(per_vertex, 0, sizeof(unsigned long long) * std::max<uint32_t>(num_nodes, 1), dev.stream),
             "memset");
    GCU_CUDA(cudaMemsetAsync(p.next.ptr, 0, sizeof(uint32_t) * kBuckets, dev.stream), "memset");
    for (int c = kBuckets - 1; c >= 0; --c) {
        if (p.buckets.host_counts[c] == 0) continue;
        GCU_TRY(launch_bucket(dev, p.dag_offsets.ptr, p.dag_targets.ptr, p.buckets, c, p.variant[c], p.next.ptr + c,
                              false, nullptr, nullptr, VertexCountSink{per_vertex, 0}));
    }
    return ok();
}

}  // namespace gcu
