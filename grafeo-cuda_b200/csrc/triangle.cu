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
//     from_edge_pairs_oriented (csr_export.rs:319-329). A count pass, a device
//     scan and an order-preserving fill pass build the DAG CSR; self-loops
//     drop out because the order is strict. Max out-degree becomes O(sqrt m).
//     A CSR that is not symmetric is oriented by id alone (keep v > u): the
//     count below is then exactly the reference's formula, the sum over
//     entries u -> v, v > u, of |{w in N(u) ∩ N(v) : w > v}|
//     (triangle_counting.cu:246-315), whatever the input.
//  2. Counting: sum over DAG edges u -> v of |N+(u) ∩ N+(v)|, which counts
//     every triangle exactly once. Vertex-centric: a warp hashes N+(u) into
//     shared memory, then walks the wedges (v, w), v in N+(u), w in N+(v), 32 at
//     a time with the (v, w) pairs balanced over the lanes by a warp scan of
//     the d+(v), and probes each w in a shared-memory hash table of N+(u)
//     (wedge.cuh). Out-lists longer than 128 entries go to a CTA-per-vertex
//     kernel with a larger table (global binary search beyond 2048 entries).
//  All indices are 64-bit where they can exceed 2^32, so there is no cap on the
//  number of edges.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"
#include "wedge.cuh"

namespace gcu {


__device__ __forceinline__ bool dag_keep(uint32_t u, uint32_t du, uint32_t v, uint32_t dv, bool by_degree) {
    return by_degree ? (du < dv || (du == dv && u < v)) : u < v;
}

// Pass 1: out-degree of every vertex in the degree-oriented DAG.
__global__ void __launch_bounds__(256) tc_orient_count_kernel(const uint32_t* __restrict__ offsets,
                                                              const uint32_t* __restrict__ targets, uint32_t V,
                                                              bool by_degree, uint32_t* __restrict__ out_deg) {
    const unsigned lane = lane_id();
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < V; base += nwarps * 32) {
        const uint32_t count = static_cast<uint32_t>(min_u64(32, V - base));
        uint32_t s = 0, e = 0;
        if (lane < count) {
            s = offsets[base + lane];
            e = offsets[base + lane + 1];
        }
        uint32_t mine = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t u = static_cast<uint32_t>(base + i);
            const uint32_t start = __shfl_sync(kFullMask, s, i), end = __shfl_sync(kFullMask, e, i);
            const uint32_t du = end - start;
            uint32_t kept = 0;
            for (uint32_t j = start + lane; j < end; j += 32) {
                const uint32_t v = ld_stream(targets + j);
                const uint32_t dv = __ldg(offsets + v + 1) - __ldg(offsets + v);
                kept += dag_keep(u, du, v, dv, by_degree) ? 1u : 0u;
            }
            kept = warp_sum(kept);
            if (lane == i) mine = kept;
        }
        if (lane < count) out_deg[base + lane] = mine;
    }
}

// Pass 2: write the kept neighbours in list order (still sorted by id).
__global__ void __launch_bounds__(256) tc_orient_fill_kernel(const uint32_t* __restrict__ offsets,
                                                             const uint32_t* __restrict__ targets, uint32_t V,
                                                             bool by_degree, const uint32_t* __restrict__ dag_offsets,
                                                             uint32_t* __restrict__ dag_targets,
                                                             const uint32_t* __restrict__ rev,
                                                             uint32_t* __restrict__ dag_eid) {
    const unsigned lane = lane_id();
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < V; base += nwarps * 32) {
        const uint32_t count = static_cast<uint32_t>(min_u64(32, V - base));
        uint32_t s = 0, e = 0, o = 0;
        if (lane < count) {
            s = offsets[base + lane];
            e = offsets[base + lane + 1];
            o = dag_offsets[base + lane];
        }
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t u = static_cast<uint32_t>(base + i);
            const uint32_t start = __shfl_sync(kFullMask, s, i), end = __shfl_sync(kFullMask, e, i);
            uint32_t out = __shfl_sync(kFullMask, o, i);
            const uint32_t du = end - start;
            for (uint32_t j0 = start; j0 < end; j0 += 32) {
                const uint32_t j = j0 + lane;
                bool keep = false;
                uint32_t v = 0;
                if (j < end) {
                    v = ld_stream(targets + j);
                    const uint32_t dv = __ldg(offsets + v + 1) - __ldg(offsets + v);
                    keep = dag_keep(u, du, v, dv, by_degree);
                }
                const unsigned mask = __ballot_sync(kFullMask, keep);
                if (keep) {
                    const uint32_t at = out + __popc(mask & ((1u << lane) - 1));
                    dag_targets[at] = v;
                    // Undirected edge id: the CSR index of its u < v entry.
                    if (dag_eid) dag_eid[at] = u < v ? j : rev[j];
                }
                out += __popc(mask);
            }
        }
    }
}

// ---------------------------------------------------------------- host

namespace {

// Counts every triangle reported by the wedge kernels.
struct CountSink {
    static constexpr bool kNeedsPos = false;
    unsigned long long* total;
    unsigned long long count;
    __device__ __forceinline__ void hit(uint32_t, uint32_t, uint32_t, uint32_t) { ++count; }
    __device__ __forceinline__ void finish() {
        unsigned long long c = warp_sum(count);
        if (lane_id() == 0 && c) atomicAdd(total, c);
    }
};

}  // namespace

Error build_dag(GraphImpl& g, bool by_degree, const uint32_t* rev, DeviceBuffer<uint32_t>* dag_offsets,
                DeviceBuffer<uint32_t>* dag_targets, DeviceBuffer<uint32_t>* dag_eid, uint32_t* m) {
    DeviceImpl& dev = *g.dev;
    const uint32_t V = g.num_nodes;
    GCU_TRY(dag_offsets->allocate(dev, static_cast<uint64_t>(V) + 1));
    const unsigned grid = static_cast<unsigned>(
        std::min<uint64_t>(ceil_div_u64(ceil_div_u64(V, 32) * 32, 256), static_cast<uint64_t>(dev.sm_count) * 16));
    GCU_LAUNCH(dev, "tc_orient_count", tc_orient_count_kernel, grid, 256, 0, g.offsets.ptr, g.targets.ptr, V,
               by_degree, dag_offsets->ptr);
    GCU_TRY(exclusive_scan_u32(dev, dag_offsets->ptr, dag_offsets->ptr, V));
    *m = 0;
    GCU_CUDA(cudaMemcpyAsync(m, dag_offsets->ptr + V, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    GCU_TRY(dag_targets->allocate(dev, std::max<uint32_t>(*m, 1)));
    if (dag_eid) GCU_TRY(dag_eid->allocate(dev, std::max<uint32_t>(*m, 1)));
    if (*m == 0) return ok();
    GCU_LAUNCH(dev, "tc_orient_fill", tc_orient_fill_kernel, grid, 256, 0, g.offsets.ptr, g.targets.ptr, V, by_degree,
               dag_offsets->ptr, dag_targets->ptr, rev, dag_eid ? dag_eid->ptr : nullptr);
    return ok();
}

static Error count_dag(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, uint32_t V,
                       uint32_t min_deg, uint64_t* total) {
    DeviceBuffer<unsigned long long> d_total;
    GCU_TRY(d_total.allocate(dev, 1));
    GCU_CUDA(cudaMemsetAsync(d_total.ptr, 0, sizeof(unsigned long long), dev.stream), "memset");
    GCU_TRY(run_wedges(dev, d_offsets, d_targets, V, min_deg, CountSink{d_total.ptr, 0}, "tc"));
    unsigned long long host_total = 0;
    GCU_CUDA(cudaMemcpyAsync(&host_total, d_total.ptr, sizeof(host_total), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    GCU_TRY(dev.sync());
    *total = host_total;
    return ok();
}

Error triangle_count(GraphImpl& g, bool oriented, uint64_t* total) {
    *total = 0;
    // triangle_counting.rs:44-49: nothing to count.
    if (g.num_edges == 0) return ok();
    DeviceImpl& dev = *g.dev;
    const uint32_t V = g.num_nodes;
    if (oriented) {
        // The input is already a DAG: count over its lists as given; a
        // self-loop entry u -> u contributes |N(u)| like in the reference.
        return count_dag(dev, g.offsets.ptr, g.targets.ptr, V, 1, total);
    }
    bool symmetric = false;
    GCU_TRY(graph_symmetry(g, &symmetric));
    DeviceBuffer<uint32_t> dag_offsets, dag_targets;
    uint32_t m = 0;
    GCU_TRY(build_dag(g, symmetric, nullptr, &dag_offsets, &dag_targets, nullptr, &m));
    if (m == 0) return ok();
    // A DAG vertex needs two out-neighbours to close a triangle.
    return count_dag(dev, dag_offsets.ptr, dag_targets.ptr, V, 2, total);
}

}  // namespace gcu
