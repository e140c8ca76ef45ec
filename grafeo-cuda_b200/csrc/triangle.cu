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
//     every triangle exactly once. Vertex-centric: a warp stages N+(u) in
//     shared memory, then walks the wedges (v, w), v in N+(u), w in N+(v), 32 at
//     a time with the (v, w) pairs balanced over the lanes by a warp scan of
//     the d+(v), and binary-searches each w in the staged list. Vertices whose
//     lists do not fit a warp's slice go to a CTA-per-vertex kernel with a
//     larger shared-memory stage (global binary search beyond that).
//  All indices are 64-bit where they can exceed 2^32, so there is no cap on the
//  number of edges.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kTcThreads = 256;
constexpr int kTcWarps = kTcThreads / 32;
constexpr uint32_t kTcWarpCap = 256;     // list entries staged per warp
constexpr uint32_t kTcBatch = 8;         // vertices fetched per warp at a time
constexpr uint32_t kTcBlockCapMax = 48 * 1024;  // entries staged per CTA for hubs (192 KB)

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
                                                             uint32_t* __restrict__ dag_targets) {
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
                if (keep) dag_targets[out + __popc(mask & ((1u << lane) - 1))] = v;
                out += __popc(mask);
            }
        }
    }
}

// Binary search for w in the sorted list a[0, n).
__device__ __forceinline__ bool contains_sorted(const uint32_t* a, uint32_t n, uint32_t w) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t x = a[mid];
        if (x < w)
            lo = mid + 1;
        else if (x > w)
            hi = mid;
        else
            return true;
    }
    return false;
}

// Wedges (v, w) of one chunk of up to 32 out-neighbours v of u, balanced over
// the lanes; each w is searched in list[0, du). Returns this lane's hits.
__device__ __forceinline__ uint32_t tc_chunk(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                             const uint32_t* list, uint32_t du, uint32_t c, uint32_t* s_excl,
                                             uint32_t* s_start) {
    const unsigned lane = lane_id();
    uint32_t vs = 0, dv = 0;
    if (c + lane < du) {
        const uint32_t v = list[c + lane];
        vs = offsets[v];
        dv = offsets[v + 1] - vs;
    }
    const uint32_t inc = warp_inclusive_scan(dv);
    const uint32_t total = __shfl_sync(kFullMask, inc, 31);
    __syncwarp();
    s_excl[lane] = inc - dv;
    s_start[lane] = vs;
    __syncwarp();
    uint32_t hits = 0;
    for (uint32_t k = lane; k < total; k += 32) {
        uint32_t lo = 0, hi = 32;  // largest j with s_excl[j] <= k
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (s_excl[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        const uint32_t w = targets[s_start[lo] + (k - s_excl[lo])];
        hits += contains_sorted(list, du, w) ? 1u : 0u;
    }
    return hits;
}

// Warp per vertex for lists of [min_deg, kTcWarpCap] entries; vertices are
// handed out dynamically kTcBatch at a time.
__global__ void __launch_bounds__(kTcThreads) tc_count_warp_kernel(const uint32_t* __restrict__ offsets,
                                                                   const uint32_t* __restrict__ targets, uint32_t V,
                                                                   uint32_t min_deg, uint32_t* __restrict__ next_vertex,
                                                                   unsigned long long* __restrict__ total) {
    __shared__ uint32_t s_list[kTcWarps][kTcWarpCap];
    __shared__ uint32_t s_excl[kTcWarps][32];
    __shared__ uint32_t s_start[kTcWarps][32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    unsigned long long count = 0;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next_vertex, kTcBatch);
        base = __shfl_sync(kFullMask, base, 0);
        if (base >= V) break;
        const uint32_t last = min(base + kTcBatch, V);
        for (uint32_t u = base; u < last; ++u) {
            const uint32_t s = offsets[u], e = offsets[u + 1], du = e - s;
            if (du < min_deg || du > kTcWarpCap) continue;
            __syncwarp();
            for (uint32_t k = lane; k < du; k += 32) s_list[warp][k] = targets[s + k];
            __syncwarp();
            for (uint32_t c = 0; c < du; c += 32)
                count += tc_chunk(offsets, targets, s_list[warp], du, c, s_excl[warp], s_start[warp]);
        }
    }
    count = warp_sum(count);
    if (lane == 0 && count) atomicAdd(total, count);
}

// Lists longer than kTcWarpCap: collect them for the CTA kernel.
__global__ void tc_collect_hubs_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t* __restrict__ hubs,
                                       uint32_t* __restrict__ hub_count) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (offsets[u + 1] - offsets[u] > kTcWarpCap) hubs[atomicAdd(hub_count, 1u)] = static_cast<uint32_t>(u);
    }
}

// CTA per hub vertex: its list is staged in dynamic shared memory when it fits
// (stage_cap entries), otherwise searched in place in global memory.
__global__ void __launch_bounds__(kTcThreads) tc_count_hub_kernel(const uint32_t* __restrict__ offsets,
                                                                  const uint32_t* __restrict__ targets,
                                                                  const uint32_t* __restrict__ hubs,
                                                                  const uint32_t* __restrict__ hub_count,
                                                                  uint32_t stage_cap,
                                                                  unsigned long long* __restrict__ total) {
    extern __shared__ uint32_t s_stage[];
    __shared__ uint32_t s_excl[kTcWarps][32];
    __shared__ uint32_t s_start[kTcWarps][32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t nhubs = *hub_count;
    unsigned long long count = 0;
    for (uint32_t h = blockIdx.x; h < nhubs; h += gridDim.x) {
        const uint32_t u = hubs[h];
        const uint32_t s = offsets[u], e = offsets[u + 1], du = e - s;
        const uint32_t* list = targets + s;
        __syncthreads();
        if (du <= stage_cap) {
            for (uint32_t k = threadIdx.x; k < du; k += blockDim.x) s_stage[k] = targets[s + k];
            list = s_stage;
        }
        __syncthreads();
        for (uint32_t c = warp * 32; c < du; c += kTcThreads)
            count += tc_chunk(offsets, targets, list, du, c, s_excl[warp], s_start[warp]);
    }
    count = warp_sum(count);
    if (lane == 0 && count) atomicAdd(total, count);
}

// ---------------------------------------------------------------- host

static Error count_dag(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, uint32_t V,
                       uint32_t min_deg, uint64_t* total) {
    // scratch: [0] next vertex, [1] hub count, [2..3] u64 total, then the hub list
    DeviceBuffer<uint32_t> scratch;
    GCU_TRY(scratch.allocate(dev, 4 + static_cast<uint64_t>(V)));
    GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, 4 * sizeof(uint32_t), dev.stream), "memset");
    uint32_t* next_vertex = scratch.ptr;
    uint32_t* hub_count = scratch.ptr + 1;
    auto* d_total = reinterpret_cast<unsigned long long*>(scratch.ptr + 2);
    uint32_t* hubs = scratch.ptr + 4;

    const unsigned grid = static_cast<unsigned>(dev.sm_count) * 8;
    GCU_LAUNCH(dev, "tc_count_warp", tc_count_warp_kernel, grid, kTcThreads, 0, d_offsets, d_targets, V, min_deg,
               next_vertex, d_total);
    const unsigned collect_blocks =
        static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), static_cast<uint64_t>(dev.sm_count) * 8));
    GCU_LAUNCH(dev, "tc_collect_hubs", tc_collect_hubs_kernel, collect_blocks, 256, 0, d_offsets, V, hubs, hub_count);
    const size_t static_smem = 2 * kTcWarps * 32 * sizeof(uint32_t);
    size_t avail = dev.max_smem_optin > 0 ? static_cast<size_t>(dev.max_smem_optin) : 48 * 1024;
    uint32_t stage_cap = static_cast<uint32_t>(std::min<size_t>((avail - static_smem) / 4, kTcBlockCapMax));
    size_t dyn = static_cast<size_t>(stage_cap) * 4;
    GCU_CUDA(cudaFuncSetAttribute(tc_count_hub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dyn)),
             "cudaFuncSetAttribute");
    GCU_LAUNCH(dev, "tc_count_hub", tc_count_hub_kernel, static_cast<unsigned>(dev.sm_count), kTcThreads, dyn,
               d_offsets, d_targets, hubs, hub_count, stage_cap, d_total);
    unsigned long long host_total = 0;
    GCU_CUDA(cudaMemcpyAsync(&host_total, d_total, sizeof(host_total), cudaMemcpyDeviceToHost, dev.stream), "copy");
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
    GCU_TRY(dag_offsets.allocate(dev, static_cast<uint64_t>(V) + 1));
    const unsigned grid = static_cast<unsigned>(
        std::min<uint64_t>(ceil_div_u64(ceil_div_u64(V, 32) * 32, 256), static_cast<uint64_t>(dev.sm_count) * 16));
    GCU_LAUNCH(dev, "tc_orient_count", tc_orient_count_kernel, grid, 256, 0, g.offsets.ptr, g.targets.ptr, V,
               symmetric, dag_offsets.ptr);
    GCU_TRY(exclusive_scan_u32(dev, dag_offsets.ptr, dag_offsets.ptr, V));
    uint32_t m = 0;
    GCU_CUDA(cudaMemcpyAsync(&m, dag_offsets.ptr + V, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    if (m == 0) return ok();
    GCU_TRY(dag_targets.allocate(dev, m));
    GCU_LAUNCH(dev, "tc_orient_fill", tc_orient_fill_kernel, grid, 256, 0, g.offsets.ptr, g.targets.ptr, V,
               symmetric, dag_offsets.ptr, dag_targets.ptr);
    // A DAG vertex needs two out-neighbours to close a triangle.
    return count_dag(dev, dag_offsets.ptr, dag_targets.ptr, V, 2, total);
}

}  // namespace gcu
