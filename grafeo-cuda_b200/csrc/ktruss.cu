// k-truss by synchronous peeling.
//
// Reference: crates/grafeo-cuda-algos/src/k_truss.rs:42-161 and
// kernels/k_truss.cu:46-124. Each round computes, for every live CSR entry
// u -> v with v > u, support = |live N(u) ∩ live N(v)| (entry-level liveness, so
// in the first round a live self-loop at u or v counts as a common neighbour
// exactly as in the reference's merge), copies it to the live reverse entry
// v -> u, and then removes every live entry whose support is below k - 2. The
// rounds repeat until one removes nothing; the number of rounds is the
// reference's `iterations`. Since every round sees the same live set as the
// reference's round, removed sets and round counts are identical.
//
// Differences from the reference's kernels, same results:
//  * a warp per entry intersects the two lists by walking the shorter one and
//    binary-searching the longer (the reference merges both lists in one
//    thread, per node);
//  * the reverse entry comes from a precomputed index (the reference scans
//    N(v) linearly for it every round);
//  * the source vertex of every entry is materialised once (COO row array);
//  * the result edge list is compacted on the device in CSR order (the
//    reference copies removed/offsets/targets back and loops on the host).
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// src[j] = row of entry j (a warp per 32 rows, coalesced writes).
__global__ void __launch_bounds__(256) kt_rows_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                                      uint32_t* __restrict__ src) {
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
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t start = __shfl_sync(kFullMask, s, i), end = __shfl_sync(kFullMask, e, i);
            for (uint32_t j = start + lane; j < end; j += 32) src[j] = static_cast<uint32_t>(base + i);
        }
    }
}

// rev[j] = index of entry v -> u for entry j = u -> v, or kNone.
__global__ void kt_reverse_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                  const uint32_t* __restrict__ src, uint32_t E, uint32_t* __restrict__ rev) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[j], v = targets[j];
        const uint32_t s = offsets[v], e = offsets[v + 1];
        const uint32_t p = lower_bound_u32(targets, s, e, u);
        rev[j] = (p < e && targets[p] == u) ? p : kNone;
    }
}

// One warp per live entry u -> v with v > u (32 candidate entries per step).
__global__ void __launch_bounds__(256) kt_support_kernel(const uint32_t* __restrict__ offsets,
                                                         const uint32_t* __restrict__ targets,
                                                         const uint32_t* __restrict__ src,
                                                         const uint32_t* __restrict__ rev,
                                                         const uint8_t* __restrict__ live, uint32_t E,
                                                         uint32_t* __restrict__ support) {
    const unsigned lane = lane_id();
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < E; base += nwarps * 32) {
        const uint64_t j = base + lane;
        uint32_t u = 0, v = 0;
        bool todo = false;
        if (j < E && live[j]) {
            u = src[j];
            v = targets[j];
            todo = v > u;
        }
        unsigned pending = __ballot_sync(kFullMask, todo);
        while (pending) {
            const int l = __ffs(pending) - 1;
            pending &= pending - 1;
            const uint32_t eu = __shfl_sync(kFullMask, u, l), ev = __shfl_sync(kFullMask, v, l);
            uint32_t as = offsets[eu], ae = offsets[eu + 1], bs = offsets[ev], be = offsets[ev + 1];
            if (ae - as > be - bs) {
                uint32_t t = as; as = bs; bs = t;
                t = ae; ae = be; be = t;
            }
            uint32_t hits = 0;
            for (uint32_t i = as + lane; i < ae; i += 32) {
                if (!live[i]) continue;
                const uint32_t x = targets[i];
                const uint32_t p = lower_bound_u32(targets, bs, be, x);
                if (p < be && targets[p] == x && live[p]) ++hits;
            }
            hits = warp_sum(hits);
            if (lane == 0) {
                const uint64_t ej = base + l;
                support[ej] = hits;
                const uint32_t r = rev[ej];
                if (r != kNone && live[r]) support[r] = hits;
            }
        }
    }
}

__global__ void kt_filter_kernel(const uint32_t* __restrict__ support, uint8_t* __restrict__ live, uint32_t E,
                                 uint32_t threshold, uint32_t* __restrict__ removed) {
    uint32_t mine = 0;
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (live[j] && support[j] < threshold) {
            live[j] = 0;
            ++mine;
        }
    }
    mine = warp_sum(mine);
    if (lane_id() == 0 && mine) atomicAdd(removed, mine);
}

__global__ void kt_flag_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src,
                               const uint8_t* __restrict__ live, uint32_t E, uint32_t* __restrict__ flag) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        flag[j] = (live[j] && targets[j] > src[j]) ? 1u : 0u;
    }
}

__global__ void kt_emit_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src,
                               const uint8_t* __restrict__ live, uint32_t E, const uint32_t* __restrict__ pos,
                               uint2* __restrict__ out) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[j], v = targets[j];
        if (live[j] && v > u) out[pos[j]] = make_uint2(u, v);
    }
}

Error k_truss(GraphImpl& g, uint32_t k, std::vector<uint32_t>* edges, uint32_t* iterations) {
    edges->clear();
    *iterations = 0;
    const uint32_t E = g.num_edges, V = g.num_nodes;
    // k_truss.rs:53-60: no edges, no truss.
    if (E == 0) return ok();
    DeviceImpl& dev = *g.dev;
    const uint32_t threshold = k - 2;
    DeviceBuffer<uint32_t> src, rev, support, scratch;
    DeviceBuffer<uint8_t> live;
    GCU_TRY(src.allocate(dev, E));
    GCU_TRY(rev.allocate(dev, static_cast<uint64_t>(E) + 1));  // + 1: reused as scan output
    GCU_TRY(support.allocate(dev, E));
    GCU_TRY(live.allocate(dev, E));
    GCU_TRY(scratch.allocate(dev, 2));
    uint32_t* host = nullptr;
    GCU_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host), sizeof(uint32_t)), "cudaMallocHost");
    struct HostFree {
        uint32_t* p;
        ~HostFree() { cudaFreeHost(p); }
    } host_guard{host};

    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned row_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), cap));
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    GCU_LAUNCH(dev, "kt_rows", kt_rows_kernel, row_grid, 256, 0, g.offsets.ptr, V, src.ptr);
    GCU_LAUNCH(dev, "kt_reverse", kt_reverse_kernel, edge_grid, 256, 0, g.offsets.ptr, g.targets.ptr, src.ptr, E,
               rev.ptr);
    GCU_CUDA(cudaMemsetAsync(live.ptr, 1, E, dev.stream), "memset");

    uint32_t rounds = 0;
    while (true) {
        GCU_CUDA(cudaMemsetAsync(support.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
        GCU_LAUNCH(dev, "kt_support", kt_support_kernel, edge_grid, 256, 0, g.offsets.ptr, g.targets.ptr, src.ptr,
                   rev.ptr, live.ptr, E, support.ptr);
        GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
        GCU_LAUNCH(dev, "kt_filter", kt_filter_kernel, edge_grid, 256, 0, support.ptr, live.ptr, E, threshold,
                   scratch.ptr);
        GCU_CUDA(cudaMemcpyAsync(host, scratch.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        rounds += 1;
        if (*host == 0) break;
    }

    // Compact the surviving u < v entries in CSR order.
    GCU_LAUNCH(dev, "kt_flag", kt_flag_kernel, edge_grid, 256, 0, g.targets.ptr, src.ptr, live.ptr, E, support.ptr);
    GCU_TRY(exclusive_scan_u32(dev, support.ptr, rev.ptr, E));  // rev is free now
    uint32_t count = 0;
    GCU_CUDA(cudaMemcpyAsync(&count, rev.ptr + E, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    if (count > 0) {
        DeviceBuffer<uint2> out;
        GCU_TRY(out.allocate(dev, count));
        GCU_LAUNCH(dev, "kt_emit", kt_emit_kernel, edge_grid, 256, 0, g.targets.ptr, src.ptr, live.ptr, E, rev.ptr,
                   out.ptr);
        edges->resize(2 * static_cast<size_t>(count));
        GCU_CUDA(cudaMemcpyAsync(edges->data(), out.ptr, sizeof(uint2) * count, cudaMemcpyDeviceToHost, dev.stream),
                 "copy edges to host");
        GCU_TRY(dev.sync());
    }
    *iterations = rounds;
    return ok();
}

}  // namespace gcu
