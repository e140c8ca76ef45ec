// Breadth-first search: direction-optimising, level synchronous.
//
// Reference: crates/grafeo-cuda-algos/src/bfs.rs:42-131 and kernels/bfs.cu:54-83
// (one thread per frontier vertex walking its whole list, an atomicCAS per
// edge on `distances`, one global atomic per discovered vertex, and a host
// sync plus a 4-byte copy per level). Here:
//
//  * Top-down step (small frontiers): the frontier's edges are split evenly
//    over blocks (an exclusive scan of frontier degrees, then a load-balanced
//    search per block over the scan staged in shared memory), so a hub's list
//    is read by many blocks with coalesced loads instead of one thread.
//    Discovery is an atomicOr on a visited bitmap (V/8 bytes, L2 resident)
//    after a plain test; the next queue is appended with one atomic per warp.
//  * Bottom-up step (large frontiers, symmetric graphs only): every unvisited
//    vertex scans its list for a parent in the frontier bitmap and stops at the
//    first hit (Beamer, Asanovic and Patterson, SC'12). No atomics: each warp
//    owns one bitmap word of 32 vertices.
//  * Direction rule: Beamer's alpha/beta heuristic (alpha = 14, beta = 24),
//    fed by the frontier and unexplored edge counts the steps emit. The
//    direction only changes the schedule; BFS levels are unique, so the
//    distances cannot change.
//  * Vertices without out-edges are counted and labelled but never queued.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kTdThreads = 256;
constexpr int kTdItems = 4;
constexpr int kTdTile = kTdThreads * kTdItems;  // frontier edges per block
constexpr int kBuThreads = 256;

struct BfsCounters {
    uint32_t discovered;  // vertices labelled this level
    uint32_t queued;      // of those, vertices with out-edges (appended to the queue)
    unsigned long long edges;  // sum of out-degrees of the vertices labelled this level
};

struct BfsWork {
    DeviceBuffer<int32_t> dist;
    DeviceBuffer<uint32_t> visited;
    DeviceBuffer<uint32_t> bitmap[2];
    DeviceBuffer<uint32_t> queue[2];
    DeviceBuffer<uint32_t> degree_scan;  // V + 1
    DeviceBuffer<BfsCounters> counters;
    BfsCounters* host_counters = nullptr;  // pinned
    int symmetric = -1;                    // -1 unknown, 0 no, 1 yes
};

void destroy_bfs_work(BfsWork* w) {
    if (!w) return;
    if (w->host_counters) cudaFreeHost(w->host_counters);
    delete w;
}

// ---------------------------------------------------------------- kernels

__device__ __forceinline__ void append_warp(bool take, uint32_t v, uint32_t* __restrict__ queue,
                                            uint32_t* __restrict__ count) {
    const unsigned mask = __ballot_sync(kFullMask, take);
    if (mask == 0) return;
    const unsigned lane = lane_id();
    uint32_t base = 0;
    if (lane == static_cast<unsigned>(__ffs(mask) - 1)) base = atomicAdd(count, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(kFullMask, base, __ffs(mask) - 1);
    if (take) queue[base + __popc(mask & ((1u << lane) - 1))] = v;
}

// Labels v (found by a parent at this level) and records it; called by all
// lanes of a warp, `found` says whether this lane discovered a vertex.
__device__ __forceinline__ void record_discovery(bool found, uint32_t v, const uint32_t* __restrict__ offsets,
                                                 int32_t* __restrict__ dist, int32_t level,
                                                 uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr) {
    uint32_t deg = 0;
    if (found) {
        dist[v] = level;
        deg = offsets[v + 1] - offsets[v];
    }
    const unsigned found_mask = __ballot_sync(kFullMask, found);
    if (found_mask == 0) return;
    unsigned long long e = warp_sum(static_cast<unsigned long long>(deg));
    append_warp(found && deg > 0, v, next_queue, &ctr->queued);
    if (lane_id() == static_cast<unsigned>(__ffs(found_mask) - 1)) {
        atomicAdd(&ctr->discovered, static_cast<uint32_t>(__popc(found_mask)));
        if (e) atomicAdd(&ctr->edges, e);
    }
}

__global__ void bfs_init_kernel(const uint32_t* __restrict__ offsets, uint32_t source, int32_t* __restrict__ dist,
                                uint32_t* __restrict__ visited, uint32_t* __restrict__ queue,
                                BfsCounters* __restrict__ ctr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    dist[source] = 0;
    visited[source >> 5] |= 1u << (source & 31);
    uint32_t deg = offsets[source + 1] - offsets[source];
    queue[0] = source;
    ctr->discovered = 1;
    ctr->queued = deg > 0 ? 1 : 0;
    ctr->edges = deg;
}

__global__ void bfs_queue_degrees_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ queue,
                                         uint32_t n, uint32_t* __restrict__ deg) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t u = queue[i];
        deg[i] = offsets[u + 1] - offsets[u];
    }
}

// Top-down: block b expands frontier edges [b*kTdTile, (b+1)*kTdTile).
__global__ void __launch_bounds__(kTdThreads) bfs_topdown_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ queue,
    uint32_t qsize, const uint32_t* __restrict__ qscan, int32_t* __restrict__ dist, uint32_t* __restrict__ visited,
    uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr, int32_t next_level) {
    __shared__ uint32_t s_scan[kTdTile + 1];
    __shared__ uint32_t s_start[kTdTile + 1];
    __shared__ uint32_t s_range[2];
    const uint32_t total = qscan[qsize];
    const uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kTdTile;
    if (e0 >= total) return;
    const uint32_t e1 = static_cast<uint32_t>(min_u64(e0 + kTdTile, total));
    if (threadIdx.x < 2) {
        // Largest frontier index i with qscan[i] <= e (each queued vertex owns >= 1 edge).
        uint32_t e = threadIdx.x == 0 ? static_cast<uint32_t>(e0) : e1 - 1;
        uint32_t lo = 0, hi = qsize;
        while (hi - lo > 1) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if (qscan[mid] <= e)
                lo = mid;
            else
                hi = mid;
        }
        s_range[threadIdx.x] = lo;
    }
    __syncthreads();
    const uint32_t i0 = s_range[0];
    const uint32_t window = s_range[1] - i0 + 1;  // <= kTdTile
    for (uint32_t k = threadIdx.x; k < window; k += kTdThreads) {
        s_scan[k] = qscan[i0 + k];
        s_start[k] = offsets[queue[i0 + k]];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kTdItems; ++q) {
        const uint32_t e = static_cast<uint32_t>(e0) + q * kTdThreads + threadIdx.x;
        bool found = false;
        uint32_t v = 0;
        if (e < e1) {
            uint32_t lo = 0, hi = window;
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (s_scan[mid] <= e)
                    lo = mid;
                else
                    hi = mid;
            }
            v = ld_stream(targets + s_start[lo] + (e - s_scan[lo]));
            const uint32_t bit = 1u << (v & 31);
            if (!(__ldcg(visited + (v >> 5)) & bit)) found = !(atomicOr(visited + (v >> 5), bit) & bit);
        }
        record_discovery(found, v, offsets, dist, next_level, next_queue, ctr);
    }
}

__global__ void bfs_queue_to_bitmap_kernel(const uint32_t* __restrict__ queue, uint32_t n,
                                           uint32_t* __restrict__ bitmap) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t u = queue[i];
        atomicOr(bitmap + (u >> 5), 1u << (u & 31));
    }
}

// Bottom-up: warp w handles the 32 vertices of bitmap word w.
__global__ void __launch_bounds__(kBuThreads) bfs_bottomup_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t V,
    const uint32_t* __restrict__ frontier, uint32_t* __restrict__ next_frontier, uint32_t* __restrict__ visited,
    int32_t* __restrict__ dist, uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr,
    int32_t next_level) {
    const unsigned lane = lane_id();
    const uint64_t words = ceil_div_u64(V, 32);
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < words; w += warps) {
        const uint32_t vis = visited[w];
        const uint32_t v = static_cast<uint32_t>(w * 32 + lane);
        bool found = false;
        if (v < V && !((vis >> lane) & 1u)) {
            const uint32_t end = offsets[v + 1];
            for (uint32_t j = offsets[v]; j < end; ++j) {
                const uint32_t u = targets[j];
                if ((__ldg(frontier + (u >> 5)) >> (u & 31)) & 1u) {
                    found = true;
                    break;
                }
            }
        }
        const unsigned mask = __ballot_sync(kFullMask, found);
        if (lane == 0) {
            next_frontier[w] = mask;
            if (mask) visited[w] = vis | mask;
        }
        record_discovery(found, v, offsets, dist, next_level, next_queue, ctr);
    }
}

// ---------------------------------------------------------------- host

static Error ensure_work(GraphImpl& g) {
    if (g.bfs_work) return ok();
    DeviceImpl& dev = *g.dev;
    auto w = std::unique_ptr<BfsWork, void (*)(BfsWork*)>(new BfsWork, destroy_bfs_work);
    const uint64_t V = g.num_nodes, words = ceil_div_u64(V, 32);
    GCU_TRY(w->dist.allocate(dev, V));
    GCU_TRY(w->visited.allocate(dev, words));
    GCU_TRY(w->bitmap[0].allocate(dev, words));
    GCU_TRY(w->bitmap[1].allocate(dev, words));
    GCU_TRY(w->queue[0].allocate(dev, V));
    GCU_TRY(w->queue[1].allocate(dev, V));
    GCU_TRY(w->degree_scan.allocate(dev, V + 1));
    GCU_TRY(w->counters.allocate(dev, 1));
    GCU_CUDA(cudaMallocHost(reinterpret_cast<void**>(&w->host_counters), sizeof(BfsCounters)), "cudaMallocHost");
    // Bottom-up steps read in-neighbours; they equal the CSR lists only when
    // the CSR is symmetric (checked once per graph).
    bool sym = false;
    GCU_TRY(graph_symmetry(g, &sym));
    w->symmetric = sym ? 1 : 0;
    g.bfs_work = w.release();
    return ok();
}

Error bfs(GraphImpl& g, uint32_t source, int32_t* host_distances, uint32_t* reachable, int32_t* max_depth) {
    DeviceImpl& dev = *g.dev;
    GCU_TRY(ensure_work(g));
    BfsWork& w = *g.bfs_work;
    const uint32_t V = g.num_nodes;
    const uint64_t words = ceil_div_u64(V, 32);
    const unsigned grid_cap = static_cast<unsigned>(dev.sm_count) * 16;

    GCU_CUDA(cudaMemsetAsync(w.dist.ptr, 0xFF, sizeof(int32_t) * V, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(w.visited.ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
    GCU_LAUNCH(dev, "bfs_init", bfs_init_kernel, 1, 32, 0, g.offsets.ptr, source, w.dist.ptr, w.visited.ptr,
               w.queue[0].ptr, w.counters.ptr);
    GCU_CUDA(cudaMemcpyAsync(w.host_counters, w.counters.ptr, sizeof(BfsCounters), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    GCU_TRY(dev.sync());

    const double alpha = 14.0, beta = 24.0;
    uint64_t unexplored = static_cast<uint64_t>(g.num_edges) - w.host_counters->edges;
    uint32_t frontier_n = w.host_counters->discovered;
    uint32_t frontier_q = w.host_counters->queued;
    uint64_t frontier_m = w.host_counters->edges;
    uint32_t reached = 1;
    int32_t level = 0;
    int cur = 0;             // queue[cur] / bitmap[cur] hold the current frontier
    bool bottom_up = false;  // direction of the previous step
    bool bitmap_valid = false;

    while (frontier_q > 0) {
        bool use_bottom_up = bottom_up;
        if (w.symmetric == 1) {
            if (!bottom_up && static_cast<double>(frontier_m) > static_cast<double>(unexplored) / alpha)
                use_bottom_up = true;
            else if (bottom_up && static_cast<double>(frontier_n) < static_cast<double>(V) / beta)
                use_bottom_up = false;
        } else {
            use_bottom_up = false;
        }
        const int nxt = cur ^ 1;
        GCU_CUDA(cudaMemsetAsync(w.counters.ptr, 0, sizeof(BfsCounters), dev.stream), "memset");
        if (use_bottom_up) {
            if (!bitmap_valid) {
                GCU_CUDA(cudaMemsetAsync(w.bitmap[cur].ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
                unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(frontier_q, 256), grid_cap));
                GCU_LAUNCH(dev, "bfs_queue_to_bitmap", bfs_queue_to_bitmap_kernel, blocks, 256, 0, w.queue[cur].ptr,
                           frontier_q, w.bitmap[cur].ptr);
            }
            unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(words * 32, kBuThreads), grid_cap));
            GCU_LAUNCH(dev, "bfs_bottomup", bfs_bottomup_kernel, blocks, kBuThreads, 0, g.offsets.ptr, g.targets.ptr,
                       V, w.bitmap[cur].ptr, w.bitmap[nxt].ptr, w.visited.ptr, w.dist.ptr, w.queue[nxt].ptr,
                       w.counters.ptr, level + 1);
            bitmap_valid = true;
        } else {
            unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(frontier_q, 256), grid_cap));
            GCU_LAUNCH(dev, "bfs_queue_degrees", bfs_queue_degrees_kernel, blocks, 256, 0, g.offsets.ptr,
                       w.queue[cur].ptr, frontier_q, w.degree_scan.ptr);
            GCU_TRY(exclusive_scan_u32(dev, w.degree_scan.ptr, w.degree_scan.ptr, frontier_q));
            unsigned td_blocks = static_cast<unsigned>(std::max<uint64_t>(1, ceil_div_u64(frontier_m, kTdTile)));
            GCU_LAUNCH(dev, "bfs_topdown", bfs_topdown_kernel, td_blocks, kTdThreads, 0, g.offsets.ptr, g.targets.ptr,
                       w.queue[cur].ptr, frontier_q, w.degree_scan.ptr, w.dist.ptr, w.visited.ptr, w.queue[nxt].ptr,
                       w.counters.ptr, level + 1);
            bitmap_valid = false;
        }
        bottom_up = use_bottom_up;
        GCU_CUDA(cudaMemcpyAsync(w.host_counters, w.counters.ptr, sizeof(BfsCounters), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        const BfsCounters c = *w.host_counters;
        if (c.discovered == 0) break;
        level += 1;
        reached += c.discovered;
        unexplored -= c.edges;
        frontier_n = c.discovered;
        frontier_q = c.queued;
        frontier_m = c.edges;
        cur = nxt;
    }
    if (host_distances) {
        GCU_CUDA(cudaMemcpyAsync(host_distances, w.dist.ptr, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, dev.stream),
                 "copy distances to host");
        GCU_TRY(dev.sync());
    }
    *reachable = reached;
    *max_depth = level;
    return ok();
}

}  // namespace gcu
