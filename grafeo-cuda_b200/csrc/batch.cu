// Batched form: many uneven graphs packed into one CSR and processed by
// persistent kernels, replayed as one captured CUDA graph.
//
// Layout: graph i owns the vertices [vbase[i], vbase[i + 1]) of a union CSR
// whose targets are union ids (no edge leaves its graph), so the union is a
// plain symmetric CSR and graph i's entries are [offsets[vbase[i]],
// offsets[vbase[i + 1]]).
//
//  * Triangles: one degree-oriented DAG of the union and its out-degree
//    buckets, one variant per bucket (the installed learned schedule's pick,
//    else the fastest of the valid variants timed once on the batch); the
//    wedge kernels add each DAG source's triangles into a per-vertex counter
//    and a block per graph sums its vertices.
//  * BFS from S <= 32 sources per graph: multi-source BFS (Then et al., VLDB
//    2015) with one S-bit mask per vertex for visited / frontier / next: a CTA
//    owns a graph and runs all its levels itself (pull: a vertex ORs its
//    neighbours' frontier masks, stopping once every missing bit is found),
//    so there is no host round trip and no grid-wide barrier; bit k of a
//    vertex's mask appearing at level L is distance L from source k.
//  * Personalised PageRank from K seeds per graph (teleport 1/K per seed,
//    repeats add up; the formula of gcu_personalized_pagerank): a CTA owns a
//    graph and iterates to its own convergence (L1 change < tol, FP64 block
//    reductions of the residual and the dangling mass), FP32 row sums (a lane
//    per short row, a warp per row of >= 32 entries).
//  * CTAs take graphs from a queue ordered by entry count, largest first
//    (longest-processing-time order). The CTA size of the BFS and PageRank
//    kernels is autotuned per batch (256 / 512 / 1024 threads, each timed
//    once on the whole batch, the fastest kept).
// No reference counterpart: the reference runs one graph per call.
#include <algorithm>
#include <numeric>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr uint32_t kMaxBatchSources = 32;

// ---------------------------------------------------------------- kernels

__global__ void batch_entry_base_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ vbase,
                                        uint32_t G, uint32_t* __restrict__ ebase) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x)
        ebase[g] = offsets[vbase[g]];
}

// First union entry whose target lies outside its row's graph (atomicMin).
__global__ void batch_check_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                   const uint32_t* __restrict__ vbase, uint32_t G,
                                   unsigned long long* __restrict__ first_bad) {
    for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
        const uint32_t vb = vbase[g], ve = vbase[g + 1];
        const uint32_t e0 = offsets[vb], e1 = offsets[ve];
        for (uint32_t j = e0 + threadIdx.x; j < e1; j += blockDim.x) {
            const uint32_t t = targets[j];
            if (t < vb || t >= ve) atomicMin(first_bad, static_cast<unsigned long long>(j));
        }
    }
}

__global__ void batch_graph_sum_kernel(const unsigned long long* __restrict__ per_vertex,
                                       const uint32_t* __restrict__ vbase, uint32_t G,
                                       unsigned long long* __restrict__ totals) {
    __shared__ unsigned long long scratch[32];
    for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
        unsigned long long acc = 0;
        for (uint32_t v = vbase[g] + threadIdx.x; v < vbase[g + 1]; v += blockDim.x) acc += per_vertex[v];
        acc = block_sum(acc, scratch);
        if (threadIdx.x == 0) totals[g] = acc;
    }
}

// Teleport vector: 1/K for every seed (local ids), repeats add up.
__global__ void batch_tele_kernel(const uint32_t* __restrict__ seeds, const uint32_t* __restrict__ vbase, uint32_t G,
                                  uint32_t K, float* __restrict__ tele) {
    const uint64_t total = static_cast<uint64_t>(G) * K;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t g = static_cast<uint32_t>(i / K);
        atomicAdd(tele + vbase[g] + seeds[i], 1.0f / static_cast<float>(K));
    }
}

// One member graph copied out with local ids.
__global__ void batch_extract_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                     uint32_t vb, uint32_t n, uint32_t eb, uint32_t m, uint32_t* __restrict__ lo,
                                     uint32_t* __restrict__ lt) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n || i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (i <= n) lo[i] = offsets[vb + i] - eb;
        if (i < m) lt[i] = targets[eb + i] - vb;
    }
}

// Multi-source BFS, one CTA per graph at a time (see the file comment).
template <int kThreads>
__global__ void __launch_bounds__(kThreads) batch_bfs_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ vbase,
    const uint32_t* __restrict__ order, uint32_t G, const uint32_t* __restrict__ sources, uint32_t S,
    uint32_t* __restrict__ visited, uint32_t* buf_a, uint32_t* buf_b, int32_t* __restrict__ dist, uint64_t Vt,
    uint32_t* __restrict__ reachable, int32_t* __restrict__ max_depth, uint32_t* __restrict__ next_graph) {
    constexpr int kWarps = kThreads / 32;
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_or[kWarps];
    __shared__ uint32_t s_count[kMaxBatchSources];
    __shared__ int32_t s_last[kMaxBatchSources];
    const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
    const uint32_t full = S >= 32 ? 0xFFFFFFFFu : ((1u << S) - 1u);
    while (true) {
        if (tid == 0) s_item = atomicAdd(next_graph, 1u);
        __syncthreads();
        const uint32_t h = s_item;
        if (h >= G) break;
        const uint32_t g = order[h];
        const uint32_t vb = vbase[g], ve = vbase[g + 1];
        uint32_t* frontier = buf_a;
        uint32_t* next = buf_b;
        for (uint32_t v = vb + tid; v < ve; v += kThreads) {
            visited[v] = 0;
            frontier[v] = 0;
        }
        if (tid < kMaxBatchSources) {
            s_count[tid] = 0;
            s_last[tid] = 0;
        }
        __syncthreads();
        if (tid < S) {
            const uint32_t s = vb + sources[static_cast<uint64_t>(g) * S + tid];
            atomicOr(visited + s, 1u << tid);
            atomicOr(frontier + s, 1u << tid);
            if (dist) dist[tid * Vt + s] = 0;
        }
        __syncthreads();
        int32_t level = 0;
        while (true) {
            uint32_t any = 0;
            for (uint32_t v = vb + tid; v < ve; v += kThreads) {
                const uint32_t vis = visited[v];
                uint32_t nw = 0;
                if (vis != full) {
                    uint32_t m = 0;
                    const uint32_t e = offsets[v + 1];
                    for (uint32_t j = offsets[v]; j < e; ++j) {
                        m |= frontier[targets[j]];
                        if ((m | vis) == full) break;
                    }
                    nw = m & ~vis;
                    if (nw && dist) {
                        uint32_t bits = nw;
                        while (bits) {
                            const uint32_t k = __ffs(bits) - 1;
                            dist[k * Vt + v] = level + 1;
                            bits &= bits - 1;
                        }
                    }
                    any |= nw;
                }
                next[v] = nw;
            }
            any = __reduce_or_sync(kFullMask, any);
            if (lane == 0) s_or[warp] = any;
            __syncthreads();
            uint32_t all = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) all |= s_or[w];
            if (all == 0) break;  // the same for every thread of the block
            if (tid < S && ((all >> tid) & 1u)) s_last[tid] = level + 1;
            for (uint32_t v = vb + tid; v < ve; v += kThreads) visited[v] |= next[v];
            uint32_t* t = frontier;
            frontier = next;
            next = t;
            ++level;
            __syncthreads();
        }
        // Reached vertices per source: lane k of every warp counts bit k.
        uint32_t cnt = 0;
        for (uint32_t base = vb + warp * 32; base < ve; base += kThreads) {
            const uint32_t v = base + lane;
            const uint32_t vis = v < ve ? visited[v] : 0u;
            for (uint32_t k = 0; k < S; ++k) {
                const unsigned b = __ballot_sync(kFullMask, (vis >> k) & 1u);
                if (lane == k) cnt += __popc(b);
            }
        }
        if (lane < S && cnt) atomicAdd(&s_count[lane], cnt);
        __syncthreads();
        if (tid < S) {
            reachable[static_cast<uint64_t>(g) * S + tid] = s_count[tid];
            max_depth[static_cast<uint64_t>(g) * S + tid] = s_last[tid];
        }
        __syncthreads();
    }
}

// Personalised PageRank, one CTA per graph at a time (see the file comment).
template <int kThreads>
__global__ void __launch_bounds__(kThreads) batch_ppr_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ vbase,
    const uint32_t* __restrict__ order, uint32_t G, const float* __restrict__ tele, float damping,
    uint32_t max_iterations, double tolerance, float* rank_a, float* rank_b, float* contrib_a, float* contrib_b,
    float* __restrict__ ranks_out, uint32_t* __restrict__ iterations, uint8_t* __restrict__ converged,
    uint32_t* __restrict__ next_graph) {
    __shared__ uint32_t s_item;
    __shared__ double scratch[32];
    const unsigned tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
    const double d = damping;
    while (true) {
        if (tid == 0) s_item = atomicAdd(next_graph, 1u);
        __syncthreads();
        const uint32_t h = s_item;
        if (h >= G) break;
        const uint32_t g = order[h];
        const uint32_t vb = vbase[g], ve = vbase[g + 1], n = ve - vb;
        if (n == 0) {
            if (tid == 0) {
                iterations[g] = 0;
                converged[g] = 1;
            }
            __syncthreads();
            continue;
        }
        const float r0 = 1.0f / static_cast<float>(n);
        double dang = 0.0;
        for (uint32_t v = vb + tid; v < ve; v += kThreads) {
            const uint32_t deg = offsets[v + 1] - offsets[v];
            rank_a[v] = r0;
            contrib_a[v] = deg ? r0 / static_cast<float>(deg) : 0.f;
            if (!deg) dang += r0;
        }
        double dangling = block_sum(dang, scratch);
        float *r = rank_a, *rn = rank_b, *c = contrib_a, *cn = contrib_b;
        uint32_t it = 0;
        bool conv = false;
        while (it < max_iterations) {
            double l1 = 0.0, dn = 0.0;
            for (uint32_t base = vb + warp * 32; base < ve; base += kThreads) {
                const uint32_t v = base + lane;
                const bool valid = v < ve;
                uint32_t s = 0, e = 0;
                if (valid) {
                    s = offsets[v];
                    e = offsets[v + 1];
                }
                const uint32_t deg = e - s;
                float sum = 0.f;
                if (valid && deg < 32)
                    for (uint32_t j = s; j < e; ++j) sum += c[targets[j]];
                unsigned longs = __ballot_sync(kFullMask, valid && deg >= 32);
                while (longs) {
                    const int i = __ffs(longs) - 1;
                    longs &= longs - 1;
                    const uint32_t rs = __shfl_sync(kFullMask, s, i), re = __shfl_sync(kFullMask, e, i);
                    float part = 0.f;
                    for (uint32_t j = rs + lane; j < re; j += 32) part += c[targets[j]];
                    part = warp_sum(part);
                    if (static_cast<int>(lane) == i) sum = part;
                }
                if (valid) {
                    const double p = tele[v];
                    const float x = static_cast<float>((1.0 - d) * p + d * (static_cast<double>(sum) + dangling * p));
                    l1 += fabs(static_cast<double>(x) - static_cast<double>(r[v]));
                    rn[v] = x;
                    cn[v] = deg ? x / static_cast<float>(deg) : 0.f;
                    if (!deg) dn += x;
                }
            }
            l1 = block_sum(l1, scratch);
            dangling = block_sum(dn, scratch);
            float* t = r;
            r = rn;
            rn = t;
            t = c;
            c = cn;
            cn = t;
            ++it;
            if (l1 < tolerance) {
                conv = true;
                break;
            }
        }
        for (uint32_t v = vb + tid; v < ve; v += kThreads) ranks_out[v] = r[v];
        if (tid == 0) {
            iterations[g] = it;
            converged[g] = conv ? 1 : 0;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- host

struct BatchImpl {
    std::shared_ptr<DeviceImpl> dev;
    GraphImpl u;  // the union CSR
    uint32_t G = 0;
    std::vector<uint32_t> vbase, ebase;
    DeviceBuffer<uint32_t> d_vbase, d_order, counters;
    BatchTcPlan* tc = nullptr;
    std::string tc_tuning;
    DeviceBuffer<unsigned long long> tri_vertex, tri_totals;
    // BFS
    uint32_t S = 0;
    bool keep_dist = true;
    int bfs_threads = 0;
    DeviceBuffer<uint32_t> sources, visited, mask_a, mask_b, reachable;
    DeviceBuffer<int32_t> dist, max_depth;
    // personalised PageRank
    uint32_t K = 0;
    float damping = 0.85f, tolerance = 1e-6f;
    uint32_t max_iterations = 100;
    int ppr_threads = 0;
    DeviceBuffer<uint32_t> seeds, iterations;
    DeviceBuffer<uint8_t> converged;
    DeviceBuffer<float> tele, rank_a, rank_b, contrib_a, contrib_b, ranks;
    // captured replay of the three
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string bfs_tuning, ppr_tuning;

    ~BatchImpl() {
        if (dev) dev->activate();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        destroy_batch_tc_plan(tc);
    }
};

void destroy_batch(BatchImpl* b) { delete b; }

namespace {

uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

unsigned small_grid(const DeviceImpl& dev, uint64_t n, unsigned threads) {
    return static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(n, threads), static_cast<uint64_t>(dev.sm_count) * 8)));
}

// vbase uploaded, ebase gathered, graphs ordered by entries (largest first).
Error finish_layout(BatchImpl& b) {
    DeviceImpl& dev = *b.dev;
    const uint32_t G = b.G;
    GCU_TRY(b.d_vbase.allocate(dev, G + 1));
    GCU_CUDA(cudaMemcpyAsync(b.d_vbase.ptr, b.vbase.data(), 4 * (G + 1), cudaMemcpyHostToDevice, dev.stream), "copy");
    DeviceBuffer<uint32_t> d_ebase;
    GCU_TRY(d_ebase.allocate(dev, G + 1));
    GCU_LAUNCH(dev, "batch_entry_base", batch_entry_base_kernel, small_grid(dev, G + 1, 256), 256, 0, b.u.offsets.ptr,
               b.d_vbase.ptr, G, d_ebase.ptr);
    b.ebase.resize(G + 1);
    GCU_CUDA(cudaMemcpyAsync(b.ebase.data(), d_ebase.ptr, 4 * (G + 1), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    std::vector<uint32_t> order(G);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return b.ebase[x + 1] - b.ebase[x] > b.ebase[y + 1] - b.ebase[y];
    });
    GCU_TRY(b.d_order.allocate(dev, std::max<uint32_t>(G, 1)));
    if (G) GCU_CUDA(cudaMemcpyAsync(b.d_order.ptr, order.data(), 4 * G, cudaMemcpyHostToDevice, dev.stream), "copy");
    GCU_TRY(b.counters.allocate(dev, 2));
    return dev.sync();
}

template <int kThreads>
Error launch_bfs_t(BatchImpl& b) {
    DeviceImpl& dev = *b.dev;
    int per_sm = 0;
    GCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_bfs_kernel<kThreads>, kThreads, 0),
             "occupancy");
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(b.G, static_cast<uint64_t>(dev.sm_count) * std::max(per_sm, 1))));
    GCU_LAUNCH(dev, "batch_bfs", batch_bfs_kernel<kThreads>, grid, kThreads, 0, b.u.offsets.ptr, b.u.targets.ptr,
               b.d_vbase.ptr, b.d_order.ptr, b.G, b.sources.ptr, b.S, b.visited.ptr, b.mask_a.ptr, b.mask_b.ptr,
               b.keep_dist ? b.dist.ptr : nullptr, static_cast<uint64_t>(b.u.num_nodes), b.reachable.ptr,
               b.max_depth.ptr, b.counters.ptr);
    return ok();
}

Error launch_bfs(BatchImpl& b, int threads) {
    DeviceImpl& dev = *b.dev;
    GCU_CUDA(cudaMemsetAsync(b.counters.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
    if (b.keep_dist)
        GCU_CUDA(cudaMemsetAsync(b.dist.ptr, 0xFF, sizeof(int32_t) * b.S * static_cast<size_t>(b.u.num_nodes),
                                 dev.stream),
                 "memset");
    if (threads == 256) return launch_bfs_t<256>(b);
    if (threads == 512) return launch_bfs_t<512>(b);
    return launch_bfs_t<1024>(b);
}

template <int kThreads>
Error launch_ppr_t(BatchImpl& b) {
    DeviceImpl& dev = *b.dev;
    int per_sm = 0;
    GCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_ppr_kernel<kThreads>, kThreads, 0),
             "occupancy");
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(b.G, static_cast<uint64_t>(dev.sm_count) * std::max(per_sm, 1))));
    GCU_LAUNCH(dev, "batch_ppr", batch_ppr_kernel<kThreads>, grid, kThreads, 0, b.u.offsets.ptr, b.u.targets.ptr,
               b.d_vbase.ptr, b.d_order.ptr, b.G, b.tele.ptr, b.damping, b.max_iterations,
               static_cast<double>(b.tolerance), b.rank_a.ptr, b.rank_b.ptr, b.contrib_a.ptr, b.contrib_b.ptr,
               b.ranks.ptr, b.iterations.ptr, b.converged.ptr, b.counters.ptr + 1);
    return ok();
}

Error launch_ppr(BatchImpl& b, int threads) {
    DeviceImpl& dev = *b.dev;
    GCU_CUDA(cudaMemsetAsync(b.counters.ptr + 1, 0, sizeof(uint32_t), dev.stream), "memset");
    if (threads == 256) return launch_ppr_t<256>(b);
    if (threads == 512) return launch_ppr_t<512>(b);
    return launch_ppr_t<1024>(b);
}

Error launch_tc(BatchImpl& b) {
    DeviceImpl& dev = *b.dev;
    GCU_TRY(batch_tc_launch(dev, *b.tc, b.tri_vertex.ptr, b.u.num_nodes));
    GCU_LAUNCH(dev, "batch_graph_sum", batch_graph_sum_kernel, small_grid(dev, b.G, 1), 256, 0, b.tri_vertex.ptr,
               b.d_vbase.ptr, b.G, b.tri_totals.ptr);
    return ok();
}

// Times each candidate CTA size once on the whole batch and keeps the fastest.
template <class Launch>
Error autotune(BatchImpl& b, Launch launch, int* best, std::string* json) {
    DeviceImpl& dev = *b.dev;
    const int cand[3] = {256, 512, 1024};
    cudaEvent_t e0, e1;
    GCU_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
    GCU_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
    float best_ms = 0.f;
    *json = "{";
    Error err = ok();
    for (int i = 0; i < 3 && err.ok(); ++i) {
        cudaEventRecord(e0, dev.stream);
        err = launch(b, cand[i]);
        cudaEventRecord(e1, dev.stream);
        if (err.ok()) err = dev.sync();
        float ms = 0.f;
        if (err.ok()) cudaEventElapsedTime(&ms, e0, e1);
        if (i == 0 || ms < best_ms) {
            best_ms = ms;
            *best = cand[i];
        }
        *json += (i ? ", \"" : "\"") + std::to_string(cand[i]) + "\": " + std::to_string(ms);
    }
    *json += ", \"chosen\": " + std::to_string(*best) + "}";
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err;
}

}  // namespace

// The generated corpus: graph i is R-MAT (scale U{8..16}, edge factor
// U{8..32}, a, b, c = 0.57, 0.19, 0.19) or Watts-Strogatz (n U{256..65536},
// k = 10, p = 0.1) with equal odds, every draw from SplitMix64 of (seed, i).
Error batch_generate(DeviceImpl& dev, std::shared_ptr<DeviceImpl> owner, uint32_t num_graphs, uint64_t seed,
                     BatchImpl** out) {
    auto b = std::make_unique<BatchImpl>();
    b->dev = owner;
    b->u.dev = owner;
    b->G = num_graphs;
    std::vector<GeneratorSpec> specs(num_graphs);
    for (uint32_t i = 0; i < num_graphs; ++i) {
        const uint64_t r = mix64(mix64(seed + 0x9E3779B97F4A7C15ull) + i);
        GeneratorSpec& s = specs[i];
        s.seed = mix64(r ^ 0xD1B54A32D192ED03ull);
        if ((r & 1) == 0) {
            s.kind = GeneratorSpec::kRmat;
            s.scale = 8 + static_cast<uint32_t>((r >> 8) % 9);
            s.edge_factor = 8 + static_cast<uint32_t>((r >> 16) % 25);
            s.a = 0.57;
            s.b = 0.19;
            s.c = 0.19;
        } else {
            s.kind = GeneratorSpec::kWattsStrogatz;
            s.n = 256 + static_cast<uint32_t>((r >> 8) % (65536 - 256 + 1));
            s.k = 10;
            s.p = 0.1;
        }
    }
    GCU_TRY(generate_union(dev, specs, &b->vbase, b->u));
    GCU_TRY(finish_layout(*b));
    *out = b.release();
    return ok();
}

Error batch_from_csr(DeviceImpl& dev, std::shared_ptr<DeviceImpl> owner, const uint32_t* vbase, size_t num_graphs,
                     const uint32_t* offsets, size_t n_offsets, const uint32_t* targets, size_t n_targets,
                     BatchImpl** out) {
    if (n_offsets == 0) return invalid_csr("offsets must have num_nodes + 1 entries, got an empty array");
    if (vbase[0] != 0 || vbase[num_graphs] != n_offsets - 1)
        return kernel_error("vertex_base must start at 0 and end at num_nodes (" + std::to_string(n_offsets - 1) +
                            ")");
    for (size_t i = 0; i < num_graphs; ++i)
        if (vbase[i + 1] < vbase[i]) return kernel_error("vertex_base must be non-decreasing");
    if (offsets[0] != 0) return invalid_csr("offsets[0] must be 0, got " + std::to_string(offsets[0]));
    if (static_cast<size_t>(offsets[n_offsets - 1]) != n_targets)
        return invalid_csr("offsets[" + std::to_string(n_offsets - 1) + "] is " +
                           std::to_string(offsets[n_offsets - 1]) + " but targets has " + std::to_string(n_targets) +
                           " entries");
    auto b = std::make_unique<BatchImpl>();
    b->dev = owner;
    b->u.dev = owner;
    b->G = static_cast<uint32_t>(num_graphs);
    b->vbase.assign(vbase, vbase + num_graphs + 1);
    GraphImpl& u = b->u;
    u.num_nodes = static_cast<uint32_t>(n_offsets - 1);
    u.num_edges = static_cast<uint32_t>(n_targets);
    GCU_TRY(u.offsets.allocate(dev, n_offsets));
    GCU_TRY(u.targets.allocate(dev, n_targets));
    GCU_CUDA(cudaMemcpyAsync(u.offsets.ptr, offsets, 4 * n_offsets, cudaMemcpyHostToDevice, dev.stream), "copy");
    if (n_targets)
        GCU_CUDA(cudaMemcpyAsync(u.targets.ptr, targets, 4 * n_targets, cudaMemcpyHostToDevice, dev.stream), "copy");
    uint32_t bad = UINT32_MAX;
    GCU_TRY(validate_csr_device(dev, u.offsets.ptr, u.targets.ptr, u.num_nodes, u.num_edges, &bad));
    if (bad != UINT32_MAX) {
        const uint32_t start = offsets[bad], end = offsets[bad + 1];
        const size_t lo = std::min<size_t>(start, n_targets), hi = std::min<size_t>(std::max(start, end), n_targets);
        return invalid_csr(describe_node_violation(bad, start, end, targets + lo, hi - lo, u.num_nodes));
    }
    GCU_TRY(finish_layout(*b));
    DeviceBuffer<unsigned long long> first;
    GCU_TRY(first.allocate(dev, 1));
    GCU_CUDA(cudaMemsetAsync(first.ptr, 0xFF, sizeof(unsigned long long), dev.stream), "memset");
    GCU_LAUNCH(dev, "batch_check", batch_check_kernel, small_grid(dev, b->G, 1), 256, 0, u.offsets.ptr, u.targets.ptr,
               b->d_vbase.ptr, b->G, first.ptr);
    unsigned long long j = 0;
    GCU_CUDA(cudaMemcpyAsync(&j, first.ptr, sizeof(j), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    if (j != ~0ull) {
        const uint32_t row = static_cast<uint32_t>(std::upper_bound(offsets, offsets + n_offsets, j) - offsets - 1);
        return kernel_error("batch: edge (" + std::to_string(row) + ", " + std::to_string(targets[j]) +
                            ") leaves its graph");
    }
    *out = b.release();
    return ok();
}

Error batch_member(BatchImpl& b, uint32_t index, GraphImpl& g) {
    DeviceImpl& dev = *b.dev;
    if (index >= b.G) return kernel_error("graph index " + std::to_string(index) + " out of range (batch of " +
                                          std::to_string(b.G) + ")");
    const uint32_t vb = b.vbase[index], n = b.vbase[index + 1] - vb;
    const uint32_t eb = b.ebase[index], m = b.ebase[index + 1] - eb;
    g.num_nodes = n;
    g.num_edges = m;
    GCU_TRY(g.offsets.allocate(dev, static_cast<uint64_t>(n) + 1));
    GCU_TRY(g.targets.allocate(dev, m));
    GCU_LAUNCH(dev, "batch_extract", batch_extract_kernel, small_grid(dev, std::max<uint64_t>(n + 1, m), 256), 256, 0,
               b.u.offsets.ptr, b.u.targets.ptr, vb, n, eb, m, g.offsets.ptr, g.targets.ptr);
    g.symmetric = b.u.symmetric;
    return dev.sync();
}

// A captured graph holds the device pointers and the per-batch parameters
// (S, K, damping, ...) by value: setting new sources or seeds reallocates the
// buffers it reads, so the capture is dropped, and gcu_batch_replay refuses
// to run until the caller captures again.
static void drop_capture(BatchImpl& b) {
    if (b.exec) {
        cudaGraphExecDestroy(b.exec);
        b.exec = nullptr;
    }
    if (b.graph) {
        cudaGraphDestroy(b.graph);
        b.graph = nullptr;
    }
}

Error batch_set_bfs(BatchImpl& b, const uint32_t* sources, uint32_t S, bool keep_distances) {
    DeviceImpl& dev = *b.dev;
    if (S == 0 || S > kMaxBatchSources) return kernel_error("sources per graph must be in 1..=32");
    for (uint32_t g = 0; g < b.G; ++g) {
        const uint32_t n = b.vbase[g + 1] - b.vbase[g];
        for (uint32_t k = 0; k < S; ++k)
            if (sources[static_cast<uint64_t>(g) * S + k] >= n)
                return kernel_error("source node " + std::to_string(sources[static_cast<uint64_t>(g) * S + k]) +
                                    " of graph " + std::to_string(g) + " out of range (num_nodes = " +
                                    std::to_string(n) + ")");
    }
    GCU_TRY(dev.sync());  // a replay in flight may still read the old buffers
    drop_capture(b);
    const uint64_t V = b.u.num_nodes;
    b.S = S;
    b.keep_dist = keep_distances;
    GCU_TRY(b.sources.allocate(dev, static_cast<uint64_t>(b.G) * S));
    GCU_CUDA(cudaMemcpyAsync(b.sources.ptr, sources, 4ull * b.G * S, cudaMemcpyHostToDevice, dev.stream), "copy");
    GCU_TRY(b.visited.allocate(dev, V));
    GCU_TRY(b.mask_a.allocate(dev, V));
    GCU_TRY(b.mask_b.allocate(dev, V));
    GCU_TRY(b.reachable.allocate(dev, static_cast<uint64_t>(b.G) * S));
    GCU_TRY(b.max_depth.allocate(dev, static_cast<uint64_t>(b.G) * S));
    if (keep_distances) GCU_TRY(b.dist.allocate(dev, V * S));
    b.bfs_threads = 0;
    return dev.sync();
}

Error batch_set_ppr(BatchImpl& b, const uint32_t* seeds, uint32_t K, float damping, uint32_t max_iterations,
                    float tolerance) {
    DeviceImpl& dev = *b.dev;
    if (K == 0) return kernel_error("personalized PageRank needs at least one seed");
    for (uint32_t g = 0; g < b.G; ++g) {
        const uint32_t n = b.vbase[g + 1] - b.vbase[g];
        for (uint32_t k = 0; k < K; ++k)
            if (seeds[static_cast<uint64_t>(g) * K + k] >= n)
                return kernel_error("seed node " + std::to_string(seeds[static_cast<uint64_t>(g) * K + k]) +
                                    " of graph " + std::to_string(g) + " out of range (num_nodes = " +
                                    std::to_string(n) + ")");
    }
    GCU_TRY(dev.sync());  // a replay in flight may still read the old buffers
    drop_capture(b);
    const uint64_t V = b.u.num_nodes;
    b.K = K;
    b.damping = damping;
    b.max_iterations = max_iterations;
    b.tolerance = tolerance;
    GCU_TRY(b.seeds.allocate(dev, static_cast<uint64_t>(b.G) * K));
    GCU_CUDA(cudaMemcpyAsync(b.seeds.ptr, seeds, 4ull * b.G * K, cudaMemcpyHostToDevice, dev.stream), "copy");
    GCU_TRY(b.tele.allocate(dev, V));
    GCU_TRY(b.rank_a.allocate(dev, V));
    GCU_TRY(b.rank_b.allocate(dev, V));
    GCU_TRY(b.contrib_a.allocate(dev, V));
    GCU_TRY(b.contrib_b.allocate(dev, V));
    GCU_TRY(b.ranks.allocate(dev, V));
    GCU_TRY(b.iterations.allocate(dev, std::max<uint32_t>(b.G, 1)));
    GCU_TRY(b.converged.allocate(dev, std::max<uint32_t>(b.G, 1)));
    GCU_CUDA(cudaMemsetAsync(b.tele.ptr, 0, 4 * std::max<uint64_t>(V, 1), dev.stream), "memset");
    GCU_LAUNCH(dev, "batch_tele", batch_tele_kernel, small_grid(dev, static_cast<uint64_t>(b.G) * K, 256), 256, 0,
               b.seeds.ptr, b.d_vbase.ptr, b.G, K, b.tele.ptr);
    b.ppr_threads = 0;
    return dev.sync();
}

Error batch_ensure_tc(BatchImpl& b) {
    if (b.tc) return ok();
    DeviceImpl& dev = *b.dev;
    GCU_TRY(b.tri_vertex.allocate(dev, std::max<uint32_t>(b.u.num_nodes, 1)));
    GCU_TRY(b.tri_totals.allocate(dev, std::max<uint32_t>(b.G, 1)));
    return batch_tc_plan(b.u, &b.tc, &b.tc_tuning);
}

Error batch_run_tc(BatchImpl& b, uint64_t* totals) {
    GCU_TRY(batch_ensure_tc(b));
    GCU_TRY(launch_tc(b));
    GCU_CUDA(cudaMemcpyAsync(totals, b.tri_totals.ptr, 8ull * b.G, cudaMemcpyDeviceToHost, b.dev->stream), "copy");
    return b.dev->sync();
}

Error batch_run_bfs(BatchImpl& b) {
    if (!b.S) return kernel_error("batch BFS sources are not set");
    if (!b.bfs_threads) return autotune(b, launch_bfs, &b.bfs_threads, &b.bfs_tuning);
    GCU_TRY(launch_bfs(b, b.bfs_threads));
    return b.dev->sync();
}

Error batch_run_ppr(BatchImpl& b) {
    if (!b.K) return kernel_error("batch PageRank seeds are not set");
    if (!b.ppr_threads) return autotune(b, launch_ppr, &b.ppr_threads, &b.ppr_tuning);
    GCU_TRY(launch_ppr(b, b.ppr_threads));
    return b.dev->sync();
}

Error batch_read_bfs(BatchImpl& b, int32_t* distances, uint32_t* reachable, int32_t* max_depth) {
    DeviceImpl& dev = *b.dev;
    const uint64_t gs = static_cast<uint64_t>(b.G) * b.S;
    if (distances && b.keep_dist) GCU_TRY(copy_to_host(dev, distances, b.dist.ptr, 4ull * b.S * b.u.num_nodes));
    if (reachable) GCU_CUDA(cudaMemcpyAsync(reachable, b.reachable.ptr, 4 * gs, cudaMemcpyDeviceToHost, dev.stream), "copy");
    if (max_depth) GCU_CUDA(cudaMemcpyAsync(max_depth, b.max_depth.ptr, 4 * gs, cudaMemcpyDeviceToHost, dev.stream), "copy");
    return dev.sync();
}

Error batch_read_ppr(BatchImpl& b, float* ranks, uint32_t* iterations, uint8_t* converged) {
    DeviceImpl& dev = *b.dev;
    if (ranks) GCU_TRY(copy_to_host(dev, ranks, b.ranks.ptr, 4ull * b.u.num_nodes));
    if (iterations)
        GCU_CUDA(cudaMemcpyAsync(iterations, b.iterations.ptr, 4ull * b.G, cudaMemcpyDeviceToHost, dev.stream), "copy");
    if (converged)
        GCU_CUDA(cudaMemcpyAsync(converged, b.converged.ptr, b.G, cudaMemcpyDeviceToHost, dev.stream), "copy");
    return dev.sync();
}

// Captures triangle counts, BFS and PageRank of the whole batch into one CUDA
// graph (plans and autotunes first: nothing in the capture allocates or syncs).
Error batch_capture(BatchImpl& b) {
    DeviceImpl& dev = *b.dev;
    if (!b.S || !b.K) return kernel_error("set the batch BFS sources and PageRank seeds before capturing");
    GCU_TRY(batch_ensure_tc(b));
    if (!b.bfs_threads) GCU_TRY(autotune(b, launch_bfs, &b.bfs_threads, &b.bfs_tuning));
    if (!b.ppr_threads) GCU_TRY(autotune(b, launch_ppr, &b.ppr_threads, &b.ppr_tuning));
    drop_capture(b);
    const bool timing = dev.kernel_timing;
    dev.kernel_timing = false;  // no event bookkeeping inside the capture
    GCU_CUDA(cudaStreamBeginCapture(dev.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    Error e = launch_tc(b);
    if (e.ok()) e = launch_bfs(b, b.bfs_threads);
    if (e.ok()) e = launch_ppr(b, b.ppr_threads);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(dev.stream, &graph);
    dev.kernel_timing = timing;
    if (!e.ok()) {
        if (graph) cudaGraphDestroy(graph);
        return e;
    }
    if (ce != cudaSuccess) return driver_error(ce, "cudaStreamEndCapture");
    b.graph = graph;
    GCU_CUDA(cudaGraphInstantiate(&b.exec, b.graph, 0), "cudaGraphInstantiate");
    return ok();
}

Error batch_replay(BatchImpl& b) {
    if (!b.exec) return kernel_error("batch has no captured graph (call gcu_batch_capture first)");
    b.dev->launches.fetch_add(1, std::memory_order_relaxed);
    GCU_CUDA(cudaGraphLaunch(b.exec, b.dev->stream), "cudaGraphLaunch");
    return ok();
}

uint32_t batch_num_graphs(const BatchImpl& b) { return b.G; }
GraphImpl& batch_union(BatchImpl& b) { return b.u; }
const std::vector<uint32_t>& batch_vertex_base(const BatchImpl& b) { return b.vbase; }

Error batch_read_tc(BatchImpl& b, uint64_t* totals) {
    if (!b.tc) return kernel_error("batch triangle counts have not run");
    GCU_CUDA(cudaMemcpyAsync(totals, b.tri_totals.ptr, 8ull * b.G, cudaMemcpyDeviceToHost, b.dev->stream), "copy");
    return b.dev->sync();
}

std::string batch_tuning(const BatchImpl& b) {
    return "{\"triangle_buckets\": " + (b.tc_tuning.empty() ? std::string("null") : b.tc_tuning) +
           ", \"bfs_threads\": " + (b.bfs_tuning.empty() ? std::string("null") : b.bfs_tuning) +
           ", \"ppr_threads\": " + (b.ppr_tuning.empty() ? std::string("null") : b.ppr_tuning) + "}";
}

}  // namespace gcu
