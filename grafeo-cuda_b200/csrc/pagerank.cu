// PageRank: pull SpMV over the CSR with the update, the L1 residual and the
// dangling mass fused into its epilogue.
//
// Reference: crates/grafeo-cuda-algos/src/pagerank.rs:46-199 and
// kernels/pagerank.cu:19-134. Per iteration the reference launches four
// kernels (dangling sum, thread-per-row SpMV, L1 diff, plus memsets), reads
// `ranks_in[u] / deg[u]` with two random gathers and a divide per edge, and
// syncs the host to read the f32 diff. Here:
//
//  * Work split: merge-path over (row ends, nonzeros) (Merrill & Garland,
//    SC'16). Every tile of kTile merge items gets the same amount of work no
//    matter how skewed the degrees are, so a 160k-degree R-MAT hub is spread
//    over ~80 tiles instead of one thread.
//  * Each tile stages its slice of `offsets` and the gathered contributions
//    c[u] = rank[u] / deg(u) of its nonzeros in shared memory with coalesced
//    loads; `targets` is streamed once (no L1 allocation), `c` (4V bytes) stays
//    resident in L2.
//  * Row sums: FP32 Kahan sums inside each thread; partial sums that cross
//    threads, tiles or rows are carried in FP64 and combined by a block-wide
//    segmented scan, then across tiles by a fix-up pass in a fixed order.
//  * Epilogue per row v: r'[v] = (1-d)/N + d (sum + dangling/N); |r' - r| and
//    the dangling mass of r' go to FP64 per-tile partials, reduced in a fixed
//    order by the last block of the fix-up pass (deterministic, no float
//    atomics); c'[v] = r'[v] / deg(v) is written for the next iteration.
//  * The iteration loop stays on the device: each kernel reads a `done` flag
//    first, so the host can queue iterations ahead and poll the flag once per
//    chunk instead of syncing every iteration.
#include <algorithm>
#include <cmath>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kPrThreads = 256;
constexpr int kPrItems = 8;                       // merge items per thread
constexpr int kPrTile = kPrThreads * kPrItems;    // merge items per tile
constexpr uint32_t kNoRow = 0xFFFFFFFFu;

// Shared-memory index with one padding word per 32: each thread walks
// kPrItems consecutive staged items, so without padding the lanes of a warp
// would hit every 8th bank (an 8-way conflict on every merge step).
__device__ __forceinline__ uint32_t pad(uint32_t k) { return k + (k >> 5); }

struct PrState {
    double dangling;   // sum of ranks of dangling vertices in the current input ranks
    double last_diff;  // L1 change of the last iteration
    uint32_t iterations;
    uint32_t done;
    uint32_t ticket;
    uint32_t pad;
};

struct PageRankPlan {
    uint64_t num_tiles = 0;
    DeviceBuffer<uint2> coords;        // merge-path coordinates (row, nonzero) per tile start
    DeviceBuffer<float> ranks;         // 2 * V: ping-pong
    DeviceBuffer<float> contrib;       // 2 * V: ping-pong
    DeviceBuffer<uint32_t> head_row;   // per tile: row finished here but started in an earlier tile
    DeviceBuffer<double> head_val;
    DeviceBuffer<uint32_t> carry_row;  // per tile: row still open at the tile end
    DeviceBuffer<double> carry_val;
    DeviceBuffer<double> tile_diff;
    DeviceBuffer<double> tile_dangle;
    DeviceBuffer<double> block_partials;  // 2 * fix-up blocks
    DeviceBuffer<PrState> state;
    PrState* host_state = nullptr;     // pinned
    uint32_t final_buffer = 0;         // which half of `ranks` holds the last result
};

void destroy_pagerank_plan(PageRankPlan* p) {
    if (!p) return;
    if (p->host_state) cudaFreeHost(p->host_state);
    delete p;
}

// ---------------------------------------------------------------- kernels

// Merge-path search: coordinate (rows finished, nonzeros consumed) of
// `diagonal` in the merge of row ends offsets[1..V] with nonzero indices 0..E-1.
__device__ __forceinline__ uint2 merge_path_search(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t E,
                                                   uint64_t diagonal) {
    uint64_t lo = diagonal > E ? diagonal - E : 0;
    uint64_t hi = diagonal < V ? diagonal : V;
    while (lo < hi) {
        uint64_t pivot = (lo + hi) >> 1;
        // Row end `pivot` comes before nonzero (diagonal - pivot - 1)?
        if (static_cast<uint64_t>(offsets[pivot + 1]) <= diagonal - pivot - 1)
            lo = pivot + 1;
        else
            hi = pivot;
    }
    return make_uint2(static_cast<uint32_t>(lo), static_cast<uint32_t>(diagonal - lo));
}

__global__ void pr_plan_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t E, uint64_t num_tiles,
                               uint2* __restrict__ coords) {
    uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > num_tiles) return;
    uint64_t total = static_cast<uint64_t>(V) + E;
    uint64_t diag = std::min<uint64_t>(t * kPrTile, total);
    coords[t] = merge_path_search(offsets, V, E, diag);
}

__global__ void __launch_bounds__(kPrThreads) pr_init_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                                             float r0, float* __restrict__ ranks,
                                                             float* __restrict__ contrib,
                                                             double* __restrict__ block_partials) {
    __shared__ double scratch[32];
    double dangle = 0.0;
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t deg = offsets[v + 1] - offsets[v];
        ranks[v] = r0;
        contrib[v] = deg > 0 ? r0 / static_cast<float>(deg) : 0.f;
        if (deg == 0) dangle += static_cast<double>(r0);
    }
    dangle = block_sum(dangle, scratch);
    if (threadIdx.x == 0) block_partials[blockIdx.x] = dangle;
}

__global__ void __launch_bounds__(1024) pr_init_reduce_kernel(const double* __restrict__ block_partials,
                                                              uint32_t nblocks, PrState* __restrict__ state) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (uint32_t i = threadIdx.x; i < nblocks; i += blockDim.x) s += block_partials[i];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0) {
        state->dangling = s;
        state->last_diff = INFINITY;
        state->iterations = 0;
        state->done = 0;
        state->ticket = 0;
    }
}

// Row update shared by the tile and fix-up kernels.
__device__ __forceinline__ void pr_finish_row(uint32_t v, double sum, uint32_t deg, const float* __restrict__ rank_in,
                                              float* __restrict__ rank_out, float* __restrict__ contrib_out,
                                              double base, double damp, double spread, double& diff,
                                              double& dangle) {
    float r = static_cast<float>(base + damp * (sum + spread));
    float old = rank_in[v];
    diff += fabs(static_cast<double>(r) - static_cast<double>(old));
    rank_out[v] = r;
    contrib_out[v] = deg > 0 ? r / static_cast<float>(deg) : 0.f;
    if (deg == 0) dangle += static_cast<double>(r);
}

__global__ void __launch_bounds__(kPrThreads) pr_tile_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint2* __restrict__ coords,
    const float* __restrict__ rank_in, const float* __restrict__ contrib_in, float* __restrict__ rank_out,
    float* __restrict__ contrib_out, uint32_t V, double base, double damp, const PrState* __restrict__ state,
    uint32_t* __restrict__ head_row, double* __restrict__ head_val, uint32_t* __restrict__ carry_row,
    double* __restrict__ carry_val, double* __restrict__ tile_diff, double* __restrict__ tile_dangle) {
    if (state->done) return;
    __shared__ uint32_t s_off[kPrTile + 2 + (kPrTile + 2) / 32 + 1];
    __shared__ float s_val[kPrTile + kPrTile / 32];
    __shared__ double s_warp_v[kPrThreads / 32];
    __shared__ int s_warp_f[kPrThreads / 32];
    __shared__ uint32_t s_defer_row;
    __shared__ double s_defer_val;
    __shared__ double scratch[32];

    const uint32_t t = blockIdx.x;
    const uint2 c0 = coords[t], c1 = coords[t + 1];
    const uint32_t r0 = c0.x, z0 = c0.y;
    const uint32_t nrows = c1.x - c0.x, nnz = c1.y - c0.y;
    const uint32_t items = nrows + nnz;
    const double spread = state->dangling / static_cast<double>(V);

    // Stage offsets[r0 .. r0 + nrows + 1] and the gathered contributions.
    for (uint32_t k = threadIdx.x; k < nrows + 2; k += kPrThreads) {
        uint64_t r = static_cast<uint64_t>(r0) + k;
        s_off[pad(k)] = r <= V ? ld_stream(offsets + r) : 0xFFFFFFFFu;
    }
    {
        // All of this thread's target loads first, then all gathers, so every
        // thread keeps kPrItems independent requests in flight.
        uint32_t u[kPrItems];
#pragma unroll
        for (int q = 0; q < kPrItems; ++q) {
            const uint32_t k = threadIdx.x + q * kPrThreads;
            u[q] = k < nnz ? ld_stream(targets + z0 + k) : 0u;
        }
#pragma unroll
        for (int q = 0; q < kPrItems; ++q) {
            const uint32_t k = threadIdx.x + q * kPrThreads;
            if (k < nnz) s_val[pad(k)] = __ldg(contrib_in + u[q]);
        }
    }
    if (threadIdx.x == 0) s_defer_row = kNoRow;
    __syncthreads();

    // This thread's start on the merge path inside the tile.
    const uint32_t dk = min(static_cast<uint32_t>(threadIdx.x) * kPrItems, items);
    uint32_t lo = dk > nnz ? dk - nnz : 0, hi = min(dk, nrows);
    while (lo < hi) {
        uint32_t p = (lo + hi) >> 1;
        if (s_off[pad(p + 1)] <= z0 + dk - p - 1)
            lo = p + 1;
        else
            hi = p;
    }
    uint32_t rr = lo, jj = dk - lo;
    const uint32_t stop = min(dk + kPrItems, items);

    float acc = 0.f, comp = 0.f;  // Kahan sum of the open row
    bool has_head = false;
    double head_partial = 0.0;
    uint32_t head_local = 0;
    double my_diff = 0.0, my_dangle = 0.0;
#pragma unroll
    for (int q = 0; q < kPrItems; ++q) {
        if (dk + q >= stop) break;
        if (jj < nnz && z0 + jj < s_off[pad(rr + 1)]) {
            float y = s_val[pad(jj)] - comp;
            float s = acc + y;
            comp = (s - acc) - y;
            acc = s;
            ++jj;
        } else {
            double sum = static_cast<double>(acc) - static_cast<double>(comp);
            if (!has_head) {
                has_head = true;
                head_partial = sum;
                head_local = rr;
            } else {
                pr_finish_row(r0 + rr, sum, s_off[pad(rr + 1)] - s_off[pad(rr)], rank_in, rank_out, contrib_out, base, damp,
                              spread, my_diff, my_dangle);
            }
            acc = 0.f;
            comp = 0.f;
            ++rr;
        }
    }

    // Block-wide segmented scan of the carries: a thread that finished a row
    // starts a new segment. The exclusive value is what earlier threads add to
    // this thread's first finished row.
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    double v = static_cast<double>(acc) - static_cast<double>(comp);
    int f = has_head ? 1 : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double pv = __shfl_up_sync(kFullMask, v, o);
        int pf = __shfl_up_sync(kFullMask, f, o);
        if (lane >= static_cast<unsigned>(o)) {
            if (!f) v += pv;
            f |= pf;
        }
    }
    if (lane == 31) {
        s_warp_v[warp] = v;
        s_warp_f[warp] = f;
    }
    __syncthreads();
    double pre_v = 0.0;
    int pre_f = 0;
    for (unsigned w = 0; w < warp; ++w) {
        if (s_warp_f[w]) {
            pre_v = s_warp_v[w];
            pre_f = 1;
        } else {
            pre_v += s_warp_v[w];
        }
    }
    if (!f) v += pre_v;
    f |= pre_f;
    double ex_v = __shfl_up_sync(kFullMask, v, 1);
    int ex_f = __shfl_up_sync(kFullMask, f, 1);
    if (lane == 0) {
        ex_v = pre_v;
        ex_f = pre_f;
    }

    if (has_head) {
        double total = head_partial + ex_v;
        uint32_t row = r0 + head_local;
        // The tile's first row began in an earlier tile: finish it in the fix-up.
        if (!ex_f && s_off[pad(0)] < z0) {
            s_defer_row = row;
            s_defer_val = total;
        } else {
            pr_finish_row(row, total, s_off[pad(head_local + 1)] - s_off[pad(head_local)], rank_in, rank_out, contrib_out,
                          base, damp, spread, my_diff, my_dangle);
        }
    }
    if (threadIdx.x == kPrThreads - 1) {
        carry_row[t] = c1.x;
        carry_val[t] = v;
    }
    my_diff = block_sum(my_diff, scratch);
    my_dangle = block_sum(my_dangle, scratch);
    if (threadIdx.x == 0) {
        tile_diff[t] = my_diff;
        tile_dangle[t] = my_dangle;
        head_row[t] = s_defer_row;
        head_val[t] = s_defer_val;
    }
}

// Finishes rows that span tiles, then the last block reduces the per-tile and
// per-block partials in a fixed order and advances the iteration state.
__global__ void __launch_bounds__(256) pr_fixup_kernel(
    const uint32_t* __restrict__ offsets, uint64_t num_tiles, const float* __restrict__ rank_in,
    float* __restrict__ rank_out, float* __restrict__ contrib_out, uint32_t V, double base, double damp,
    PrState* __restrict__ state, double tolerance, const uint32_t* __restrict__ head_row,
    const double* __restrict__ head_val, const uint32_t* __restrict__ carry_row,
    const double* __restrict__ carry_val, const double* __restrict__ tile_diff,
    const double* __restrict__ tile_dangle, double* __restrict__ block_partials) {
    if (state->done) return;
    __shared__ double scratch[32];
    __shared__ bool s_last;
    const double spread = state->dangling / static_cast<double>(V);
    double d = 0.0, g = 0.0;
    uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < num_tiles) {
        d = tile_diff[t];
        g = tile_dangle[t];
        uint32_t row = head_row[t];
        if (row != kNoRow) {
            double sum = head_val[t];
            for (int64_t s = static_cast<int64_t>(t) - 1; s >= 0 && carry_row[s] == row; --s) sum += carry_val[s];
            pr_finish_row(row, sum, offsets[row + 1] - offsets[row], rank_in, rank_out, contrib_out, base, damp,
                          spread, d, g);
        }
    }
    d = block_sum(d, scratch);
    g = block_sum(g, scratch);
    if (threadIdx.x == 0) {
        block_partials[2 * blockIdx.x] = d;
        block_partials[2 * blockIdx.x + 1] = g;
        __threadfence();
        unsigned ticket = atomicAdd(&state->ticket, 1u);
        s_last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double dd = 0.0, gg = 0.0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        dd += __ldcg(block_partials + 2 * b);
        gg += __ldcg(block_partials + 2 * b + 1);
    }
    dd = block_sum(dd, scratch);
    gg = block_sum(gg, scratch);
    if (threadIdx.x == 0) {
        state->iterations += 1;
        state->last_diff = dd;
        state->dangling = gg;
        if (dd < tolerance) state->done = 1;
        state->ticket = 0;
    }
}

// ---------------------------------------------------------------- host

static Error ensure_plan(GraphImpl& g) {
    if (g.pr_plan) return ok();
    DeviceImpl& dev = *g.dev;
    auto plan = std::unique_ptr<PageRankPlan, void (*)(PageRankPlan*)>(new PageRankPlan, destroy_pagerank_plan);
    const uint32_t V = g.num_nodes, E = g.num_edges;
    const uint64_t total = static_cast<uint64_t>(V) + E;
    plan->num_tiles = ceil_div_u64(total, kPrTile);
    const uint64_t nt = plan->num_tiles;
    GCU_TRY(plan->coords.allocate(dev, nt + 1));
    GCU_TRY(plan->ranks.allocate(dev, 2 * static_cast<uint64_t>(V)));
    GCU_TRY(plan->contrib.allocate(dev, 2 * static_cast<uint64_t>(V)));
    GCU_TRY(plan->head_row.allocate(dev, nt));
    GCU_TRY(plan->head_val.allocate(dev, nt));
    GCU_TRY(plan->carry_row.allocate(dev, nt));
    GCU_TRY(plan->carry_val.allocate(dev, nt));
    GCU_TRY(plan->tile_diff.allocate(dev, nt));
    GCU_TRY(plan->tile_dangle.allocate(dev, nt));
    uint64_t fix_blocks = ceil_div_u64(nt, 256);
    uint64_t init_blocks = std::min<uint64_t>(ceil_div_u64(V, kPrThreads), static_cast<uint64_t>(dev.sm_count) * 8);
    GCU_TRY(plan->block_partials.allocate(dev, 2 * std::max(fix_blocks, init_blocks)));
    GCU_TRY(plan->state.allocate(dev, 1));
    GCU_CUDA(cudaMallocHost(reinterpret_cast<void**>(&plan->host_state), sizeof(PrState)), "cudaMallocHost");
    GCU_LAUNCH(dev, "pr_plan", pr_plan_kernel, static_cast<unsigned>(ceil_div_u64(nt + 1, 256)), 256, 0,
               g.offsets.ptr, V, E, nt, plan->coords.ptr);
    g.pr_plan = plan.release();
    return ok();
}

Error pagerank(GraphImpl& g, float damping, uint32_t max_iterations, float tolerance, float* host_ranks,
               uint32_t* iterations, bool* converged) {
    const uint32_t V = g.num_nodes;
    // pagerank.rs:56-63: no nodes, no ranks.
    if (V == 0) {
        *iterations = 0;
        *converged = true;
        return ok();
    }
    DeviceImpl& dev = *g.dev;
    GCU_TRY(ensure_plan(g));
    PageRankPlan& p = *g.pr_plan;
    const uint64_t nt = p.num_tiles;
    float* ranks[2] = {p.ranks.ptr, p.ranks.ptr + V};
    float* contrib[2] = {p.contrib.ptr, p.contrib.ptr + V};

    const float r0 = 1.0f / static_cast<float>(V);  // pagerank.rs:83
    const unsigned init_blocks =
        static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, kPrThreads), static_cast<uint64_t>(dev.sm_count) * 8));
    GCU_LAUNCH(dev, "pr_init", pr_init_kernel, init_blocks, kPrThreads, 0, g.offsets.ptr, V, r0, ranks[0],
               contrib[0], p.block_partials.ptr);
    GCU_LAUNCH(dev, "pr_init_reduce", pr_init_reduce_kernel, 1, 1024, 0, p.block_partials.ptr, init_blocks,
               p.state.ptr);

    const double damp = static_cast<double>(damping);
    const double base = (1.0 - damp) / static_cast<double>(V);
    const double tol = static_cast<double>(tolerance);
    const unsigned fix_blocks = static_cast<unsigned>(ceil_div_u64(nt, 256));

    // Queue iterations in chunks; the device stops itself once converged, so
    // the host only polls the state between chunks.
    uint32_t launched = 0;
    uint32_t chunk = 4;
    cudaEvent_t polled = nullptr;
    GCU_CUDA(cudaEventCreateWithFlags(&polled, cudaEventDisableTiming), "cudaEventCreate");
    bool stop = false;
    Error err = ok();
    while (launched < max_iterations && !stop) {
        uint32_t n = std::min(chunk, max_iterations - launched);
        for (uint32_t i = 0; i < n && err.ok(); ++i) {
            const uint32_t it = launched + i;
            const int in = it & 1, out = in ^ 1;
            err = [&]() -> Error {
                GCU_LAUNCH(dev, "pr_tile", pr_tile_kernel, static_cast<unsigned>(nt), kPrThreads, 0, g.offsets.ptr,
                           g.targets.ptr, p.coords.ptr, ranks[in], contrib[in], ranks[out], contrib[out], V, base,
                           damp, p.state.ptr, p.head_row.ptr, p.head_val.ptr, p.carry_row.ptr, p.carry_val.ptr,
                           p.tile_diff.ptr, p.tile_dangle.ptr);
                GCU_LAUNCH(dev, "pr_fixup", pr_fixup_kernel, fix_blocks, 256, 0, g.offsets.ptr, nt, ranks[in],
                           ranks[out], contrib[out], V, base, damp, p.state.ptr, tol, p.head_row.ptr, p.head_val.ptr,
                           p.carry_row.ptr, p.carry_val.ptr, p.tile_diff.ptr, p.tile_dangle.ptr,
                           p.block_partials.ptr);
                return ok();
            }();
        }
        if (!err.ok()) break;
        launched += n;
        cudaError_t c = cudaMemcpyAsync(p.host_state, p.state.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, dev.stream);
        if (c == cudaSuccess) c = cudaEventRecord(polled, dev.stream);
        if (c == cudaSuccess) c = cudaEventSynchronize(polled);
        if (c != cudaSuccess) {
            err = kernel_error(std::string("PageRank iteration failed: ") + cudaGetErrorString(c));
            break;
        }
        stop = p.host_state->done != 0;
        chunk = std::min<uint32_t>(chunk * 2, 64);
    }
    cudaEventDestroy(polled);
    GCU_TRY(err);
    GCU_TRY(dev.sync());
    if (launched == 0) {
        p.host_state->iterations = 0;
        p.host_state->done = 0;
    }
    const uint32_t iters = p.host_state->iterations;
    p.final_buffer = iters & 1;
    if (host_ranks) {
        GCU_CUDA(cudaMemcpyAsync(host_ranks, ranks[p.final_buffer], sizeof(float) * V, cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy ranks to host");
        GCU_TRY(dev.sync());
    }
    *iterations = iters;
    *converged = p.host_state->done != 0;
    return ok();
}

}  // namespace gcu
