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
//    owns one bitmap word of 32 vertices; a lane checks the first entries of
//    its vertex's list alone and longer lists are walked by the whole warp,
//    32 coalesced entries per step.
//  * Three step variants: push with one warp per frontier vertex (one
//    launch), load-balanced push (above), pull (above).
//  * Schedule: Beamer's alpha/beta rule (alpha = 14, beta = 24) over the
//    balanced push and the pull, fed by the frontier and unexplored edge
//    counts the steps emit; or, when a learned schedule is installed on the
//    device, a one-warp kernel after every step that turns the step's
//    counters into features and picks the variant with the smallest predicted
//    time (sched.cuh), with the alpha/beta rule as its fallback. The schedule
//    only changes which kernels run; BFS levels are unique, so the distances
//    cannot change.
//  * Trace mode (bfs_trace) times every valid variant at every level from the
//    same frontier: the training data of the learned schedule.
//  * Vertices without out-edges are counted and labelled but never queued.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"
#include "sched.cuh"

namespace gcu {

constexpr int kTdThreads = 256;
constexpr int kTdItems = 4;
constexpr int kTdTile = kTdThreads * kTdItems;  // frontier edges per block
constexpr int kBuThreads = 256;

struct BfsCounters {
    uint32_t discovered;  // vertices labelled this level
    uint32_t queued;      // of those, vertices with out-edges (appended to the queue)
    unsigned long long edges;  // sum of out-degrees of the vertices labelled this level
    int32_t choice;       // learned schedule's variant for the next step (-1: use the fixed rule)
    uint32_t pad;
};

// Step variants (the learned schedule's three outputs for a BFS level).
enum BfsVariant : int {
    kPushWarp = 0,      // top-down, one warp per frontier vertex, one launch
    kPushBalanced = 1,  // top-down, frontier edges split evenly over blocks (degrees + scan + expand)
    kPull = 2,          // bottom-up over the frontier bitmap (symmetric graphs only)
};

// Where a device-driven run stands between two steps (the device twin of the
// host loop's BfsState, kept in device memory and read by every step kernel).
struct BfsDevState {
    unsigned long long frontier_m;  // out-edges of the frontier
    unsigned long long unexplored;  // out-edges of vertices not labelled yet
    uint32_t frontier_n;            // vertices labelled by the last step
    uint32_t frontier_q;            // of those, queued (out-degree > 0)
    uint32_t reached;
    int32_t level;                  // level of the frontier
    uint32_t cur;                   // queue[cur] / bitmap[cur] hold the frontier
    uint32_t bitmap_valid;          // the last step was a pull: bitmap[cur] holds the frontier
    int32_t variant;                // the step the SWITCH node runs next (kSchedOut: none)
    uint32_t first;                 // the counters are the source's, not a step's
    uint32_t failed;                // the loop stopped on a state no search can reach
};

struct BfsWork {
    DeviceBuffer<int32_t> dist;
    DeviceBuffer<uint32_t> visited;
    DeviceBuffer<uint32_t> bitmap[2];
    DeviceBuffer<uint32_t> queue[2];
    DeviceBuffer<uint32_t> degree_scan;  // V + 1
    DeviceBuffer<BfsCounters> counters;
    BfsCounters host_counters{};  // host copy, read after a synchronisation (plain memory)
    int symmetric = -1;                    // -1 unknown, 0 no, 1 yes
    DeviceBuffer<uint32_t> active;         // vertices with edges, ascending (symmetric graphs)
    uint32_t n_active = 0;
    bool pull_list = false;                // the pull walks `active` instead of every bitmap word
    // device-driven level loop (built on first use, per schedule network)
    DeviceBuffer<BfsDevState> loop_state;
    DeviceBuffer<uint32_t> loop_scan_sums;
    BfsDevState host_loop_state{};  // host copy of the loop's final state (plain memory)
    cudaGraph_t loop_graph = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    const void* loop_net = nullptr;  // the schedule network the graph reads (NULL: fixed rule)
    bool loop_unavailable = false;   // the driver refused the graph: the host drives the levels
};

void destroy_bfs_work(BfsWork* w) {
    if (!w) return;
    if (w->loop_exec) cudaGraphExecDestroy(w->loop_exec);
    if (w->loop_graph) cudaGraphDestroy(w->loop_graph);
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

// Per-lane totals of what a lane labelled; a warp adds them to the level's
// counters once, when it is done (flush_tally), instead of one atomic pair on
// the same two words per warp step.
struct Tally {
    uint32_t found = 0;
    unsigned long long edges = 0;
};

// Labels v (found by a parent at this level) and records it; called by all
// lanes of a warp, `found` says whether this lane discovered a vertex.
__device__ __forceinline__ void record_discovery(bool found, uint32_t v, const uint32_t* __restrict__ offsets,
                                                 int32_t* __restrict__ dist, int32_t level,
                                                 uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr,
                                                 Tally& tally) {
    uint32_t deg = 0;
    if (found) {
        dist[v] = level;
        deg = offsets[v + 1] - offsets[v];
        tally.found += 1;
        tally.edges += deg;
    }
    if (__ballot_sync(kFullMask, found) == 0) return;
    append_warp(found && deg > 0, v, next_queue, &ctr->queued);
}

// All 32 lanes call it once, at the end of the kernel.
__device__ __forceinline__ void flush_tally(const Tally& tally, BfsCounters* __restrict__ ctr) {
    const uint32_t found = warp_sum(tally.found);
    const unsigned long long edges = warp_sum(tally.edges);
    if (lane_id() == 0) {
        if (found) atomicAdd(&ctr->discovered, found);
        if (edges) atomicAdd(&ctr->edges, edges);
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

// Top-down: the block expands frontier edges [e0, e0 + kTdTile) of `total`
// (every thread of the block calls it with the same tile).
__device__ __forceinline__ void topdown_tile(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                             const uint32_t* __restrict__ queue, uint32_t qsize,
                                             const uint32_t* __restrict__ qscan, uint32_t total, uint64_t e0,
                                             int32_t* __restrict__ dist, uint32_t* __restrict__ visited,
                                             uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr,
                                             int32_t next_level, Tally& tally) {
    __shared__ uint32_t s_scan[kTdTile + 1];
    __shared__ uint32_t s_start[kTdTile + 1];
    __shared__ uint32_t s_range[2];
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
        record_discovery(found, v, offsets, dist, next_level, next_queue, ctr, tally);
    }
}

// Top-down: block b expands frontier edges [b*kTdTile, (b+1)*kTdTile).
__global__ void __launch_bounds__(kTdThreads) bfs_topdown_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ queue,
    uint32_t qsize, const uint32_t* __restrict__ qscan, int32_t* __restrict__ dist, uint32_t* __restrict__ visited,
    uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr, int32_t next_level) {
    const uint32_t total = qscan[qsize];
    const uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kTdTile;
    if (e0 >= total) return;
    Tally tally;
    topdown_tile(offsets, targets, queue, qsize, qscan, total, e0, dist, visited, next_queue, ctr, next_level, tally);
    flush_tally(tally, ctr);
}

__global__ void bfs_queue_to_bitmap_kernel(const uint32_t* __restrict__ queue, uint32_t n,
                                           uint32_t* __restrict__ bitmap) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t u = queue[i];
        atomicOr(bitmap + (u >> 5), 1u << (u & 31));
    }
}

constexpr uint32_t kBuSolo = 8;  // entries a lane checks alone before its warp takes over the list
// The pull step walks the list of vertices with edges when at least
// 1 / kBuListFraction of the vertices are isolated (R-MAT 22: 43 %; list
// 7.5 % faster than the word form there, 10 % at R-MAT 24), and every word of
// the visited bitmap otherwise (Erdos-Renyi 2^22, almost no isolated vertex:
// the word form is 9 % faster, without the list's atomics and indirection).
constexpr uint32_t kBuListFraction = 8;

__device__ __forceinline__ bool in_frontier(const uint32_t* __restrict__ frontier, uint32_t u) {
    return (__ldg(frontier + (u >> 5)) >> (u & 31)) & 1u;
}

// Bottom-up: warp w handles the 32 vertices of bitmap word w. Each unvisited
// vertex first checks its first kBuSolo entries alone (4 loads in flight);
// most vertices that have a parent in a large frontier find it there. The
// lists that are left are then walked by the whole warp, one list at a time,
// 32 consecutive entries per step (coalesced) with a ballot to stop at the
// first parent, so a long list neither serialises one lane nor stalls the
// other 31.
// Whether this lane's vertex (list [s, e); e == s: nothing to probe) has a
// neighbour in the frontier. Called by all 32 lanes: the lists left after
// the solo probes are walked by the whole warp.
__device__ __forceinline__ bool probe_parent(uint32_t s, uint32_t e, const uint32_t* __restrict__ frontier,
                                             const uint32_t* __restrict__ targets) {
    const unsigned lane = lane_id();
    bool found = false;
    const uint32_t solo = min(e - s, kBuSolo);
    for (uint32_t k = 0; k < solo && !found; k += 4) {
        uint32_t t[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = k + q < solo ? targets[s + k + q] : 0xFFFFFFFFu;
#pragma unroll
        for (int q = 0; q < 4; ++q) found = found || (t[q] != 0xFFFFFFFFu && in_frontier(frontier, t[q]));
    }
    unsigned pending = __ballot_sync(kFullMask, !found && e - s > kBuSolo);
    while (pending) {
        const int p = __ffs(pending) - 1;
        pending &= pending - 1;
        const uint64_t ps = static_cast<uint64_t>(__shfl_sync(kFullMask, s, p)) + kBuSolo;
        const uint64_t pe = __shfl_sync(kFullMask, e, p);
        bool hit = false;
        for (uint64_t base = ps; base < pe; base += 32) {
            const uint64_t j = base + lane;
            const bool h = j < pe && in_frontier(frontier, targets[j]);
            if (__ballot_sync(kFullMask, h)) {
                hit = true;
                break;
            }
        }
        if (static_cast<int>(lane) == p) found = hit;
    }
    return found;
}

// Word form: warp w handles the 32 vertices of bitmap word w (it owns that
// word of `visited` and writes the word of `next_frontier`, found or not).
__device__ __forceinline__ void bottomup_body(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t V,
    const uint32_t* __restrict__ frontier, uint32_t* __restrict__ next_frontier, uint32_t* __restrict__ visited,
    int32_t* __restrict__ dist, uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr,
    int32_t next_level) {
    const unsigned lane = lane_id();
    const uint64_t words = ceil_div_u64(V, 32);
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    Tally tally;
    for (uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < words; w += warps) {
        // The word's visited bits and its lanes' list bounds, loaded side by
        // side (the bounds of visited vertices are read too, then ignored).
        const uint32_t vis = visited[w];
        const uint32_t v = static_cast<uint32_t>(w * 32 + lane);
        uint32_t s = 0, e = 0;
        if (v < V) {
            s = offsets[v];
            e = offsets[v + 1];
        }
        const bool open = v < V && !((vis >> lane) & 1u);
        if (!open) e = s;
        const bool found = probe_parent(s, e, frontier, targets);
        const unsigned mask = __ballot_sync(kFullMask, found);
        if (lane == 0) {
            next_frontier[w] = mask;
            if (mask) visited[w] = vis | mask;
        }
        record_discovery(found, v, offsets, dist, next_level, next_queue, ctr, tally);
    }
    flush_tally(tally, ctr);
}

// List form: the warps stride over the graph's vertices with edges (`active`,
// ascending), 32 at a time, so no lane sits on an isolated vertex (43 % of
// R-MAT 22's). A word of the bitmaps can span two warps' batches, so found
// vertices set their bits with atomicOr; the caller clears next_frontier.
__device__ __forceinline__ void bottomup_list_body(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
    const uint32_t* __restrict__ active, uint32_t n_active, const uint32_t* __restrict__ frontier,
    uint32_t* __restrict__ next_frontier, uint32_t* visited, int32_t* __restrict__ dist,
    uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr, int32_t next_level) {
    const unsigned lane = lane_id();
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    Tally tally;
    for (uint64_t base = ((static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * 32; base < n_active;
         base += warps * 32) {
        const uint64_t i = base + lane;
        uint32_t v = 0, s = 0, e = 0;
        bool open = false;
        if (i < n_active) {
            v = active[i];
            // Only this lane sets its vertex's bit, so a word another warp is
            // updating still shows this bit as it is.
            const uint32_t vis = visited[v >> 5];
            s = offsets[v];
            e = offsets[v + 1];
            open = !((vis >> (v & 31)) & 1u);
        }
        if (!open) e = s;
        const bool found = probe_parent(s, e, frontier, targets);
        if (found) {
            const uint32_t bit = 1u << (v & 31);
            atomicOr(next_frontier + (v >> 5), bit);
            atomicOr(visited + (v >> 5), bit);
        }
        record_discovery(found, v, offsets, dist, next_level, next_queue, ctr, tally);
    }
    flush_tally(tally, ctr);
}

// One instantiation per pull form (kList: walk `active`; else every bitmap
// word), so that each keeps its own body's register count: the word form
// needs 32 registers, a kernel holding both bodies 38, which costs a quarter
// of the resident warps of whichever form runs.
template <bool kList>
__global__ void __launch_bounds__(kBuThreads) bfs_bottomup_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t V,
    const uint32_t* __restrict__ active, uint32_t n_active, const uint32_t* __restrict__ frontier,
    uint32_t* __restrict__ next_frontier, uint32_t* __restrict__ visited, int32_t* __restrict__ dist,
    uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ ctr, int32_t next_level) {
    if (kList)
        bottomup_list_body(offsets, targets, active, n_active, frontier, next_frontier, visited, dist, next_queue, ctr,
                           next_level);
    else
        bottomup_body(offsets, targets, V, frontier, next_frontier, visited, dist, next_queue, ctr, next_level);
}

// Top-down, one warp per frontier vertex (no degree scan: one launch, for
// frontiers whose edges are few or evenly spread).
__device__ __forceinline__ void topdown_warp_body(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ queue,
    uint32_t qsize, int32_t* __restrict__ dist, uint32_t* __restrict__ visited, uint32_t* __restrict__ next_queue,
    BfsCounters* __restrict__ ctr, int32_t next_level) {
    const unsigned lane = lane_id();
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    Tally tally;
    for (uint64_t i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; i < qsize; i += nwarps) {
        const uint32_t u = queue[i];
        const uint64_t s = offsets[u], e = offsets[u + 1];
        for (uint64_t b = s; b < e; b += 32) {
            const uint64_t j = b + lane;
            bool found = false;
            uint32_t v = 0;
            if (j < e) {
                v = ld_stream(targets + j);
                const uint32_t bit = 1u << (v & 31);
                if (!(__ldcg(visited + (v >> 5)) & bit)) found = !(atomicOr(visited + (v >> 5), bit) & bit);
            }
            record_discovery(found, v, offsets, dist, next_level, next_queue, ctr, tally);
        }
    }
    flush_tally(tally, ctr);
}

__global__ void __launch_bounds__(kTdThreads) bfs_topdown_warp_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint32_t* __restrict__ queue,
    uint32_t qsize, int32_t* __restrict__ dist, uint32_t* __restrict__ visited, uint32_t* __restrict__ next_queue,
    BfsCounters* __restrict__ ctr, int32_t next_level) {
    topdown_warp_body(offsets, targets, queue, qsize, dist, visited, next_queue, ctr, next_level);
}

// Beamer's direction-optimising thresholds (Beamer, Asanovic and Patterson,
// SC'12): pull when the frontier's edges exceed the unexplored edges / alpha,
// back to push when the frontier falls below V / beta.
constexpr int kAlpha = 14;
constexpr int kBeta = 24;

// Beamer's direction rule over the balanced push and the pull, from the
// state after a step: the fixed schedule, the fallback of the learned one,
// and the variant the learned pick has to beat by a margin.
__host__ __device__ __forceinline__ int bfs_fixed_variant(bool symmetric, bool bottom_up, uint64_t frontier_n,
                                                          uint64_t frontier_m, uint64_t unexplored, uint32_t V) {
    const double alpha = kAlpha, beta = kBeta;
    if (!symmetric) return kPushBalanced;
    if (!bottom_up && static_cast<double>(frontier_m) > static_cast<double>(unexplored) / alpha) return kPull;
    if (bottom_up && static_cast<double>(frontier_n) < static_cast<double>(V) / beta) return kPushBalanced;
    return bottom_up ? kPull : kPushBalanced;
}

// One warp: the features of the decision before expanding the frontier the
// last step produced (its counters, plus the host's totals before that step),
// written to features_out when given; with a network, the chosen variant goes
// to ctr->choice for the host to read with the counters.
__global__ void bfs_decide_kernel(const __nv_bfloat16* __restrict__ w, BfsCounters* __restrict__ ctr,
                                  DegreeStats stats, unsigned long long prior_unexplored, uint32_t prior_reached,
                                  int32_t frontier_level, int frontier_bitmap, unsigned valid_mask, uint32_t num_nodes,
                                  float* __restrict__ features_out) {
    const BfsCounters c = *ctr;
    float f[kSchedIn];
    bfs_features(f, static_cast<float>(c.discovered), static_cast<float>(c.edges),
                 static_cast<float>(prior_unexplored - c.edges), frontier_level, stats, frontier_bitmap != 0,
                 static_cast<float>(prior_reached + c.discovered));
    if (features_out && lane_id() == 0)
        for (int k = 0; k < kSchedIn; ++k) features_out[k] = f[k];
    if (w) {
        float out[kSchedOut];
        sched_forward_warp(w, f, out);
        const int fixed = bfs_fixed_variant((valid_mask >> kPull) & 1u, frontier_bitmap != 0, c.discovered, c.edges,
                                            prior_unexplored - c.edges, num_nodes);
        if (lane_id() == 0) ctr->choice = sched_pick_over(out, valid_mask, fixed);
    }
}

// ---------------------------------------------------------------- device-driven level loop
//
// The host-driven loop reads the level counters back after every step (one
// copy and one synchronisation per level). The device-driven loop runs a
// whole search as one CUDA graph: a WHILE node whose body is a one-warp
// decide kernel followed by a SWITCH node over the three step variants. The
// decide kernel folds the last step's counters into BfsDevState exactly as
// the host's `advance` does, ends the loop where the host loop stops (empty
// frontier, or a step that labelled nothing), picks the next variant (the
// alpha/beta rule, or the learned schedule with its margin), and sets the
// SWITCH value; each step kernel reads its frontier size, level and queue
// parity from the state. The grids are fixed when the graph is captured and
// the kernels stride over what the state holds.

__global__ void bfs_loop_init_kernel(const uint32_t* __restrict__ offsets, uint32_t source,
                                     int32_t* __restrict__ dist, uint32_t* __restrict__ visited,
                                     uint32_t* __restrict__ queue0, BfsCounters* __restrict__ ctr,
                                     BfsDevState* __restrict__ st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    dist[source] = 0;
    visited[source >> 5] |= 1u << (source & 31);
    const uint32_t deg = offsets[source + 1] - offsets[source];
    queue0[0] = source;
    BfsCounters c{};
    c.discovered = 1;
    c.queued = deg > 0 ? 1u : 0u;
    c.edges = deg;
    *ctr = c;
    BfsDevState s{};
    s.first = 1;
    s.variant = kSchedOut;
    *st = s;
}

__global__ void bfs_loop_decide_kernel(const __nv_bfloat16* __restrict__ w, BfsCounters* __restrict__ ctr,
                                       BfsDevState* __restrict__ st, DegreeStats stats, unsigned long long num_edges,
                                       uint32_t V, unsigned valid_mask, cudaGraphConditionalHandle h_loop,
                                       cudaGraphConditionalHandle h_step) {
    const BfsCounters c = *ctr;
    BfsDevState s = *st;
    bool stop = false;
    if (s.first) {
        s.first = 0;
        s.unexplored = num_edges - c.edges;
        s.reached = 1;
        s.level = 0;
    } else if (c.discovered == 0) {
        stop = true;  // the step labelled nothing: level and reached stay
    } else {
        s.level += 1;
        s.reached += c.discovered;
        s.unexplored -= c.edges;
        s.cur ^= 1u;
        s.bitmap_valid = s.variant == kPull ? 1u : 0u;
    }
    if (!stop) {
        s.frontier_n = c.discovered;
        s.frontier_q = c.queued;
        s.frontier_m = c.edges;
        stop = s.frontier_q == 0;
    }
    // A search labels each vertex once, so it ends within V levels with at
    // most V vertices reached and at most V queued; state past these bounds
    // can only come from a fault, and it ends the loop with the error flag
    // set instead of looping or indexing past the queues.
    if (!stop && (static_cast<uint64_t>(s.level) >= V || s.reached > V || s.frontier_q > V)) {
        stop = true;
        s.failed = 1;
    }
    int variant = kSchedOut;
    if (!stop) {
        variant = bfs_fixed_variant((valid_mask >> kPull) & 1u, s.bitmap_valid != 0, s.frontier_n, s.frontier_m,
                                    s.unexplored, V);
        if (w) {
            float f[kSchedIn];
            bfs_features(f, static_cast<float>(s.frontier_n), static_cast<float>(s.frontier_m),
                         static_cast<float>(s.unexplored), s.level, stats, s.bitmap_valid != 0,
                         static_cast<float>(s.reached));
            float out[kSchedOut];
            sched_forward_warp(w, f, out);
            const int pick = sched_pick_over(out, valid_mask, variant);
            if (pick >= 0) variant = pick;
        }
    }
    __syncwarp();
    if (lane_id() == 0) {
        s.variant = variant;
        *st = s;
        *ctr = BfsCounters{};
        cudaGraphSetConditional(h_step, static_cast<unsigned>(variant));
        cudaGraphSetConditional(h_loop, stop ? 0u : 1u);
    }
}

__global__ void __launch_bounds__(kTdThreads) bfs_topdown_warp_loop_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t* queue0, uint32_t* queue1,
    int32_t* __restrict__ dist, uint32_t* __restrict__ visited, BfsCounters* __restrict__ ctr,
    const BfsDevState* __restrict__ st) {
    const uint32_t cur = st->cur;
    topdown_warp_body(offsets, targets, cur ? queue1 : queue0, st->frontier_q, dist, visited, cur ? queue0 : queue1,
                      ctr, st->level + 1);
}

// Also sets the IF node that picks the scan: three kernels above
// kScanOneLaunchMax frontier vertices, one below.
__global__ void bfs_queue_degrees_loop_kernel(const uint32_t* __restrict__ offsets, const uint32_t* queue0,
                                              const uint32_t* queue1, const BfsDevState* __restrict__ st,
                                              uint32_t* __restrict__ deg, int set_big,
                                              cudaGraphConditionalHandle h_big) {
    const uint32_t* queue = st->cur ? queue1 : queue0;
    const uint32_t n = st->frontier_q;
    if (set_big && blockIdx.x == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(h_big, n > kScanOneLaunchMax ? 1u : 0u);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = queue[i];
        deg[i] = offsets[u + 1] - offsets[u];
    }
}

// Balanced top-down over the scanned frontier degrees: blocks stride over the
// kTdTile-edge tiles of the frontier.
__global__ void __launch_bounds__(kTdThreads) bfs_topdown_loop_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t* queue0, uint32_t* queue1,
    const uint32_t* __restrict__ qscan, int32_t* __restrict__ dist, uint32_t* __restrict__ visited,
    BfsCounters* __restrict__ ctr, const BfsDevState* __restrict__ st) {
    const uint32_t cur = st->cur, qsize = st->frontier_q;
    const int32_t next_level = st->level + 1;
    const uint32_t total = qscan[qsize];
    const uint32_t* queue = cur ? queue1 : queue0;
    uint32_t* next_queue = cur ? queue0 : queue1;
    Tally tally;
    const uint64_t tiles = ceil_div_u64(total, kTdTile);
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        topdown_tile(offsets, targets, queue, qsize, qscan, total, t * kTdTile, dist, visited, next_queue, ctr,
                     next_level, tally);
        __syncthreads();  // the tile's shared arrays are reused by the next tile
    }
    flush_tally(tally, ctr);
}

// Before a pull that follows a push: the frontier bitmap from the queue.
__global__ void bfs_bitmap_clear_loop_kernel(uint32_t* bitmap0, uint32_t* bitmap1, uint64_t words,
                                             const BfsDevState* __restrict__ st) {
    if (st->bitmap_valid) return;
    uint32_t* bitmap = st->cur ? bitmap1 : bitmap0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < words;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        bitmap[i] = 0;
}

__global__ void bfs_queue_to_bitmap_loop_kernel(const uint32_t* queue0, const uint32_t* queue1, uint32_t* bitmap0,
                                                uint32_t* bitmap1, const BfsDevState* __restrict__ st) {
    if (st->bitmap_valid) return;
    const uint32_t* queue = st->cur ? queue1 : queue0;
    uint32_t* bitmap = st->cur ? bitmap1 : bitmap0;
    const uint32_t n = st->frontier_q;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = queue[i];
        atomicOr(bitmap + (u >> 5), 1u << (u & 31));
    }
}

template <bool kList>  // one instantiation per pull form, as bfs_bottomup_kernel
__global__ void __launch_bounds__(kBuThreads) bfs_bottomup_loop_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, uint32_t V,
    const uint32_t* __restrict__ active, uint32_t n_active, uint32_t* bitmap0, uint32_t* bitmap1,
    uint32_t* __restrict__ visited, int32_t* __restrict__ dist, uint32_t* queue0, uint32_t* queue1,
    BfsCounters* __restrict__ ctr, const BfsDevState* __restrict__ st) {
    const uint32_t cur = st->cur;
    if (kList)
        bottomup_list_body(offsets, targets, active, n_active, cur ? bitmap1 : bitmap0, cur ? bitmap0 : bitmap1,
                           visited, dist, cur ? queue0 : queue1, ctr, st->level + 1);
    else
        bottomup_body(offsets, targets, V, cur ? bitmap1 : bitmap0, cur ? bitmap0 : bitmap1, visited, dist,
                      cur ? queue0 : queue1, ctr, st->level + 1);
}

// The list form of the pull sets only found bits: clear the bitmap it fills.
__global__ void bfs_next_bitmap_clear_loop_kernel(uint32_t* bitmap0, uint32_t* bitmap1, uint64_t words,
                                                  const BfsDevState* __restrict__ st) {
    uint32_t* bitmap = st->cur ? bitmap0 : bitmap1;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < words;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        bitmap[i] = 0;
}

// ---------------------------------------------------------------- host

// The vertices with at least one entry, ascending (flags, scan, scatter).
__global__ void bfs_has_edges_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t* __restrict__ flags) {
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        flags[v] = offsets[v + 1] > offsets[v] ? 1u : 0u;
}

__global__ void bfs_active_scatter_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                          const uint32_t* __restrict__ pos, uint32_t* __restrict__ active) {
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (offsets[v + 1] > offsets[v]) active[pos[v]] = static_cast<uint32_t>(v);
}

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
    // Bottom-up steps read in-neighbours; they equal the CSR lists only when
    // the CSR is symmetric (checked once per graph).
    bool sym = false;
    GCU_TRY(graph_symmetry(g, &sym));
    w->symmetric = sym ? 1 : 0;
    if (sym && V > 0) {
        // degree_scan is free until the first balanced push: flags, then positions.
        const unsigned grid = static_cast<unsigned>(
            std::min<uint64_t>(ceil_div_u64(V, 256), static_cast<uint64_t>(dev.sm_count) * 16));
        GCU_LAUNCH(dev, "bfs_has_edges", bfs_has_edges_kernel, grid, 256, 0, g.offsets.ptr, static_cast<uint32_t>(V),
                   w->degree_scan.ptr);
        GCU_TRY(exclusive_scan_u32(dev, w->degree_scan.ptr, w->degree_scan.ptr, V));
        uint32_t n = 0;
        GCU_CUDA(cudaMemcpyAsync(&n, w->degree_scan.ptr + V, sizeof(n), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        w->n_active = n;
        w->pull_list = V - n >= V / kBuListFraction;
        if (w->pull_list) {
            GCU_TRY(w->active.allocate(dev, std::max<uint32_t>(n, 1)));
            GCU_LAUNCH(dev, "bfs_active_scatter", bfs_active_scatter_kernel, grid, 256, 0, g.offsets.ptr,
                       static_cast<uint32_t>(V), w->degree_scan.ptr, w->active.ptr);
        }
    }
    g.bfs_work = w.release();
    return ok();
}

namespace {

// Where a level-synchronous run stands between two steps.
struct BfsState {
    uint32_t frontier_n = 0;    // vertices labelled by the last step
    uint32_t frontier_q = 0;    // of those, queued (out-degree > 0)
    uint64_t frontier_m = 0;    // their out-edges
    uint64_t unexplored = 0;    // out-edges of vertices not labelled yet
    uint32_t reached = 0;
    int32_t level = 0;          // level of the frontier
    int cur = 0;                // queue[cur] / bitmap[cur] hold the frontier
    bool bottom_up = false;     // the last step was a pull
    bool bitmap_valid = false;  // bitmap[cur] holds the frontier
};

int fixed_rule(const BfsState& st, bool symmetric, uint32_t V) {
    return bfs_fixed_variant(symmetric, st.bottom_up, st.frontier_n, st.frontier_m, st.unexplored, V);
}

unsigned valid_variants(bool symmetric) {
    return (1u << kPushWarp) | (1u << kPushBalanced) | (symmetric ? (1u << kPull) : 0u);
}

// Launches one step of `variant` from the frontier in st (counters reset).
Error launch_step(GraphImpl& g, BfsWork& w, int variant, const BfsState& st) {
    DeviceImpl& dev = *g.dev;
    const uint32_t V = g.num_nodes;
    const uint64_t words = ceil_div_u64(V, 32);
    const unsigned grid_cap = static_cast<unsigned>(dev.sm_count) * 16;
    const int cur = st.cur, nxt = cur ^ 1;
    GCU_CUDA(cudaMemsetAsync(w.counters.ptr, 0, sizeof(BfsCounters), dev.stream), "memset");
    if (variant == kPull) {
        if (!st.bitmap_valid) {
            GCU_CUDA(cudaMemsetAsync(w.bitmap[cur].ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
            unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(st.frontier_q, 256), grid_cap));
            GCU_LAUNCH(dev, "bfs_queue_to_bitmap", bfs_queue_to_bitmap_kernel, blocks, 256, 0, w.queue[cur].ptr,
                       st.frontier_q, w.bitmap[cur].ptr);
        }
        const uint64_t lanes = w.pull_list ? w.n_active : words * 32;
        if (w.pull_list)
            GCU_CUDA(cudaMemsetAsync(w.bitmap[nxt].ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
        unsigned blocks = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(lanes, kBuThreads), grid_cap)));
        const auto bottomup = w.pull_list ? bfs_bottomup_kernel<true> : bfs_bottomup_kernel<false>;
        GCU_LAUNCH(dev, "bfs_bottomup", bottomup, blocks, kBuThreads, 0, g.offsets.ptr, g.targets.ptr, V,
                   w.pull_list ? w.active.ptr : nullptr, w.n_active, w.bitmap[cur].ptr, w.bitmap[nxt].ptr, w.visited.ptr, w.dist.ptr,
                   w.queue[nxt].ptr, w.counters.ptr, st.level + 1);
    } else if (variant == kPushWarp) {
        unsigned blocks = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(st.frontier_q, kTdThreads / 32), grid_cap)));
        GCU_LAUNCH(dev, "bfs_topdown_warp", bfs_topdown_warp_kernel, blocks, kTdThreads, 0, g.offsets.ptr,
                   g.targets.ptr, w.queue[cur].ptr, st.frontier_q, w.dist.ptr, w.visited.ptr, w.queue[nxt].ptr,
                   w.counters.ptr, st.level + 1);
    } else {
        unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(st.frontier_q, 256), grid_cap));
        GCU_LAUNCH(dev, "bfs_queue_degrees", bfs_queue_degrees_kernel, blocks, 256, 0, g.offsets.ptr,
                   w.queue[cur].ptr, st.frontier_q, w.degree_scan.ptr);
        GCU_TRY(exclusive_scan_u32(dev, w.degree_scan.ptr, w.degree_scan.ptr, st.frontier_q));
        unsigned td_blocks = static_cast<unsigned>(std::max<uint64_t>(1, ceil_div_u64(st.frontier_m, kTdTile)));
        GCU_LAUNCH(dev, "bfs_topdown", bfs_topdown_kernel, td_blocks, kTdThreads, 0, g.offsets.ptr, g.targets.ptr,
                   w.queue[cur].ptr, st.frontier_q, w.degree_scan.ptr, w.dist.ptr, w.visited.ptr, w.queue[nxt].ptr,
                   w.counters.ptr, st.level + 1);
    }
    return ok();
}

// Resets the work buffers and labels the source; st describes level 0.
Error start_run(GraphImpl& g, BfsWork& w, uint32_t source) {
    DeviceImpl& dev = *g.dev;
    const uint64_t words = ceil_div_u64(g.num_nodes, 32);
    GCU_CUDA(cudaMemsetAsync(w.dist.ptr, 0xFF, sizeof(int32_t) * g.num_nodes, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(w.visited.ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(w.counters.ptr, 0, sizeof(BfsCounters), dev.stream), "memset");
    GCU_LAUNCH(dev, "bfs_init", bfs_init_kernel, 1, 32, 0, g.offsets.ptr, source, w.dist.ptr, w.visited.ptr,
               w.queue[0].ptr, w.counters.ptr);
    return ok();
}

Error read_counters(DeviceImpl& dev, BfsWork& w) {
    GCU_CUDA(cudaMemcpyAsync(&w.host_counters, w.counters.ptr, sizeof(BfsCounters), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    return dev.sync();
}

// Folds the counters of the step just run (or of the init) into st.
void advance(BfsState& st, const BfsCounters& c, bool first, int variant, uint64_t num_edges) {
    if (first) {
        st.unexplored = num_edges - c.edges;
        st.reached = 1;
        st.level = 0;
    } else {
        st.level += 1;
        st.reached += c.discovered;
        st.unexplored -= c.edges;
        st.cur ^= 1;
        st.bottom_up = variant == kPull;
        st.bitmap_valid = variant == kPull;
    }
    st.frontier_n = c.discovered;
    st.frontier_q = c.queued;
    st.frontier_m = c.edges;
}

// Captures the launches `f` makes on the device stream into `target` (a
// conditional node's body graph), after the node `after` when given.
template <class F>
Error capture_into(DeviceImpl& dev, cudaGraph_t target, F&& f, const cudaGraphNode_t* after = nullptr) {
    GCU_CUDA(cudaStreamBeginCaptureToGraph(dev.stream, target, after, nullptr, after ? 1 : 0,
                                           cudaStreamCaptureModeThreadLocal),
             "cudaStreamBeginCaptureToGraph");
    const Error e = f();
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(dev.stream, &captured);
    GCU_TRY(e);
    if (ce != cudaSuccess) return driver_error(ce, "cudaStreamEndCapture");
    return ok();
}

// The graph of a device-driven search: WHILE(loop) { decide; SWITCH(step) {
// push with a warp per vertex | balanced push | pull } }. Everything it reads
// lives in the BfsWork buffers and the graph's CSR; the source is labelled by
// bfs_loop_init_kernel before each launch.
Error build_loop_graph(GraphImpl& g, BfsWork& w) {
    DeviceImpl& dev = *g.dev;
    if (w.loop_exec) {
        cudaGraphExecDestroy(w.loop_exec);
        w.loop_exec = nullptr;
    }
    if (w.loop_graph) {
        cudaGraphDestroy(w.loop_graph);
        w.loop_graph = nullptr;
    }
    const uint32_t V = g.num_nodes;
    const uint64_t words = ceil_div_u64(V, 32);
    if (!w.loop_state.ptr) {
        GCU_TRY(w.loop_state.allocate(dev, 1));
        GCU_TRY(w.loop_scan_sums.allocate(dev, scan_device_n_tiles(V)));
    }
    const __nv_bfloat16* net = reinterpret_cast<const __nv_bfloat16*>(dev.schedule);
    DegreeStats stats;
    if (net) GCU_TRY(degree_stats(g, &stats));
    const bool sym = w.symmetric == 1;
    const unsigned valid = valid_variants(sym);
    BfsDevState* st = w.loop_state.ptr;
    const uint32_t* n_ptr = &st->frontier_q;
    const unsigned cap = static_cast<unsigned>(dev.sm_count) * 16;
    const unsigned vgrid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(V, 256), cap)));
    const unsigned bu_grid = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div_u64(w.pull_list ? w.n_active : words * 32, kBuThreads), cap)));
    const unsigned wgrid =
        static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(V, kTdThreads / 32), cap)));
    const unsigned td_grid = static_cast<unsigned>(dev.sm_count) * 8;

    cudaGraph_t graph = nullptr;
    GCU_CUDA(cudaGraphCreate(&graph, 0), "cudaGraphCreate");
    struct Owner {
        cudaGraph_t g;
        ~Owner() {
            if (g) cudaGraphDestroy(g);
        }
    } owner{graph};
    cudaGraphConditionalHandle h_loop = 0, h_step = 0;
    GCU_CUDA(cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault),
             "cudaGraphConditionalHandleCreate");
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t while_node = nullptr;
    GCU_CUDA(cudaGraphAddNode(&while_node, graph, nullptr, 0, &wp), "cudaGraphAddNode (while)");
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    GCU_CUDA(cudaGraphConditionalHandleCreate(&h_step, body, 0, 0), "cudaGraphConditionalHandleCreate");
    GCU_TRY(capture_into(dev, body, [&]() -> Error {
        GCU_LAUNCH(dev, "bfs_loop_decide", bfs_loop_decide_kernel, 1, 32, 0, net, w.counters.ptr, st, stats,
                   static_cast<unsigned long long>(g.num_edges), V, valid, h_loop, h_step);
        return ok();
    }));
    cudaGraphNode_t decide_node = nullptr;
    size_t nodes = 1;
    GCU_CUDA(cudaGraphGetNodes(body, &decide_node, &nodes), "cudaGraphGetNodes");
    if (nodes != 1) return kernel_error("BFS loop graph: unexpected body");
    cudaGraphNodeParams sp = {};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = h_step;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = kSchedOut;
    cudaGraphNode_t switch_node = nullptr;
    GCU_CUDA(cudaGraphAddNode(&switch_node, body, &decide_node, 1, &sp), "cudaGraphAddNode (switch)");
    cudaGraph_t* branch = sp.conditional.phGraph_out;
    GCU_TRY(capture_into(dev, branch[kPushWarp], [&]() -> Error {
        GCU_LAUNCH(dev, "bfs_topdown_warp", bfs_topdown_warp_loop_kernel, wgrid, kTdThreads, 0, g.offsets.ptr,
                   g.targets.ptr, w.queue[0].ptr, w.queue[1].ptr, w.dist.ptr, w.visited.ptr, w.counters.ptr, st);
        return ok();
    }));
    // Balanced push: degrees (which set the scan's IF), IF(n > 8192) { three-kernel
    // scan } ELSE { one-kernel scan }, expand. Graphs of at most 8192
    // vertices only ever take the one-kernel scan: no IF node.
    cudaGraph_t balanced = branch[kPushBalanced];
    const bool big = V > kScanOneLaunchMax;
    cudaGraphConditionalHandle h_big = 0;
    if (big)
        GCU_CUDA(cudaGraphConditionalHandleCreate(&h_big, balanced, 0, 0), "cudaGraphConditionalHandleCreate");
    auto launch_expand = [&]() -> Error {
        GCU_LAUNCH(dev, "bfs_topdown", bfs_topdown_loop_kernel, td_grid, kTdThreads, 0, g.offsets.ptr, g.targets.ptr,
                   w.queue[0].ptr, w.queue[1].ptr, w.degree_scan.ptr, w.dist.ptr, w.visited.ptr, w.counters.ptr, st);
        return ok();
    };
    GCU_TRY(capture_into(dev, balanced, [&]() -> Error {
        GCU_LAUNCH(dev, "bfs_queue_degrees", bfs_queue_degrees_loop_kernel, vgrid, 256, 0, g.offsets.ptr,
                   w.queue[0].ptr, w.queue[1].ptr, st, w.degree_scan.ptr, big ? 1 : 0, h_big);
        if (big) return ok();
        GCU_TRY(exclusive_scan_u32_device_n(dev, w.degree_scan.ptr, w.degree_scan.ptr, n_ptr, V,
                                            w.loop_scan_sums.ptr, ScanLaunches::kOneTile));
        return launch_expand();
    }));
    if (big) {
        cudaGraphNode_t degrees_node = nullptr;
        nodes = 1;
        GCU_CUDA(cudaGraphGetNodes(balanced, &degrees_node, &nodes), "cudaGraphGetNodes");
        if (nodes != 1) return kernel_error("BFS loop graph: unexpected balanced branch");
        cudaGraphNodeParams ip = {};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = h_big;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 2;
        cudaGraphNode_t if_node = nullptr;
        GCU_CUDA(cudaGraphAddNode(&if_node, balanced, &degrees_node, 1, &ip), "cudaGraphAddNode (if)");
        GCU_TRY(capture_into(dev, ip.conditional.phGraph_out[0], [&]() -> Error {
            return exclusive_scan_u32_device_n(dev, w.degree_scan.ptr, w.degree_scan.ptr, n_ptr, V,
                                               w.loop_scan_sums.ptr, ScanLaunches::kMultiTile);
        }));
        GCU_TRY(capture_into(dev, ip.conditional.phGraph_out[1], [&]() -> Error {
            return exclusive_scan_u32_device_n(dev, w.degree_scan.ptr, w.degree_scan.ptr, n_ptr, V,
                                               w.loop_scan_sums.ptr, ScanLaunches::kOneTile);
        }));
        GCU_TRY(capture_into(dev, balanced, launch_expand, &if_node));
    }
    GCU_TRY(capture_into(dev, branch[kPull], [&]() -> Error {
        GCU_LAUNCH(dev, "bfs_bitmap_clear", bfs_bitmap_clear_loop_kernel, vgrid, 256, 0, w.bitmap[0].ptr,
                   w.bitmap[1].ptr, words, st);
        GCU_LAUNCH(dev, "bfs_queue_to_bitmap", bfs_queue_to_bitmap_loop_kernel, vgrid, 256, 0, w.queue[0].ptr,
                   w.queue[1].ptr, w.bitmap[0].ptr, w.bitmap[1].ptr, st);
        if (w.pull_list)
            GCU_LAUNCH(dev, "bfs_next_bitmap_clear", bfs_next_bitmap_clear_loop_kernel, vgrid, 256, 0,
                       w.bitmap[0].ptr, w.bitmap[1].ptr, words, st);
        const auto bottomup = w.pull_list ? bfs_bottomup_loop_kernel<true> : bfs_bottomup_loop_kernel<false>;
        GCU_LAUNCH(dev, "bfs_bottomup", bottomup, bu_grid, kBuThreads, 0, g.offsets.ptr,
                   g.targets.ptr, V, w.pull_list ? w.active.ptr : nullptr, w.n_active, w.bitmap[0].ptr, w.bitmap[1].ptr, w.visited.ptr,
                   w.dist.ptr, w.queue[0].ptr, w.queue[1].ptr, w.counters.ptr, st);
        return ok();
    }));
    cudaGraphExec_t exec = nullptr;
    GCU_CUDA(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    w.loop_graph = graph;
    owner.g = nullptr;
    w.loop_exec = exec;
    w.loop_net = net;
    return ok();
}

// One search through the loop graph; the final state gives reachable and
// max_depth.
Error run_loop(GraphImpl& g, BfsWork& w, uint32_t source, BfsDevState* final_state) {
    DeviceImpl& dev = *g.dev;
    const uint64_t words = ceil_div_u64(g.num_nodes, 32);
    GCU_CUDA(cudaMemsetAsync(w.dist.ptr, 0xFF, sizeof(int32_t) * g.num_nodes, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(w.visited.ptr, 0, sizeof(uint32_t) * words, dev.stream), "memset");
    GCU_LAUNCH(dev, "bfs_init", bfs_loop_init_kernel, 1, 32, 0, g.offsets.ptr, source, w.dist.ptr, w.visited.ptr,
               w.queue[0].ptr, w.counters.ptr, w.loop_state.ptr);
    dev.launches.fetch_add(1, std::memory_order_relaxed);
    GCU_CUDA(cudaGraphLaunch(w.loop_exec, dev.stream), "cudaGraphLaunch");
    GCU_CUDA(cudaMemcpyAsync(&w.host_loop_state, w.loop_state.ptr, sizeof(BfsDevState), cudaMemcpyDeviceToHost,
                             dev.stream),
             "copy");
    GCU_TRY(dev.sync());
    *final_state = w.host_loop_state;
    return ok();
}

uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

Error bfs(GraphImpl& g, uint32_t source, int32_t* host_distances, uint32_t* reachable, int32_t* max_depth) {
    DeviceImpl& dev = *g.dev;
    GCU_TRY(ensure_work(g));
    BfsWork& w = *g.bfs_work;
    const bool sym = w.symmetric == 1;
    const unsigned valid = valid_variants(sym);
    const __nv_bfloat16* net = reinterpret_cast<const __nv_bfloat16*>(dev.schedule);
    DegreeStats stats;
    if (net) GCU_TRY(degree_stats(g, &stats));

    if (dev.bfs_device_loop && !dev.kernel_timing && !w.loop_unavailable) {
        if (!w.loop_exec || w.loop_net != static_cast<const void*>(net)) {
            // A driver that cannot build the conditional graph leaves the
            // search to the host-driven loop below (same kernels, same result).
            if (!build_loop_graph(g, w).ok()) w.loop_unavailable = true;
        }
        if (w.loop_exec) {
            BfsDevState fin{};
            GCU_TRY(run_loop(g, w, source, &fin));
            if (fin.failed) return kernel_error("BFS level loop stopped on an impossible state");
            if (host_distances)
                GCU_TRY(copy_to_host(dev, host_distances, w.dist.ptr, sizeof(int32_t) * g.num_nodes));
            *reachable = fin.reached;
            *max_depth = fin.level;
            return ok();
        }
    }

    GCU_TRY(start_run(g, w, source));
    if (net)
        GCU_LAUNCH(dev, "bfs_decide", bfs_decide_kernel, 1, 32, 0, net, w.counters.ptr, stats,
                   static_cast<unsigned long long>(g.num_edges), 0u, 0, 0, valid, g.num_nodes, nullptr);
    GCU_TRY(read_counters(dev, w));
    BfsState st;
    advance(st, w.host_counters, true, 0, g.num_edges);
    while (st.frontier_q > 0) {
        int variant = fixed_rule(st, sym, g.num_nodes);
        if (net) {
            const int c = w.host_counters.choice;
            if (c >= 0 && ((valid >> c) & 1u)) variant = c;
        }
        GCU_TRY(launch_step(g, w, variant, st));
        if (net)
            GCU_LAUNCH(dev, "bfs_decide", bfs_decide_kernel, 1, 32, 0, net, w.counters.ptr, stats,
                       static_cast<unsigned long long>(st.unexplored), st.reached, st.level + 1,
                       variant == kPull ? 1 : 0, valid, g.num_nodes, nullptr);
        GCU_TRY(read_counters(dev, w));
        if (w.host_counters.discovered == 0) break;
        advance(st, w.host_counters, false, variant, g.num_edges);
    }
    if (host_distances) GCU_TRY(copy_to_host(dev, host_distances, w.dist.ptr, sizeof(int32_t) * g.num_nodes));
    *reachable = st.reached;
    *max_depth = st.level;
    return ok();
}

// Trace: at every level, each valid variant runs from the same frontier
// (visited bitmap and distances restored from a snapshot in between) and is
// timed with events on the stream; all must label the same vertices. The run
// then continues with the fixed rule's variant, or, for 3 levels in 10 chosen
// by explore_seed, a uniformly drawn valid one (so that the traces also hold
// states the fixed rule never reaches).
Error bfs_trace(GraphImpl& g, uint32_t source, uint64_t explore_seed, std::vector<BfsTraceLevel>* levels) {
    DeviceImpl& dev = *g.dev;
    GCU_TRY(ensure_work(g));
    BfsWork& w = *g.bfs_work;
    const bool sym = w.symmetric == 1;
    const unsigned valid = valid_variants(sym);
    DegreeStats stats;
    GCU_TRY(degree_stats(g, &stats));
    const uint64_t V = g.num_nodes, words = ceil_div_u64(V, 32);
    DeviceBuffer<uint32_t> visited_snap;
    DeviceBuffer<int32_t> dist_snap;
    DeviceBuffer<BfsCounters> variant_ctr;
    DeviceBuffer<float> feats;
    GCU_TRY(visited_snap.allocate(dev, words));
    GCU_TRY(dist_snap.allocate(dev, V));
    GCU_TRY(variant_ctr.allocate(dev, kSchedOut));
    cudaEvent_t ev[2 * kSchedOut];
    for (auto& e : ev) GCU_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    struct Events {
        cudaEvent_t* e;
        ~Events() {
            for (int i = 0; i < 2 * kSchedOut; ++i) cudaEventDestroy(e[i]);
        }
    } guard{ev};

    levels->clear();
    GCU_TRY(feats.allocate(dev, kSchedIn));
    GCU_TRY(start_run(g, w, source));
    GCU_LAUNCH(dev, "bfs_decide", bfs_decide_kernel, 1, 32, 0, nullptr, w.counters.ptr, stats,
               static_cast<unsigned long long>(g.num_edges), 0u, 0, 0, valid, g.num_nodes, feats.ptr);
    GCU_TRY(read_counters(dev, w));
    BfsState st;
    advance(st, w.host_counters, true, 0, g.num_edges);
    std::vector<float> host_feats(kSchedIn);
    GCU_CUDA(cudaMemcpy(host_feats.data(), feats.ptr, 4 * kSchedIn, cudaMemcpyDeviceToHost), "copy");
    while (st.frontier_q > 0) {
        BfsTraceLevel rec{};
        for (int k = 0; k < kSchedIn; ++k) rec.features[k] = host_feats[k];
        rec.valid = static_cast<uint8_t>(valid);
        const int fixed = fixed_rule(st, sym, g.num_nodes);
        rec.fixed_rule = static_cast<uint8_t>(fixed);
        int take = fixed;
        const uint64_t r = mix64(explore_seed * 0x9E3779B97F4A7C15ull + static_cast<uint64_t>(st.level) + 1);
        if (r % 10 < 3) {
            const int nvalid = __builtin_popcount(valid);
            int pick = static_cast<int>((r >> 32) % nvalid);
            for (int c = 0; c < kSchedOut; ++c)
                if ((valid >> c) & 1u) {
                    if (pick == 0) {
                        take = c;
                        break;
                    }
                    --pick;
                }
        }
        rec.taken = static_cast<uint8_t>(take);
        GCU_CUDA(cudaMemcpyAsync(visited_snap.ptr, w.visited.ptr, 4 * words, cudaMemcpyDeviceToDevice, dev.stream),
                 "copy");
        GCU_CUDA(cudaMemcpyAsync(dist_snap.ptr, w.dist.ptr, 4 * V, cudaMemcpyDeviceToDevice, dev.stream), "copy");
        for (int k = 0; k < kSchedOut; ++k) {
            const int c = (k + st.level) % kSchedOut;  // rotate which variant goes first
            if (!((valid >> c) & 1u)) continue;
            GCU_CUDA(cudaEventRecord(ev[2 * c], dev.stream), "cudaEventRecord");
            GCU_TRY(launch_step(g, w, c, st));
            GCU_CUDA(cudaEventRecord(ev[2 * c + 1], dev.stream), "cudaEventRecord");
            GCU_CUDA(cudaMemcpyAsync(variant_ctr.ptr + c, w.counters.ptr, sizeof(BfsCounters),
                                     cudaMemcpyDeviceToDevice, dev.stream),
                     "copy");
            GCU_CUDA(cudaMemcpyAsync(w.visited.ptr, visited_snap.ptr, 4 * words, cudaMemcpyDeviceToDevice, dev.stream),
                     "copy");
            GCU_CUDA(cudaMemcpyAsync(w.dist.ptr, dist_snap.ptr, 4 * V, cudaMemcpyDeviceToDevice, dev.stream), "copy");
        }
        GCU_TRY(launch_step(g, w, take, st));
        GCU_LAUNCH(dev, "bfs_decide", bfs_decide_kernel, 1, 32, 0, nullptr, w.counters.ptr, stats,
                   static_cast<unsigned long long>(st.unexplored), st.reached, st.level + 1, take == kPull ? 1 : 0,
                   valid, g.num_nodes, feats.ptr);
        BfsCounters vc[kSchedOut];
        GCU_CUDA(cudaMemcpyAsync(vc, variant_ctr.ptr, sizeof(vc), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_CUDA(cudaMemcpyAsync(host_feats.data(), feats.ptr, 4 * kSchedIn, cudaMemcpyDeviceToHost, dev.stream),
                 "copy");
        GCU_TRY(read_counters(dev, w));
        const BfsCounters c = w.host_counters;
        for (int v = 0; v < kSchedOut; ++v) {
            rec.times_us[v] = __builtin_nanf("");
            if (!((valid >> v) & 1u)) continue;
            if (vc[v].discovered != c.discovered || vc[v].queued != c.queued || vc[v].edges != c.edges)
                return kernel_error("BFS step variants disagree at level " + std::to_string(st.level));
            float ms = 0.f;
            GCU_CUDA(cudaEventElapsedTime(&ms, ev[2 * v], ev[2 * v + 1]), "cudaEventElapsedTime");
            rec.times_us[v] = 1000.f * ms;
        }
        levels->push_back(rec);
        if (c.discovered == 0) break;
        advance(st, c, false, take, g.num_edges);
    }
    return ok();
}

}  // namespace gcu
