// k-truss by synchronous peeling.
//
// Reference: crates/grafeo-cuda-algos/src/k_truss.rs:42-161 and
// kernels/k_truss.cu:46-124. Each reference round computes, for every live CSR
// entry u -> v with v > u, support = |live N(u) ∩ live N(v)| (entry-level
// liveness, so in the first round a live self-loop at u or v counts as a
// common neighbour, as the reference's merge of the raw lists does), copies it
// to the live reverse entry v -> u, and then removes every live entry whose
// support is below k - 2. Rounds repeat until one removes nothing; their count
// is the reference's `iterations`. Two paths give exactly the same removed
// sets round by round, hence the same edges and round count:
//
//  * Symmetric CSR (every graph exported from Grafeo): the support of every
//    undirected edge is its triangle count, found once by enumerating the
//    triangles of the degree-oriented DAG (wedge.cuh) with three atomic adds
//    per triangle; round 1 adds one for a self-loop at either end. After a
//    round removes a set R of edges, each triangle with an edge in R that was
//    alive at the start of the round is destroyed once (credited to its
//    removed edge with the smallest id) and its surviving edges lose one
//    support, so the supports stay exact for the next round without
//    recomputing them. Work per round is proportional to the edges removed.
//  * Any other CSR: the reference's per-entry rules with all supports
//    recomputed each round (a warp per entry, binary-search intersection).
//
// Both paths use a reverse-entry index instead of the reference's linear scan
// of N(v), and compact the result edge list on the device in CSR order (the
// reference copies removed/offsets/targets back and loops on the host).
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"
#include "wedge.cuh"

namespace gcu {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// src[j] = row of entry j.
__global__ void __launch_bounds__(256) kt_rows_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t E,
                                                      uint32_t* __restrict__ src) {
    for_each_entry<256, 4>(offsets, V, E, [&](uint32_t j, uint32_t row) { src[j] = row; });
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

struct LiveFlag {
    const uint8_t* live;
    __device__ __forceinline__ bool operator()(uint64_t j) const { return live[j] != 0; }
};
struct RoundState {
    const uint32_t* state;  // 0 = alive, r = removed in round r
    __device__ __forceinline__ bool operator()(uint64_t j) const { return state[j] == 0; }
};

template <class Alive>
__global__ void kt_flag_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src, Alive alive,
                               uint32_t E, uint32_t* __restrict__ flag) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        flag[j] = (targets[j] > src[j] && alive(j)) ? 1u : 0u;
    }
}

template <class Alive>
__global__ void kt_emit_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src, Alive alive,
                               uint32_t E, const uint32_t* __restrict__ pos, uint2* __restrict__ out) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[j], v = targets[j];
        if (v > u && alive(j)) out[pos[j]] = make_uint2(u, v);
    }
}

// ---------------------------------------------------------------- symmetric CSR: incremental peeling

namespace {

// Adds each triangle found on the DAG to the support of its three edges.
struct SupportSink {
    static constexpr bool kNeedsPos = true;
    const uint32_t* dag_eid;
    uint32_t* support;
    __device__ __forceinline__ void hit(uint32_t base, uint32_t pv, uint32_t pw, uint32_t evw) {
        atomicAdd(support + dag_eid[base + pv], 1u);
        atomicAdd(support + dag_eid[base + pw], 1u);
        atomicAdd(support + dag_eid[evw], 1u);
    }
    __device__ __forceinline__ void finish() {}
};

}  // namespace

// loop[u] = 1 for every vertex with a self-loop entry; counts them in *loops.
__global__ void kt_loops_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src, uint32_t E,
                                uint8_t* __restrict__ loop, uint32_t* __restrict__ loops) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[j];
        if (targets[j] == u) {
            loop[u] = 1;
            atomicAdd(loops, 1u);
        }
    }
}

// Round r: every alive u < v entry whose support is below the threshold is
// removed (state = r) and listed. With `loop` in round 1 a self-loop at either
// end adds one to the support, as the reference's merge of the raw lists
// does. With `truss`, every removed entry also gets truss_value there.
__global__ void kt_round_filter_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src,
                                       const uint8_t* __restrict__ loop, const uint32_t* __restrict__ support,
                                       uint32_t* __restrict__ state, uint32_t E, uint32_t threshold, uint32_t round,
                                       uint32_t* __restrict__ removed, uint32_t* __restrict__ removed_count,
                                       uint32_t* __restrict__ truss, uint32_t truss_value) {
    const unsigned lane = lane_id();
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~31ull; base < E;
         base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t j = base + lane;
        bool take = false;
        if (j < E && state[j] == 0) {
            const uint32_t u = src[j], v = targets[j];
            if (v > u) {
                uint32_t s = support[j];
                if (loop && round == 1) s += loop[u] + loop[v];
                take = s < threshold;
                if (take && truss) truss[j] = truss_value;
            }
        }
        const unsigned mask = __ballot_sync(kFullMask, take);
        if (mask == 0) continue;
        uint32_t at = 0;
        const int leader = __ffs(mask) - 1;
        if (lane == static_cast<unsigned>(leader)) at = atomicAdd(removed_count, static_cast<uint32_t>(__popc(mask)));
        at = __shfl_sync(kFullMask, at, leader);
        if (take) {
            state[j] = round;
            removed[at + __popc(mask & ((1u << lane) - 1))] = static_cast<uint32_t>(j);
        }
    }
}

// For every edge (a, b) removed in round r, every triangle {a, b, w} still
// alive at the start of the round is destroyed: each of its edges that
// survives the round loses one support. A triangle with several edges removed
// in this round is handled once, by the removed edge with the smallest id.
// With `next`, an edge whose support falls from `threshold` to below it is
// listed there: supports only fall by one at a time, so every surviving edge
// that the next round removes is listed exactly once, and that round needs no
// scan of the alive edges.
//
// The shorter of the two lists is walked (the longer one binary-searched) in
// chunks of kPeelChunk entries, one warp per chunk, so that a round that
// removes a few hub edges spreads their lists over the whole GPU instead of
// waiting on one warp per edge.
constexpr uint32_t kPeelChunk = 256;

struct PeelEdge {
    uint32_t a, b;       // the removed edge
    uint32_t x, y;       // the walked end and the searched end
    uint32_t xs, xe, ys, ye;
};

// Lists of the live CSR `lv` (the graph's CSR, or its alive entries after a
// compaction); e is an entry of the graph's CSR.
struct LiveCsr {
    const uint32_t* offsets;
    const uint32_t* targets;
    const uint32_t* eid;  // graph entry of each live entry (nullptr: the graph's CSR itself)
    __device__ __forceinline__ uint32_t entry(uint32_t p) const { return eid ? eid[p] : p; }
};

__device__ __forceinline__ PeelEdge peel_edge(const LiveCsr& lv, const uint32_t* __restrict__ targets,
                                              const uint32_t* __restrict__ src, uint32_t e) {
    const uint32_t* __restrict__ offsets = lv.offsets;
    PeelEdge p;
    p.a = src[e];
    p.b = targets[e];
    p.xs = offsets[p.a];
    p.xe = offsets[p.a + 1];
    p.ys = offsets[p.b];
    p.ye = offsets[p.b + 1];
    p.x = p.a;
    p.y = p.b;
    if (p.xe - p.xs > p.ye - p.ys) {
        uint32_t t = p.xs; p.xs = p.ys; p.ys = t;
        t = p.xe; p.xe = p.ye; p.ye = t;
        p.x = p.b;
        p.y = p.a;
    }
    return p;
}

// chunks[i] = the walk chunks of removed edge i (at least one).
__global__ void kt_peel_chunks_kernel(const LiveCsr lv, const uint32_t* __restrict__ targets,
                                      const uint32_t* __restrict__ src, const uint32_t* __restrict__ removed,
                                      const uint32_t* __restrict__ removed_count, uint32_t* __restrict__ chunks) {
    const uint32_t n = *removed_count;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const PeelEdge p = peel_edge(lv, targets, src, removed[i]);
        chunks[i] = max(1u, (p.xe - p.xs + kPeelChunk - 1) / kPeelChunk);
    }
}

// Warp per chunk: chunk_start (n + 1 words) is the exclusive scan of the
// chunk counts; each warp finds its edge by a binary search of it.
__global__ void __launch_bounds__(256) kt_peel_kernel(const LiveCsr lv,
                                                      const uint32_t* __restrict__ targets,
                                                      const uint32_t* __restrict__ src,
                                                      const uint32_t* __restrict__ rev,
                                                      const uint32_t* __restrict__ state,
                                                      uint32_t* __restrict__ support,
                                                      const uint32_t* __restrict__ removed,
                                                      const uint32_t* __restrict__ removed_count,
                                                      const uint32_t* __restrict__ chunk_start, uint32_t round,
                                                      uint32_t threshold, uint32_t* __restrict__ next,
                                                      uint32_t* __restrict__ next_count) {
    const unsigned lane = lane_id();
    const uint32_t n = *removed_count;
    const uint32_t total = chunk_start[n];
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < total; w += nwarps) {
        // i = the largest index with chunk_start[i] <= w (every edge has a chunk).
        uint32_t lo = 0, hi = n;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (chunk_start[mid] <= w)
                lo = mid;
            else
                hi = mid;
        }
        const uint32_t e = removed[lo];
        const PeelEdge pe = peel_edge(lv, targets, src, e);
        const uint32_t begin = pe.xs + (static_cast<uint32_t>(w) - chunk_start[lo]) * kPeelChunk;
        const uint32_t end = min(begin + kPeelChunk, pe.xe);
        for (uint32_t p = begin + lane; p < end; p += 32) {
            const uint32_t wv = lv.targets[p];
            if (wv == pe.a || wv == pe.b) continue;
            const uint32_t j1 = lv.entry(p);
            const uint32_t e1 = pe.x < wv ? j1 : rev[j1];
            const uint32_t s1 = state[e1];
            if (s1 != 0 && s1 != round) continue;
            const uint32_t q = lower_bound_u32(lv.targets, pe.ys, pe.ye, wv);
            if (q == pe.ye || lv.targets[q] != wv) continue;
            const uint32_t j2 = lv.entry(q);
            const uint32_t e2 = pe.y < wv ? j2 : rev[j2];
            const uint32_t s2 = state[e2];
            if (s2 != 0 && s2 != round) continue;
            if ((s1 == round && e1 < e) || (s2 == round && e2 < e)) continue;
            if (s1 == 0 && atomicSub(support + e1, 1u) == threshold && next) next[atomicAdd(next_count, 1u)] = e1;
            if (s2 == 0 && atomicSub(support + e2, 1u) == threshold && next) next[atomicAdd(next_count, 1u)] = e2;
        }
    }
}

// One peel: chunk counts of the n removed edges, their scan, the chunk walk.
// chunks holds n + 1 words.
static Error launch_peel(DeviceImpl& dev, GraphImpl& g, const LiveCsr& lv, const uint32_t* src,
                         const uint32_t* rev, const uint32_t* state, uint32_t* support, const uint32_t* list,
                         const uint32_t* count, uint32_t n, uint32_t* chunks, uint32_t round, uint32_t threshold,
                         uint32_t* next, uint32_t* next_count) {
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(n, 256), cap)));
    GCU_LAUNCH(dev, "kt_peel_chunks", kt_peel_chunks_kernel, grid, 256, 0, lv, g.targets.ptr, src, list, count,
               chunks);
    GCU_TRY(exclusive_scan_u32(dev, chunks, chunks, n));
    GCU_LAUNCH(dev, "kt_peel", kt_peel_kernel, static_cast<unsigned>(cap), 256, 0, lv, g.targets.ptr, src, rev,
               state, support, list, count, chunks, round, threshold, next, next_count);
    return ok();
}

// ---------------------------------------------------------------- live CSR compaction

// keep[p] for every live entry p = u -> w: not a self-loop and its edge alive.
__global__ void __launch_bounds__(256) kt_live_flag_kernel(const LiveCsr lv, uint32_t V, uint32_t L,
                                                           const uint32_t* __restrict__ rev,
                                                           const uint32_t* __restrict__ state,
                                                           uint32_t* __restrict__ keep) {
    for_each_entry<256, 4>(lv.offsets, V, L, [&](uint32_t p, uint32_t u) {
        const uint32_t w = lv.targets[p];
        const uint32_t j = lv.entry(p);
        keep[p] = (u != w && state[u < w ? j : rev[j]] == 0) ? 1u : 0u;
    });
}

__global__ void kt_live_offsets_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                       const uint32_t* __restrict__ pos, uint32_t* __restrict__ out) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u <= V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[u] = pos[offsets[u]];
}

__global__ void kt_live_fill_kernel(const LiveCsr lv, uint32_t L, const uint32_t* __restrict__ pos,
                                    uint32_t* __restrict__ targets, uint32_t* __restrict__ eid) {
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < L;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t at = pos[p];
        if (pos[p + 1] == at) continue;
        targets[at] = lv.targets[p];
        eid[at] = lv.entry(p);
    }
}

// The alive entries of `lv` (L entries) in a new CSR (same order), so that
// the peel of later rounds walks alive lists only.
struct LiveBuffers {
    DeviceBuffer<uint32_t> offsets, targets, eid;
    uint32_t entries = 0;
};

static Error compact_live(DeviceImpl& dev, uint32_t V, const LiveCsr& lv, uint32_t L, const uint32_t* rev,
                          const uint32_t* state, LiveBuffers* out) {
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    DeviceBuffer<uint32_t> pos;
    GCU_TRY(pos.allocate(dev, static_cast<uint64_t>(L) + 1));
    GCU_TRY(out->offsets.allocate(dev, static_cast<uint64_t>(V) + 1));
    const unsigned tiles = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(L, 1024), cap)));
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(L, 256), cap)));
    const unsigned vgrid =
        static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(static_cast<uint64_t>(V) + 1, 256), cap));
    if (L > 0)
        GCU_LAUNCH(dev, "kt_live_flag", kt_live_flag_kernel, tiles, 256, 0, lv, V, L, rev, state, pos.ptr);
    GCU_TRY(exclusive_scan_u32(dev, pos.ptr, pos.ptr, L));
    GCU_LAUNCH(dev, "kt_live_offsets", kt_live_offsets_kernel, vgrid, 256, 0, lv.offsets, V, pos.ptr,
               out->offsets.ptr);
    GCU_CUDA(cudaMemcpyAsync(&out->entries, pos.ptr + L, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    GCU_TRY(dev.sync());
    GCU_TRY(out->targets.allocate(dev, std::max<uint32_t>(out->entries, 1)));
    GCU_TRY(out->eid.allocate(dev, std::max<uint32_t>(out->entries, 1)));
    if (out->entries > 0)
        GCU_LAUNCH(dev, "kt_live_fill", kt_live_fill_kernel, grid, 256, 0, lv, L, pos.ptr, out->targets.ptr,
                   out->eid.ptr);
    GCU_TRY(dev.sync());  // pos is freed on return
    return ok();
}

// The entries listed for round r are removed in it (state = r); with truss,
// they also get truss_value.
__global__ void kt_mark_kernel(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                               uint32_t* __restrict__ state, uint32_t round, uint32_t* __restrict__ truss,
                               uint32_t truss_value) {
    const uint32_t n = *count;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t j = list[i];
        state[j] = round;
        if (truss) truss[j] = truss_value;
    }
}

// Compacts the alive u < v entries, in CSR order, into host pairs.
template <class Alive>
static Error emit_edges(DeviceImpl& dev, GraphImpl& g, const uint32_t* src, Alive alive, uint32_t* flag,
                        uint32_t* pos, std::vector<uint32_t>* edges) {
    const uint32_t E = g.num_edges;
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    GCU_LAUNCH(dev, "kt_flag", kt_flag_kernel<Alive>, edge_grid, 256, 0, g.targets.ptr, src, alive, E, flag);
    GCU_TRY(exclusive_scan_u32(dev, flag, pos, E));
    uint32_t count = 0;
    GCU_CUDA(cudaMemcpyAsync(&count, pos + E, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    if (count > 0) {
        DeviceBuffer<uint2> out;
        GCU_TRY(out.allocate(dev, count));
        GCU_LAUNCH(dev, "kt_emit", kt_emit_kernel<Alive>, edge_grid, 256, 0, g.targets.ptr, src, alive, E, pos,
                   out.ptr);
        edges->resize(2 * static_cast<size_t>(count));
        GCU_TRY(copy_to_host(dev, edges->data(), out.ptr, sizeof(uint2) * count));
    }
    return ok();
}

// Any CSR: the reference's rounds, recomputing every support each round.
static Error k_truss_general(GraphImpl& g, uint32_t k, const uint32_t* src, const uint32_t* rev,
                             std::vector<uint32_t>* edges, uint32_t* iterations) {
    DeviceImpl& dev = *g.dev;
    const uint32_t E = g.num_edges;
    const uint32_t threshold = k - 2;
    DeviceBuffer<uint32_t> support, pos, scratch;
    DeviceBuffer<uint8_t> live;
    GCU_TRY(support.allocate(dev, E));
    GCU_TRY(pos.allocate(dev, static_cast<uint64_t>(E) + 1));
    GCU_TRY(live.allocate(dev, E));
    GCU_TRY(scratch.allocate(dev, 1));
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    GCU_CUDA(cudaMemsetAsync(live.ptr, 1, E, dev.stream), "memset");
    uint32_t rounds = 0;
    while (true) {
        GCU_CUDA(cudaMemsetAsync(support.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
        GCU_LAUNCH(dev, "kt_support", kt_support_kernel, edge_grid, 256, 0, g.offsets.ptr, g.targets.ptr, src, rev,
                   live.ptr, E, support.ptr);
        GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
        GCU_LAUNCH(dev, "kt_filter", kt_filter_kernel, edge_grid, 256, 0, support.ptr, live.ptr, E, threshold,
                   scratch.ptr);
        uint32_t removed = 0;
        GCU_CUDA(cudaMemcpyAsync(&removed, scratch.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        rounds += 1;
        if (removed == 0) break;
    }
    *iterations = rounds;
    return emit_edges(dev, g, src, LiveFlag{live.ptr}, support.ptr, pos.ptr, edges);
}

// support[j] += triangles of the undirected edge whose u < v entry is j,
// counted once on the degree DAG (symmetric CSR).
static Error triangle_support(GraphImpl& g, const uint32_t* rev, uint32_t* support) {
    DeviceBuffer<uint32_t> dag_offsets, dag_targets, dag_eid;
    uint32_t m = 0;
    GCU_TRY(build_dag(g, true, rev, &dag_offsets, &dag_targets, &dag_eid, &m));
    if (m > 0) {
        GCU_TRY(run_wedges(*g.dev, dag_offsets.ptr, dag_targets.ptr, g.num_nodes, 2,
                           SupportSink{dag_eid.ptr, support}, "kt"));
    }
    return ok();
}

// Per-graph state of the symmetric k-truss: row of every entry, reverse
// entries, self-loop flags and the triangle support of every u < v entry. It
// depends only on the graph, so it is computed once and reused by every
// k_truss call and by the truss decomposition (3 E + V words of HBM, kept
// with the graph like the PageRank plan).
struct KtCache {
    DeviceBuffer<uint32_t> src, rev, support;
    DeviceBuffer<uint8_t> loop;
    uint32_t loops = 0;  // self-loop entries
};

void destroy_kt_cache(KtCache* c) { delete c; }

static Error ensure_kt_cache(GraphImpl& g, KtCache** out) {
    if (!g.kt_cache) {
        DeviceImpl& dev = *g.dev;
        const uint32_t E = g.num_edges, V = g.num_nodes;
        auto c = std::unique_ptr<KtCache, void (*)(KtCache*)>(new KtCache, destroy_kt_cache);
        GCU_TRY(c->src.allocate(dev, E));
        GCU_TRY(c->rev.allocate(dev, E));
        GCU_TRY(c->support.allocate(dev, E));
        GCU_TRY(c->loop.allocate(dev, V));
        DeviceBuffer<uint32_t> count;
        GCU_TRY(count.allocate(dev, 1));
        const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
        const unsigned tile_grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(E, 1024), cap)));
        const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
        GCU_LAUNCH(dev, "kt_rows", kt_rows_kernel, tile_grid, 256, 0, g.offsets.ptr, V, E, c->src.ptr);
        GCU_LAUNCH(dev, "kt_reverse", kt_reverse_kernel, edge_grid, 256, 0, g.offsets.ptr, g.targets.ptr, c->src.ptr,
                   E, c->rev.ptr);
        GCU_CUDA(cudaMemsetAsync(c->loop.ptr, 0, V, dev.stream), "memset");
        GCU_CUDA(cudaMemsetAsync(count.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
        GCU_LAUNCH(dev, "kt_loops", kt_loops_kernel, edge_grid, 256, 0, g.targets.ptr, c->src.ptr, E, c->loop.ptr,
                   count.ptr);
        GCU_CUDA(cudaMemsetAsync(c->support.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
        GCU_TRY(triangle_support(g, c->rev.ptr, c->support.ptr));
        GCU_CUDA(cudaMemcpyAsync(&c->loops, count.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
        GCU_TRY(dev.sync());
        g.kt_cache = c.release();
    }
    *out = g.kt_cache;
    return ok();
}

// Symmetric CSR: per-edge triangle counts from the DAG (cached), then
// incremental peeling. Every round removes exactly the entries the
// reference's round removes, so the edge list and the round count are the
// same.
static Error k_truss_symmetric(GraphImpl& g, uint32_t k, std::vector<uint32_t>* edges, uint32_t* iterations) {
    DeviceImpl& dev = *g.dev;
    const uint32_t E = g.num_edges;
    const uint32_t threshold = k - 2;
    KtCache* c = nullptr;
    GCU_TRY(ensure_kt_cache(g, &c));
    const uint32_t* src = c->src.ptr;
    const uint32_t* rev = c->rev.ptr;
    DeviceBuffer<uint32_t> support, state, removed, scratch, lists[2];
    GCU_TRY(support.allocate(dev, static_cast<uint64_t>(E) + 1));
    GCU_TRY(state.allocate(dev, static_cast<uint64_t>(E) + 1));
    GCU_TRY(removed.allocate(dev, E));
    GCU_TRY(lists[0].allocate(dev, E));
    GCU_TRY(lists[1].allocate(dev, E));
    DeviceBuffer<uint32_t> chunks;  // peel chunk counts, then their scan
    GCU_TRY(chunks.allocate(dev, static_cast<uint64_t>(E) + 1));
    GCU_TRY(scratch.allocate(dev, 3));  // [0] removed by a scan, [1 + b] entries of lists[b]
    GCU_CUDA(cudaMemcpyAsync(support.ptr, c->support.ptr, sizeof(uint32_t) * static_cast<size_t>(E),
                             cudaMemcpyDeviceToDevice, dev.stream),
             "copy");
    GCU_CUDA(cudaMemsetAsync(state.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    const uint32_t loops = c->loops;

    // Rounds 1 and (with self-loops) 2 scan every entry: round 1 adds the
    // self-loop terms, so an edge it keeps may be below the threshold in
    // round 2 without losing a triangle. Later rounds remove exactly the
    // edges that the previous round's peel brought below the threshold.
    uint32_t round = 1;
    int cur = 0;       // the peel of this round lists the next round's removals in lists[cur]
    uint32_t n = 0;    // entries removed in this round
    while (true) {
        const bool scan = round == 1 || (round == 2 && loops > 0);
        const uint32_t* list = removed.ptr;
        const uint32_t* count = scratch.ptr;
        if (scan) {
            GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
            GCU_LAUNCH(dev, "kt_round_filter", kt_round_filter_kernel, edge_grid, 256, 0, g.targets.ptr, src,
                       c->loop.ptr, support.ptr, state.ptr, E, threshold, round, removed.ptr, scratch.ptr, nullptr,
                       0u);
            GCU_CUDA(cudaMemcpyAsync(&n, scratch.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
            GCU_TRY(dev.sync());
        } else {
            // n = the previous peel's list (read below); mark it removed in this round.
            list = lists[cur ^ 1].ptr;
            count = scratch.ptr + 1 + (cur ^ 1);
            if (n > 0) {
                const unsigned grid =
                    static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(n, 256), cap));
                GCU_LAUNCH(dev, "kt_mark", kt_mark_kernel, grid, 256, 0, list, count, state.ptr, round,
                           static_cast<uint32_t*>(nullptr), 0u);
            }
        }
        // Round 1 also removes the self-loop entries (their support is 0).
        const bool removed_any = n > 0 || (round == 1 && loops > 0);
        if (!removed_any) break;
        uint32_t next_n = 0;
        GCU_CUDA(cudaMemsetAsync(scratch.ptr + 1 + cur, 0, sizeof(uint32_t), dev.stream), "memset");
        if (n > 0) {
            GCU_TRY(launch_peel(dev, g, LiveCsr{g.offsets.ptr, g.targets.ptr, nullptr}, src, rev, state.ptr,
                                support.ptr, list, count, n, chunks.ptr, round, threshold, lists[cur].ptr,
                                scratch.ptr + 1 + cur));
            GCU_CUDA(cudaMemcpyAsync(&next_n, scratch.ptr + 1 + cur, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     dev.stream),
                     "copy");
            GCU_TRY(dev.sync());
        }
        n = next_n;
        cur ^= 1;
        round += 1;
    }
    *iterations = round;
    // `removed` (E entries) and `support` (E + 1) are reused as the compaction's flag and scan buffers.
    return emit_edges(dev, g, src, RoundState{state.ptr}, removed.ptr, support.ptr, edges);
}

Error k_truss(GraphImpl& g, uint32_t k, std::vector<uint32_t>* edges, uint32_t* iterations) {
    edges->clear();
    *iterations = 0;
    const uint32_t E = g.num_edges, V = g.num_nodes;
    // k_truss.rs:53-60: no edges, no truss.
    if (E == 0) return ok();
    DeviceImpl& dev = *g.dev;
    bool symmetric = false;
    GCU_TRY(graph_symmetry(g, &symmetric));
    if (symmetric) return k_truss_symmetric(g, k, edges, iterations);
    DeviceBuffer<uint32_t> src, rev;
    GCU_TRY(src.allocate(dev, E));
    GCU_TRY(rev.allocate(dev, E));
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned tile_grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(E, 1024), cap)));
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    GCU_LAUNCH(dev, "kt_rows", kt_rows_kernel, tile_grid, 256, 0, g.offsets.ptr, V, E, src.ptr);
    GCU_LAUNCH(dev, "kt_reverse", kt_reverse_kernel, edge_grid, 256, 0, g.offsets.ptr, g.targets.ptr, src.ptr, E,
               rev.ptr);
    return k_truss_general(g, k, src.ptr, rev.ptr, edges, iterations);
}

// ---------------------------------------------------------------- truss decomposition

// Appends, warp-aggregated, the entries with take set (all 32 lanes call it).
__device__ __forceinline__ void kt_append(bool take, uint32_t j, uint32_t* __restrict__ list,
                                          uint32_t* __restrict__ count) {
    const unsigned mask = __ballot_sync(kFullMask, take);
    if (mask == 0) return;
    const unsigned lane = lane_id();
    const int leader = __ffs(mask) - 1;
    uint32_t at = 0;
    if (lane == static_cast<unsigned>(leader)) at = atomicAdd(count, static_cast<uint32_t>(__popc(mask)));
    at = __shfl_sync(kFullMask, at, leader);
    if (take) list[at + __popc(mask & ((1u << lane) - 1))] = j;
}

// The alive u < v entries: from all E entries (list == nullptr) or from a
// previous active list of n entries.
__global__ void kt_active_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src,
                                 const uint32_t* __restrict__ state, const uint32_t* __restrict__ list, uint32_t n,
                                 uint32_t* __restrict__ out, uint32_t* __restrict__ count) {
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~31ull; base < n;
         base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i = base + lane_id();
        bool take = false;
        uint32_t j = 0;
        if (i < n) {
            j = list ? list[i] : static_cast<uint32_t>(i);
            take = state[j] == 0 && targets[j] > src[j];
        }
        kt_append(take, j, out, count);
    }
}

// kt_round_filter_kernel over an active list: every listed entry still alive
// with support < threshold is removed in this round (state = round), listed in
// `removed` and given truss_value.
__global__ void kt_active_filter_kernel(const uint32_t* __restrict__ active, uint32_t n,
                                        const uint32_t* __restrict__ support, uint32_t* __restrict__ state,
                                        uint32_t threshold, uint32_t round, uint32_t* __restrict__ removed,
                                        uint32_t* __restrict__ removed_count, uint32_t* __restrict__ truss,
                                        uint32_t truss_value) {
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~31ull; base < n;
         base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i = base + lane_id();
        bool take = false;
        uint32_t j = 0;
        if (i < n) {
            j = active[i];
            take = state[j] == 0 && support[j] < threshold;
            if (take) {
                state[j] = round;
                truss[j] = truss_value;
            }
        }
        kt_append(take, j, removed, removed_count);
    }
}

// Spreads the u < v entries' trussness to every entry: the reverse entry gets
// the same value, self-loops 0.
__global__ void kt_truss_spread_kernel(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ src,
                                       const uint32_t* __restrict__ rev, const uint32_t* __restrict__ truss,
                                       uint32_t E, uint32_t* __restrict__ out) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = src[j], v = targets[j];
        out[j] = u == v ? 0u : truss[u < v ? j : rev[j]];
    }
}

// Trussness of every edge of a symmetric CSR: the peeling of k_truss_symmetric
// continued level by level without restarting. At level k the rounds remove
// every alive edge with fewer than k - 2 alive triangles until none is left
// below; the edges removed at level k have trussness k - 1. Self-loops take no
// part (they are in no k-truss for k >= 3).
Error truss_decomposition(GraphImpl& g, uint32_t* host_truss, uint32_t* max_truss, uint32_t* rounds) {
    *max_truss = 0;
    *rounds = 0;
    const uint32_t E = g.num_edges;
    if (E == 0) return ok();
    DeviceImpl& dev = *g.dev;
    bool symmetric = false;
    GCU_TRY(graph_symmetry(g, &symmetric));
    if (!symmetric) return kernel_error("truss decomposition needs a symmetric CSR (every u -> v with its v -> u)");
    KtCache* c = nullptr;
    GCU_TRY(ensure_kt_cache(g, &c));
    const uint32_t* src = c->src.ptr;
    const uint32_t* rev = c->rev.ptr;
    DeviceBuffer<uint32_t> support, state, removed, truss, scratch, active[2], lists[2];
    GCU_TRY(support.allocate(dev, E));
    GCU_TRY(state.allocate(dev, E));
    GCU_TRY(removed.allocate(dev, E));
    GCU_TRY(truss.allocate(dev, E));
    GCU_TRY(lists[0].allocate(dev, E));
    GCU_TRY(lists[1].allocate(dev, E));
    DeviceBuffer<uint32_t> chunks;  // peel chunk counts, then their scan
    GCU_TRY(chunks.allocate(dev, static_cast<uint64_t>(E) + 1));
    GCU_TRY(scratch.allocate(dev, 4));  // [0] removed by a scan, [1] active count, [2 + b] entries of lists[b]
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned edge_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(E, 256), cap));
    GCU_CUDA(cudaMemcpyAsync(support.ptr, c->support.ptr, sizeof(uint32_t) * static_cast<size_t>(E),
                             cudaMemcpyDeviceToDevice, dev.stream),
             "copy");
    GCU_CUDA(cudaMemsetAsync(state.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(truss.ptr, 0, sizeof(uint32_t) * static_cast<size_t>(E), dev.stream), "memset");
    // Undirected edges alive: in a symmetric CSR every edge but a self-loop
    // has two entries, so there are (E - self-loop entries) / 2 of them; the
    // active list holds their u < v entries and is compacted whenever half
    // of it has been peeled, so late rounds only touch the remaining core.
    uint64_t alive = (static_cast<uint64_t>(E) - c->loops) / 2;
    const uint64_t list_cap = std::max<uint64_t>(alive, 1);
    GCU_TRY(active[0].allocate(dev, list_cap));
    GCU_TRY(active[1].allocate(dev, list_cap));
    GCU_CUDA(cudaMemsetAsync(scratch.ptr + 1, 0, sizeof(uint32_t), dev.stream), "memset");
    GCU_LAUNCH(dev, "kt_active", kt_active_kernel, edge_grid, 256, 0, g.targets.ptr, src, state.ptr,
               static_cast<const uint32_t*>(nullptr), E, active[0].ptr, scratch.ptr + 1);
    int cur = 0;              // active list in use
    int out = 0;              // the peel lists the next round's removals in lists[out]
    LiveCsr live{g.offsets.ptr, g.targets.ptr, nullptr};  // the peel's lists
    uint32_t live_entries = E;
    LiveBuffers live_bufs[2];
    int live_cur = 0;
    uint64_t listed = alive;  // entries in active[cur]
    uint32_t round = 0, k = 3, top = alive > 0 ? 2 : 0;
    // The first round of every level scans the active list for the edges
    // below the new threshold; every later round of the level removes
    // exactly the edges that the previous peel brought below it.
    bool level_start = true;
    uint32_t n = 0;  // entries removed in this round
    while (alive > 0) {
        round += 1;
        const unsigned grid =
            static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(listed, 256), cap)));
        const uint32_t* list = removed.ptr;
        const uint32_t* count = scratch.ptr;
        if (level_start) {
            GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
            GCU_LAUNCH(dev, "kt_active_filter", kt_active_filter_kernel, grid, 256, 0, active[cur].ptr,
                       static_cast<uint32_t>(listed), support.ptr, state.ptr, k - 2, round, removed.ptr,
                       scratch.ptr, truss.ptr, k - 1);
            GCU_CUDA(cudaMemcpyAsync(&n, scratch.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
            GCU_TRY(dev.sync());
        } else {
            list = lists[out ^ 1].ptr;
            count = scratch.ptr + 2 + (out ^ 1);
            if (n > 0) {
                const unsigned mark_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(n, 256), cap));
                GCU_LAUNCH(dev, "kt_mark", kt_mark_kernel, mark_grid, 256, 0, list, count, state.ptr, round,
                           truss.ptr, k - 1);
            }
        }
        if (n == 0) {
            // Every alive edge has at least k - 2 alive triangles: it is in the k-truss.
            top = k;
            k += 1;
            level_start = true;
            continue;
        }
        alive -= n;
        GCU_CUDA(cudaMemsetAsync(scratch.ptr + 2 + out, 0, sizeof(uint32_t), dev.stream), "memset");
        GCU_TRY(launch_peel(dev, g, live, src, rev, state.ptr, support.ptr, list, count, n, chunks.ptr, round, k - 2,
                            lists[out].ptr, scratch.ptr + 2 + out));
        GCU_CUDA(cudaMemcpyAsync(&n, scratch.ptr + 2 + out, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        out ^= 1;
        level_start = false;
        if (alive > 0 && 2 * alive < listed) {
            GCU_CUDA(cudaMemsetAsync(scratch.ptr + 1, 0, sizeof(uint32_t), dev.stream), "memset");
            GCU_LAUNCH(dev, "kt_active", kt_active_kernel, grid, 256, 0, g.targets.ptr, src, state.ptr,
                       active[cur].ptr, static_cast<uint32_t>(listed), active[cur ^ 1].ptr, scratch.ptr + 1);
            cur ^= 1;
            listed = alive;
            // The peel's lists too: the alive entries only (the removals
            // listed for the next round are still alive and stay).
            GCU_TRY(compact_live(dev, g.num_nodes, live, live_entries, rev, state.ptr, &live_bufs[live_cur ^ 1]));
            live_cur ^= 1;
            live = LiveCsr{live_bufs[live_cur].offsets.ptr, live_bufs[live_cur].targets.ptr,
                           live_bufs[live_cur].eid.ptr};
            live_entries = live_bufs[live_cur].entries;
        }
    }
    *max_truss = top;
    *rounds = round;
    if (host_truss) {
        GCU_LAUNCH(dev, "kt_truss_spread", kt_truss_spread_kernel, edge_grid, 256, 0, g.targets.ptr, src, rev,
                   truss.ptr, E, support.ptr);
        GCU_TRY(copy_to_host(dev, host_truss, support.ptr, sizeof(uint32_t) * static_cast<size_t>(E)));
    }
    return ok();
}

}  // namespace gcu
