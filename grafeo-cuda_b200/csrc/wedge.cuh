// Wedge enumeration over a DAG CSR with shared-memory tables.
//
// Shared by triangle counting and k-truss support counting. For a vertex u
// with out-list N+(u), the keys of N+(u) go into a table in shared memory: an
// open-addressing hash table (multiplicative hashing, linear probing, load
// <= 1/2, <= 1/4 where the slots allow) or, when the DAG is oriented by a
// vertex rank and u's rank fits, a bitmap of the ranks below u's. Then every
// wedge (v, w), v in N+(u), w in N+(v), is probed: a hit is a triangle
// {u, v, w}. The wedges of up to 32 v's at a time are spread evenly over the
// lanes of a warp by a warp scan of the d+(v) (a load-balanced search), so the
// reads of the N+(v) lists are coalesced and no lane idles on short lists.
#pragma once

#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr uint32_t kNotFound = 0xFFFFFFFFu;

// Smallest b >= 6 with 2^b >= 4n, at most max_bits: a table of 2^b slots at
// load <= 1/4 where the slots allow (most probes miss, and a miss walks the
// run to the next empty slot: 1.4 slots on average at load 1/4, 2.5 at 1/2).
// Callers keep n <= 2^(max_bits - 1), so the load never exceeds 1/2.
__host__ __device__ __forceinline__ uint32_t table_bits(uint32_t n, uint32_t max_bits) {
    uint32_t b = 6;
    while (b < max_bits && (1u << b) < 4 * n) ++b;
    return b;
}

__device__ __forceinline__ uint32_t hash_home(uint32_t key, uint32_t bits) {
    return (key * 2654435761u) >> (32 - bits);
}

// Inserts a key that is not yet present. Keys are distinct (sorted lists), so
// only the slot claim needs an atomic. Gives up after one sweep of the table,
// which cannot happen below load 1.
template <bool kWithPos>
__device__ __forceinline__ void hash_insert(uint32_t* keys, uint32_t* pos, uint32_t bits, uint32_t key,
                                            uint32_t value) {
    const uint32_t mask = (1u << bits) - 1;
    uint32_t s = hash_home(key, bits);
    for (uint32_t i = 0; i <= mask; ++i) {
        if (atomicCAS(keys + s, kEmptyKey, key) == kEmptyKey) {
            if (kWithPos) pos[s] = value;
            return;
        }
        s = (s + 1) & mask;
    }
}

// Position stored with `key`, kNotFound if absent (1 when kWithPos is false
// and the key is present).
template <bool kWithPos>
__device__ __forceinline__ uint32_t hash_find(const uint32_t* keys, const uint32_t* pos, uint32_t bits,
                                              uint32_t key) {
    const uint32_t mask = (1u << bits) - 1;
    uint32_t s = hash_home(key, bits);
    for (uint32_t i = 0; i <= mask; ++i) {
        const uint32_t k = keys[s];
        if (k == key) return kWithPos ? pos[s] : 1u;
        if (k == kEmptyKey) return kNotFound;
        s = (s + 1) & mask;
    }
    return kNotFound;
}

// Position of w in the sorted list a[0, n) or kNotFound (for lists too long
// for a shared-memory table).
__device__ __forceinline__ uint32_t sorted_find(const uint32_t* a, uint32_t n, uint32_t w) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t x = a[mid];
        if (x < w)
            lo = mid + 1;
        else if (x > w)
            hi = mid;
        else
            return mid;
    }
    return kNotFound;
}

// Walks the wedges of the out-neighbours v = list[c .. c + 31] of u (list =
// N+(u), du entries); for every entry v -> w whose value values[entry] (the
// target w itself, or its rank) find() locates in N+(u) calls
// hit(pos_v, pos_w, entry_vw): positions of v and w in N+(u) and the CSR entry
// index of v -> w. Out-neighbours with more than max_dv out-edges are skipped
// (their edges are counted from the other end). s_excl (33 words) / s_start
// (32 words) are per-warp scratch.
template <class Find, class Hit>
__device__ __forceinline__ void wedge_chunk(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ values,
                                            const uint32_t* list, uint32_t du, uint32_t c, uint32_t* s_excl,
                                            uint32_t* s_start, uint32_t max_dv, Find find, Hit hit) {
    const unsigned lane = lane_id();
    uint32_t vs = 0, dv = 0;
    if (c + lane < du) {
        const uint32_t v = list[c + lane];
        vs = offsets[v];
        dv = offsets[v + 1] - vs;
        if (dv > max_dv) dv = 0;
    }
    const uint32_t inc = warp_inclusive_scan(dv);
    const uint32_t total = __shfl_sync(kFullMask, inc, 31);
    __syncwarp();
    s_excl[lane] = inc - dv;
    s_start[lane] = vs;
    if (lane == 0) s_excl[32] = 0xFFFFFFFFu;  // stops the walk
    __syncwarp();
    // lo = the largest j with s_excl[j] <= k (the v owning wedge k); k only
    // grows, so each lane walks forward from its last v, with that v's first
    // wedge, list start and the next v's first wedge kept in registers: no
    // shared-memory read per wedge while a lane stays on one v.
    uint32_t lo = 0, first = 0, start = s_start[0], next = s_excl[1];
    for (uint32_t k = lane; k < total; k += 32) {
        while (next <= k) {
            ++lo;
            first = next;
            start = s_start[lo];
            next = s_excl[lo + 1];
        }
        const uint32_t entry = start + (k - first);
        const uint32_t p = find(values[entry]);
        if (p != kNotFound) hit(c + lo, p, entry);
    }
}

// First list entry of the next 32-entry chunk of the current CTA item
// (shared counter reset with the item): the warps of a CTA take chunks as
// they finish, so one long chunk does not keep the others at the barrier.
__device__ __forceinline__ uint32_t next_chunk(uint32_t* s_chunk) {
    uint32_t c = 0;
    if (lane_id() == 0) c = atomicAdd(s_chunk, 32u);
    return __shfl_sync(kFullMask, c, 0);
}

// ---------------------------------------------------------------- kernels

constexpr int kWedgeThreads = 256;
constexpr int kWedgeWarps = kWedgeThreads / 32;
constexpr uint32_t kWarpMaxDeg = 128;   // warp kernel: out-lists up to this length
constexpr uint32_t kWarpBits = 8;
constexpr uint32_t kWarpSlots = 1u << kWarpBits;  // hash slots per warp (load <= 1/2)
constexpr uint32_t kCtaMaxDeg = 2048;   // CTA kernel: hash table up to this length
constexpr uint32_t kCtaBits = 12;
constexpr uint32_t kCtaSlots = 1u << kCtaBits;
constexpr uint32_t kVertexBatch = 8;    // vertices fetched per warp at a time

// The lookup structure of a CTA item whose owner x has the out-list
// entries [s, s + d):
//  kBitmap: with ranks (a DAG oriented by a vertex order, rank[entry] = the
//    position of the entry's target in that order, every out-neighbour
//    ranked below its owner), a bitmap of the ranks below vrank[x] when it
//    fits the shared array: one bit test per probe, no probe loop, no hash;
//  kHash: a hash table of the values probed (ranks, or the targets);
//  kSearch: binary search of the sorted targets in global memory.
enum : int { kSearch = 0, kHash = 1, kBitmap = 2 };
struct CtaTable {
    int kind;
    uint32_t bits;             // kHash: log2 of the slots
    uint32_t limit;            // kBitmap: ranks below this are covered
    const uint32_t* values;    // what the probes look up (ranks or targets)
};

template <bool kPos>
__device__ __forceinline__ CtaTable build_cta_table(uint32_t* s_keys, uint32_t* pos,
                                                    const uint32_t* __restrict__ targets,
                                                    const uint32_t* __restrict__ rank,
                                                    const uint32_t* __restrict__ vrank, uint32_t x, uint32_t s,
                                                    uint32_t d, int search) {
    CtaTable t{kSearch, 0, 0, targets};
    if (search) return t;
    if (!kPos && rank) {
        t.values = rank;
        const uint32_t r = vrank[x];
        if (r <= kCtaSlots * 32) {
            t.kind = kBitmap;
            t.limit = r;
            for (uint32_t k = threadIdx.x; k < (r + 31) / 32; k += kWedgeThreads) s_keys[k] = 0;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < d; k += kWedgeThreads) {
                const uint32_t w = rank[s + k];
                if (w < r) atomicOr(s_keys + (w >> 5), 1u << (w & 31));
            }
            __syncthreads();
            return t;
        }
    }
    if (d <= kCtaMaxDeg) {
        t.kind = kHash;
        t.bits = table_bits(d, kCtaBits);
        for (uint32_t k = threadIdx.x; k < (1u << t.bits); k += kWedgeThreads) s_keys[k] = kEmptyKey;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < d; k += kWedgeThreads)
            hash_insert<kPos>(s_keys, pos, t.bits, t.values[s + k], k);
        __syncthreads();
        return t;
    }
    t.values = targets;
    return t;
}

// Position of the probed value w in the owner's list (kNotFound if absent; 0
// for any hit in a bitmap, which keeps no positions).
template <bool kPos>
__device__ __forceinline__ uint32_t cta_find(const CtaTable& t, const uint32_t* s_keys, const uint32_t* pos,
                                             const uint32_t* sorted_list, uint32_t d, uint32_t w) {
    if (t.kind == kBitmap) return (w < t.limit && ((s_keys[w >> 5] >> (w & 31)) & 1u)) ? 0u : kNotFound;
    if (t.kind == kHash) return hash_find<kPos>(s_keys, pos, t.bits, w);
    return sorted_find(sorted_list, d, w);
}

// A Sink receives every triangle: hit(row_base, pos_v, pos_w, entry_vw) with
// row_base = offsets[u] (so row_base + pos_v is the entry u -> v) and
// finish() once per thread at the end. Sink::kNeedsPos says whether the hash
// table has to keep the positions of the keys.

// Warp per vertex for out-lists of [min_deg, kWarpMaxDeg] entries; vertices
// are handed out dynamically kVertexBatch at a time.
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_warp_kernel(const uint32_t* __restrict__ offsets,
                                                                   const uint32_t* __restrict__ targets, uint32_t V,
                                                                   uint32_t min_deg, uint32_t* __restrict__ next_vertex,
                                                                   Sink sink) {
    constexpr bool kPos = Sink::kNeedsPos;
    __shared__ uint32_t s_keys[kWedgeWarps][kWarpSlots];
    __shared__ uint32_t s_pos[kPos ? kWedgeWarps : 1][kPos ? kWarpSlots : 1];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t* keys = s_keys[warp];
    uint32_t* pos = kPos ? s_pos[warp] : nullptr;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next_vertex, kVertexBatch);
        base = __shfl_sync(kFullMask, base, 0);
        if (base >= V) break;
        const uint32_t last = min(base + kVertexBatch, V);
        for (uint32_t u = base; u < last; ++u) {
            const uint32_t s = offsets[u], du = offsets[u + 1] - s;
            if (du < min_deg || du > kWarpMaxDeg) continue;
            const uint32_t bits = table_bits(du, kWarpBits);
            __syncwarp();
            for (uint32_t k = lane; k < (1u << bits); k += 32) keys[k] = kEmptyKey;
            __syncwarp();
            for (uint32_t k = lane; k < du; k += 32) hash_insert<kPos>(keys, pos, bits, targets[s + k], k);
            __syncwarp();
            for (uint32_t c = 0; c < du; c += 32)
                wedge_chunk(
                    offsets, targets, targets + s, du, c, s_excl[warp], s_start[warp], 0xFFFFFFFFu,
                    [&](uint32_t w) { return hash_find<kPos>(keys, pos, bits, w); },
                    [&](uint32_t pv, uint32_t pw, uint32_t evw) { sink.hit(s, pv, pw, evw); });
        }
    }
    sink.finish();
}

// Out-lists longer than kWarpMaxDeg: collect them for the CTA kernel.
static __global__ void wedge_collect_long_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                          uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (offsets[u + 1] - offsets[u] > kWarpMaxDeg) list[atomicAdd(count, 1u)] = static_cast<uint32_t>(u);
    }
}

// CTA per long out-list, handed out dynamically: a shared hash table when the
// list has at most kCtaMaxDeg entries, otherwise binary search of the list in
// global memory.
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_cta_kernel(const uint32_t* __restrict__ offsets,
                                                                  const uint32_t* __restrict__ targets,
                                                                  const uint32_t* __restrict__ long_list,
                                                                  const uint32_t* __restrict__ long_count,
                                                                  uint32_t* __restrict__ next_item, Sink sink) {
    constexpr bool kPos = Sink::kNeedsPos;
    __shared__ uint32_t s_keys[kCtaSlots];
    __shared__ uint32_t s_pos[kPos ? kCtaSlots : 1];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    __shared__ uint32_t s_item, s_chunk;
    const unsigned warp = threadIdx.x >> 5;
    const uint32_t n = *long_count;
    uint32_t* pos = kPos ? s_pos : nullptr;
    while (true) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(next_item, 1u);
            s_chunk = 0;
        }
        __syncthreads();
        const uint32_t h = s_item;
        if (h >= n) break;
        const uint32_t u = long_list[h];
        const uint32_t s = offsets[u], du = offsets[u + 1] - s;
        const uint32_t* list = targets + s;
        const bool use_table = du <= kCtaMaxDeg;
        const uint32_t bits = use_table ? table_bits(du, kCtaBits) : 0;
        if (use_table) {
            for (uint32_t k = threadIdx.x; k < (1u << bits); k += kWedgeThreads) s_keys[k] = kEmptyKey;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < du; k += kWedgeThreads) hash_insert<kPos>(s_keys, pos, bits, list[k], k);
            __syncthreads();
        }
        for (uint32_t c = next_chunk(&s_chunk); c < du; c = next_chunk(&s_chunk))
            wedge_chunk(
                offsets, targets, list, du, c, s_excl[warp], s_start[warp], 0xFFFFFFFFu,
                [&](uint32_t w) {
                    return use_table ? hash_find<kPos>(s_keys, pos, bits, w) : sorted_find(list, du, w);
                },
                [&](uint32_t pv, uint32_t pw, uint32_t evw) { sink.hit(s, pv, pw, evw); });
        __syncthreads();  // the table and s_item are reused by the next list
    }
    sink.finish();
}

// ---------------------------------------------------------------- bucket kernels
// The same intersections over an explicit vertex list (one out-degree bucket
// of a DAG), so that a schedule can pick the variant per bucket. Their sinks
// also get end_vertex(u) from every warp that worked on u, once it is done
// with u (all 32 lanes call it). With `split`, an edge u -> v whose head has
// more out-edges than its tail (d+(v) > d+(u) >= 2) is left to the head-side
// kernels below, which stream the shorter list N+(u) against a table of
// N+(v): every edge then costs min(d+(u), d+(v)) probes instead of d+(v).

// Warp per listed vertex; a shared hash table per warp for out-lists of at
// most kWarpMaxDeg entries, binary search in global memory beyond (the
// schedule only sends buckets within the limit here; the guard keeps the
// table in bounds whatever the list holds).
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_warp_list_kernel(const uint32_t* __restrict__ offsets,
                                                                        const uint32_t* __restrict__ targets,
                                                                        const uint32_t* __restrict__ list, uint32_t n,
                                                                        uint32_t* __restrict__ next, bool split,
                                                                        Sink sink) {
    constexpr bool kPos = Sink::kNeedsPos;
    __shared__ uint32_t s_keys[kWedgeWarps][kWarpSlots];
    __shared__ uint32_t s_pos[kPos ? kWedgeWarps : 1][kPos ? kWarpSlots : 1];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t* keys = s_keys[warp];
    uint32_t* pos = kPos ? s_pos[warp] : nullptr;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next, kVertexBatch);
        base = __shfl_sync(kFullMask, base, 0);
        if (base >= n) break;
        const uint32_t last = min(base + kVertexBatch, n);
        for (uint32_t h = base; h < last; ++h) {
            const uint32_t u = list[h];
            const uint32_t s = offsets[u], du = offsets[u + 1] - s;
            const bool use_table = du <= kWarpMaxDeg;
            const uint32_t bits = use_table ? table_bits(du, kWarpBits) : 0;
            __syncwarp();
            if (use_table) {
                for (uint32_t k = lane; k < (1u << bits); k += 32) keys[k] = kEmptyKey;
                __syncwarp();
                for (uint32_t k = lane; k < du; k += 32) hash_insert<kPos>(keys, pos, bits, targets[s + k], k);
                __syncwarp();
            }
            const uint32_t* ulist = targets + s;
            const uint32_t max_dv = split && du >= 2 ? du : 0xFFFFFFFFu;
            for (uint32_t c = 0; c < du; c += 32)
                wedge_chunk(
                    offsets, targets, ulist, du, c, s_excl[warp], s_start[warp], max_dv,
                    [&](uint32_t w) {
                        return use_table ? hash_find<kPos>(keys, pos, bits, w) : sorted_find(ulist, du, w);
                    },
                    [&](uint32_t pv, uint32_t pw, uint32_t evw) { sink.hit(s, pv, pw, evw); });
            sink.end_vertex(u);
        }
    }
    sink.finish();
}

// CTA per listed vertex: a shared bitmap of ranks (`rank` given, the owner's
// rank within the shared array), a shared hash table (out-lists of at most
// kCtaMaxDeg entries, unless `search`) or binary search of the out-list in
// global memory (build_cta_table).
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_cta_list_kernel(const uint32_t* __restrict__ offsets,
                                                                       const uint32_t* __restrict__ targets,
                                                                       const uint32_t* __restrict__ list, uint32_t n,
                                                                       uint32_t* __restrict__ next, int search,
                                                                       bool split, const uint32_t* __restrict__ rank,
                                                                       const uint32_t* __restrict__ vrank, Sink sink) {
    constexpr bool kPos = Sink::kNeedsPos;
    __shared__ uint32_t s_keys[kCtaSlots];
    __shared__ uint32_t s_pos[kPos ? kCtaSlots : 1];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    __shared__ uint32_t s_item, s_chunk;
    const unsigned warp = threadIdx.x >> 5;
    uint32_t* pos = kPos ? s_pos : nullptr;
    while (true) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(next, 1u);
            s_chunk = 0;
        }
        __syncthreads();
        const uint32_t h = s_item;
        if (h >= n) break;
        const uint32_t u = list[h];
        const uint32_t s = offsets[u], du = offsets[u + 1] - s;
        const uint32_t* ulist = targets + s;
        const CtaTable tab = build_cta_table<kPos>(s_keys, pos, targets, rank, vrank, u, s, du, search);
        const uint32_t max_dv = split && du >= 2 ? du : 0xFFFFFFFFu;
        for (uint32_t c = next_chunk(&s_chunk); c < du; c = next_chunk(&s_chunk))
            wedge_chunk(
                offsets, tab.values, ulist, du, c, s_excl[warp], s_start[warp], max_dv,
                [&](uint32_t w) { return cta_find<kPos>(tab, s_keys, pos, ulist, du, w); },
                [&](uint32_t pv, uint32_t pw, uint32_t evw) { sink.hit(s, pv, pw, evw); });
        sink.end_vertex(u);
        __syncthreads();  // the table and s_item are reused by the next list
    }
    sink.finish();
}

// ---------------------------------------------------------------- head-side kernels
// Item (v, k): the k-th slice of `slice` tails of v's in-list (in_src from
// in_off[v], the tails u with 2 <= d+(u) < d+(v)); slices are short enough
// that no single item holds up the end of a launch. The table holds N+(v);
// the out-lists of the slice's tails are streamed against it, balanced over
// the lanes by wedge_chunk; a hit w is a triangle u -> v, u -> w, v -> w.
// Sinks only count (hit positions are not the tail's).
constexpr uint32_t kHeadWarpSlice = 256;   // tails per item of the warp kernel
constexpr uint32_t kHeadCtaSlice = 1024;   // tails per item of the CTA kernel

__device__ __forceinline__ void head_slice(const uint2 item, const uint32_t* __restrict__ in_off,
                                           const uint32_t* __restrict__ in_src, uint32_t slice,
                                           const uint32_t*& tails, uint32_t& count) {
    const uint32_t b = in_off[item.x] + item.y * slice, e = in_off[item.x + 1];
    tails = in_src + b;
    count = min(slice, e - b);
}

// Warp per item, heads with at most kWarpMaxDeg out-edges (binary search of
// N+(v) beyond, to stay in bounds whatever the items hold).
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_head_warp_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint2* __restrict__ items,
    uint32_t n, const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_src, uint32_t* __restrict__ next,
    Sink sink) {
    __shared__ uint32_t s_keys[kWedgeWarps][kWarpSlots];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t* keys = s_keys[warp];
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(next, kVertexBatch);
        base = __shfl_sync(kFullMask, base, 0);
        if (base >= n) break;
        const uint32_t last = min(base + kVertexBatch, n);
        for (uint32_t h = base; h < last; ++h) {
            const uint2 item = items[h];
            const uint32_t s = offsets[item.x], dv = offsets[item.x + 1] - s;
            const uint32_t* vlist = targets + s;
            const bool use_table = dv <= kWarpMaxDeg;
            const uint32_t bits = use_table ? table_bits(dv, kWarpBits) : 0;
            __syncwarp();
            if (use_table) {
                for (uint32_t k = lane; k < (1u << bits); k += 32) keys[k] = kEmptyKey;
                __syncwarp();
                for (uint32_t k = lane; k < dv; k += 32) hash_insert<false>(keys, nullptr, bits, vlist[k], k);
                __syncwarp();
            }
            const uint32_t* tails;
            uint32_t count;
            head_slice(item, in_off, in_src, kHeadWarpSlice, tails, count);
            for (uint32_t c = 0; c < count; c += 32)
                wedge_chunk(
                    offsets, targets, tails, count, c, s_excl[warp], s_start[warp], 0xFFFFFFFFu,
                    [&](uint32_t w) {
                        return use_table ? hash_find<false>(keys, nullptr, bits, w) : sorted_find(vlist, dv, w);
                    },
                    [&](uint32_t pu, uint32_t pw, uint32_t e) { sink.hit(s, pu, pw, e); });
        }
    }
    sink.finish();
}

// CTA per item: a shared table of N+(v) (at most kCtaMaxDeg entries, unless
// `search`) or binary search of N+(v) in global memory.
template <class Sink>
__global__ void __launch_bounds__(kWedgeThreads) wedge_head_cta_kernel(
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets, const uint2* __restrict__ items,
    uint32_t n, const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_src, uint32_t* __restrict__ next,
    int search, const uint32_t* __restrict__ rank, const uint32_t* __restrict__ vrank, Sink sink) {
    __shared__ uint32_t s_keys[kCtaSlots];
    __shared__ uint32_t s_excl[kWedgeWarps][33];
    __shared__ uint32_t s_start[kWedgeWarps][32];
    __shared__ uint32_t s_item, s_chunk;
    const unsigned warp = threadIdx.x >> 5;
    while (true) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(next, 1u);
            s_chunk = 0;
        }
        __syncthreads();
        const uint32_t h = s_item;
        if (h >= n) break;
        const uint2 item = items[h];
        const uint32_t s = offsets[item.x], dv = offsets[item.x + 1] - s;
        const uint32_t* vlist = targets + s;
        const CtaTable tab = build_cta_table<false>(s_keys, nullptr, targets, rank, vrank, item.x, s, dv, search);
        const uint32_t* tails;
        uint32_t count;
        head_slice(item, in_off, in_src, kHeadCtaSlice, tails, count);
        for (uint32_t c = next_chunk(&s_chunk); c < count; c = next_chunk(&s_chunk))
            wedge_chunk(
                offsets, tab.values, tails, count, c, s_excl[warp], s_start[warp], 0xFFFFFFFFu,
                [&](uint32_t w) { return cta_find<false>(tab, s_keys, nullptr, vlist, dv, w); },
                [&](uint32_t pu, uint32_t pw, uint32_t e) { sink.hit(s, pu, pw, e); });
        __syncthreads();  // the table and s_item are reused by the next item
    }
    sink.finish();
}

// Runs both wedge kernels over a DAG CSR: long out-lists by CTAs first (they
// hold the heaviest work), then everything else by warps.
template <class Sink>
Error run_wedges(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets, uint32_t V, uint32_t min_deg,
                 Sink sink, const char* tag) {
    (void)tag;
    // scratch: [0] next vertex, [1] long-list count, [2] next long list, then the long lists
    DeviceBuffer<uint32_t> scratch;
    GCU_TRY(scratch.allocate(dev, 4 + static_cast<uint64_t>(V)));
    GCU_CUDA(cudaMemsetAsync(scratch.ptr, 0, 4 * sizeof(uint32_t), dev.stream), "memset");
    const unsigned grid = static_cast<unsigned>(dev.sm_count) * 8;
    const unsigned collect_blocks =
        static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), static_cast<uint64_t>(dev.sm_count) * 8));
    GCU_LAUNCH(dev, "wedge_collect_long", wedge_collect_long_kernel, collect_blocks, 256, 0, d_offsets, V,
               scratch.ptr + 4, scratch.ptr + 1);
    GCU_LAUNCH(dev, "wedge_cta", wedge_cta_kernel<Sink>, grid, kWedgeThreads, 0, d_offsets, d_targets,
               scratch.ptr + 4, scratch.ptr + 1, scratch.ptr + 2, sink);
    GCU_LAUNCH(dev, "wedge_warp", wedge_warp_kernel<Sink>, grid, kWedgeThreads, 0, d_offsets, d_targets, V, min_deg,
               scratch.ptr, sink);
    return ok();
}

}  // namespace gcu
