// PageRank: pull SpMV over a degree-relabelled copy of the CSR, with the rank
// update, the L1 residual and the dangling mass fused into its epilogue.
//
// Reference: crates/grafeo-cuda-algos/src/pagerank.rs:46-199 and
// kernels/pagerank.cu:19-134. Per iteration the reference launches four
// kernels (dangling sum, thread-per-row SpMV, L1 diff, plus memsets), reads
// `ranks_in[u] / deg[u]` with two random gathers and a divide per edge, and
// syncs the host to read the f32 diff. What bounds a pull SpMV on a power-law
// graph is the random gather of the source contributions (one L1TEX sector
// per edge), not the streamed CSR; the design follows from that:
//
//  * Relabelling (once per graph, cached): vertices are stably partitioned by
//    degree class, class c holding degrees in [2^(c-1), 2^c), highest class
//    first and ids ascending inside a class. Hubs get the smallest new ids,
//    so their contributions share sectors and cache lines and most gathers
//    hit L1/L2 lines that are already hot. The relabelled CSR keeps every
//    list in its original order, so each row's summation order is the
//    original one.
//  * Rows of 1024 or more entries (the relabelling puts them first) are split
//    into 1024-entry segments, one warp each, 8 loads in flight per lane, and
//    their partial sums are added in segment order by the finishing kernel.
//  * Rows of 1 to 1023 entries (pr_chunks_kernel) are read as a stream of
//    256-entry chunks, one warp per chunk and 8 consecutive entries per lane
//    (two 128-bit target loads and one 64-bit load of the entries' row deltas,
//    a byte each), so every lane keeps 8 gathers in flight whatever the row
//    lengths; runs of equal rows are summed per lane, joined across lanes by a
//    warp segmented scan, and finished by the lane where they end, and the
//    rows that cross chunks are finished from their per-chunk parts, in chunk
//    order, by the finishing kernel. The lane-group form it replaced (a group
//    of 2^(c-1) lanes per row of class c, 1 to 2 entries per lane and row)
//    stays behind kChunkRows = false.
//  * Work units (a long-row segment, a chunk, or 32 rows without entries)
//    are dealt round-robin to the warps of persistent grids: the warps in
//    flight read one contiguous window of the CSR, and no block barrier ties
//    the warps of a CTA together.
//  * Row sums: FP32 Kahan sums per lane and FP64 across lanes and segments for
//    the long rows, FP64 for the chunked rows. Epilogue per row v: r'[v] = (1-d)/N + d (sum +
//    dangling/N); |r' - r| and the dangling mass of r' are summed as 64-bit
//    fixed-point integers (2^-62 units) in registers per lane, then per warp
//    and per CTA, and reduced by the last block of the finishing kernel (no
//    shared-memory atomics: same-address atomics of a warp's rows cost a
//    quarter of the L1TEX wavefronts); integer sums do not depend on the order, so the
//    result is deterministic whatever the grid size (no float atomics);
//    c'[v] = r'[v] / deg(v) is written for the next iteration.
//  * The iteration loop stays on the device: each kernel reads a `done` flag
//    first, so the host queues iterations ahead and polls the flag once per
//    chunk instead of syncing every iteration.
#include <algorithm>
#include <cmath>
#include <vector>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

// Two CTAs of 1024 threads per SM: the 32 warps of a CTA hold consecutive
// work units, so an SM works on two contiguous windows of rows at a time
// instead of eight, and their gathers share more L1 lines; 32 registers, 64
// warps per SM. Measured per iteration (R-MAT 24 directed / R-MAT 22 /
// Erdos-Renyi 2^22; same ranks bit for bit): 8 x 256 threads 1.871 / 0.448 /
// 0.893 ms, 4 x 512 1.833 / 0.434 / -, 2 x 1024 1.778 / 0.437 / 0.882, 2 x 768
// (40 registers, 48 warps) 1.759 / 0.429 / 0.992: with fewer warps the
// Erdos-Renyi gathers, none of which hit L1, have fewer loads in flight.
constexpr int kPrThreads = 1024;
constexpr int kDegClasses = 33;       // class 0: degree 0; class c: degree in [2^(c-1), 2^c)
constexpr int kLongClass = 11;        // degree >= 1024
constexpr uint32_t kSegment = 1024;   // entries per long-row segment (one warp)
constexpr int kClassBlock = 1024;     // vertices per block of the class partition
constexpr int kMaxPhases = 16;
constexpr int kRowsPerGroup = 2;      // rows a lane group works on in lockstep
constexpr int kUnroll = 2;            // steps per loop trip: kRowsPerGroup * kUnroll loads in flight
constexpr int kRowCtasPerSm = 2;      // persistent CTAs of the row kernel per SM
// Hub cache: every CTA of the row kernel copies the contributions of the new
// ids [0, kHubEntries) (the highest-degree vertices, which take the largest
// share of the gathers) into shared memory at the start of a launch and
// gathers below that bound from there; 0 turns it off. Measured on B200
// (same ranks bit for bit): 16K entries (40 % of the gathers at R-MAT 22) with
// two 768-thread CTAs per SM ran R-MAT 22 2.6 % faster than the plain 8 x 256
// kernel but R-MAT 24 no faster than two 1024-thread CTAs without it; 24K and
// 32K entries ran slower (the carve-out shrinks L1). Off.
constexpr uint32_t kHubEntries = 0;
// Load the next group-phase unit's row offsets while working on this one.
// It needs 40 registers; measured slower (2 x 768 threads: 1.923 against
// 1.759 ms per iteration at R-MAT 24 directed, 0.480 against 0.429 ms at
// R-MAT 22): off.
constexpr bool kPrefetchRows = false;

// Rows of 1 to 1023 entries, read as a stream of chunks: kChunk consecutive
// entries of the relabelled CSR per warp (rows packed back to back, a row
// that crosses a chunk boundary split between the chunks), 8 consecutive
// entries per lane, loaded as two 128-bit target loads and one 64-bit load of
// their row deltas (row minus the chunk's first row: a chunk holds at most
// kChunk rows, each with an entry, so a byte holds it). A lane sums its runs
// of equal rows, a segmented scan over the warp joins the runs that cross
// lanes, and the lane where a row ends finishes it; the parts of a row that
// crosses chunks are added, in chunk order, by the finishing kernel. Every
// lane keeps 8 gathers in flight with no row offsets in the chain, against
// 1 to 2 entries per lane and row in the lane-group form (kChunkRows = false:
// rows of class c served by groups of 2^(c-1) lanes).
constexpr bool kChunkRows = true;
constexpr uint32_t kChunk = 256;
constexpr int kChunkThreads = 512;
constexpr int kChunkCtasPerSm = 2;
constexpr uint32_t kNoRow = 0xFFFFFFFFu;

enum : uint32_t { kPhaseLong = 0, kPhaseGroup = 1, kPhaseEmpty = 2 };

struct PrPhase {
    uint32_t first_block;  // first work unit of this phase
    uint32_t row_begin, row_end;
    uint32_t kind;
    uint32_t log2g;        // lanes per row = 1 << log2g (group phases)
    uint32_t rows_per_group;  // rows a lane group works on together (group phases)
};

struct PrSchedule {
    uint32_t nphases;
    uint32_t total_blocks;
    PrPhase phase[kMaxPhases];
};

struct PrState {
    double dangling;   // sum of ranks of dangling vertices in the current input ranks
    double last_diff;  // L1 change of the last iteration
    uint32_t iterations;
    uint32_t done;
    uint32_t ticket;
    uint32_t pad;
};

struct PageRankPlan {
    uint32_t long_rows = 0;   // rows [0, long_rows) of the relabelled CSR have >= 1024 entries
    uint32_t empty_rows = 0;  // rows without entries (the last class)
    uint32_t dangling_rows = 0;  // vertices without out-edges
    uint32_t fin_blocks = 1;
    uint32_t row_ctas = 1;    // persistent CTAs of the row kernel
    PrSchedule sched{};
    DeviceBuffer<uint32_t> perm;       // new id -> original id
    DeviceBuffer<uint32_t> inv;        // original id -> new id
    DeviceBuffer<uint32_t> poff;       // relabelled offsets (V + 1)
    DeviceBuffer<uint32_t> ptgt;       // relabelled targets (E)
    DeviceBuffer<uint32_t> outdeg;     // out-degrees, relabelled order (only when pulling over the transpose)
    DeviceBuffer<uint2> units;         // long-row segments: (row, segment)
    DeviceBuffer<uint32_t> unit_begin; // long row i owns units [unit_begin[i], unit_begin[i+1])
    DeviceBuffer<double> seg_partial;  // one partial sum per unit
    DeviceBuffer<float> ranks;         // 2 * V: ping-pong, relabelled order
    DeviceBuffer<float> contrib;       // 2 * V: ping-pong, relabelled order
    DeviceBuffer<float> ranks_out;     // V: result in original order
    DeviceBuffer<unsigned long long> row_partials; // 2 fixed-point sums per CTA of the row kernel
    DeviceBuffer<unsigned long long> fin_partials; // 2 per block of the finishing kernel
    DeviceBuffer<PrState> state;
    // Host copy of the state, read after each poll's synchronisation: plain
    // memory (a 32-byte copy needs no pinned page, and a graph's setup and
    // release then make no page-locking calls).
    PrState host_state{};
    // Chunked rows (kChunkRows): entries [chunk_lo, chunk_hi) of the relabelled
    // CSR, chunk c covering entries chunk_origin + kChunk c .. + kChunk - 1.
    uint32_t chunk_origin = 0, chunk_lo = 0, chunk_hi = 0;
    uint32_t n_chunks = 0, n_split = 0, chunk_ctas = 0;
    DeviceBuffer<uint32_t> chunk_row;   // first row of each chunk
    DeviceBuffer<uint8_t> chunk_delta;  // per entry: its row minus its chunk's first row
    DeviceBuffer<uint4> split_rows;     // (row, first chunk, last chunk, 0) of the rows that cross chunks
    DeviceBuffer<double> chunk_part;    // per chunk: the part of its first row (begun before it), of its last row (going on)
};

void destroy_pagerank_plan(PageRankPlan* p) {
    if (!p) return;
    delete p;
}

// ---------------------------------------------------------------- relabelling kernels

__host__ __device__ __forceinline__ uint32_t degree_class(uint32_t d) {
#ifdef __CUDA_ARCH__
    return d == 0 ? 0u : 32u - static_cast<uint32_t>(__clz(d));
#else
    uint32_t c = 0;
    while (d) {
        ++c;
        d >>= 1;
    }
    return c;
#endif
}

// counts[(K-1-c) * nblk + blk] = vertices of class c in block blk, so that an
// exclusive scan gives every (class, block) its first new id, classes descending.
__global__ void __launch_bounds__(kClassBlock) pr_class_count_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                                                     uint32_t nblk, uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[kDegClasses];
    if (threadIdx.x < kDegClasses) h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t v = static_cast<uint64_t>(blockIdx.x) * kClassBlock + threadIdx.x;
    if (v < V) atomicAdd(&h[degree_class(offsets[v + 1] - offsets[v])], 1u);
    __syncthreads();
    if (threadIdx.x < kDegClasses) counts[(kDegClasses - 1 - threadIdx.x) * nblk + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: the rank of v among the vertices of its class in its block
// comes from per-warp class matches and a prefix over the warps.
__global__ void __launch_bounds__(kClassBlock) pr_class_scatter_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                                                       uint32_t nblk, const uint32_t* __restrict__ cpos,
                                                                       uint32_t* __restrict__ perm,
                                                                       uint32_t* __restrict__ inv) {
    __shared__ uint32_t wcnt[kClassBlock / 32][kDegClasses];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint32_t k = threadIdx.x; k < (kClassBlock / 32) * kDegClasses; k += kClassBlock) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    const uint64_t v = static_cast<uint64_t>(blockIdx.x) * kClassBlock + threadIdx.x;
    const uint32_t c = v < V ? degree_class(offsets[v + 1] - offsets[v]) : kDegClasses;
    const unsigned same = __match_any_sync(kFullMask, c);
    const uint32_t rank = __popc(same & ((1u << lane) - 1));
    if (c < kDegClasses && lane == static_cast<unsigned>(__ffs(same) - 1)) wcnt[warp][c] = __popc(same);
    __syncthreads();
    if (threadIdx.x < kDegClasses) {
        uint32_t run = 0;
        for (int w = 0; w < kClassBlock / 32; ++w) {
            const uint32_t t = wcnt[w][threadIdx.x];
            wcnt[w][threadIdx.x] = run;
            run += t;
        }
    }
    __syncthreads();
    if (v < V) {
        const uint32_t pos = cpos[(kDegClasses - 1 - c) * nblk + blockIdx.x] + wcnt[warp][c] + rank;
        perm[pos] = static_cast<uint32_t>(v);
        inv[v] = pos;
    }
}

// First new id of every class (index c), plus V at index K.
__global__ void pr_class_starts_kernel(const uint32_t* __restrict__ cpos, uint32_t nblk, uint32_t* __restrict__ starts) {
    const uint32_t c = threadIdx.x;
    if (c < kDegClasses) starts[c] = cpos[(kDegClasses - 1 - c) * nblk];
    if (c == kDegClasses) starts[c] = cpos[kDegClasses * nblk];
}

__global__ void pr_perm_degree_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ perm,
                                      uint32_t V, uint32_t* __restrict__ pdeg) {
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < V;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = perm[r];
        pdeg[r] = offsets[u + 1] - offsets[u];
    }
}

Error degree_class_order(DeviceImpl& dev, const uint32_t* offsets, uint32_t V, DeviceBuffer<uint32_t>* inv) {
    GCU_TRY(inv->allocate(dev, std::max<uint32_t>(V, 1)));
    if (V == 0) return ok();
    const uint32_t nblk = static_cast<uint32_t>(ceil_div_u64(V, kClassBlock));
    const uint64_t ncount = static_cast<uint64_t>(kDegClasses) * nblk;
    DeviceBuffer<uint32_t> counts, cpos, perm;
    GCU_TRY(counts.allocate(dev, ncount));
    GCU_TRY(cpos.allocate(dev, ncount + 1));
    GCU_TRY(perm.allocate(dev, V));
    GCU_LAUNCH(dev, "pr_class_count", pr_class_count_kernel, nblk, kClassBlock, 0, offsets, V, nblk, counts.ptr);
    GCU_TRY(exclusive_scan_u32(dev, counts.ptr, cpos.ptr, ncount));
    GCU_LAUNCH(dev, "pr_class_scatter", pr_class_scatter_kernel, nblk, kClassBlock, 0, offsets, V, nblk, cpos.ptr,
               perm.ptr, inv->ptr);
    return ok();
}

// Relabelled CSR entry k of row r is original entry offsets[perm[r]] +
// (k - poff[r]) with its target renamed. Blocks work on tiles of consecutive
// output entries (rows found through the staged row starts), so a hub's list
// is copied by many blocks, reads and writes coalesced.
constexpr int kFillThreads = 256;
constexpr int kFillItems = 4;
constexpr int kFillTile = kFillThreads * kFillItems;

// With `delta`, entries in [lo, hi) also get their chunk row delta.
__global__ void __launch_bounds__(kFillThreads) pr_perm_fill_kernel(const uint32_t* __restrict__ offsets,
                                                                    const uint32_t* __restrict__ targets,
                                                                    const uint32_t* __restrict__ perm,
                                                                    const uint32_t* __restrict__ inv,
                                                                    const uint32_t* __restrict__ poff, uint32_t V,
                                                                    uint32_t E, uint32_t* __restrict__ ptgt,
                                                                    const uint32_t* __restrict__ chunk_row,
                                                                    uint32_t origin, uint32_t lo, uint32_t hi,
                                                                    uint8_t* __restrict__ delta) {
    __shared__ uint32_t s_start[kFillTile];
    __shared__ uint32_t s_meta[2];
    for (uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kFillTile; e0 < E;
         e0 += static_cast<uint64_t>(gridDim.x) * kFillTile) {
        const uint64_t e1 = min_u64(e0 + kFillTile, E);
        const bool staged = stage_tile_rows<kFillTile>(poff, V, e0, e1, s_start, s_meta);
        const uint32_t r0 = s_meta[0], nrows = s_meta[1] - r0 + 1;
#pragma unroll
        for (int q = 0; q < kFillItems; ++q) {
            const uint64_t k = e0 + q * kFillThreads + threadIdx.x;
            if (k >= e1) continue;
            const uint32_t r = tile_row(poff, V, s_start, staged, r0, nrows, static_cast<uint32_t>(k));
            const uint32_t src = offsets[perm[r]] + static_cast<uint32_t>(k - poff[r]);
            ptgt[k] = inv[ld_stream(targets + src)];
            if (delta && k >= lo && k < hi) {
                const uint32_t rel = static_cast<uint32_t>(k) - origin;
                delta[rel] = static_cast<uint8_t>(r - chunk_row[rel / kChunk]);
            }
        }
        __syncthreads();  // the staged starts are rewritten for the next tile
    }
}

// Chunk c's first row is the row holding its first entry (chunk 0: the first
// chunked row, which may begin a few entries into it); a row of the chunked
// range [r0, r1) is split when its entries fall in more than one chunk.
__global__ void pr_chunk_rows_kernel(const uint32_t* __restrict__ poff, uint32_t r0, uint32_t r1, uint32_t origin,
                                     uint32_t* __restrict__ chunk_row, uint32_t* __restrict__ split_flag) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < r1 - r0;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t r = r0 + static_cast<uint32_t>(i);
        const uint32_t s = poff[r] - origin, e = poff[r + 1] - origin;  // e > s: every chunked row has entries
        const uint32_t c_first = s / kChunk, c_last = (e - 1) / kChunk;
        for (uint32_t c = r == r0 ? 0 : (s + kChunk - 1) / kChunk; c <= c_last; ++c) chunk_row[c] = r;
        split_flag[i] = c_first != c_last ? 1u : 0u;
    }
}

__global__ void pr_split_rows_kernel(const uint32_t* __restrict__ poff, uint32_t r0, uint32_t n, uint32_t origin,
                                     const uint32_t* __restrict__ split_pos, uint4* __restrict__ split_rows) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (split_pos[i + 1] == split_pos[i]) continue;
        const uint32_t r = r0 + static_cast<uint32_t>(i);
        split_rows[split_pos[i]] =
            make_uint4(r, (poff[r] - origin) / kChunk, (poff[r + 1] - 1 - origin) / kChunk, 0u);
    }
}

// Segment count of every long row (a row of d entries has ceil(d / kSegment)).
__global__ void pr_unit_count_kernel(const uint32_t* __restrict__ poff, uint32_t long_rows,
                                     uint32_t* __restrict__ counts) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < long_rows;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        counts[i] = static_cast<uint32_t>(ceil_div_u64(poff[i + 1] - poff[i], kSegment));
}

// units[unit_begin[i] + s] = (i, s) for every segment s of long row i.
__global__ void pr_unit_fill_kernel(const uint32_t* __restrict__ poff, uint32_t long_rows,
                                    const uint32_t* __restrict__ unit_begin, uint2* __restrict__ units) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < long_rows;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint32_t u = unit_begin[i], sgm = 0; u < unit_begin[i + 1]; ++u, ++sgm)
            units[u] = make_uint2(static_cast<uint32_t>(i), sgm);
}

__global__ void pr_init_kernel(const uint32_t* __restrict__ poff, const uint32_t* __restrict__ outdeg, uint32_t V,
                               float r0, float* __restrict__ ranks, float* __restrict__ contrib) {
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t deg = outdeg ? outdeg[v] : poff[v + 1] - poff[v];
        ranks[v] = r0;
        contrib[v] = deg > 0 ? r0 / static_cast<float>(deg) : 0.f;
    }
}

// Out-degrees from the original CSR, in relabelled order; counts the vertices
// without out-edges (the dangling ones).
__global__ void pr_outdeg_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ perm, uint32_t V,
                                 uint32_t* __restrict__ outdeg, uint32_t* __restrict__ dangling_count) {
    uint32_t zeros = 0;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < V;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t u = perm[r];
        const uint32_t d = offsets[u + 1] - offsets[u];
        outdeg[r] = d;
        zeros += d == 0 ? 1u : 0u;
    }
    zeros = warp_sum(zeros);
    if (lane_id() == 0 && zeros) atomicAdd(dangling_count, zeros);
}

// Personalisation vector in relabelled order.
__global__ void pr_permute_tele_kernel(const float* __restrict__ tele, const uint32_t* __restrict__ perm, uint32_t V,
                                       float* __restrict__ out) {
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < V;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        out[r] = tele[perm[r]];
    }
}

__global__ void pr_unpermute_kernel(const float* __restrict__ ranks, const uint32_t* __restrict__ inv, uint32_t V,
                                    float* __restrict__ out) {
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        out[v] = ranks[inv[v]];
    }
}

// ---------------------------------------------------------------- iteration kernels

// Row update shared by the row and finishing kernels. row_len is the length
// of the pulled row; the out-degree is that length (symmetric graph) or
// outdeg[v] (pull over the transpose). Uniform teleport: r = (1-d)/N +
// d (sum + dangling/N); with a personalisation vector p: r = (1-d) p[v] +
// d (sum + dangling p[v]).
__device__ __forceinline__ void pr_finish_row(uint32_t v, double sum, uint32_t row_len,
                                              const float* __restrict__ rank_in, float* __restrict__ rank_out,
                                              float* __restrict__ contrib_out, const uint32_t* __restrict__ outdeg,
                                              const float* __restrict__ tele, double base, double damp,
                                              double spread, double dangling, double& diff, double& dangle) {
    const uint32_t deg = outdeg ? outdeg[v] : row_len;
    float r;
    if (tele) {
        const double pv = static_cast<double>(tele[v]);
        r = static_cast<float>((1.0 - damp) * pv + damp * (sum + dangling * pv));
    } else {
        r = static_cast<float>(base + damp * (sum + spread));
    }
    const float old = rank_in[v];
    diff += fabs(static_cast<double>(r) - static_cast<double>(old));
    rank_out[v] = r;
    contrib_out[v] = deg > 0 ? r / static_cast<float>(deg) : 0.f;
    if (deg == 0) dangle += static_cast<double>(r);
}

// The L1 change and the dangling mass are summed as 64-bit fixed-point
// integers (units of 2^-62; every term lies in [0, 2] and so does every sum):
// integer addition is associative, so the totals do not depend on which CTA
// handled which rows, and the dynamic block handout stays deterministic.
__device__ __forceinline__ unsigned long long to_fixed(double x) {
    return __double2ull_rz(x * 4611686018427387904.0);
}
__device__ __forceinline__ double from_fixed(unsigned long long q) {
    return static_cast<double>(q) * (1.0 / 4611686018427387904.0);
}

__device__ __forceinline__ void kahan_add(float& acc, float& comp, float x) {
    const float y = x - comp;
    const float t = acc + y;
    comp = (t - acc) - y;
    acc = t;
}

// Sum over lanes of an aligned group of 2^log2g lanes (all 32 lanes call it).
__device__ __forceinline__ double group_sum(double v, uint32_t log2g) {
    for (uint32_t o = (1u << log2g) >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

// Persistent: warp w of W works on units w, w + W, w + 2W, ... (a unit is a
// 1024-entry segment of a long row, the 2 rows per lane group of one warp in a
// degree class, or 32 rows without entries). Every phase's units are spread
// evenly over the warps, the warps in flight read one contiguous window of
// the CSR, and no block barrier ties the warps of a CTA together inside the
// loop. 2 CTAs of 1024 threads per SM.

// Phase of work unit b.
__device__ __forceinline__ uint32_t unit_phase(const PrSchedule& sched, uint32_t b) {
    uint32_t pi = 0;
    while (pi + 1 < sched.nphases && sched.phase[pi + 1].first_block <= b) ++pi;
    return pi;
}

// Row bounds of this lane's kRowsPerGroup rows in work unit b of a group
// phase (0, 0 past the phase's last row).
__device__ __forceinline__ void unit_rows(const PrPhase& ph, uint32_t b, unsigned lane,
                                          const uint32_t* __restrict__ poff, uint32_t* rs, uint32_t* re) {
    const uint32_t groups = 32u >> ph.log2g, group = lane >> ph.log2g;
    const uint32_t first = ph.row_begin + (b - ph.first_block) * groups * kRowsPerGroup;
#pragma unroll
    for (int q = 0; q < kRowsPerGroup; ++q) {
        const uint32_t row = first + q * groups + group;
        rs[q] = 0;
        re[q] = 0;
        if (row < ph.row_end) {
            rs[q] = poff[row];
            re[q] = poff[row + 1];
        }
    }
}

// Contribution of source t: from the shared hub copy when t < kHubEntries
// (every target is below V, so such a t is inside the copied min(V,
// kHubEntries) entries), else a gather from global memory.
__device__ __forceinline__ float gather_contrib(const float* s_hub, const float* __restrict__ contrib, uint32_t t) {
    if (kHubEntries > 0 && t < kHubEntries) return s_hub[t];
    return __ldg(contrib + t);
}

__global__ void __launch_bounds__(kPrThreads, kRowCtasPerSm) pr_rows_kernel(
    const uint32_t* __restrict__ poff, const uint32_t* __restrict__ ptgt, const float* __restrict__ rank_in,
    const float* __restrict__ contrib_in, float* __restrict__ rank_out, float* __restrict__ contrib_out,
    const uint32_t* __restrict__ outdeg, const float* __restrict__ tele, uint32_t V, double base, double damp,
    const PrState* __restrict__ state, const PrSchedule sched,
    const uint2* __restrict__ units, double* __restrict__ seg_partial,
    unsigned long long* __restrict__ row_partials) {
    if (state->done) return;
    // Loop invariants live in shared memory, so that the unrolled gather loop
    // keeps its loads in flight within the register budget of two CTAs per
    // SM; the fixed-point sums stay in registers per lane until the end.
    constexpr int kWarps = kPrThreads / 32;
    __shared__ double s_mass[2];                     // dangling mass, its uniform share
    __shared__ unsigned long long s_sum[2 * kWarps];  // per warp: L1 change, dangling mass of r'
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_mass[0] = state->dangling;
        s_mass[1] = state->dangling / static_cast<double>(V);
    }
    if (threadIdx.x < 2 * kWarps) s_sum[threadIdx.x] = 0;
    extern __shared__ float s_hub[];  // kHubEntries floats (dynamic shared memory)
    if (kHubEntries > 0) {
        const uint32_t hub = V < kHubEntries ? V : kHubEntries;
        for (uint32_t i = threadIdx.x; i < hub; i += blockDim.x) s_hub[i] = __ldg(contrib_in + i);
    }
    __syncthreads();
    const uint32_t total_warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t first_unit = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long my_diff = 0, my_dangle = 0;
    {
        // The row bounds of the next group-phase unit are loaded while this
        // unit is worked on: a unit's loads form a chain (row offsets, then
        // targets, then gathers), and most lanes finish a unit in one trip,
        // so the offsets' latency would otherwise be paid in full each time.
        uint32_t b = first_unit;
        uint32_t pi = 0, rs[kRowsPerGroup] = {}, re[kRowsPerGroup] = {};
        if (b < sched.total_blocks) {
            pi = unit_phase(sched, b);
            if (sched.phase[pi].kind == kPhaseGroup) unit_rows(sched.phase[pi], b, lane, poff, rs, re);
        }
        while (b < sched.total_blocks) {
            const uint32_t nb = b + total_warps;
            uint32_t npi = 0, nrs[kRowsPerGroup] = {}, nre[kRowsPerGroup] = {};
            if (kPrefetchRows && nb < sched.total_blocks) {
                npi = unit_phase(sched, nb);
                if (sched.phase[npi].kind == kPhaseGroup) unit_rows(sched.phase[npi], nb, lane, poff, nrs, nre);
            }
            const PrPhase ph = sched.phase[pi];
            if (ph.kind == kPhaseLong) {
                // One segment of a long row: 32 entries per lane, 8 loads in flight.
                const uint2 unit = units[b - ph.first_block];
                const uint32_t row_start = poff[unit.x], row_end = poff[unit.x + 1];
                const uint32_t s0 = row_start + unit.y * kSegment;
                const uint32_t s1 = min(s0 + kSegment, row_end);
                float acc = 0.f, comp = 0.f;
                uint32_t j = s0 + lane;
                for (; j + 7 * 32 < s1; j += 8 * 32) {
                    uint32_t t[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) t[q] = ld_stream(ptgt + j + q * 32);
                    float c[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) c[q] = gather_contrib(s_hub, contrib_in, t[q]);
#pragma unroll
                    for (int q = 0; q < 8; ++q) kahan_add(acc, comp, c[q]);
                }
                for (; j < s1; j += 32) kahan_add(acc, comp, gather_contrib(s_hub, contrib_in, ld_stream(ptgt + j)));
                const double part = warp_sum(static_cast<double>(acc) - static_cast<double>(comp));
                if (lane == 0) seg_partial[b - ph.first_block] = part;
            } else if (ph.kind == kPhaseGroup) {
                // Rows of one class, 2^log2g lanes per row, kRowsPerGroup rows per
                // group worked on in lockstep: each step issues one target load and
                // one gather per row (kRowsPerGroup * kUnroll in flight per lane),
                // so no row waits on the previous one's memory round trips.
                const uint32_t log2g = ph.log2g, g = 1u << log2g;
                const uint32_t groups = 32u >> log2g;
                const uint32_t group = lane >> log2g, lig = lane & (g - 1);
                const uint32_t first = ph.row_begin + (b - ph.first_block) * groups * kRowsPerGroup;
                uint32_t longest = 0;
#pragma unroll
                for (int q = 0; q < kRowsPerGroup; ++q) longest = max(longest, re[q] - rs[q]);
                float acc[kRowsPerGroup], comp[kRowsPerGroup];
#pragma unroll
                for (int q = 0; q < kRowsPerGroup; ++q) {
                    acc[q] = 0.f;
                    comp[q] = 0.f;
                }
                for (uint32_t off = lig; off < longest; off += kUnroll * g) {
                    uint32_t t[kUnroll][kRowsPerGroup];
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
                        for (int q = 0; q < kRowsPerGroup; ++q) {
                            const uint32_t j = rs[q] + off + u * g;
                            t[u][q] = j < re[q] ? ld_stream(ptgt + j) : 0xFFFFFFFFu;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
                        for (int q = 0; q < kRowsPerGroup; ++q) {
                            if (t[u][q] != 0xFFFFFFFFu) kahan_add(acc[q], comp[q], gather_contrib(s_hub, contrib_in, t[u][q]));
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kRowsPerGroup; ++q) {
                    const uint32_t row = first + q * groups + group;
                    const double v = group_sum(static_cast<double>(acc[q]) - static_cast<double>(comp[q]), log2g);
                    if (lig == 0 && row < ph.row_end) {
                        double d = 0.0, dg = 0.0;
                        pr_finish_row(row, v, re[q] - rs[q], rank_in, rank_out, contrib_out, outdeg, tele, base,
                                      damp, s_mass[1], s_mass[0], d, dg);
                        my_diff += to_fixed(d);
                        my_dangle += to_fixed(dg);
                    }
                }
            } else {
                // Rows without entries: the teleport and dangling share only.
                const uint32_t row = ph.row_begin + (b - ph.first_block) * 32 + lane;
                if (row < ph.row_end) {
                    double d = 0.0, dg = 0.0;
                    pr_finish_row(row, 0.0, 0, rank_in, rank_out, contrib_out, outdeg, tele, base, damp, s_mass[1],
                                  s_mass[0], d, dg);
                    my_diff += to_fixed(d);
                    my_dangle += to_fixed(dg);
                }
            }
            if (!kPrefetchRows && nb < sched.total_blocks) {
                npi = unit_phase(sched, nb);
                if (sched.phase[npi].kind == kPhaseGroup) unit_rows(sched.phase[npi], nb, lane, poff, nrs, nre);
            }
            b = nb;
            pi = npi;
#pragma unroll
            for (int q = 0; q < kRowsPerGroup; ++q) {
                rs[q] = nrs[q];
                re[q] = nre[q];
            }
        }
    }
    my_diff = warp_sum(my_diff);
    my_dangle = warp_sum(my_dangle);
    if (lane == 0) {
        s_sum[2 * warp] = my_diff;
        s_sum[2 * warp + 1] = my_dangle;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long diff = 0, dangle = 0;
        for (int w = 0; w < kWarps; ++w) {
            diff += s_sum[2 * w];
            dangle += s_sum[2 * w + 1];
        }
        row_partials[2 * blockIdx.x] = diff;
        row_partials[2 * blockIdx.x + 1] = dangle;
    }
}

// One warp per chunk of kChunk entries (chunks dealt round-robin to the warps
// of a persistent grid), 8 consecutive entries per lane. Row sums are FP64
// (the contributions are FP32). A run of equal rows inside a lane that is
// neither its first nor its last is a whole row; the first and last runs are
// joined across lanes by a segmented scan, and the lane where a run ends
// finishes its row, except for the parts of rows that cross chunks:
// chunk_part[2c] takes the part of chunk c's first row when that row began
// in an earlier chunk, chunk_part[2c + 1] the part of its last row when that
// row goes on into the next chunk (the whole chunk when one row covers it).
__global__ void __launch_bounds__(kChunkThreads, kChunkCtasPerSm) pr_chunks_kernel(
    const uint32_t* __restrict__ poff, const uint32_t* __restrict__ ptgt, const uint8_t* __restrict__ delta,
    const uint32_t* __restrict__ chunk_row, uint32_t origin, uint32_t lo, uint32_t hi, uint32_t n_chunks,
    const float* __restrict__ rank_in, const float* __restrict__ contrib_in, float* __restrict__ rank_out,
    float* __restrict__ contrib_out, const uint32_t* __restrict__ outdeg, const float* __restrict__ tele, uint32_t V,
    double base, double damp, const PrState* __restrict__ state, double* __restrict__ chunk_part,
    unsigned long long* __restrict__ partials) {
    if (state->done) return;
    constexpr int kWarps = kChunkThreads / 32;
    __shared__ double s_mass[2];
    __shared__ unsigned long long s_sum[2 * kWarps];
    if (threadIdx.x == 0) {
        s_mass[0] = state->dangling;
        s_mass[1] = state->dangling / static_cast<double>(V);
    }
    __syncthreads();
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t total_warps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long my_diff = 0, my_dangle = 0;
    auto finish = [&](uint32_t r, double sum) {
        double d = 0.0, dg = 0.0;
        pr_finish_row(r, sum, poff[r + 1] - poff[r], rank_in, rank_out, contrib_out, outdeg, tele, base, damp,
                      s_mass[1], s_mass[0], d, dg);
        my_diff += to_fixed(d);
        my_dangle += to_fixed(dg);
    };
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_chunks; c += total_warps) {
        const uint32_t e0 = origin + c * kChunk;   // chunk start; entries [e0, e0 + kChunk)
        const uint32_t eb = e0 + 8 * lane;         // this lane's first entry (32-byte aligned)
        const uint32_t rbase = __ldg(chunk_row + c);
        const uint4 ta = ld_stream4(reinterpret_cast<const uint4*>(ptgt + eb));
        const uint4 tb = ld_stream4(reinterpret_cast<const uint4*>(ptgt + eb + 4));
        const uint2 dl = ld_stream2(reinterpret_cast<const uint2*>(delta + (eb - origin)));
        const bool first_split = __ldg(poff + rbase) < e0;  // the first row began in an earlier chunk
        const uint32_t t[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
        uint32_t row[8];
        float val[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t e = eb + i;
            const bool ok = e >= lo && e < hi;
            row[i] = ok ? rbase + (((i < 4 ? dl.x : dl.y) >> (8 * (i & 3))) & 0xFFu) : kNoRow;
            val[i] = ok ? __ldg(contrib_in + t[i]) : 0.f;
        }
        const uint32_t rlast = __shfl_sync(kFullMask, row[7], 31);
        // Only the last chunk has slots past `hi`, and its last row ends inside it.
        const bool last_split = rlast != kNoRow && __ldg(poff + rlast + 1) > e0 + kChunk;
        double head = 0.0, acc = 0.0;
        bool multi = false;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            acc += static_cast<double>(val[i]);
            if (i < 7 && row[i + 1] != row[i]) {
                if (!multi) {
                    head = acc;
                    multi = true;
                } else {
                    finish(row[i], acc);  // a whole row inside this lane (never kNoRow: those runs lead or trail)
                }
                acc = 0.0;
            }
        }
        // Segmented inclusive scan of the lanes' last runs: a lane continues the
        // run of the lane before when it holds one row only and that row is the
        // previous lane's last.
        const uint32_t rf = row[0], rl = row[7];
        const uint32_t prev_last = __shfl_up_sync(kFullMask, rl, 1);
        const uint32_t next_first = __shfl_down_sync(kFullMask, rf, 1);
        const bool carry_in = lane > 0 && prev_last == rf;
        bool head_flag = multi || !carry_in;
        double S = acc;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double su = __shfl_up_sync(kFullMask, S, d);
            const bool fu = __shfl_up_sync(kFullMask, head_flag, d);
            if (lane >= static_cast<unsigned>(d)) {
                if (!head_flag) S += su;
                head_flag = head_flag || fu;
            }
        }
        const double carry = __shfl_up_sync(kFullMask, S, 1);
        if (multi && rf != kNoRow) {  // the first run ends in this lane
            const double total = head + (carry_in ? carry : 0.0);
            if (rf == rbase && first_split) chunk_part[2 * static_cast<uint64_t>(c)] = total;
            else finish(rf, total);
        }
        const bool continues = lane < 31 && next_first == rl;
        if (!continues && rl != kNoRow) {  // the last run ends at this lane's end
            if (lane == 31 && last_split) chunk_part[2 * static_cast<uint64_t>(c) + 1] = S;
            else if (rl == rbase && first_split) chunk_part[2 * static_cast<uint64_t>(c)] = S;
            else finish(rl, S);
        }
    }
    my_diff = warp_sum(my_diff);
    my_dangle = warp_sum(my_dangle);
    if (lane == 0) {
        s_sum[2 * warp] = my_diff;
        s_sum[2 * warp + 1] = my_dangle;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long diff = 0, dangle = 0;
        for (int w = 0; w < kWarps; ++w) {
            diff += s_sum[2 * w];
            dangle += s_sum[2 * w + 1];
        }
        partials[2 * blockIdx.x] = diff;
        partials[2 * blockIdx.x + 1] = dangle;
    }
}

// Finishes the long rows from their segment partials (in segment order) and
// the chunked rows that cross chunks from their chunk parts (in chunk order),
// and folds a fixed slice of kFinSlice row-kernel block partials per block; then
// the last block reduces the per-block results in a fixed order and advances
// the state.
constexpr uint32_t kFinSlice = 2048;

__global__ void __launch_bounds__(256) pr_finish_kernel(
    const uint32_t* __restrict__ poff, uint32_t long_rows, const uint32_t* __restrict__ unit_begin,
    const double* __restrict__ seg_partial, const uint4* __restrict__ split_rows, uint32_t n_split,
    const double* __restrict__ chunk_part, const float* __restrict__ rank_in, float* __restrict__ rank_out,
    float* __restrict__ contrib_out, const uint32_t* __restrict__ outdeg, const float* __restrict__ tele, uint32_t V,
    double base, double damp, PrState* __restrict__ state,
    double tolerance, const unsigned long long* __restrict__ row_partials, uint32_t row_blocks,
    unsigned long long* __restrict__ fin_partials) {
    if (state->done) return;
    __shared__ unsigned long long scratch[32];
    __shared__ bool s_last;
    const double dangling = state->dangling;
    const double spread = dangling / static_cast<double>(V);
    unsigned long long d = 0, g = 0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < long_rows) {
        double sum = 0.0, rd = 0.0, rg = 0.0;
        for (uint32_t u = unit_begin[i]; u < unit_begin[i + 1]; ++u) sum += seg_partial[u];
        pr_finish_row(i, sum, poff[i + 1] - poff[i], rank_in, rank_out, contrib_out, outdeg, tele, base, damp,
                      spread, dangling, rd, rg);
        d = to_fixed(rd);
        g = to_fixed(rg);
    } else if (i - long_rows < n_split) {
        // A chunked row that crosses chunks: its part in its first chunk (that
        // chunk's last row), every chunk it covers whole, its part in its last.
        const uint4 sr = split_rows[i - long_rows];
        double sum = chunk_part[2 * static_cast<uint64_t>(sr.y) + 1], rd = 0.0, rg = 0.0;
        for (uint32_t c = sr.y + 1; c < sr.z; ++c) sum += chunk_part[2 * static_cast<uint64_t>(c) + 1];
        sum += chunk_part[2 * static_cast<uint64_t>(sr.z)];
        pr_finish_row(sr.x, sum, poff[sr.x + 1] - poff[sr.x], rank_in, rank_out, contrib_out, outdeg, tele, base,
                      damp, spread, dangling, rd, rg);
        d = to_fixed(rd);
        g = to_fixed(rg);
    }
    const uint64_t slice_end = std::min<uint64_t>(static_cast<uint64_t>(blockIdx.x + 1) * kFinSlice, row_blocks);
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * kFinSlice + threadIdx.x; k < slice_end; k += blockDim.x) {
        d += row_partials[2 * k];
        g += row_partials[2 * k + 1];
    }
    d = block_sum(d, scratch);
    g = block_sum(g, scratch);
    if (threadIdx.x == 0) {
        fin_partials[2 * blockIdx.x] = d;
        fin_partials[2 * blockIdx.x + 1] = g;
        __threadfence();
        const unsigned ticket = atomicAdd(&state->ticket, 1u);
        s_last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    unsigned long long dd = 0, gg = 0;
    for (uint32_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        dd += __ldcg(fin_partials + 2 * k);
        gg += __ldcg(fin_partials + 2 * k + 1);
    }
    dd = block_sum(dd, scratch);
    gg = block_sum(gg, scratch);
    if (threadIdx.x == 0) {
        const double diff = from_fixed(dd);
        state->iterations += 1;
        state->last_diff = diff;
        state->dangling = from_fixed(gg);
        if (diff < tolerance) state->done = 1;
        state->ticket = 0;
    }
}

// ---------------------------------------------------------------- host

// Builds the relabelled pull CSR and the schedule for pulling over
// (pull_offsets, pull_targets); `out_offsets`, when given, is the CSR whose
// list lengths are the out-degrees (the graph itself when pulling over its
// transpose).
static Error build_plan(GraphImpl& g, const uint32_t* pull_offsets, const uint32_t* pull_targets,
                        const uint32_t* out_offsets, PageRankPlan** out) {
    DeviceImpl& dev = *g.dev;
    auto plan = std::unique_ptr<PageRankPlan, void (*)(PageRankPlan*)>(new PageRankPlan, destroy_pagerank_plan);
    PageRankPlan& p = *plan;
    const uint32_t V = g.num_nodes, E = g.num_edges;
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned vgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), cap));

    // 1. Stable partition of the vertices by degree class, highest first.
    const uint32_t nblk = static_cast<uint32_t>(ceil_div_u64(V, kClassBlock));
    const uint64_t ncount = static_cast<uint64_t>(kDegClasses) * nblk;
    DeviceBuffer<uint32_t> counts, cpos, starts;
    GCU_TRY(counts.allocate(dev, ncount));
    GCU_TRY(cpos.allocate(dev, ncount + 1));
    GCU_TRY(starts.allocate(dev, kDegClasses + 2));
    GCU_TRY(p.perm.allocate(dev, V));
    GCU_TRY(p.inv.allocate(dev, V));
    GCU_LAUNCH(dev, "pr_class_count", pr_class_count_kernel, nblk, kClassBlock, 0, pull_offsets, V, nblk,
               counts.ptr);
    GCU_TRY(exclusive_scan_u32(dev, counts.ptr, cpos.ptr, ncount));
    GCU_LAUNCH(dev, "pr_class_scatter", pr_class_scatter_kernel, nblk, kClassBlock, 0, pull_offsets, V, nblk,
               cpos.ptr, p.perm.ptr, p.inv.ptr);
    GCU_CUDA(cudaMemsetAsync(starts.ptr + kDegClasses + 1, 0, sizeof(uint32_t), dev.stream), "memset");
    GCU_LAUNCH(dev, "pr_class_starts", pr_class_starts_kernel, 1, 64, 0, cpos.ptr, nblk, starts.ptr);

    uint32_t cls[kDegClasses + 2];
    GCU_CUDA(cudaMemcpyAsync(cls, starts.ptr, sizeof(cls), cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_TRY(dev.sync());
    // Rows of class c (new ids) are [begin[c], end[c]); classes are laid out
    // from K-1 down to 0, so class c ends where class c-1 begins.
    std::vector<uint32_t> begin(kDegClasses), end(kDegClasses);
    for (int c = 0; c < kDegClasses; ++c) {
        begin[c] = cls[c];
        end[c] = c == 0 ? V : cls[c - 1];
    }
    p.long_rows = begin[kLongClass - 1];  // classes >= kLongClass occupy [0, begin[kLongClass - 1])
    p.empty_rows = end[0] - begin[0];

    // 2. Relabelled CSR (and out-degrees when they differ from the row lengths).
    GCU_TRY(p.poff.allocate(dev, static_cast<uint64_t>(V) + 1));
    GCU_LAUNCH(dev, "pr_perm_degree", pr_perm_degree_kernel, vgrid, 256, 0, pull_offsets, p.perm.ptr, V, p.poff.ptr);
    GCU_TRY(exclusive_scan_u32(dev, p.poff.ptr, p.poff.ptr, V));
    // Chunked rows: [long_rows, begin[0]), entries [chunk_lo, chunk_hi). The
    // chunk kernel indexes entries in 32 bits up to kChunk past E, so graphs
    // within 2 kChunk of 2^32 entries keep the lane-group form.
    const uint32_t short_rows = begin[0] - p.long_rows;
    if (kChunkRows && short_rows > 0 && E <= 0xFFFFFFFFu - 2 * kChunk) {
        uint32_t bounds[2];
        GCU_CUDA(cudaMemcpyAsync(&bounds[0], p.poff.ptr + p.long_rows, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_CUDA(cudaMemcpyAsync(&bounds[1], p.poff.ptr + begin[0], sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        p.chunk_lo = bounds[0];
        p.chunk_hi = bounds[1];
        p.chunk_origin = p.chunk_lo & ~7u;  // 32-byte aligned target loads
        p.n_chunks = static_cast<uint32_t>(ceil_div_u64(p.chunk_hi - p.chunk_origin, kChunk));
        GCU_TRY(p.chunk_row.allocate(dev, p.n_chunks));
        GCU_TRY(p.chunk_delta.allocate(dev, static_cast<uint64_t>(p.n_chunks) * kChunk));
        GCU_TRY(p.chunk_part.allocate(dev, 2 * static_cast<uint64_t>(p.n_chunks)));
        GCU_CUDA(cudaMemsetAsync(p.chunk_delta.ptr, 0, static_cast<size_t>(p.n_chunks) * kChunk, dev.stream),
                 "memset");
        DeviceBuffer<uint32_t> split_pos;
        GCU_TRY(split_pos.allocate(dev, static_cast<uint64_t>(short_rows) + 1));
        const unsigned sgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(short_rows, 256), cap));
        GCU_LAUNCH(dev, "pr_chunk_rows", pr_chunk_rows_kernel, sgrid, 256, 0, p.poff.ptr, p.long_rows, begin[0],
                   p.chunk_origin, p.chunk_row.ptr, split_pos.ptr);
        GCU_TRY(exclusive_scan_u32(dev, split_pos.ptr, split_pos.ptr, short_rows));
        GCU_CUDA(cudaMemcpyAsync(&p.n_split, split_pos.ptr + short_rows, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        GCU_TRY(p.split_rows.allocate(dev, std::max<uint32_t>(p.n_split, 1)));
        GCU_LAUNCH(dev, "pr_split_rows", pr_split_rows_kernel, sgrid, 256, 0, p.poff.ptr, p.long_rows, short_rows,
                   p.chunk_origin, split_pos.ptr, p.split_rows.ptr);
    }
    // The last chunk's loads run up to kChunk entries past E: padding of valid ids.
    const uint64_t tgt_pad = p.n_chunks ? kChunk : 0;
    GCU_TRY(p.ptgt.allocate(dev, static_cast<uint64_t>(E) + tgt_pad));
    if (tgt_pad) GCU_CUDA(cudaMemsetAsync(p.ptgt.ptr + E, 0, sizeof(uint32_t) * tgt_pad, dev.stream), "memset");
    if (E > 0) {
        const unsigned fill_grid =
            static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(E, kFillTile), cap)));
        GCU_LAUNCH(dev, "pr_perm_fill", pr_perm_fill_kernel, fill_grid, kFillThreads, 0, pull_offsets, pull_targets,
                   p.perm.ptr, p.inv.ptr, p.poff.ptr, V, E, p.ptgt.ptr, p.chunk_row.ptr, p.chunk_origin, p.chunk_lo,
                   p.chunk_hi, p.n_chunks ? p.chunk_delta.ptr : nullptr);
    }
    if (out_offsets) {
        GCU_TRY(p.outdeg.allocate(dev, V));
        GCU_LAUNCH(dev, "pr_outdeg", pr_outdeg_kernel, vgrid, 256, 0, out_offsets, p.perm.ptr, V, p.outdeg.ptr,
                   starts.ptr + kDegClasses + 1);
        uint32_t dangling = 0;
        GCU_CUDA(cudaMemcpyAsync(&dangling, starts.ptr + kDegClasses + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        p.dangling_rows = dangling;
    } else {
        p.dangling_rows = p.empty_rows;
    }

    // 3. Long-row segments, listed on the device: unit_begin[i] = the first
    // unit of long row i (a scan of the segment counts), units = (row, segment).
    GCU_TRY(p.unit_begin.allocate(dev, static_cast<uint64_t>(p.long_rows) + 1));
    uint32_t n_units = 0;
    if (p.long_rows > 0) {
        const unsigned lgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(p.long_rows, 256), cap));
        GCU_LAUNCH(dev, "pr_unit_count", pr_unit_count_kernel, lgrid, 256, 0, p.poff.ptr, p.long_rows,
                   p.unit_begin.ptr);
        GCU_TRY(exclusive_scan_u32(dev, p.unit_begin.ptr, p.unit_begin.ptr, p.long_rows));
        GCU_CUDA(cudaMemcpyAsync(&n_units, p.unit_begin.ptr + p.long_rows, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
    } else {
        GCU_CUDA(cudaMemsetAsync(p.unit_begin.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
    }
    GCU_TRY(p.units.allocate(dev, std::max<uint32_t>(n_units, 1)));
    GCU_TRY(p.seg_partial.allocate(dev, std::max<uint32_t>(n_units, 1)));
    if (n_units > 0) {
        const unsigned lgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(p.long_rows, 256), cap));
        GCU_LAUNCH(dev, "pr_unit_fill", pr_unit_fill_kernel, lgrid, 256, 0, p.poff.ptr, p.long_rows,
                   p.unit_begin.ptr, p.units.ptr);
    }

    // 4. Block schedule: long segments, then (unless chunked) classes
    // kLongClass-1 .. 1, then empty rows.
    PrSchedule& s = p.sched;
    s.nphases = 0;
    uint32_t blocks = 0;
    auto add = [&](uint32_t kind, uint32_t rb, uint32_t re, uint32_t log2g, uint32_t rpg, uint32_t nb) {
        if (nb == 0) return;
        PrPhase& ph = s.phase[s.nphases++];
        ph.first_block = blocks;
        ph.row_begin = rb;
        ph.row_end = re;
        ph.kind = kind;
        ph.log2g = log2g;
        ph.rows_per_group = rpg;
        blocks += nb;
    };
    add(kPhaseLong, 0, p.long_rows, 0, 0, n_units);
    for (int c = kLongClass - 1; c >= 1 && p.n_chunks == 0; --c) {
        // Class c (degrees [2^(c-1), 2^c)): 2^(c-1) lanes per row up to a warp.
        const uint32_t rows = end[c] - begin[c];
        const uint32_t log2g = std::min<uint32_t>(static_cast<uint32_t>(c - 1), 5);
        const uint32_t per_unit = (32u >> log2g) * kRowsPerGroup;  // one warp's rows
        add(kPhaseGroup, begin[c], end[c], log2g, kRowsPerGroup, static_cast<uint32_t>(ceil_div_u64(rows, per_unit)));
    }
    add(kPhaseEmpty, begin[0], end[0], 0, 0, static_cast<uint32_t>(ceil_div_u64(p.empty_rows, 32)));
    s.total_blocks = blocks;
    p.row_ctas = std::max<uint32_t>(
        1, std::min<uint32_t>(ceil_div_u64(blocks, kPrThreads / 32), static_cast<uint32_t>(dev.sm_count) * kRowCtasPerSm));

    if (kHubEntries * sizeof(float) > 48 * 1024)
        GCU_CUDA(cudaFuncSetAttribute(pr_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kHubEntries * sizeof(float))),
                 "cudaFuncSetAttribute");
    p.chunk_ctas = p.n_chunks == 0 ? 0
                                   : std::max<uint32_t>(1, std::min<uint32_t>(
                                                               ceil_div_u64(p.n_chunks, kChunkThreads / 32),
                                                               static_cast<uint32_t>(dev.sm_count) * kChunkCtasPerSm));
    p.fin_blocks = static_cast<uint32_t>(std::max<uint64_t>(
        {1, ceil_div_u64(static_cast<uint64_t>(p.long_rows) + p.n_split, 256),
         ceil_div_u64(static_cast<uint64_t>(p.row_ctas) + p.chunk_ctas, kFinSlice)}));

    GCU_TRY(p.ranks.allocate(dev, 2 * static_cast<uint64_t>(V)));
    GCU_TRY(p.contrib.allocate(dev, 2 * static_cast<uint64_t>(V)));
    GCU_TRY(p.ranks_out.allocate(dev, V));
    GCU_TRY(p.row_partials.allocate(dev, 2 * (static_cast<uint64_t>(p.row_ctas) + p.chunk_ctas)));
    GCU_TRY(p.fin_partials.allocate(dev, 2 * static_cast<uint64_t>(p.fin_blocks)));
    GCU_TRY(p.state.allocate(dev, 1));
    GCU_TRY(dev.sync());
    *out = plan.release();
    return ok();
}

static Error ensure_plan(GraphImpl& g, bool directed, PageRankPlan** plan) {
    PageRankPlan*& slot = directed ? g.pr_plan_directed : g.pr_plan;
    if (!slot) {
        if (directed) {
            // Pull over the in-lists (transpose); out-degrees from the lists.
            DeviceBuffer<uint32_t> t_offsets, t_targets;
            GCU_TRY(transpose_csr(*g.dev, g.offsets.ptr, g.targets.ptr, g.num_nodes, g.num_edges, &t_offsets,
                                  &t_targets));
            GCU_TRY(build_plan(g, t_offsets.ptr, t_targets.ptr, g.offsets.ptr, &slot));
        } else {
            GCU_TRY(build_plan(g, g.offsets.ptr, g.targets.ptr, nullptr, &slot));
        }
    }
    *plan = slot;
    return ok();
}

// Gather probe: the relabelled targets streamed coalesced and contrib[t]
// gathered, with nothing else (no row offsets, no row structure, no
// epilogue). Same grid, CTA shape and load pattern (8 targets, then 8
// gathers, in flight per lane) as the long-row segments of pr_rows, over the
// same plan, so its time per pass is the floor of a pull SpMV on this layout
// (the grid is the row kernel's full persistent grid, 2 CTAs per SM).
// Each warp folds its sums into one float atomic so that nothing is dropped.
__global__ void __launch_bounds__(kPrThreads, kRowCtasPerSm) pr_gather_probe_kernel(
    const uint32_t* __restrict__ ptgt, uint32_t E, const float* __restrict__ contrib, float* __restrict__ sink) {
    const uint32_t total_warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = lane_id();
    float acc = 0.f;
    for (uint64_t base = static_cast<uint64_t>(warp) * kSegment; base < E;
         base += static_cast<uint64_t>(total_warps) * kSegment) {
        const uint64_t end = min_u64(base + kSegment, E);
        uint64_t j = base + lane;
        for (; j + 7 * 32 < end; j += 8 * 32) {
            uint32_t t[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) t[q] = ld_stream(ptgt + j + q * 32);
            float c[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) c[q] = __ldg(contrib + t[q]);
#pragma unroll
            for (int q = 0; q < 8; ++q) acc += c[q];
        }
        for (; j < end; j += 32) acc += __ldg(contrib + ld_stream(ptgt + j));
    }
    acc = warp_sum(acc);
    if (lane == 0) atomicAdd(sink, acc);
}

Error pagerank_gather_probe(GraphImpl& g, bool directed, uint32_t passes, double* ms_per_pass) {
    *ms_per_pass = 0.0;
    const uint32_t V = g.num_nodes, E = g.num_edges;
    if (V == 0 || E == 0 || passes == 0) return ok();
    DeviceImpl& dev = *g.dev;
    PageRankPlan* plan = nullptr;
    GCU_TRY(ensure_plan(g, directed, &plan));
    PageRankPlan& p = *plan;
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned vgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), cap));
    GCU_LAUNCH(dev, "pr_init", pr_init_kernel, vgrid, 256, 0, p.poff.ptr, directed ? p.outdeg.ptr : nullptr, V,
               1.0f / static_cast<float>(V), p.ranks.ptr, p.contrib.ptr);
    const unsigned grid = static_cast<unsigned>(dev.sm_count) * kRowCtasPerSm;  // the row kernel's full grid
    DeviceBuffer<float> sink;
    GCU_TRY(sink.allocate(dev, 1));
    GCU_CUDA(cudaMemsetAsync(sink.ptr, 0, sizeof(float), dev.stream), "memset");
    cudaEvent_t ev[2] = {nullptr, nullptr};
    GCU_CUDA(cudaEventCreate(&ev[0]), "cudaEventCreate");
    cudaError_t c = cudaEventCreate(&ev[1]);
    Error err = ok();
    if (c != cudaSuccess) err = kernel_error(std::string("cudaEventCreate: ") + cudaGetErrorString(c));
    if (err.ok()) {
        err = [&]() -> Error {
            GCU_LAUNCH(dev, "pr_gather_probe", pr_gather_probe_kernel, grid, kPrThreads, 0, p.ptgt.ptr, E,
                       p.contrib.ptr, sink.ptr);  // warm-up
            GCU_CUDA(cudaEventRecord(ev[0], dev.stream), "cudaEventRecord");
            for (uint32_t i = 0; i < passes; ++i)
                GCU_LAUNCH(dev, "pr_gather_probe", pr_gather_probe_kernel, grid, kPrThreads, 0, p.ptgt.ptr, E,
                           p.contrib.ptr, sink.ptr);
            GCU_CUDA(cudaEventRecord(ev[1], dev.stream), "cudaEventRecord");
            GCU_CUDA(cudaEventSynchronize(ev[1]), "cudaEventSynchronize");
            float ms = 0.f;
            GCU_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]), "cudaEventElapsedTime");
            *ms_per_pass = static_cast<double>(ms) / passes;
            return ok();
        }();
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    GCU_TRY(err);
    return dev.sync();
}

Error pagerank_ex(GraphImpl& g, bool directed, const float* tele_host, float damping, uint32_t max_iterations,
                  float tolerance, float* host_ranks, uint32_t* iterations, bool* converged) {
    const uint32_t V = g.num_nodes;
    // pagerank.rs:56-63: no nodes, no ranks.
    if (V == 0) {
        *iterations = 0;
        *converged = true;
        return ok();
    }
    DeviceImpl& dev = *g.dev;
    PageRankPlan* plan = nullptr;
    GCU_TRY(ensure_plan(g, directed, &plan));
    PageRankPlan& p = *plan;
    float* ranks[2] = {p.ranks.ptr, p.ranks.ptr + V};
    float* contrib[2] = {p.contrib.ptr, p.contrib.ptr + V};
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned vgrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), cap));
    const uint32_t* outdeg = directed ? p.outdeg.ptr : nullptr;

    DeviceBuffer<float> tele_raw, tele;
    if (tele_host) {
        GCU_TRY(tele_raw.allocate(dev, V));
        GCU_TRY(tele.allocate(dev, V));
        GCU_CUDA(cudaMemcpyAsync(tele_raw.ptr, tele_host, sizeof(float) * V, cudaMemcpyHostToDevice, dev.stream),
                 "copy personalisation vector");
        GCU_LAUNCH(dev, "pr_permute_tele", pr_permute_tele_kernel, vgrid, 256, 0, tele_raw.ptr, p.perm.ptr, V,
                   tele.ptr);
    }
    const float* d_tele = tele_host ? tele.ptr : nullptr;

    const float r0 = 1.0f / static_cast<float>(V);  // pagerank.rs:83
    GCU_LAUNCH(dev, "pr_init", pr_init_kernel, vgrid, 256, 0, p.poff.ptr, outdeg, V, r0, ranks[0], contrib[0]);
    PrState init{};
    init.dangling = static_cast<double>(p.dangling_rows) * static_cast<double>(r0);
    init.last_diff = INFINITY;
    p.host_state = init;
    GCU_CUDA(cudaMemcpyAsync(p.state.ptr, &p.host_state, sizeof(PrState), cudaMemcpyHostToDevice, dev.stream), "copy");

    const double damp = static_cast<double>(damping);
    const double base = (1.0 - damp) / static_cast<double>(V);
    const double tol = static_cast<double>(tolerance);

    // Queue iterations in chunks; the device stops itself once converged, so
    // the host only polls the state between chunks.
    uint32_t launched = 0;
    uint32_t chunk = 4;
    cudaEvent_t polled = nullptr;
    GCU_CUDA(cudaEventCreateWithFlags(&polled, cudaEventDisableTiming), "cudaEventCreate");
    bool stop = false;
    Error err = ok();
    while (launched < max_iterations && !stop) {
        const uint32_t n = std::min(chunk, max_iterations - launched);
        for (uint32_t i = 0; i < n && err.ok(); ++i) {
            const uint32_t it = launched + i;
            const int in = it & 1, out = in ^ 1;
            err = [&]() -> Error {
                GCU_LAUNCH(dev, "pr_rows", pr_rows_kernel, p.row_ctas, kPrThreads, kHubEntries * sizeof(float),
                           p.poff.ptr, p.ptgt.ptr,
                           ranks[in], contrib[in], ranks[out], contrib[out], outdeg, d_tele, V, base, damp,
                           p.state.ptr, p.sched, p.units.ptr, p.seg_partial.ptr, p.row_partials.ptr);
                if (p.n_chunks > 0)
                    GCU_LAUNCH(dev, "pr_chunks", pr_chunks_kernel, p.chunk_ctas, kChunkThreads, 0, p.poff.ptr,
                               p.ptgt.ptr, p.chunk_delta.ptr, p.chunk_row.ptr, p.chunk_origin, p.chunk_lo,
                               p.chunk_hi, p.n_chunks, ranks[in], contrib[in], ranks[out], contrib[out], outdeg,
                               d_tele, V, base, damp, p.state.ptr, p.chunk_part.ptr,
                               p.row_partials.ptr + 2 * static_cast<uint64_t>(p.row_ctas));
                GCU_LAUNCH(dev, "pr_finish", pr_finish_kernel, p.fin_blocks, 256, 0, p.poff.ptr, p.long_rows,
                           p.unit_begin.ptr, p.seg_partial.ptr, p.split_rows.ptr, p.n_split, p.chunk_part.ptr,
                           ranks[in], ranks[out], contrib[out], outdeg, d_tele, V, base, damp, p.state.ptr, tol,
                           p.row_partials.ptr, p.row_ctas + p.chunk_ctas, p.fin_partials.ptr);
                return ok();
            }();
        }
        if (!err.ok()) break;
        launched += n;
        cudaError_t c = cudaMemcpyAsync(&p.host_state, p.state.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, dev.stream);
        if (c == cudaSuccess) c = cudaEventRecord(polled, dev.stream);
        if (c == cudaSuccess) c = cudaEventSynchronize(polled);
        if (c != cudaSuccess) {
            err = kernel_error(std::string("PageRank iteration failed: ") + cudaGetErrorString(c));
            break;
        }
        stop = p.host_state.done != 0;
        chunk = std::min<uint32_t>(chunk * 2, 64);
    }
    cudaEventDestroy(polled);
    GCU_TRY(err);
    GCU_TRY(dev.sync());
    if (launched == 0) p.host_state = init;
    const uint32_t iters = p.host_state.iterations;
    GCU_LAUNCH(dev, "pr_unpermute", pr_unpermute_kernel, vgrid, 256, 0, ranks[iters & 1], p.inv.ptr, V,
               p.ranks_out.ptr);
    if (host_ranks) GCU_TRY(copy_to_host(dev, host_ranks, p.ranks_out.ptr, sizeof(float) * V));
    GCU_TRY(dev.sync());
    *iterations = iters;
    *converged = p.host_state.done != 0;
    return ok();
}

Error pagerank(GraphImpl& g, float damping, uint32_t max_iterations, float tolerance, float* host_ranks,
               uint32_t* iterations, bool* converged) {
    return pagerank_ex(g, false, nullptr, damping, max_iterations, tolerance, host_ranks, iterations, converged);
}

}  // namespace gcu
