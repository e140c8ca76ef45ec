// Stable LSD radix sort of 64-bit keys, and the CSR transpose built on it.
//
// Each pass sorts by one 8-bit digit: digit histograms per CTA range of
// kCtaKeys keys (digit-major, so one exclusive scan gives every (digit, CTA)
// its output base), then a stable scatter in which each CTA walks its range
// tile by tile (kSortTile keys): it ranks the tile's keys by digit inside each
// warp, stages them in shared memory in digit order and writes them out as
// contiguous runs, carrying every digit's output base on to its next tile.
// Stability makes the sort of (target << 32 | source) keys by their high word
// keep every in-list ordered by source, so the transpose is deterministic.
//
// Scatter forms, 3-pass transpose of R-MAT 24's directed copy (505 M keys) on
// one B200, ms of scatter per transpose (same output in every form):
//   each key written to its own address (radix_scatter_kernel)     23.0
//   staged in shared memory, warp ranks by match.any               18.2
//   ... ranks from 8 ballots per key (kMatchBallots)                15.0
//   ... 8 tiles per CTA instead of 1 (kTilesPerCta)                 13.2
//   ... ranks kept from the counting pass (kCacheRanks), 8 keys
//       per lane, 16 tiles per CTA, 4 CTAs per SM                   11.7
//   ... keys in shared memory, next tile loaded over the write-out
//       (kKeysInSmem, kPrefetchNextTile; shipped)                   11.4
// ncu of one pass at R-MAT 22 (126 M keys): with the ranks computed twice the
// integer ALU pipe was 88 % busy (the ballots' bit tests, 5.9 warp
// instructions per key) and DRAM 22 %; in the shipped form the ALU pipe is at
// 66 % and the shared-memory data pipe at 79 %, half of its wavefronts bank
// conflicts of the digit-ordered stores and per-digit counter updates.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;  // keys per tile
constexpr int kRadix = 256;
// Consecutive tiles per CTA of the staged scatter: the digit histograms, and
// so the output bases, are per CTA range (kCtaKeys keys) rather than per tile,
// and the CTA carries each digit's running base from one tile to the next.
// One 4,096-key tile per CTA made the digit-major histogram 256 counters per
// 4,096 keys (126 MB per pass at 505 M keys, every counter in its own cache
// line, written by the histogram, scanned, and read back by the scatter).
constexpr int kTilesPerCta = 16;
constexpr int kCtaKeys = kSortTile * kTilesPerCta;

// Digit counts of every CTA range (digit-major: hist[d * nctas + cta]).
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                                                  uint32_t shift, uint32_t nctas,
                                                                  uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kCtaKeys;
    for (int r = 0; r < kSortRounds * kTilesPerCta; ++r) {
        const uint64_t i = base + static_cast<uint64_t>(r) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    hist[static_cast<uint64_t>(threadIdx.x) * nctas + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint64_t* __restrict__ in,
                                                                     uint64_t* __restrict__ out, uint64_t n,
                                                                     uint32_t shift, uint32_t ntiles,
                                                                     const uint32_t* __restrict__ bases) {
    __shared__ uint32_t s_base[kRadix];
    __shared__ uint32_t s_run[kRadix];
    __shared__ uint32_t s_wcount[kSortThreads / 32][kRadix];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    s_base[threadIdx.x] = bases[static_cast<uint64_t>(threadIdx.x) * ntiles + blockIdx.x];
    s_run[threadIdx.x] = 0;
    for (int w = 0; w < kSortThreads / 32; ++w) s_wcount[w][threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t i = base + static_cast<uint64_t>(r) * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint64_t key = valid ? in[i] : 0;
        const uint32_t d = valid ? static_cast<uint32_t>((key >> shift) & 0xFF) : kRadix;  // kRadix: no key
        const unsigned same = __match_any_sync(kFullMask, d);
        const uint32_t rank = __popc(same & ((1u << lane) - 1));
        if (valid && lane == static_cast<unsigned>(__ffs(same) - 1)) s_wcount[warp][d] = __popc(same);
        __syncthreads();
        if (valid) {
            uint32_t before = 0;
            for (unsigned w = 0; w < warp; ++w) before += s_wcount[w][d];
            out[s_base[d] + s_run[d] + before + rank] = key;
        }
        __syncthreads();
        uint32_t round_total = 0;
        for (int w = 0; w < kSortThreads / 32; ++w) {
            round_total += s_wcount[w][threadIdx.x];
            s_wcount[w][threadIdx.x] = 0;
        }
        s_run[threadIdx.x] += round_total;
        __syncthreads();
    }
}

// The stable scatter with the tile staged in shared memory. Each warp owns a
// contiguous slice of kSliceKeys keys (kKeysPerLane per lane, loaded
// coalesced). Pass 1 counts the slice's digits with warp-level equal-digit
// masks; one barrier later every digit has its start inside the tile and
// every warp its offset inside each digit; pass 2 places the keys in shared
// memory in digit order (index order inside a digit: stable); the block then
// writes the tile out run by run, consecutive threads to consecutive
// addresses of a digit's output range.
constexpr bool kStagedScatter = true;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSliceKeys = kSortTile / kSortWarps;
constexpr int kKeysPerLane = kSliceKeys / 32;
static_assert(kSortThreads == kRadix, "one thread per digit in the block scans");
static_assert(kSliceKeys % 32 == 0, "whole warp rounds per slice");
static_assert(kStagedScatter || kTilesPerCta == 1, "the first scatter form takes one tile per CTA");

// Lanes of the warp holding the same digit (kRadix: a lane with no key), from
// one ballot per digit bit (kMatchBallots) or one match instruction (12.1
// against 11.4 ms in the shipped form, where it runs once per key).
constexpr bool kMatchBallots = true;
__device__ __forceinline__ unsigned same_digit_lanes(uint32_t d) {
    if (!kMatchBallots) return __match_any_sync(kFullMask, d);
    unsigned m = __ballot_sync(kFullMask, d == kRadix) ^ (d == kRadix ? 0u : kFullMask);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const unsigned bits = __ballot_sync(kFullMask, (d >> b) & 1u);
        m &= ((d >> b) & 1u) ? bits : ~bits;
    }
    return m;
}

constexpr int kScatterMinCtas = 4;  // __launch_bounds__ minimum CTAs per SM of the staged scatter
// Register form (kKeysInSmem off): with kCacheRanks the second pass over a
// tile's keys reuses each key's rank, digit count and first-lane flag from the
// first (packed in registers) instead of redoing the 8 ballots per key.
constexpr bool kCacheRanks = true;
static_assert(!kCacheRanks || kKeysPerLane % 2 == 0, "two keys' rank words per register");

__global__ void __launch_bounds__(kSortThreads, kScatterMinCtas) radix_scatter_staged_kernel(
    const uint64_t* __restrict__ in, uint64_t* __restrict__ out, uint64_t n, uint32_t shift, uint32_t nctas,
    const uint32_t* __restrict__ bases) {
    __shared__ uint64_t s_keys[kSortTile];
    __shared__ uint32_t s_woff[kSortWarps][kRadix];  // per warp: digit counts, then running offsets
    __shared__ uint32_t s_start[kRadix];             // digit start inside the tile
    __shared__ uint32_t s_base[kRadix];              // digit's output base for the current tile
    __shared__ uint32_t s_wtot[kSortWarps];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1;
    s_base[threadIdx.x] = bases[static_cast<uint64_t>(threadIdx.x) * nctas + blockIdx.x];
    for (int t = 0; t < kTilesPerCta; ++t) {
        const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kCtaKeys + static_cast<uint64_t>(t) * kSortTile;
        if (tile0 >= n) break;  // the same for every thread of the block
        for (int w = 0; w < kSortWarps; ++w) s_woff[w][threadIdx.x] = 0;
        const uint64_t slice = tile0 + static_cast<uint64_t>(warp) * kSliceKeys;
        uint64_t key[kKeysPerLane];
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint64_t i = slice + static_cast<uint64_t>(q) * 32 + lane;
            key[q] = i < n ? in[i] : 0;
        }
        // Digit of key q (kRadix: past the end of the input).
        auto digit = [&](int q) -> uint32_t {
            return slice + static_cast<uint64_t>(q) * 32 + lane < n ? static_cast<uint32_t>((key[q] >> shift) & 0xFF)
                                                                     : static_cast<uint32_t>(kRadix);
        };
        // Per key, with kCacheRanks: its rank among the warp's lanes of the
        // same digit (bits 0-4), that digit's lane count (bits 5-10) and
        // whether this lane is the digit's first (bit 11), two keys per word.
        uint32_t info[kCacheRanks ? kKeysPerLane / 2 : 1];
        __syncthreads();  // counters cleared; the previous tile's base update visible
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint32_t d = digit(q);
            const unsigned same = same_digit_lanes(d);
            const bool first = d < kRadix && lane == static_cast<unsigned>(__ffs(same) - 1);
            if (first) s_woff[warp][d] += __popc(same);
            if (kCacheRanks) {
                const uint32_t v = __popc(same & below) | (__popc(same) << 5) | (first ? 1u << 11 : 0u);
                if (q & 1) info[q / 2] |= v << 16;
                else info[q / 2] = v;
            }
            __syncwarp();
        }
        __syncthreads();
        // Thread d: the warps' exclusive offsets inside digit d, then the
        // digits' exclusive starts inside the tile (block-wide scan); `tot`
        // (the tile's count of digit d) advances the digit's base afterwards.
        uint32_t tot = 0;
        {
            const uint32_t d = threadIdx.x;
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t c = s_woff[w][d];
                s_woff[w][d] = tot;
                tot += c;
            }
            const uint32_t inc = warp_inclusive_scan(tot);
            if (lane == 31) s_wtot[warp] = inc;
            __syncthreads();
            uint32_t before = 0;
            for (unsigned w = 0; w < warp; ++w) before += s_wtot[w];
            s_start[d] = before + inc - tot;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint32_t d = digit(q);
            uint32_t rank, count;
            bool first;
            if (kCacheRanks) {
                const uint32_t v = (info[q / 2] >> (q & 1 ? 16 : 0)) & 0xFFFFu;
                rank = v & 31u;
                count = (v >> 5) & 63u;
                first = (v >> 11) & 1u;
            } else {
                const unsigned same = same_digit_lanes(d);
                rank = __popc(same & below);
                count = __popc(same);
                first = d < kRadix && lane == static_cast<unsigned>(__ffs(same) - 1);
            }
            if (d < kRadix) s_keys[s_start[d] + s_woff[warp][d] + rank] = key[q];
            __syncwarp();
            if (first) s_woff[warp][d] += count;
            __syncwarp();
        }
        __syncthreads();
        const uint32_t valid = static_cast<uint32_t>(min_u64(kSortTile, n - tile0));
        for (uint32_t j = threadIdx.x; j < valid; j += kSortThreads) {
            const uint64_t k = s_keys[j];
            const uint32_t d = static_cast<uint32_t>((k >> shift) & 0xFF);
            out[s_base[d] + (j - s_start[d])] = k;
        }
        __syncthreads();  // every read of s_base, s_start and s_keys done
        s_base[threadIdx.x] += tot;
    }
}

// The staged scatter with the tile's keys in shared memory instead of
// registers (kKeysInSmem): each warp copies its slice into s_in, ranks from
// there and places from there, so the rank words are the only per-key
// registers; with kPrefetchNextTile the loads of the CTA's next tile are
// issued before the current tile's write-out and land in s_in after it (the
// write-out hides their latency). Dynamic shared memory: s_in then s_keys,
// kSortTile keys each.
constexpr bool kKeysInSmem = true;
constexpr bool kPrefetchNextTile = true;
constexpr size_t kSmemScatterBytes = 2 * sizeof(uint64_t) * kSortTile;
static_assert(!kKeysInSmem || kKeysPerLane % 2 == 0, "two keys' rank words per register");

__global__ void __launch_bounds__(kSortThreads, kScatterMinCtas) radix_scatter_smem_kernel(
    const uint64_t* __restrict__ in, uint64_t* __restrict__ out, uint64_t n, uint32_t shift, uint32_t nctas,
    const uint32_t* __restrict__ bases) {
    extern __shared__ uint64_t s_dyn[];
    uint64_t* s_keys = s_dyn + kSortTile;            // the tile in digit order
    __shared__ uint32_t s_woff[kSortWarps][kRadix];  // per warp: digit counts, then running offsets
    __shared__ uint32_t s_start[kRadix];             // digit start inside the tile
    __shared__ uint32_t s_base[kRadix];              // digit's output base for the current tile
    __shared__ uint32_t s_wtot[kSortWarps];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1;
    uint64_t* my_in = s_dyn + warp * kSliceKeys;     // this warp's slice, in input order
    s_base[threadIdx.x] = bases[static_cast<uint64_t>(threadIdx.x) * nctas + blockIdx.x];
    const uint64_t cta0 = static_cast<uint64_t>(blockIdx.x) * kCtaKeys;
    {
        const uint64_t slice = cta0 + static_cast<uint64_t>(warp) * kSliceKeys;
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint64_t i = slice + static_cast<uint64_t>(q) * 32 + lane;
            my_in[q * 32 + lane] = i < n ? in[i] : 0;
        }
    }
    for (int t = 0; t < kTilesPerCta; ++t) {
        const uint64_t tile0 = cta0 + static_cast<uint64_t>(t) * kSortTile;
        if (tile0 >= n) break;  // the same for every thread of the block
        for (int w = 0; w < kSortWarps; ++w) s_woff[w][threadIdx.x] = 0;
        const uint64_t slice = tile0 + static_cast<uint64_t>(warp) * kSliceKeys;
        if (!kPrefetchNextTile && t > 0) {
#pragma unroll
            for (int q = 0; q < kKeysPerLane; ++q) {
                const uint64_t i = slice + static_cast<uint64_t>(q) * 32 + lane;
                my_in[q * 32 + lane] = i < n ? in[i] : 0;
            }
        }
        auto digit = [&](int q) -> uint32_t {
            return slice + static_cast<uint64_t>(q) * 32 + lane < n
                       ? static_cast<uint32_t>((my_in[q * 32 + lane] >> shift) & 0xFF)
                       : static_cast<uint32_t>(kRadix);
        };
        // Per key: rank among the warp's lanes of the same digit (bits 0-4),
        // that digit's lane count (bits 5-10), first lane of the digit (bit
        // 11); two keys per word.
        uint32_t info[kKeysPerLane / 2];
        __syncthreads();  // counters cleared; slices stored; the previous tile's base update visible
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint32_t d = digit(q);
            const unsigned same = same_digit_lanes(d);
            const bool first = d < kRadix && lane == static_cast<unsigned>(__ffs(same) - 1);
            if (first) s_woff[warp][d] += __popc(same);
            const uint32_t v = __popc(same & below) | (__popc(same) << 5) | (first ? 1u << 11 : 0u);
            if (q & 1) info[q / 2] |= v << 16;
            else info[q / 2] = v;
            __syncwarp();
        }
        __syncthreads();
        uint32_t tot = 0;  // the tile's count of digit threadIdx.x
        {
            const uint32_t d = threadIdx.x;
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t c = s_woff[w][d];
                s_woff[w][d] = tot;
                tot += c;
            }
            const uint32_t inc = warp_inclusive_scan(tot);
            if (lane == 31) s_wtot[warp] = inc;
            __syncthreads();
            uint32_t before = 0;
            for (unsigned w = 0; w < warp; ++w) before += s_wtot[w];
            s_start[d] = before + inc - tot;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kKeysPerLane; ++q) {
            const uint32_t d = digit(q);
            const uint32_t v = (info[q / 2] >> (q & 1 ? 16 : 0)) & 0xFFFFu;
            if (d < kRadix) s_keys[s_start[d] + s_woff[warp][d] + (v & 31u)] = my_in[q * 32 + lane];
            __syncwarp();
            if ((v >> 11) & 1u) s_woff[warp][d] += (v >> 5) & 63u;
            __syncwarp();
        }
        __syncthreads();
        // The next tile's slice: loads in flight over the write-out, stored
        // into this warp's s_in slice after it (only this warp reads it).
        const bool more = kPrefetchNextTile && t + 1 < kTilesPerCta && tile0 + kSortTile < n;
        uint64_t nxt[kKeysPerLane];
        if (more) {
#pragma unroll
            for (int q = 0; q < kKeysPerLane; ++q) {
                const uint64_t i = slice + kSortTile + static_cast<uint64_t>(q) * 32 + lane;
                nxt[q] = i < n ? in[i] : 0;
            }
        }
        const uint32_t valid = static_cast<uint32_t>(min_u64(kSortTile, n - tile0));
        for (uint32_t j = threadIdx.x; j < valid; j += kSortThreads) {
            const uint64_t k = s_keys[j];
            const uint32_t d = static_cast<uint32_t>((k >> shift) & 0xFF);
            out[s_base[d] + (j - s_start[d])] = k;
        }
        if (more) {
#pragma unroll
            for (int q = 0; q < kKeysPerLane; ++q) my_in[q * 32 + lane] = nxt[q];
        }
        __syncthreads();  // every read of s_base, s_start and s_keys done
        s_base[threadIdx.x] += tot;
    }
}

Error radix_sort_u64(DeviceImpl& dev, uint64_t* keys, uint64_t* tmp, uint64_t n, uint32_t low_bit, uint32_t high_bit,
                     uint64_t** sorted) {
    *sorted = keys;
    if (n <= 1 || high_bit <= low_bit) return ok();
    // One histogram column and one scatter CTA per range of kCtaKeys keys.
    const uint64_t nctas64 = ceil_div_u64(n, kCtaKeys);
    if (nctas64 * kRadix > 0xFFFFFFFFull || n > 0xFFFFFFFFull) return kernel_error("radix sort input too large");
    const uint32_t nctas = static_cast<uint32_t>(nctas64);
    DeviceBuffer<uint32_t> hist, bases;
    GCU_TRY(hist.allocate(dev, static_cast<uint64_t>(nctas) * kRadix));
    GCU_TRY(bases.allocate(dev, static_cast<uint64_t>(nctas) * kRadix + 1));
    if (kStagedScatter && kKeysInSmem && kSmemScatterBytes > 48 * 1024)
        GCU_CUDA(cudaFuncSetAttribute(radix_scatter_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSmemScatterBytes)),
                 "cudaFuncSetAttribute");
    uint64_t* src = keys;
    uint64_t* dst = tmp;
    for (uint32_t shift = low_bit; shift < high_bit; shift += 8) {
        GCU_LAUNCH(dev, "radix_hist", radix_hist_kernel, nctas, kSortThreads, 0, src, n, shift, nctas, hist.ptr);
        GCU_TRY(exclusive_scan_u32(dev, hist.ptr, bases.ptr, static_cast<uint64_t>(nctas) * kRadix));
        if (kStagedScatter && kKeysInSmem)
            GCU_LAUNCH(dev, "radix_scatter", radix_scatter_smem_kernel, nctas, kSortThreads, kSmemScatterBytes, src,
                       dst, n, shift, nctas, bases.ptr);
        else if (kStagedScatter)
            GCU_LAUNCH(dev, "radix_scatter", radix_scatter_staged_kernel, nctas, kSortThreads, 0, src, dst, n, shift,
                       nctas, bases.ptr);
        else
            GCU_LAUNCH(dev, "radix_scatter", radix_scatter_kernel, nctas, kSortThreads, 0, src, dst, n, shift, nctas,
                       bases.ptr);
        std::swap(src, dst);
    }
    *sorted = src;
    return ok();
}

// ---------------------------------------------------------------- transpose

// keys[j] = (target << 32) | source for every entry j.
__global__ void __launch_bounds__(256) transpose_keys_kernel(const uint32_t* __restrict__ offsets,
                                                             const uint32_t* __restrict__ targets, uint32_t V,
                                                             uint32_t E, uint64_t* __restrict__ keys) {
    for_each_entry<256, 4>(offsets, V, E, [&](uint32_t j, uint32_t u) {
        keys[j] = (static_cast<uint64_t>(targets[j]) << 32) | u;
    });
}

// Sorted keys -> transposed lists: t_targets[j] = the source of key j, and
// in-list v starts at the first key whose target is >= v (rows prev < v <=
// cur get the boundary between keys j - 1 and j; every row one writer, no
// atomics on the hubs' in-degrees).
__global__ void transpose_split_kernel(const uint64_t* __restrict__ keys, uint32_t E, uint32_t V,
                                       uint32_t* __restrict__ t_targets, uint32_t* __restrict__ t_offsets) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j <= E;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int64_t prev = j == 0 ? -1 : static_cast<int64_t>(keys[j - 1] >> 32);
        const int64_t cur = j < E ? static_cast<int64_t>(keys[j] >> 32) : static_cast<int64_t>(V);
        if (j < E) t_targets[j] = static_cast<uint32_t>(keys[j]);
        for (int64_t r = prev + 1; r <= cur; ++r) t_offsets[r] = static_cast<uint32_t>(j);
    }
}

Error transpose_csr(DeviceImpl& dev, const uint32_t* offsets, const uint32_t* targets, uint32_t V, uint32_t E,
                    DeviceBuffer<uint32_t>* t_offsets, DeviceBuffer<uint32_t>* t_targets) {
    GCU_TRY(t_offsets->allocate(dev, static_cast<uint64_t>(V) + 1));
    GCU_TRY(t_targets->allocate(dev, E));
    GCU_CUDA(cudaMemsetAsync(t_offsets->ptr, 0, sizeof(uint32_t) * (static_cast<size_t>(V) + 1), dev.stream), "memset");
    if (E == 0) return ok();
    DeviceBuffer<uint64_t> keys, tmp;
    GCU_TRY(keys.allocate(dev, E));
    GCU_TRY(tmp.allocate(dev, E));
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned tgrid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(E, 1024), cap)));
    const unsigned egrid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(static_cast<uint64_t>(E) + 1, 256), cap));
    GCU_LAUNCH(dev, "transpose_keys", transpose_keys_kernel, tgrid, 256, 0, offsets, targets, V, E, keys.ptr);
    uint32_t bits = 0;
    while (bits < 32 && (static_cast<uint64_t>(1) << bits) < V) ++bits;
    uint64_t* sorted = nullptr;
    // Stable sort by target only: sources stay ascending inside each in-list.
    GCU_TRY(radix_sort_u64(dev, keys.ptr, tmp.ptr, E, 32, 32 + ((bits + 7) / 8) * 8, &sorted));
    GCU_LAUNCH(dev, "transpose_split", transpose_split_kernel, egrid, 256, 0, sorted, E, V, t_targets->ptr,
               t_offsets->ptr);
    GCU_TRY(dev.sync());  // keys/tmp are freed on return
    return ok();
}

}  // namespace gcu
