// Stable LSD radix sort of 64-bit keys, and the CSR transpose built on it.
//
// Each pass sorts by one 8-bit digit: per-tile digit histograms (digit-major,
// so one exclusive scan gives every (digit, tile) its output base), then a
// stable scatter of each tile of kSortTile keys, staged in shared memory in
// digit order and written out as contiguous runs (radix_scatter_staged_kernel;
// the first form, radix_scatter_kernel, walked the tile in rounds of 256 keys
// and wrote every key to its own address).
// Stability makes the sort of (target << 32 | source) keys by their high word
// keep every in-list ordered by source, so the transpose is deterministic.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // keys per tile
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                                                  uint32_t shift, uint32_t ntiles,
                                                                  uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t i = base + static_cast<uint64_t>(r) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    hist[static_cast<uint64_t>(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];
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

// The same stable scatter with the tile staged in shared memory. Each warp
// owns a contiguous slice of kSliceKeys keys (kKeysPerLane per lane, loaded
// coalesced and kept in registers). Pass 1 counts the slice's digits with
// warp matches; one barrier later every digit has its start inside the tile
// and every warp its offset inside each digit; pass 2 ranks the keys again in
// the same order and stores them in shared memory in digit order (index order
// inside a digit: stable); the block then writes the tile out run by run,
// consecutive threads to consecutive addresses of a digit's output range.
// Measured on the transpose of R-MAT 24's directed copy (505 M keys, 3
// passes): 23.0 ms with the scatter above (each key written to its own
// address, three block barriers per 256-key round), 18.2 ms staged.
constexpr bool kStagedScatter = true;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSliceKeys = kSortTile / kSortWarps;
constexpr int kKeysPerLane = kSliceKeys / 32;

// Lanes of the warp holding the same digit (kRadix: a lane with no key), from
// one ballot per digit bit (kMatchBallots) or one match instruction. The
// ballots took the staged scatter of the same transpose from 18.2 to 15.0 ms.
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

__global__ void __launch_bounds__(kSortThreads, 3) radix_scatter_staged_kernel(const uint64_t* __restrict__ in,
                                                                            uint64_t* __restrict__ out, uint64_t n,
                                                                            uint32_t shift, uint32_t ntiles,
                                                                            const uint32_t* __restrict__ bases) {
    __shared__ uint64_t s_keys[kSortTile];
    __shared__ uint32_t s_woff[kSortWarps][kRadix];  // per warp: digit counts, then running offsets
    __shared__ uint32_t s_start[kRadix];             // digit start inside the tile
    __shared__ uint32_t s_base[kRadix];              // digit's output base for this tile
    __shared__ uint32_t s_wtot[kSortWarps];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1;
    for (int w = 0; w < kSortWarps; ++w) s_woff[w][threadIdx.x] = 0;
    s_base[threadIdx.x] = bases[static_cast<uint64_t>(threadIdx.x) * ntiles + blockIdx.x];
    const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kSortTile;
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
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kKeysPerLane; ++q) {
        const uint32_t d = digit(q);
        const unsigned same = same_digit_lanes(d);
        if (d < kRadix && lane == static_cast<unsigned>(__ffs(same) - 1)) s_woff[warp][d] += __popc(same);
        __syncwarp();
    }
    __syncthreads();
    {
        // Thread d: the warps' exclusive offsets inside digit d, then the
        // digits' exclusive starts inside the tile (block-wide scan).
        const uint32_t d = threadIdx.x;
        uint32_t tot = 0;
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
        const unsigned same = same_digit_lanes(d);
        if (d < kRadix) s_keys[s_start[d] + s_woff[warp][d] + __popc(same & below)] = key[q];
        __syncwarp();
        if (d < kRadix && lane == static_cast<unsigned>(__ffs(same) - 1)) s_woff[warp][d] += __popc(same);
        __syncwarp();
    }
    __syncthreads();
    const uint32_t valid = static_cast<uint32_t>(min_u64(kSortTile, n - tile0));
    for (uint32_t j = threadIdx.x; j < valid; j += kSortThreads) {
        const uint64_t k = s_keys[j];
        const uint32_t d = static_cast<uint32_t>((k >> shift) & 0xFF);
        out[s_base[d] + (j - s_start[d])] = k;
    }
}

Error radix_sort_u64(DeviceImpl& dev, uint64_t* keys, uint64_t* tmp, uint64_t n, uint32_t low_bit, uint32_t high_bit,
                     uint64_t** sorted) {
    *sorted = keys;
    if (n <= 1 || high_bit <= low_bit) return ok();
    const uint64_t ntiles64 = ceil_div_u64(n, kSortTile);
    if (ntiles64 * kRadix > 0xFFFFFFFFull || n > 0xFFFFFFFFull) return kernel_error("radix sort input too large");
    const uint32_t ntiles = static_cast<uint32_t>(ntiles64);
    DeviceBuffer<uint32_t> hist, bases;
    GCU_TRY(hist.allocate(dev, static_cast<uint64_t>(ntiles) * kRadix));
    GCU_TRY(bases.allocate(dev, static_cast<uint64_t>(ntiles) * kRadix + 1));
    uint64_t* src = keys;
    uint64_t* dst = tmp;
    for (uint32_t shift = low_bit; shift < high_bit; shift += 8) {
        GCU_LAUNCH(dev, "radix_hist", radix_hist_kernel, ntiles, kSortThreads, 0, src, n, shift, ntiles, hist.ptr);
        GCU_TRY(exclusive_scan_u32(dev, hist.ptr, bases.ptr, static_cast<uint64_t>(ntiles) * kRadix));
        if (kStagedScatter)
            GCU_LAUNCH(dev, "radix_scatter", radix_scatter_staged_kernel, ntiles, kSortThreads, 0, src, dst, n, shift,
                       ntiles, bases.ptr);
        else
            GCU_LAUNCH(dev, "radix_scatter", radix_scatter_kernel, ntiles, kSortThreads, 0, src, dst, n, shift, ntiles,
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
