// Device-wide exclusive scan of u32 counts into CSR-style offsets.
//
// Replaces the reference's single-thread `prefix_sum_kernel`
// (crates/grafeo-cuda-algos/kernels/triangle_counting.cu:223-237), a serial
// O(V) loop on one GPU thread. Three passes: per-tile sums, a scan of the tile
// sums in one block, then the per-tile scan with its carry-in. Each tile is
// 1024 threads x 8 items; the input is read twice and the output written once.
// Inputs of one tile take a single launch.
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(const uint32_t* __restrict__ in, uint64_t n,
                                                                     uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t scratch[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + static_cast<uint64_t>(k) * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    s = block_sum(s, scratch);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = s;
}

// Exclusive scan of the tile sums in place; writes the grand total to *total.
__global__ void __launch_bounds__(kScanThreads) scan_tile_prefix_kernel(uint32_t* __restrict__ tile_sums,
                                                                       uint64_t num_tiles, uint32_t* __restrict__ total) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint64_t base = 0; base < num_tiles; base += kScanThreads) {
        uint64_t i = base + threadIdx.x;
        uint32_t v = i < num_tiles ? tile_sums[i] : 0;
        uint32_t inc = warp_inclusive_scan(v);
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_tot[lane];
            uint32_t winc = warp_inclusive_scan(w);
            warp_tot[lane] = winc - w;
        }
        __syncthreads();
        uint32_t excl = carry + warp_tot[warp] + inc - v;
        if (i < num_tiles) tile_sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// `in` and `out` may be the same array (callers scan in place), so neither is
// __restrict__: every thread loads its items into registers before it stores.
__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(const uint32_t* in, uint64_t n,
                                                                 const uint32_t* __restrict__ tile_prefix,
                                                                 uint32_t* out) {
    __shared__ uint32_t warp_tot[32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
    // Thread t owns items base + t*8 .. base + t*8 + 7 (a blocked layout).
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + static_cast<uint64_t>(threadIdx.x) * kScanItems + k;
        v[k] = i < n ? in[i] : 0;
        local += v[k];
    }
    uint32_t inc = warp_inclusive_scan(local);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_tot[lane];
        warp_tot[lane] = warp_inclusive_scan(w) - w;
    }
    __syncthreads();
    uint32_t run = tile_prefix[blockIdx.x] + warp_tot[warp] + inc - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint64_t i = base + static_cast<uint64_t>(threadIdx.x) * kScanItems + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// One tile (n <= kScanTile): the whole scan in one launch, the total in
// out[n]. Every thread reads its items before it writes them, so in == out
// is fine.
__global__ void __launch_bounds__(kScanThreads) scan_one_tile_kernel(const uint32_t* in, uint32_t n,
                                                                    uint32_t* out) {
    __shared__ uint32_t warp_tot[32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = threadIdx.x * kScanItems + k;
        v[k] = i < n ? in[i] : 0;
        local += v[k];
    }
    const uint32_t inc = warp_inclusive_scan(local);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_tot[lane];
        warp_tot[lane] = warp_inclusive_scan(w) - w;
    }
    __syncthreads();
    uint32_t run = warp_tot[warp] + inc - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = threadIdx.x * kScanItems + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) out[n] = run;
}

// ---- the same scan with its length read on the device (*n_ptr), for launch
// sequences captured into a CUDA graph whose sizes the host never sees. The
// grids are fixed; tile loops stride over them. One tile: one kernel does
// the scan; more: tile sums, their scan, then the tiles. Each kernel returns
// at once when the length is not its case.

__global__ void __launch_bounds__(kScanThreads) scan_one_tile_dn_kernel(const uint32_t* in, const uint32_t* n_ptr,
                                                                       uint32_t* out) {
    const uint32_t n = *n_ptr;
    if (n > static_cast<uint32_t>(kScanTile)) return;
    __shared__ uint32_t warp_tot[32];
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = threadIdx.x * kScanItems + k;
        v[k] = i < n ? in[i] : 0;
        local += v[k];
    }
    const uint32_t inc = warp_inclusive_scan(local);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_tot[lane];
        warp_tot[lane] = warp_inclusive_scan(w) - w;
    }
    __syncthreads();
    uint32_t run = warp_tot[warp] + inc - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = threadIdx.x * kScanItems + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) out[n] = run;
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_dn_kernel(const uint32_t* __restrict__ in,
                                                                        const uint32_t* __restrict__ n_ptr,
                                                                        uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t scratch[32];
    const uint64_t n = *n_ptr;
    if (n <= static_cast<uint64_t>(kScanTile)) return;
    const uint64_t tiles = ceil_div_u64(n, kScanTile);
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t base = t * kScanTile;
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const uint64_t i = base + static_cast<uint64_t>(k) * kScanThreads + threadIdx.x;
            if (i < n) s += in[i];
        }
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) tile_sums[t] = s;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_prefix_dn_kernel(uint32_t* __restrict__ tile_sums,
                                                                          const uint32_t* __restrict__ n_ptr,
                                                                          uint32_t* __restrict__ out) {
    const uint64_t n = *n_ptr;
    if (n <= static_cast<uint64_t>(kScanTile)) return;
    const uint64_t num_tiles = ceil_div_u64(n, kScanTile);
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint64_t base = 0; base < num_tiles; base += kScanThreads) {
        const uint64_t i = base + threadIdx.x;
        const uint32_t v = i < num_tiles ? tile_sums[i] : 0;
        const uint32_t inc = warp_inclusive_scan(v);
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = warp_tot[lane];
            warp_tot[lane] = warp_inclusive_scan(w) - w;
        }
        __syncthreads();
        const uint32_t excl = carry + warp_tot[warp] + inc - v;
        if (i < num_tiles) tile_sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// `in` and `out` may be the same array (each tile is read into registers
// before it is written).
__global__ void __launch_bounds__(kScanThreads) scan_tiles_dn_kernel(const uint32_t* in, const uint32_t* n_ptr,
                                                                    const uint32_t* __restrict__ tile_prefix,
                                                                    uint32_t* out) {
    __shared__ uint32_t warp_tot[32];
    const uint64_t n = *n_ptr;
    if (n <= static_cast<uint64_t>(kScanTile)) return;
    const uint64_t tiles = ceil_div_u64(n, kScanTile);
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t base = t * kScanTile;
        uint32_t v[kScanItems];
        uint32_t local = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const uint64_t i = base + static_cast<uint64_t>(threadIdx.x) * kScanItems + k;
            v[k] = i < n ? in[i] : 0;
            local += v[k];
        }
        const uint32_t inc = warp_inclusive_scan(local);
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = warp_tot[lane];
            warp_tot[lane] = warp_inclusive_scan(w) - w;
        }
        __syncthreads();
        uint32_t run = tile_prefix[t] + warp_tot[warp] + inc - local;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const uint64_t i = base + static_cast<uint64_t>(threadIdx.x) * kScanItems + k;
            if (i < n) out[i] = run;
            run += v[k];
        }
        __syncthreads();  // warp_tot is reused by the next tile
    }
}

uint64_t scan_device_n_tiles(uint64_t max_n) { return std::max<uint64_t>(1, ceil_div_u64(max_n, kScanTile)); }

static_assert(kScanTile == kScanOneLaunchMax, "one-launch scan size");

Error exclusive_scan_u32_device_n(DeviceImpl& dev, const uint32_t* d_in, uint32_t* d_out, const uint32_t* d_n,
                                  uint64_t max_n, uint32_t* tile_sums, ScanLaunches which) {
    const unsigned grid = static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>(scan_device_n_tiles(max_n), static_cast<uint64_t>(dev.sm_count) * 2)));
    if (which != ScanLaunches::kMultiTile)
        GCU_LAUNCH(dev, "scan_one_tile", scan_one_tile_dn_kernel, 1, kScanThreads, 0, d_in, d_n, d_out);
    if (which != ScanLaunches::kOneTile && max_n > static_cast<uint64_t>(kScanTile)) {
        GCU_LAUNCH(dev, "scan_tile_sums", scan_tile_sums_dn_kernel, grid, kScanThreads, 0, d_in, d_n, tile_sums);
        GCU_LAUNCH(dev, "scan_tile_prefix", scan_tile_prefix_dn_kernel, 1, kScanThreads, 0, tile_sums, d_n, d_out);
        GCU_LAUNCH(dev, "scan_tiles", scan_tiles_dn_kernel, grid, kScanThreads, 0, d_in, d_n, tile_sums, d_out);
    }
    return ok();
}

Error exclusive_scan_u32(DeviceImpl& dev, const uint32_t* d_in, uint32_t* d_out, uint64_t n) {
    if (n == 0) {
        GCU_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint32_t), dev.stream), "memset");
        return ok();
    }
    if (n <= static_cast<uint64_t>(kScanTile)) {
        // Small inputs (BFS frontiers, per-round peel lists): one launch.
        GCU_LAUNCH(dev, "scan_one_tile", scan_one_tile_kernel, 1, kScanThreads, 0, d_in, static_cast<uint32_t>(n),
                   d_out);
        return ok();
    }
    const uint64_t tiles = ceil_div_u64(n, kScanTile);
    DeviceBuffer<uint32_t> sums;
    GCU_TRY(sums.allocate(dev, tiles));
    GCU_LAUNCH(dev, "scan_tile_sums", scan_tile_sums_kernel, static_cast<unsigned>(tiles), kScanThreads, 0, d_in, n,
               sums.ptr);
    GCU_LAUNCH(dev, "scan_tile_prefix", scan_tile_prefix_kernel, 1, kScanThreads, 0, sums.ptr, tiles, d_out + n);
    GCU_LAUNCH(dev, "scan_tiles", scan_tiles_kernel, static_cast<unsigned>(tiles), kScanThreads, 0, d_in, n, sums.ptr,
               d_out);
    return ok();
}

}  // namespace gcu
