// Device helpers shared by the kernel files (sm_100a, 32-lane warps).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace gcu {

constexpr int kWarp = 32;
constexpr unsigned kFullMask = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(kFullMask, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Inclusive warp scan.
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const unsigned lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T w = __shfl_up_sync(kFullMask, v, o);
        if (lane >= static_cast<unsigned>(o)) v += w;
    }
    return v;
}

// Block-wide sum; every thread gets the result. `scratch` holds >= 32 values.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
    const unsigned nwarps = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = (threadIdx.x < nwarps) ? scratch[threadIdx.x] : T(0);
    if (warp == 0) r = warp_sum(r);
    if (threadIdx.x == 0) scratch[0] = r;
    __syncthreads();
    r = scratch[0];
    __syncthreads();
    return r;
}

// Streaming load that does not allocate in L1 (data read once).
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ uint2 ld_stream2(const uint2* p) {
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0,%1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ uint4 ld_stream4(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// First index in [lo, hi) with a[idx] >= val.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t val) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < val)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Largest row r in [0, n) with offsets[r] <= pos (offsets non-decreasing,
// offsets[0] == 0 <= pos).
__device__ __forceinline__ uint32_t row_of_entry(const uint32_t* offsets, uint32_t n, uint32_t pos) {
    uint32_t lo = 0, hi = n;  // answer in [lo, hi)
    while (hi - lo > 1) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (offsets[mid] <= pos)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------- entry tiles
// A block that works on a tile of consecutive CSR entries [e0, e1) finds the
// row of each entry from the row starts of the tile, staged in shared memory
// (s_start, kTile words; s_meta, 2 words); when the tile spans more rows than
// fit (runs of empty rows), each entry searches the global offsets instead.

// Largest row r in [0, n) with offsets[r] <= pos (defined above) picks, among
// empty rows that share a start, the non-empty row that holds the entry.
template <int kTile>
__device__ __forceinline__ bool stage_tile_rows(const uint32_t* __restrict__ offsets, uint32_t V, uint64_t e0,
                                                uint64_t e1, uint32_t* s_start, uint32_t* s_meta) {
    if (threadIdx.x < 2)
        s_meta[threadIdx.x] = row_of_entry(offsets, V, static_cast<uint32_t>(threadIdx.x == 0 ? e0 : e1 - 1));
    __syncthreads();
    const uint32_t r0 = s_meta[0], nrows = s_meta[1] - r0 + 1;
    const bool staged = nrows <= static_cast<uint32_t>(kTile);
    if (staged)
        for (uint32_t k = threadIdx.x; k < nrows; k += blockDim.x) s_start[k] = offsets[r0 + k];
    __syncthreads();
    return staged;
}

__device__ __forceinline__ uint32_t tile_row(const uint32_t* __restrict__ offsets, uint32_t V, const uint32_t* s_start,
                                             bool staged, uint32_t r0, uint32_t nrows, uint32_t j) {
    if (!staged) return row_of_entry(offsets, V, j);
    uint32_t lo = 0, hi = nrows;  // largest k with s_start[k] <= j
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_start[mid] <= j)
            lo = mid;
        else
            hi = mid;
    }
    return r0 + lo;
}

__host__ __device__ __forceinline__ uint64_t min_u64(uint64_t a, uint64_t b) { return a < b ? a : b; }

__host__ __device__ __forceinline__ uint64_t ceil_div_u64(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Calls f(j, row) for every entry j of a CSR with V rows and E entries: each
// block takes tiles of kThreads * kItems consecutive entries (grid-stride),
// so long rows are shared by many blocks and every access to the entries is
// coalesced. All threads of the block must call it.
template <int kThreads, int kItems, class F>
__device__ __forceinline__ void for_each_entry(const uint32_t* __restrict__ offsets, uint32_t V, uint64_t E, F f) {
    constexpr int kTile = kThreads * kItems;
    __shared__ uint32_t s_start[kTile];
    __shared__ uint32_t s_meta[2];
    for (uint64_t e0 = static_cast<uint64_t>(blockIdx.x) * kTile; e0 < E;
         e0 += static_cast<uint64_t>(gridDim.x) * kTile) {
        const uint64_t e1 = min_u64(e0 + kTile, E);
        const bool staged = stage_tile_rows<kTile>(offsets, V, e0, e1, s_start, s_meta);
        const uint32_t r0 = s_meta[0], nrows = s_meta[1] - r0 + 1;
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
            const uint64_t j = e0 + q * kThreads + threadIdx.x;
            if (j < e1) f(static_cast<uint32_t>(j), tile_row(offsets, V, s_start, staged, r0, nrows,
                                                              static_cast<uint32_t>(j)));
        }
        __syncthreads();  // the staged starts are rewritten for the next tile
    }
}

}  // namespace gcu
