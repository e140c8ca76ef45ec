// Oriented triangle count that allocates nothing on the device.
//
// Some callers cannot allocate device memory at the moment they need a
// result: code running under a fixed memory budget that hands out all device
// memory up front (a serving process that pre-reserves its pool), code inside
// a framework whose allocator owns the device and forbids side allocations,
// or code on a path where an allocation could block or fail late. They already
// hold the graph on the device and only need the count. This entry point takes
// the caller's device CSR and stream and uses, as its only working memory, the
// file-scope array below, which is part of the library image and exists on
// every device that loads the library until the process exits.
//
// Limits and rules (also in include/grafeo_cuda.h):
//  * at most kNoAllocMaxNodes vertices; larger graphs are rejected with
//    GCU_ERR_KERNEL before anything runs;
//  * the array is shared by every call on a device and keeps the last call's
//    contents; each call clears the counters it needs first. Calls that
//    overlap on the GPU (two host threads, or two streams) race on it;
//  * the first call on a device looks up the array's device address with that
//    device current (cudaGetSymbolAddress); make that first call before any
//    stream capture. The address is kept for the life of the process, which
//    assumes the device's primary context is never reset (cudaDeviceReset)
//    between calls;
//  * each call waits for the caller's stream to finish before it returns (the
//    count is copied to the host);
//  * the CSR is not validated here: it must satisfy validate_csr (sorted,
//    duplicate-free lists, targets < num_nodes), as every GpuGraph does.
#include <mutex>

#include "device_common.cuh"
#include "gcu_internal.h"
#include "wedge.cuh"

namespace gcu {

constexpr uint32_t kNoAllocMaxNodes = 1u << 20;  // 4 MiB of queue space per device
constexpr uint32_t kNoAllocHeader = 8;            // [0] next vertex [1] long count [2] next long [4..5] u64 total

// The working memory: counters, then the queue of long out-lists.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocHeader + kNoAllocMaxNodes];

namespace {

struct NoAllocCountSink {
    static constexpr bool kNeedsPos = false;
    unsigned long long* total;
    unsigned long long count;
    __device__ __forceinline__ void hit(uint32_t, uint32_t, uint32_t, uint32_t) { ++count; }
    __device__ __forceinline__ void finish() {
        const unsigned long long c = warp_sum(count);
        if (lane_id() == 0 && c) atomicAdd(total, c);
    }
};

std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[256] = {};  // device address of the array, per device ordinal

// Device address of the array on the current device (looked up once).
Error noalloc_scratch(int device, uint32_t** out) {
    if (device < 0 || device >= 256) return kernel_error("device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        GCU_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
        g_noalloc_ptr[device] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_ptr[device];
    return ok();
}

Error triangle_count_oriented_noalloc(const uint32_t* d_offsets, const uint32_t* d_targets, uint32_t num_nodes,
                                      uint32_t num_edges, cudaStream_t stream, uint64_t* total) {
    *total = 0;
    if (num_nodes > kNoAllocMaxNodes) {
        return kernel_error("graph has " + std::to_string(num_nodes) +
                            " nodes; the allocation-free triangle count takes at most " +
                            std::to_string(kNoAllocMaxNodes));
    }
    if (num_nodes == 0 || num_edges == 0) return ok();
    if (!d_offsets || !d_targets) return kernel_error("CSR pointer is NULL");
    int device = 0;
    GCU_CUDA(cudaGetDevice(&device), "cudaGetDevice");
    uint32_t* scratch = nullptr;
    GCU_TRY(noalloc_scratch(device, &scratch));
    int sms = 0;
    GCU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");

    uint32_t* next_vertex = scratch;
    uint32_t* long_count = scratch + 1;
    uint32_t* next_long = scratch + 2;
    auto* d_total = reinterpret_cast<unsigned long long*>(scratch + 4);
    uint32_t* long_list = scratch + kNoAllocHeader;
    GCU_CUDA(cudaMemsetAsync(scratch, 0, kNoAllocHeader * sizeof(uint32_t), stream), "memset");

    const unsigned grid = static_cast<unsigned>(sms) * 8;
    const unsigned collect_blocks = static_cast<unsigned>(
        std::min<uint64_t>(ceil_div_u64(num_nodes, 256), static_cast<uint64_t>(sms) * 8));
    const NoAllocCountSink sink{d_total, 0};
    wedge_collect_long_kernel<<<collect_blocks, 256, 0, stream>>>(d_offsets, num_nodes, long_list, long_count);
    GCU_CUDA(cudaGetLastError(), "launch");
    wedge_cta_kernel<NoAllocCountSink><<<grid, kWedgeThreads, 0, stream>>>(d_offsets, d_targets, long_list,
                                                                            long_count, next_long, sink);
    GCU_CUDA(cudaGetLastError(), "launch");
    wedge_warp_kernel<NoAllocCountSink><<<grid, kWedgeThreads, 0, stream>>>(d_offsets, d_targets, num_nodes, 1,
                                                                             next_vertex, sink);
    GCU_CUDA(cudaGetLastError(), "launch");
    unsigned long long host_total = 0;
    GCU_CUDA(cudaMemcpyAsync(&host_total, d_total, sizeof(host_total), cudaMemcpyDeviceToHost, stream), "copy");
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return kernel_error(std::string("synchronize failed: ") + cudaGetErrorString(e));
    *total = host_total;
    return ok();
}

}  // namespace
}  // namespace gcu

extern "C" GCU_API gcu_status gcu_triangle_count_oriented_noalloc(const uint32_t* d_offsets,
                                                                  const uint32_t* d_targets, uint32_t num_nodes,
                                                                  uint32_t num_edges, void* stream,
                                                                  uint64_t* total) {
    if (!total) return gcu::fail(gcu::kernel_error("total is NULL"));
    gcu::Error e = gcu::triangle_count_oriented_noalloc(d_offsets, d_targets, num_nodes, num_edges,
                                                        static_cast<cudaStream_t>(stream), total);
    return e.ok() ? gcu::succeed() : gcu::fail(e);
}
