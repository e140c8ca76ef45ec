// CSR validation on the device.
//
// The reference checks every CSR on the host before the copy
// (crates/grafeo-cuda-core/src/csr_export.rs:71-120): a serial O(V + E) scan
// that takes longer than the algorithms themselves at scale. Here the arrays
// are copied first and one coalesced pass on the device finds the first node
// that breaks a rule; the host then rebuilds the exact reference message for
// that node alone (describe_node_violation). The rules, per node in order:
//   offsets[node + 1] >= offsets[node]                 ("offsets decrease ...")
//   every target < num_nodes                           ("... has neighbor ...")
//   every list strictly increasing                     ("... not strictly increasing ...")
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

// One warp walks 32 consecutive nodes; for each node all lanes check its list
// in coalesced 32-entry strides. The smallest offending node wins (atomicMin).
__global__ void __launch_bounds__(256) csr_validate_kernel(const uint32_t* __restrict__ offsets,
                                                           const uint32_t* __restrict__ targets,
                                                           uint32_t num_nodes, uint32_t num_edges,
                                                           uint32_t* __restrict__ first_bad) {
    const unsigned lane = lane_id();
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < num_nodes; base += nwarps * 32) {
        // Lane i loads the bounds of node base + i.
        uint64_t my = base + lane;
        uint32_t s = 0, e = 0;
        if (my < num_nodes) {
            s = offsets[my];
            e = offsets[my + 1];
        }
        const uint32_t count = static_cast<uint32_t>(min_u64(32, num_nodes - base));
        for (uint32_t i = 0; i < count; ++i) {
            uint32_t start = __shfl_sync(kFullMask, s, i);
            uint32_t end = __shfl_sync(kFullMask, e, i);
            bool bad = end < start || end > num_edges;
            if (!bad) {
                for (uint32_t j = start + lane; j < end; j += 32) {
                    uint32_t t = targets[j];
                    bool wrong = t >= num_nodes || (j > start && targets[j - 1] >= t);
                    if (__any_sync(__activemask(), wrong)) {
                        bad = true;
                        break;
                    }
                }
                bad = __any_sync(kFullMask, bad);
            }
            if (bad) {
                if (lane == 0) atomicMin(first_bad, static_cast<uint32_t>(base + i));
                break;  // later nodes of this warp cannot be first
            }
        }
    }
}

Error validate_csr_device(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets,
                          uint32_t num_nodes, uint32_t num_edges, uint32_t* first_bad_node) {
    *first_bad_node = UINT32_MAX;
    if (num_nodes == 0) return ok();
    DeviceBuffer<uint32_t> flag;
    GCU_TRY(flag.allocate(dev, 1));
    GCU_CUDA(cudaMemsetAsync(flag.ptr, 0xFF, sizeof(uint32_t), dev.stream), "memset");
    uint64_t warps = ceil_div_u64(num_nodes, 32);
    uint64_t blocks = std::min<uint64_t>(ceil_div_u64(warps * 32, 256), static_cast<uint64_t>(dev.sm_count) * 16);
    GCU_LAUNCH(dev, "csr_validate", csr_validate_kernel, static_cast<unsigned>(blocks), 256, 0, d_offsets,
               d_targets, num_nodes, num_edges, flag.ptr);
    uint32_t host = UINT32_MAX;
    GCU_CUDA(cudaMemcpyAsync(&host, flag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy flag");
    GCU_TRY(dev.sync());
    *first_bad_node = host;
    return ok();
}

// Symmetry test: every entry u -> v needs v -> u. A warp walks 32 rows; the
// lanes stride over each row and binary-search u in the neighbour's list.
__global__ void csr_symmetry_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                    uint32_t V, uint32_t* __restrict__ asymmetric) {
    const unsigned lane = lane_id();
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < V; base += nwarps * 32) {
        const uint32_t count = static_cast<uint32_t>(min_u64(32, V - base));
        uint32_t s = 0, e = 0;
        if (lane < count) {
            s = offsets[base + lane];
            e = offsets[base + lane + 1];
        }
        bool bad = false;
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t u = static_cast<uint32_t>(base + i);
            const uint32_t start = __shfl_sync(kFullMask, s, i), end = __shfl_sync(kFullMask, e, i);
            for (uint32_t j = start + lane; j < end; j += 32) {
                const uint32_t v = targets[j];
                const uint32_t vs = offsets[v], ve = offsets[v + 1];
                const uint32_t p = lower_bound_u32(targets, vs, ve, u);
                if (p == ve || targets[p] != u) bad = true;
            }
        }
        if (__any_sync(kFullMask, bad)) {
            if (lane == 0) atomicOr(asymmetric, 1u);
            return;
        }
    }
}


Error graph_symmetry(GraphImpl& g, bool* symmetric) {
    if (g.symmetric < 0) {
        if (g.num_edges == 0) {
            g.symmetric = 1;
        } else {
            DeviceImpl& dev = *g.dev;
            DeviceBuffer<uint32_t> flag;
            GCU_TRY(flag.allocate(dev, 1));
            GCU_CUDA(cudaMemsetAsync(flag.ptr, 0, sizeof(uint32_t), dev.stream), "memset");
            unsigned blocks = static_cast<unsigned>(
                std::min<uint64_t>(ceil_div_u64(g.num_nodes, 256), static_cast<uint64_t>(dev.sm_count) * 16));
            GCU_LAUNCH(dev, "csr_symmetry", csr_symmetry_kernel, blocks, 256, 0, g.offsets.ptr, g.targets.ptr,
                       g.num_nodes, flag.ptr);
            uint32_t host = 0;
            GCU_CUDA(cudaMemcpyAsync(&host, flag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, dev.stream), "copy");
            GCU_TRY(dev.sync());
            g.symmetric = host == 0 ? 1 : 0;
        }
    }
    *symmetric = g.symmetric == 1;
    return ok();
}

}  // namespace gcu
