// CSR validation on the device.
//
// The reference checks every CSR on the host before the copy
// (crates/grafeo-cuda-core/src/csr_export.rs:71-120): a serial O(V + E) scan
// that takes longer than the algorithms themselves at scale. Here the arrays
// are copied first and coalesced passes on the device find the first node
// that breaks a rule; the host then rebuilds the exact reference message for
// that node alone (describe_node_violation). The rules, per node in order:
//   offsets[node + 1] >= offsets[node]                 ("offsets decrease ...")
//   every target < num_nodes                           ("... has neighbor ...")
//   every list strictly increasing                     ("... not strictly increasing ...")
#include <algorithm>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

// Three coalesced passes, each O(V) or O(E), with the smallest offending node
// kept by atomicMin (flags[0..2] = decrease, past-the-end, list error):
//  1. per node: offsets[u+1] < offsets[u] (decrease) or offsets[u+1] > E;
//  2. per node below the first such node: mark the first entry of every
//     non-empty list in a bitmap over the entries;
//  3. per entry below that node's offset: target >= V, or not a list start
//     and not above its predecessor; the offending entry's node is found by
//     a binary search over the (monotone) offsets.
// A node's own rules are checked before later nodes' ones, so the smallest
// node reported is the first node the reference's serial scan would reject.
__global__ void csr_check_offsets_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint32_t E,
                                         uint32_t* __restrict__ flags) {
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < V;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t s = offsets[u], e = offsets[u + 1];
        if (e < s) atomicMin(flags + 0, static_cast<uint32_t>(u));
        if (e > E) atomicMin(flags + 1, static_cast<uint32_t>(u));
    }
}

__device__ __forceinline__ uint32_t checked_limit(const uint32_t* flags, uint32_t V) {
    return min(min(flags[0], flags[1]), V);
}

__global__ void csr_mark_starts_kernel(const uint32_t* __restrict__ offsets, uint32_t V,
                                       const uint32_t* __restrict__ flags, uint32_t* __restrict__ starts) {
    const uint32_t limit = checked_limit(flags, V);
    for (uint64_t u = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < limit;
         u += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t s = offsets[u];
        if (offsets[u + 1] > s) atomicOr(starts + (s >> 5), 1u << (s & 31));
    }
}

// Entries [j0, j1) (those below the first offset violation); entry j - 1 must
// be on the device too.
__global__ void csr_check_entries_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ targets,
                                         uint32_t V, const uint32_t* __restrict__ starts,
                                         uint32_t* __restrict__ flags, uint64_t j0, uint64_t j1) {
    const uint32_t limit = checked_limit(flags, V);
    const uint64_t end = min_u64(offsets[limit], j1);
    for (uint64_t j = j0 + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < end;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t t = ld_stream(targets + j);
        const bool first = (starts[j >> 5] >> (j & 31)) & 1u;
        const bool bad = t >= V || (!first && targets[j - 1] >= t);
        if (bad) atomicMin(flags + 2, row_of_entry(offsets, limit, static_cast<uint32_t>(j)));
    }
}

// Entries per chunk of the overlapped upload (64 MB of targets).
constexpr uint64_t kUploadChunk = uint64_t{1} << 24;

// With h_targets, the targets are copied here, chunk by chunk on the copy
// stream, and the entry checks of each chunk wait for its copy only.
static Error check_csr(DeviceImpl& dev, const uint32_t* d_offsets, uint32_t* d_targets, const uint32_t* h_targets,
                       uint32_t num_nodes, uint32_t num_edges, uint32_t* first_bad_node) {
    *first_bad_node = UINT32_MAX;
    if (num_nodes == 0) {
        if (h_targets && num_edges)
            GCU_CUDA(cudaMemcpyAsync(d_targets, h_targets, sizeof(uint32_t) * num_edges, cudaMemcpyHostToDevice,
                                     dev.stream),
                     "copy CSR to device");
        return ok();
    }
    const uint64_t words = ceil_div_u64(num_edges, 32);
    DeviceBuffer<uint32_t> scratch;  // 4 flags, then the list-start bitmap
    GCU_TRY(scratch.allocate(dev, 4 + words));
    uint32_t* flags = scratch.ptr;
    uint32_t* starts = scratch.ptr + 4;
    GCU_CUDA(cudaMemsetAsync(flags, 0xFF, 4 * sizeof(uint32_t), dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(starts, 0, words * sizeof(uint32_t), dev.stream), "memset");
    const uint64_t cap = static_cast<uint64_t>(dev.sm_count) * 16;
    const unsigned node_grid = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(num_nodes, 256), cap));
    const unsigned entry_grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(num_edges, 256), cap)));
    GCU_LAUNCH(dev, "csr_check_offsets", csr_check_offsets_kernel, node_grid, 256, 0, d_offsets, num_nodes, num_edges,
               flags);
    GCU_LAUNCH(dev, "csr_mark_starts", csr_mark_starts_kernel, node_grid, 256, 0, d_offsets, num_nodes, flags,
               starts);
    if (!h_targets) {
        GCU_LAUNCH(dev, "csr_check_entries", csr_check_entries_kernel, entry_grid, 256, 0, d_offsets, d_targets,
                   num_nodes, starts, flags, uint64_t{0}, static_cast<uint64_t>(num_edges));
    } else if (num_edges > 0) {
        // The copy stream starts once the buffers above exist (they are
        // stream-ordered allocations of dev.stream); dev.stream then waits for
        // each chunk before checking it.
        GCU_CUDA(cudaEventRecord(dev.copy_event, dev.stream), "cudaEventRecord");
        GCU_CUDA(cudaStreamWaitEvent(dev.copy_stream, dev.copy_event, 0), "cudaStreamWaitEvent");
        Error err = ok();
        for (uint64_t c0 = 0; c0 < num_edges && err.ok(); c0 += kUploadChunk) {
            const uint64_t c1 = std::min<uint64_t>(c0 + kUploadChunk, num_edges);
            cudaError_t c = cudaMemcpyAsync(d_targets + c0, h_targets + c0, sizeof(uint32_t) * (c1 - c0),
                                            cudaMemcpyHostToDevice, dev.copy_stream);
            if (c == cudaSuccess) c = cudaEventRecord(dev.copy_event, dev.copy_stream);
            if (c == cudaSuccess) c = cudaStreamWaitEvent(dev.stream, dev.copy_event, 0);
            if (c != cudaSuccess) {
                err = driver_error(c, "copy CSR to device");
                break;
            }
            const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ceil_div_u64(c1 - c0, 256), cap)));
            err = [&]() -> Error {
                GCU_LAUNCH(dev, "csr_check_entries", csr_check_entries_kernel, grid, 256, 0, d_offsets, d_targets,
                           num_nodes, starts, flags, c0, c1);
                return ok();
            }();
        }
        if (!err.ok()) {
            cudaStreamSynchronize(dev.copy_stream);  // no copy may outlive the buffers
            return err;
        }
    }
    uint32_t host[4];
    GCU_CUDA(cudaMemcpyAsync(host, flags, sizeof(host), cudaMemcpyDeviceToHost, dev.stream), "copy flags");
    GCU_TRY(dev.sync());
    *first_bad_node = std::min(std::min(host[0], host[1]), host[2]);
    return ok();
}

Error validate_csr_device(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets,
                          uint32_t num_nodes, uint32_t num_edges, uint32_t* first_bad_node) {
    return check_csr(dev, d_offsets, const_cast<uint32_t*>(d_targets), nullptr, num_nodes, num_edges,
                     first_bad_node);
}

Error upload_and_validate_csr(DeviceImpl& dev, const uint32_t* d_offsets, uint32_t* d_targets,
                              const uint32_t* h_targets, uint32_t num_nodes, uint32_t num_edges,
                              uint32_t* first_bad_node) {
    return check_csr(dev, d_offsets, d_targets, h_targets, num_nodes, num_edges, first_bad_node);
}

// Symmetry test: every entry u -> v needs v -> u; each entry binary-searches
// u in the neighbour's list (entries taken in tiles, so hub lists are shared
// by many blocks).
__global__ void __launch_bounds__(256) csr_symmetry_kernel(const uint32_t* __restrict__ offsets,
                                                           const uint32_t* __restrict__ targets, uint32_t V,
                                                           uint32_t E, uint32_t* __restrict__ asymmetric) {
    bool bad = false;
    for_each_entry<256, 4>(offsets, V, E, [&](uint32_t j, uint32_t u) {
        const uint32_t v = targets[j];
        const uint32_t vs = offsets[v], ve = offsets[v + 1];
        const uint32_t p = lower_bound_u32(targets, vs, ve, u);
        if (p == ve || targets[p] != u) bad = true;
    });
    if (bad) atomicOr(asymmetric, 1u);
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
            unsigned blocks = static_cast<unsigned>(std::max<uint64_t>(
                1, std::min<uint64_t>(ceil_div_u64(g.num_edges, 1024), static_cast<uint64_t>(dev.sm_count) * 16)));
            GCU_LAUNCH(dev, "csr_symmetry", csr_symmetry_kernel, blocks, 256, 0, g.offsets.ptr, g.targets.ptr,
                       g.num_nodes, g.num_edges, flag.ptr);
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
