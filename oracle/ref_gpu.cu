// Reference GPU kernels driver — TEST INFRASTRUCTURE ONLY.
//
// Compiles grafeo-cuda's own CUDA kernels (crates/grafeo-cuda-algos/kernels/
// pagerank.cu, bfs.cu, triangle_counting.cu, k_truss.cu, included from where they lie in
// the reference checkout; REF_KERNELS is that directory) for sm_100a and runs
// them with the launch sequences of the reference's Rust drivers, restated
// here in C++ (the Rust host code cannot be built in this image):
//   pagerank    crates/grafeo-cuda-algos/src/pagerank.rs:46-199
//   bfs         crates/grafeo-cuda-algos/src/bfs.rs:42-131
//   triangles   crates/grafeo-cuda-algos/src/triangle_counting.rs:40-152
//   k-truss     crates/grafeo-cuda-algos/src/k_truss.rs:42-161
// It gives the tests a second oracle (the reference code itself) and the
// reference kernels' device time on the same B200. Built into oracle/_ref/ by
// `make -C oracle ref`; nothing in the library links it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_KERNELS/pagerank.cu)
#include REF_STR(REF_KERNELS/bfs.cu)
#include REF_STR(REF_KERNELS/triangle_counting.cu)
// k_truss.cu's device helper `binary_search` is file-local in the reference's
// own build (one module per kernel file); its namespace keeps it apart here.
namespace ref_kt_kernels {
#include REF_STR(REF_KERNELS/k_truss.cu)
}  // namespace ref_kt_kernels

namespace {

constexpr unsigned kThreads = 256;  // THREADS_PER_BLOCK, launch.rs:7

unsigned grid_for(unsigned items) { return (items + kThreads - 1) / kThreads; }

struct Csr {
    unsigned *offsets = nullptr, *targets = nullptr;
    ~Csr() {
        cudaFree(offsets);
        cudaFree(targets);
    }
};

int upload(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t nnz, Csr& c) {
    if (cudaMalloc(&c.offsets, 4ull * (n + 1)) != cudaSuccess) return 1;
    if (cudaMalloc(&c.targets, 4ull * (nnz ? nnz : 1)) != cudaSuccess) return 1;
    if (cudaMemcpy(c.offsets, offsets, 4ull * (n + 1), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    if (nnz && cudaMemcpy(c.targets, targets, 4ull * nnz, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    return 0;
}

struct Timer {
    cudaEvent_t a, b;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a);
    }
    double stop() {
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return ms;
    }
};

}  // namespace

extern "C" {

// pagerank.rs:46-199 (n > 0). Returns 0 on success.
int ref_pagerank(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t nnz, float damping,
                 uint32_t max_iterations, float tolerance, float* ranks, uint32_t* iterations, int* converged,
                 double* device_ms) {
    Csr c;
    if (n == 0 || upload(offsets, targets, n, nnz, c)) return 1;
    float *a = nullptr, *b = nullptr, *dangling = nullptr, *diff = nullptr;
    unsigned* deg = nullptr;
    cudaMalloc(&a, 4ull * n);
    cudaMalloc(&b, 4ull * n);
    cudaMalloc(&deg, 4ull * n);
    cudaMalloc(&dangling, 4);
    cudaMalloc(&diff, 4);
    std::vector<float> init(n, 1.0f / static_cast<float>(n));
    Timer t;
    cudaMemcpy(a, init.data(), 4ull * n, cudaMemcpyHostToDevice);
    cudaMemset(b, 0, 4ull * n);
    compute_out_degrees_kernel<<<grid_for(n), kThreads>>>(c.offsets, n, deg);
    *converged = 0;
    *iterations = 0;
    for (uint32_t it = 0; it < max_iterations; ++it) {
        cudaMemset(dangling, 0, 4);
        pagerank_dangling_sum_kernel<<<grid_for(n), kThreads, kThreads * 4>>>(a, deg, n, dangling);
        pagerank_iteration_kernel<<<grid_for(n), kThreads>>>(c.offsets, c.targets, a, b, deg, dangling, n, damping);
        *iterations += 1;
        cudaMemset(diff, 0, 4);
        pagerank_diff_kernel<<<grid_for(n), kThreads, kThreads * 4>>>(a, b, n, diff);
        cudaDeviceSynchronize();
        float h = 0.f;
        cudaMemcpy(&h, diff, 4, cudaMemcpyDeviceToHost);
        float* s = a;
        a = b;
        b = s;
        if (h < tolerance) {
            *converged = 1;
            break;
        }
    }
    cudaDeviceSynchronize();
    cudaMemcpy(ranks, a, 4ull * n, cudaMemcpyDeviceToHost);
    *device_ms = t.stop();
    const int err = cudaGetLastError() != cudaSuccess;
    cudaFree(a);
    cudaFree(b);
    cudaFree(deg);
    cudaFree(dangling);
    cudaFree(diff);
    return err;
}

// bfs.rs:42-131 (source < n). distances: n values.
int ref_bfs(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t nnz, uint32_t source,
            int32_t* distances, uint32_t* reachable, int32_t* max_depth, double* device_ms) {
    Csr c;
    if (source >= n || upload(offsets, targets, n, nnz, c)) return 1;
    int* dist = nullptr;
    unsigned *fa = nullptr, *fb = nullptr, *size = nullptr;
    cudaMalloc(&dist, 4ull * n);
    cudaMalloc(&fa, 4ull * n);
    cudaMalloc(&fb, 4ull * n);
    cudaMalloc(&size, 4);
    std::vector<int32_t> init(n, -1);
    init[source] = 0;
    Timer t;
    cudaMemcpy(dist, init.data(), 4ull * n, cudaMemcpyHostToDevice);
    cudaMemset(fa, 0, 4ull * n);
    cudaMemcpy(fa, &source, 4, cudaMemcpyHostToDevice);
    cudaMemset(fb, 0, 4ull * n);
    unsigned frontier = 1;
    int depth = 0;
    while (true) {
        const unsigned zero = 0;
        cudaMemcpy(size, &zero, 4, cudaMemcpyHostToDevice);
        bfs_expand_kernel<<<grid_for(frontier), kThreads>>>(c.offsets, c.targets, dist, fa, frontier, fb, size, depth);
        cudaDeviceSynchronize();
        cudaMemcpy(&frontier, size, 4, cudaMemcpyDeviceToHost);
        if (frontier == 0) break;
        depth += 1;
        unsigned* s = fa;
        fa = fb;
        fb = s;
    }
    cudaMemcpy(distances, dist, 4ull * n, cudaMemcpyDeviceToHost);
    *device_ms = t.stop();
    uint32_t r = 0;
    for (uint32_t v = 0; v < n; ++v) r += distances[v] >= 0;
    *reachable = r;
    *max_depth = depth;
    const int err = cudaGetLastError() != cudaSuccess;
    cudaFree(dist);
    cudaFree(fa);
    cudaFree(fb);
    cudaFree(size);
    return err;
}

// triangle_counting.rs:40-152 (the default, symmetric-CSR path). Refuses,
// like warp_per_item (launch.rs:27-35), more than 134,217,727 forward edges
// (returns 2).
int ref_triangle_count(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t nnz, uint64_t* total,
                       double* device_ms) {
    *total = 0;
    if (nnz == 0) return 0;
    Csr c;
    if (upload(offsets, targets, n, nnz, c)) return 1;
    unsigned *fwd = nullptr, *fwd_off = nullptr;
    unsigned long long* result = nullptr;
    cudaMalloc(&fwd, 4ull * n);
    cudaMalloc(&fwd_off, 4ull * (n + 1));
    cudaMalloc(&result, 8);
    cudaMemset(fwd, 0, 4ull * n);
    cudaMemset(fwd_off, 0, 4ull * (n + 1));
    Timer t;
    compute_forward_counts_kernel<<<grid_for(n), kThreads>>>(c.offsets, c.targets, n, fwd);
    prefix_sum_kernel<<<1, 1>>>(fwd, fwd_off, n);
    cudaDeviceSynchronize();
    std::vector<unsigned> host_off(static_cast<size_t>(n) + 1);
    cudaMemcpy(host_off.data(), fwd_off, 4ull * (n + 1), cudaMemcpyDeviceToHost);
    const unsigned forward = host_off[n];
    int rc = 0;
    if (forward > 0) {
        if (static_cast<uint64_t>(forward) * 32 > 0xFFFFFFFFull) {
            rc = 2;
        } else {
            const unsigned long long zero = 0;
            cudaMemcpy(result, &zero, 8, cudaMemcpyHostToDevice);
            const unsigned blocks = static_cast<unsigned>((static_cast<uint64_t>(forward) * 32 + kThreads - 1) / kThreads);
            triangle_count_edge_parallel_kernel<<<blocks, kThreads>>>(c.offsets, c.targets, fwd_off, n, forward,
                                                                     result);
            cudaDeviceSynchronize();
            unsigned long long h = 0;
            cudaMemcpy(&h, result, 8, cudaMemcpyDeviceToHost);
            *total = h;
        }
    }
    *device_ms = t.stop();
    if (cudaGetLastError() != cudaSuccess) rc = 1;
    cudaFree(fwd);
    cudaFree(fwd_off);
    cudaFree(result);
    return rc;
}

// k_truss.rs:42-161: per round, support recomputed over the alive entries
// (thread per node), then every alive entry below k - 2 removed (thread per
// entry); rounds until one removes nothing; edges u < v that survive, in CSR
// order. k < 3 returns 3 (the reference's Kernel error); out holds 2 values
// per surviving edge (at most nnz / 2 edges).
int ref_k_truss(const uint32_t* offsets, const uint32_t* targets, uint32_t n, uint32_t nnz, uint32_t k, uint32_t* out,
                uint64_t* num_out, uint32_t* iterations, double* device_ms) {
    *num_out = 0;
    *iterations = 0;
    *device_ms = 0.0;
    if (k < 3) return 3;
    if (nnz == 0) return 0;
    Csr c;
    if (upload(offsets, targets, n, nnz, c)) return 1;
    unsigned *support = nullptr, *removed_count = nullptr;
    unsigned char* removed = nullptr;
    cudaMalloc(&support, 4ull * nnz);
    cudaMalloc(&removed, nnz);
    cudaMalloc(&removed_count, 4);
    cudaMemset(removed, 0, nnz);
    const unsigned threshold = k - 2;
    Timer t;
    for (;;) {
        cudaMemset(support, 0, 4ull * nnz);
        ref_kt_kernels::edge_triangle_support_kernel<<<grid_for(n), kThreads>>>(c.offsets, c.targets, removed, n, support);
        cudaMemset(removed_count, 0, 4);
        ref_kt_kernels::edge_filter_kernel<<<grid_for(nnz), kThreads>>>(support, removed, nnz, threshold, removed_count);
        cudaDeviceSynchronize();
        *iterations += 1;
        unsigned h = 0;
        cudaMemcpy(&h, removed_count, 4, cudaMemcpyDeviceToHost);
        if (h == 0) break;
    }
    *device_ms = t.stop();
    std::vector<unsigned char> mask(nnz);
    cudaMemcpy(mask.data(), removed, nnz, cudaMemcpyDeviceToHost);
    const int err = cudaGetLastError() != cudaSuccess;
    uint64_t m = 0;
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t idx = offsets[u]; idx < offsets[u + 1]; ++idx)
            if (targets[idx] > u && !mask[idx]) {
                out[2 * m] = u;
                out[2 * m + 1] = targets[idx];
                ++m;
            }
    *num_out = m;
    cudaFree(support);
    cudaFree(removed);
    cudaFree(removed_count);
    return err;
}

}  // extern "C"
