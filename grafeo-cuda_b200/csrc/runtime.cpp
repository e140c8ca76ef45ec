// Host runtime: errors, devices, graphs, timing, and the C ABI entry points
// for them and for the algorithms.
//
// Mirrors crates/grafeo-cuda-core/src/{error.rs,device.rs,gpu_graph.rs} and the
// PyO3-facing algorithm calls in crates/grafeo-cuda-algos/src/*.rs. Every call
// runs on the device's own stream and synchronizes before returning, like the
// reference's default-stream calls (device.rs:38).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <sstream>
#include <thread>

#include "gcu_internal.h"

namespace gcu {

// ---------------------------------------------------------------- errors

static thread_local std::string t_last_error;

Error ok() { return Error{}; }
Error no_device() { return Error{GCU_ERR_NO_DEVICE, "no CUDA device found"}; }
Error driver_error(cudaError_t e, const char* what) {
    std::string msg = "CUDA driver error: ";
    if (what && *what) {
        msg += what;
        msg += ": ";
    }
    msg += cudaGetErrorName(e);
    msg += " (";
    msg += cudaGetErrorString(e);
    msg += ")";
    return Error{GCU_ERR_DRIVER, msg};
}
Error out_of_memory(size_t required, size_t available) {
    return Error{GCU_ERR_OUT_OF_MEMORY, "graph too large for GPU memory: " +
                                            std::to_string(required) + " bytes required, " +
                                            std::to_string(available) + " bytes available"};
}
Error kernel_error(const std::string& msg) { return Error{GCU_ERR_KERNEL, "kernel error: " + msg}; }
Error export_error(const std::string& msg) {
    return Error{GCU_ERR_EXPORT, "CSR export failed: " + msg};
}
Error invalid_csr(const std::string& msg) { return Error{GCU_ERR_INVALID_CSR, "invalid CSR: " + msg}; }

gcu_status fail(const Error& e) {
    t_last_error = e.message;
    return e.status;
}
gcu_status succeed() {
    t_last_error.clear();
    return GCU_OK;
}

// ---------------------------------------------------------------- device

DeviceImpl::~DeviceImpl() {
    cudaSetDevice(ordinal);
    if (schedule && stream) cudaFreeAsync(schedule, stream);
    if (stream) cudaStreamSynchronize(stream);
    collect_pending();
    for (auto e : event_pool) cudaEventDestroy(e);
    if (timer_start) cudaEventDestroy(timer_start);
    if (timer_stop) cudaEventDestroy(timer_stop);
    if (copy_stream) {
        cudaStreamSynchronize(copy_stream);
        cudaStreamDestroy(copy_stream);
    }
    if (copy_event) cudaEventDestroy(copy_event);
    for (int i = 0; i < 2; ++i) {
        if (stage[i]) cudaFreeHost(stage[i]);
        if (stage_ev[i]) cudaEventDestroy(stage_ev[i]);
    }
    if (stream) cudaStreamDestroy(stream);
}

namespace {
constexpr size_t kStageMin = size_t(4) << 20;
constexpr size_t kStageChunk = size_t(32) << 20;
constexpr unsigned kStageThreads = 4;

// memcpy split into contiguous parts over up to kStageThreads threads.
void parallel_copy(void* dst, const void* src, size_t bytes) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned parts = std::min<unsigned>(kStageThreads, hw);
    const size_t part = (bytes + parts - 1) / parts;
    std::vector<std::thread> workers;
    for (unsigned i = 1; i < parts; ++i) {
        const size_t off = std::min(bytes, i * part);
        const size_t len = std::min(part, bytes - off);
        if (len == 0) break;
        workers.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len); });
    }
    std::memcpy(dst, src, std::min(part, bytes));
    for (auto& w : workers) w.join();
}
}  // namespace

Error copy_to_host(DeviceImpl& dev, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return ok();
    if (bytes <= kStageMin) {
        GCU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, dev.stream), "copy to host");
        return dev.sync();
    }
    if (!dev.stage[0] || !dev.stage[1]) {
        GCU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, dev.stream), "copy to host");
        return dev.sync();
    }
    std::lock_guard<std::mutex> lock(dev.stage_mu);
    const size_t chunks = (bytes + kStageChunk - 1) / kStageChunk;
    auto issue = [&](size_t k) -> Error {
        const size_t off = k * kStageChunk;
        const size_t len = std::min(kStageChunk, bytes - off);
        GCU_CUDA(cudaMemcpyAsync(dev.stage[k & 1], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost,
                                 dev.stream),
                 "copy to host");
        GCU_CUDA(cudaEventRecord(dev.stage_ev[k & 1], dev.stream), "cudaEventRecord");
        return ok();
    };
    Error err = [&]() -> Error {
        GCU_TRY(issue(0));
        for (size_t k = 0; k < chunks; ++k) {
            if (k + 1 < chunks) GCU_TRY(issue(k + 1));  // buffer (k + 1) & 1 was emptied at step k - 1
            GCU_CUDA(cudaEventSynchronize(dev.stage_ev[k & 1]), "cudaEventSynchronize");
            const size_t off = k * kStageChunk;
            parallel_copy(static_cast<char*>(dst) + off, dev.stage[k & 1], std::min(kStageChunk, bytes - off));
        }
        return ok();
    }();
    if (!err.ok()) cudaStreamSynchronize(dev.stream);  // no copy into the staging buffers outlives the lock
    GCU_TRY(err);
    return dev.sync();
}

Error DeviceImpl::activate() const {
    GCU_CUDA(cudaSetDevice(ordinal), "cudaSetDevice");
    return ok();
}

Error DeviceImpl::sync() {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return kernel_error(std::string("synchronize failed: ") + cudaGetErrorString(e));
    collect_pending();
    return ok();
}

void DeviceImpl::before_launch(const char* name, cudaEvent_t* start) {
    (void)name;
    launches.fetch_add(1, std::memory_order_relaxed);
    *start = nullptr;
    if (!kernel_timing) return;
    cudaEvent_t e;
    if (!event_pool.empty()) {
        e = event_pool.back();
        event_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        return;
    }
    cudaEventRecord(e, stream);
    *start = e;
}

void DeviceImpl::after_launch(const char* name, cudaEvent_t start) {
    if (!kernel_timing || start == nullptr) return;
    cudaEvent_t e;
    if (!event_pool.empty()) {
        e = event_pool.back();
        event_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        event_pool.push_back(start);
        return;
    }
    cudaEventRecord(e, stream);
    pending.push_back(Pending{name, start, e});
    // Bound the number of outstanding events.
    if (pending.size() > 4096) {
        cudaStreamSynchronize(stream);
        collect_pending();
    }
}

void DeviceImpl::collect_pending() {
    if (pending.empty()) return;
    std::lock_guard<std::mutex> lock(stats_mu);
    for (auto& p : pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.stop) == cudaSuccess &&
            cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
            KernelStat& s = stats[p.name];
            s.launches += 1;
            s.total_ms += ms;
        }
        event_pool.push_back(p.start);
        event_pool.push_back(p.stop);
    }
    pending.clear();
}

Error device_alloc(DeviceImpl& dev, void** ptr, size_t bytes) {
    *ptr = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(ptr, bytes, dev.stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        *ptr = nullptr;
        return out_of_memory(bytes, free_b);
    }
    if (e != cudaSuccess) return driver_error(e, "cudaMallocAsync");
    return ok();
}

void device_free(DeviceImpl& dev, void* ptr) {
    if (ptr) cudaFreeAsync(ptr, dev.stream);
}

GraphImpl::~GraphImpl() {
    if (dev) {
        dev->activate();
        destroy_pagerank_plan(pr_plan);
        destroy_pagerank_plan(pr_plan_directed);
        destroy_bfs_work(bfs_work);
        destroy_kt_cache(kt_cache);
        kt_cache = nullptr;
        pr_plan = nullptr;
        pr_plan_directed = nullptr;
        bfs_work = nullptr;
        offsets.reset();
        targets.reset();
        cudaStreamSynchronize(dev->stream);
    }
}

static Error create_device(int ordinal, std::shared_ptr<DeviceImpl>* out) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || (e == cudaSuccess && count == 0)) {
        cudaGetLastError();
        return no_device();
    }
    if (e != cudaSuccess) return driver_error(e, "cudaGetDeviceCount");
    if (ordinal < 0 || ordinal >= count) {
        return driver_error(cudaErrorInvalidDevice, ("device ordinal " + std::to_string(ordinal)).c_str());
    }
    auto dev = std::make_shared<DeviceImpl>();
    dev->ordinal = ordinal;
    GCU_CUDA(cudaSetDevice(ordinal), "cudaSetDevice");
    cudaDeviceProp prop;
    GCU_CUDA(cudaGetDeviceProperties(&prop, ordinal), "cudaGetDeviceProperties");
    dev->name = prop.name;
    dev->total_memory = prop.totalGlobalMem;
    dev->sm_count = prop.multiProcessorCount;
    dev->l2_bytes = prop.l2CacheSize;
    dev->max_smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
    GCU_CUDA(cudaStreamCreateWithFlags(&dev->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    GCU_CUDA(cudaEventCreate(&dev->timer_start), "cudaEventCreate");
    GCU_CUDA(cudaEventCreate(&dev->timer_stop), "cudaEventCreate");
    GCU_CUDA(cudaStreamCreateWithFlags(&dev->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    GCU_CUDA(cudaEventCreateWithFlags(&dev->copy_event, cudaEventDisableTiming), "cudaEventCreate");
    // Keep freed stream-ordered allocations cached in the pool, so repeated
    // algorithm calls do not return memory to the driver between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ordinal) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    // The staging pair of copy_to_host, page-locked once here (about 70 ms for
    // 64 MB) rather than in the first call that copies a large result; without
    // it (no page-locked memory left) large copies go straight to the caller.
    for (int i = 0; i < 2; ++i) {
        if (cudaMallocHost(&dev->stage[i], kStageChunk) != cudaSuccess) {
            cudaGetLastError();
            dev->stage[i] = nullptr;
        }
        GCU_CUDA(cudaEventCreateWithFlags(&dev->stage_ev[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    *out = dev;
    return ok();
}

}  // namespace gcu

using namespace gcu;

struct gcu_device {
    std::shared_ptr<DeviceImpl> impl;
};
struct gcu_graph {
    std::unique_ptr<GraphImpl> impl;
};
struct gcu_edge_list {
    std::vector<uint32_t> data;
};
struct gcu_batch {
    BatchImpl* impl = nullptr;
    ~gcu_batch() { destroy_batch(impl); }
};

// ---------------------------------------------------------------- C ABI

extern "C" {

GCU_API const char* gcu_last_error(void) { return t_last_error.c_str(); }
GCU_API const char* gcu_version(void) { return "0.3.0+b200"; }

GCU_API int gcu_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count;
}

GCU_API gcu_status gcu_device_create(int ordinal, gcu_device** out) {
    if (!out) return fail(kernel_error("gcu_device_create: out is NULL"));
    *out = nullptr;
    std::shared_ptr<DeviceImpl> impl;
    Error e = create_device(ordinal, &impl);
    if (!e.ok()) return fail(e);
    *out = new gcu_device{impl};
    return succeed();
}

GCU_API void gcu_device_destroy(gcu_device* dev) { delete dev; }
GCU_API const char* gcu_device_name(const gcu_device* dev) { return dev ? dev->impl->name.c_str() : ""; }
GCU_API int gcu_device_ordinal(const gcu_device* dev) { return dev ? dev->impl->ordinal : -1; }
GCU_API uint64_t gcu_device_total_memory(const gcu_device* dev) { return dev ? dev->impl->total_memory : 0; }
GCU_API int gcu_device_sm_count(const gcu_device* dev) { return dev ? dev->impl->sm_count : 0; }
GCU_API void* gcu_device_stream(gcu_device* dev) { return dev ? static_cast<void*>(dev->impl->stream) : nullptr; }

GCU_API gcu_status gcu_device_synchronize(gcu_device* dev) {
    if (!dev) return fail(kernel_error("device is NULL"));
    Error e = dev->impl->activate();
    if (e.ok()) e = dev->impl->sync();
    return e.ok() ? succeed() : fail(e);
}

GCU_API gcu_status gcu_device_timer_start(gcu_device* dev) {
    if (!dev) return fail(kernel_error("device is NULL"));
    DeviceImpl& d = *dev->impl;
    Error e = d.activate();
    if (!e.ok()) return fail(e);
    cudaError_t c = cudaEventRecord(d.timer_start, d.stream);
    if (c != cudaSuccess) return fail(driver_error(c, "cudaEventRecord"));
    return succeed();
}

GCU_API gcu_status gcu_device_timer_stop(gcu_device* dev, float* ms) {
    if (!dev) return fail(kernel_error("device is NULL"));
    DeviceImpl& d = *dev->impl;
    Error e = d.activate();
    if (!e.ok()) return fail(e);
    cudaError_t c = cudaEventRecord(d.timer_stop, d.stream);
    if (c == cudaSuccess) c = cudaEventSynchronize(d.timer_stop);
    float t = 0.f;
    if (c == cudaSuccess) c = cudaEventElapsedTime(&t, d.timer_start, d.timer_stop);
    if (c != cudaSuccess) return fail(driver_error(c, "event timing"));
    if (ms) *ms = t;
    return succeed();
}

GCU_API uint64_t gcu_device_launch_count(const gcu_device* dev) {
    return dev ? dev->impl->launches.load() : 0;
}

GCU_API void gcu_device_set_kernel_timing(gcu_device* dev, int on) {
    if (!dev) return;
    dev->impl->activate();
    cudaStreamSynchronize(dev->impl->stream);
    dev->impl->collect_pending();
    dev->impl->kernel_timing = on != 0;
}

GCU_API void gcu_device_set_bfs_device_loop(gcu_device* dev, int on) {
    if (!dev) return;
    dev->impl->bfs_device_loop = on != 0;
}

GCU_API size_t gcu_device_kernel_stats(gcu_device* dev, char* buf, size_t buflen) {
    if (!dev) return 0;
    DeviceImpl& d = *dev->impl;
    d.activate();
    cudaStreamSynchronize(d.stream);
    d.collect_pending();
    std::ostringstream os;
    os.precision(9);
    os << "{";
    {
        std::lock_guard<std::mutex> lock(d.stats_mu);
        bool first = true;
        for (auto& kv : d.stats) {
            if (!first) os << ", ";
            first = false;
            os << "\"" << kv.first << "\": [" << kv.second.launches << ", " << kv.second.total_ms << "]";
        }
    }
    os << "}";
    std::string s = os.str();
    if (buf && buflen) {
        size_t n = std::min(buflen - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size() + 1;
}

GCU_API void gcu_device_reset_stats(gcu_device* dev) {
    if (!dev) return;
    DeviceImpl& d = *dev->impl;
    d.activate();
    cudaStreamSynchronize(d.stream);
    d.collect_pending();
    std::lock_guard<std::mutex> lock(d.stats_mu);
    d.stats.clear();
    d.launches.store(0);
}

GCU_API gcu_status gcu_graph_from_csr(gcu_device* dev, const uint32_t* offsets, size_t n_offsets,
                                      const uint32_t* targets, size_t n_targets, gcu_graph** out) {
    if (!out) return fail(kernel_error("gcu_graph_from_csr: out is NULL"));
    *out = nullptr;
    if (!dev) return fail(kernel_error("device is NULL"));
    // Shape checks need only a few host reads; the per-entry rules run on the
    // device after the copy (csr_export.rs:71-96 for the order of the checks).
    if (n_offsets == 0) {
        return fail(invalid_csr("offsets must have num_nodes + 1 entries, got an empty array"));
    }
    if (n_offsets > 0xFFFFFFFFull || n_targets > 0xFFFFFFFFull) {
        return fail(invalid_csr("graph too large for u32 indices: " + std::to_string(n_offsets) +
                                " offsets, " + std::to_string(n_targets) + " targets"));
    }
    if (!offsets || (n_targets > 0 && !targets)) return fail(kernel_error("CSR pointer is NULL"));
    if (offsets[0] != 0) {
        return fail(invalid_csr("offsets[0] must be 0, got " + std::to_string(offsets[0])));
    }
    const size_t num_nodes = n_offsets - 1;
    if (static_cast<size_t>(offsets[num_nodes]) != n_targets) {
        return fail(invalid_csr("offsets[" + std::to_string(num_nodes) + "] is " +
                                std::to_string(offsets[num_nodes]) + " but targets has " +
                                std::to_string(n_targets) + " entries"));
    }

    auto g = std::make_unique<GraphImpl>();
    g->dev = dev->impl;
    DeviceImpl& d = *g->dev;
    Error e = d.activate();
    if (!e.ok()) return fail(e);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        size_t required = n_offsets * 4 + n_targets * 4;
        if (required > free_b) return fail(out_of_memory(required, free_b));
    }
    g->num_nodes = static_cast<uint32_t>(num_nodes);
    g->num_edges = static_cast<uint32_t>(n_targets);
    e = g->offsets.allocate(d, n_offsets);
    if (e.ok()) e = g->targets.allocate(d, n_targets);
    if (!e.ok()) return fail(e);
    cudaError_t c = cudaMemcpyAsync(g->offsets.ptr, offsets, n_offsets * 4, cudaMemcpyHostToDevice, d.stream);
    if (c != cudaSuccess) return fail(driver_error(c, "copy CSR to device"));

    // The targets are copied in chunks that the entry checks follow.
    uint32_t bad = UINT32_MAX;
    e = upload_and_validate_csr(d, g->offsets.ptr, g->targets.ptr, targets, g->num_nodes, g->num_edges, &bad);
    if (!e.ok()) return fail(e);
    if (bad != UINT32_MAX) {
        // Reproduce the exact reference message for that node on the host.
        uint32_t start = offsets[bad], end = offsets[bad + 1];
        size_t lo = std::min<size_t>(start, n_targets), hi = std::min<size_t>(std::max(start, end), n_targets);
        std::string msg = describe_node_violation(bad, start, end, targets + lo, hi - lo, g->num_nodes);
        return fail(invalid_csr(msg));
    }
    *out = new gcu_graph{std::move(g)};
    return succeed();
}

GCU_API uint32_t gcu_graph_num_nodes(const gcu_graph* g) { return g ? g->impl->num_nodes : 0; }
GCU_API uint32_t gcu_graph_num_edges(const gcu_graph* g) { return g ? g->impl->num_edges : 0; }
GCU_API void gcu_graph_destroy(gcu_graph* g) { delete g; }

GCU_API gcu_status gcu_graph_copy_csr(const gcu_graph* g, uint32_t* offsets, uint32_t* targets) {
    if (!g || !offsets || (g->impl->num_edges && !targets)) return fail(kernel_error("gcu_graph_copy_csr: NULL argument"));
    GraphImpl& gi = *g->impl;
    DeviceImpl& d = *gi.dev;
    Error e = d.activate();
    if (!e.ok()) return fail(e);
    e = copy_to_host(d, offsets, gi.offsets.ptr, 4 * (static_cast<size_t>(gi.num_nodes) + 1));
    if (e.ok() && gi.num_edges) e = copy_to_host(d, targets, gi.targets.ptr, 4 * static_cast<size_t>(gi.num_edges));
    return e.ok() ? succeed() : fail(e);
}

}  // extern "C"

namespace {

// Runs a device CSR build into a new graph handle.
template <typename Build>
gcu_status new_device_graph(gcu_device* dev, gcu_graph** out, Build&& build) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    if (!dev) return fail(kernel_error("device is NULL"));
    auto g = std::make_unique<GraphImpl>();
    g->dev = dev->impl;
    Error e = g->dev->activate();
    if (e.ok()) e = build(*g->dev, *g);
    if (!e.ok()) return fail(e);
    *out = new gcu_graph{std::move(g)};
    return succeed();
}

}  // namespace

extern "C" {

GCU_API gcu_status gcu_graph_from_edge_pairs(gcu_device* dev, const uint32_t* pairs, size_t n_pairs,
                                             uint32_t num_nodes, int symmetric, gcu_graph** out) {
    if (n_pairs && !pairs) return fail(kernel_error("pairs is NULL"));
    return new_device_graph(dev, out, [&](DeviceImpl& d, GraphImpl& g) {
        return build_graph_from_pairs(d, pairs, n_pairs, num_nodes, symmetric ? 1 : 0, g);
    });
}

GCU_API gcu_status gcu_graph_from_edge_pairs_oriented(gcu_device* dev, const uint32_t* pairs, size_t n_pairs,
                                                      uint32_t num_nodes, gcu_graph** out) {
    if (n_pairs && !pairs) return fail(kernel_error("pairs is NULL"));
    return new_device_graph(dev, out, [&](DeviceImpl& d, GraphImpl& g) {
        return build_graph_from_pairs(d, pairs, n_pairs, num_nodes, 2, g);
    });
}

static gcu_status generate(gcu_device* dev, const GeneratorSpec& spec, gcu_graph** out) {
    return new_device_graph(dev, out, [&](DeviceImpl& d, GraphImpl& g) { return generate_graph(d, spec, g); });
}

GCU_API gcu_status gcu_graph_generate_rmat(gcu_device* dev, uint32_t scale, uint32_t edge_factor, double a, double b,
                                           double c, uint64_t seed, gcu_graph** out) {
    GeneratorSpec s;
    s.kind = GeneratorSpec::kRmat;
    s.scale = scale;
    s.edge_factor = edge_factor;
    s.a = a;
    s.b = b;
    s.c = c;
    s.seed = seed;
    return generate(dev, s, out);
}

GCU_API gcu_status gcu_graph_generate_erdos_renyi(gcu_device* dev, uint32_t num_nodes, uint64_t num_pairs,
                                                  uint64_t seed, gcu_graph** out) {
    GeneratorSpec s;
    s.kind = GeneratorSpec::kErdosRenyi;
    s.n = num_nodes;
    s.pairs = num_pairs;
    s.seed = seed;
    return generate(dev, s, out);
}

GCU_API gcu_status gcu_graph_generate_grid(gcu_device* dev, uint32_t width, uint32_t height, double drop,
                                           uint64_t seed, gcu_graph** out) {
    GeneratorSpec s;
    s.kind = GeneratorSpec::kGrid;
    s.width = width;
    s.height = height;
    s.p = drop;
    s.seed = seed;
    return generate(dev, s, out);
}

GCU_API gcu_status gcu_graph_generate_watts_strogatz(gcu_device* dev, uint32_t num_nodes, uint32_t k, double p,
                                                     uint64_t seed, gcu_graph** out) {
    GeneratorSpec s;
    s.kind = GeneratorSpec::kWattsStrogatz;
    s.n = num_nodes;
    s.k = k;
    s.p = p;
    s.seed = seed;
    return generate(dev, s, out);
}

GCU_API gcu_status gcu_graph_generate_geometric(gcu_device* dev, uint32_t num_nodes, double avg_degree, uint64_t seed,
                                                gcu_graph** out) {
    GeneratorSpec s;
    s.kind = GeneratorSpec::kGeometric;
    s.n = num_nodes;
    s.avg_degree = avg_degree;
    s.seed = seed;
    return generate(dev, s, out);
}

GCU_API gcu_status gcu_triangle_count(gcu_graph* g, uint64_t* total, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    std::lock_guard<std::mutex> lock(g->impl->mu);
    Error e = g->impl->dev->activate();
    uint64_t t = 0;
    if (e.ok()) e = triangle_count(*g->impl, false, &t);
    if (!e.ok()) return fail(e);
    if (total) *total = t;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_triangle_count_oriented(gcu_graph* g, uint64_t* total, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    std::lock_guard<std::mutex> lock(g->impl->mu);
    Error e = g->impl->dev->activate();
    uint64_t t = 0;
    if (e.ok()) e = triangle_count(*g->impl, true, &t);
    if (!e.ok()) return fail(e);
    if (total) *total = t;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_bfs(gcu_graph* g, uint32_t source, int32_t* distances, uint32_t* reachable,
                           int32_t* max_depth, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    GraphImpl& gi = *g->impl;
    // bfs.rs:46-51
    if (source >= gi.num_nodes) {
        return fail(kernel_error("source node " + std::to_string(source) +
                                 " out of range (num_nodes = " + std::to_string(gi.num_nodes) + ")"));
    }
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    uint32_t r = 0;
    int32_t depth = 0;
    if (e.ok()) e = bfs(gi, source, distances, &r, &depth);
    if (!e.ok()) return fail(e);
    if (reachable) *reachable = r;
    if (max_depth) *max_depth = depth;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_pagerank(gcu_graph* g, float damping, uint32_t max_iterations, float tolerance,
                                float* ranks, uint32_t* iterations, int* converged, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    uint32_t it = 0;
    bool conv = false;
    if (e.ok()) e = pagerank(gi, damping, max_iterations, tolerance, ranks, &it, &conv);
    if (!e.ok()) return fail(e);
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_pagerank_directed(gcu_graph* g, float damping, uint32_t max_iterations, float tolerance,
                                         float* ranks, uint32_t* iterations, int* converged, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    uint32_t it = 0;
    bool conv = false;
    if (e.ok()) e = pagerank_ex(gi, true, nullptr, damping, max_iterations, tolerance, ranks, &it, &conv);
    if (!e.ok()) return fail(e);
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_pagerank_gather_probe(gcu_graph* g, int directed, uint32_t passes, double* ms_per_pass) {
    if (!g || !ms_per_pass) return fail(kernel_error("graph or result pointer is NULL"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    if (e.ok()) e = pagerank_gather_probe(gi, directed != 0, passes, ms_per_pass);
    if (!e.ok()) return fail(e);
    return succeed();
}

GCU_API gcu_status gcu_personalized_pagerank(gcu_graph* g, const uint32_t* seeds, size_t n_seeds, int directed,
                                             float damping, uint32_t max_iterations, float tolerance, float* ranks,
                                             uint32_t* iterations, int* converged, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    GraphImpl& gi = *g->impl;
    if (n_seeds == 0 || !seeds) return fail(kernel_error("personalized PageRank needs at least one seed"));
    std::vector<float> tele(gi.num_nodes, 0.f);
    for (size_t i = 0; i < n_seeds; ++i) {
        if (seeds[i] >= gi.num_nodes) {
            return fail(kernel_error("seed node " + std::to_string(seeds[i]) + " out of range (num_nodes = " +
                                     std::to_string(gi.num_nodes) + ")"));
        }
        tele[seeds[i]] += static_cast<float>(1.0 / static_cast<double>(n_seeds));
    }
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    uint32_t it = 0;
    bool conv = false;
    if (e.ok())
        e = pagerank_ex(gi, directed != 0, tele.data(), damping, max_iterations, tolerance, ranks, &it, &conv);
    if (!e.ok()) return fail(e);
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

GCU_API gcu_status gcu_k_truss(gcu_graph* g, uint32_t k, gcu_edge_list** edges, uint32_t* iterations,
                               double* seconds) {
    WallTimer wall;
    if (edges) *edges = nullptr;
    if (!g) return fail(kernel_error("graph is NULL"));
    // k_truss.rs:43-47
    if (k < 3) return fail(kernel_error("k must be >= 3 for k-truss decomposition"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    auto list = std::make_unique<gcu_edge_list>();
    uint32_t it = 0;
    if (e.ok()) e = k_truss(gi, k, &list->data, &it);
    if (!e.ok()) return fail(e);
    if (iterations) *iterations = it;
    if (seconds) *seconds = wall.seconds();
    if (edges) *edges = list.release();
    return succeed();
}

GCU_API gcu_status gcu_truss_decomposition(gcu_graph* g, uint32_t* trussness, uint32_t* max_trussness,
                                           uint32_t* rounds, double* seconds) {
    WallTimer wall;
    if (!g) return fail(kernel_error("graph is NULL"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    uint32_t top = 0, r = 0;
    if (e.ok()) e = truss_decomposition(gi, trussness, &top, &r);
    if (!e.ok()) return fail(e);
    if (max_trussness) *max_trussness = top;
    if (rounds) *rounds = r;
    if (seconds) *seconds = wall.seconds();
    return succeed();
}

static gcu_status on_device(gcu_device* dev, const std::function<Error(DeviceImpl&)>& body) {
    if (!dev) return fail(kernel_error("device is NULL"));
    DeviceImpl& d = *dev->impl;
    Error e = d.activate();
    if (e.ok()) e = body(d);
    return e.ok() ? succeed() : fail(e);
}

GCU_API gcu_status gcu_device_set_schedule(gcu_device* dev, const uint16_t* weights) {
    return on_device(dev, [&](DeviceImpl& d) { return set_schedule(d, weights); });
}

GCU_API gcu_status gcu_schedule_forward(gcu_device* dev, const uint16_t* weights, const float* features, size_t n,
                                        float* out) {
    if (!weights || (n && (!features || !out))) return fail(kernel_error("gcu_schedule_forward: NULL argument"));
    return on_device(dev, [&](DeviceImpl& d) { return sched_forward(d, weights, features, n, out); });
}

GCU_API gcu_status gcu_schedule_gradient(gcu_device* dev, const uint16_t* weights, const float* features,
                                         const float* targets, const uint8_t* mask, size_t n, double* loss,
                                         float* grad) {
    if (!weights || !loss || !grad || (n && (!features || !targets || !mask)))
        return fail(kernel_error("gcu_schedule_gradient: NULL argument"));
    return on_device(dev, [&](DeviceImpl& d) { return sched_gradient(d, weights, features, targets, mask, n, loss, grad); });
}

GCU_API gcu_status gcu_schedule_train(gcu_device* dev, float* master, uint16_t* weights, const float* features,
                                      const float* targets, const uint8_t* mask, size_t n, uint32_t steps,
                                      uint32_t batch, float lr, uint64_t seed, double* final_loss) {
    if (!master || !weights || !final_loss || (n && (!features || !targets || !mask)))
        return fail(kernel_error("gcu_schedule_train: NULL argument"));
    return on_device(dev, [&](DeviceImpl& d) {
        return sched_train(d, master, weights, features, targets, mask, n, steps, batch, lr, seed, final_loss);
    });
}

GCU_API gcu_status gcu_bfs_trace(gcu_graph* g, uint32_t source, uint64_t explore_seed, float* features,
                                 float* times_us, uint8_t* valid, uint8_t* fixed_rule, uint8_t* taken,
                                 size_t capacity, size_t* levels) {
    if (!g || !levels) return fail(kernel_error("gcu_bfs_trace: NULL argument"));
    if (capacity && (!features || !times_us || !valid || !fixed_rule || !taken))
        return fail(kernel_error("gcu_bfs_trace: NULL output array"));
    GraphImpl& gi = *g->impl;
    if (source >= gi.num_nodes)
        return fail(kernel_error("source node " + std::to_string(source) + " out of range (num_nodes = " +
                                 std::to_string(gi.num_nodes) + ")"));
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    std::vector<BfsTraceLevel> rec;
    if (e.ok()) e = bfs_trace(gi, source, explore_seed, &rec);
    if (!e.ok()) return fail(e);
    for (size_t i = 0; i < std::min(capacity, rec.size()); ++i) {
        std::memcpy(features + 12 * i, rec[i].features, sizeof(rec[i].features));
        std::memcpy(times_us + 3 * i, rec[i].times_us, sizeof(rec[i].times_us));
        valid[i] = rec[i].valid;
        fixed_rule[i] = rec[i].fixed_rule;
        taken[i] = rec[i].taken;
    }
    *levels = rec.size();
    return succeed();
}

GCU_API gcu_status gcu_triangle_trace(gcu_graph* g, float* features, float* times_us, uint8_t* valid,
                                      uint8_t* fixed_rule, size_t capacity, size_t* buckets, uint64_t* total) {
    if (!g || !buckets || !total) return fail(kernel_error("gcu_triangle_trace: NULL argument"));
    if (capacity && (!features || !times_us || !valid || !fixed_rule))
        return fail(kernel_error("gcu_triangle_trace: NULL output array"));
    GraphImpl& gi = *g->impl;
    std::lock_guard<std::mutex> lock(gi.mu);
    Error e = gi.dev->activate();
    std::vector<TcTraceBucket> rec;
    uint64_t t = 0;
    if (e.ok()) e = triangle_trace(gi, &rec, &t);
    if (!e.ok()) return fail(e);
    for (size_t i = 0; i < std::min(capacity, rec.size()); ++i) {
        std::memcpy(features + 12 * i, rec[i].features, sizeof(rec[i].features));
        std::memcpy(times_us + 3 * i, rec[i].times_us, sizeof(rec[i].times_us));
        valid[i] = rec[i].valid;
        fixed_rule[i] = rec[i].fixed_rule;
    }
    *buckets = rec.size();
    *total = t;
    return succeed();
}

// ---------------------------------------------------------------- batch

static gcu_status on_batch(gcu_batch* b, const std::function<Error(BatchImpl&)>& body) {
    if (!b || !b->impl) return fail(kernel_error("batch is NULL"));
    Error e = batch_union(*b->impl).dev->activate();
    if (e.ok()) e = body(*b->impl);
    return e.ok() ? succeed() : fail(e);
}

GCU_API gcu_status gcu_batch_generate(gcu_device* dev, uint32_t num_graphs, uint64_t seed, gcu_batch** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    return on_device(dev, [&](DeviceImpl& d) {
        BatchImpl* impl = nullptr;
        GCU_TRY(batch_generate(d, dev->impl, num_graphs, seed, &impl));
        *out = new gcu_batch{impl};
        return ok();
    });
}

GCU_API gcu_status gcu_batch_from_csr(gcu_device* dev, const uint32_t* vertex_base, size_t num_graphs,
                                      const uint32_t* offsets, size_t n_offsets, const uint32_t* targets,
                                      size_t n_targets, gcu_batch** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    if (!vertex_base || !offsets || (n_targets && !targets)) return fail(kernel_error("batch CSR pointer is NULL"));
    if (n_offsets > 0xFFFFFFFFull || n_targets > 0xFFFFFFFFull)
        return fail(invalid_csr("graph too large for u32 indices: " + std::to_string(n_offsets) + " offsets, " +
                                std::to_string(n_targets) + " targets"));
    return on_device(dev, [&](DeviceImpl& d) {
        BatchImpl* impl = nullptr;
        GCU_TRY(batch_from_csr(d, dev->impl, vertex_base, num_graphs, offsets, n_offsets, targets, n_targets, &impl));
        *out = new gcu_batch{impl};
        return ok();
    });
}

GCU_API void gcu_batch_destroy(gcu_batch* b) { delete b; }
GCU_API uint32_t gcu_batch_num_graphs(const gcu_batch* b) { return b && b->impl ? batch_num_graphs(*b->impl) : 0; }
GCU_API uint32_t gcu_batch_num_nodes(const gcu_batch* b) {
    return b && b->impl ? batch_union(*b->impl).num_nodes : 0;
}
GCU_API uint32_t gcu_batch_num_edges(const gcu_batch* b) {
    return b && b->impl ? batch_union(*b->impl).num_edges : 0;
}

GCU_API gcu_status gcu_batch_vertex_base(const gcu_batch* b, uint32_t* vertex_base) {
    if (!b || !b->impl || !vertex_base) return fail(kernel_error("gcu_batch_vertex_base: NULL argument"));
    const auto& v = batch_vertex_base(*b->impl);
    std::copy(v.begin(), v.end(), vertex_base);
    return succeed();
}

GCU_API gcu_status gcu_batch_copy_csr(const gcu_batch* b, uint32_t* offsets, uint32_t* targets) {
    if (!b || !b->impl) return fail(kernel_error("batch is NULL"));
    GraphImpl& u = batch_union(*b->impl);
    if (!offsets || (u.num_edges && !targets)) return fail(kernel_error("gcu_batch_copy_csr: NULL argument"));
    DeviceImpl& d = *u.dev;
    Error e = d.activate();
    if (!e.ok()) return fail(e);
    cudaError_t c = cudaMemcpyAsync(offsets, u.offsets.ptr, 4 * (static_cast<size_t>(u.num_nodes) + 1),
                                    cudaMemcpyDeviceToHost, d.stream);
    if (c == cudaSuccess && u.num_edges)
        c = cudaMemcpyAsync(targets, u.targets.ptr, 4 * static_cast<size_t>(u.num_edges), cudaMemcpyDeviceToHost,
                            d.stream);
    if (c != cudaSuccess) return fail(driver_error(c, "copy CSR to host"));
    e = d.sync();
    return e.ok() ? succeed() : fail(e);
}

GCU_API gcu_status gcu_batch_member(gcu_batch* b, uint32_t index, gcu_graph** out) {
    if (!out) return fail(kernel_error("out is NULL"));
    *out = nullptr;
    return on_batch(b, [&](BatchImpl& bi) {
        auto g = std::make_unique<GraphImpl>();
        g->dev = batch_union(bi).dev;
        GCU_TRY(batch_member(bi, index, *g));
        *out = new gcu_graph{std::move(g)};
        return ok();
    });
}

GCU_API gcu_status gcu_batch_triangle_count(gcu_batch* b, uint64_t* totals, double* seconds) {
    WallTimer wall;
    if (!totals) return fail(kernel_error("totals is NULL"));
    gcu_status s = on_batch(b, [&](BatchImpl& bi) { return batch_run_tc(bi, totals); });
    if (s == GCU_OK && seconds) *seconds = wall.seconds();
    return s;
}

GCU_API gcu_status gcu_batch_set_bfs_sources(gcu_batch* b, const uint32_t* sources, uint32_t S, int keep_distances) {
    if (!sources) return fail(kernel_error("sources is NULL"));
    return on_batch(b, [&](BatchImpl& bi) { return batch_set_bfs(bi, sources, S, keep_distances != 0); });
}

GCU_API gcu_status gcu_batch_bfs(gcu_batch* b, int32_t* distances, uint32_t* reachable, int32_t* max_depth,
                                 double* seconds) {
    WallTimer wall;
    gcu_status s = on_batch(b, [&](BatchImpl& bi) {
        GCU_TRY(batch_run_bfs(bi));
        return batch_read_bfs(bi, distances, reachable, max_depth);
    });
    if (s == GCU_OK && seconds) *seconds = wall.seconds();
    return s;
}

GCU_API gcu_status gcu_batch_set_pagerank_seeds(gcu_batch* b, const uint32_t* seeds, uint32_t K, float damping,
                                                uint32_t max_iterations, float tolerance) {
    if (!seeds) return fail(kernel_error("seeds is NULL"));
    return on_batch(b,
                    [&](BatchImpl& bi) { return batch_set_ppr(bi, seeds, K, damping, max_iterations, tolerance); });
}

GCU_API gcu_status gcu_batch_personalized_pagerank(gcu_batch* b, float* ranks, uint32_t* iterations,
                                                   uint8_t* converged, double* seconds) {
    WallTimer wall;
    gcu_status s = on_batch(b, [&](BatchImpl& bi) {
        GCU_TRY(batch_run_ppr(bi));
        return batch_read_ppr(bi, ranks, iterations, converged);
    });
    if (s == GCU_OK && seconds) *seconds = wall.seconds();
    return s;
}

GCU_API gcu_status gcu_batch_capture(gcu_batch* b) {
    return on_batch(b, [&](BatchImpl& bi) { return batch_capture(bi); });
}

GCU_API gcu_status gcu_batch_replay(gcu_batch* b) {
    return on_batch(b, [&](BatchImpl& bi) { return batch_replay(bi); });
}

GCU_API gcu_status gcu_batch_results(gcu_batch* b, uint64_t* triangles, int32_t* distances, uint32_t* reachable,
                                     int32_t* max_depth, float* ranks, uint32_t* iterations, uint8_t* converged) {
    return on_batch(b, [&](BatchImpl& bi) {
        GCU_TRY(batch_union(bi).dev->sync());
        if (triangles) GCU_TRY(batch_read_tc(bi, triangles));
        GCU_TRY(batch_read_bfs(bi, distances, reachable, max_depth));
        return batch_read_ppr(bi, ranks, iterations, converged);
    });
}

GCU_API size_t gcu_batch_tuning(const gcu_batch* b, char* buf, size_t buflen) {
    if (!b || !b->impl) return 0;
    const std::string s = batch_tuning(*b->impl);
    if (buf && buflen) {
        const size_t n = std::min(buflen - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return s.size() + 1;
}

GCU_API size_t gcu_edge_list_len(const gcu_edge_list* list) { return list ? list->data.size() / 2 : 0; }
GCU_API const uint32_t* gcu_edge_list_data(const gcu_edge_list* list) {
    return list && !list->data.empty() ? list->data.data() : nullptr;
}
GCU_API void gcu_edge_list_free(gcu_edge_list* list) { delete list; }

}  // extern "C"
