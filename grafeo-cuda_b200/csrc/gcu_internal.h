// Internal declarations shared by the host runtime and the kernel files.
//
// Layout of a graph in HBM (one allocation each, 256-byte aligned, padded to a
// multiple of 16 bytes plus 16 so that 16-byte vector and bulk loads of the
// last partial chunk stay inside the allocation):
//   offsets  u32[V + 1]   CSR row pointers   (GpuGraph::offsets, gpu_graph.rs:17)
//   targets  u32[E]       sorted neighbours  (GpuGraph::targets, gpu_graph.rs:19)
// Derived per-algorithm state (PageRank tile plan, BFS work buffers, ...) is
// built lazily on first use and cached on the graph, like the reference caches
// its kernel modules per context (module_cache.rs:23-87).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/grafeo_cuda.h"

namespace gcu {

// ---------------------------------------------------------------- errors

// Error value carried through the host code; converted to gcu_status plus the
// thread-local message at the C boundary.
struct Error {
    gcu_status status = GCU_OK;
    std::string message;
    bool ok() const { return status == GCU_OK; }
};

Error ok();
Error no_device();
Error driver_error(cudaError_t e, const char* what);
Error out_of_memory(size_t required, size_t available);
Error kernel_error(const std::string& msg);
Error export_error(const std::string& msg);
Error invalid_csr(const std::string& msg);

// Records `e` as this thread's last error and returns its status.
gcu_status fail(const Error& e);
gcu_status succeed();

#define GCU_TRY(expr)                       \
    do {                                    \
        ::gcu::Error _e = (expr);           \
        if (!_e.ok()) return _e;            \
    } while (0)

#define GCU_CUDA(call, what)                                          \
    do {                                                              \
        cudaError_t _c = (call);                                      \
        if (_c != cudaSuccess) return ::gcu::driver_error(_c, what);  \
    } while (0)

// ---------------------------------------------------------------- timing

class WallTimer {
  public:
    WallTimer() : t0_(std::chrono::steady_clock::now()) {}
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }

  private:
    std::chrono::steady_clock::time_point t0_;
};

// ---------------------------------------------------------------- device

struct KernelStat {
    uint64_t launches = 0;
    double total_ms = 0.0;
};

struct DeviceImpl {
    int ordinal = 0;
    std::string name;
    uint64_t total_memory = 0;
    int sm_count = 0;
    int l2_bytes = 0;
    int max_smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t timer_start = nullptr;
    cudaEvent_t timer_stop = nullptr;
    cudaStream_t copy_stream = nullptr;  // chunked host-to-device copies that overlap the checks
    cudaEvent_t copy_event = nullptr;

    std::atomic<uint64_t> launches{0};
    bool kernel_timing = false;
    // BFS runs its level loop on the device (one CUDA graph per search)
    // unless this is off or per-kernel timing is on.
    bool bfs_device_loop = true;
    std::mutex stats_mu;
    std::map<std::string, KernelStat> stats;
    struct Pending {
        const char* name;
        cudaEvent_t start, stop;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;

    // Installed learned-schedule network (BF16 bit patterns, device copy);
    // NULL: the fixed rules (alpha/beta BFS direction, degree-range buckets).
    uint16_t* schedule = nullptr;

    // Two page-locked staging buffers for large device-to-host copies into
    // pageable memory (copy_to_host), allocated with the device (NULL if
    // page-locked memory ran out: those copies then go straight to the caller).
    std::mutex stage_mu;
    void* stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};

    ~DeviceImpl();

    // Makes this device current on the calling thread.
    Error activate() const;
    // Synchronizes the stream and folds pending per-kernel timings into stats.
    Error sync();
    // Called around each kernel launch by GCU_LAUNCH.
    void before_launch(const char* name, cudaEvent_t* start);
    void after_launch(const char* name, cudaEvent_t start);
    void collect_pending();
};

// Copies `bytes` of device memory to pageable host memory and waits for it.
// Up to kStageMin bytes: one copy. Beyond: chunks of kStageChunk bytes go
// through two page-locked staging buffers, the DMA of the next chunk
// overlapping the host copy of the current one, which is split over up to
// kStageThreads threads. Measured on the B200 box: 67 MB in 5.1 ms against
// 13.5 ms for the driver's pageable copy (2.7x), 396 MB of batch ranks in
// about a third of the time; one host thread instead of four gained 7 %.
Error copy_to_host(DeviceImpl& dev, void* dst, const void* src, size_t bytes);

// Stream-ordered device allocation that reports OutOfMemory with the
// reference's required/available fields (error.rs:18-26).
Error device_alloc(DeviceImpl& dev, void** ptr, size_t bytes);
void device_free(DeviceImpl& dev, void* ptr);

// Owning device buffer, freed on the device stream.
template <typename T>
struct DeviceBuffer {
    DeviceImpl* dev = nullptr;
    T* ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept { *this = std::move(o); }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        reset();
        dev = o.dev; ptr = o.ptr; count = o.count;
        o.ptr = nullptr; o.count = 0;
        return *this;
    }
    ~DeviceBuffer() { reset(); }
    Error allocate(DeviceImpl& d, size_t n) {
        reset();
        dev = &d;
        count = n;
        // Pad so that 16-byte vector loads of the tail stay in bounds.
        size_t bytes = ((n * sizeof(T) + 15) / 16) * 16 + 16;
        return device_alloc(d, reinterpret_cast<void**>(&ptr), bytes);
    }
    void reset() {
        if (ptr && dev) device_free(*dev, ptr);
        ptr = nullptr;
        count = 0;
    }
};

// ---------------------------------------------------------------- graph

struct PageRankPlan;
struct BfsWork;
struct KtCache;

// Per-graph degree statistics that the learned schedule's features use.
struct DegreeStats {
    float mean_degree = 0.f;
    float max_degree = 0.f;
    float gini = 0.f;  // Gini coefficient of the degree distribution
    float num_nodes = 0.f;
};

struct GraphImpl {
    std::shared_ptr<DeviceImpl> dev;
    uint32_t num_nodes = 0;
    uint32_t num_edges = 0;
    DeviceBuffer<uint32_t> offsets;
    DeviceBuffer<uint32_t> targets;
    std::mutex mu;  // guards the lazily built caches below
    int symmetric = -1;  // every entry u -> v has v -> u: -1 unknown, 0 no, 1 yes
    PageRankPlan* pr_plan = nullptr;  // owned; freed by destroy_pagerank_plan
    PageRankPlan* pr_plan_directed = nullptr;  // pull over the transpose; owned
    BfsWork* bfs_work = nullptr;      // owned; freed by destroy_bfs_work
    KtCache* kt_cache = nullptr;      // owned; freed by destroy_kt_cache
    bool has_degree_stats = false;
    DegreeStats degree_stats;
    ~GraphImpl();
};

// Host CSR arrays (CsrArrays, csr_export.rs:16-30).
struct HostCsr {
    std::vector<uint32_t> offsets;
    std::vector<uint32_t> targets;
    uint32_t num_nodes = 0;
};

// ---------------------------------------------------------------- host CSR

Error validate_csr_host(const uint32_t* offsets, size_t n_offsets, const uint32_t* targets,
                        size_t n_targets);
// Exact validate_csr message for the first violation at or after `node`,
// checking only that node (used after the device scan found it).
std::string describe_node_violation(uint32_t node, uint32_t start, uint32_t end,
                                    const uint32_t* list, size_t list_len, uint32_t num_nodes);

// ---------------------------------------------------------------- kernels (host wrappers)

// Finds the first node that breaks a CSR rule on the device; UINT32_MAX if none.
Error validate_csr_device(DeviceImpl& dev, const uint32_t* d_offsets, const uint32_t* d_targets,
                          uint32_t num_nodes, uint32_t num_edges, uint32_t* first_bad_node);
// The same checks while copying the targets from the host: the offsets are
// already on the device (or queued on dev.stream); the targets go up in chunks
// on dev.copy_stream and each chunk's entries are checked as soon as it lands.
Error upload_and_validate_csr(DeviceImpl& dev, const uint32_t* d_offsets, uint32_t* d_targets,
                              const uint32_t* h_targets, uint32_t num_nodes, uint32_t num_edges,
                              uint32_t* first_bad_node);

// New id of every vertex in the stable partition by degree class (class c:
// list lengths in [2^(c-1), 2^c)), highest class first: the order the
// PageRank plan relabels by, and the triangle count orients by.
Error degree_class_order(DeviceImpl& dev, const uint32_t* offsets, uint32_t V, DeviceBuffer<uint32_t>* inv);

// Whether every entry u -> v has its reverse v -> u (cached on the graph).
Error graph_symmetry(GraphImpl& g, bool* symmetric);

// Degree-oriented (by_degree) or id-oriented DAG of the CSR: every undirected
// edge once, lists still sorted. With `rev` (reverse-entry index) and dag_eid,
// also the CSR index of each DAG edge's u < v entry. *m = DAG edges.
Error build_dag(GraphImpl& g, bool by_degree, const uint32_t* rev, DeviceBuffer<uint32_t>* dag_offsets,
                DeviceBuffer<uint32_t>* dag_targets, DeviceBuffer<uint32_t>* dag_eid, uint32_t* m);

Error triangle_count(GraphImpl& g, bool oriented, uint64_t* total);
Error bfs(GraphImpl& g, uint32_t source, int32_t* host_distances, uint32_t* reachable,
          int32_t* max_depth);
Error pagerank(GraphImpl& g, float damping, uint32_t max_iterations, float tolerance,
               float* host_ranks, uint32_t* iterations, bool* converged);
Error k_truss(GraphImpl& g, uint32_t k, std::vector<uint32_t>* edges, uint32_t* iterations);
// Trussness of every CSR entry's edge (host_truss may be NULL), symmetric CSR.
Error truss_decomposition(GraphImpl& g, uint32_t* host_truss, uint32_t* max_truss, uint32_t* rounds);

// Exclusive scan of u32 counts into u32 offsets (out has n + 1 entries);
// returns the total through the device (out[n]).
Error exclusive_scan_u32(DeviceImpl& dev, const uint32_t* d_in, uint32_t* d_out, uint64_t n);
// The same scan with its length n = *d_n read on the device (n <= max_n),
// for launch sequences captured into a CUDA graph: out[0..n) = exclusive
// prefix, out[n] = total. tile_sums holds scan_device_n_tiles(max_n) values.
// Lengths up to kScanOneLaunchMax take one kernel, longer ones three; each
// kernel returns at once when the length is not its case, and `which` leaves
// out the launches a caller's graph never needs (an IF node on the length).
constexpr uint64_t kScanOneLaunchMax = 8192;
enum class ScanLaunches { kBoth, kOneTile, kMultiTile };
Error exclusive_scan_u32_device_n(DeviceImpl& dev, const uint32_t* d_in, uint32_t* d_out, const uint32_t* d_n,
                                  uint64_t max_n, uint32_t* tile_sums, ScanLaunches which = ScanLaunches::kBoth);
uint64_t scan_device_n_tiles(uint64_t max_n);

// Stable LSD radix sort of n 64-bit keys by bits [low_bit, high_bit), 8 per
// pass, ping-ponging between keys and tmp; *sorted is whichever holds the result.
Error radix_sort_u64(DeviceImpl& dev, uint64_t* keys, uint64_t* tmp, uint64_t n, uint32_t low_bit, uint32_t high_bit,
                     uint64_t** sorted);

// In-lists of a CSR (the transpose), every in-list ordered by source.
Error transpose_csr(DeviceImpl& dev, const uint32_t* offsets, const uint32_t* targets, uint32_t V, uint32_t E,
                    DeviceBuffer<uint32_t>* t_offsets, DeviceBuffer<uint32_t>* t_targets);

// PageRank over the CSR lists (directed = false: symmetric graph, pagerank.rs)
// or over their transpose with out-degrees from the lists (directed = true).
// tele (nullable, V floats, original ids): personalisation vector that takes
// the teleport and the dangling mass instead of the uniform 1/N.
Error pagerank_ex(GraphImpl& g, bool directed, const float* tele, float damping, uint32_t max_iterations,
                  float tolerance, float* host_ranks, uint32_t* iterations, bool* converged);

// Times `passes` launches of the gather probe (the plan's target stream and
// contribution gathers alone) over the plan of pagerank_ex(directed); builds
// the plan if needed. *ms_per_pass = device time per launch.
Error pagerank_gather_probe(GraphImpl& g, bool directed, uint32_t passes, double* ms_per_pass);

void destroy_pagerank_plan(PageRankPlan* p);
void destroy_bfs_work(BfsWork* w);
void destroy_kt_cache(KtCache* c);

// ---------------------------------------------------------------- device CSR build

// Edge pairs (host, interleaved src/dst) -> the graph's CSR, built on the
// device. mode 0: directed (from_edge_pairs, symmetric = false), 1: symmetric
// (from_edge_pairs, symmetric = true), 2: degree-oriented
// (from_edge_pairs_oriented).
Error build_graph_from_pairs(DeviceImpl& dev, const uint32_t* host_pairs, uint64_t n_pairs, uint32_t num_nodes,
                             int mode, GraphImpl& g);

// Synthetic graph drawn on the device (symmetric, loop-free, deduplicated).
struct GeneratorSpec {
    enum Kind { kRmat, kErdosRenyi, kGrid, kWattsStrogatz, kGeometric } kind = kRmat;
    uint64_t seed = 0;
    uint32_t scale = 0, edge_factor = 0;  // R-MAT
    double a = 0, b = 0, c = 0;           // R-MAT quadrant probabilities
    uint32_t n = 0;                       // Erdos-Renyi, Watts-Strogatz, geometric vertices
    uint64_t pairs = 0;                   // Erdos-Renyi drawn pairs
    uint32_t width = 0, height = 0;       // grid
    uint32_t k = 0;                       // Watts-Strogatz lattice degree (even)
    double p = 0;                         // grid drop / Watts-Strogatz rewire probability
    double avg_degree = 0;                // geometric
};
Error generate_graph(DeviceImpl& dev, const GeneratorSpec& spec, GraphImpl& g);
// Many R-MAT / Watts-Strogatz graphs drawn into one CSR: graph i holds the
// vertices [vbase[i], vbase[i + 1]) and each graph's lists equal its own
// generate_graph CSR shifted by vbase[i].
Error generate_union(DeviceImpl& dev, const std::vector<GeneratorSpec>& specs, std::vector<uint32_t>* vbase,
                     GraphImpl& u);

// ---------------------------------------------------------------- learned schedule

// Degree statistics of the CSR lists (computed on the device once, cached;
// the caller holds g.mu like every algorithm entry point).
Error degree_stats(GraphImpl& g, DegreeStats* out);

// Batched forward pass: out[n][3] predictions of features x[n][12].
Error sched_forward(DeviceImpl& dev, const uint16_t* weights, const float* x, uint64_t n, float* out);
// Masked mean squared error of the predictions against y[n][3] (mask[n][3]
// selects the recorded variants) and its gradient w.r.t. the 1571 parameters.
Error sched_gradient(DeviceImpl& dev, const uint16_t* weights, const float* x, const float* y, const uint8_t* mask,
                     uint64_t n, double* loss, float* grad);
// Adam on the device over minibatches drawn with replacement; master (FP32)
// is updated in place and weights receives its BF16 rounding.
Error sched_train(DeviceImpl& dev, float* master, uint16_t* weights, const float* x, const float* y,
                  const uint8_t* mask, uint64_t n, uint32_t steps, uint32_t batch, float lr, uint64_t seed,
                  double* final_loss);
Error set_schedule(DeviceImpl& dev, const uint16_t* weights);

// Per-level BFS trace: every valid step variant timed from the same frontier.
struct BfsTraceLevel {
    float features[12];
    float times_us[3];  // NaN for a variant that is not valid here
    uint8_t valid;      // bit c: variant c valid
    uint8_t fixed_rule; // what the alpha/beta rule picks
    uint8_t taken;      // the variant the traced run continued with
};
Error bfs_trace(GraphImpl& g, uint32_t source, uint64_t explore_seed, std::vector<BfsTraceLevel>* levels);

// Per-bucket triangle trace: every valid intersection variant timed per
// out-degree bucket of the DAG; *total = the triangle count (all agree).
struct TcTraceBucket {
    float features[12];
    float times_us[3];
    uint8_t valid;
    uint8_t fixed_rule;
};
Error triangle_trace(GraphImpl& g, std::vector<TcTraceBucket>* buckets, uint64_t* total);

// ---------------------------------------------------------------- batched form

// Triangle counting over a union of disjoint graphs: the union's DAG and
// out-degree buckets with one variant per bucket (learned, or timed once),
// planned once; batch_tc_launch then only enqueues kernels (capturable), which
// add every DAG source vertex's triangles into per_vertex[u].
struct BatchTcPlan;
Error batch_tc_plan(GraphImpl& u, BatchTcPlan** out, std::string* tuning);
Error batch_tc_launch(DeviceImpl& dev, BatchTcPlan& p, unsigned long long* per_vertex, uint32_t num_nodes);
void destroy_batch_tc_plan(BatchTcPlan* p);

// A packed batch of graphs (batch.cu).
struct BatchImpl;
void destroy_batch(BatchImpl* b);
Error batch_generate(DeviceImpl& dev, std::shared_ptr<DeviceImpl> owner, uint32_t num_graphs, uint64_t seed,
                     BatchImpl** out);
Error batch_from_csr(DeviceImpl& dev, std::shared_ptr<DeviceImpl> owner, const uint32_t* vbase, size_t num_graphs,
                     const uint32_t* offsets, size_t n_offsets, const uint32_t* targets, size_t n_targets,
                     BatchImpl** out);
uint32_t batch_num_graphs(const BatchImpl& b);
GraphImpl& batch_union(BatchImpl& b);
const std::vector<uint32_t>& batch_vertex_base(const BatchImpl& b);
Error batch_member(BatchImpl& b, uint32_t index, GraphImpl& g);
Error batch_set_bfs(BatchImpl& b, const uint32_t* sources, uint32_t S, bool keep_distances);
Error batch_set_ppr(BatchImpl& b, const uint32_t* seeds, uint32_t K, float damping, uint32_t max_iterations,
                    float tolerance);
Error batch_run_tc(BatchImpl& b, uint64_t* totals);
Error batch_run_bfs(BatchImpl& b);
Error batch_run_ppr(BatchImpl& b);
Error batch_read_tc(BatchImpl& b, uint64_t* totals);
Error batch_read_bfs(BatchImpl& b, int32_t* distances, uint32_t* reachable, int32_t* max_depth);
Error batch_read_ppr(BatchImpl& b, float* ranks, uint32_t* iterations, uint8_t* converged);
Error batch_capture(BatchImpl& b);
Error batch_replay(BatchImpl& b);
std::string batch_tuning(const BatchImpl& b);

}  // namespace gcu

// Launch helper: counts the launch, brackets it with events when per-kernel
// timing is on, and turns a launch failure into CudaError::Kernel.
#define GCU_LAUNCH(devref, name, kernel, grid, block, smem, ...)                           \
    do {                                                                                   \
        cudaEvent_t _ev = nullptr;                                                         \
        (devref).before_launch(name, &_ev);                                                \
        kernel<<<(grid), (block), (smem), (devref).stream>>>(__VA_ARGS__);                 \
        cudaError_t _le = cudaGetLastError();                                              \
        (devref).after_launch(name, _ev);                                                  \
        if (_le != cudaSuccess)                                                            \
            return ::gcu::kernel_error(std::string(name) + " launch failed: " +            \
                                       cudaGetErrorString(_le));                           \
    } while (0)
