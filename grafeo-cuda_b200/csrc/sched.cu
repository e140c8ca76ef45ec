// Learned schedule: training and inference kernels of the 12-32-32-3 network
// (layout and forward pass in sched.cuh), and the degree statistics that its
// features use.
//
// Training is minibatch Adam on the device. One gradient launch covers a
// minibatch in blocks of 64 samples: each thread runs the forward and
// backward pass of one sample into shared memory, then the block sums the
// per-sample products for every parameter in sample order and writes one row
// of partial sums; a second kernel adds the rows in block order (FP64), and a
// third applies Adam to the FP32 master weights and rounds them to BF16. The
// sums never depend on timing, so a training run is reproducible bit for bit.
// The loss is the masked mean squared error between the predicted and the
// measured log2(time in microseconds) of the variants a trace recorded.
#include <algorithm>
#include <cmath>

#include "sched.cuh"

namespace gcu {

namespace {

constexpr int kGradSamples = 64;                 // samples (threads) per gradient block
constexpr int kGradRow = kSchedParams + 2;       // partial sums: gradient, loss, count
constexpr int kPad = kSchedHidden + 1;           // padded row of per-sample activations

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void sched_to_bf16_kernel(const float* __restrict__ master, __nv_bfloat16* __restrict__ w) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kSchedParams; p += gridDim.x * blockDim.x)
        w[p] = __float2bfloat16_rn(master[p]);
}

__global__ void __launch_bounds__(128) sched_forward_kernel(const __nv_bfloat16* __restrict__ w16,
                                                            const float* __restrict__ x, uint64_t n,
                                                            float* __restrict__ out) {
    __shared__ float sw[kSchedParams];
    for (int p = threadIdx.x; p < kSchedParams; p += blockDim.x) sw[p] = __bfloat162float(w16[p]);
    __syncthreads();
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float xs[kSchedIn], h1[kSchedHidden], h2[kSchedHidden], o[kSchedOut];
        for (int k = 0; k < kSchedIn; ++k) xs[k] = x[i * kSchedIn + k];
        sched_forward_thread(sw, xs, h1, h2, o);
        for (int c = 0; c < kSchedOut; ++c) out[i * kSchedOut + c] = o[c];
    }
}

// One row of partial sums per block. Sample slot s of block b is minibatch
// position b * 64 + s: sample index = that position (sample_state == 0, the
// whole data set in order) or a draw from the SplitMix64 stream of
// sample_state at step * batch + position (with replacement).
__global__ void __launch_bounds__(kGradSamples) sched_grad_kernel(const __nv_bfloat16* __restrict__ w16,
                                                                  const float* __restrict__ x,
                                                                  const float* __restrict__ y,
                                                                  const uint8_t* __restrict__ mask, uint64_t n,
                                                                  uint64_t sample_state, uint64_t step,
                                                                  uint32_t batch, double* __restrict__ partials) {
    __shared__ float sw[kSchedParams];
    __shared__ float sx[kGradSamples][kSchedIn];
    __shared__ float sh1[kGradSamples][kPad], sh2[kGradSamples][kPad];
    __shared__ float sd1[kGradSamples][kPad], sd2[kGradSamples][kPad];
    __shared__ float sd3[kGradSamples][kSchedOut];
    __shared__ float sloss[kGradSamples], scount[kGradSamples];
    const int t = threadIdx.x;
    for (int p = t; p < kSchedParams; p += kGradSamples) sw[p] = __bfloat162float(w16[p]);
    __syncthreads();

    const uint64_t pos = static_cast<uint64_t>(blockIdx.x) * kGradSamples + t;
    bool valid;
    uint64_t idx = 0;
    if (sample_state) {
        valid = pos < batch;
        if (valid) idx = __umul64hi(mix64(sample_state + (step * batch + pos + 1) * 0x9E3779B97F4A7C15ull), n);
    } else {
        valid = pos < n;
        idx = pos;
    }
    float xs[kSchedIn], h1[kSchedHidden], h2[kSchedHidden], o[kSchedOut], d3[kSchedOut];
    for (int k = 0; k < kSchedIn; ++k) xs[k] = valid ? x[idx * kSchedIn + k] : 0.f;
    sched_forward_thread(sw, xs, h1, h2, o);
    float loss = 0.f, count = 0.f;
    for (int c = 0; c < kSchedOut; ++c) {
        const bool m = valid && mask[idx * kSchedOut + c];
        const float r = m ? o[c] - y[idx * kSchedOut + c] : 0.f;
        d3[c] = 2.f * r;
        loss = fmaf(r, r, loss);
        count += m ? 1.f : 0.f;
    }
    for (int k = 0; k < kSchedIn; ++k) sx[t][k] = xs[k];
    for (int j = 0; j < kSchedHidden; ++j) {
        sh1[t][j] = h1[j];
        sh2[t][j] = h2[j];
        float g = 0.f;
        for (int c = 0; c < kSchedOut; ++c) g = fmaf(sw[kSchedW3 + c * kSchedHidden + j], d3[c], g);
        sd2[t][j] = h2[j] > 0.f ? g : 0.f;
    }
    for (int c = 0; c < kSchedOut; ++c) sd3[t][c] = d3[c];
    for (int j = 0; j < kSchedHidden; ++j) {
        float g = 0.f;
        for (int i = 0; i < kSchedHidden; ++i) g = fmaf(sw[kSchedW2 + i * kSchedHidden + j], sd2[t][i], g);
        sd1[t][j] = h1[j] > 0.f ? g : 0.f;
    }
    sloss[t] = loss;
    scount[t] = count;
    __syncthreads();

    double* row = partials + static_cast<uint64_t>(blockIdx.x) * kGradRow;
    for (int p = t; p < kSchedParams; p += kGradSamples) {
        float g = 0.f;
        if (p < kSchedB1) {
            const int j = p / kSchedIn, k = p % kSchedIn;
            for (int s = 0; s < kGradSamples; ++s) g = fmaf(sd1[s][j], sx[s][k], g);
        } else if (p < kSchedW2) {
            const int j = p - kSchedB1;
            for (int s = 0; s < kGradSamples; ++s) g += sd1[s][j];
        } else if (p < kSchedB2) {
            const int i = (p - kSchedW2) / kSchedHidden, j = (p - kSchedW2) % kSchedHidden;
            for (int s = 0; s < kGradSamples; ++s) g = fmaf(sd2[s][i], sh1[s][j], g);
        } else if (p < kSchedW3) {
            const int i = p - kSchedB2;
            for (int s = 0; s < kGradSamples; ++s) g += sd2[s][i];
        } else if (p < kSchedB3) {
            const int c = (p - kSchedW3) / kSchedHidden, j = (p - kSchedW3) % kSchedHidden;
            for (int s = 0; s < kGradSamples; ++s) g = fmaf(sd3[s][c], sh2[s][j], g);
        } else {
            const int c = p - kSchedB3;
            for (int s = 0; s < kGradSamples; ++s) g += sd3[s][c];
        }
        row[p] = g;
    }
    if (t == 0) {
        double l = 0.0, c = 0.0;
        for (int s = 0; s < kGradSamples; ++s) {
            l += sloss[s];
            c += scount[s];
        }
        row[kSchedParams] = l;
        row[kSchedParams + 1] = c;
    }
}

// sums[p] = sum over blocks (in block order) of partials[b][p].
__global__ void sched_reduce_kernel(const double* __restrict__ partials, uint32_t blocks, double* __restrict__ sums) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kGradRow; p += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < blocks; ++b) s += partials[static_cast<uint64_t>(b) * kGradRow + p];
        sums[p] = s;
    }
}

// Adam (Kingma and Ba, 2015) with bias correction; b1t = beta1^t, b2t = beta2^t.
__global__ void sched_adam_kernel(const double* __restrict__ sums, float* __restrict__ master, float* __restrict__ m1,
                                  float* __restrict__ m2, __nv_bfloat16* __restrict__ w16, float lr, float b1t,
                                  float b2t) {
    constexpr float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    const double count = sums[kSchedParams + 1];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kSchedParams; p += gridDim.x * blockDim.x) {
        const float g = count > 0.0 ? static_cast<float>(sums[p] / count) : 0.f;
        const float a = beta1 * m1[p] + (1.f - beta1) * g;
        const float b = beta2 * m2[p] + (1.f - beta2) * g * g;
        m1[p] = a;
        m2[p] = b;
        const float mh = a / (1.f - b1t), vh = b / (1.f - b2t);
        master[p] -= lr * mh / (sqrtf(vh) + eps);
        w16[p] = __float2bfloat16_rn(master[p]);
    }
}

// ---------------------------------------------------------------- degree statistics

__global__ void degree_keys_kernel(const uint32_t* __restrict__ offsets, uint32_t V, uint64_t* __restrict__ keys) {
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < V;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        keys[v] = offsets[v + 1] - offsets[v];
}

// Block partials of sum_i (2 i - V + 1) d_(i) over the ascending degrees; the
// Gini coefficient is that sum / (V * sum d).
__global__ void gini_partial_kernel(const uint64_t* __restrict__ sorted, uint32_t V, double* __restrict__ partials) {
    __shared__ double scratch[32];
    double acc = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < V;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        acc += (2.0 * static_cast<double>(i) - V + 1.0) * static_cast<double>(sorted[i]);
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

struct Uploaded {
    DeviceBuffer<float> x, y;
    DeviceBuffer<uint8_t> mask;
    DeviceBuffer<__nv_bfloat16> w16;
};

Error upload(DeviceImpl& dev, Uploaded& u, const uint16_t* weights, const float* x, const float* y,
             const uint8_t* mask, uint64_t n) {
    GCU_TRY(u.x.allocate(dev, std::max<uint64_t>(n * kSchedIn, 1)));
    GCU_TRY(u.w16.allocate(dev, kSchedParams));
    if (n) GCU_CUDA(cudaMemcpyAsync(u.x.ptr, x, 4 * n * kSchedIn, cudaMemcpyHostToDevice, dev.stream), "copy");
    if (weights)
        GCU_CUDA(cudaMemcpyAsync(u.w16.ptr, weights, 2 * kSchedParams, cudaMemcpyHostToDevice, dev.stream), "copy");
    if (y) {
        GCU_TRY(u.y.allocate(dev, std::max<uint64_t>(n * kSchedOut, 1)));
        GCU_TRY(u.mask.allocate(dev, std::max<uint64_t>(n * kSchedOut, 1)));
        if (n) {
            GCU_CUDA(cudaMemcpyAsync(u.y.ptr, y, 4 * n * kSchedOut, cudaMemcpyHostToDevice, dev.stream), "copy");
            GCU_CUDA(cudaMemcpyAsync(u.mask.ptr, mask, n * kSchedOut, cudaMemcpyHostToDevice, dev.stream), "copy");
        }
    }
    return ok();
}

// Loss and gradient sums over the whole data set in order.
Error full_gradient(DeviceImpl& dev, const Uploaded& u, uint64_t n, std::vector<double>* sums) {
    const uint64_t blocks = std::max<uint64_t>(1, ceil_div_u64(n, kGradSamples));
    if (blocks > 0x7FFFFFFFull) return kernel_error("schedule data set too large");
    DeviceBuffer<double> partials, dsums;
    GCU_TRY(partials.allocate(dev, blocks * kGradRow));
    GCU_TRY(dsums.allocate(dev, kGradRow));
    GCU_LAUNCH(dev, "sched_grad", sched_grad_kernel, static_cast<unsigned>(blocks), kGradSamples, 0, u.w16.ptr,
               u.x.ptr, u.y.ptr, u.mask.ptr, n, 0ull, 0ull, 0u, partials.ptr);
    GCU_LAUNCH(dev, "sched_reduce", sched_reduce_kernel, ceil_div_u64(kGradRow, 256), 256, 0, partials.ptr,
               static_cast<uint32_t>(blocks), dsums.ptr);
    sums->resize(kGradRow);
    GCU_CUDA(cudaMemcpyAsync(sums->data(), dsums.ptr, sizeof(double) * kGradRow, cudaMemcpyDeviceToHost, dev.stream),
             "copy");
    return dev.sync();
}

}  // namespace

Error sched_forward(DeviceImpl& dev, const uint16_t* weights, const float* x, uint64_t n, float* out) {
    Uploaded u;
    GCU_TRY(upload(dev, u, weights, x, nullptr, nullptr, n));
    if (n == 0) return ok();
    DeviceBuffer<float> d_out;
    GCU_TRY(d_out.allocate(dev, n * kSchedOut));
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(n, 128), 4096));
    GCU_LAUNCH(dev, "sched_forward", sched_forward_kernel, blocks, 128, 0, u.w16.ptr, u.x.ptr, n, d_out.ptr);
    GCU_CUDA(cudaMemcpyAsync(out, d_out.ptr, 4 * n * kSchedOut, cudaMemcpyDeviceToHost, dev.stream), "copy");
    return dev.sync();
}

Error sched_gradient(DeviceImpl& dev, const uint16_t* weights, const float* x, const float* y, const uint8_t* mask,
                     uint64_t n, double* loss, float* grad) {
    Uploaded u;
    GCU_TRY(upload(dev, u, weights, x, y, mask, n));
    std::vector<double> sums;
    GCU_TRY(full_gradient(dev, u, n, &sums));
    const double count = sums[kSchedParams + 1];
    *loss = count > 0 ? sums[kSchedParams] / count : 0.0;
    for (int p = 0; p < kSchedParams; ++p) grad[p] = count > 0 ? static_cast<float>(sums[p] / count) : 0.f;
    return ok();
}

Error sched_train(DeviceImpl& dev, float* master, uint16_t* weights, const float* x, const float* y,
                  const uint8_t* mask, uint64_t n, uint32_t steps, uint32_t batch, float lr, uint64_t seed,
                  double* final_loss) {
    if (n == 0) return kernel_error("schedule training needs at least one sample");
    if (batch == 0 || batch > (1u << 20)) return kernel_error("schedule training batch must be in 1..=1048576");
    Uploaded u;
    GCU_TRY(upload(dev, u, nullptr, x, y, mask, n));
    DeviceBuffer<float> d_master, m1, m2;
    GCU_TRY(d_master.allocate(dev, kSchedParams));
    GCU_TRY(m1.allocate(dev, kSchedParams));
    GCU_TRY(m2.allocate(dev, kSchedParams));
    GCU_CUDA(cudaMemcpyAsync(d_master.ptr, master, 4 * kSchedParams, cudaMemcpyHostToDevice, dev.stream), "copy");
    GCU_CUDA(cudaMemsetAsync(m1.ptr, 0, 4 * kSchedParams, dev.stream), "memset");
    GCU_CUDA(cudaMemsetAsync(m2.ptr, 0, 4 * kSchedParams, dev.stream), "memset");
    GCU_LAUNCH(dev, "sched_to_bf16", sched_to_bf16_kernel, 7, 256, 0, d_master.ptr, u.w16.ptr);
    const uint32_t blocks = static_cast<uint32_t>(ceil_div_u64(batch, kGradSamples));
    DeviceBuffer<double> partials, sums;
    GCU_TRY(partials.allocate(dev, static_cast<uint64_t>(blocks) * kGradRow));
    GCU_TRY(sums.allocate(dev, kGradRow));
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    const uint64_t state = (z ^ (z >> 31)) | 1ull;  // nonzero: sampled minibatches
    double b1t = 1.0, b2t = 1.0;
    for (uint32_t s = 0; s < steps; ++s) {
        b1t *= 0.9;
        b2t *= 0.999;
        GCU_LAUNCH(dev, "sched_grad", sched_grad_kernel, blocks, kGradSamples, 0, u.w16.ptr, u.x.ptr, u.y.ptr,
                   u.mask.ptr, n, state, static_cast<uint64_t>(s), batch, partials.ptr);
        GCU_LAUNCH(dev, "sched_reduce", sched_reduce_kernel, ceil_div_u64(kGradRow, 256), 256, 0, partials.ptr,
                   blocks, sums.ptr);
        GCU_LAUNCH(dev, "sched_adam", sched_adam_kernel, 7, 256, 0, sums.ptr, d_master.ptr, m1.ptr, m2.ptr, u.w16.ptr,
                   lr, static_cast<float>(b1t), static_cast<float>(b2t));
        if ((s & 1023) == 1023) GCU_TRY(dev.sync());  // bound the queued launches
    }
    std::vector<double> all;
    GCU_TRY(full_gradient(dev, u, n, &all));
    *final_loss = all[kSchedParams + 1] > 0 ? all[kSchedParams] / all[kSchedParams + 1] : 0.0;
    GCU_CUDA(cudaMemcpyAsync(master, d_master.ptr, 4 * kSchedParams, cudaMemcpyDeviceToHost, dev.stream), "copy");
    GCU_CUDA(cudaMemcpyAsync(weights, u.w16.ptr, 2 * kSchedParams, cudaMemcpyDeviceToHost, dev.stream), "copy");
    return dev.sync();
}

Error set_schedule(DeviceImpl& dev, const uint16_t* weights) {
    if (!weights) {
        if (dev.schedule) {
            GCU_TRY(dev.sync());
            device_free(dev, dev.schedule);
            dev.schedule = nullptr;
        }
        return ok();
    }
    if (!dev.schedule) GCU_TRY(device_alloc(dev, reinterpret_cast<void**>(&dev.schedule), 2 * kSchedParams + 16));
    GCU_CUDA(cudaMemcpyAsync(dev.schedule, weights, 2 * kSchedParams, cudaMemcpyHostToDevice, dev.stream), "copy");
    return dev.sync();
}

Error degree_stats(GraphImpl& g, DegreeStats* out) {
    if (g.has_degree_stats) {
        *out = g.degree_stats;
        return ok();
    }
    DeviceImpl& dev = *g.dev;
    DegreeStats s;
    const uint32_t V = g.num_nodes;
    s.num_nodes = static_cast<float>(V);
    s.mean_degree = V ? static_cast<float>(static_cast<double>(g.num_edges) / V) : 0.f;
    if (V && g.num_edges) {
        DeviceBuffer<uint64_t> keys, tmp;
        GCU_TRY(keys.allocate(dev, V));
        GCU_TRY(tmp.allocate(dev, V));
        const unsigned grid =
            static_cast<unsigned>(std::min<uint64_t>(ceil_div_u64(V, 256), static_cast<uint64_t>(dev.sm_count) * 8));
        GCU_LAUNCH(dev, "degree_keys", degree_keys_kernel, grid, 256, 0, g.offsets.ptr, V, keys.ptr);
        uint32_t bits = 0;
        while (bits < 32 && (static_cast<uint64_t>(1) << bits) <= g.num_edges) ++bits;
        uint64_t* sorted = nullptr;
        GCU_TRY(radix_sort_u64(dev, keys.ptr, tmp.ptr, V, 0, bits, &sorted));
        DeviceBuffer<double> partials;
        GCU_TRY(partials.allocate(dev, grid));
        GCU_LAUNCH(dev, "degree_gini", gini_partial_kernel, grid, 256, 0, sorted, V, partials.ptr);
        std::vector<double> host(grid);
        uint64_t maxdeg = 0;
        GCU_CUDA(cudaMemcpyAsync(host.data(), partials.ptr, sizeof(double) * grid, cudaMemcpyDeviceToHost, dev.stream),
                 "copy");
        GCU_CUDA(cudaMemcpyAsync(&maxdeg, sorted + (V - 1), sizeof(uint64_t), cudaMemcpyDeviceToHost, dev.stream),
                 "copy");
        GCU_TRY(dev.sync());
        double acc = 0.0;
        for (double h : host) acc += h;
        s.max_degree = static_cast<float>(maxdeg);
        s.gini = static_cast<float>(acc / (static_cast<double>(V) * static_cast<double>(g.num_edges)));
    }
    g.degree_stats = s;
    g.has_degree_stats = true;
    *out = s;
    return ok();
}

}  // namespace gcu
