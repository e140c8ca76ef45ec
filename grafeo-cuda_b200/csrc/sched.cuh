// Learned schedule: the 12-32-32-3 network that picks a BFS step variant per
// level and a wedge-intersection variant per degree bucket.
//
// Parameters are BF16 (round to nearest even from FP32 master copies);
// activations and sums are FP32 with explicit fused multiply-adds in a fixed
// order, so the per-decision warp forward pass, the batched forward kernel and
// the training kernels compute the same numbers. Layout (GCU_SCHEDULE_PARAMS
// = 1571 values): W1[32][12], b1[32], W2[32][32], b2[32], W3[3][32], b3[3];
// hidden layers ReLU, outputs linear: the predicted log2 of each variant's
// time in microseconds. A decision is the valid variant with the smallest
// prediction. No reference counterpart: the reference has one fixed schedule.
#pragma once

#include <cuda_bf16.h>

#include "device_common.cuh"
#include "gcu_internal.h"

namespace gcu {

constexpr int kSchedIn = 12;
constexpr int kSchedHidden = 32;
constexpr int kSchedOut = 3;
constexpr int kSchedW1 = 0;
constexpr int kSchedB1 = kSchedW1 + kSchedHidden * kSchedIn;
constexpr int kSchedW2 = kSchedB1 + kSchedHidden;
constexpr int kSchedB2 = kSchedW2 + kSchedHidden * kSchedHidden;
constexpr int kSchedW3 = kSchedB2 + kSchedHidden;
constexpr int kSchedB3 = kSchedW3 + kSchedOut * kSchedHidden;
constexpr int kSchedParams = kSchedB3 + kSchedOut;
static_assert(kSchedParams == 1571, "schedule network layout");

__host__ __device__ __forceinline__ float sched_log(float x) { return log2f(1.0f + x); }

// Features of the BFS decision taken before expanding the frontier of `level`
// (12 values; index 0 = 0 marks a BFS level).
__host__ __device__ __forceinline__ void bfs_features(float* f, float frontier_n, float frontier_m, float unexplored,
                                                      int level, const DegreeStats& s, bool frontier_bitmap,
                                                      float reached) {
    f[0] = 0.f;
    f[1] = sched_log(frontier_n) / 32.f;
    f[2] = sched_log(frontier_m) / 32.f;
    f[3] = sched_log(unexplored) / 32.f;
    f[4] = fminf(static_cast<float>(level), 64.f) / 32.f;
    f[5] = sched_log(s.mean_degree) / 16.f;
    f[6] = sched_log(s.max_degree) / 32.f;
    f[7] = s.gini;
    f[8] = sched_log(s.num_nodes) / 32.f;
    f[9] = frontier_bitmap ? 1.f : 0.f;
    f[10] = s.num_nodes > 0.f ? (s.num_nodes - reached) / s.num_nodes : 0.f;
    f[11] = (sched_log(frontier_m) - sched_log(unexplored)) / 32.f;
}

// Features of the intersection decision for one degree bucket of a DAG:
// vertices with out-degree in [lo, hi] (index 0 = 1 marks a bucket).
__host__ __device__ __forceinline__ void bucket_features(float* f, float vertices, float entries, float dag_edges,
                                                         const DegreeStats& s, float lo, float hi, float mean_out) {
    f[0] = 1.f;
    f[1] = sched_log(vertices) / 32.f;
    f[2] = sched_log(entries) / 32.f;
    f[3] = sched_log(dag_edges) / 32.f;
    f[4] = 0.f;
    f[5] = sched_log(s.mean_degree) / 16.f;
    f[6] = sched_log(s.max_degree) / 32.f;
    f[7] = s.gini;
    f[8] = sched_log(s.num_nodes) / 32.f;
    f[9] = sched_log(lo) / 16.f;
    f[10] = sched_log(hi) / 16.f;
    f[11] = sched_log(mean_out) / 16.f;
}

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// Forward pass of one sample by one warp: lane j owns hidden unit j; every
// lane ends with the three outputs. Sums run over inputs in index order.
__device__ __forceinline__ void sched_forward_warp(const __nv_bfloat16* __restrict__ w, const float* x, float* out) {
    const int j = static_cast<int>(lane_id());
    float z1 = bf(w, kSchedB1 + j);
#pragma unroll
    for (int k = 0; k < kSchedIn; ++k) z1 = fmaf(bf(w, kSchedW1 + j * kSchedIn + k), x[k], z1);
    const float h1 = fmaxf(z1, 0.f);
    float z2 = bf(w, kSchedB2 + j);
#pragma unroll
    for (int k = 0; k < kSchedHidden; ++k)
        z2 = fmaf(bf(w, kSchedW2 + j * kSchedHidden + k), __shfl_sync(kFullMask, h1, k), z2);
    const float h2 = fmaxf(z2, 0.f);
#pragma unroll
    for (int c = 0; c < kSchedOut; ++c) {
        float o = bf(w, kSchedB3 + c);
#pragma unroll
        for (int k = 0; k < kSchedHidden; ++k)
            o = fmaf(bf(w, kSchedW3 + c * kSchedHidden + k), __shfl_sync(kFullMask, h2, k), o);
        out[c] = o;
    }
}

// Forward pass of one sample by one thread with FP32 weights (already
// converted from BF16), the same order of operations as the warp version.
// h1/h2 receive the hidden activations (the backward pass needs them).
__device__ __forceinline__ void sched_forward_thread(const float* __restrict__ w, const float* x, float* h1, float* h2,
                                                     float* out) {
    for (int j = 0; j < kSchedHidden; ++j) {
        float z = w[kSchedB1 + j];
#pragma unroll
        for (int k = 0; k < kSchedIn; ++k) z = fmaf(w[kSchedW1 + j * kSchedIn + k], x[k], z);
        h1[j] = fmaxf(z, 0.f);
    }
    for (int j = 0; j < kSchedHidden; ++j) {
        float z = w[kSchedB2 + j];
#pragma unroll 8
        for (int k = 0; k < kSchedHidden; ++k) z = fmaf(w[kSchedW2 + j * kSchedHidden + k], h1[k], z);
        h2[j] = fmaxf(z, 0.f);
    }
#pragma unroll
    for (int c = 0; c < kSchedOut; ++c) {
        float o = w[kSchedB3 + c];
#pragma unroll 8
        for (int k = 0; k < kSchedHidden; ++k) o = fmaf(w[kSchedW3 + c * kSchedHidden + k], h2[k], o);
        out[c] = o;
    }
}

// Valid variant with the smallest predicted time; -1 when the prediction is
// not finite (the caller falls back to its fixed rule).
__host__ __device__ __forceinline__ int sched_pick(const float* out, unsigned valid_mask) {
    int best = -1;
    for (int c = 0; c < kSchedOut; ++c) {
        if (!((valid_mask >> c) & 1u)) continue;
        if (!(out[c] == out[c]) || out[c] > 3.0e38f || out[c] < -3.0e38f) return -1;
        if (best < 0 || out[c] < out[best]) best = c;
    }
    return best;
}

// The network's pick replaces the fixed rule's variant only where it predicts
// that variant at least 2^kSchedMarginLog2 (1.15x) slower than its pick. On
// graphs the fixed rule already serves well (R-MAT and Erdos-Renyi levels,
// where the alpha/beta rule is near the best schedule) the remaining predicted
// gains are within the network's error, and following them costs time; the
// large gains (long-diameter graphs, small frontiers) are far above the margin.
constexpr float kSchedMarginLog2 = 0.2f;

__host__ __device__ __forceinline__ int sched_pick_over(const float* out, unsigned valid_mask, int fixed) {
    const int best = sched_pick(out, valid_mask);
    if (best < 0 || best == fixed || fixed < 0 || !((valid_mask >> fixed) & 1u)) return best;
    return out[fixed] - out[best] >= kSchedMarginLog2 ? best : fixed;
}

}  // namespace gcu
