// Learned style selector: layout of the MLP parameter blob, the feature vector,
// and the block-level inference routine used inside the relax kernels' epilogue.
//
// Network: x (16 features) -> standardise with (mu, sd) -> 64 ReLU -> 64 ReLU -> 8
// outputs, one predicted log2 launch time (ns) per variant. The selector picks
// the allowed variant with the smallest prediction. Weights are stored
// [in][out] so that, for a fixed input, consecutive outputs are consecutive in memory.
#pragma once
#include "common.cuh"

namespace i2 {

constexpr int kOut = kNumVariants;
constexpr int kOffMu = 0;
constexpr int kOffSd = kOffMu + kFeatures;
constexpr int kOffW1 = kOffSd + kFeatures;
constexpr int kOffB1 = kOffW1 + kFeatures * kHidden;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden * kOut;
constexpr int kParams = kOffB3 + kOut;

// Features of a frontier about to be consumed. All are finite and O(1..40).
__device__ __forceinline__ void frontier_features(const GStats& gs, int algo, int iter, int size, int hsize,
                                                  unsigned long long edges, int maxdeg, long long visited,
                                                  float* f) {
  const float fs = (float)size + (float)hsize;
  const float fe = (float)edges;
  const float V = (float)gs.nodes;
  const float E = (float)gs.edges > 0.f ? (float)gs.edges : 1.f;
  f[0] = log2f(1.f + fs);
  f[1] = log2f(1.f + fe);
  f[2] = fs / V;
  f[3] = fe / E;
  f[4] = log2f(1.f + fe / fmaxf(1.f, fs));
  f[5] = log2f(1.f + (float)maxdeg);
  f[6] = (float)visited / V;
  f[7] = log2f(1.f + (float)iter);
  f[8] = log2f(V);
  f[9] = log2f(1.f + (float)gs.edges);
  f[10] = log2f(1.f + gs.avgdeg);
  f[11] = log2f(1.f + (float)gs.maxdeg);
  f[12] = log2f(1.f + gs.degcv);
  f[13] = algo == kSSSP ? 1.f : 0.f;
  f[14] = algo == kCC ? 1.f : 0.f;
  f[15] = fs > 0.f ? (float)hsize / fs : 0.f;
}

// Block-cooperative forward pass (any block size >= kHidden). x and y live in
// shared memory; the hidden activations use the two scratch arrays.
__device__ __forceinline__ void mlp_forward_block(const float* __restrict__ P, const float* x, float* h1,
                                                  float* h2, float* y) {
  const int t = threadIdx.x;
  if (t < kHidden) {
    float acc = P[kOffB1 + t];
#pragma unroll
    for (int k = 0; k < kFeatures; ++k) {
      const float xs = (x[k] - P[kOffMu + k]) / P[kOffSd + k];
      acc = fmaf(xs, P[kOffW1 + k * kHidden + t], acc);
    }
    h1[t] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  if (t < kHidden) {
    float acc = P[kOffB2 + t];
#pragma unroll 8
    for (int k = 0; k < kHidden; ++k) acc = fmaf(h1[k], P[kOffW2 + k * kHidden + t], acc);
    h2[t] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  if (t < kOut) {
    float acc = P[kOffB3 + t];
#pragma unroll 8
    for (int k = 0; k < kHidden; ++k) acc = fmaf(h2[k], P[kOffW3 + k * kOut + t], acc);
    y[t] = acc;
  }
  __syncthreads();
}

}  // namespace i2
